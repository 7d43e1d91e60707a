"""The oracle's plain sampler replays the reference RMCSampler's golden
traces exactly: the same accepted swaps, exchanges and final states."""
import numpy as np
import pytest

from cases import oracle_problem, trace_inputs
from oracle import sampler as OS


@pytest.mark.parametrize("name", ["rmc_trace.npz", "rmc_trace_disp.npz", "rmc_trace_ms.npz"])
def test_oracle_replays_reference_trace(name):
    d = trace_inputs(name)
    prob = oracle_problem(d)
    smp = OS.PlainSampler(prob, int(d["nrep"]), float(d["tmin"]), float(d["tmax"]),
                          int(d["seed"]), float(d["swap_frac"]), 0.012, 0.10)
    smp.init_state(d["species0"], d["ideal"])
    trace, c2 = [], []
    for it in range(int(d["nsteps"])):
        trace.append(smp.step())
        c2.append(smp.chi2.copy())
        if (it + 1) % 25 == 0:
            smp.replica_exchange()
    assert np.array_equal(np.array(trace), d["accepted"])
    assert np.allclose(np.array(c2), d["chi2_log"], rtol=1e-10, atol=0)
    assert np.array_equal(smp.species, d["final_species"])
    assert np.allclose(smp.pos, d["final_pos"], rtol=0, atol=1e-14)
    assert np.allclose(smp.chi, d["final_chi"], rtol=1e-10, atol=1e-12)
    if "ms_C_final" in d:
        assert np.array_equal(smp.C, d["ms_C_final"])
