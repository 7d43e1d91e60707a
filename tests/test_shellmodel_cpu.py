"""The pair-count calibration objective: the CPU restatement (oracle) against
the reference's own ShellModel.r_factor (tests/golden/shellmodel.npz), and
the host side of chimera_b200.shellmodel."""
import numpy as np
import pytest

from conftest import golden
from oracle import shellmodel as OS


def model_of(g):
    return dict(k=g["k"], f=g["f"], delta=g["delta"], lam=g["lam"], shells_ref=g["shells_ref"],
                shell_mult=g["shell_mult"], sigma2_ref=g["sigma2_shell_ref"],
                a0_ref=float(g["a0_ref"]), s02=float(g["s02"]), dk_win=float(g["dk_win"]),
                etok=float(g["etok"]))


@pytest.mark.parametrize("kind", ["complex", "magnitude"])
def test_oracle_matches_reference_r_factor(kind):
    """24 parameter sets over the calibration's search ranges (window, E0
    shifts, a0, sigma^2 scales, dr, C3, C4, per-pair widths): R-factor and
    per-edge amplitudes of the reference's ShellModel to 1e-10 relative."""
    g = golden("shellmodel.npz")
    m = model_of(g)
    mask = g["mask"]
    bins = g["idx"][mask]
    mag = kind == "magnitude"
    data = (g["data_m"] if mag else g["data_c"])[:, mask]
    rf_ref = g["rf_m"] if mag else g["rf_c"]
    sc_ref = g["scales_m"] if mag else g["scales_c"]
    for q, x in enumerate(g["params"]):
        rf, sc = OS.r_factor(x, g["N1"], m, data, bins, g["kweight"], magnitude=mag)
        assert abs(rf - rf_ref[q]) <= 1e-10 * abs(rf_ref[q]), (q, rf, rf_ref[q])
        assert np.allclose(sc, sc_ref[q], rtol=1e-10, atol=0), (q, sc, sc_ref[q])


def test_oracle_random_alloy_counts():
    g = golden("shellmodel.npz")
    m = model_of(g)
    mask = g["mask"]
    for q in range(0, 24, 6):
        rf, _ = OS.r_factor(g["params"][q], g["N0"], m, g["data_c"][:, mask], g["idx"][mask],
                            g["kweight"])
        assert abs(rf - g["rf_n0"][q]) <= 1e-10 * g["rf_n0"][q]


def host_model(g):
    from chimera_b200.shellmodel import ShellModel
    return ShellModel(g["k"], (None, g["f"], g["delta"], g["lam"]), g["shells_ref"],
                      g["shell_mult"], g["sigma2_shell_ref"], int(g["natoms"]),
                      float(g["a0_ref"]), s02=float(g["s02"]), dk_win=float(g["dk_win"]),
                      composition=(0.5, 0.5))


def test_flat_layout_roundtrip():
    g = golden("shellmodel.npz")
    sm = host_model(g)
    assert sm.nparam == g["params"].shape[1]
    for row in g["params"][:5]:
        sm.set_flat(row)
        assert np.array_equal(sm.flat(), row)


def test_stage1_vector_matches_reference():
    """The global stage's search vector (names, bounds, default start) and
    its mapping to model parameters equal the reference's Stage1
    (chimera/calibrate.py:126-247) with every optional block switched on."""
    from chimera_b200.calibrate import Stage1
    g = golden("shellmodel.npz")
    sm = host_model(g)
    sm.set_flat(g["stage_base"])
    st = Stage1(sm, (0.5, 0.5), ms=True, free_window=True, free_dr=True, free_c3=True,
                free_shell_sigma=True, free_c4=True, free_sigma_pair=True, free_ms_edge=True,
                elements=("Fe", "Ni"), dE0_start=float(g["stage_dE0_start"]))
    assert st.names == [str(x) for x in g["stage_names"]]
    assert np.allclose(st.bounds, g["stage_bounds"], rtol=0, atol=0)
    assert np.array_equal(st.x0(), g["stage_x0"])
    rows = st.rows(g["stage_X"], a0=3.59)
    assert np.allclose(rows, g["stage_rows"], rtol=1e-15, atol=0)
    assert np.array_equal(sm.flat(), g["stage_base"])      # the model's own state is untouched


@pytest.mark.parametrize("flags", [dict(), dict(free_c4=True, free_sigma_pair=True,
                                               free_ms_edge=True, free_a0=True),
                                   dict(ms=False, free_window=False, free_dr=False)])
def test_stage1_rows_fast_equal_rows(flags):
    """The population-at-once mapping gives the rows of one unpack +
    set_params per vector, to rounding (exp of a sum of logs)."""
    from chimera_b200.calibrate import Stage1
    g = golden("shellmodel.npz")
    sm = host_model(g)
    sm.set_flat(g["stage_base"])
    st = Stage1(sm, (0.5, 0.5), elements=("Fe", "Ni"), **flags)
    lo, hi = np.array(st.bounds).T
    X = lo + (hi - lo) * np.random.default_rng(1).uniform(size=(40, lo.size))
    a0 = None if flags.get("free_a0") else 3.59
    assert np.allclose(st.rows_fast(X, a0=a0), st.rows(X, a0=a0), rtol=1e-13, atol=1e-16)
