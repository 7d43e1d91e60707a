"""The device FP64 sampler over the whole plain-method configuration run
(500-atom fcc Fe-Ni, exact multiple scattering, 8 rungs, 20,000 swap
attempts), against the oracle's FP64 run of it (tests/golden/config0.npz,
made by tests/golden/make_config0.py): fed the reference's random streams,
the device run makes the same decisions, so its final states, best chi^2,
best state's R-factor and posterior Warren-Cowley parameters are the
oracle's."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def test_fp64_sampler_reproduces_the_config0_run(cuda):
    torch = cuda
    from chimera_b200 import configs
    from chimera_b200.sampler import RMCSampler
    g = golden("config0.npz")
    prob = configs.Problem(ncell=(5, 5, 5), rmax=5.0, ms=True)
    nsteps = int(g["nsteps"])
    smp = RMCSampler(prob.fm, prob.ft, g["target"], prob.mask, prob.sigma_R(), nrep=8,
                     tmin=1e-4, tmax=1e-1, seed=int(g["seed"]), swap_frac=1.0, disp_sigma=0.012,
                     max_disp=0.10, ms_library=prob.ms, precision=0, reproduce=True,
                     collect_after=int(0.6 * nsteps), collect_every=50, collect_beta=0.5,
                     n_collect=4)
    smp.init_state(g["species0"], prob.cell.ideal)
    smp.run(nsteps, exchange_every=25, log_every=10 ** 9)
    assert smp.lad.device_error() == 0
    assert np.array_equal(smp.species.cpu().numpy(), g["final_species"].astype(np.int32))
    bsp, bpos, bc2 = smp.best()
    assert np.array_equal(bsp, g["best_species"].astype(np.int32))
    assert abs(bc2 - float(g["best_chi2"])) <= 1e-9 * abs(float(g["best_chi2"]))
    # the best state's R-factor, by the device path sum, MS and transform
    sp_d = torch.from_numpy(bsp[None]).cuda()
    chi = prob.fm.chi_full(torch.from_numpy(bpos[None]).cuda(), sp_d) + prob.ms.full(sp_d)
    cnt = torch.bincount(sp_d[0].long(), minlength=2).double()
    m = prob.ft.to_R(chi[0] / cnt[:, None]).cpu().numpy()[:, prob.mask]
    d = g["target"][:, prob.mask]
    edge = prob.ft.chan_edge
    num = np.bincount(edge, np.real((np.conj(m) * d).sum(1)), 2)
    den = np.bincount(edge, np.real((np.conj(m) * m).sum(1)), 2)
    sc = (num / den)[edge]
    r = (np.abs(m * sc[:, None] - d) ** 2).sum() / (np.abs(d) ** 2).sum()
    assert abs(r - float(g["best_rfactor"])) <= 1e-9 * float(g["best_rfactor"])
    mean, sd, n = smp.posterior_wc(float(prob.top.r_shell[0]), prob.top.i, prob.top.j,
                                   prob.top.shift, prob.cell, nsp=2)
    assert n == int(g["post_n"])
    np.testing.assert_allclose(mean, g["post_alpha_mean"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(sd, g["post_alpha_sd"], rtol=0, atol=1e-12)
