"""Full path sum (A1) and MS counts (A2) on the device against the oracle's
pinned references."""
import types

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _fm(g, cumulant):
    from chimera_b200.forward import ForwardModel
    from chimera_b200.tables import ScatteringTables
    cell = types.SimpleNamespace(ideal=g["ideal"], natoms=g["ideal"].shape[0])
    t = ScatteringTables(k=g["k"], f=g["f"], delta=g["delta"], lam=g["lam"], s02=float(g["s02"]))
    fm = ForwardModel(cell, t, g["i"], g["j"], g["shift"], sigma2=g["sig2"], shell=g["shell"])
    if cumulant:
        fm.set_dr(g["dr"]).set_c3(g["c3"]).set_sig2_types(g["s2types"])
    return fm


@pytest.mark.parametrize("which", ["chi_plain", "chi_cumulant"])
def test_chi_full_fp64_and_fp32c(cuda, which):
    from chimera_b200.forward import FP64, FP32C
    g = golden("forward.npz")
    fm = _fm(g, which == "chi_cumulant")
    ref = g[which]
    c64 = fm.chi(g["pos"], g["species"], precision=FP64).cpu().numpy()
    assert np.abs(c64 - ref).max() <= 1e-12 * np.abs(ref).max()
    c32 = fm.chi(g["pos"], g["species"], precision=FP32C).cpu().numpy()
    # chi(k) within 1e-6 absolute of FP64
    assert np.abs(c32 - ref).max() <= 1e-6
    # the reference-kernel route (r and ptype given) agrees too
    r, _ = fm.distances(g["pos"])
    pt = fm.ptypes(g["species"])
    cr = fm.chi(g["pos"], g["species"], r=r, ptype=pt).cpu().numpy()
    assert np.abs(cr - ref).max() <= 1e-12 * np.abs(ref).max()


def test_chi_full_4000_atoms_fp32c_within_1e6(cuda):
    """Config-1 size: 4,000-atom fcc Fe-Ni, 78 neighbours, smooth tables, 241 k."""
    from chimera_b200 import lattice as L
    from chimera_b200.forward import ForwardModel, FP64, FP32C
    from chimera_b200.tables import smooth_tables, uniform_k
    cell = L.CrystalSupercell("fcc", (10, 10, 10), 3.59)
    top = L.Topology(cell, 6.2, sigma2=0.006)
    fm = ForwardModel(cell, smooth_tables(uniform_k(), ("Fe", "Ni")), top.i, top.j, top.shift,
                      sigma2=top.sigma2, shell=top.shell)
    rng = np.random.default_rng(0)
    sp = np.stack([L.random_config(cell.natoms, (0.5, 0.5), s) for s in range(4)])
    pos = np.repeat(cell.ideal[None], 4, 0)
    pos[2:] += rng.normal(0, 0.02, pos[2:].shape)
    c64 = fm.chi(pos, sp, precision=FP64).cpu().numpy()
    c32 = fm.chi(pos, sp, precision=FP32C).cpu().numpy()
    err = np.abs(c32 - c64)
    assert err.max() <= 1e-6, err.max()


def test_ms_counts_delta_chi_of(cuda):
    torch = cuda
    from chimera_b200 import lattice as L
    from chimera_b200 import mspaths as MP
    g = golden("ms.npz")
    classes = MP.enumerate_classes(3.59, 5.5)
    cell = L.CrystalSupercell("fcc", (5, 5, 5), 3.59)
    for nsp in (2, 3):
        key = f"sc{nsp}_"
        paths = MP.SupercellPaths(classes, cell.ideal, cell.H, 3.59, nsp)
        T = np.random.default_rng(5).normal(0, 0.01, (paths.nent, 320))
        ms = MP.SupercellMS(paths, T)
        C = ms.counts(g[key + "species"]).cpu().numpy()
        assert np.array_equal(C, g[key + "counts"])
        chi_d = ms.delta(g[key + "species"], g[key + "a"], g[key + "b"], g[key + "nsa"],
                         g[key + "nsb"]).cpu().numpy()
        assert np.array_equal(ms._dC.cpu().numpy(), g[key + "dC"])
        assert np.allclose(chi_d, g[key + "chi_delta"], rtol=0, atol=1e-13)
        full = ms.full(g[key + "species"]).cpu().numpy()
        ref = np.stack([g[key + "counts"][:, a * paths.nblk:(a + 1) * paths.nblk]
                        @ T[a * paths.nblk:(a + 1) * paths.nblk] for a in range(nsp)], axis=1)
        assert np.allclose(full, ref, rtol=0, atol=1e-12)


def test_chi_full_reports_device_errors(cuda):
    """Out-of-range species and pair indices are caught on the device: the
    error word is set (ChxError from ForwardModel.chi_full) and chi is NaN."""
    import torch
    from chimera_b200 import _native as N
    from chimera_b200.forward import FP64
    g = golden("forward.npz")
    fm = _fm(g, False)
    sp = np.array(g["species"], np.int32).copy()
    sp[0, 3] = fm.nsp
    with pytest.raises(N.ChxError, match="error word"):
        fm.chi_full(torch.from_numpy(np.asarray(g["pos"])).cuda(), torch.from_numpy(sp).cuda(),
                    precision=FP64)
    out = fm.chi_full(torch.from_numpy(np.asarray(g["pos"])).cuda(),
                      torch.from_numpy(sp).cuda(), precision=FP64, check=False)
    assert torch.isnan(out).all()
    good = fm.chi_full(torch.from_numpy(np.asarray(g["pos"])).cuda(),
                       torch.from_numpy(np.array(g["species"], np.int32)).cuda(), precision=FP64)
    assert torch.isfinite(good).all()
