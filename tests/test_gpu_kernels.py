"""Device kernels against the oracle, through the C ABI."""
import numpy as np
import pytest

from cases import trace_inputs
from oracle import kernels as K

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def test_reference_kernels_match_oracle(cuda):
    torch = cuda
    from chimera_b200 import _native as N
    d = trace_inputs("rmc_trace_disp.npz")
    nsp = d["nsp"]
    natoms = d["ideal"].shape[0]
    npairs = d["i"].size
    ncoord = npairs // natoms
    nrep, nk = 6, d["k"].size
    rng = np.random.default_rng(1)
    sp = np.stack([rng.permutation(d["species0"]) for _ in range(nrep)]).astype(np.int32)
    pos = np.repeat(d["ideal"][None], nrep, 0) + rng.normal(0, 0.01, (nrep, natoms, 3))
    ideal = np.repeat(d["ideal"][None], nrep, 0)
    S = N.stream()
    # compute_r, build_ptype
    r = torch.empty((nrep, npairs), dtype=torch.float64, device="cuda")
    ev = torch.empty((nrep, npairs, 3), dtype=torch.float64, device="cuda")
    gp, gi, gj, gs = _dev(torch, pos), _dev(torch, d["i"]), _dev(torch, d["j"]), _dev(torch, d["shift"])
    N.call("chx_compute_r", N.ptr(gp), N.ptr(gi), N.ptr(gj), N.ptr(gs), N.ptr(r), N.ptr(ev),
           npairs, natoms, nrep, S)
    r_o = np.zeros((nrep, npairs)); ev_o = np.zeros((nrep, npairs, 3))
    K.compute_r(pos, d["i"], d["j"], d["shift"], r_o, ev_o, npairs, natoms, nrep)
    assert np.allclose(r.cpu().numpy(), r_o, rtol=1e-15, atol=0)
    assert np.allclose(ev.cpu().numpy(), ev_o, rtol=0, atol=1e-15)
    pt = torch.empty((nrep, npairs), dtype=torch.int32, device="cuda")
    gsp = _dev(torch, sp)
    N.call("chx_build_ptype", N.ptr(gsp), N.ptr(gi), N.ptr(gj), N.ptr(pt), npairs, natoms, nrep,
           nsp, S)
    pt_o = np.zeros((nrep, npairs), np.int32)
    K.build_ptype(sp, d["i"], d["j"], pt_o, npairs, natoms, nrep, nsp)
    assert np.array_equal(pt.cpu().numpy(), pt_o)
    # chi_forward FP64
    nshell = int(d["shell"].max()) + 1
    dr = rng.normal(0, 0.01, nshell * nsp * nsp); c3 = rng.normal(0, 1e-4, nshell)
    s2 = np.abs(rng.normal(0, 1e-3, nshell * nsp * nsp))
    delta = np.ascontiguousarray(d["delta"].reshape(nsp * nsp, -1))
    tabs = [_dev(torch, x) for x in (d["shell"], d["sig2"], d["f"], delta, d["lam"], d["k"], dr, c3, s2)]
    chi = torch.empty((nrep, nsp, nk), dtype=torch.float64, device="cuda")
    N.call("chx_chi_forward", N.ptr(r), N.ptr(pt), *[N.ptr(t) for t in tabs], N.ptr(chi),
           npairs, nk, nrep, float(d["s02"]), nsp, S)
    chi_o = np.zeros((nrep, nsp, nk))
    K.chi_forward(r_o, pt_o, d["shell"], d["sig2"], d["f"], delta, d["lam"], d["k"], dr, c3, s2,
                  chi_o, npairs, nk, nrep, float(d["s02"]), nsp)
    assert np.abs(chi.cpu().numpy() - chi_o).max() <= 1e-12 * np.abs(chi_o).max()
    # propose_select: bit-identical integers, FP64 positions to rounding
    outs = dict(a=torch.empty(nrep, dtype=torch.int32, device="cuda"))
    for k_ in ("b", "nsa", "nsb"):
        outs[k_] = torch.empty(nrep, dtype=torch.int32, device="cuda")
    npa = torch.empty((nrep, 3), dtype=torch.float64, device="cuda")
    isw = torch.empty(nrep, dtype=torch.uint8, device="cuda")
    gid = _dev(torch, ideal)
    for stepc, sf in ((1, 1.0), (2, 0.5), (3, 0.0), (77, 0.75)):
        N.call("chx_propose_select", N.ptr(gsp), N.ptr(gp), N.ptr(gid), N.ptr(outs["a"]),
               N.ptr(outs["b"]), N.ptr(outs["nsa"]), N.ptr(outs["nsb"]), N.ptr(npa), N.ptr(isw),
               natoms, nrep, 12345, stepc, sf, 0.012, 0.10, S)
        o = dict(a=np.zeros(nrep, np.int32), b=np.zeros(nrep, np.int32),
                 nsa=np.zeros(nrep, np.int32), nsb=np.zeros(nrep, np.int32))
        npa_o = np.zeros((nrep, 3)); isw_o = np.zeros(nrep, np.uint8)
        K.propose_select(sp, pos, ideal, o["a"], o["b"], o["nsa"], o["nsb"], npa_o, isw_o, natoms,
                         nrep, 12345, stepc, sf, 0.012, 0.10)
        for k_ in o:
            assert np.array_equal(outs[k_].cpu().numpy(), o[k_]), (stepc, k_)
        assert np.array_equal(isw.cpu().numpy(), isw_o)
        assert np.allclose(npa.cpu().numpy(), npa_o, rtol=0, atol=1e-14)
    # propose_build + chi_delta + commits on the last proposal
    maxaff = 4 * ncoord
    rev = np.argsort(d["i"].astype(np.int64) * natoms + d["j"])[np.searchsorted(
        np.sort(d["i"].astype(np.int64) * natoms + d["j"]), d["j"].astype(np.int64) * natoms + d["i"])]
    rev = rev.astype(np.int32)
    nbr = np.arange(npairs, dtype=np.int32).reshape(natoms, ncoord)
    aff = torch.empty((nrep, maxaff), dtype=torch.int32, device="cuda")
    rnew = torch.empty((nrep, maxaff), dtype=torch.float64, device="cuda")
    ptn = torch.empty((nrep, maxaff), dtype=torch.int32, device="cuda")
    g_nbr, g_rev = _dev(torch, nbr), _dev(torch, rev)
    N.call("chx_propose_build", N.ptr(gsp), N.ptr(gp), N.ptr(g_nbr), N.ptr(g_rev), N.ptr(gi),
           N.ptr(gj), N.ptr(gs), N.ptr(outs["a"]), N.ptr(outs["b"]), N.ptr(outs["nsa"]),
           N.ptr(outs["nsb"]), N.ptr(npa), N.ptr(aff), N.ptr(rnew), N.ptr(ptn), natoms, ncoord,
           npairs, nrep, maxaff, nsp, S)
    aff_o = np.zeros((nrep, maxaff), np.int32); rn_o = np.zeros((nrep, maxaff)); ptn_o = np.zeros((nrep, maxaff), np.int32)
    K.propose_build(sp, pos, nbr, rev, d["i"], d["j"], d["shift"], o["a"], o["b"], o["nsa"],
                    o["nsb"], npa_o, aff_o, rn_o, ptn_o, natoms, ncoord, npairs, nrep, maxaff, nsp)
    assert np.array_equal(aff.cpu().numpy(), aff_o)
    assert np.array_equal(ptn.cpu().numpy(), ptn_o)
    assert np.allclose(rnew.cpu().numpy(), rn_o, rtol=1e-14, atol=0)
    dchi = torch.empty((nrep, nsp, nk), dtype=torch.float64, device="cuda")
    N.call("chx_chi_delta", N.ptr(r), N.ptr(pt), N.ptr(tabs[0]), N.ptr(aff), N.ptr(rnew),
           N.ptr(ptn), *[N.ptr(t) for t in tabs[1:]], N.ptr(dchi), npairs, nk, nrep, maxaff,
           float(d["s02"]), nsp, S)
    dchi_o = np.zeros((nrep, nsp, nk))
    K.chi_delta(r_o, pt_o, d["shell"], aff_o, rn_o, ptn_o, d["sig2"], d["f"], delta, d["lam"],
                d["k"], dr, c3, s2, dchi_o, npairs, nk, nrep, maxaff, float(d["s02"]), nsp)
    assert np.abs(dchi.cpu().numpy() - dchi_o).max() <= 1e-12 * max(np.abs(dchi_o).max(), 1e-30)
    acc = np.array([1, 0, 1, 1, 0, 1], np.uint8)
    gacc = _dev(torch, acc)
    N.call("chx_commit_move", N.ptr(aff), N.ptr(rnew), N.ptr(ptn), N.ptr(gacc), N.ptr(r),
           N.ptr(pt), npairs, nrep, maxaff, S)
    K.commit_move(aff_o, rn_o, ptn_o, acc, r_o, pt_o, npairs, nrep, maxaff)
    assert np.array_equal(pt.cpu().numpy(), pt_o)
    N.call("chx_commit_state", N.ptr(gacc), N.ptr(outs["a"]), N.ptr(outs["b"]), N.ptr(outs["nsa"]),
           N.ptr(outs["nsb"]), N.ptr(npa), N.ptr(isw), N.ptr(gsp), N.ptr(gp), natoms, nrep, S)
    K.commit_state(acc, o["a"], o["b"], o["nsa"], o["nsb"], npa_o, isw_o, sp, pos, natoms, nrep)
    assert np.array_equal(gsp.cpu().numpy(), sp)
    assert np.allclose(gp.cpu().numpy(), pos, rtol=0, atol=1e-14)


def test_kernels_get_forwards_reference_argument_tuples(cuda):
    """chimera_b200.kernels.get(name, nsp) takes the reference's call form."""
    torch = cuda
    from chimera_b200 import kernels as KK
    d = trace_inputs("rmc_trace_disp.npz")
    nsp = d["nsp"]
    natoms = d["ideal"].shape[0]
    npairs = d["i"].size
    nrep = 2
    rng = np.random.default_rng(5)
    pos = np.repeat(d["ideal"][None], nrep, 0) + rng.normal(0, 0.01, (nrep, natoms, 3))
    sp = np.stack([rng.permutation(d["species0"]) for _ in range(nrep)]).astype(np.int32)
    r = torch.empty((nrep, npairs), dtype=torch.float64, device="cuda")
    ev = torch.empty((nrep, npairs, 3), dtype=torch.float64, device="cuda")
    KK.get("compute_r", nsp)((1,), (256,), (_dev(torch, pos), _dev(torch, d["i"]),
                                            _dev(torch, d["j"]), _dev(torch, d["shift"]), r, ev,
                                            np.int32(npairs), np.int32(natoms), np.int32(nrep)))
    r_o = np.zeros((nrep, npairs))
    K.compute_r(pos, d["i"], d["j"], d["shift"], r_o, None, npairs, natoms, nrep)
    assert np.allclose(r.cpu().numpy(), r_o, rtol=1e-15, atol=0)
    pt = torch.empty((nrep, npairs), dtype=torch.int32, device="cuda")
    KK.get("build_ptype", nsp)((1,), (256,), (_dev(torch, sp), _dev(torch, d["i"]),
                                              _dev(torch, d["j"]), pt, np.int32(npairs),
                                              np.int32(natoms), np.int32(nrep)))
    pt_o = np.zeros((nrep, npairs), np.int32)
    K.build_ptype(sp, d["i"], d["j"], pt_o, npairs, natoms, nrep, nsp)
    assert np.array_equal(pt.cpu().numpy(), pt_o)
