"""Generate the golden vectors in tests/golden/ from the reference itself.

Run in a container that has the reference checked out (its path is the first
argument, or the CHIMERA_REFERENCE environment variable):

    python tests/golden/make_golden.py /path/to/reference   (or CHIMERA_REFERENCE=...)

The reference's own Python modules are imported with `cupy` resolved to the
NumPy stand-in in tests/golden/_stub (its RawModule runs the C oracle's
restatements of the reference's NVRTC kernels). Everything saved here is
computed by reference code paths:

  lattice_*.npz   CrystalSupercell.neighbour_list           exafs_gpu/lattice.py:224-286
                  shell index, model.py:199-201; warren_cowley lattice.py:167-185
  forward.npz     ForwardModel.chi_reference (NumPy twin)   exafs_gpu/forward.py:265-293
  fourier.npz     FourierTransform(xp=np) set-up and to_R   exafs_gpu/fourier.py:21-83
  rmc_trace*.npz  RMCSampler.step/run/replica_exchange      methods/method_a_rmc.py:166-455
  ms.npz          canonical/PathClass/entry_list + SupercellMS.counts/delta
                                                            chimera/mslibrary.py:86-198, 341-492
The large neighbour lists are stored as SHA-256 digests of the arrays.
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _refpath import reference_path  # noqa: E402

REF = reference_path()
sys.path.insert(0, os.path.join(HERE, "_stub"))
sys.path.insert(0, REPO)
sys.path.insert(0, REF)

from exafs_gpu import lattice as L                      # noqa: E402
from exafs_gpu.fourier import FourierTransform          # noqa: E402
from exafs_gpu.abinitio.paths import enumerate_paths    # noqa: E402
from chimera import system as SYS, model as M           # noqa: E402
from chimera import mslibrary as ML                     # noqa: E402
from chimera.multift import MultiEdgeFT                 # noqa: E402
from methods.method_a_rmc import RMCSampler, build_reverse_index  # noqa: E402


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode() + str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def save(name, **kw):
    np.savez_compressed(os.path.join(HERE, name), **kw)
    print(f"  wrote {name}: {sorted(kw)}", flush=True)


def shell_index(cell, i, j, shift):
    """model.py:199-201, applied to the reference's own arrays."""
    d0 = np.linalg.norm((cell.ideal[j] + shift) - cell.ideal[i], axis=1)
    _, sh = np.unique(np.round(d0, 3), return_inverse=True)
    return sh.astype(np.int32), d0


def lattices():
    cases = [("fcc", (3, 3, 3), 3.59, None, 5.0, True),
             ("fcc", (5, 5, 5), 3.59, None, 6.2, True),
             ("fcc", (5, 5, 5), 3.59, None, 5.0, True),
             ("bcc", (5, 5, 10), 2.87, None, 5.0, True),
             ("hcp", (5, 5, 5), 2.50, 1.633, 5.0, True),
             ("fcc", (10, 10, 10), 3.59, None, 6.2, False)]
    out = {}
    for n, (lat, nc, a0, ca, rmax, full) in enumerate(cases):
        t = time.time()
        cell = L.CrystalSupercell(lat, nc, a0=a0, c_over_a=ca)
        i, j, sh, off = cell.neighbour_list(rmax)
        shell, d0 = shell_index(cell, i, j, sh)
        rng = np.random.default_rng(100 + n)
        sp = rng.permutation(np.repeat(np.arange(2), [cell.natoms // 2,
                                                       cell.natoms - cell.natoms // 2])
                             ).astype(np.int32)
        vals, _ = cell.shell_radii(rmax)
        wc = L.warren_cowley(sp, i, j, sh, cell, float(vals[0]), nsp=2)
        key = f"c{n}"
        out[key + "_meta"] = np.array([lat, str(nc), repr(a0), repr(ca), repr(rmax)])
        out[key + "_digest"] = np.array(digest(i, j, sh, off, shell))
        out[key + "_npairs"] = np.int64(i.size)
        out[key + "_species"] = sp
        out[key + "_wc"] = wc
        out[key + "_shell_radii"] = vals
        if full:
            out[key + "_ideal"] = cell.ideal
            out[key + "_H"] = cell.H
            out[key + "_i"], out[key + "_j"], out[key + "_shift"] = i, j, sh
            out[key + "_off"], out[key + "_shell"] = off, shell
            out[key + "_rev"] = build_reverse_index(i, j, cell.natoms)
        print(f"  lattice {lat}{nc} rmax {rmax}: {i.size} pairs [{time.time() - t:.1f}s]",
              flush=True)
    save("lattice.npz", **out)


def spectrum(ncell, rmax, kweight=(1, 2, 3)):
    sysm = SYS.AlloySystem(elements=("Fe", "Ni"), a0_ref=3.59, tables_name="analytic")
    return M.Spectrum(system=sysm, ncell=ncell, rmax=rmax, ms=False, tables="analytic",
                      kweight=kweight, kmin=3.0, kmax=13.0)


def forward():
    S = spectrum((3, 3, 3), 5.0)
    fm = S.fm
    rng = np.random.default_rng(7)
    nconf = 3
    sp = np.stack([S.random_config(s) for s in range(nconf)]).astype(np.int32)
    pos = np.repeat(S.cell.ideal[None], nconf, 0).copy()
    pos[1:] += rng.normal(0, 0.02, pos[1:].shape)
    plain = fm.chi_reference(pos, sp)
    # the same configurations with non-zero bond offsets, C3 and pair-type sigma^2
    dr = rng.normal(0, 0.01, (fm.nshell, 2, 2))
    c3 = rng.normal(0, 1e-4, fm.nshell)
    s2 = np.abs(rng.normal(0, 1e-3, (fm.nshell, 2, 2)))
    fm.set_dr(dr).set_c3(c3).set_sig2_types(s2)
    cumul = fm.chi_reference(pos, sp)
    k, f, delta, lam = S.tables.as_float64()
    save("forward.npz", k=k, f=f, delta=delta, lam=lam, s02=np.float64(fm.s02),
         i=S.i, j=S.j, shift=S.shift, shell=S.shell_idx, sig2=S.sigma2_ref,
         ideal=S.cell.ideal, species=sp, pos=pos, chi_plain=plain,
         dr=dr, c3=c3, s2types=s2, chi_cumulant=cumul)


def fourier():
    out = {}
    rng = np.random.default_rng(3)
    grids = {"model": np.linspace(M.K_LO, M.K_HI, M.NKMODEL),
             "uniform": np.arange(241) * 0.05 + 2.0,
             "shifted": M.k_exp_axis(np.linspace(M.K_LO, M.K_HI, M.NKMODEL), 9.5)}
    for gname, k in grids.items():
        for kw in (1, 2, 3):
            ft = FourierTransform(k, 3.0, 13.0, kw, dk_win=1.0, xp=np)
            chi = rng.normal(0, 0.05, (2, k.size)) * np.exp(-0.01 * k ** 2) * np.sin(5 * k)
            z = ft.to_R(chi)
            key = f"{gname}_w{kw}"
            out[key + "_k"] = k
            out[key + "_idx"], out[key + "_frac"] = ft._idx, ft._frac
            out[key + "_inside"], out[key + "_w"] = ft._inside, ft._w
            out[key + "_norm"] = np.float64(ft._norm)
            out[key + "_chi"] = chi
            out[key + "_R256"] = z[:, :256]
    # the reference's multi-edge adapter (chimera/multift.py) over its own
    # channels: edge 0 on the model axis, edge 1 on an E0-shifted axis, k^1..k^3,
    # with a fixed chi_extra added before the transform
    per_edge = [[FourierTransform(grids[g], 3.0, 13.0, kw, dk_win=1.0, xp=np) for kw in (1, 2, 3)]
                for g in ("model", "shifted")]
    mft = MultiEdgeFT([f for ch in per_edge for f in ch], chan_edge=np.repeat(np.arange(2), 3),
                      chi_extra=rng.normal(0, 0.01, (2, M.NKMODEL)))
    mchi = rng.normal(0, 0.05, (3, 2, M.NKMODEL)) * np.sin(5 * grids["model"])
    out["multi_chi"] = mchi
    out["multi_extra"] = np.asarray(mft.chi_extra)
    out["multi_R256"] = np.asarray(mft.to_R(mchi))[..., :256]
    ft = FourierTransform(grids["uniform"], 3.0, 13.0, 2, xp=np)
    out["R"] = ft.R
    out["mask_14_50"] = ft.window_mask(1.4, 5.0)
    save("fourier.npz", **out)


def make_target(S, sp_t, noise, seed):
    """A complex chi(R) target on the FFT grid: the model of configuration
    sp_t plus Gaussian noise on chi(k), through the spectrum's own transforms."""
    chi = S.fm.chi(np.asarray(S.cell.ideal[None]), sp_t[None].astype(np.int32))[0]
    chi = chi + np.random.default_rng(seed).normal(0, noise, chi.shape)
    return np.array([f.to_R(chi[e]) for f, e in zip(S.ft, S.chan_edge)])


def rmc_trace(name, ncell, rmax, nrep, nsteps, seed, swap_frac, ms_lib=None,
              energy=False):
    S = spectrum(ncell, rmax)
    sp_t = S.random_config(1000 + seed)
    target = make_target(S, sp_t, 5e-4, seed)
    mask = S.ft[0].window_mask(1.4, 5.0)
    sigR = np.full(target.shape, 2e-3)
    ft = MultiEdgeFT.from_spectrum(S)
    ep = None
    if energy:
        V = np.zeros((S.nshell, 2, 2))
        V[0] = [[0.0, -0.01], [-0.01, 0.0]]
        ep = (V, 800.0)
    ms = None
    if ms_lib is not None:
        ms = ML.SupercellMS(ms_lib, S)
        ms.set_params(sigma2_nn=0.006, r_nn=float(S.shells[0]), c_ms=1.3, amp=1.0,
                      s02=S.s02, a_scale=1.0)
    smp = RMCSampler(S.fm, ft, target, mask, sigR, nrep=nrep, seed=seed,
                     tmin=1e-4, tmax=1e-1, swap_frac=swap_frac, max_disp=0.10,
                     disp_sigma=0.012, energy_prior=ep, ms_library=ms)
    sp0 = S.random_config(seed)
    smp.init_state(sp0, S.cell.ideal)
    acc_log, c2_log, order_log = [], [], []
    step0 = smp.step
    exch0 = smp.replica_exchange

    def step():
        a = step0()
        acc_log.append(np.asarray(a).copy())
        c2_log.append(np.asarray(smp.chi2).copy())
        return a

    def exch(return_rates=False):
        # the permutation the reference applies is read off the index array it
        # gathers `count` with (method_a_rmc.py:357-362)
        seen = []

        class _Rec(np.ndarray):
            def __getitem__(self, key):
                if isinstance(key, np.ndarray) and key.dtype.kind in "iu":
                    seen.append(key.copy())
                return np.asarray(np.ndarray.__getitem__(np.asarray(self), key))
        smp.count = smp.count.view(_Rec)
        out = exch0(return_rates=return_rates)
        smp.count = np.asarray(smp.count)
        order_log.append(seen[0] if seen else np.arange(nrep))
        return out
    smp.step = step
    smp.replica_exchange = exch
    t = time.time()
    smp.run(nsteps, exchange_every=25, log_every=10 ** 9)
    print(f"  {name}: {nrep} replicas x {nsteps} steps [{time.time() - t:.1f}s], "
          f"accept {np.mean(acc_log):.3f}", flush=True)
    bsp, bpos, bc2 = smp.best()
    kw = dict(species0=sp0, target=target, mask=mask, sigR=sigR, seed=np.int64(seed),
              nrep=np.int64(nrep), nsteps=np.int64(nsteps), swap_frac=np.float64(swap_frac),
              tmin=np.float64(1e-4), tmax=np.float64(1e-1), ncell=np.array(ncell),
              rmax=np.float64(rmax), accepted=np.array(acc_log), chi2_log=np.array(c2_log),
              exch_order=np.array(order_log), final_species=smp.species,
              final_pos=smp.pos, final_chi=smp.chi, best_species=bsp, best_pos=bpos,
              best_chi2=np.float64(bc2), best_verified=np.float64(smp.best_verified),
              exchange_rate=smp.exchange_rate, chi2_init=np.array(c2_log[0]),
              energy=np.int64(bool(energy)))
    # the exact inputs the reference used, so the trace can be replayed
    k, f, delta, lam = S.tables.as_float64()
    kw.update(k=k, f=f, delta=delta, lam=lam, s02=np.float64(S.fm.s02), i=S.i, j=S.j,
              shift=S.shift, shell=S.shell_idx, sig2=S.sigma2_ref, ideal=S.cell.ideal,
              H=S.cell.H, ft_idx=np.array([f_._idx for f_ in S.ft]),
              ft_frac=np.array([f_._frac for f_ in S.ft]),
              ft_inside=np.array([f_._inside for f_ in S.ft]),
              ft_w=np.array([f_._w for f_ in S.ft]), ft_norm=np.float64(S.ft[0]._norm),
              ft_kmodel=np.array([f_.k_model for f_ in S.ft]))
    if energy:
        kw["V"], kw["T_ann"] = ep[0], np.float64(ep[1])
    if ms is not None:
        kw["ms_table_seed"] = np.int64(9)
    if ms is not None:
        kw["ms_C_final"] = ms.C
    save(name, **kw)


def ms_classes(a0=3.59, rmax_half=5.5):
    """Classes from the reference's own path enumeration and canonical form,
    ordered as classes_from_feff orders them (mslibrary.py:148)."""
    unit = a0 / 2.0
    g = np.array([[i, j, k] for i in range(-4, 5) for j in range(-4, 5) for k in range(-4, 5)])
    q = g[(g.sum(1) % 2) == 0]
    pos = q * unit
    sel = np.linalg.norm(pos, axis=1) <= rmax_half + 1e-6
    pos, q = pos[sel], q[sel]
    order = np.argsort(np.linalg.norm(pos, axis=1), kind="stable")
    pos, q = pos[order], q[order]
    groups = enumerate_paths(pos, np.zeros(len(pos), int), rmax_half, nleg_max=4,
                             group=False, absorber=0)
    keys = {}
    for G in groups:
        if G.nleg < 3:
            continue
        for s in G.members:
            k = ML.canonical(q[list(s)])
            keys[k] = keys.get(k, 0) + 1
    ks = sorted(keys, key=lambda k: (len(k), ML.PathClass(k).reff_units(), k))
    return [ML.PathClass(k) for k in ks]


class _Lib:
    """The parts of PathLibrary that SupercellMS reads (mslibrary.py:261-321),
    with the classes from ms_classes() and a seeded per-entry table."""

    def __init__(self, classes, nsp, nk, seed=5):
        self.classes = classes
        self.nsp = nsp
        self.entries = ML.entry_list(classes, nsp)
        self.nblk = len(self.entries)
        self.cls_off = np.cumsum([0] + [nsp ** c.nslot for c in classes])[:-1]
        self.T = np.random.default_rng(seed).normal(0, 0.01, (nsp * self.nblk, nk))

    def table(self, *a, **k):
        return self.T


def ms():
    classes = ms_classes()
    out = {"n_classes": np.int64(len(classes))}
    out["rep_len"] = np.array([c.rep.shape[0] for c in classes])
    out["rep"] = np.concatenate([c.rep for c in classes])
    out["nslot"] = np.array([c.nslot for c in classes])
    out["deg"] = np.array([c.deg for c in classes])
    out["reff_units"] = np.array([c.reff_units() for c in classes])
    out["slot_of"] = np.concatenate([c.slot_of for c in classes])
    imgs, img_slot = [], []
    for c in classes:
        for img, so in c.images:
            imgs.append(np.pad(img, ((0, 3 - img.shape[0]), (0, 0)), constant_values=99))
            img_slot.append(np.pad(so, (0, 3 - so.size), constant_values=99))
    out["images"] = np.array(imgs)
    out["image_slot_of"] = np.array(img_slot)
    for nsp in (2, 3):
        lib = _Lib(classes, nsp, 8)
        out[f"nblk{nsp}"] = np.int64(lib.nblk)
        out[f"cls_off{nsp}"] = lib.cls_off
        ent = np.array([[ci for ci, c in enumerate(classes) if c is cl][0] * 1000
                        + sum(s * 10 ** q for q, s in enumerate(sp))
                        for cl, sp in lib.entries])
        out[f"entries{nsp}"] = ent
    # SupercellMS on a 500-atom supercell, binary and ternary
    for nsp, els in ((2, ("Fe", "Ni")), (3, ("Fe", "Ni", "Cr"))):
        sysm = SYS.AlloySystem(elements=els, a0_ref=3.59, tables_name="analytic")
        S = M.Spectrum(system=sysm, ncell=(5, 5, 5), rmax=5.0, ms=False, tables="analytic")
        lib = _Lib(classes, nsp, S.fm.nk)
        sm = ML.SupercellMS(lib, S)
        sm.set_params(0.006, float(S.shells[0]))
        rng = np.random.default_rng(11 + nsp)
        nrep = 4
        sp = np.stack([S.random_config(s) for s in range(nrep)]).astype(np.int32)
        C = sm.counts(sp)
        a = rng.integers(0, S.cell.natoms, nrep).astype(np.int32)
        b = rng.integers(0, S.cell.natoms, nrep).astype(np.int32)
        b[0] = a[0]                          # a displacement: no change
        # make replica 1 swap two neighbours (paths through both sites)
        b[1] = S.j[a[1] * (S.i.size // S.cell.natoms)]
        nsa = sp[np.arange(nrep), b].astype(np.int32)
        nsb = sp[np.arange(nrep), a].astype(np.int32)
        nsa[0] = nsb[0] = sp[0, a[0]]
        chi_d = sm.delta(sp, a, b, nsa, nsb)
        key = f"sc{nsp}_"
        out[key + "npath"] = np.int64(sm.npath)
        out[key + "M"] = np.int64(sm.M)
        out[key + "digest"] = np.array(digest(np.asarray(sm.d_abs), np.asarray(sm.d_cls),
                                              np.asarray(sm.d_slot), np.asarray(sm.d_inc)))
        out[key + "abs_head"] = np.asarray(sm.d_abs)[:3000]
        out[key + "cls_head"] = np.asarray(sm.d_cls)[:3000]
        out[key + "slot_head"] = np.asarray(sm.d_slot)[:3000]
        out[key + "inc_head"] = np.asarray(sm.d_inc)[:3]
        out[key + "species"] = sp
        out[key + "counts"] = C
        out[key + "a"], out[key + "b"], out[key + "nsa"], out[key + "nsb"] = a, b, nsa, nsb
        out[key + "dC"] = sm._dC
        out[key + "chi_delta"] = chi_d
        print(f"  SupercellMS nsp={nsp}: {sm.npath} paths, M={sm.M}", flush=True)
    save("ms.npz", **out)


if __name__ == "__main__":
    which = sys.argv[2:] or ["lattice", "forward", "fourier", "ms", "rmc"]
    if "lattice" in which:
        lattices()
    if "forward" in which:
        forward()
    if "fourier" in which:
        fourier()
    if "ms" in which:
        ms()
    if "rmc" in which:
        rmc_trace("rmc_trace.npz", (5, 5, 5), 5.0, 8, 300, 3, 1.0)
        rmc_trace("rmc_trace_disp.npz", (3, 3, 3), 5.0, 6, 200, 4, 0.5, energy=True)
        cls = ms_classes()
        rmc_trace("rmc_trace_ms.npz", (5, 5, 5), 5.0, 4, 150, 5, 1.0,
                  ms_lib=_Lib(cls, 2, M.NKMODEL, seed=9))
