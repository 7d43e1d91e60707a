"""Golden vectors of the pair-count calibration objective, from the reference.

Run where the reference is checked out (its path is the first argument
or the CHIMERA_REFERENCE environment variable):

    python tests/golden/make_shellmodel_golden.py /path/to/reference   (or CHIMERA_REFERENCE=...)

It builds the reference's own `model.Spectrum` (fcc Fe-Ni, 4x4x4 cells,
rmax 6.2 A, its analytic Z-parameterised tables, no multiple-scattering
library) and `shellmodel.ShellModel.from_spectrum`, then evaluates
`ShellModel.r_factor` (chimera/shellmodel.py:427-440) at seeded random
parameter sets spanning the calibration's search ranges
(chimera/calibrate.py:129-193), against complex chi(R) data and against
|chi(R)| data made by the same model at a reference parameter set plus
seeded noise. It saves the model inputs, the data, every parameter set in
the flat layout of chimera_b200.shellmodel, the reference's R-factors and
per-edge amplitudes, its global-stage search vector (calibrate.Stage1) and
its Cramer-Rao bounds (shellmodel.crlb, :449-593) at the data's parameters
(shellmodel.npz).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _refpath import reference_path  # noqa: E402

REF = reference_path()
sys.path.insert(0, os.path.join(HERE, "_stub"))
sys.path.insert(0, REF)

from chimera import model as M                     # noqa: E402
from chimera import shellmodel as SM                # noqa: E402
from chimera import calibrate as CAL                # noqa: E402


def flat(p, nsp, nshell):
    """The parameter dict as chimera_b200.shellmodel lays it out."""
    return np.concatenate([[p["a0"], p["sigma_scale"], p["ms_amp"], p["ms_c"],
                            float(np.atleast_1d(p["kmin"])[0]), float(np.atleast_1d(p["kmax"])[0])],
                           np.asarray(p["dE0"], float).ravel(),
                           np.asarray(p["sigma_shell_scale"], float).ravel(),
                           np.asarray(p["dr"], float).ravel(),
                           np.asarray(p["c3"], float).ravel(),
                           np.asarray(p["c4"], float).ravel(),
                           np.asarray(p["sigma_pair"], float).ravel(),
                           np.asarray(p["ms_amp_edge"], float).ravel()])


def main():
    S = M.Spectrum(elements=("Fe", "Ni"), composition=(0.5, 0.5), a0_ref=3.59,
                   lattice="fcc", tables="analytic", ms=False, ncell=(4, 4, 4), rmax=6.2)
    sm = SM.ShellModel.from_spectrum(S)
    nsp, nshell = sm.nsp, sm.nshell
    kw = (1, 2, 3)
    comp = np.array([0.5, 0.5])
    N0 = sm.random_counts()
    rng = np.random.default_rng(0)
    sp = rng.permutation(np.repeat(np.arange(nsp), sm.natoms // nsp))
    N1 = sm.counts_of(sp)
    # data: the model at a reference parameter set, plus seeded noise
    true = dict(a0=3.585, dE0=np.array([1.5, -0.8]), kmin=3.0, kmax=13.0, kweight=kw,
                sigma_scale=1.2, sigma_shell_scale=np.array([1, 1.1, 0.9, 1.05, 1.0]),
                dr=SM.dr_from_free([0.01, -0.004], comp), c3=[2e-4])
    sm.set_params(**true)
    R_data = sm.R[:200].copy()
    idx = M.match_grid(sm.R, R_data)
    mask = (R_data > 1.4) & (R_data < 5.0)
    z = sm.chi_R(N1, idx)
    noise = rng.normal(0, 2e-4, z.shape) + 1j * rng.normal(0, 2e-4, z.shape)
    data_c = z + noise
    data_m = np.abs(z) + rng.normal(0, 2e-4, z.shape)
    sets, rf_c, sc_c, rf_m, sc_m, rf_n0 = [], [], [], [], [], []
    for q in range(24):
        p = dict(a0=3.59 * rng.uniform(0.97, 1.02), dE0=rng.uniform(-6, 8, nsp),
                 kmin=rng.uniform(2.6, 3.8), kmax=rng.uniform(11.5, 14.5), kweight=kw,
                 sigma_scale=np.exp(rng.uniform(np.log(0.6), np.log(4))),
                 sigma_shell_scale=np.r_[1.0, np.exp(rng.uniform(np.log(0.5), np.log(2), nshell - 1))],
                 dr=SM.dr_from_free(rng.uniform(-0.05, 0.05, 2), comp),
                 c3=[rng.uniform(-5e-4, 5e-4)],
                 c4=[rng.uniform(-2e-5, 2e-5) if q % 3 == 0 else 0.0],
                 sigma_pair=(SM.pair_log_from_free(rng.uniform(-0.5, 0.5, 2), comp)
                             if q % 2 else np.ones((nsp, nsp))))
        sm.set_params(**p)
        sets.append(flat(sm.p, nsp, nshell))
        r, s = sm.r_factor(N1, data_c, mask, idx, return_scales=True)
        rf_c.append(r)
        sc_c.append(s)
        r, s = sm.r_factor(N1, data_m, mask, idx, return_scales=True)
        rf_m.append(r)
        sc_m.append(s)
        rf_n0.append(sm.r_factor(N0, data_c, mask, idx))
    # the global stage's search vector (calibrate.py:126-247) -> parameters
    stage = CAL.Stage1(sm, comp, ms=True, free_window=True, free_dr=True, free_c3=True,
                       free_shell_sigma=True, free_c4=True, free_sigma_pair=True,
                       free_ms_edge=True, elements=("Fe", "Ni"))
    lo = np.array([b[0] for b in stage.bounds]); hi = np.array([b[1] for b in stage.bounds])
    X = lo + (hi - lo) * rng.uniform(size=(6, lo.size))
    base = dict(sm.p)
    stage_rows = []
    for x in X:
        sm.p = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in base.items()}
        q = stage.unpack(x)
        q.setdefault("a0", 3.59)
        sm.set_params(kweight=kw, **q)
        stage_rows.append(flat(sm.p, nsp, nshell))
    sm.p = base
    # Cramer-Rao bounds (shellmodel.py:449-593) at the data's parameters
    sm.set_params(**true)
    crlb_base = flat(sm.p, nsp, nshell)
    sig = np.full(nsp * len(kw), 2e-4)
    cr = {}
    for tag, dat in (("c", data_c), ("m", data_m)):
        r = SM.crlb(sm, N1, dat, sig, mask, idx)
        ns = r["nuisance_sd"]
        cr[f"crlb_{tag}_alpha_sd"] = np.array(r["alpha_sd"])
        cr[f"crlb_{tag}_eig_sd"] = np.array(r["eig_sd"])
        cr[f"crlb_{tag}_alpha_cov"] = np.array(r["alpha_cov"])
        cr[f"crlb_{tag}_nuis"] = np.concatenate([np.atleast_1d(ns[k]) for k in
                                                 ("a0", "sigma_scale", "ms_amp", "dE0", "dr",
                                                  "c3")])
        cr[f"crlb_{tag}_dr_entry_sd"] = np.array(r["dr_entry_sd"])
    _, f, delta, lam = S.tables.as_float64()
    out = dict(k=np.asarray(sm.k, float), f=f, delta=delta.reshape(nsp * nsp, -1), lam=lam,
               shells_ref=sm.shells_ref, shell_mult=sm.z, sigma2_shell_ref=sm.sigma2_shell_ref,
               natoms=np.int64(sm.natoms), a0_ref=np.float64(sm.a0_ref),
               s02=np.float64(sm.s02), dk_win=np.float64(sm.dk_win), etok=np.float64(M.ETOK),
               kweight=np.array(kw), N0=N0, N1=N1, R_data=R_data, idx=idx, mask=mask,
               data_c=data_c, data_m=data_m, params=np.array(sets),
               rf_c=np.array(rf_c), scales_c=np.array(sc_c), rf_m=np.array(rf_m),
               scales_m=np.array(sc_m), rf_n0=np.array(rf_n0),
               stage_names=np.array(stage.names), stage_bounds=np.array(stage.bounds),
               stage_x0=stage.x0(), stage_dE0_start=np.float64(stage.dE0_start),
               stage_X=X, stage_rows=np.array(stage_rows),
               stage_base=flat(base, nsp, nshell), crlb_base=crlb_base, crlb_sigma=sig, **cr)
    np.savez_compressed(os.path.join(HERE, "shellmodel.npz"), **out)
    print("wrote shellmodel.npz:", {k: np.shape(v) for k, v in out.items()})
    print("R-factors (complex):", np.round(out["rf_c"], 4))


if __name__ == "__main__":
    main()
