"""The systematic band: the fit under each calibration variant, in one launch.

The reference refits the data once per calibration variant, one after the
other (chimera/fitrun.py:652-718, the variants :466-488), and reads the
spread of the Warren-Cowley parameters over the variants the data cannot
reject as the systematic error (band_from_variants, :491-536). Each variant
changes the model (a0, sigma^2 scale, MS amplitude, E0 shift), the
transform (k weights, k window) or the fitted R range, never the data; so
every variant is one temperature ladder with its own forward model,
transform, target and fit mask, and `systematic_band` runs all of them (times
the sample seeds) as one `BatchedSampler`: one step launch per exchange
period for the whole band.

`variant_specs` builds the ladders from a `configs.Problem` (the baseline
calibration): variants of a0 and sigma^2 get a supercell / forward model of
their own, E0 shifts move the model's k axis (k^2 - 0.2624682843 dE0,
chimera/model.py:120-130) while the data keep theirs, k-weight and k-window
variants re-transform the data as well as the model (the chi(k)-data case of
the reference), R-range variants change the fit mask, MS variants scale the
exact MS table. The result of a variant is its best state's first-shell
Warren-Cowley vector and R-factors (its own R range and the baseline's).
"""
from __future__ import annotations

import numpy as np

from . import configs
from .fourier import EdgeTransforms

ETOK = 0.2624682843

# the reference's variant table (chimera/fitrun.py:466-488)
CALIB_VARIANTS = [
    ("baseline", {}),
    ("a0 -0.005 A", dict(da0=-0.005)),
    ("a0 +0.005 A", dict(da0=+0.005)),
    ("dE0 -2 eV", dict(ddE0=-2.0)),
    ("dE0 +2 eV", dict(ddE0=+2.0)),
    ("sigma x0.85", dict(fsig=0.85)),
    ("sigma x1.15", dict(fsig=1.15)),
    ("k weight 2", dict(kweight=2)),
    ("k weight 4", dict(kweight=4)),
    ("k min +0.5", dict(dkmin=+0.5)),
    ("k max -1.0", dict(dkmax=-1.0)),
    ("R min +0.1", dict(drmin=+0.1)),
    ("R max -0.4", dict(drmax=-0.4)),
    ("R max +0.2", dict(drmax=+0.2)),
    ("ms_amp x0.85", dict(fms=0.85)),
    ("ms_amp x1.15", dict(fms=1.15)),
    ("no dr", dict(dr_off=True)),
    ("no C3", dict(c3_off=True)),
]


def band_from_variants(rows, tol=1.3):
    """The Warren-Cowley spread over the variants the data cannot reject
    (chimera/fitrun.py:491-536): variants with another number of channels are
    not comparable; among the comparable ones a variant counts when its
    R-factor (on the common R range) is within `tol` of the baseline's
    (rows[0]), and one that fits better always counts."""
    W = np.array([r["wc"] for r in rows])
    rf = np.array([r["r_factor_common"] if r.get("r_factor_common") is not None
                   else r["r_factor"] for r in rows])
    nch = np.array([r.get("n_channels", 0) for r in rows])
    comparable = nch == nch[0]
    keep = comparable & (rf <= tol * rf[0])
    keep[0] = True
    Wk = W[keep]
    better = [r["variant"] for r, k, c in zip(rows, rf < rf[0], comparable) if k and c]
    return dict(wc_mean=W[comparable].mean(0).tolist(), wc_sd=W[comparable].std(0).tolist(),
                wc_min=Wk.min(0).tolist(), wc_max=Wk.max(0).tolist(),
                wc_min_all=W[comparable].min(0).tolist(),
                wc_max_all=W[comparable].max(0).tolist(),
                n_admissible=int(keep.sum()), n_variants=int(len(rows)),
                n_comparable=int(comparable.sum()),
                admissible=[r["variant"] for r, k in zip(rows, keep) if k],
                excluded_incomparable=[r["variant"] for r, c in zip(rows, comparable) if not c],
                fit_better_than_baseline=better, r_factor_baseline=float(rf[0]),
                r_factor_range=[float(rf[comparable].min()), float(rf[comparable].max())])


class Variant:
    """One variant's model, transforms, target and masks."""

    def __init__(self, name, prob, ft_model, ft_data, kweights, rwin, ms, dE0):
        self.name, self.prob, self.ft, self.ft_data = name, prob, ft_model, ft_data
        self.kweights, self.rwin, self.ms, self.dE0 = kweights, rwin, ms, dE0


def _fts(prob, k_model, kmin, kmax, kweights, window):
    return EdgeTransforms.build([k_model[e] for e in range(prob.nsp)], kmin, kmax, kweights,
                                window=window)


def build_variants(base_kw, variants=CALIB_VARIANTS, window=None):
    """Variant models around the baseline problem built from `base_kw`
    (configs.Problem keywords). Problems are shared between variants that do
    not change the supercell."""
    base = configs.Problem(**base_kw)
    window = window or base_kw.get("window", "kaiser")
    kw0 = tuple(base_kw.get("kweights", (1, 2, 3)))
    kmin0, kmax0 = base_kw.get("kmin", 3.0), base_kw.get("kmax", 13.0)
    rwin0 = tuple(base_kw.get("rwin", (1.4, 5.0)))
    a0, s2 = base_kw.get("a0", 3.59), base_kw.get("sigma2", 0.006)
    out = []
    for name, ch in variants:
        prob = base
        if "da0" in ch or "fsig" in ch:
            kw = dict(base_kw)
            kw["a0"] = a0 + ch.get("da0", 0.0)
            kw["sigma2"] = s2 * ch.get("fsig", 1.0)
            prob = configs.Problem(**kw)
        kws = (int(ch["kweight"]),) if "kweight" in ch else kw0
        kmin = kmin0 + ch.get("dkmin", 0.0)
        kmax = kmax0 + ch.get("dkmax", 0.0)
        rwin = (rwin0[0] + ch.get("drmin", 0.0), rwin0[1] + ch.get("drmax", 0.0))
        dE0 = ch.get("ddE0", 0.0)
        k = prob.k
        k_model = [np.sqrt(np.maximum(k ** 2 - ETOK * dE0, 1e-4))] * prob.nsp
        ft_model = _fts(prob, k_model, kmin, kmax, kws, window)
        ft_data = _fts(prob, [k] * prob.nsp, kmin, kmax, kws, window)
        ms = prob.ms
        if ms is not None and "fms" in ch:
            from .mspaths import SupercellMS
            ms = SupercellMS(prob.paths, prob.ms_table * ch["fms"])
        out.append(Variant(name, prob, ft_model, ft_data, kws, rwin, ms, dE0))
    return base, out


def variant_specs(base, variants, positions=(0,), nrep=16, tmin=1e-4, tmax=1e-1, seed0=0,
                  swap_frac=1.0):
    """LadderSpecs of every (variant, position): the data of a position are
    the baseline's noisy chi(k), transformed with the variant's own k
    weights and window; its sigma_R is the noise through that transform."""
    from .sampler import LadderSpec
    specs, meta = [], []
    for p in positions:
        data_k = base.target_chi() + base.noise_k(p)
        for v in variants:
            fd = v.ft_data
            target = np.array([f.to_R(data_k[e]) for f, e in zip(fd.fts, fd.chan_edge)])
            sig = np.array([base.noise * np.sqrt(0.5 * (np.abs(f.basis()) ** 2).sum(0))
                            for f in fd.fts])
            mask = fd.window_mask(*v.rwin)
            specs.append(LadderSpec(v.prob.fm, v.ft, target, mask, np.maximum(sig, 1e-12),
                                    nrep=nrep, tmin=tmin, tmax=tmax, seed=seed0 + len(specs),
                                    swap_frac=swap_frac, ms_library=v.ms))
            meta.append((v, p))
    return specs, meta


def variant_result(bs, li, v, spec, common_mask):
    """Best state of ladder li: first-shell Warren-Cowley vector (a <= b)
    and R-factors on the variant's range and on the common range
    (chimera/model.py:497-545 with per-edge amplitudes)."""
    import torch
    sp, _ = bs.best(li)
    prob = v.prob
    sp_d = torch.from_numpy(sp[None].astype(np.int32)).cuda()
    chi = prob.fm.chi_full(torch.from_numpy(prob.cell.ideal[None]).cuda(), sp_d)
    if v.ms is not None:
        chi = chi + v.ms.full(sp_d)
    cnt = np.bincount(sp, minlength=prob.nsp).astype(np.float64)
    chi = chi[0].cpu().numpy() / np.maximum(cnt, 1)[:, None]
    m = np.array([f.to_R(chi[e]) for f, e in zip(v.ft.fts, v.ft.chan_edge)])
    d = spec.target
    edge = np.asarray(v.ft.chan_edge)

    def rf(mask):
        num = np.real((np.conj(m[:, mask]) * d[:, mask]).sum(1))
        den = np.real((np.conj(m[:, mask]) * m[:, mask]).sum(1))
        ne = int(edge.max()) + 1
        sc = (np.bincount(edge, num, ne) / np.maximum(np.bincount(edge, den, ne), 1e-30))[edge]
        return float((np.abs(m[:, mask] * sc[:, None] - d[:, mask]) ** 2).sum()
                     / max((np.abs(d[:, mask]) ** 2).sum(), 1e-30))

    alpha = prob.alpha1(sp)
    iu = np.triu_indices(prob.nsp)
    return dict(variant=v.name, wc=alpha[iu].tolist(), r_factor=rf(spec.mask),
                r_factor_common=rf(common_mask), n_channels=int(m.shape[0]),
                kweights=list(v.kweights))


def systematic_band(base_kw, variants=CALIB_VARIANTS, positions=(0,), nrep=16, blocks=240,
                    tmin=1e-4, tmax=1e-1, precision=1, tol=1.3, starts_seed=100):
    """Every variant x position as one batched sampler (one launch per
    exchange period for the whole band); returns (rows, band, sampler)."""
    from .sampler import BatchedSampler
    base, vs = build_variants(base_kw, variants)
    specs, meta = variant_specs(base, vs, positions, nrep, tmin, tmax)
    bs = BatchedSampler(specs, precision=precision, exchange_every=25, reanchor_every=1000)
    bs.init_state([v.prob.random_config(starts_seed + i) for i, (v, _) in enumerate(meta)],
                  [v.prob.cell.ideal for v, _ in meta])
    bs.run_blocks(blocks)
    common = vs[0].ft_data.window_mask(*vs[0].rwin)
    rows = [variant_result(bs, li, v, specs[li], common) for li, (v, _) in enumerate(meta)]
    return rows, band_from_variants(rows[:len(vs)], tol=tol), bs
