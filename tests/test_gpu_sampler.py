"""The fused device sampler step (A3-A8) against the reference's golden
traces and against full recomputes."""
import numpy as np
import pytest

from cases import device_objects, trace_inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["rmc_trace.npz", "rmc_trace_disp.npz", "rmc_trace_ms.npz"])
def test_fp64_reproduces_reference_accept_sequence(cuda, name):
    """FP64 acceptance fed the reference's RNG streams gives the reference's
    accepted-swap sequence, exchanges and final configuration."""
    d = trace_inputs(name)
    smp, fm = device_objects(d, precision=0, reproduce=True)
    smp.init_state(d["species0"], d["ideal"])
    acc, c2 = [], []
    for it in range(int(d["nsteps"])):
        acc.append(smp.step().cpu().numpy())
        c2.append(smp.chi2.cpu().numpy())
        if (it + 1) % 25 == 0:
            smp.replica_exchange()
    acc = np.array(acc)
    mism = np.argwhere(acc != d["accepted"])
    assert mism.size == 0, f"first mismatch at step/rung {mism[0]}"
    assert np.allclose(np.array(c2), d["chi2_log"], rtol=1e-9, atol=0)
    assert np.array_equal(smp.species.cpu().numpy(), d["final_species"])
    assert np.allclose(smp.pos.cpu().numpy(), d["final_pos"], rtol=0, atol=1e-13)
    assert np.allclose(smp.chi.cpu().numpy(), d["final_chi"], rtol=1e-9, atol=1e-11)
    assert smp.lad.device_error() == 0


def test_run_matches_reference_run_summary(cuda):
    d = trace_inputs("rmc_trace.npz")
    smp, fm = device_objects(d, precision=0, reproduce=True)
    smp.init_state(d["species0"], d["ideal"])
    smp.run(int(d["nsteps"]), exchange_every=25, log_every=10 ** 9)
    bsp, bpos, bc2 = smp.best()
    assert np.array_equal(bsp, d["best_species"])
    assert abs(bc2 - float(d["best_chi2"])) <= 1e-9 * abs(float(d["best_chi2"]))
    assert abs(smp.best_verified - float(d["best_verified"])) <= 1e-9 * abs(float(d["best_verified"]))
    assert np.allclose(smp.exchange_rate, d["exchange_rate"], equal_nan=True)


@pytest.mark.parametrize("name", ["rmc_trace.npz", "rmc_trace_disp.npz", "rmc_trace_ms.npz"])
def test_fp32c_tracks_full_recompute(cuda, name):
    """FP32C (tabulated ideal shells, FP32 transforms): after a device-only run
    the running chi equals an FP64 recompute of the state to 1e-6 (per absorber),
    the composition is conserved and the best state verifies."""
    torch = cuda
    d = trace_inputs(name)
    smp, fm = device_objects(d, precision=1, reproduce=False)
    smp.init_state(d["species0"], d["ideal"])
    smp.run(300, exchange_every=25, log_every=10 ** 9)
    lad, b = smp.lad, smp.b
    chi = b["chi"].cpu().numpy()
    full = fm.chi_full(b["pos"], b["species"]).cpu().numpy()
    if smp.ms is not None:
        full = full + smp.ms.chi_of(b["ms_C"]).cpu().numpy()
        assert np.array_equal(b["ms_C"].cpu().numpy(), smp.ms.counts(b["species"]).cpu().numpy())
    cnt = b["count"].cpu().numpy()[:, :, None]
    assert np.abs(chi / cnt - full / cnt).max() <= 1e-6
    sp = b["species"].cpu().numpy()
    assert (np.bincount(sp[0], minlength=2) == np.bincount(d["species0"], minlength=2)).all()
    assert all((np.sort(s) == np.sort(d["species0"])).all() for s in sp)
    assert abs(smp.best_verified - smp.best()[2]) <= 1e-3 * abs(smp.best()[2])
    assert lad.device_error() == 0


def test_reanchor_kernel_equals_fp64_recompute(cuda):
    """The pair-count FP64 re-anchoring of chx_reanchor gives the state's FP64
    path sum (ideal pairs via the shell table, displaced pairs directly, exact
    MS counts) to rounding, on the slots it is asked to recompute only."""
    torch = cuda
    d = trace_inputs("rmc_trace_ms.npz")
    d["swap_frac"] = np.float64(0.7)            # make displaced atoms appear
    smp, fm = device_objects(d, precision=1, reproduce=False)
    smp.init_state(d["species0"], d["ideal"])
    smp.run(200, exchange_every=25, log_every=10 ** 9)
    lad, b = smp.lad, smp.b
    assert int(b["moved"].sum()) > 0
    before = b["chi"].clone()
    mask = np.zeros(lad.nslots, bool)
    mask[::2] = True
    lad.reanchor(mask)
    after = b["chi"].cpu().numpy()
    full = fm.chi_full(b["pos"], b["species"]).cpu().numpy() + smp.ms.chi_of(b["ms_C"]).cpu().numpy()
    scale = np.abs(full).max()
    assert np.abs(after[mask] - full[mask]).max() <= 1e-12 * scale
    assert np.array_equal(after[~mask], before.cpu().numpy()[~mask])
    assert (b["n_acc"].cpu().numpy()[mask] == 0).all()
    assert lad.device_error() == 0


def test_uneven_batch_equals_separate_runs(cuda):
    """Ladders of different supercells (108, 256, 500 and 864 sites, each
    with its own exact MS templates and targets) run in one launch per step
    give, bit for bit, what each ladder gives in a batch of its own: the
    shared launch plan (largest extents) changes no arithmetic."""
    from chimera_b200 import configs
    from chimera_b200.sampler import BatchedSampler, LadderSpec
    specs, init = [], []
    for n in (3, 4, 5, 6):
        prob = configs.Problem(ncell=(n, n, n), ms=n >= 4)
        pos = prob.position(n)
        specs.append(LadderSpec(prob.fm, prob.ft, pos.target, pos.mask, pos.sigma_R,
                                nrep=4 + n, tmin=1e-3, tmax=1e-1, seed=n, swap_frac=0.9,
                                ms_library=prob.ms))
        init.append((prob.random_config(n), prob.cell.ideal))

    def run(sp):
        bs = BatchedSampler(sp, precision=1, exchange_every=25, reanchor_every=0)
        idx = [specs.index(x) for x in sp]
        bs.init_state([init[i][0] for i in idx], [init[i][1] for i in idx])
        bs.run_blocks(6)
        assert bs.lad.device_error() == 0
        return [{k: b[k].cpu().numpy().copy() for k in ("species", "pos", "chi", "chi2",
                                                        "rung_of", "best_chi2")}
                for b in bs.lad.bufs]

    together = run(specs)
    for i, s in enumerate(specs):
        alone = run([s])[0]
        for k, v in alone.items():
            assert np.array_equal(together[i][k], v), (i, k)


def test_mixed_species_counts_equal_separate_runs(cuda):
    """A batch of binary and ternary ladders (two step kernels, one per
    species count, on parallel streams inside one graph) gives, bit for bit,
    what each ladder gives alone."""
    from chimera_b200 import configs
    from chimera_b200.sampler import BatchedSampler, LadderSpec
    specs, init = [], []
    for q, (els, comp, n) in enumerate(((("Fe", "Ni"), (0.5, 0.5), 4),
                                        (("Fe", "Ni", "Cr"), (0.4, 0.4, 0.2), 4),
                                        (("Fe", "Ni"), (0.5, 0.5), 5),
                                        (("Fe", "Ni", "Cr"), (0.4, 0.4, 0.2), 5))):
        prob = configs.Problem(elements=els, composition=comp, ncell=(n, n, n))
        pos = prob.position(q)
        specs.append(LadderSpec(prob.fm, prob.ft, pos.target, pos.mask, pos.sigma_R,
                                nrep=6 + q, tmin=1e-3, tmax=1e-1, seed=q, swap_frac=1.0,
                                ms_library=prob.ms))
        init.append((prob.random_config(q), prob.cell.ideal))

    def run(sp):
        bs = BatchedSampler(sp, precision=1, exchange_every=25, reanchor_every=0)
        idx = [specs.index(x) for x in sp]
        bs.init_state([init[i][0] for i in idx], [init[i][1] for i in idx])
        bs.run_blocks(6)
        assert bs.device_error() == 0
        out = []
        for li in range(bs.nladders):
            lad, q = bs.ladder(li)
            b = lad.bufs[q]
            out.append({k: b[k].cpu().numpy().copy() for k in ("species", "chi", "chi2",
                                                               "rung_of", "best_chi2")})
        return bs, out

    bs, together = run(specs)
    assert len(bs.groups) == 2 and [g.nsp for g in bs.groups] == [2, 3]
    assert [bs.where[i] for i in range(4)] == [(0, 0), (1, 0), (0, 1), (1, 1)]
    for i, s in enumerate(specs):
        _, alone = run([s])
        for k, v in alone[0].items():
            assert np.array_equal(together[i][k], v), (i, k)


def test_hcp_exact_ms_tracks_recount(cuda):
    """hcp with exact MS (classes in hexagonal coordinates, B sites reading
    the inverted template offsets): after FP32C batched steps each slot's
    running MS entry counts equal a recount of its state, and its running
    chi equals the FP64 recompute to 1e-6 per absorber."""
    from chimera_b200 import configs
    from chimera_b200.sampler import BatchedSampler, LadderSpec
    prob = configs.Problem(elements=("Co", "Ni"), a0=2.507, lattice="hcp", ncell=(8, 8, 6),
                           alpha1=-0.05)
    assert prob.paths is not None and prob.paths.hex
    pos = prob.position(0)
    spec = LadderSpec(prob.fm, prob.ft, pos.target, pos.mask, pos.sigma_R, nrep=16, tmin=1e-3,
                      tmax=1e-1, seed=1, swap_frac=1.0, ms_library=prob.ms)
    bs = BatchedSampler([spec], precision=1, exchange_every=25, reanchor_every=0)
    bs.init_state([prob.random_config(1)], [prob.cell.ideal])
    bs.run_blocks(8)
    assert bs.device_error() == 0
    b = bs.lad.bufs[0]
    assert int(b["n_acc"].sum()) > 50
    assert np.array_equal(b["ms_C"].cpu().numpy(), prob.ms.counts(b["species"]).cpu().numpy())
    full = (prob.fm.chi_full(b["pos"], b["species"]) + prob.ms.chi_of(b["ms_C"])).cpu().numpy()
    cnt = b["count"].cpu().numpy()[:, :, None]
    assert np.abs(b["chi"].cpu().numpy() / cnt - full / cnt).max() <= 1e-6


@pytest.mark.parametrize("els,comp", [(("Fe", "Ni"), (0.5, 0.5)),
                                      (("Fe", "Ni", "Cr"), (0.4, 0.4, 0.2))])
def test_fp32_transform_chi2_matches_fp64(cuda, els, comp):
    """The FP32C step's fit-window transform and chi^2 (FP32 taps and
    twiddles, FP64 sums of the chi^2 terms) agree with the FP64 path on the
    same states to 2e-5 relative: 16 random configurations of a 4x4x4 cell
    with exact MS, binary and ternary."""
    from chimera_b200 import configs
    from chimera_b200.sampler import BatchedSampler, LadderSpec
    prob = configs.Problem(elements=els, composition=comp, ncell=(4, 4, 4))
    pos = prob.position(3)
    spec = LadderSpec(prob.fm, prob.ft, pos.target, pos.mask, pos.sigma_R, nrep=16, tmin=1e-3,
                      tmax=1e-1, seed=2, swap_frac=1.0, ms_library=prob.ms)
    out = []
    for prec in (0, 1):
        bs = BatchedSampler([spec], precision=prec, exchange_every=25, reanchor_every=0)
        bs.init_state([prob.random_config(5)], [prob.cell.ideal])
        b = bs.lad.bufs[0]
        for r in range(16):          # a different configuration in every slot
            b["species"][r].copy_(torch_from(prob.random_config(100 + r)))
        chi = prob.fm.chi_full(b["pos"], b["species"]) + prob.ms.full(b["species"])
        b["chi"].copy_(chi)
        bs.lad.refresh_chi2()
        out.append(b["chi2"].cpu().numpy().copy())
        assert bs.device_error() == 0
    rel = np.abs(out[1] - out[0]) / np.abs(out[0])
    assert np.ptp(out[0]) > 0
    assert rel.max() <= 2e-5, rel.max()


def torch_from(a):
    import torch
    return torch.as_tensor(np.asarray(a, np.int32), device="cuda")


def test_best_state_is_the_state_of_the_best_chi2(cuda):
    """The best state is written once per launch (or when its log of later
    moves fills up) as the current state with the moves after the best
    undone. After single launches of 250 FP64 steps with displacements on,
    enough for that log to fill, every slot's best species and positions
    give back its best chi^2 exactly."""
    import torch
    d = trace_inputs("rmc_trace.npz")
    d["swap_frac"] = np.float64(0.5)
    d["tmin"], d["tmax"] = np.float64(1e2), np.float64(1e4)
    smp, fm = device_objects(d, precision=0, reproduce=False)
    smp.init_state(d["species0"], d["ideal"])
    lad, b = smp.lad, smp.b
    most = 0
    for _ in range(3):
        flags = smp.steps(250)
        most = max(most, int(flags.sum(0).max()))
    assert most >= 40          # some rung accepted more moves than the log holds
    assert int(b["moved"].sum()) > 0
    bsp, bpos = b["best_sp"], b["best_pos"]
    chi = fm.chi_full(bpos, bsp)
    cnt = torch.stack([(bsp == s).sum(1) for s in range(d["nsp"])], 1).double()
    c2 = lad.eval_chi2(chi.contiguous(), cnt.contiguous()).cpu().numpy()
    best = b["best_chi2"].cpu().numpy()
    assert np.allclose(c2, best, rtol=1e-10, atol=0), (c2, best)
    assert (best <= b["chi2"].cpu().numpy() + 1e-12).all()
    assert lad.device_error() == 0


def test_systematic_band_variants_in_one_launch_equal_separate_runs(cuda):
    """Six calibration variants (baseline; a0 +0.005 A with its own
    supercell; dE0 +2 eV on the model's k axis; k weight 2 alone; R max
    -0.4; MS amplitude x1.15) as ladders of one batched sampler give, bit for
    bit, what each gives alone; the band reduction then leaves out the k-weight
    variant as not comparable."""
    from chimera_b200 import band as B
    from chimera_b200.sampler import BatchedSampler
    pick = ["baseline", "a0 +0.005 A", "dE0 +2 eV", "k weight 2", "R max -0.4", "ms_amp x1.15"]
    variants = [v for v in B.CALIB_VARIANTS if v[0] in pick]
    base, vs = B.build_variants(dict(ncell=(4, 4, 4)), variants)
    specs, meta = B.variant_specs(base, vs, positions=(0,), nrep=8)
    assert vs[1].prob is not base and vs[2].prob is base
    assert not np.allclose(vs[2].ft.fts[0].k_model, base.k)
    assert specs[3].target.shape[0] == base.nsp                 # one k weight
    assert specs[4].mask.sum() < specs[0].mask.sum()
    starts = [v.prob.random_config(7 + i) for i, (v, _) in enumerate(meta)]
    ideal = [v.prob.cell.ideal for v, _ in meta]

    def run(idx):
        bs = BatchedSampler([specs[i] for i in idx], precision=1, exchange_every=25,
                            reanchor_every=0)
        bs.init_state([starts[i] for i in idx], [ideal[i] for i in idx])
        bs.run_blocks(6)
        assert bs.device_error() == 0
        return bs, [{k: b[k].cpu().numpy().copy() for k in ("species", "chi2", "best_chi2")}
                    for b in bs.lad.bufs]

    bs, together = run(range(len(specs)))
    for i in range(len(specs)):
        _, alone = run([i])
        for k, v in alone[0].items():
            assert np.array_equal(together[i][k], v), (pick[i], k)
    common = vs[0].ft_data.window_mask(*vs[0].rwin)
    rows = [B.variant_result(bs, li, v, specs[li], common) for li, (v, _) in enumerate(meta)]
    band = B.band_from_variants(rows)
    assert band["excluded_incomparable"] == ["k weight 2"]
    assert all(np.isfinite(r["r_factor"]) and len(r["wc"]) == 3 for r in rows)


def test_device_reanchoring_equals_host_reanchoring(cuda):
    """Re-anchoring decided on the device inside each exchange period's graph
    (chx_reanchor_due, its per-period cap at the slot count) re-anchors exactly
    the slots the host-side check finds due after the same period, so the
    chains are identical bit for bit; the device counter counts the
    re-anchored slots."""
    from chimera_b200 import configs
    from chimera_b200.sampler import BatchedSampler, LadderSpec
    prob = configs.Problem(ncell=(5, 5, 5), ms=True)
    specs = []
    for p in range(2):
        pos = prob.position(p)
        specs.append(LadderSpec(prob.fm, prob.ft, pos.target, pos.mask, pos.sigma_R, nrep=8,
                                tmin=1e-3, tmax=1e-1, seed=p, swap_frac=0.98,
                                ms_library=prob.ms))
    init = [prob.random_config(40 + p) for p in range(2)]
    out = []
    for dev in (True, False):
        bs = BatchedSampler(specs, precision=1, exchange_every=25, reanchor_every=6,
                            check_every=1, device_reanchor=dev, reanchor_cap=16)
        bs.init_state(init, prob.cell.ideal)
        bs.run_blocks(10)
        assert bs.lad.device_error() == 0
        keys = ("species", "chi", "chi2", "n_acc", "best_chi2", "rung_of")
        out.append(({(li, k): bb[k].cpu().numpy().copy() for li, bb in enumerate(bs.lad.bufs)
                     for k in keys}, bs))
    (a, bs_dev), (b, bs_host) = out
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert bs_dev.reanchors > 0 and bs_host.host_reanchors > 0


def test_posterior_warren_cowley_matches_lattice_definition(cuda):
    """Posterior samples reduced on the device (chx_pair_counts over the first
    shell) give the Warren-Cowley vector of lattice.warren_cowley (the
    reference's definition, exafs_gpu/lattice.py:167-185) for the sampled
    rungs' configurations."""
    from chimera_b200 import configs
    from chimera_b200 import lattice as L
    from chimera_b200.sampler import BatchedSampler, LadderSpec
    prob = configs.Problem(elements=("Fe", "Ni", "Cr"), composition=(0.4, 0.4, 0.2),
                           ncell=(4, 4, 4), ms=False)
    pos = prob.position(0)
    spec = LadderSpec(prob.fm, prob.ft, pos.target, pos.mask, pos.sigma_R, nrep=8, tmin=1e-3,
                      tmax=1e-1, seed=3, swap_frac=1.0)
    bs = BatchedSampler([spec], precision=1, exchange_every=25, reanchor_every=0)
    bs.init_state([prob.random_config(5)], prob.cell.ideal)
    bs.enable_collect(from_block=10 ** 9)            # manual collection only
    want = []
    for blocks in (0, 3, 4):
        bs.run_blocks(blocks) if blocks else None
        bs.collect()
        b = bs.lad.bufs[0]
        rungs = b["_collect_rungs"].cpu().numpy()
        slots = b["slot_of"].cpu().numpy()[rungs]
        for sp in b["species"].cpu().numpy()[slots]:
            a = L.warren_cowley(sp, prob.top.i, prob.top.j, prob.top.shift, prob.cell,
                                float(prob.top.r_shell[0]), nsp=3)
            want.append(a[np.triu_indices(3)])
    want = np.array(want)
    mean, sd, n = bs.posterior_wc(0)
    assert n == len(want) == 12
    np.testing.assert_allclose(mean, want.mean(0), rtol=0, atol=1e-12)
    np.testing.assert_allclose(sd, want.std(0), rtol=0, atol=1e-12)
    assert bs.lad.device_error() == 0


@pytest.mark.parametrize("name", ["rmc_trace.npz", "rmc_trace_disp.npz", "rmc_trace_ms.npz"])
def test_fp32c_decisions_shadow_fp64_over_1000_steps(cuda, name):
    """Decision agreement of FP32C with FP64 on the same states: an FP64
    chain runs 1,000 steps on the reference's streams; before each of its
    steps an FP32C sampler takes its exact state (species, positions, FP64
    chi and chi^2, MS counts, rung maps; its FP64 chi(R) from a refresh) and
    step counter, and makes the same proposal. Every (step, rung) decision
    is compared. FP32C evaluates a move with FP32 terms and an FP32
    transform of the change, re-deciding near ties with FP64 transforms;
    the measured disagreement stays below one decision in 1,000."""
    torch = cuda
    d = trace_inputs(name)
    s64, fm = device_objects(d, precision=0, reproduce=True)
    s32, _ = device_objects(d, precision=1, reproduce=True)
    s64.init_state(d["species0"], d["ideal"])
    s32.init_state(d["species0"], d["ideal"])
    keys = ("species", "pos", "moved", "chi", "chi2", "ms_C", "rung_of", "slot_of", "count")
    diff, total = [], 0
    for it in range(1000):
        for k in keys:
            s32.b[k].copy_(s64.b[k])
        s32.lad.refresh_chi2()                  # chi^2 and chi(R) of that state in FP64
        assert torch.allclose(s32.b["chi2"], s64.b["chi2"], rtol=1e-12, atol=0)
        s32.lad.stepc.copy_(s64.lad.stepc)
        s32._stepc = s64._stepc
        a32 = s32.step().cpu().numpy()
        a64 = s64.step().cpu().numpy()
        total += a64.size
        diff += [(it, r) for r in np.nonzero(a32 != a64)[0]]
        if (it + 1) % 25 == 0:
            s64.replica_exchange()
    assert s64.lad.device_error() == 0 and s32.lad.device_error() == 0
    ties = s32.lad.tie_stats().sum(0)
    rate = len(diff) / total
    print(f"{name}: {len(diff)} of {total} decisions differ ({rate:.2e}); "
          f"{ties[0]:.0f} near-tie FP64 re-checks, {ties[1]:.0f} decisions changed by them")
    assert rate <= 1e-3, (diff[:5], ties)
