"""The swap surrogate's kernels and delayed acceptance on the device, checked
against the CPU oracle (oracle/mlp.py) and against the plain sampler."""
import numpy as np
import pytest

from cases import device_objects, oracle_problem, trace_inputs
from oracle import mlp as OM

pytestmark = pytest.mark.gpu


def _codes(rng, nsp, D, B):
    npt = nsp * (nsp - 1) // 2
    return np.concatenate([rng.integers(0, npt, (B, 1)), rng.integers(0, nsp + 1, (B, 2 * D))],
                          1).astype(np.uint8)


@pytest.mark.parametrize("nsp,D,H,nchain", [(2, 42, 256, 512), (3, 12, 64, 0)])
def test_predict_matches_oracle(cuda, nsp, D, H, nchain):
    """The per-CTA surrogate evaluation the sampler step runs equals the BF16
    oracle to FP32 summation order."""
    from chimera_b200.surrogate import SwapSurrogate
    rng = np.random.default_rng(1)
    sur = SwapSurrogate(nsp, D, H, nchain=nchain, seed=2)
    sur.host.feat_shift, sur.host.feat_scale = 0.3, 1.7
    sur.upload()
    B = 200
    codes, lnb = _codes(rng, nsp, D, B), rng.normal(0, 2, B).astype(np.float32)
    chain = rng.integers(0, nchain, B).astype(np.int32) if nchain else None
    y = sur.predict(codes, lnb, chain).cpu().numpy()
    want, _ = OM.forward(sur.theta.cpu().numpy(), codes, lnb, nsp, D, H, 0.3, 1.7,
                         chain=chain, nchain=nchain)
    scale = np.abs(want).max()
    assert np.abs(y - want).max() <= 1e-2 * scale
    assert np.median(np.abs(y - want)) <= 1e-4 * scale
    # bit-reproducible
    assert np.array_equal(y, sur.predict(codes, lnb, chain).cpu().numpy())


@pytest.mark.parametrize("nsp,D,H,B,nchain", [(2, 42, 256, 1024, 512), (3, 12, 64, 300, 0)])
def test_gradient_matches_oracle(cuda, nsp, D, H, B, nchain):
    """Training forward (tensor-core GEMMs), loss and every gradient block
    against the oracle's back-propagation with the same BF16 rounding points."""
    from chimera_b200.surrogate import SwapSurrogate
    rng = np.random.default_rng(3)
    sur = SwapSurrogate(nsp, D, H, nchain=nchain, seed=4)
    sur.host.feat_shift, sur.host.feat_scale = -0.2, 0.9
    sur.upload()
    codes, lnb = _codes(rng, nsp, D, B), rng.normal(0, 1, B).astype(np.float32)
    chain = np.sort(rng.integers(0, nchain, B)).astype(np.int32) if nchain else None
    t = rng.normal(0, 1, B).astype(np.float32)
    loss, y, g = sur.grad(codes, lnb, t, chain)
    theta = sur.theta.cpu().numpy()
    y_or, cache = OM.forward(theta, codes, lnb, nsp, D, H, -0.2, 0.9, chain=chain, nchain=nchain)
    loss_or, g_or = OM.backward(theta, cache, y_or, t.astype(np.float64), nsp, D, H)
    y = y.cpu().numpy()
    assert np.abs(y - y_or).max() <= 1e-2 * np.abs(y_or).max()
    assert abs(float(loss[0]) - loss_or) <= 1e-3 * loss_or
    yp = sur.predict(codes, lnb, chain).cpu().numpy()
    assert np.abs(y - yp).max() <= 1e-2 * np.abs(y_or).max()
    g = g.cpu().numpy()
    o = sur.offsets()
    bounds = [("W1", o["W1"], o["b1"]), ("b1", o["b1"], o["W2"]), ("W2", o["W2"], o["b2"]),
              ("b2", o["b2"], o["W3"]), ("W3", o["W3"], o["b3"]), ("b3", o["b3"], o["w4"]),
              ("w4", o["w4"], o["b4"]), ("b4", o["b4"], o["b4"] + 1)]
    for name, a, b in bounds:
        err = np.linalg.norm(g[a:b] - g_or[a:b]) / max(np.linalg.norm(g_or[a:b]), 1e-30)
        assert err <= 2e-2, (name, err)
    # reproducible bit for bit (fixed-order reductions, no atomics)
    _, _, g2 = sur.grad(codes, lnb, t, chain)
    assert np.array_equal(g, g2.cpu().numpy())


def test_adam_step_matches_formula(cuda):
    import torch
    from chimera_b200.surrogate import SwapSurrogate
    sur = SwapSurrogate(2, 4, 16, seed=5)
    rng = np.random.default_rng(6)
    th0 = sur.theta.cpu().numpy().astype(np.float64)
    m = np.zeros_like(th0)
    v = np.zeros_like(th0)
    for t in range(1, 4):
        g = rng.normal(0, 1, th0.size).astype(np.float32)
        sur.grad_buf.copy_(torch.from_numpy(g))
        sur.adam(lr=1e-2)
        m = 0.9 * m + 0.1 * g
        v = 0.999 * v + 0.001 * g.astype(np.float64) ** 2
        th0 = th0 - 1e-2 * (m / (1 - 0.9 ** t)) / (np.sqrt(v / (1 - 0.999 ** t)) + 1e-8)
    th = sur.theta.cpu().numpy()
    assert np.abs(th - th0).max() <= 1e-5
    b16 = sur.theta16.view(torch.bfloat16).float().cpu().numpy()
    assert np.array_equal(b16, OM.bf16(th))


def test_training_fits_a_site_additive_target(cuda):
    """Adam on the library's gradients learns a target that is a sum of
    per-site terms plus a beta term (the form of a first-order chi^2 change)."""
    from chimera_b200.surrogate import SwapSurrogate
    rng = np.random.default_rng(7)
    nsp, D, B = 2, 16, 20000
    codes = _codes(rng, nsp, D, B)
    lnb = rng.uniform(3, 9, B).astype(np.float32)
    c = rng.normal(0, 1, (2 * D + 1, nsp + 1))
    y = c[np.arange(2 * D + 1)[None, :], codes].sum(1) + 0.3 * lnb
    sur = SwapSurrogate(nsp, D, 128, seed=8)
    rep = sur.fit(codes, lnb, y.astype(np.float32), epochs=25, batch=1024, lr=2e-3)
    assert rep["loss"][-1] < 0.05 * rep["loss"][0]
    assert rep["rmse_d"] < 0.25 * rep["std_d"]


def test_zero_screen_reproduces_the_reference_sequence(cuda):
    """Delayed acceptance with the zero surrogate (d^ = 0, no prior) passes
    every swap to the exact stage, whose test is then the plain one: the
    FP64 run consumes the reference's streams and reproduces its accepted
    sequence and final state bit for bit."""
    from chimera_b200.surrogate import SwapSurrogate
    d = trace_inputs("rmc_trace.npz")
    assert int(d["energy"]) == 0
    smp, fm = device_objects(d, precision=0, reproduce=True)
    D = smp.lad.feature_table(0).shape[1]
    sur = SwapSurrogate(d["nsp"], D, 64)
    sur.init(zero=True)
    smp.lad.attach_surrogate(sur)
    smp.init_state(d["species0"], d["ideal"])
    acc = []
    for it in range(int(d["nsteps"])):
        acc.append(smp.step().cpu().numpy())
        if (it + 1) % 25 == 0:
            smp.replica_exchange()
    acc = np.array(acc)
    mism = np.argwhere(acc != d["accepted"])
    assert mism.size == 0, f"first mismatch at step/rung {mism[0]}"
    assert np.array_equal(smp.species.cpu().numpy(), d["final_species"])
    st = smp.lad.da_stats()[0]
    assert st[0] > 0 and st[1] == st[0] and 0 < st[2] <= d["accepted"].sum()
    assert smp.lad.device_error() == 0


def test_logged_swaps_match_the_oracle(cuda):
    """The step kernel's swap log (features, sigma * d, ln beta, chain, step)
    equals the oracle's restatement for every swap of an FP64 run on the
    reference's streams (energy prior and displacements on)."""
    from oracle.sampler import PlainSampler
    d = trace_inputs("rmc_trace_disp.npz")
    nsp, nrep = d["nsp"], int(d["nrep"])
    smp, fm = device_objects(d, precision=0, reproduce=True)
    lad = smp.lad
    nbr = lad.feature_table(0)
    nsteps = 60
    lad.enable_log(nsteps * nrep)
    prob = oracle_problem(d)
    ref = PlainSampler(prob, nrep, float(d["tmin"]), float(d["tmax"]), int(d["seed"]),
                       float(d["swap_frac"]), 0.012, 0.10)
    ref.init_state(d["species0"], d["ideal"])
    smp.init_state(d["species0"], d["ideal"])
    nlog = 0
    beta = 1.0 / np.geomspace(float(d["tmin"]), float(d["tmax"]), nrep)
    for s in range(1, nsteps + 1):
        slot_of = smp.b["slot_of"].cpu().numpy()
        ref.step()
        smp.step()
        L = ref.last
        codes = lad.bufs[0]["log_codes"].cpu().numpy()
        ylog = lad.bufs[0]["log_y"].cpu().numpy()
        for r in range(nrep):
            row = (s - 1) * nrep + slot_of[r]
            a, b = int(L["a"][r]), int(L["b"][r])
            sp = L["species"][r]
            if not L["swap"][r] or sp[a] == sp[b]:
                assert np.isnan(ylog[row, 0])
                continue
            want, sigma = OM.swap_codes(sp, a, b, nbr, nsp)
            assert np.array_equal(codes[row], want), (s, r)
            assert np.isclose(ylog[row, 0], sigma * L["d"][r], rtol=1e-6,
                              atol=1e-7 * abs(L["d"][r]) + 1e-30)
            assert np.isclose(ylog[row, 1], np.log(np.float32(beta[r])), rtol=1e-6)
            assert ylog[row, 2] == r and ylog[row, 3] == s
            nlog += 1
        if s % 25 == 0:
            ref.replica_exchange()
            smp.replica_exchange()
    assert nlog > nsteps * nrep // 3
    c, l, y = lad.swap_log()
    assert c.shape[0] == nlog
    assert lad.device_error() == 0


def _same_temperature_run(d, sur, nblocks, scale=None):
    smp, fm = device_objects(d, precision=1, reproduce=False)
    if sur is not None:
        sur.host.out_scale = scale
        sur.upload()
        smp.lad.attach_surrogate(sur)
    smp.init_state(d["species0"], d["ideal"])
    c2 = []
    for blk in range(nblocks):
        smp.steps(25)
        smp.lad.exchange_device()
        c2.append(smp.b["chi2"].cpu().numpy().copy())
    return smp, np.array(c2)


def test_delayed_acceptance_samples_the_plain_distribution(cuda):
    """With an untrained (random) surrogate as the screen, the chains still
    sample the target: at a temperature where the chains are stationary, the
    mean chi^2 of 64 independent same-temperature chains agrees with plain
    sampling within the statistical error, while the screen sent a large
    share of the moves back before the exact stage."""
    from chimera_b200.surrogate import SwapSurrogate
    d = trace_inputs("rmc_trace.npz")
    d["nrep"] = np.int64(64)
    d["tmin"] = d["tmax"] = np.float64(1e4)
    nblocks, burn = 400, 80
    smp0, plain = _same_temperature_run(d, None, nblocks)
    D = smp0.lad.feature_table(0).shape[1]
    sur = SwapSurrogate(d["nsp"], D, 64, seed=11)
    # screen errors of order one in the log acceptance
    smp1, da = _same_temperature_run(d, sur, nblocks, scale=float(d["tmin"]) / smp0.lad.nfit_of[0])
    st = smp1.lad.da_stats()[0]
    assert st[1] < 0.95 * st[0], st          # the screen did work
    a = plain[burn:].mean(0)
    b = da[burn:].mean(0)
    se = np.sqrt(a.var(ddof=1) / a.size + b.var(ddof=1) / b.size)
    assert abs(a.mean() - b.mean()) <= 5 * se, (a.mean(), b.mean(), se)
    assert smp1.lad.device_error() == 0


def test_bad_screen_falls_back_to_plain_steps(cuda):
    """A ladder whose screening error exceeds the threshold stops screening."""
    from chimera_b200.sampler import BatchedSampler
    from chimera_b200.surrogate import SwapSurrogate
    d = trace_inputs("rmc_trace.npz")
    smp, fm = device_objects(d, precision=1, reproduce=False)
    spec = smp.spec
    bs = BatchedSampler([spec, spec], precision=1, exchange_every=25, check_every=4,
                        reanchor_every=0)
    bs.init_state(d["species0"], d["ideal"])
    D = bs.lad.feature_table(0).shape[1]
    sur = SwapSurrogate(d["nsp"], D, 64, seed=3)
    sur.host.out_scale = 1e3
    sur.upload()
    bs.surrogate = sur
    bs.lad.attach_surrogate(sur, ladders=[0])
    bs.run_blocks(8)
    assert bs.fallbacks >= 1
    assert bs.lad.screening_on() == [False, False]
    assert bs.lad.device_error() == 0


def test_learned_screen_saves_exact_evaluations(cuda):
    """After learning from its own logged swaps (one input row per chain),
    the screen sends a third or more of the swaps of a warm ladder back
    before the exact path sum, transform and chi^2, with a screening error
    below the fallback threshold, so every ladder keeps screening."""
    from chimera_b200 import configs
    from chimera_b200.sampler import BatchedSampler, LadderSpec
    prob = configs.Problem(ncell=(10, 10, 10))
    specs = []
    for p in range(16):
        pos = prob.position(p)
        specs.append(LadderSpec(prob.fm, prob.ft, pos.target, pos.mask, pos.sigma_R, nrep=32,
                                tmin=0.05, tmax=0.5, seed=p, swap_frac=1.0, ms_library=prob.ms))
    bs = BatchedSampler(specs, precision=1, exchange_every=25, reanchor_every=0, check_every=10)
    bs.init_state([prob.random_config(p) for p in range(16)], prob.cell.ideal)
    bs.run_blocks(20)
    rep = bs.learn(blocks=40, epochs=8, H=64)
    assert rep["rmse_d"] < 0.7 * rep["std_d"], rep
    bs.run_blocks(20)
    st = bs.last_screen.sum(0)
    passed, err = st[1] / st[0], 1.0 - st[3] / st[1]
    print(f"pass {passed:.3f} screening error {err:.3f} fit {rep['rmse_d'] / rep['std_d']:.3f}")
    assert passed < 0.75 and err < bs.da_max_err
    assert all(bs.lad.screening_on()) and bs.fallbacks == 0
    assert bs.lad.device_error() == 0


def test_learn_on_mixed_lattices_and_species_counts(cuda):
    """A batch of fcc and bcc binaries and an fcc ternary learns one
    surrogate per (species count, feature width) class, each fitted on its
    own ladders' logged swaps, and every ladder then screens with the
    surrogate of its class: screened moves are counted on every ladder and
    the chains stay error-free."""
    from chimera_b200 import configs
    from chimera_b200.sampler import BatchedSampler, LadderSpec
    probs = [configs.Problem(ncell=(5, 5, 5)),
             configs.Problem(elements=("Fe", "Cr"), a0=2.87, lattice="bcc", ncell=(6, 6, 6)),
             configs.Problem(elements=("Fe", "Ni", "Cr"), composition=(0.4, 0.4, 0.2),
                             ncell=(5, 5, 5))]
    specs, starts = [], []
    for q, prob in enumerate(probs):
        for p in range(2):
            pos = prob.position(10 * q + p)
            specs.append(LadderSpec(prob.fm, prob.ft, pos.target, pos.mask, pos.sigma_R,
                                    nrep=16, tmin=0.05, tmax=0.5, seed=10 * q + p,
                                    swap_frac=1.0, ms_library=prob.ms))
            starts.append((prob.random_config(q + p), prob.cell.ideal))
    bs = BatchedSampler(specs, precision=1, exchange_every=25, reanchor_every=0,
                        check_every=10 ** 6)
    bs.init_state([s for s, _ in starts], [x for _, x in starts])
    bs.run_blocks(4)
    reps = bs.learn(blocks=8, epochs=2, H=64)
    assert isinstance(reps, list) and len(reps) == 3
    keys = sorted(bs.surrogates)
    assert [k[0] for k in keys] == [0, 0, 1]          # binaries: fcc and bcc widths; ternary
    widths = {bs.ladder(li)[0].host[bs.ladder(li)[1]].feat_D for li in range(6)}
    assert len(widths) == 2
    for (g, D), sur in bs.surrogates.items():
        assert sur.nsp == bs.groups[g].nsp and sur.D == D
    bs.run_blocks(10)
    bs._check_screen()                 # the first screening window after learning
    st = bs.last_screen
    assert (st[:, 0] > 0).all(), st
    assert (st[:, 1] <= st[:, 0]).all() and (st[:, 2] <= st[:, 1]).all()
    assert bs.device_error() == 0
