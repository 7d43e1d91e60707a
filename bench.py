"""Benchmark of the batched PT-RMC hot path on one node.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the batched plain-sampler configuration): fcc Fe50Ni50, 10x10x10
conventional cells (4,000 atoms), a0 = 3.59 A, single scattering to 5.0 A (42
neighbours), exact 3-/4-leg multiple scattering to 5.5 A (25 classes, 3,204
paths per site), 2 K edges, 241 k points, k^1/k^2/k^3 Kaiser-windowed complex
chi(R) fitted on 1.4-5.0 A; 16 sample positions (seeded noise) x 32 PT rungs =
512 replicas per GPU, advanced together, FP32 transcendentals with FP64 phase
reduction and accumulation, FP64 re-anchoring every 1,000 accepted moves.

One bench "step" is one exchange period: 25 sampler steps of every replica
(one persistent fused launch), one device replica exchange and the FP64
re-anchoring of the slots that reached 1,000 accepted moves, replayed as a
CUDA graph. The chains are aged by an untimed burn-in (--burnin) first. value = swap attempts per second over all ranks. With --gpus N every
rank runs its own 16 ladders (weak scaling, no collective in the timed loop).

--impl reference times the CPU restatement of the reference sampler (oracle/,
the reference itself is CuPy and cannot run here) on the host cores, one
process per ladder.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PT-RMC GPU-s to plain's R-factor: learned+batched vs plain GPU; chi err vs FP64"
UNIT = "swap attempts/s"
NPOS, NREP, EXCH = 16, 32, 25      # positions (ladders) per GPU, rungs, steps per block


def workload_config():
    return {"workload": "batched plain PT-RMC, fcc Fe50Ni50 4000 atoms (10x10x10, a0 3.59 A), "
                        "SS to 5.0 A + exact 3/4-leg MS to 5.5 A, 2 edges, 241 k, "
                        "k^1/k^2/k^3 Kaiser complex chi(R) 1.4-5.0 A",
            "positions": NPOS, "rungs": NREP, "replicas_per_gpu": NPOS * NREP,
            "steps_per_bench_step": EXCH, "precision": "FP32 terms/transform, FP64 phase+accum",
            "l2": "flushed between timed periods (256 MB write outside each period's "
                  "CUDA events)"}


def build_problem():
    from chimera_b200.configs import Problem
    return Problem(ncell=(10, 10, 10), rmax=5.0, ms=True)


def make_sampler(prob, rank=0):
    from chimera_b200.sampler import BatchedSampler, LadderSpec
    specs = []
    for p in range(NPOS):
        pos = prob.position(rank * NPOS + p)
        specs.append(LadderSpec(prob.fm, prob.ft, pos.target, pos.mask, pos.sigma_R, nrep=NREP,
                                tmin=1e-4, tmax=1e-1, seed=1000 * rank + p, swap_frac=1.0,
                                disp_sigma=0.012, max_disp=0.10, ms_library=prob.ms))
    return BatchedSampler(specs, precision=1, exchange_every=EXCH, reanchor_every=1000)


class Clocks:
    """nvidia-smi samples while the timed region runs."""

    def __init__(self, index=0):
        self.index = index
        self.lines = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def step_bytes(prob):
    """Algorithmic bytes of one swap attempt in the reference's own int32
    layout: for both sites, the z pair ids (4 B) and neighbour species (1 B),
    and the M incident MS paths (4 B path id, 4 B absorber/class, 12 B slot
    ids, 4 B species); the delta chi is fused into the transform, so it is not
    written back. The kernel reads far less (the MS paths come from shared
    templates and the species from shared memory): see `traffic`."""
    z = prob.top.ncoord
    M = prob.paths.M if prob.paths is not None else 0
    return 2 * z * (4 + 1) + 2 * M * 24


def time_graph(fn, reps):
    import torch
    s = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    for _ in range(reps):
        fn()
    b.record(s)
    b.synchronize()
    return a.elapsed_time(b) / 1e3


def oracle_problem(prob, p):
    """The oracle's problem for sample position p, built on the host only:
    the target comes from the oracle's own path sum, MS counts and FFT."""
    from oracle import kernels as K
    from oracle import sampler as OS
    chans = [OS.Channel(f._idx, f._frac, f._inside, f._w, f.nfft, f._norm,
                        int(prob.ft.chan_edge[c])) for c, f in enumerate(prob.ft.fts)]
    msd = None
    if prob.paths is not None:
        P = prob.paths
        msd = dict(p_abs=P.p_abs, p_cls=P.p_cls, p_slot=P.p_slot, inc=P.inc, cls_off=P.cls_off,
                   nblk=P.nblk, T=prob.ms_table)
    nchan = len(chans)
    pr = OS.Problem(prob.cell.ideal, prob.top.i, prob.top.j, prob.top.shift, prob.top.shell,
                    prob.top.sigma2, prob.k, prob.tables.f, prob.tables.delta, prob.tables.lam,
                    prob.tables.s02, chans, np.zeros((nchan, 1024), complex), prob.mask,
                    prob.sigma_R(), prob.nsp, ms=msd)
    sp = prob.target_species[None]
    chi, _, _ = pr.chi_full(prob.cell.ideal[None], sp)
    if msd is not None:
        chi = chi + pr.ms_chi(pr.ms_counts(sp))
    cnt = np.bincount(prob.target_species, minlength=prob.nsp).astype(float)
    chi = chi[0] / np.maximum(cnt, 1)[:, None] + prob.noise_k(p)
    target = pr.observe(chi[None])[0]
    pr.target, pr.tm = target, np.ascontiguousarray(target[:, prob.mask])
    del K
    return pr


def cpu_baseline(prob, nsteps=40, nrep=NREP, p=0):
    """The oracle's plain sampler on one ladder of this workload, one core."""
    from oracle import sampler as OS
    pr = oracle_problem(prob, p)
    smp = OS.PlainSampler(pr, nrep, 1e-4, 1e-1, p, 1.0, 0.012, 0.10)
    smp.init_state(prob.random_config(p), prob.cell.ideal)
    smp.step()
    t0 = time.perf_counter()
    for it in range(nsteps):
        smp.step()
        if (it + 1) % EXCH == 0:
            smp.replica_exchange()
    dt = time.perf_counter() - t0
    return {"value": nsteps * nrep / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"oracle plain sampler (C kernels + NumPy FFT), one ladder of {nrep} "
                      f"replicas on the 4,000-atom workload, {nsteps} steps after 1 warm-up"}


def run_reference(args):
    """--impl reference: the CPU restatement of the reference sampler, one
    process per ladder on the host cores. A bench step is one exchange period
    (25 sampler steps of every rung, then the exchange) when the whole
    --warmup W --steps K run fits in about two minutes of host time, else a
    bounded sample of fewer sampler steps per bench step; the rate (swap
    attempts per second) is what is compared."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import multiprocessing as mp
    ncores = os.cpu_count() or 1
    nproc = max(1, min(NPOS, ncores))
    W, K = max(0, args.warmup), max(1, args.steps)
    per_step = max(1, min(EXCH, int(120.0 / (0.065 * (W + K)))))   # ~65 ms per sampler step
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(nproc) as pool:
        res = pool.map(_ref_worker, [(p, W, K, per_step) for p in range(nproc)])
    wall = time.perf_counter() - t0
    attempts = sum(r["attempts"] for r in res)
    busy = max(r["seconds"] for r in res)
    val = attempts / busy
    sample = (f"{nproc} ladders x {NREP} replicas, {per_step} sampler steps per bench step "
              f"({'one exchange period' if per_step == EXCH else 'bounded sample'}), {W} "
              f"untimed + {K} timed bench steps, one process per ladder (oracle C kernels + "
              f"NumPy FFT)")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": 0,
            "steps": K, "warmup": W, "ms_per_step": busy / K * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(),
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": nproc, "kind": "port",
                             "sample": sample},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line), flush=True)
    return 0


def _ref_worker(arg):
    p, W, K, per_step = arg
    sys.path.insert(0, ROOT)
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    from oracle import sampler as OS
    prob = build_problem()
    pr = oracle_problem(prob, p)
    smp = OS.PlainSampler(pr, NREP, 1e-4, 1e-1, p, 1.0, 0.012, 0.10)
    smp.init_state(prob.random_config(p), prob.cell.ideal)

    def bench_step():
        for _ in range(per_step):
            smp.step()
        smp.replica_exchange()

    for _ in range(W):
        bench_step()
    t0 = time.perf_counter()
    for _ in range(K):
        bench_step()
    dt = time.perf_counter() - t0
    return {"attempts": K * per_step * NREP, "seconds": dt}


def bench_ft(args):
    """The windowed FT contraction of the series configuration: 4,096 seeded
    chi(k) on 241 k points, values N(0, 0.05) shaped by exp(-0.01 k^2)
    sin(2k 2.5), each at k^1, k^2 and k^3 (one basis per weight, Kaiser
    window dk = 1, k 3-13), onto complex chi(R) at R 0-6 A (200 bins of
    0.0307 A). Per precision (0 FP64 SIMT, 1 FP32 SIMT, 2 split-BF16 tcgen05,
    3 TF32 tcgen05): device time of the three calls (inputs resident, L2
    flushed with a 256 MB write before each call), and the error against
    FP64: max and rms of Re and Im chi(R) relative to max |chi(R)|, and the
    R-factor sum|z - z64|^2 / sum|z64|^2 per spectrum (max and mean). The
    three weights share chi, so one call contracts it with their bases side
    by side (1,200 real columns)."""
    import torch
    from chimera_b200 import _native as N
    from chimera_b200.fourier import FourierTransform
    from chimera_b200.tables import uniform_k
    N.lib()
    k = uniform_k()
    nspec, nk = 4096, k.size
    bins = np.arange(200)
    rng = np.random.default_rng(0)
    chi = rng.normal(0, 0.05, (nspec, nk)) * (np.exp(-0.01 * k * k) * np.sin(2 * k * 2.5))[None]
    x = torch.from_numpy(chi).cuda()
    # the three k weights share chi: one contraction against their bases side by side
    Bs = [FourierTransform(k, 3.0, 13.0, w, window="kaiser").basis(bins) for w in (1, 2, 3)]
    Bc = np.concatenate(Bs, axis=1)                                    # (nk, 3 nR)
    basis = torch.from_numpy(np.ascontiguousarray(
        np.stack([Bc.real, Bc.imag], -1).reshape(nk, -1))).cuda()
    nR = 3 * bins.size
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream()
    res, ref = {}, None
    for prec in (0, 1, 2, 3):
        out = torch.empty((nspec, 2 * nR), dtype=torch.float64, device="cuda")
        nsc = int(N.lib().chx_ft_batch_scratch_bytes(nspec, nk, nR, prec))
        scr = torch.empty(max(nsc, 1), dtype=torch.uint8, device="cuda")

        def call():
            N.call("chx_ft_batch", N.ptr(x), nspec, nk, N.ptr(basis), nR, prec, N.ptr(out),
                   N.ptr(scr), nsc, N.stream())
        for _ in range(max(3, args.warmup)):
            call()
        ts = []
        for _ in range(max(5, min(args.steps, 30))):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            call()
            b.record(s)
            b.synchronize()
            ts.append(a.elapsed_time(b) * 1e-3)
        if prec in (2, 3):
            assert int(scr[:4].view(torch.int32).item()) == 0, "device error word set"
        z = out.view(nspec, 3, nR // 3, 2).transpose(0, 1)              # (3, nspec, nR, 2)
        if ref is None:
            ref = z.clone()
        scale = float(ref.abs().max())
        dz = z - ref
        rf = (dz ** 2).sum((2, 3)) / (ref ** 2).sum((2, 3)).clamp_min(1e-300)
        t = float(np.median(ts))
        byts = (nspec * nk + nk * 2 * nR + nspec * 2 * nR) * 8
        res[str(prec)] = {
            "us": t * 1e6, "GB_per_s": byts / t / 1e9,
            "useful_TFLOP_per_s": 2.0 * nspec * nk * 2 * nR / t / 1e12,
            "max_err_re": float(dz[..., 0].abs().max()) / scale,
            "max_err_im": float(dz[..., 1].abs().max()) / scale,
            "rms_err_re": float(dz[..., 0].pow(2).mean().sqrt()) / scale,
            "rms_err_im": float(dz[..., 1].pow(2).mean().sqrt()) / scale,
            "rfactor_max": float(rf.max()), "rfactor_mean": float(rf.mean())}
    # the fused form (chx_ft_window_sums): the same contraction, its epilogue
    # summing each spectrum against a target over the fit window (1.4-5.0 A)
    # instead of writing chi(R); the three weights are the channels of one
    # edge, so the sums over all 600 bins are the edge's sums; anchored at
    # s0 = 1 (the targets are near scale 1)
    from chimera_b200.fourier import WindowSums, FourierTransform as _FT
    z64 = ref.transpose(0, 1).reshape(nspec, nR, 2)
    zc = torch.complex(z64[..., 0], z64[..., 1])                      # FP64 chi(R)
    Rg = _FT(k, 3.0, 13.0, 1).R[bins]
    win = np.tile((Rg >= 1.4) & (Rg <= 5.0), 3)
    tgt = zc[0].cpu().numpy() * 1.05 + rng.normal(0, 1e-3, nR) * (1 + 1j)
    wgt = np.where(win, 1.0 / 2e-3 ** 2, 0.0)
    tg = torch.from_numpy(tgt).cuda()
    wg = torch.from_numpy(wgt).cuda()
    wn = torch.from_numpy(win).cuda()
    T0 = float((tg.abs() ** 2 * wn).sum())
    sc64 = (zc * tg.conj()).real.mul(wn).sum(1) / (zc.abs() ** 2 * wn).sum(1)
    c64 = ((sc64[:, None] * zc - tg).abs() ** 2 * wg).sum(1)
    r64 = ((sc64[:, None] * zc - tg).abs() ** 2 * wn).sum(1) / T0
    for prec in (2, 3):
        ws = WindowSums(Bc, tgt, wgt, nspec, prec, s0=1.0, Bd=basis)
        for _ in range(max(3, args.warmup)):
            ws(x)
        ts = []
        for _ in range(max(5, min(args.steps, 30))):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            o5 = ws(x)
            b.record(s)
            b.synchronize()
            ts.append(a.elapsed_time(b) * 1e-3)
        assert ws.device_error() == 0, "device error word set"
        sc, c, rn = WindowSums.chi2(o5, 1.0)
        r = rn / T0              # the R-factor from the same sums (model.py:535-540)
        t = float(np.median(ts))
        byts = (nspec * nk + nk * 2 * nR + nspec * 7) * 8
        res[f"fused_{prec}"] = {
            "us": t * 1e6, "GB_per_s": byts / t / 1e9,
            "useful_TFLOP_per_s": 2.0 * nspec * nk * 2 * nR / t / 1e12,
            "chi2_rel_err_max": float(((c - c64).abs() / c64.abs()).max()),
            "rfactor_rel_err_max": float(((r - r64).abs() / r64.abs()).max()),
            "bytes_out_per_spectrum": 56}
    hbm, src = peaks()
    tc = res["2"]
    line = {"metric": "windowed FT contraction chi(k) -> chi(R)", "kernel": "chx_ft_batch",
            "config": {"workload": "4,096 spectra x k^1/k^2/k^3, 241 k -> 200 R points (0-6 A), "
                                   "Kaiser dk 1, k 3-13",
                       "spectra": nspec, "nk": nk, "nR": nR, "l2": "flushed before each call"},
            "precisions": {"0": "FP64 SIMT", "1": "FP32 SIMT", "2": "split-BF16 tcgen05",
                           "3": "TF32 tcgen05",
                           "fused_2": "split-BF16 tcgen05, window-sums epilogue "
                                      "(chx_ft_window_sums)", "fused_3": "TF32, fused"},
            "results": res,
            "roofline": {"bound": "hbm", "achieved": tc["GB_per_s"], "peak": hbm,
                         "unit": "GB/s", "frac": tc["GB_per_s"] / hbm, "peak_source": src,
                         "bytes": "chi + basis read, chi(R) written, FP64; the three k "
                                  "weights in one call against their bases side by side"}}
    print(json.dumps(line), flush=True)
    return 0


def r_factors(bs, prob):
    """R-factor of each ladder's best state (chimera/model.py:535-540 with the
    per-edge profiled scales of model.py:495-510): sum |s m - d|^2 / sum |d|^2
    over the fit window, m the model chi(R) of the state, d the target."""
    import torch
    out = []
    for li, spec in enumerate(bs.lad.specs):
        sp, _ = bs.best(li)
        sp_d = torch.from_numpy(sp[None].astype(np.int32)).cuda()
        chi = spec.fm.chi_full(torch.from_numpy(prob.cell.ideal[None]).cuda(), sp_d)
        if spec.ms is not None:
            chi = chi + spec.ms.full(sp_d)
        cnt = torch.from_numpy(np.bincount(sp, minlength=prob.nsp).astype(np.float64)).cuda()
        m = prob.ft.to_R(chi[0] / cnt.clamp_min(1)[:, None]).cpu().numpy()
        d, mask = spec.target, spec.mask
        edge = prob.ft.chan_edge
        num = np.real((np.conj(m[:, mask]) * d[:, mask]).sum(1))
        den = np.real((np.conj(m[:, mask]) * m[:, mask]).sum(1))
        ne = int(edge.max()) + 1
        sc = (np.bincount(edge, num, ne) / np.maximum(np.bincount(edge, den, ne), 1e-30))[edge]
        r = (np.abs(m[:, mask] * sc[:, None] - d[:, mask]) ** 2).sum() / (np.abs(d[:, mask]) ** 2).sum()
        out.append(float(r))
    return np.array(out)


DA_POS = 8              # the learned configuration's sample positions
DA_ATTEMPTS = 200_000   # swap attempts per replica
DA_LOGGED = 1_000_000   # swaps logged by plain steps to train the surrogate


def _da_problem():
    from chimera_b200 import configs
    return configs.Problem(elements=("Fe", "Ni", "Cr"), composition=(0.4, 0.4, 0.2), a0=3.57,
                           alpha1=-0.12, alpha_pair=(0, 2))


def _da_run(specs, starts, prob, periods, chunk, timed, learned=None, stop=None, early=True):
    """One sampler over `specs` for `periods` exchange periods in chunks of
    `chunk` (GPU time by events; the R-factors and posterior checks after
    each chunk are untimed). Posterior samples every 2 periods, those of the
    last 40 % of the run made so far kept (the reference's 60 % start,
    fitrun.py:311). learned: (H, burn_blocks, log_blocks, epochs): plain
    burn-in periods, then log, train and screen. stop(rf, wc): stop once it
    holds for the R-factors and posterior alpha after a chunk. Returns a
    summary dict with the trajectory (early False: the rule is recorded at
    every chunk and the run goes on)."""
    from chimera_b200.sampler import BatchedSampler
    bs = BatchedSampler(specs, precision=1, exchange_every=EXCH, reanchor_every=1000,
                        threads=256, min_blocks=4)
    bs.init_state(starts, prob.cell.ideal)
    bs.capture()
    out = {"ladders": len(specs), "replicas": bs.nslots}
    start = bs.blocks
    bs.enable_collect(from_block=start, every_blocks=2)
    t = 0.0
    if learned is not None:
        H, burn, log_blocks, epochs = learned
        t += timed(lambda: bs.run_blocks(burn))
        tl = timed(lambda: bs.learn(blocks=log_blocks, epochs=epochs, H=H))
        t += tl
        rep = bs.train_report
        out.update(gpu_s_burn_log_train=t, burn_periods=burn, logged_swaps=rep.get("n"),
                   surrogate_rmse_over_sd=rep.get("rmse_d", 0) / max(rep.get("std_d", 1), 1e-30))
    traj = []

    def window_wc():
        done_ = bs.blocks - start
        try:
            return [bs.posterior_wc(li, from_block=start + int(0.6 * done_))
                    for li in range(bs.nladders)]
        except RuntimeError:
            return None

    while bs.blocks - start < periods:
        n = min(chunk, periods - (bs.blocks - start))
        t += timed(lambda: bs.run_blocks(n))
        rf = r_factors(bs, prob)
        wc = window_wc()
        hit = bool(stop(rf, wc)) if (stop is not None and wc is not None) else False
        traj.append((t, float(rf.mean()), hit))
        if hit and early:
            break
    done = bs.blocks - start
    rf = r_factors(bs, prob)
    wc = window_wc()
    out.update(gpu_s=t, periods=done, attempts_per_replica=done * EXCH,
               r_factor=[float(x) for x in rf], r_factor_mean=float(rf.mean()),
               alpha_mean=[w[0].tolist() for w in wc], alpha_sd=[w[1].tolist() for w in wc],
               alpha_samples=[int(w[2]) for w in wc], trajectory=traj,
               device_error=bs.device_error())
    if learned is not None:
        st = np.concatenate([lad.da_stats() for lad in bs.groups]).sum(0)
        out.update(exact_fraction=float(st[1] / max(st[0], 1)),
                   screening_error=float(1 - st[3] / max(st[1], 1)), fallbacks=bs.fallbacks,
                   screened_moves=float(st[0]))
    return out


def bench_da(args):
    """GPU-s of the learned + batched sampler to the plain GPU sampler's final
    R-factor, on the learned configuration: fcc Fe-Ni-Cr 40/40/20, 4,000
    sites (10x10x10, a0 3.57 A), target order alpha1(Fe-Cr) = -0.12 plus
    noise 5e-4, three K edges, 8 sample positions x 32 rungs, 2e5 swap
    attempts per replica, a surrogate trained on 1e6 swaps logged by plain
    steps.

    - plain GPU sampler: each position's ladder on its own (one ladder per
      launch, as the reference's fit loop runs its seeds, fitrun.py:306),
      2e5 attempts per replica; GPU-s summed over the positions;
    - batched plain: the 8 ladders in one launch, same length (for context);
    - learned + batched: the 8 ladders in one launch, a plain burn-in (5 %
      of the run, so the logged swaps see the converged residual), ~1e6 plain
      swaps logged and the surrogate trained, then delayed acceptance until
      the mean best R-factor is within 1 % of the plain one (fitrun.py:378
      definition) and every position's posterior alpha is within plain's
      posterior sd, at most 2e5 attempts per replica; all of it counted.
    Each reports its R-factors and posterior first-shell Warren-Cowley alpha
    (mean, sd; the reference's collection: 60 % into the run, every 50 steps,
    the 4 rungs nearest beta 0.5). --steps other than the default sets the
    periods (a short run)."""
    import torch
    from chimera_b200 import _native as N
    from chimera_b200.sampler import LadderSpec
    N.lib()
    prob = _da_problem()
    npos = DA_POS if args.positions == 16 else args.positions
    periods = DA_ATTEMPTS // EXCH if args.steps == 1200 else args.steps
    chunk = max(1, periods // 20)
    specs = []
    for p in range(npos):
        pos = prob.position(p)
        specs.append(LadderSpec(prob.fm, prob.ft, pos.target, pos.mask, pos.sigma_R, nrep=NREP,
                                tmin=1e-4, tmax=1e-1, seed=p, swap_frac=1.0,
                                disp_sigma=0.012, max_disp=0.10, ms_library=prob.ms))
    starts = [prob.random_config(1000 + p) for p in range(npos)]
    s = torch.cuda.current_stream()

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        fn()
        b.record(s)
        b.synchronize()
        return a.elapsed_time(b) * 1e-3

    # plain GPU sampler: one ladder per launch, position after position
    singles = [_da_run([specs[p]], [starts[p]], prob, periods, chunk, timed)
               for p in range(npos)]
    plain = {"gpu_s": float(sum(r["gpu_s"] for r in singles)),
             "r_factor": [r["r_factor"][0] for r in singles],
             "alpha_mean": [r["alpha_mean"][0] for r in singles],
             "alpha_sd": [r["alpha_sd"][0] for r in singles],
             "periods": periods, "per_position_gpu_s": [r["gpu_s"] for r in singles]}
    plain["r_factor_mean"] = float(np.mean(plain["r_factor"]))
    # plain's own time to within 1 % of its final R-factor (trajectories summed)
    target = 1.01 * plain["r_factor_mean"]
    npts = min(len(r["trajectory"]) for r in singles)
    reach = None
    for q in range(npts):
        if np.mean([r["trajectory"][q][1] for r in singles]) <= target:
            reach = float(sum(r["trajectory"][q][0] for r in singles))
            break
    plain["gpu_s_to_within_1pct"] = reach
    am, asd = np.array(plain["alpha_mean"]), np.array(plain["alpha_sd"])

    def reached(rf, wc):
        """plain's final R-factor within 1 % (mean over positions) and every
        position's posterior alpha within plain's posterior sd"""
        if rf.mean() > target:
            return False
        return all(np.all(np.abs(np.asarray(wc[p][0]) - am[p]) <= asd[p]) for p in range(npos))

    batched = _da_run(specs, starts, prob, periods, chunk, timed, stop=reached, early=False)
    hits = [t for t, _, h in batched["trajectory"] if h]
    batched["gpu_s_to_reach"] = hits[0] if hits else None
    log_blocks = max(1, -(-DA_LOGGED // (npos * NREP * EXCH)))
    burn = max(1, periods // 20)
    learned = _da_run(specs, starts, prob, periods, chunk, timed,
                      learned=(64, burn, log_blocks, 4), stop=reached)
    lr = learned
    lr["reached"] = bool(lr["trajectory"] and lr["trajectory"][-1][2])

    def alpha_agree(run):
        """positions whose posterior alpha lies within the plain posterior sd"""
        ok = []
        for p in range(npos):
            d = np.abs(np.array(run["alpha_mean"][p]) - np.array(plain["alpha_mean"][p]))
            ok.append(bool(np.all(d <= np.array(plain["alpha_sd"][p]) + 1e-12)))
        return ok

    line = {"metric": METRIC, "kernel": "learned + batched vs plain GPU sampler",
            "config": {"workload": "fcc Fe40Ni40Cr20 4000 atoms (10x10x10, a0 3.57 A), "
                                   "alpha1(Fe-Cr) -0.12 + noise 5e-4, 3 K edges, SS 5.0 A + "
                                   "exact MS 5.5 A, k^1/k^2/k^3 Kaiser complex chi(R) 1.4-5.0 A",
                       "positions": npos, "rungs": NREP, "periods": periods,
                       "attempts_per_replica": periods * EXCH, "logged_swaps": DA_LOGGED,
                       "surrogate": "BF16 MLP 3 x 64 hidden"},
            "plain": plain, "batched_plain": batched, "learned_batched": learned,
            "ratio_plain_over_learned": plain["gpu_s"] / lr["gpu_s"],
            "ratio_plain_over_batched_plain": plain["gpu_s"] / batched["gpu_s"],
            "learned_reached": lr["reached"],
            "reach_rule": "mean best R-factor within 1 % of plain's and every position's "
                          "posterior alpha (last 40 % of the run) within plain's posterior sd",
            "alpha_within_plain_sd": {"learned": alpha_agree(lr), "batched": alpha_agree(batched)},
            "alpha_index": "first shell, upper triangle (FeFe, FeNi, FeCr, NiNi, NiCr, CrCr)"}
    print(json.dumps(line), flush=True)
    return 0


# the uneven series: (lattice, elements, composition, a0, cells, alpha1 target);
# exact 3-/4-leg MS to 5.5 A on every point
UNEVEN = (("fcc", ("Fe", "Ni"), (0.5, 0.5), 3.55, (5, 5, 5), -0.05),
          ("fcc", ("Fe", "Ni"), (0.5, 0.5), 3.57, (8, 8, 8), -0.10),
          ("fcc", ("Fe", "Ni"), (0.5, 0.5), 3.59, (10, 10, 10), -0.08),
          ("fcc", ("Fe", "Ni"), (0.5, 0.5), 3.60, (20, 20, 10), -0.06),
          ("fcc", ("Fe", "Ni"), (0.5, 0.5), 3.62, (20, 20, 20), -0.04),
          ("bcc", ("Fe", "Cr"), (0.5, 0.5), 2.87, (5, 5, 10), -0.06),
          ("bcc", ("Fe", "Cr"), (0.5, 0.5), 2.87, (10, 10, 10), -0.12),
          ("hcp", ("Co", "Ni"), (0.5, 0.5), 2.507, (8, 8, 6), -0.05),
          ("hcp", ("Co", "Ni"), (0.5, 0.5), 2.507, (12, 12, 10), -0.08),
          ("fcc", ("Fe", "Ni", "Cr"), (0.4, 0.4, 0.2), 3.59, (8, 8, 8), -0.08),
          ("fcc", ("Fe", "Ni", "Cr"), (0.4, 0.4, 0.2), 3.59, (10, 10, 10), -0.12),
          ("bcc", ("Fe", "Cr", "Ni"), (0.4, 0.4, 0.2), 2.87, (8, 8, 8), -0.06))
UNEVEN_POS = 2


def bench_uneven(args):
    """The uneven serving-style batch: 24 series points (12 supercells of
    500-32,000 sites: fcc Fe-Ni a0 3.55-3.62 A, bcc Fe-Cr 2.87 A, hcp Co-Ni
    2.507 A, and fcc / bcc Fe-Ni-Cr ternaries; exact MS to 5.5 A; seeded SRO targets alpha1 -0.12..-0.04 plus noise, 2 sample
    positions each), 16 rungs per point. All 24 ladders run in one graph
    replay per exchange period (one step launch per species count, the two on
    parallel streams), against the same ladders run one ladder per launch one
    after the other (the reference's host loop over points). Swap
    attempts/s of both, device time by CUDA events."""
    import torch
    from chimera_b200 import _native as N
    from chimera_b200 import configs
    from chimera_b200.sampler import BatchedSampler, LadderSpec
    N.lib()
    specs, starts = [], []
    for q, (lat, els, comp, a0, nc, al) in enumerate(UNEVEN):
        prob = configs.Problem(elements=els, composition=comp, a0=a0, lattice=lat, ncell=nc,
                               alpha1=al, order_seed=q)
        for p in range(UNEVEN_POS):
            pos = prob.position(10 * q + p)
            specs.append(LadderSpec(prob.fm, prob.ft, pos.target, pos.mask, pos.sigma_R,
                                    nrep=16, tmin=1e-4, tmax=1e-1, seed=10 * q + p,
                                    swap_frac=1.0, ms_library=prob.ms))
            starts.append((prob.random_config(100 + 10 * q + p), prob.cell.ideal))
    nb = 40 if args.steps == 1200 else max(4, min(args.steps, 200))
    s = torch.cuda.current_stream()

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        fn()
        b.record(s)
        b.synchronize()
        return a.elapsed_time(b) * 1e-3

    bs = BatchedSampler(specs, precision=1, exchange_every=EXCH, reanchor_every=1000)
    bs.init_state([x[0] for x in starts], [x[1] for x in starts])
    bs.autotune()
    bs.capture()
    bs.run_blocks(max(3, args.warmup))
    t_batch = timed(lambda: bs.run_blocks(nb))
    t_sep = 0.0
    for li, (sp, (s0, p0)) in enumerate(zip(specs, starts)):
        lad, _ = bs.ladder(li)
        one = BatchedSampler([sp], precision=1, exchange_every=EXCH, reanchor_every=1000,
                             threads=lad.threads, min_blocks=lad.min_blocks)
        one.init_state([s0], [p0])
        one.capture()
        one.run_blocks(2)
        t_sep += timed(lambda: one.run_blocks(nb))
        del one
    att = bs.nslots * EXCH * nb
    # the same batch with delayed acceptance: one surrogate per (species
    # count, feature width) class, learned from 40 periods of its own swaps
    rep = bs.learn(blocks=40, epochs=4, H=256)
    bs.capture()
    bs.run_blocks(2)
    t_learned = timed(lambda: bs.run_blocks(nb))
    st = bs.last_screen.sum(0) if hasattr(bs, "last_screen") else np.zeros(4)
    line = {"metric": METRIC, "kernel": "uneven batch",
            "config": {"workload": "24 series points: fcc Fe-Ni a0 3.55-3.62 A (500-32,000 "
                                   "sites), bcc Fe-Cr 2.87 A, hcp Co-Ni 2.507 A, fcc/bcc "
                                   "Fe-Ni-Cr ternaries; exact 3-/4-leg MS 5.5 A on all; one K "
                                   "edge per species, 16 rungs",
                       "sites": sorted({int(sp.fm.natoms) for sp in specs}),
                       "lattices": sorted({u[0] for u in UNEVEN}),
                       "species_counts": [g.nsp for g in bs.groups],
                       "ladders": len(specs), "replicas": bs.nslots, "periods": nb},
            "batched": {"attempts_per_s": att / t_batch, "gpu_s": t_batch,
                        "launch_shapes": [list(t["shape"]) for t in bs.tuning],
                        "tuning": [{"nsp": g.nsp, "ladders": g.nladders, "replicas": g.nslots,
                                    "shape": list(t["shape"]),
                                    "tensor_core_transform": t.get("tensor_core_transform"),
                                    "us_per_step": t["us_per_step"]}
                                   for g, t in zip(bs.groups, bs.tuning)]},
            "one_ladder_per_launch": {"attempts_per_s": att / t_sep, "gpu_s": t_sep},
            "learned": {"attempts_per_s": att / t_learned, "gpu_s": t_learned,
                        "surrogates": len(bs.surrogates),
                        "fit_rmse_over_sd": [round(r["rmse_d"] / r["std_d"], 3)
                                             for r in (rep if isinstance(rep, list) else [rep])],
                        "passed_to_exact": float(st[1] / max(st[0], 1)),
                        "fallbacks": bs.fallbacks},
            "speedup": t_sep / t_batch, "unit": UNIT,
            "device_error": bs.device_error()}
    print(json.dumps(line), flush=True)
    return 0


def bench_calib(args):
    """The calibration objective (chimera/calibrate.py's differential
    evolution over the pair-count model): an fcc Fe-Ni 4x4x4 model to
    6.2 A (5 shells), 241 k points, k^1/k^2/k^3 complex chi(R) data of an
    ordered configuration (its path sum through the Hanning-window transform,
    fitted over 1.4-5.0 A). Times (1) the population objective, members per
    second, for the reference's stage-1 population (popsize 12 x 12
    parameters = 144 members) and for 4,096 members, CUDA events; (2) the
    reference's whole global stage (maxiter 120, popsize 12, tol 1e-8,
    polished) with one launch per generation, wall clock; beside the CPU
    restatement of the objective per member on one core."""
    import time
    import torch
    from chimera_b200 import _native as N
    from chimera_b200 import configs
    from chimera_b200.calibrate import Stage1, de_stage1
    from chimera_b200.fourier import FourierTransform
    from chimera_b200.shellmodel import ShellModel
    N.lib()
    prob = configs.Problem(ncell=(4, 4, 4), rmax=6.2, ms=False, alpha1=-0.08)
    top = prob.top
    z = np.bincount(top.shell, minlength=top.nshell) / top.natoms
    sm = ShellModel(prob.k, prob.tables, top.r_shell, z, top.s2_shell, top.natoms, 3.59,
                    s02=0.85, pairs=(top.i, top.j, top.shell), composition=(0.5, 0.5),
                    elements=("Fe", "Ni"))
    kw = (1, 2, 3)
    sm.set_params(kweight=kw)
    chi = prob.target_chi()
    fts = [FourierTransform(prob.k, 3.0, 13.0, w) for e in range(2) for w in kw]
    bins = np.arange(200)
    data = np.array([f.to_R(chi[e], bins=bins) for f, e in zip(fts, (0, 0, 0, 1, 1, 1))])
    R = fts[0].R[:200]
    mask = (R > 1.4) & (R < 5.0)
    Nc = sm.counts_of(prob.target_species)
    st = Stage1(sm, (0.5, 0.5), ms=False, elements=("Fe", "Ni"))
    rng = np.random.default_rng(0)
    lo, hi = np.array(st.bounds).T

    def pop(n):
        return st.rows(lo + (hi - lo) * rng.uniform(size=(n, lo.size)), a0=3.59)

    s = torch.cuda.current_stream()
    out = {}
    for P in (12 * len(st.names), 4096):
        X = pop(P)
        for _ in range(3):
            sm.r_factor_batch(Nc, data, mask, bins, X)
        reps = 10
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        a.record(s)
        for _ in range(reps):
            sm.r_factor_batch(Nc, data, mask, bins, X)
        b.record(s)
        b.synchronize()
        wall = (time.perf_counter() - t0) / reps
        out[P] = dict(members_per_s_device_span=P * reps / (a.elapsed_time(b) * 1e-3),
                      members_per_s_with_host=P / wall)
    # the whole global stage, wall clock
    t0 = time.perf_counter()
    gens = 120 if args.steps == 1200 else max(1, min(args.steps, 120))   # small profiling case
    res, nev = de_stage1(sm, Nc, data, mask, bins, st, a0=3.59, maxiter=gens, popsize=12,
                         seed=0, tol=1e-8, polish=gens == 120)
    t_de = time.perf_counter() - t0
    # CPU: the restatement of the objective, one member at a time
    cpu = None
    if not args.no_cpu:
        sys.path.insert(0, ROOT)
        from oracle import shellmodel as OS
        m = dict(k=sm.k, f=sm.f, delta=sm.delta, lam=sm.lam, shells_ref=sm.shells_ref,
                 shell_mult=sm.z, sigma2_ref=sm.sigma2_shell_ref, a0_ref=sm.a0_ref,
                 s02=sm.s02, dk_win=sm.dk_win, etok=sm.etok)
        X = pop(40)
        t0 = time.perf_counter()
        for x in X:
            OS.r_factor(x, Nc, m, data[:, mask], bins[mask], kw)
        cpu = 40 / (time.perf_counter() - t0)
    line = {"metric": "calibration objective: pair-count R-factor per parameter set",
            "kernel": "calibration population (chx_shell_rfactor)", "unit": "members/s",
            "config": {"workload": "fcc Fe50Ni50 pair-count model, 4x4x4 cells, SS to 6.2 A "
                                   "(5 shells), 241 k, k^1/k^2/k^3 complex chi(R), Hanning "
                                   "window 3-13 A^-1, fitted 1.4-5.0 A",
                       "parameters": len(st.names), "fitted_bins": int(mask.sum())},
            "population": {str(k): v for k, v in out.items()},
            "de_stage1": {"wall_s": t_de, "members_evaluated": nev, "generations": int(res.nit),
                          "r_factor": float(res.fun),
                          "cpu_estimate_s": (nev / cpu) if cpu else None},
            "cpu_baseline": None if cpu is None else {
                "value": cpu, "unit": "members/s", "cores": 1, "kind": "port",
                "sample": "CPU restatement of the objective, 40 members one at a time"}}
    print(json.dumps(line), flush=True)
    return 0


def bench_band(args):
    """The systematic band (chimera/fitrun.py:652-718): the reference's 18
    calibration variants of the 4,000-site fcc Fe-Ni workload (exact MS,
    k^1/k^2/k^3 Kaiser complex chi(R)), 48 rungs each (its nrep), 6,000 steps
    (240 exchange periods, its nsteps) of every variant as ONE batched sampler,
    against the same variants run one after the other (the reference's loop).
    Device time by CUDA events; swap attempts/s of both; the band of the
    batched run."""
    import torch
    from chimera_b200 import _native as N
    from chimera_b200 import band as B
    from chimera_b200.sampler import BatchedSampler
    N.lib()
    nb = 240 if args.steps == 1200 else max(4, min(args.steps, 240))
    base, vs = B.build_variants(dict(ncell=(10, 10, 10)))
    specs, meta = B.variant_specs(base, vs, positions=(0,), nrep=48)
    starts = [v.prob.random_config(100 + i) for i, (v, _) in enumerate(meta)]
    ideal = [v.prob.cell.ideal for v, _ in meta]
    s = torch.cuda.current_stream()

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        fn()
        b.record(s)
        b.synchronize()
        return a.elapsed_time(b) * 1e-3

    bs = BatchedSampler(specs, precision=1, exchange_every=EXCH, reanchor_every=1000,
                        threads=256, min_blocks=4)
    bs.init_state(starts, ideal)
    bs.capture()
    t_batch = timed(lambda: bs.run_blocks(nb))
    common = vs[0].ft_data.window_mask(*vs[0].rwin)
    rows = [B.variant_result(bs, li, v, specs[li], common) for li, (v, _) in enumerate(meta)]
    band = B.band_from_variants(rows)
    t_seq = 0.0
    for li in range(len(specs)):
        one = BatchedSampler([specs[li]], precision=1, exchange_every=EXCH,
                             reanchor_every=1000, threads=256, min_blocks=4)
        one.init_state([starts[li]], [ideal[li]])
        one.capture()
        t_seq += timed(lambda: one.run_blocks(nb))
        del one
    att = bs.nslots * EXCH * nb
    line = {"metric": METRIC, "kernel": "systematic band (18 calibration variants)",
            "unit": UNIT,
            "config": {"workload": "fcc Fe50Ni50 4000 atoms, SS 5.0 A + exact MS 5.5 A, "
                                   "k^1/k^2/k^3 Kaiser complex chi(R) 1.4-5.0 A; the 18 "
                                   "calibration variants (a0, dE0, sigma^2, k weight, k and R "
                                   "window, MS amplitude, dr, C3)",
                       "variants": len(vs), "rungs": 48, "replicas": bs.nslots,
                       "steps": nb * EXCH},
            "batched": {"attempts_per_s": att / t_batch, "gpu_s": t_batch},
            "one_variant_per_launch": {"attempts_per_s": att / t_seq, "gpu_s": t_seq},
            "speedup": t_seq / t_batch,
            "band": {k: band[k] for k in ("wc_min", "wc_max", "n_admissible", "n_comparable",
                                          "excluded_incomparable", "r_factor_baseline",
                                          "r_factor_range")},
            "device_error": bs.device_error()}
    print(json.dumps(line), flush=True)
    return 0


def bench_pathtrace(args):
    """The curved-wave path trace (exafs_gpu/abinitio/pathsum.py): every
    3- and 4-leg path class of fcc to 5.5 A half length (25 classes) and the
    first three single-scattering shells, Fe-Ni alternating along the path,
    at 120 energies (k 2-18 A^-1) with smooth synthetic complex phase shifts
    of two types; lmax per (path, energy) where |t_l| > 1e-6 (at most 40).
    Traces per second of one chx_path_trace launch (CUDA events) and of the
    whole call from host arrays; beside the CPU evaluation (oracle, dense
    matrices) on a bounded sample."""
    import time
    import torch
    from chimera_b200 import _native as N
    from chimera_b200 import mspaths as MP
    from chimera_b200 import pathtrace as PT
    N.lib()
    bohr = 0.529177210903
    a0 = 3.59
    unit = a0 / 2.0 / bohr
    cls = MP.enumerate_classes(a0, 5.5, "fcc")
    sites = [np.array([[1, 1, 0]]) * unit, np.array([[2, 0, 0]]) * unit,
             np.array([[2, 1, 1]]) * unit]
    for c in cls:
        rep = np.asarray(c.rep, float) * unit
        sites.append(rep)
    # a 4-leg class may pass through the absorber (q2 = 0); the trace needs
    # scatterers off the origin, so such classes are left out
    sites = [s_ for s_ in sites if np.all(np.linalg.norm(s_, axis=1) > 1e-9)]
    types = [tuple(q % 2 for q in range(len(s_))) for s_ in sites]
    nE, nl = 120, 41
    k = np.linspace(2.0, 18.0, nE)
    kb = k * bohr
    p = kb + 1j * (0.02 + 0.002 * kb)
    l = np.arange(nl)
    S = np.empty((2, nE, nl), complex)
    for ty in range(2):
        width = 0.75 * kb[:, None] * (2.3 + 0.3 * ty) + 1.0
        d = (0.9 + 0.25 * ty) * np.exp(-(l[None, :] / width) ** 2)
        S[ty] = np.exp(2j * (d + 0.02j * np.exp(-(l[None, :] / width) ** 2)))
    t = 0.5 * (S - 1.0)
    big = np.abs(t).max(0) > 1e-6
    lm_e = np.array([max(2, int(np.nonzero(row)[0].max())) for row in big])
    lmax = np.minimum(np.tile(lm_e, (len(sites), 1)), PT.MAX_L).astype(np.int32)
    PT.path_trace(sites, types, p, t, lmax)                  # tables, attributes
    s = torch.cuda.current_stream()
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        tr = PT.path_trace(sites, types, p, t, lmax)
    wall = (time.perf_counter() - t0) / reps
    # device time of the launch alone: re-run through the entry with CUDA events
    a_, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a_.record(s)
    PT.path_trace(sites, types, p, t, lmax)
    b_.record(s)
    b_.synchronize()
    span = a_.elapsed_time(b_) * 1e-3
    ntr = len(sites) * nE
    cpu = None
    if not args.no_cpu:
        sys.path.insert(0, ROOT)
        from oracle import pathtrace as OP
        sample = [(q, e) for q in (0, 5, 12) for e in (10, 60)]
        t0 = time.perf_counter()
        for q, e in sample:
            OP.trace(sites[q], types[q], p[e], t[:, e], int(lmax[q, e]))
        cpu = len(sample) / (time.perf_counter() - t0)
    line = {"metric": "curved-wave path trace (ab initio path sum)", "unit": "traces/s",
            "kernel": "chx_path_trace",
            "config": {"workload": "fcc Fe-Ni: 3 SS shells + MS classes to 5.5 A, 120 energies "
                                   "k 2-18 A^-1, synthetic phase shifts of two types",
                       "paths": len(sites), "energies": nE,
                       "lmax_range": [int(lmax.min()), int(lmax.max())]},
            "traces_per_s_with_host": ntr / wall, "traces_per_s_span": ntr / span,
            "finite": bool(np.isfinite(tr).all()),
            "cpu_baseline": None if cpu is None else {
                "value": cpu, "unit": "traces/s", "cores": 1, "kind": "port",
                "sample": "CPU evaluation with dense Wigner matrices, 6 traces (3 paths x 2 energies)"}}
    print(json.dumps(line), flush=True)
    return 0


def bench_pathsum(args):
    """The full path sum (A1/A2): every single-scattering pair of a 4,000-site
    fcc Fe-Ni cell to 6.2 A (z = 78, 312,000 pairs) at 241 k points for 256
    configurations, FP32C and FP64 (chx_chi_full, CUDA events), and the exact
    MS entry counts of the same configurations (3.94 M paths each,
    chx_ms_counts + chx_ms_chi_of). Terms/s (one (pair, k) term each) and
    paths/s; beside the CPU restatement of the reference kernels (oracle, C)
    on one configuration."""
    import time
    import torch
    from chimera_b200 import _native as N
    from chimera_b200 import configs
    from chimera_b200.forward import FP32C, FP64
    N.lib()
    prob = configs.Problem(ncell=(10, 10, 10), rmax=6.2, ms=True)
    fm, ms = prob.fm, prob.ms
    nconf = 256 if args.steps == 1200 else max(8, min(args.steps, 256))
    rng = np.random.default_rng(0)
    sp = torch.from_numpy(np.stack([prob.random_config(int(rng.integers(1 << 30)))
                                    for _ in range(nconf)])).cuda()
    pos = torch.from_numpy(np.repeat(prob.cell.ideal[None], nconf, 0)).cuda()
    s = torch.cuda.current_stream()

    def timed(fn, reps=3):
        fn()
        a_, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a_.record(s)
        for _ in range(reps):
            fn()
        b_.record(s)
        b_.synchronize()
        return a_.elapsed_time(b_) * 1e-3 / reps

    terms = nconf * fm.npairs * fm.nk
    t32 = timed(lambda: fm.chi_full(pos, sp, precision=FP32C))
    t64 = timed(lambda: fm.chi_full(pos, sp, precision=FP64))
    tms = timed(lambda: ms.full(sp))
    c32 = fm.chi_full(pos[:4], sp[:4], precision=FP32C)
    c64 = fm.chi_full(pos[:4], sp[:4], precision=FP64)
    err = float((c32 - c64).abs().max() / (c64.abs().max()))
    cpu = None
    if not args.no_cpu:
        sys.path.insert(0, ROOT)
        from oracle import sampler as OS
        pr = OS.Problem(prob.cell.ideal, prob.top.i, prob.top.j, prob.top.shift, prob.top.shell,
                        prob.top.sigma2, prob.k, prob.tables.f, prob.tables.delta,
                        prob.tables.lam, prob.tables.s02, [], np.zeros((0, 1024), complex),
                        np.zeros(1024, bool), np.ones((0, 1024)), prob.nsp)
        sp0 = sp[:1].cpu().numpy()
        t0 = time.perf_counter()
        pr.chi_full(prob.cell.ideal[None], sp0)
        cpu = fm.npairs * fm.nk / (time.perf_counter() - t0)
    line = {"metric": "full path sum (single + exact multiple scattering)", "unit": "terms/s",
            "kernel": "chx_chi_full, chx_ms_counts",
            "config": {"workload": "fcc Fe50Ni50 4000 atoms, SS to 6.2 A (z 78), exact MS 5.5 A, "
                                   "241 k", "configurations": nconf, "pairs": fm.npairs,
                       "ms_paths": int(prob.paths.npath)},
            "fp32c_terms_per_s": terms / t32, "fp64_terms_per_s": terms / t64,
            "fp32c_ms_per_config": t32 / nconf * 1e3, "fp64_ms_per_config": t64 / nconf * 1e3,
            "ms_paths_per_s": nconf * prob.paths.npath / tms,
            "fp32c_vs_fp64_max_rel": err,
            "cpu_baseline": None if cpu is None else {
                "value": cpu, "unit": "terms/s", "cores": 1, "kind": "port",
                "sample": "C restatement of the reference's compute_r / build_ptype / "
                          "chi_forward, one configuration"}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    global NPOS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=30)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--positions", type=int, default=16,
                    help="ladders per GPU (fewer for a small profiling case)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--burnin", type=int, default=2000,
                    help="untimed exchange periods before tuning and timing (2,000 = 5e4 "
                         "attempts per replica, the middle of the configuration's run)")
    ap.add_argument("--e2e-periods", type=int, default=3999,
                    help="exchange periods of the end-to-end run after its first (4,000 "
                         "periods x 25 steps = the configuration's 1e5 attempts per replica)")
    ap.add_argument("--kernel", default="sampler",
                    choices=["sampler", "ft", "da", "uneven", "calib", "band", "pathtrace",
                             "pathsum"],
                    help="ft: time the windowed FT contraction (chx_ft_batch); da: GPU-s of "
                         "the learned (delayed-acceptance) sampler to the plain sampler's "
                         "R-factor on the ternary configuration")
    args = ap.parse_args()
    NPOS = args.positions
    if args.impl == "reference":
        return run_reference(args)
    if args.kernel == "ft":
        return bench_ft(args)
    if args.kernel == "da":
        return bench_da(args)
    if args.kernel == "uneven":
        return bench_uneven(args)
    if args.kernel == "calib":
        return bench_calib(args)
    if args.kernel == "band":
        return bench_band(args)
    if args.kernel == "pathtrace":
        return bench_pathtrace(args)
    if args.kernel == "pathsum":
        return bench_pathsum(args)

    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from chimera_b200 import _native as N
    N.lib()
    prob = build_problem()
    smp = make_sampler(prob, rank)
    rng = np.random.default_rng(rank)
    sp0 = [prob.random_config(int(rng.integers(1 << 30))) for _ in range(NPOS)]
    smp.init_state(sp0, prob.cell.ideal)
    # clocks are sampled from the burn-in through the timed region (the timed
    # periods alone are shorter than the sampling interval)
    clk = Clocks(local).__enter__()
    # untimed burn-in: the chains are aged to the middle of the configuration's
    # run (displaced atoms accumulate and make later steps slower), then the
    # launch shape is tuned on those states and the warm-up periods run
    smp.capture()
    smp.run_blocks(args.burnin)
    tuning = smp.autotune()
    smp.capture()
    smp.run_blocks(max(3, args.warmup))
    torch.cuda.synchronize()

    # ---- timed region: device-resident inputs
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    # each exchange period is timed by its own pair of events; between
    # periods a 256 MB write (twice the L2) flushes the cache, outside the
    # events, so no period starts from the previous one's cached state
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    for a, b in evs:
        flush.fill_(1)
        a.record(s)
        smp.run_blocks(1)
        b.record(s)
    evs[-1][1].synchronize()
    torch.cuda.synchronize()
    clk.__exit__(None, None, None)
    dt = sum(a.elapsed_time(b) for a, b in evs) / 1e3
    if world > 1:
        t = torch.tensor([dt], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dt = float(t)
        dist.barrier()
    attempts = smp.nslots * EXCH * args.steps * world
    value = attempts / dt

    # ---- dominant kernel: the fused step (one launch = 25 steps of every
    # replica), timed alone on its stream; per_step = one replica-step sweep
    smp.lad.step(EXCH)
    torch.cuda.synchronize()
    reps = 20
    t_steps = time_graph(lambda: smp.lad.step(EXCH), reps)
    per_launch = t_steps / reps
    per_step = per_launch / EXCH
    hbm, src = peaks()
    achieved = step_bytes(prob) * smp.nslots * EXCH / per_launch / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "step_traffic.json")
    if os.path.exists(tp):
        t = json.load(open(tp))
        # DRAM bytes per replica-step from the capture, scaled to this launch
        traffic = t["dram_bytes_per_replica_step"] * smp.nslots * EXCH

    # ---- end to end through the public API with host buffers: the whole
    # configuration's job (a fresh sampler from host arrays, 1e5 swap attempts
    # per replica, every period's best chi^2 read back, the best states back)
    torch.cuda.synchronize()
    e2e_blocks = args.e2e_periods
    phases = {}
    t0 = time.perf_counter()
    if not args.no_e2e:
        smp2 = make_sampler(prob, rank)
        smp2.lad.threads, smp2.lad.min_blocks = smp.lad.threads, smp.lad.min_blocks
        phases["build_s"] = time.perf_counter() - t0
        smp2.init_state(sp0, prob.cell.ideal)
        torch.cuda.synchronize()
        phases["init_s"] = time.perf_counter() - t0 - sum(phases.values())
        smp2.capture()
        torch.cuda.synchronize()
        phases["capture_s"] = time.perf_counter() - t0 - sum(phases.values())
        # every exchange period's result, every ladder's best chi^2 so far,
        # gathered and read back into pinned host memory (asynchronously, so
        # that the replays stay queued back to back)
        bests = [bb["best_chi2"] for lad in smp2.groups for bb in lad.bufs]
        res_dev = torch.empty(sum(int(x.numel()) for x in bests), dtype=torch.float64,
                              device="cuda")
        res_host = torch.empty(res_dev.shape, dtype=torch.float64).pin_memory()
        for _ in range(e2e_blocks):
            smp2.run_blocks(1)
            torch.cat(bests, out=res_dev)
            res_host.copy_(res_dev, non_blocking=True)
        per_period = res_dev.numel() * 8
        e2e_steps = smp2.nslots * EXCH * (e2e_blocks + 1)       # capture ran one period
    else:
        smp2, per_period, e2e_steps = smp, 0, 0
    best = [smp2.best(li) for li in range(NPOS)]
    torch.cuda.synchronize()
    e2e_dt = time.perf_counter() - t0
    phases["run_and_readback_s"] = e2e_dt - sum(phases.values())
    # host -> device: one species array per ladder and the shared start
    # positions; device -> host: the per-period best chi^2 and the best states
    h2d = NPOS * prob.cell.natoms * 4 + prob.cell.natoms * 24
    d2h = NPOS * (prob.cell.natoms * 4 + 8) + e2e_blocks * per_period
    e2e_val = e2e_steps / e2e_dt if e2e_steps else None
    err = smp.lad.device_error()
    # chi error vs FP64: the running FP32C chi of every replica against an
    # FP64 recompute of its state (per absorber), after the timed run
    chi_err = 0.0
    for li, bb in enumerate(smp.lad.bufs):
        spec = smp.lad.specs[li]
        full = spec.fm.chi_full(bb["pos"], bb["species"])
        if spec.ms is not None:
            full = full + spec.ms.chi_of(bb["ms_C"])
        chi_err = max(chi_err, float(((bb["chi"] - full) / bb["count"][:, :, None]).abs().max()))
    best_all = np.array([[b[1]] for b in best])
    if world > 1:
        # the one collective of the sharded run: per-ladder summaries (ladders
        # rank * NPOS + i live on rank `rank`), after the timed region
        from chimera_b200.shard import gather_summaries
        parts = [[r * NPOS + i for i in range(NPOS)] for r in range(world)]
        best_all = gather_summaries(best_all, world * NPOS, parts)

    if rank == 0:
        cpu = None
        if not args.no_cpu:
            cpu = cpu_baseline(prob, nsteps=args.cpu_steps)
        clocks = clk.summary()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic", "config": workload_config(),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                         "peak_source": src, "kernel": "k_step (fused sampler step)",
                         "launch_us": per_launch * 1e6, "step_us": per_step * 1e6,
                         "bytes_per_launch": step_bytes(prob) * smp.nslots * EXCH,
                         "bytes_layout": "reference int32 layout (algorithmic); traffic = "
                                         "measured DRAM bytes of the same launch (ncu)"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": UNIT,
                    "h2d_bytes_per_step": h2d / (e2e_blocks + 1),
                    "d2h_bytes_per_step": d2h / (e2e_blocks + 1),
                    "periods": e2e_blocks + 1, "wall_s": e2e_dt, "phases": phases,
                    "note": "the configuration's whole job from host arrays (1e5 swap "
                            "attempts per replica): build, upload, init, capture, run with "
                            "every ladder's best chi^2 read back after each exchange period, "
                            "best configs back at the end; bytes averaged over its periods"},
            "gpu_launches": args.steps * 4,
            "burn_in_periods": args.burnin,
            "clocks": clocks,
            "device_error": err,
            "chi_err_vs_fp64": {"value": chi_err, "unit": "max |chi - chi_FP64| per absorber",
                                "note": "running FP32C chi of all replicas after the timed "
                                        "run vs an FP64 path sum of their states"},
            "reanchors": smp.reanchors,
            "autotune": tuning,
            "best_chi2_min": float(np.nanmin(best_all)),
            "ladders": int(best_all.shape[0]),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
