"""Launch-shape autotuner for the fused sampler step.

The step kernel is built in three launch shapes (CTA size, CTAs kept
resident per SM): (256, 3), (256, 4) and (128, 6). In FP32C with the kept
chi(R) it also has two forms of the window transform of a move's change:
split-BF16 tensor-core products (mma m16n8k16) or the FP32 rotation DFT.
Which combination is fastest depends on the supercell size, species count,
k grid, transform window (the tensor-core form pads the window's bins to
tiles of 8 and the channels to 8) and number of replicas (how many waves of
CTAs one launch takes on 148 SMs), so it is measured on the live problem:
each candidate runs a few real blocks of sampler steps, timed with CUDA
events on the launching stream, and the fastest is kept. The timed steps are
ordinary steps of the chains (they are not discarded), so tuning costs no
sampling work.

Results are cached per problem key in memory and, when `path` is given, in a
JSON file, so repeated runs on the same shapes skip the measurement.
"""
from __future__ import annotations

import json
import os

SHAPES = ((256, 3), (256, 4), (128, 6))
_CACHE = {}


def problem_key(lad, nsteps):
    h = lad.host[0]
    return (f"natoms={h.natoms},nsp={lad.nsp},nk={h.nk},nchan={h.nchan},nwin={h.nwin},"
            f"ncoef={h.ncoef},ms={int(h.ms_nblk > 0)},slots={lad.nslots},"
            f"prec={lad.precision},steps={nsteps}")


def _name(shape, tc):
    t, m = shape
    return f"{t}x{m}" + ("" if tc is None else ("+tc" if tc else "+dft"))


def tune(lad, nsteps=25, reps=3, shapes=SHAPES, path=None, force=False):
    """Pick the fastest launch shape and transform form for `lad` (a
    sampler.Ladders) and set them. Returns {"shape": (threads, min_blocks),
    "tensor_core_transform": bool or None, "us_per_step": {candidate: us}}."""
    import torch
    key = problem_key(lad, nsteps)
    disk = {}
    if path and os.path.exists(path):
        try:
            disk = json.load(open(path))
        except (OSError, ValueError):
            disk = {}
    hit = _CACHE.get(key) or disk.get(key)
    if hit and not force:
        lad.threads, lad.min_blocks = hit["shape"]
        if hit.get("tensor_core_transform") is not None:
            lad.set_transform(hit["tensor_core_transform"])
        return hit
    forms = (True, False) if lad.has_tc_transform() else (None,)
    s = torch.cuda.current_stream()
    times = {}
    for tc in forms:
        if tc is not None:
            lad.set_transform(tc)
        for shape in shapes:
            lad.threads, lad.min_blocks = shape
            lad.step(nsteps)                  # first launch sets the kernel attributes
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            for _ in range(reps):
                lad.step(nsteps)
            b.record(s)
            b.synchronize()
            times[(shape, tc)] = a.elapsed_time(b) * 1e3 / (reps * nsteps)
    (best, tc), _ = min(times.items(), key=lambda kv: kv[1])
    lad.threads, lad.min_blocks = best
    if tc is not None:
        lad.set_transform(tc)
    out = {"shape": list(best), "tensor_core_transform": tc,
           "us_per_step": {_name(sh, f): v for (sh, f), v in times.items()}}
    _CACHE[key] = out
    if path:
        disk[key] = out
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        tmp = path + f".{os.getpid()}.tmp"
        json.dump(disk, open(tmp, "w"), indent=1)
        os.replace(tmp, path)
    return out
