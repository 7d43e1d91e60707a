"""Golden vectors of the systematic-band reduction, from the reference.

    python tests/golden/make_band_golden.py /path/to/reference   (or CHIMERA_REFERENCE=...)

Runs the reference's own chimera.fitrun.band_from_variants (fitrun.py:491-536)
on seeded synthetic variant rows (Warren-Cowley vectors, R-factors on the
common range, channel counts; two variants with another channel count, some
fitting better and some far worse than the baseline) and saves the rows and
its result (band.npz).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _refpath import reference_path  # noqa: E402

REF = reference_path()
sys.path.insert(0, os.path.join(HERE, "_stub"))
sys.path.insert(0, REF)

from chimera import fitrun as FR                    # noqa: E402


def main():
    rng = np.random.default_rng(4)
    out = {}
    for case in range(3):
        rows = []
        for q, (name, ch) in enumerate(FR.CALIB_VARIANTS):
            rf = 0.02 * (1.0 + (rng.uniform(-0.2, 0.6) if q else 0.0))
            rows.append(dict(variant=name, wc=rng.normal(-0.08, 0.03, 3).tolist(),
                             r_factor=rf * 1.1, r_factor_common=rf if case != 2 or q % 4 else None,
                             n_channels=2 if "kweight" in ch else 6))
        tol = (1.3, 1.1, 1.5)[case]
        res = FR.band_from_variants(rows, tol=tol)
        out[f"case{case}"] = json.dumps(dict(rows=rows, tol=tol, result=res))
    np.savez_compressed(os.path.join(HERE, "band.npz"), **out)
    print("wrote band.npz")


if __name__ == "__main__":
    main()
