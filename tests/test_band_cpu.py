"""The systematic-band reduction against the reference's own
band_from_variants (tests/golden/band.npz) and the variant table."""
import json

import numpy as np
import pytest

from conftest import golden
from chimera_b200 import band as B


@pytest.mark.parametrize("case", range(3))
def test_band_from_variants_matches_reference(case):
    g = golden("band.npz")
    d = json.loads(str(g[f"case{case}"]))
    got = B.band_from_variants(d["rows"], tol=d["tol"])
    ref = d["result"]
    assert set(got) == set(ref)
    for k, v in ref.items():
        if isinstance(v, list) and v and isinstance(v[0], float):
            assert np.allclose(got[k], v, rtol=1e-15, atol=0), k
        else:
            assert got[k] == v, k


def test_variant_table_names_and_changes():
    g = golden("band.npz")
    rows = json.loads(str(g["case0"]))["rows"]
    assert [r["variant"] for r in rows] == [n for n, _ in B.CALIB_VARIANTS]
    assert len(B.CALIB_VARIANTS) == 18
