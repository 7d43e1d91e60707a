"""Integer topology is bit-identical to the reference (exafs_gpu/lattice.py)."""
import hashlib

import numpy as np
import pytest

from conftest import golden
from chimera_b200 import lattice as L


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode() + str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def case(g, n):
    lat, nc, a0, ca, rmax = g[f"c{n}_meta"]
    return lat, eval(nc), eval(a0), eval(ca), eval(rmax)


@pytest.mark.parametrize("n", range(6))
def test_neighbour_list_shells_and_wc(n):
    g = golden("lattice.npz")
    lat, nc, a0, ca, rmax = case(g, n)
    cell = L.CrystalSupercell(lat, nc, a0=a0, c_over_a=ca)
    i, j, sh, off = cell.neighbour_list(rmax)
    shell, _ = L.shell_index(cell, i, j, sh)
    assert i.size == int(g[f"c{n}_npairs"])
    assert digest(i, j, sh, off, shell) == str(g[f"c{n}_digest"])
    if f"c{n}_ideal" in g.files:
        assert np.array_equal(cell.ideal, g[f"c{n}_ideal"])
        assert np.array_equal(L.build_reverse_index(i, j, cell.natoms), g[f"c{n}_rev"])
    vals, _ = cell.shell_radii(rmax)
    assert np.array_equal(vals, g[f"c{n}_shell_radii"])
    wc = L.warren_cowley(g[f"c{n}_species"], i, j, sh, cell, float(vals[0]), nsp=2)
    assert np.array_equal(wc, g[f"c{n}_wc"])


@pytest.mark.parametrize("lat,nc,a0,rmax", [("fcc", (8, 9, 10), 3.59, 5.0),
                                             ("bcc", (10, 8, 9), 2.87, 5.0),
                                             ("hcp", (10, 11, 8), 2.5, 5.0),
                                             ("sc", (10, 11, 12), 2.9, 6.2)])
def test_offset_image_shortcut_equals_27_image_search(lat, nc, a0, rmax):
    """Large cells read each candidate's image off its cell offset; the
    result is bit-identical to the reference's 27-image argmin."""
    cell = L.CrystalSupercell(lat, nc, a0)
    assert cell._offset_images(rmax) is not None
    fast = cell.neighbour_list(rmax)
    cell._offset_images = lambda r: None
    exact = cell.neighbour_list(rmax)
    assert digest(*fast) == digest(*exact)


def test_topology_uniform_and_tabulable():
    cell = L.CrystalSupercell("fcc", (4, 4, 4), 3.59)
    t = L.Topology(cell, 6.2, sigma2=0.006)
    assert t.ncoord == 78 and t.nshell == 5
    assert t.pair_tab.all()
    assert np.allclose(t.r_shell, 3.59 * np.sqrt([0.5, 1, 1.5, 2, 2.5]))


def test_random_config_and_counts():
    sp = L.random_config(4000, (0.4, 0.4, 0.2), seed=3)
    assert np.bincount(sp).tolist() == [1600, 1600, 800]
    assert L.integer_counts((1, 1), 5).tolist() == [2, 3]
