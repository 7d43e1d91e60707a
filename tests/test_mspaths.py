"""MS path classes, entries and supercell paths match the reference
(chimera/mslibrary.py), and the oracle's counts/deltas match its output."""
import hashlib

import numpy as np
import pytest

from conftest import golden
from chimera_b200 import lattice as L
from chimera_b200 import mspaths as MP
from oracle import kernels as K


@pytest.fixture(scope="module")
def classes():
    return MP.enumerate_classes(3.59, 5.5)


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode() + str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def test_classes_images_and_entries(classes):
    g = golden("ms.npz")
    assert len(classes) == int(g["n_classes"]) == 25
    assert sum(c.deg for c in classes) == 984
    assert np.array_equal(np.concatenate([c.rep for c in classes]), g["rep"])
    assert np.array_equal([c.deg for c in classes], g["deg"])
    assert np.array_equal([c.nslot for c in classes], g["nslot"])
    assert np.allclose([c.reff_units() for c in classes], g["reff_units"], rtol=0, atol=1e-15)
    assert np.array_equal(np.concatenate([c.slot_of for c in classes]), g["slot_of"])
    imgs, slots = [], []
    for c in classes:
        for img, so in c.images:
            imgs.append(np.pad(img, ((0, 3 - img.shape[0]), (0, 0)), constant_values=99))
            slots.append(np.pad(so, (0, 3 - so.size), constant_values=99))
    assert np.array_equal(np.array(imgs), g["images"])
    assert np.array_equal(np.array(slots), g["image_slot_of"])
    for nsp in (2, 3):
        assert np.array_equal(MP.class_offsets(classes, nsp), g[f"cls_off{nsp}"])
        ent = np.array([gi * 1000 + sum(s * 10 ** q for q, s in enumerate(sp))
                        for gi, sp in MP.entry_list(classes, nsp)])
        assert np.array_equal(ent, g[f"entries{nsp}"])
    assert [len(MP.entry_list(classes, n)) for n in (2, 3)] == [122, 327]


@pytest.mark.parametrize("nsp", [2, 3])
def test_supercell_paths_and_oracle_counts(classes, nsp):
    g = golden("ms.npz")
    cell = L.CrystalSupercell("fcc", (5, 5, 5), 3.59)
    sp = MP.SupercellPaths(classes, cell.ideal, cell.H, 3.59, nsp)
    key = f"sc{nsp}_"
    assert sp.npath == int(g[key + "npath"]) and sp.M == int(g[key + "M"])
    P_abs = np.r_[sp.p_abs, 0].astype(np.int32)
    P_cls = np.r_[sp.p_cls, 0].astype(np.int32)
    P_slot = np.vstack([sp.p_slot, -np.ones((1, 3), np.int32)]).astype(np.int32)
    assert digest(P_abs, P_cls, P_slot, sp.inc) == str(g[key + "digest"])
    # device records are the same paths, packed
    assert np.array_equal(sp.records[:, 0] & 0xFFFFF, sp.p_abs)
    assert np.array_equal(sp.records[:, 0] >> 20, sp.cls_off[sp.p_cls])
    assert np.array_equal(sp.inc_rec[5, :, 1:], np.vstack([sp.p_slot, -np.ones((1, 3))])[sp.inc[5]])
    C = K.ms_counts(g[key + "species"], sp.p_abs, sp.p_cls, sp.p_slot, sp.cls_off, nsp, sp.nblk)
    assert np.array_equal(C, g[key + "counts"])
    dC = K.ms_delta(g[key + "species"], sp.inc, sp.p_abs, sp.p_cls, sp.p_slot, sp.npath,
                    sp.cls_off, nsp, sp.nblk, g[key + "a"], g[key + "b"], g[key + "nsa"],
                    g[key + "nsb"])
    assert np.array_equal(dC, g[key + "dC"])
    # every path contributes -1 and +1: the count change sums to zero
    assert np.all(dC.sum(1) == 0)
    # chi_of(dC) = the reference's delta chi with the seeded table
    T = np.random.default_rng(5).normal(0, 0.01, (sp.nent, 320))
    chi = np.stack([dC[:, a * sp.nblk:(a + 1) * sp.nblk] @ T[a * sp.nblk:(a + 1) * sp.nblk]
                    for a in range(nsp)], axis=1)
    assert np.allclose(chi, g[key + "chi_delta"], rtol=0, atol=1e-13)


@pytest.mark.parametrize("nsp", [2, 3])
def test_templates_give_the_incident_paths_entries(classes, nsp):
    """Every site's paths, rebuilt from the shared templates and the site's
    neighbourhood table, carry the same entries as its incidence records,
    before and after a swap."""
    from oracle import kernels as K
    cell = L.CrystalSupercell("fcc", (5, 5, 5), 3.59)
    sp = MP.SupercellPaths(classes, cell.ideal, cell.H, 3.59, nsp)
    assert sp.tpl.shape == (sp.M, 2) and sp.nbr.shape == (sp.natoms, sp.D)
    assert sp.D < 0xFE
    rng = np.random.default_rng(nsp)
    species = rng.integers(0, nsp, sp.natoms).astype(np.int32)
    for site in rng.integers(0, sp.natoms, 4):
        pids = sp.inc[site]
        pids = pids[pids < sp.npath]
        rec = []
        for pid in pids:
            e = species[sp.p_abs[pid]] * sp.nblk + sp.cls_off[sp.p_cls[pid]]
            for q in range(3):
                if sp.p_slot[pid, q] >= 0:
                    e += species[sp.p_slot[pid, q]] * nsp ** q
            rec.append(e)
        assert np.array_equal(np.sort(sp.template_entries(species, site)), np.sort(rec))
    # the count change of a swap, from templates, equals the oracle's
    a, b = 17, int(sp.nbr[17, 3])
    while species[a] == species[b]:
        species[b] = (species[b] + 1) % nsp
    nsa, nsb = int(species[b]), int(species[a])
    dC = np.zeros(sp.nent)
    for site, skip_a in ((a, False), (b, True)):
        old = sp.template_entries(species, site)
        new = sp.template_entries(species, site, a, b, nsa, nsb)
        for t, (eo, en) in enumerate(zip(old, new)):
            code = int(sp.tpl[t, 1])
            sites = [site if ((code >> 8 * p) & 0xFF) == sp.SELF else
                     (-1 if ((code >> 8 * p) & 0xFF) == sp.NONE else
                      int(sp.nbr[site, (code >> 8 * p) & 0xFF])) for p in range(4)]
            if skip_a and a in sites:
                continue
            dC[en] += 1
            dC[eo] -= 1
    ref = K.ms_delta(species[None], sp.inc, sp.p_abs, sp.p_cls, sp.p_slot, sp.npath,
                     sp.cls_off, nsp, sp.nblk, np.array([a], np.int32), np.array([b], np.int32),
                     np.array([nsa], np.int32), np.array([nsb], np.int32))[0]
    assert np.array_equal(dC, ref)


def _closed_walks(pts, norm_of, Lmax, nleg_max=4):
    """Every closed walk 0 -> q1 -> q2 (-> q3) -> 0 by brute force: q1 and
    the last point off the absorber, consecutive points distinct, total
    length <= Lmax (the 4-leg middle point may be the absorber)."""
    nz = [tuple(q) for q in pts if any(q)]
    walks = set()
    for q1 in nz:
        for q2 in nz:
            if q2 != q1 and (norm_of(q1) + norm_of(np.subtract(q2, q1)) + norm_of(q2)) <= Lmax:
                walks.add((q1, q2))
        if nleg_max < 4:
            continue
        for q2 in map(tuple, pts):
            if q2 == q1:
                continue
            l12 = norm_of(q1) + norm_of(np.subtract(q2, q1))
            for q3 in nz:
                if q3 != q2 and l12 + norm_of(np.subtract(q3, q2)) + norm_of(q3) <= Lmax:
                    walks.add((q1, q2, q3))
    return walks


@pytest.mark.parametrize("lattice", ["fcc", "hcp"])
def test_class_images_are_every_closed_walk(lattice):
    """The directed images of all classes are exactly the closed walks of
    the lattice (each once), fcc in units of a0/2 under O_h and hcp in
    hexagonal integer coordinates under its 12 site operations, to a half
    length of 4.6 A (3- and 4-leg)."""
    if lattice == "fcc":
        a0, rh = 3.59, 4.6
        cls = MP.enumerate_classes(a0, rh, "fcc")
        pts = MP.lattice_points("fcc", rh / (a0 / 2))
        Lmax = 2 * rh / (a0 / 2) + 1e-9

        def norm_of(x):
            return float(np.linalg.norm(x))
    else:
        a0, rh = 2.507, 4.6
        cls = MP.enumerate_classes(a0, rh, "hcp")
        pts = MP.hcp_points(a0, rh)
        G = MP.hcp_gram(a0)
        Lmax = 2 * rh + 1e-9

        def norm_of(x):
            x = np.asarray(x, float)
            return float(np.sqrt(x @ G @ x))
    imgs = [tuple(map(tuple, img)) for c in cls for img, _ in c.images]
    assert len(imgs) == len(set(imgs))
    assert set(imgs) == _closed_walks(pts, norm_of, Lmax)
    assert all(c.nleg in (3, 4) for c in cls)


def test_hcp_operations_are_the_site_group():
    """The 12 hcp operations form a group, preserve the metric and map A->A
    and A->B displacements onto themselves; the 60-degree rotation (a screw
    axis in hcp) is not among them."""
    ops = MP.HCP_OPS
    G = MP.hcp_gram(2.507)
    keys = {tuple(A.ravel()) for A in ops}
    assert len(keys) == 12
    for A in ops:
        assert np.allclose(A.T @ G @ A, G)
        for B in ops:
            assert tuple((A @ B).ravel()) in keys
    assert (1, -1, 0, 1, 0, 0, 0, 0, 1) not in keys
    pts = MP.hcp_points(2.507, 6.0)
    kind = MP._hcp_site_type(pts)
    for A in ops:
        assert np.array_equal(MP._hcp_site_type(pts @ A.T), kind)


@pytest.mark.parametrize("lattice,a0,nc", [("bcc", 2.87, (6, 6, 6)), ("hcp", 2.507, (8, 8, 6))])
def test_templates_cover_incident_paths_on_bcc_and_hcp(lattice, a0, nc):
    """On bcc and on hcp (both sublattices, B sites reading the inverted
    offsets), each site's template paths carry the entries of its incidence
    records, every site has the same number of incident paths, and a swap's
    count change from templates equals the oracle's recount difference."""
    cell = L.CrystalSupercell(lattice, nc, a0)
    cls = MP.enumerate_classes(a0, 5.5, lattice)
    nsp = 2
    sp = MP.SupercellPaths(cls, cell.ideal, cell.H, a0, nsp, conv=cell.cell_matrix)
    cnt = np.bincount(sp.p_abs, minlength=sp.natoms)
    for q in range(3):
        s = sp.p_slot[:, q]
        cnt += np.bincount(s[s >= 0], minlength=sp.natoms)
    assert cnt.min() == cnt.max() == sp.M
    rng = np.random.default_rng(7)
    species = rng.integers(0, nsp, sp.natoms).astype(np.int32)
    sites = list(rng.integers(0, sp.natoms, 3)) + [1, 2]      # hcp: sites 0/1 are A/B
    for site in sites:
        pids = sp.inc[site]
        pids = pids[pids < sp.npath]
        rec = []
        for pid in pids:
            e = species[sp.p_abs[pid]] * sp.nblk + sp.cls_off[sp.p_cls[pid]]
            for q in range(3):
                if sp.p_slot[pid, q] >= 0:
                    e += species[sp.p_slot[pid, q]] * nsp ** q
            rec.append(e)
        assert np.array_equal(np.sort(sp.template_entries(species, site)), np.sort(rec))
    if lattice == "hcp":
        assert set(sp.sign[:2]) == {1, -1}
    a, b = 3, int(sp.nbr[3, 5])
    while species[a] == species[b]:
        species[b] = 1 - species[b]
    C0 = K.ms_counts(species[None], sp.p_abs, sp.p_cls, sp.p_slot, sp.cls_off, nsp, sp.nblk)[0]
    sw = species.copy()
    sw[a], sw[b] = species[b], species[a]
    C1 = K.ms_counts(sw[None], sp.p_abs, sp.p_cls, sp.p_slot, sp.cls_off, nsp, sp.nblk)[0]
    dC = K.ms_delta(species[None], sp.inc, sp.p_abs, sp.p_cls, sp.p_slot, sp.npath,
                    sp.cls_off, nsp, sp.nblk, np.array([a], np.int32), np.array([b], np.int32),
                    np.array([species[b]], np.int32), np.array([species[a]], np.int32))[0]
    assert np.array_equal(C1 - C0, dC)


@pytest.mark.parametrize("nsp", [2, 3])
def test_reference_construction_lays_the_same_paths(classes, nsp):
    """SupercellMS(lib, S), the call chimera/model.py:335 makes with its path
    library and spectrum, lays the reference's path arrays (the golden digest
    of SupercellMS.__init__, mslibrary.py:351-404) on the spectrum's reference
    supercell; set_params then takes the library's table, as the reference."""
    import types
    g = golden("ms.npz")
    cell = L.CrystalSupercell("fcc", (5, 5, 5), 3.59)
    calls = []

    class Lib:                  # the parts of PathLibrary the construction reads
        def __init__(self):
            self.classes, self.nsp = classes, nsp

        def table(self, *args):
            calls.append(args)
            return np.zeros((nsp * sum(nsp ** c.nslot for c in classes), 4))

    S = types.SimpleNamespace(a0_ref=3.59, ideal0=cell.ideal, H0=cell.H)
    ms = MP.SupercellMS(Lib(), S)
    sp = ms.paths
    key = f"sc{nsp}_"
    assert sp.npath == int(g[key + "npath"]) and sp.M == int(g[key + "M"])
    P_abs = np.r_[sp.p_abs, 0].astype(np.int32)
    P_cls = np.r_[sp.p_cls, 0].astype(np.int32)
    P_slot = np.vstack([sp.p_slot, -np.ones((1, 3), np.int32)]).astype(np.int32)
    assert digest(P_abs, P_cls, P_slot, sp.inc) == str(g[key + "digest"])
    assert ms.T is None and ms.lib is not None


@pytest.mark.parametrize("nsp", [2, 3])
def test_device_templates_resolve_the_swap_from_packed_words(classes, nsp):
    """The sampler step's form of the template walk: device templates (class-
    interleaved, SELF/NONE as neighbourhood slots D and D + 1) against packed
    neighbourhood words (old entry bits 0-13, new entry 14-27, occurrences of
    site a 28-31), summed per template, give the oracle's count change."""
    from oracle import kernels as K
    cell = L.CrystalSupercell("fcc", (5, 5, 5), 3.59)
    sp = MP.SupercellPaths(classes, cell.ideal, cell.H, 3.59, nsp)
    assert sp.nent < 1 << 14
    t = sp.device_templates()
    assert np.array_equal(np.sort(t[:, 0]), np.sort(sp.tpl[:, 0]))
    rng = np.random.default_rng(10 + nsp)
    species = rng.integers(0, nsp, sp.natoms).astype(np.int32)
    a, b = 23, int(sp.nbr[23, 5])
    while species[a] == species[b]:
        species[b] = (species[b] + 1) % nsp
    nsa, nsb = int(species[b]), int(species[a])
    D = sp.D
    mul = [sp.nblk, 1, nsp, nsp * nsp]
    words = np.zeros((2, 4, D + 2), np.int64)
    for half, site in enumerate((a, b)):
        for d in range(D + 1):
            s = site if d == D else int(sp.nbr[site, d])
            so = int(species[s])
            sn = nsa if s == a else (nsb if s == b else so)
            fa = int(s == a and d < D)
            for pp in range(4):
                words[half, pp, d] = (so | sn << 14) * mul[pp] + (fa << 28)
    dC = np.zeros(sp.nent)
    for off, code in t:
        code = int(code) & 0xFFFFFFFF
        for half in range(2):
            acc = int(off) | int(off) << 14
            for pp in range(4):
                acc += int(words[half, pp, (code >> 8 * pp) & 0xFF])
            eo, en, hasa = acc & 0x3FFF, (acc >> 14) & 0x3FFF, acc >> 28
            if half == 1 and hasa:
                continue
            dC[en] += 1
            dC[eo] -= 1
    ref = K.ms_delta(species[None], sp.inc, sp.p_abs, sp.p_cls, sp.p_slot, sp.npath,
                     sp.cls_off, nsp, sp.nblk, np.array([a], np.int32), np.array([b], np.int32),
                     np.array([nsa], np.int32), np.array([nsb], np.int32))[0]
    assert np.array_equal(dC, ref)
