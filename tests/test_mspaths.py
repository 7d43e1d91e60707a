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
