"""Exact supercell multiple scattering: path classes, entries and counts.

On a lattice with swap-only moves the geometry of every 3- and 4-leg path is
fixed and only the species on its sites change, so chi_MS of a configuration
is a table of per-entry spectra contracted with how often every (class,
absorber species, slot species) entry occurs (chimera/mslibrary.py:1-33).

This module builds the same classes, images, entry order and incidence the
reference uses, from its own enumeration:

  * `enumerate_classes` walks the closed lattice paths 0 -> q1 -> q2 (-> q3)
    -> 0 with consecutive points distinct, q1 and q_last off the absorber and
    half length <= rmax, and names each by its canonical form: the smallest
    image under the 48 signed permutations of the cube and time reversal
    (mslibrary.py:86-97). Classes are ordered by (legs, half length, key) as
    mslibrary.py:148 orders them.
  * `PathClass` lists a class's directed images in the reference's order
    (reversal outer, the 48 operations inner, first occurrence kept) with the
    slot each point fills (mslibrary.py:100-132).
  * `entry_list` / `cls_off` give the entry layout: class-major, slot species
    with slot 0 fastest (mslibrary.py:190-198, 275).
  * `SupercellPaths` places every image at every site of a periodic fcc/bcc/sc
    supercell (mslibrary.py:357-404) and packs, per site, the records of the
    paths through it {absorber | class entry offset << 20, slot0, slot1,
    slot2} that the device kernels stream.

The per-entry spectra come from a path library on the model's k grid; with
no FEFF library available, `synthetic_table` defines a smooth seeded one.
"""
from __future__ import annotations

import itertools

import numpy as np

from . import _native as N


def cubic_ops():
    """The 48 signed permutation matrices, permutation outer, signs inner."""
    out = []
    for perm in itertools.permutations(range(3)):
        for sg in itertools.product((1, -1), repeat=3):
            A = np.zeros((3, 3), int)
            for r, c in enumerate(perm):
                A[r, c] = sg[r]
            out.append(A)
    return out


OPS = cubic_ops()


def canonical(seq):
    """Smallest image of a path (points after the absorber) under O_h and
    reversal, as a tuple of tuples."""
    s0 = np.asarray(seq, int)
    best = None
    for s in (s0, s0[::-1]):
        for A in OPS:
            t = tuple(map(tuple, s @ A.T))
            if best is None or t < best:
                best = t
    return best


class PathClass:
    """One geometric class: representative, slots and directed images."""

    def __init__(self, rep):
        self.rep = np.asarray(rep, int)
        self.nleg = self.rep.shape[0] + 1
        slot_of, seen = [], {}
        for q in map(tuple, self.rep):
            if q == (0, 0, 0):
                slot_of.append(-1)
            else:
                if q not in seen:
                    seen[q] = len(seen)
                slot_of.append(seen[q])
        self.slot_of = np.array(slot_of, int)
        self.nslot = len(seen)
        imgs = {}
        for rev in (False, True):
            s = self.rep[::-1] if rev else self.rep
            so = self.slot_of[::-1] if rev else self.slot_of
            for A in OPS:
                t = tuple(map(tuple, s @ A.T))
                if t not in imgs:
                    imgs[t] = so.copy()
        self.images = [(np.array(k, int), v) for k, v in imgs.items()]
        self.deg = len(self.images)

    def reff_units(self):
        pts = np.vstack([np.zeros((1, 3)), self.rep, np.zeros((1, 3))])
        return 0.5 * float(np.linalg.norm(np.diff(pts, axis=0), axis=1).sum())


def lattice_points(lattice, radius):
    """Integer points (units of a0/2) of the cubic lattice within radius."""
    R = int(np.ceil(radius)) + 1
    g = np.array(list(itertools.product(range(-R, R + 1), repeat=3)))
    if lattice == "fcc":
        g = g[(g.sum(1) % 2) == 0]
    elif lattice == "bcc":
        g = g[np.all(g % 2 == 0, axis=1) | np.all(g % 2 == 1, axis=1)]
    elif lattice == "sc":
        g = g[np.all(g % 2 == 0, axis=1)]
    else:
        raise NotImplementedError(f"multiple-scattering classes for {lattice!r} are not built "
                                  "(the lattice needs integer coordinates in units of a0/2)")
    return g[np.linalg.norm(g, axis=1) <= radius + 1e-9]


def enumerate_classes(a0, rmax_half, lattice="fcc", nleg_max=4):
    """The 3- and 4-leg path classes of a cubic lattice to half length rmax."""
    unit = a0 / 2.0
    Lmax = 2.0 * rmax_half / unit + 1e-9
    pts = lattice_points(lattice, rmax_half / unit)
    nz = pts[np.any(pts != 0, axis=1)]
    norm = np.linalg.norm(pts, axis=1)
    keys = set()
    zero = np.zeros(3, int)
    for q1 in nz:
        l1 = np.linalg.norm(q1)
        # 3 legs: 0 -> q1 -> q2 -> 0
        for q2 in nz:
            if np.array_equal(q2, q1):
                continue
            L = l1 + np.linalg.norm(q2 - q1) + np.linalg.norm(q2)
            if L <= Lmax:
                keys.add(canonical([q1, q2]))
        if nleg_max < 4:
            continue
        # 4 legs: 0 -> q1 -> q2 -> q3 -> 0 (q2 may be the absorber)
        for i2, q2 in enumerate(pts):
            if np.array_equal(q2, q1):
                continue
            l12 = l1 + np.linalg.norm(q2 - q1)
            if l12 + norm[i2] > Lmax:
                continue
            for q3 in nz:
                if np.array_equal(q3, q2):
                    continue
                L = l12 + np.linalg.norm(q3 - q2) + np.linalg.norm(q3)
                if L <= Lmax:
                    keys.add(canonical([q1, q2, q3]))
    del zero
    ks = sorted(keys, key=lambda k: (len(k), PathClass(k).reff_units(), k))
    return [PathClass(k) for k in ks]


def entry_list(classes, nsp):
    """[(class index, species tuple)], class-major, slot 0 fastest."""
    out = []
    for g, cl in enumerate(classes):
        for code in range(nsp ** cl.nslot):
            out.append((g, tuple((code // nsp ** q) % nsp for q in range(cl.nslot))))
    return out


def class_offsets(classes, nsp):
    return np.cumsum([0] + [nsp ** c.nslot for c in classes])[:-1].astype(np.int32)


def synthetic_table(classes, nsp, k, f, delta, lam, sigma2_nn, r_nn, unit, c_ms=1.3,
                    s02=1.0, amp=1.0):
    """Per-entry chi of one path occurrence (nsp * nblk, nk), absorber-major,
    for runs without a FEFF path library: the single-scattering form with the
    reference's MS length and Debye-Waller conventions (mslibrary.py:304-313,
    sigma^2_path = c_ms sigma^2_NN reff / (2 r_NN)), an amplitude of 0.2 times
    the mean backscattering amplitude of the slot species, and the phase of the
    absorber to the last slot plus 0.3 rad per class index."""
    k = np.asarray(k, float)
    rows = []
    for a in range(nsp):
        for g, sp in entry_list(classes, nsp):
            cl = classes[g]
            r = cl.reff_units() * unit
            s2 = c_ms * sigma2_nn * r / (2.0 * r_nn)
            F = 0.2 * np.mean([f[s] for s in sp], axis=0)
            ph = delta[a, sp[-1]] + 0.3 * g
            rows.append(amp * s02 * F / np.maximum(k * r * r, 1e-12)
                        * np.exp(-2.0 * r / np.maximum(lam, 1e-6) - 2.0 * k * k * s2)
                        * np.sin(2.0 * k * r + ph))
    return np.array(rows)


class SupercellPaths:
    """Every image of every class at every site of a periodic cubic supercell.

    ideal (natoms, 3) and H (3, 3) of the supercell; a0 its lattice constant.
    Arrays (as mslibrary.py:357-404): p_abs, p_cls (npath), p_slot (npath, 3);
    inc (natoms, M) incident path ids padded with npath; records (npath, 4)
    and inc_rec (natoms, M, 4) for the device.
    """

    def __init__(self, classes, ideal, H, a0, nsp):
        self.classes = classes
        self.nsp = nsp
        self.nblk = int(sum(nsp ** c.nslot for c in classes))
        self.nent = nsp * self.nblk
        self.cls_off = class_offsets(classes, nsp)
        unit = a0 / 2.0
        X = np.asarray(ideal, float) / unit
        Xi = np.rint(X).astype(int)
        if not np.allclose(X, Xi, atol=1e-6):
            raise ValueError("supercell sites are not lattice points in units of a0/2")
        Hu = np.asarray(H, float) / unit
        if not np.allclose(Hu, np.diag(np.diag(Hu))):
            raise ValueError("exact multiple scattering needs an orthogonal box")
        box = np.rint(np.diag(Hu)).astype(int)
        Xi %= box
        look = -np.ones(tuple(box), int)
        look[Xi[:, 0], Xi[:, 1], Xi[:, 2]] = np.arange(len(Xi))
        n = self.natoms = len(Xi)
        P_abs, P_cls, P_slot = [], [], []
        for g, cl in enumerate(classes):
            if 2 * np.abs(cl.rep).max() >= box.min():
                raise ValueError("supercell too small for the paths")
            for img, so in cl.images:
                p = (Xi[:, None, :] + img[None]) % box
                sites = look[p[..., 0], p[..., 1], p[..., 2]]
                if (sites < 0).any():
                    raise ValueError("an image lands off the lattice")
                slot = -np.ones((n, 3), int)
                for q in range(cl.nslot):
                    slot[:, q] = sites[:, int(np.argmax(so == q))]
                P_abs.append(np.arange(n))
                P_cls.append(np.full(n, g))
                P_slot.append(slot)
        self.p_abs = np.concatenate(P_abs).astype(np.int32)
        self.p_cls = np.concatenate(P_cls).astype(np.int32)
        self.p_slot = np.concatenate(P_slot).astype(np.int32)
        self.npath = int(self.p_abs.size)
        cnt = np.bincount(self.p_abs, minlength=n)
        for q in range(3):
            s = self.p_slot[:, q]
            cnt += np.bincount(s[s >= 0], minlength=n)
        self.M = int(cnt.max())
        self.records = np.empty((self.npath, 4), np.int32)
        self.records[:, 0] = self.p_abs | (self.cls_off[self.p_cls] << 20)
        self.records[:, 1:] = self.p_slot
        self._inc = self._inc_rec = None

        self._templates(Xi, box, look)

    @property
    def inc(self):
        """(natoms, M) ids of the paths through each site, ascending, padded
        with npath (mslibrary.py:399-404); built on first use."""
        if self._inc is None:
            n = self.natoms
            site = np.concatenate([self.p_abs] + [self.p_slot[:, q] for q in range(3)])
            pid = np.tile(np.arange(self.npath), 4)
            keep = site >= 0
            site, pid = site[keep], pid[keep]
            order = np.argsort(site, kind="stable")
            site, pid = site[order], pid[order]
            cnt = np.bincount(site, minlength=n)
            inc = np.full((n, self.M), self.npath, np.int64)
            start = np.r_[0, np.cumsum(cnt)[:-1]]
            inc[site, np.arange(site.size) - start[site]] = pid
            self._inc = inc.astype(np.int32)
        return self._inc

    @property
    def inc_rec(self):
        """(natoms, M, 4) records of the paths through each site (-1 rows as
        padding), for the reference-interface delta; built on first use."""
        if self._inc_rec is None:
            pad = np.full((1, 4), -1, np.int32)
            self._inc_rec = np.concatenate([self.records, pad])[self.inc]
        return self._inc_rec

    # Every site of a cubic Bravais supercell sees the same paths up to a
    # translation, so the paths through a site are one shared list of
    # templates plus the site's own table of nearby sites.
    SELF, NONE = 0xFE, 0xFF

    def _templates(self, Xi, box, look):
        """tpl (M, 2) int32: [class entry offset, 4 position bytes (absorber,
        slot0, slot1, slot2): local index of the site in the neighbourhood
        table, SELF for the site itself, NONE for an unused slot]; nbr
        (natoms, D) int32: site index of every neighbourhood offset."""
        offs = {}
        rows = []
        for g, cl in enumerate(self.classes):
            for img, so in cl.images:
                pos = [(0, 0, 0)] + [tuple(img[int(np.argmax(so == q))])
                                     for q in range(cl.nslot)]
                pos += [None] * (4 - len(pos))
                for r in range(1 + cl.nslot):              # the site at position r
                    code = 0
                    for p in range(4):
                        if p == r:
                            v = self.SELF
                        elif pos[p] is None:
                            v = self.NONE
                        else:
                            d = tuple(int(x) for x in np.subtract(pos[p], pos[r]))
                            v = offs.setdefault(d, len(offs))
                        code |= v << (8 * p)
                    rows.append((int(self.cls_off[g]), code))
        if len(offs) >= self.SELF:
            raise ValueError(f"{len(offs)} neighbourhood sites do not fit one byte")
        if len(rows) != self.M:
            raise ValueError("templates do not cover the incident paths")
        self.D = len(offs)
        D = np.array(list(offs.keys()), int)
        t = np.array(rows, np.int64)
        self.tpl = np.empty((len(rows), 2), np.int32)
        self.tpl[:, 0] = t[:, 0]
        self.tpl[:, 1] = (t[:, 1] & 0xFFFFFFFF).astype(np.uint32).view(np.int32)
        q = (Xi[:, None, :] + D[None, :, :]) % box
        self.nbr = look[q[..., 0], q[..., 1], q[..., 2]].astype(np.int32)
        if (self.nbr < 0).any():
            raise ValueError("a neighbourhood offset lands off the lattice")

    def template_entries(self, species, site, a=-1, b=-1, nsa=0, nsb=0):
        """Entries of the paths through `site` from the templates (host check),
        with the species of a and b replaced by nsa and nsb when given."""
        sp = np.asarray(species).copy()
        if a >= 0:
            sp[a], sp[b] = nsa, nsb
        out = []
        mult = [self.nblk, 1, self.nsp, self.nsp ** 2]
        for off, code in self.tpl:
            e = int(off)
            for p in range(4):
                v = (int(code) >> (8 * p)) & 0xFF
                if v == self.NONE:
                    continue
                st = site if v == self.SELF else int(self.nbr[site, v])
                e += int(sp[st]) * mult[p]
            out.append(e)
        return np.array(out)

    def device(self, what=("records", "inc_rec", "tpl", "nbr")):
        """Device copies (created on first use) of the per-path records, the
        per-site incidence records, the templates and the neighbourhoods."""
        if not hasattr(self, "_dev"):
            self._dev = {}
        for k in what:
            if k not in self._dev:
                self._dev[k] = N.to_dev(getattr(self, k))
        return self._dev


class SupercellMS:
    """Per-replica entry counts on the device (chimera/mslibrary.py:341-492).

    `table` (nsp * nblk, nk) per-entry spectra. `counts(species)` and
    `init`/`full` run chx_ms_counts + chx_ms_chi_of; `delta` runs
    chx_ms_delta. The sampler itself applies the deltas inside its fused step.
    """

    def __init__(self, paths: SupercellPaths, table):
        import torch
        self.paths = paths
        self.nsp, self.nblk, self.nent = paths.nsp, paths.nblk, paths.nent
        self.natoms, self.npath, self.M = paths.natoms, paths.npath, paths.M
        T = np.ascontiguousarray(table, np.float64)
        assert T.shape[0] == self.nent, f"table has {T.shape[0]} rows, need {self.nent}"
        self.T = N.to_dev(T)
        self.nk = T.shape[1]
        self.C = None
        self._torch = torch

    def set_table(self, table):
        self.T = N.to_dev(np.ascontiguousarray(table, np.float64))
        return self

    def counts(self, species):
        torch = self._torch
        sp = torch.as_tensor(species).to("cuda", torch.int32).contiguous()
        nrep = sp.shape[0]
        d = self.paths.device(("records",))
        out = torch.empty((nrep, self.nent), dtype=torch.int32, device="cuda")
        N.call("chx_ms_counts", N.ptr(sp), nrep, self.natoms, N.ptr(d["records"]), self.npath,
               self.nsp, self.nblk, N.ptr(out), N.stream())
        return out

    def chi_of(self, C):
        torch = self._torch
        C = C.to(torch.int32).contiguous()
        nrep = C.shape[0]
        chi = torch.zeros((nrep, self.nsp, self.nk), dtype=torch.float64, device="cuda")
        N.call("chx_ms_chi_of", N.ptr(C), N.ptr(self.T), nrep, self.nsp, self.nblk, self.nk,
               N.ptr(chi), N.stream())
        return chi

    def init(self, species):
        self.C = self.counts(species)
        return self.chi_of(self.C)

    def full(self, species):
        return self.chi_of(self.counts(species))

    def delta(self, species, a, b, nsa, nsb):
        torch = self._torch
        sp = torch.as_tensor(species).to("cuda", torch.int32).contiguous()
        nrep = sp.shape[0]
        d = self.paths.device(("inc_rec",))
        args = [torch.as_tensor(x).to("cuda", torch.int32).contiguous() for x in (a, b, nsa, nsb)]
        dC = torch.empty((nrep, self.nent), dtype=torch.int32, device="cuda")
        N.call("chx_ms_delta", N.ptr(sp), nrep, self.natoms, N.ptr(d["inc_rec"]), self.M,
               self.nsp, self.nblk, *[N.ptr(x) for x in args], N.ptr(dC), N.stream())
        self._dC = dC
        return self.chi_of(dC)
