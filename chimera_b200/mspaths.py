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

The reference builds classes for fcc only. The same construction runs here
on bcc and sc (integer coordinates in units of a0/2, O_h) and on hcp, in the
hexagonal integer coordinates (u, v, w) = (3 f1, 3 f2, 2 f3) under the 12
operations of the hcp site group, with A-site classes placed inverted at B
sites.

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


# hcp: integer coordinates (u, v, w) = (3 f1, 3 f2, 2 f3) of the conventional
# hexagonal cell (a1, a2 at 120 degrees, c), so A sites have u, v = 0 mod 3
# and w even, B sites (basis 1/3, 2/3, 1/2) u, v = 1, 2 mod 3 and w odd.
HCP_SCALE = np.array([3.0, 3.0, 2.0])


def hcp_gram(a0, c_over_a=None):
    """Gram matrix (A^2) of the hcp integer coordinates: |x|^2 = x G x."""
    ca = np.sqrt(8.0 / 3.0) if c_over_a is None else float(c_over_a)
    c = ca * a0
    return np.array([[a0 * a0 / 9.0, -a0 * a0 / 18.0, 0.0],
                     [-a0 * a0 / 18.0, a0 * a0 / 9.0, 0.0],
                     [0.0, 0.0, c * c / 4.0]])


def _hcp_site_type(x):
    """0 for a displacement from an A site to an A site, 1 to a B site,
    -1 for no site (x integer (..., 3))."""
    x = np.asarray(x)
    a = (x[..., 0] % 3 == 0) & (x[..., 1] % 3 == 0) & (x[..., 2] % 2 == 0)
    b = (x[..., 0] % 3 == 1) & (x[..., 1] % 3 == 2) & (x[..., 2] % 2 == 1)
    return np.where(a, 0, np.where(b, 1, -1))


def hcp_ops():
    """The 12 operations of the hcp site symmetry (D3h) in (u, v, w): the
    elements of the hexagonal holohedry D6h, generated by the 60 degree
    rotation (u, v) -> (u - v, u), the mirror (u, v) -> (v, u) and w -> -w,
    that map the environment of an A site onto itself."""
    R = np.array([[1, -1, 0], [1, 0, 0], [0, 0, 1]])
    Mx = np.array([[0, 1, 0], [1, 0, 0], [0, 0, 1]])
    Mz = np.diag([1, 1, -1])
    group = {tuple(np.eye(3, dtype=int).ravel())}
    frontier = list(group)
    while frontier:
        nxt = []
        for g in frontier:
            G = np.array(g).reshape(3, 3)
            for h in (R, Mx, Mz):
                k = tuple((h @ G).ravel())
                if k not in group:
                    group.add(k)
                    nxt.append(k)
        frontier = nxt
    g = np.array(list(itertools.product(range(-6, 7), repeat=3)))
    env = g[_hcp_site_type(g) >= 0]
    key = {tuple(x) for x in env}
    ops = []
    for k in sorted(group):
        A = np.array(k).reshape(3, 3)
        img = env @ A.T
        inside = np.all(np.abs(img) <= 6, axis=1)
        if all(tuple(x) in key for x in img[inside]) and \
                np.array_equal(_hcp_site_type(img[inside]), _hcp_site_type(env[inside])):
            ops.append(A)
    assert len(group) == 24 and len(ops) == 12, (len(group), len(ops))
    return ops


HCP_OPS = hcp_ops()


def canonical(seq, ops=None):
    """Smallest image of a path (points after the absorber) under the point
    group (O_h by default) and reversal, as a tuple of tuples."""
    ops = OPS if ops is None else ops
    s0 = np.asarray(seq, int)
    best = None
    for s in (s0, s0[::-1]):
        for A in ops:
            t = tuple(map(tuple, s @ A.T))
            if best is None or t < best:
                best = t
    return best


class PathClass:
    """One geometric class: representative, slots and directed images.

    `ops` is the point group (O_h by default) and `gram` the metric of the
    integer coordinates (None: Euclidean, lengths in units of a0/2)."""

    def __init__(self, rep, ops=None, gram=None):
        ops = OPS if ops is None else ops
        self.gram = gram
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
            for A in ops:
                t = tuple(map(tuple, s @ A.T))
                if t not in imgs:
                    imgs[t] = so.copy()
        self.images = [(np.array(k, int), v) for k, v in imgs.items()]
        self.deg = len(self.images)

    def reff_units(self):
        """Half path length, in units of a0/2 (cubic) or A (with a gram)."""
        pts = np.vstack([np.zeros((1, 3)), self.rep, np.zeros((1, 3))])
        d = np.diff(pts, axis=0)
        if self.gram is None:
            return 0.5 * float(np.linalg.norm(d, axis=1).sum())
        return 0.5 * float(np.sqrt(np.einsum("ni,ij,nj->n", d, self.gram, d)).sum())


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


def hcp_points(a0, radius, c_over_a=None):
    """Integer (u, v, w) points of the sites around an hcp A site within
    radius (A)."""
    G = hcp_gram(a0, c_over_a)
    R = int(np.ceil(2.0 * np.sqrt(3.0) * radius / a0)) + 1    # u^2 - uv + v^2 >= 3u^2/4
    W = int(np.ceil(2.0 * radius / np.sqrt(G[2, 2] * 4.0))) + 2
    g = np.array(list(itertools.product(range(-R, R + 1), range(-R, R + 1),
                                        range(-W, W + 1))))
    g = g[_hcp_site_type(g) >= 0]
    return g[np.sqrt(np.einsum("ni,ij,nj->n", g, G, g)) <= radius + 1e-9]


def length_unit(lattice, a0):
    """Length of one unit of a class's reff_units(): a0/2 on the cubic
    lattices, 1 A on hcp."""
    return 1.0 if lattice == "hcp" else a0 / 2.0


def enumerate_classes(a0, rmax_half, lattice="fcc", nleg_max=4, c_over_a=None):
    """The 3- and 4-leg path classes of a lattice to half length rmax: the
    cubic lattices in units of a0/2 under O_h; hcp (A absorbers; B absorbers
    see the inverted paths) in (u, v, w) under its 12 site operations."""
    if lattice == "hcp":
        ops, gram = HCP_OPS, hcp_gram(a0, c_over_a)
        Lmax = 2.0 * rmax_half + 1e-9
        pts = hcp_points(a0, rmax_half, c_over_a)

        def norm_of(x):
            x = np.atleast_2d(x)
            return np.sqrt(np.einsum("ni,ij,nj->n", x, gram, x))
    else:
        ops, gram = OPS, None
        unit = a0 / 2.0
        Lmax = 2.0 * rmax_half / unit + 1e-9
        pts = lattice_points(lattice, rmax_half / unit)

        def norm_of(x):
            return np.linalg.norm(np.atleast_2d(x), axis=1)
    nz = pts[np.any(pts != 0, axis=1)]
    norm = norm_of(pts)
    nzn = norm_of(nz)
    keys = set()
    if gram is None:
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
    else:
        # the same walks, leg lengths through the metric, vectorised over
        # the last point
        for q1, l1 in zip(nz, nzn):
            L3 = l1 + norm_of(nz - q1) + nzn
            for q2 in nz[(L3 <= Lmax) & np.any(nz != q1, axis=1)]:
                keys.add(canonical([q1, q2], ops))
            if nleg_max < 4:
                continue
            l12 = l1 + norm_of(pts - q1)
            for i2 in np.nonzero((l12 + norm <= Lmax) & np.any(pts != q1, axis=1))[0]:
                q2 = pts[i2]
                L4 = l12[i2] + norm_of(nz - q2) + nzn
                for q3 in nz[(L4 <= Lmax) & np.any(nz != q2, axis=1)]:
                    keys.add(canonical([q1, q2, q3], ops))
    ks = sorted(keys, key=lambda k: (len(k), PathClass(k, ops, gram).reff_units(), k))
    return [PathClass(k, ops, gram) for k in ks]


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
    """Every image of every class at every site of a periodic supercell.

    ideal (natoms, 3) and H (3, 3) of the supercell; a0 its lattice constant.
    Arrays (as mslibrary.py:357-404): p_abs, p_cls (npath), p_slot (npath, 3);
    inc (natoms, M) incident path ids padded with npath; records (npath, 4)
    and inc_rec (natoms, M, 4) for the device.

    Cubic lattices (fcc, bcc, sc) need an orthogonal box and use integer
    coordinates in units of a0/2. hcp is selected by passing its hexagonal
    conventional cell `conv` (lattice.CrystalSupercell.cell_matrix): sites
    then have integer coordinates (u, v, w), the box is periodic in them, and
    the classes (enumerated for an A absorber) are placed at A sites as they
    are and at B sites inverted, since inversion through the midpoint of an
    A-B bond maps the hcp structure onto itself with A and B exchanged.
    """

    def __init__(self, classes, ideal, H, a0, nsp, conv=None):
        self.classes = classes
        self.nsp = nsp
        self.nblk = int(sum(nsp ** c.nslot for c in classes))
        self.nent = nsp * self.nblk
        self.cls_off = class_offsets(classes, nsp)
        self.hex = conv is not None and abs(float(np.asarray(conv)[1, 0])) > 1e-12
        if self.hex:
            Ainv = np.linalg.inv(np.asarray(conv, float))
            X = (np.asarray(ideal, float) @ Ainv) * HCP_SCALE
            Xi = np.rint(X).astype(int)
            if not np.allclose(X, Xi, atol=1e-6):
                raise ValueError("supercell sites are not hcp lattice points")
            Hu = (np.asarray(H, float) @ Ainv) * HCP_SCALE
            if not np.allclose(Hu, np.diag(np.diag(Hu))):
                raise ValueError("exact multiple scattering needs a box of whole hexagonal cells")
            box = np.rint(np.diag(Hu)).astype(int)
            Xi %= box
            kind = _hcp_site_type(Xi)
            if (kind < 0).any():
                raise ValueError("supercell sites are not hcp lattice points")
            self.sign = (1 - 2 * kind).astype(int)           # +1 on A sites, -1 on B
        else:
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
            self.sign = np.ones(len(Xi), int)
        look = -np.ones(tuple(box), int)
        look[Xi[:, 0], Xi[:, 1], Xi[:, 2]] = np.arange(len(Xi))
        n = self.natoms = len(Xi)
        sgn = self.sign[:, None, None]
        P_abs, P_cls, P_slot = [], [], []
        for g, cl in enumerate(classes):
            small = (np.any(2 * np.abs(cl.rep).max(0) >= box) if self.hex
                     else 2 * np.abs(cl.rep).max() >= box.min())
            if small:
                raise ValueError("supercell too small for the paths")
            for img, so in cl.images:
                p = (Xi[:, None, :] + sgn * img[None]) % box
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
                    # hcp: a site at an A->B position of an A-absorber image
                    # is a B site, and the same paths seen from a B site are
                    # the inverted ones; B sites read their neighbourhood
                    # table at the inverted offsets, so the row stores the
                    # offsets inverted and serves both sublattices.
                    flip = -1 if (self.hex and _hcp_site_type(np.array(pos[r])) == 1) else 1
                    code = 0
                    for p in range(4):
                        if p == r:
                            v = self.SELF
                        elif pos[p] is None:
                            v = self.NONE
                        else:
                            d = tuple(flip * int(x) for x in np.subtract(pos[p], pos[r]))
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
        q = (Xi[:, None, :] + self.sign[:, None, None] * D[None, :, :]) % box
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
                a = getattr(self, k)
                if k == "tpl":
                    a = self.device_templates()
                self._dev[k] = N.to_dev(np.ascontiguousarray(a))
        return self._dev

    def tpl_order(self):
        """Device order of the templates: the classes interleaved (the i-th
        template of every class, then the (i+1)-th ...), so that the lanes of
        a warp, which take consecutive templates, resolve them to different
        MS entries and their shared-memory count updates rarely collide. The
        counts are integer sums, so the order does not change them."""
        off = self.tpl[:, 0].astype(np.int64)
        first = np.r_[True, off[1:] != off[:-1]]
        start = np.maximum.accumulate(np.where(first, np.arange(len(off)), 0))
        rank = np.arange(len(off)) - start
        return np.lexsort((off, rank))

    def device_templates(self):
        """The templates as the sampler step reads them: in tpl_order, with
        the position bytes SELF and NONE replaced by D and D + 1, the two
        slots the step appends to each site's neighbourhood (the site itself
        and a zero), so that every position is a plain table index."""
        if self.D + 1 >= self.SELF:
            raise ValueError(f"{self.D} neighbourhood sites leave no room for the extra slots")
        t = np.ascontiguousarray(self.tpl[self.tpl_order()])
        pos = np.ascontiguousarray(t[:, 1]).view(np.uint8).reshape(-1, 4)  # position p: byte p
        pos[pos == self.SELF] = self.D
        pos[pos == self.NONE] = self.D + 1
        t[:, 1] = pos.reshape(-1).view(np.int32)
        return t


def _host_array(x):
    """NumPy copy of a host or device array (a torch tensor, or an object
    with a `get()` or `cpu()` method)."""
    if hasattr(x, "detach"):
        return x.detach().cpu().numpy()
    if hasattr(x, "get"):
        return np.asarray(x.get())
    return np.asarray(x)


class SupercellMS:
    """Per-replica entry counts on the device (chimera/mslibrary.py:341-492).

    `table` (nsp * nblk, nk) per-entry spectra. `counts(species)` and
    `init`/`full` run chx_ms_counts + chx_ms_chi_of; `delta` runs
    chx_ms_delta. The sampler itself applies the deltas inside its fused step.
    """

    def __init__(self, paths, table=None):
        """SupercellMS(SupercellPaths, table), or the reference's own call
        SupercellMS(lib, S) (chimera/mslibrary.py:351-404): lib a path library
        (its classes, species count and `table`), S the spectrum whose
        reference supercell (a0_ref, ideal0, H0) the paths are laid on; the
        table then comes from set_params, as in the reference."""
        import torch
        self.lib = None
        if not isinstance(paths, SupercellPaths):
            lib, S = paths, table
            paths = SupercellPaths(list(lib.classes), S.ideal0, S.H0, float(S.a0_ref),
                                   int(lib.nsp))
            self.lib, table = lib, None
        self.paths = paths
        self.nsp, self.nblk, self.nent = paths.nsp, paths.nblk, paths.nent
        self.natoms, self.npath, self.M = paths.natoms, paths.npath, paths.M
        self.T, self.nk = None, None
        if table is not None:
            self.set_table(table)
        self.C = None
        self._dC = None
        self._torch = torch

    @classmethod
    def adopt(cls, ms, cell):
        """This class for an MS object built elsewhere: the reference's own
        SupercellMS (it carries its library `lib` and device table `T` but no
        paths of this package), laid on `cell` (ideal, H, a0: the forward
        model's supercell); objects of this class are returned as they are."""
        if ms is None or isinstance(ms, cls):
            return ms
        lib = getattr(ms, "lib", None)
        if lib is None or getattr(ms, "T", None) is None:
            raise TypeError("an MS library needs its path library (lib) and table (T)")
        paths = SupercellPaths(list(lib.classes), np.asarray(cell.ideal), np.asarray(cell.H),
                               float(cell.a0), int(lib.nsp))
        out = cls(paths, _host_array(ms.T))
        out.lib = lib
        return out

    def set_table(self, table):
        T = np.ascontiguousarray(table, np.float64)
        if T.shape[0] != self.nent:
            raise ValueError(f"table has {T.shape[0]} rows, need {self.nent}")
        self.T = N.to_dev(T)
        self.nk = T.shape[1]
        return self

    def set_params(self, sigma2_nn, r_nn, c_ms=1.3, amp=1.0, s02=1.0, a_scale=1.0):
        """The library's table at these parameters (mslibrary.py:406-408)."""
        if self.lib is None:
            raise ValueError("set_params needs the path library (SupercellMS(lib, S))")
        return self.set_table(_host_array(self.lib.table(sigma2_nn, r_nn, c_ms, amp, s02,
                                                         a_scale)))

    def expected_chi(self, composition=None):
        """Random-alloy chi_MS per absorbing atom (nsp, nk), NumPy
        (mslibrary.py:410-413)."""
        return self.lib.chi_counts(self.lib.expected_counts(composition), _host_array(self.T))

    def commit(self, acc):
        """Apply the last delta where accepted (mslibrary.py:488-489)."""
        torch = self._torch
        a = torch.as_tensor(acc).to("cuda").to(self.C.dtype)
        self.C = self.C + self._dC * a[:, None]

    def permute(self, ix):
        """Follow a replica exchange (mslibrary.py:491-492)."""
        self.C = self.C[self._torch.as_tensor(ix).to("cuda").long()]

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
