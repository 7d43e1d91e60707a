"""Supercell topology: sites, neighbour lists, shells, Warren-Cowley.

The outputs are bit-identical to the reference's exafs_gpu/lattice.py
(CrystalSupercell :214-295, warren_cowley :167-185) and the shell index of
chimera/model.py:199-201, but the neighbour search is O(N * candidates)
instead of O(N^2 * 27): for each site only the sites in the surrounding cells
that can lie within rmax are examined, with the reference's own arithmetic
(27-image minimum image, first minimum on ties, the same FP64 expressions)
applied to them, so every kept pair, shift and distance comes out the same.
That makes 32,000-atom cells practical.
"""
from __future__ import annotations

import numpy as np

KB = 8.617333262e-5

# Bravais basis in fractional coordinates of the conventional cell; every site
# equivalent (uniform coordination), as the reference requires (lattice.py:205-211)
LATTICES = {
    "sc": dict(basis=[[0, 0, 0]], hex=False),
    "bcc": dict(basis=[[0, 0, 0], [.5, .5, .5]], hex=False),
    "fcc": dict(basis=[[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]], hex=False),
    "hcp": dict(basis=[[0, 0, 0], [1 / 3, 2 / 3, .5]], hex=True),
}


class CrystalSupercell:
    """Periodic supercell of a Bravais lattice + equivalent basis.

    Same attributes as the reference class: lattice, ncell, a0, cell_matrix,
    H (rows = supercell vectors), ideal (natoms, 3), frac, natoms, box.
    """

    def __init__(self, lattice="fcc", ncell=(5, 5, 5), a0=3.56, c_over_a=None):
        if lattice not in LATTICES:
            raise ValueError(f"unknown lattice {lattice!r}; have {list(LATTICES)}")
        spec = LATTICES[lattice]
        self.lattice = lattice
        self.ncell = tuple(int(n) for n in ncell)
        self.a0 = float(a0)
        if spec["hex"]:
            ca = c_over_a if c_over_a is not None else np.sqrt(8.0 / 3.0)
            A = np.array([[1.0, 0.0, 0.0], [-0.5, np.sqrt(3) / 2, 0.0], [0.0, 0.0, ca]]) * a0
        else:
            A = np.eye(3) * a0
        self.cell_matrix = A
        self.H = np.diag(self.ncell).astype(float) @ A
        self.basis = np.asarray(spec["basis"], float)
        nx, ny, nz = self.ncell
        cells = np.array([(i, j, k) for i in range(nx) for j in range(ny) for k in range(nz)],
                         float)
        frac_conv = (cells[:, None, :] + self.basis[None, :, :]).reshape(-1, 3)
        self.ideal = np.ascontiguousarray(frac_conv @ A)
        self.frac = frac_conv / np.array(self.ncell, float)
        self.natoms = self.ideal.shape[0]
        self.box = np.diag(self.H).copy()
        self._images = np.array([(i, j, k) for i in (-1, 0, 1) for j in (-1, 0, 1)
                                 for k in (-1, 0, 1)], float) @ self.H

    # ------------------------------------------------------------ candidates
    def _cell_reach(self, rmax):
        """Cell offsets along each axis that can hold a site within rmax."""
        A = self.cell_matrix
        vol = abs(np.linalg.det(A))
        out = []
        for ax in range(3):
            other = [A[(ax + 1) % 3], A[(ax + 2) % 3]]
            height = vol / np.linalg.norm(np.cross(other[0], other[1]))
            out.append(int(np.ceil(rmax / height)) + 1)
        return out

    def _candidates(self, rmax):
        """(natoms, ncand) site indices, ascending per row, that include every
        site within rmax of each site under the minimum image."""
        nx, ny, nz = self.ncell
        nb = self.basis.shape[0]
        reach = self._cell_reach(rmax)
        axes = []
        for n, r in zip(self.ncell, reach):
            axes.append(np.arange(n) if 2 * r + 1 >= n else np.arange(-r, r + 1))
        off = np.array(np.meshgrid(*axes, indexing="ij")).reshape(3, -1).T   # (noff, 3)
        site = np.arange(self.natoms)
        cell = site // nb
        ci = np.stack([cell // (ny * nz), (cell // nz) % ny, cell % nz], axis=1)
        cand_cells = (ci[:, None, :] + off[None, :, :]) % np.array(self.ncell)
        flat = (cand_cells[..., 0] * ny + cand_cells[..., 1]) * nz + cand_cells[..., 2]
        cand = (flat[:, :, None] * nb + np.arange(nb)[None, None, :]).reshape(self.natoms, -1)
        cand = np.sort(cand, axis=1)
        # wrapped offsets can repeat a cell only when an axis is fully covered,
        # which the arange(n) branch already handles without repetition
        return cand

    def _heights(self):
        """Supercell heights: the distance between opposite faces, per axis."""
        H = self.H
        vol = abs(np.linalg.det(H))
        return np.array([vol / np.linalg.norm(np.cross(H[(a + 1) % 3], H[(a + 2) % 3]))
                         for a in range(3)])

    def _offset_images(self, rmax):
        """(natoms, ncand) candidates with the 27-image index of each
        candidate's unwrapped cell, j ascending per row, or None when the
        supercell is too small for the shortcut.

        When every supercell height exceeds 2 rmax, a pair within rmax has
        exactly one image within rmax, and that image is the one its
        candidate cell offset names (the offset does not wrap twice, since
        2 reach + 1 < ncell on every axis). The 27-image argmin of the
        reference then picks the same image for every kept pair, so it can be
        read off the offset instead of searched."""
        reach = self._cell_reach(rmax)
        if np.any(self._heights() <= 2.0 * rmax + 1e-9):
            return None
        if any(2 * r + 1 >= n for n, r in zip(self.ncell, reach)):
            return None
        nx, ny, nz = self.ncell
        nb = self.basis.shape[0]
        off = np.array(np.meshgrid(*[np.arange(-r, r + 1) for r in reach],
                                   indexing="ij")).reshape(3, -1).T
        cell = np.arange(self.natoms) // nb
        ci = np.stack([cell // (ny * nz), (cell // nz) % ny, cell % nz], axis=1)
        raw = ci[:, None, :] + off[None, :, :]                   # unwrapped cell
        n = np.array(self.ncell)
        wrap = np.floor_divide(raw, n)                           # -1, 0 or 1 per axis
        cc = raw - wrap * n
        flat = (cc[..., 0] * ny + cc[..., 1]) * nz + cc[..., 2]
        cand = (flat[:, :, None] * nb + np.arange(nb)[None, None, :]).reshape(self.natoms, -1)
        img = ((wrap[..., 0] + 1) * 9 + (wrap[..., 1] + 1) * 3 + (wrap[..., 2] + 1))
        img = np.repeat(img, nb, axis=1)
        order = np.argsort(cand, axis=1, kind="stable")
        return (np.take_along_axis(cand, order, 1), np.take_along_axis(img, order, 1))

    def min_image(self, d):
        """Exact minimum image by explicit search over the 27 nearest images."""
        d = np.atleast_2d(d)
        cand = d[:, None, :] + self._images[None, :, :]
        n2 = (cand ** 2).sum(-1)
        return cand[np.arange(d.shape[0]), n2.argmin(1)]

    def neighbour_list(self, rmax, batch=64):
        """(i_idx, j_idx, shift, off): i-major, j ascending, as the reference."""
        pos = self.ideal
        n = self.natoms
        imgs = self._images
        fast = self._offset_images(rmax)
        if fast is not None:
            return self._neighbour_list_offsets(rmax, *fast)
        cand = self._candidates(rmax)
        I, J, SH = [], [], []
        for s0 in range(0, n, batch):
            rows = np.arange(s0, min(n, s0 + batch))
            cj = cand[rows]                                        # (b, m)
            d0 = pos[cj] - pos[rows][:, None, :]                   # (b, m, 3)
            c = d0[:, :, None, :] + imgs[None, None, :, :]         # (b, m, 27, 3)
            n2 = (c ** 2).sum(-1)
            best = n2.argmin(-1)                                   # (b, m)
            d = np.take_along_axis(c, best[..., None, None], axis=2)[:, :, 0, :]
            r = np.linalg.norm(d.reshape(-1, 3), axis=1).reshape(d.shape[:2])
            keep = (r <= rmax) & (r > 1e-6)
            for q in range(rows.size):
                sel = np.nonzero(keep[q])[0]
                I.append(np.full(sel.size, rows[q]))
                J.append(cj[q, sel])
                SH.append(imgs[best[q, sel]])
        i_idx = np.concatenate(I).astype(np.int32)
        j_idx = np.concatenate(J).astype(np.int32)
        shift = np.ascontiguousarray(np.concatenate(SH), np.float64)
        counts = np.bincount(i_idx, minlength=n)
        off = np.zeros(n + 1, np.int32)
        off[1:] = np.cumsum(counts)
        return i_idx, j_idx, shift, off

    def _neighbour_list_offsets(self, rmax, cand, img, batch=2048):
        """neighbour_list when the image of each candidate is known: the same
        expressions (d0 + image, its norm, the rmax test) on one image per
        candidate instead of 27."""
        pos, n, imgs = self.ideal, self.natoms, self._images
        I, J, SH = [], [], []
        for s0 in range(0, n, batch):
            rows = np.arange(s0, min(n, s0 + batch))
            cj, ik = cand[rows], img[rows]
            d0 = pos[cj] - pos[rows][:, None, :]
            d = d0 + imgs[ik]
            r = np.linalg.norm(d.reshape(-1, 3), axis=1).reshape(d.shape[:2])
            keep = (r <= rmax) & (r > 1e-6)
            q, c = np.nonzero(keep)                               # row-major: j ascending
            I.append(rows[q])
            J.append(cj[q, c])
            SH.append(imgs[ik[q, c]])
        i_idx = np.concatenate(I).astype(np.int32)
        j_idx = np.concatenate(J).astype(np.int32)
        shift = np.ascontiguousarray(np.concatenate(SH), np.float64)
        counts = np.bincount(i_idx, minlength=n)
        off = np.zeros(n + 1, np.int32)
        off[1:] = np.cumsum(counts)
        return i_idx, j_idx, shift, off

    def shell_radii(self, rmax):
        d = self.min_image(self.ideal - self.ideal[0])
        r = np.linalg.norm(d, axis=1)
        r = r[(r > 1e-6) & (r <= rmax)]
        vals, cnt = np.unique(np.round(r, 3), return_counts=True)
        return vals, cnt

    def nn_distance(self):
        v, _ = self.shell_radii(self.a0 * 1.5)
        return float(v[0])


def shell_index(cell, i_idx, j_idx, shift):
    """Coordination-shell index of every pair and the exact pair distances,
    as chimera/model.py:199-201 defines them (radii rounded to 1e-3 A)."""
    d0 = np.linalg.norm((cell.ideal[j_idx] + shift) - cell.ideal[i_idx], axis=1)
    _, sh = np.unique(np.round(d0, 3), return_inverse=True)
    return sh.astype(np.int32), d0


def build_reverse_index(i_idx, j_idx, natoms):
    """rev[p] = index of the pair (j, i) given p = (i, j)
    (methods/method_a_rmc.py:51-60)."""
    key = i_idx.astype(np.int64) * natoms + j_idx
    rkey = j_idx.astype(np.int64) * natoms + i_idx
    order = np.argsort(key, kind="stable")
    at = np.searchsorted(key[order], rkey)
    rev = order[np.clip(at, 0, key.size - 1)]
    if not (np.array_equal(i_idx[rev], j_idx) and np.array_equal(j_idx[rev], i_idx)):
        raise ValueError("neighbour list is not symmetric")
    return rev.astype(np.int32)


def pair_vectors(cell, pos, i_idx, j_idx, shift):
    return (pos[j_idx] + shift) - pos[i_idx]


def warren_cowley(species, i_idx, j_idx, shift, cell, shell_r, tol=0.15, comp=None, nsp=None):
    """alpha_AB = 1 - P(B|A)/c_B over the pairs within tol of shell_r
    (exafs_gpu/lattice.py:167-185)."""
    NSP = int(nsp) if nsp is not None else int(species.max()) + 1
    d = pair_vectors(cell, cell.ideal, i_idx, j_idx, shift)
    r = np.linalg.norm(d, axis=1)
    m = np.abs(r - shell_r) < tol
    a, b = species[i_idx[m]], species[j_idx[m]]
    c = comp if comp is not None else np.bincount(species, minlength=NSP) / species.size
    # pair counts by (A, B) in one pass, then the same ratios
    cnt = np.bincount(a * NSP + b, minlength=NSP * NSP).reshape(NSP, NSP)
    tot = cnt.sum(1)
    alpha = np.zeros((NSP, NSP))
    for A in range(NSP):
        if tot[A] == 0:
            continue
        for B in range(NSP):
            P = cnt[A, B] / tot[A]
            alpha[A, B] = 1.0 - P / c[B]
    return alpha


def integer_counts(composition, natoms):
    """Species counts summing to natoms, the last species taking the
    remainder (chimera/system.py:83-90)."""
    comp = np.asarray(composition, float)
    comp = comp / comp.sum()
    cnt = np.round(comp * natoms).astype(int)
    cnt[-1] = natoms - cnt[:-1].sum()
    return cnt


def random_config(natoms, composition, seed=0):
    """A random arrangement at the composition (chimera/model.py:451-459)."""
    cnt = integer_counts(composition, natoms)
    sp = np.repeat(np.arange(len(cnt)), cnt).astype(np.int32)
    np.random.default_rng(seed).shuffle(sp)
    return sp


class Topology:
    """Everything the device kernels need about one supercell, built once:
    neighbour list (uniform coordination, i-major), reverse index, shells,
    ideal shell radii and the pair-table flag."""

    def __init__(self, cell, rmax, sigma2=None):
        self.cell = cell
        self.rmax = float(rmax)
        self.i, self.j, self.shift, self.off = cell.neighbour_list(rmax)
        self.natoms = cell.natoms
        self.npairs = int(self.i.size)
        z = np.bincount(self.i, minlength=self.natoms)
        if z.min() != z.max():
            raise ValueError("expected uniform coordination")
        self.ncoord = int(z[0])
        self.rev = build_reverse_index(self.i, self.j, self.natoms)
        self.shell, self.d0 = shell_index(cell, self.i, self.j, self.shift)
        self.nshell = int(self.shell.max()) + 1
        self.sigma2 = (np.zeros(self.npairs) if sigma2 is None
                       else np.broadcast_to(np.asarray(sigma2, float), (self.npairs,)).copy())
        # representative (first) pair of every shell; a pair may use the
        # shell's tabulated term when its ideal distance and sigma^2 match it
        first = np.array([np.argmax(self.shell == s) for s in range(self.nshell)])
        self.r_shell = self.d0[first]
        self.s2_shell = self.sigma2[first]
        self.pair_tab = ((np.abs(self.d0 - self.r_shell[self.shell]) <= 1e-12 * self.r_shell[self.shell])
                         & (self.sigma2 == self.s2_shell[self.shell])).astype(np.uint8)
        self.shells = np.array([self.d0[self.shell == s].mean() for s in range(self.nshell)])
