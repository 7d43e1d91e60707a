"""The swap surrogate on the CPU (test infrastructure: the checker of the
library's surrogate kernels and of its delayed acceptance). This component
has no counterpart in the reference; what it restates is the library's own
specification of it:

  swap_codes     the features of a swap (pair row, neighbour codes, sigma)
  bf16           round-to-nearest-even to BF16, as __float2bfloat16_rn
  forward        BF16 weights, activations rounded to BF16 between layers,
                 sums in FP64 here (FP32 on the device)
  backward       gradient of mean (y - t)^2 with the device's rounding points
                 (dZ rounded to BF16 before every product)
  da_decision    the two-stage delayed-acceptance test (Christen & Fox 2005,
                 J. Comput. Graph. Stat. 14:795) as the step kernel applies it

Parameter layout: W1 (nin+1, H) | b1 | W2 (H, H) | b2 | W3 (H, H) | b3 | w4 (H) |
b4 (1), row-major [in][out], nin = nsp(nsp-1)/2 + 2 D (nsp+1) + nchain.
"""
from __future__ import annotations

import numpy as np


def nin_of(nsp, D, nchain=0):
    return nsp * (nsp - 1) // 2 + 2 * D * (nsp + 1) + nchain


def unpack(theta, nsp, D, H, nchain=0):
    nin = nin_of(nsp, D, nchain)
    th = np.asarray(theta)
    th = th if th.dtype == np.float64 else th.astype(np.float32)   # float64 for FD checks
    o = 0

    def take(n, shape):
        nonlocal o
        a = th[o:o + n].reshape(shape)
        o += n
        return a
    W1 = take((nin + 1) * H, (nin + 1, H))
    b1 = take(H, (H,))
    W2 = take(H * H, (H, H))
    b2 = take(H, (H,))
    W3 = take(H * H, (H, H))
    b3 = take(H, (H,))
    w4 = take(H, (H,))
    b4 = take(1, (1,))
    assert o == th.size
    return dict(W1=W1, b1=b1, W2=W2, b2=b2, W3=W3, b3=b3, w4=w4, b4=b4)


def pack(p):
    return np.concatenate([p[k].reshape(-1) for k in ("W1", "b1", "W2", "b2", "W3", "b3", "w4",
                                                      "b4")])


def bf16(x):
    """Nearest BF16 value (ties to even) of float32 x, as float32."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


def swap_codes(species, a, b, nbr, nsp):
    """Features of a swap of sites a and b: (codes (1 + 2D,) uint8, sigma).
    codes[0] is the row of the unordered species pair, codes[1 + k] the
    species of neighbour k (the D neighbours of lo = min(a, b), then of hi) or
    nsp where that neighbour is a or b; sigma = +1 if S[lo] < S[hi] else -1."""
    lo, hi = min(a, b), max(a, b)
    p, q = int(species[lo]), int(species[hi])
    assert p != q, "a swap exchanges two different species"
    D = nbr.shape[1]
    codes = np.empty(1 + 2 * D, np.uint8)
    x, y = min(p, q), max(p, q)
    codes[0] = x * nsp - x * (x + 1) // 2 + (y - x - 1)
    for k in range(2 * D):
        site = int(nbr[hi if k >= D else lo, k % D])
        codes[1 + k] = nsp if site in (a, b) else int(species[site])
    return codes, (1.0 if p < q else -1.0)


def rows_of(codes, nsp, chain=None):
    """One-hot row indices of W1 for a batch of codes: (B, 1 + 2D), plus the
    chain's row (B, 2 + 2D) when chain is given."""
    codes = np.asarray(codes, np.int64)
    npt = nsp * (nsp - 1) // 2
    k = np.arange(codes.shape[1] - 1)
    r = np.empty_like(codes)
    r[:, 0] = codes[:, 0]
    r[:, 1:] = npt + k[None, :] * (nsp + 1) + codes[:, 1:]
    if chain is not None:
        r = np.concatenate([r, npt + k.size * (nsp + 1) + np.asarray(chain, np.int64)[:, None]], 1)
    return r


def forward(theta, codes, lnbeta, nsp, D, H, feat_shift=0.0, feat_scale=1.0, rounding=True,
            chain=None, nchain=0):
    """Network output (B,) and the cache backward needs. rounding=False drops
    every BF16 rounding (the exact function, for finite-difference checks);
    chain (B,) adds each sample's chain row (nchain rows in the layout)."""
    p = unpack(theta, nsp, D, H, nchain)
    rnd = (lambda x: bf16(x)) if rounding else (lambda x: np.asarray(x))
    W1, W2, W3, w4 = (np.asarray(rnd(p[k]), np.float64) for k in ("W1", "W2", "W3", "w4"))
    rows = rows_of(codes, nsp, chain)
    f = ((np.asarray(lnbeta, np.float32) - np.float32(feat_shift)) *
         np.float32(feat_scale)).astype(np.float64)
    nin = nin_of(nsp, D, nchain)
    Z1 = W1[rows].sum(1) + f[:, None] * W1[nin][None, :] + p["b1"][None, :]
    act = ((lambda z: bf16(np.maximum(z, 0).astype(np.float32)).astype(np.float64)) if rounding
           else (lambda z: np.maximum(z, 0)))
    H1 = act(Z1)
    Z2 = H1 @ W2 + p["b2"][None, :]
    H2 = act(Z2)
    Z3 = H2 @ W3 + p["b3"][None, :]
    H3 = act(Z3)
    y = H3 @ w4 + float(p["b4"][0])
    cache = dict(rows=rows, f=f, Z1=Z1, Z2=Z2, Z3=Z3, H1=H1, H2=H2, H3=H3, W2=W2, W3=W3, w4=w4,
                 nin=nin, rounding=rounding)
    return y, cache


def backward(theta, cache, y, target, nsp, D, H):
    """(loss, grad) of mean (y - target)^2, grad in the parameter layout."""
    c = cache
    B = y.shape[0]
    t = np.asarray(target, np.float64)
    loss = float(((y - t) ** 2).mean())
    dy = 2.0 * (y - t) / B
    g = {}
    g["b4"] = np.array([dy.sum()])
    g["w4"] = c["H3"].T @ dy

    def r16(x):
        return bf16(x.astype(np.float32)).astype(np.float64) if c["rounding"] else x
    dZ3 = r16(np.where(c["Z3"] > 0, dy[:, None] * c["w4"][None, :], 0.0))
    g["W3"] = c["H2"].T @ dZ3
    g["b3"] = dZ3.sum(0)
    dZ2 = r16(np.where(c["Z2"] > 0, dZ3 @ c["W3"].T, 0.0))
    g["W2"] = c["H1"].T @ dZ2
    g["b2"] = dZ2.sum(0)
    dZ1 = r16(np.where(c["Z1"] > 0, dZ2 @ c["W2"].T, 0.0))
    g["b1"] = dZ1.sum(0)
    gW1 = np.zeros((c["nin"] + 1, H))
    np.add.at(gW1, c["rows"].reshape(-1), np.repeat(dZ1, c["rows"].shape[1], axis=0))
    gW1[c["nin"]] = c["f"] @ dZ1
    g["W1"] = gW1
    return loss, pack({k: np.asarray(v, np.float64) for k, v in g.items()})


def da_probs(beta, nfit, d, dhat, de, energy_beta):
    """Stage probabilities of the step kernel's delayed-acceptance test of one
    swap: stage 1 min(1, exp(-x1)), x1 = beta nfit d^ + energy_beta de;
    stage 2 min(1, exp(-x2)), x2 = beta nfit (d - d^)."""
    x1 = beta * nfit * dhat + energy_beta * de
    x2 = beta * nfit * (d - dhat)
    return min(1.0, float(np.exp(-min(x1, 60.0)))), min(1.0, float(np.exp(-min(x2, 60.0))))


def da_decision(beta, nfit, d, dhat, de, energy_beta, u1, u2):
    """The same test with uniforms u1 (stage 1) and u2 (stage 2): a stage
    passes when x <= 0 or u < exp(-min(x, 60)). Returns (passed stage 1,
    accepted)."""
    x1 = beta * nfit * dhat + energy_beta * de
    s1 = x1 <= 0.0 or u1 < np.exp(-min(x1, 60.0))
    if not s1:
        return False, False
    x2 = beta * nfit * (d - dhat)
    return True, bool(x2 <= 0.0 or u2 < np.exp(-min(x2, 60.0)))
