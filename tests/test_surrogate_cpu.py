"""The swap surrogate's oracle and the delayed-acceptance rule, on the CPU."""
import itertools

import numpy as np
import pytest

from conftest import golden
from oracle import mlp as OM


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.normal(0, 1, 4000), rng.normal(0, 1e-30, 100),
                        rng.normal(0, 1e30, 100)]).astype(np.float32)
    want = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(OM.bf16(x), want)
    # ties go to the even mantissa
    assert OM.bf16(np.float32(1 + 2 ** -8)) == np.float32(1.0)
    assert OM.bf16(np.float32(1 + 3 * 2 ** -8)) == np.float32(1 + 2 ** -6)


def _rand_problem(nsp=2, D=4, H=16, B=8, seed=0, nchain=0):
    rng = np.random.default_rng(seed)
    nin = OM.nin_of(nsp, D, nchain)
    npt = nsp * (nsp - 1) // 2
    theta = rng.normal(0, 0.3, (nin + 1) * H + 3 * H + 2 * H * H + H + 1).astype(np.float32)
    codes = np.concatenate([rng.integers(0, npt, (B, 1)), rng.integers(0, nsp + 1, (B, 2 * D))],
                           1).astype(np.uint8)
    lnb = rng.normal(0, 1, B).astype(np.float32)
    t = rng.normal(0, 1, B)
    return theta, codes, lnb, t


@pytest.mark.parametrize("nchain", [0, 5])
def test_oracle_backward_matches_finite_differences(nchain):
    """Without BF16 rounding the oracle's gradient is the exact derivative."""
    nsp, D, H = 3, 3, 12
    theta, codes, lnb, t = _rand_problem(nsp, D, H, B=6, seed=2, nchain=nchain)
    chain = np.array([0, 3, 3, 1, 4, 0]) if nchain else None
    theta = theta.astype(np.float64)
    kw = dict(rounding=False, chain=chain, nchain=nchain)
    y, cache = OM.forward(theta, codes, lnb, nsp, D, H, 0.1, 0.7, **kw)
    loss, g = OM.backward(theta, cache, y, t, nsp, D, H)

    def f(th):
        yy, _ = OM.forward(th, codes, lnb, nsp, D, H, 0.1, 0.7, **kw)
        return ((yy - t) ** 2).mean()
    rng = np.random.default_rng(3)
    idx = rng.choice(theta.size, 60, replace=False)
    # every row of W1 a sample uses, plus random entries
    rows = OM.rows_of(codes, nsp, chain)[0]
    idx = np.concatenate([idx, rows * H, [OM.nin_of(nsp, D, nchain) * H + 1]])
    for q in idx:
        e = np.zeros_like(theta)
        e[q] = 1e-6
        fd = (f(theta + e) - f(theta - e)) / 2e-6
        assert abs(fd - g[q]) <= 1e-6 + 1e-5 * abs(fd), q


def test_oracle_loss_and_rounding_points():
    nsp, D, H = 2, 4, 16
    theta, codes, lnb, t = _rand_problem(nsp, D, H)
    y, cache = OM.forward(theta, codes, lnb, nsp, D, H)
    loss, g = OM.backward(theta, cache, y, t, nsp, D, H)
    assert np.isclose(loss, ((y - t) ** 2).mean())
    for k in ("H1", "H2", "H3"):   # activations are BF16 values
        a = cache[k].astype(np.float32)
        assert np.array_equal(OM.bf16(a), a)
    assert g.size == theta.size


def _fcc():
    d = golden("rmc_trace.npz")
    return d["ideal"], d["i"], d["j"], d["shift"], int(np.bincount(d["i"])[0])


def test_feature_neighbours_share_one_order():
    from chimera_b200.surrogate import feature_neighbours
    ideal, i, j, shift, z = _fcc()
    nbr = feature_neighbours(ideal, i, j, shift, z)
    natoms = ideal.shape[0]
    pos_of = {}
    for p in range(i.size):
        pos_of[(int(i[p]), int(j[p]))] = ideal[j[p]] + shift[p] - ideal[i[p]]
    disp = np.array([[pos_of[(s, int(nbr[s, k]))] for k in range(z)] for s in range(natoms)])
    assert np.allclose(disp, disp[:1], atol=1e-9)
    assert all(len(set(r)) == z for r in nbr.tolist())


def test_swap_features_are_the_same_for_a_swap_and_its_reverse():
    from chimera_b200.surrogate import feature_neighbours
    ideal, i, j, shift, z = _fcc()
    nbr = feature_neighbours(ideal, i, j, shift, z)
    rng = np.random.default_rng(5)
    nsp = 3
    S = rng.integers(0, nsp, ideal.shape[0])
    n = 0
    for _ in range(200):
        a, b = rng.choice(ideal.shape[0], 2, replace=False)
        if S[a] == S[b]:
            continue
        c1, s1 = OM.swap_codes(S, a, b, nbr, nsp)
        T = S.copy()
        T[a], T[b] = S[b], S[a]
        c2, s2 = OM.swap_codes(T, b, a, nbr, nsp)
        assert np.array_equal(c1, c2) and s1 == -s2
        assert c1[0] < nsp * (nsp - 1) // 2 and c1[1:].max() <= nsp
        n += 1
        if b in nbr[a]:        # a neighbouring pair codes the partner as nsp
            assert (c1[1:] == nsp).sum() >= 2
    assert n > 50


# ---------------------------------------------------------------------------
# delayed acceptance on a state space small enough to enumerate: 4 + 4 atoms
# on a ring of 8 sites, uniform proposal of an ordered pair of sites
def _toy(antisymmetric=True, seed=0):
    rng = np.random.default_rng(seed)
    n = 8
    states = [s for s in itertools.product((0, 1), repeat=n) if sum(s) == 4]
    index = {s: q for q, s in enumerate(states)}
    w, v, e = rng.normal(0, 1, n), rng.normal(0, 1, n), rng.normal(0, 1, n)

    def chi(s):
        return sum(w[i] * s[i] * s[(i + 1) % n] for i in range(n)) + float(np.dot(v, s))

    def ene(s):
        return sum(e[i] * s[i] * s[(i + 2) % n] for i in range(n))
    beta_nfit, eb = 1.3, 0.8
    logp = np.array([-beta_nfit * chi(s) - eb * ene(s) for s in states])
    pi = np.exp(logp - logp.max())
    pi /= pi.sum()

    def screen(s, lo, hi):
        # any function of the pair and of the other sites, times the sign
        rest = tuple(2 if q in (lo, hi) else s[q] for q in range(n))
        h = np.random.default_rng(abs(hash((lo, hi, rest))) % (2 ** 32)).normal(0, 1.5)
        sigma = 1.0 if s[lo] < s[hi] else -1.0
        return sigma * h if antisymmetric else h + 0.4 * s[lo]

    P = np.zeros((len(states), len(states)))
    for x, s in enumerate(states):
        for lo, hi in itertools.combinations(range(n), 2):
            if s[lo] == s[hi]:
                continue
            t = list(s)
            t[lo], t[hi] = t[hi], t[lo]
            t = tuple(t)
            p1, p2 = OM.da_probs(1.0, beta_nfit, chi(t) - chi(s), screen(s, lo, hi) / beta_nfit,
                                 ene(t) - ene(s), eb)
            P[x, index[t]] += (2.0 / (n * (n - 1))) * p1 * p2
        P[x, x] = 1.0 - P[x].sum()
    return pi, P


def test_delayed_acceptance_keeps_the_target_distribution():
    pi, P = _toy(antisymmetric=True)
    flow = pi[:, None] * P
    assert np.abs(flow - flow.T).max() <= 1e-14
    assert np.abs(pi @ P - pi).max() <= 1e-14


def test_delayed_acceptance_needs_the_antisymmetric_screen():
    """The oracle toy with a screen that is not odd under reversal breaks
    detailed balance: the sign construction is what makes the rule exact."""
    pi, P = _toy(antisymmetric=False)
    flow = pi[:, None] * P
    assert np.abs(flow - flow.T).max() > 1e-4


def test_zero_screen_is_the_plain_rule():
    rng = np.random.default_rng(9)
    for _ in range(2000):
        beta, nfit, d = rng.uniform(0.1, 5), rng.uniform(10, 500), rng.normal(0, 0.01)
        u = rng.random()
        s1, acc = OM.da_decision(beta, nfit, d, 0.0, 0.0, 0.0, rng.random(), u)
        x = beta * d * nfit
        assert s1 and acc == bool(x <= 0 or u < np.exp(-min(x, 60.0)))
