"""The oracle's primitive entry points (vo_ntt, vo_external_product,
vo_key_switch), which the GPU primitive tests compare against.

The oracle's NTT, gadget product and external product are pinned by the
reference's layer-3/4 KATs (test_oracle_kats.py); these tests pin the flat
buffer layouts of the new entry points: the NTT is a negacyclic transform
(round trip, products), an external product with the trivial RGSW of 1 is the
identity up to the gadget's rounding (so neg_s_m comes first and sample 0 pairs
with the largest gadget entry), and a key switch under the trivial key of 1
returns (0, X^k body - X^k mask) up to the same rounding.
"""
import numpy as np
import pytest

from via_rs_b200.params import PAPER_Q1, PAPER_Q2

Q1 = tuple(PAPER_Q1)


def _negacyclic(a, b, q):
    n = len(a)
    out = [0] * n
    for i in range(n):
        for j in range(n):
            k = i + j
            v = int(a[i]) * int(b[j])
            if k >= n:
                out[k - n] -= v
            else:
                out[k] += v
    return np.array([x % q for x in out], dtype=np.uint64)


def _rand(rng, q, n, count):
    return np.concatenate([rng.integers(0, qi, size=(count, 1, n), dtype=np.uint64) for qi in q], axis=1)


def _crt_centered(limbs, q):
    """[nl][n] residues -> centered Python ints modulo prod(q)."""
    if len(q) == 1:
        Q = q[0]
        vals = [int(v) for v in limbs[0]]
    else:
        q0, q1 = q
        Q = q0 * q1
        inv = pow(q0, -1, q1)
        vals = [int(a) + q0 * (((int(b) - int(a)) * inv) % q1) for a, b in zip(limbs[0], limbs[1])]
    return [v - Q if v > Q // 2 else v for v in vals], Q


def _gadget(Q, base, L):
    return [(Q + base ** (i + 1) // 2) // base ** (i + 1) for i in range(L)]


def _const_poly(value, q, n):
    out = np.zeros((len(q), n), dtype=np.uint64)
    for l, qi in enumerate(q):
        out[l, 0] = value % qi
    return out


@pytest.mark.parametrize("q", [Q1, (PAPER_Q2,)])
def test_oracle_ntt_is_negacyclic(oracle, q):
    rng = np.random.default_rng(1)
    n = 32
    a = _rand(rng, q, n, 2)
    fa = oracle.ntt(q, n, a)
    assert np.array_equal(oracle.ntt(q, n, fa, inverse=True), a)
    fb = fa[1]
    prod_eval = np.zeros_like(fa[0])
    for l, qi in enumerate(q):
        prod_eval[l] = np.array([(int(x) * int(y)) % qi for x, y in zip(fa[0][l], fb[l])], dtype=np.uint64)
    got = oracle.ntt(q, n, prod_eval[None], inverse=True)[0]
    for l, qi in enumerate(q):
        assert np.array_equal(got[l], _negacyclic(a[0][l], a[1][l], qi))


@pytest.mark.parametrize("q,base,L,bound", [(Q1, 55879, 2, 2**46), ((PAPER_Q2,), 81, 2, 2**22)])
def test_oracle_external_product_trivial_rgsw_of_one(oracle, q, base, L, bound):
    rng = np.random.default_rng(2)
    n = 64
    Q = int(np.prod([int(x) for x in q], dtype=object))
    g = _gadget(Q, base, L)
    rgsw = np.zeros((2 * L, 2, len(q), n), dtype=np.uint64)
    for i in range(L):
        rgsw[i, 0] = _const_poly(g[i], q, n)      # neg_s_m[i] = (g_i, 0)
        rgsw[L + i, 1] = _const_poly(g[i], q, n)  # m[i] = (0, g_i)
    ct = _rand(rng, q, n, 2)
    out = oracle.external_product(q, n, base, L, rgsw, ct, threads=1).reshape(2, len(q), n)
    for part in range(2):
        got, _ = _crt_centered(out[part], q)
        want, _ = _crt_centered(ct[part], q)
        assert max(abs(a - b) for a, b in zip(got, want)) < bound


def test_oracle_key_switch_trivial_key_of_one(oracle):
    rng = np.random.default_rng(3)
    q, n, base, L = Q1, 64, 18, 18
    Q = q[0] * q[1]
    g = _gadget(Q, base, L)
    key = np.zeros((L, 2, 2, n), dtype=np.uint64)
    for i in range(L):
        key[i, 1] = _const_poly(g[i], q, n)  # RLev of 1: (0, g_i)
    cts = _rand(rng, q, n, 6).reshape(3, 2, len(q), n)
    shifts = np.array([0, 5, 2 * n - 1], dtype=np.uint64)
    out = oracle.key_switch(q, n, base, L, key, cts.reshape(-1), shifts, threads=1).reshape(3, 2, 2, n)

    def rot(poly_limbs, k):
        res = np.zeros_like(poly_limbs)
        for l, qi in enumerate(q):
            for i in range(n):
                pos = i + int(k)
                v = int(poly_limbs[l][i])
                sign = -1 if (pos // n) % 2 else 1
                res[l][pos % n] = (sign * v) % qi
        return res

    for c in range(3):
        assert not out[c, 0].any(), "mask of a key switch under a trivial key is zero"
        want_rns = np.stack([(rot(cts[c, 1], shifts[c])[l].astype(object) - rot(cts[c, 0], shifts[c])[l].astype(object))
                             % q[l] for l in range(2)]).astype(np.uint64)
        got, _ = _crt_centered(out[c, 1], q)
        want, _ = _crt_centered(want_rns, q)
        assert max(abs(a - b) for a, b in zip(got, want)) < 2**10
