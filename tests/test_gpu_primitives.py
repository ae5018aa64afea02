"""GPU parity of the ring/RNS primitives against the oracle, bit for bit.

Mirrors the reference's shared-case GPU tests (crates/ckks-train-cuda/tests/cases/mod.rs):
several inputs per op spread over levels, all-(q-1) inputs, and the near-tie fixtures
that catch an FMA-contracted overflow estimate in exact base conversion.
"""

import numpy as np
import pytest

from gpu_util import (PARAM_SETS, assert_same, empty_dev, from_dev, make_pair, near_tie_limbs, ptr, to_dev)

pytestmark = pytest.mark.gpu


def levels(L):
    """The levels of the reference's INPUTS (cases/mod.rs:54-57)."""
    return sorted({L, L - 1, 3 * L // 4, L // 2, L // 3, 2, 1, 0} & set(range(L + 1)), reverse=True)


@pytest.fixture(scope="module", params=["tiny", "small", "cfg1", "n14", "n15", "cfg2"])
def pair(request, ckg, oracle):
    return make_pair(ckg, oracle, request.param)


def test_ntt_forward_inverse(pair):
    P, ctx = pair
    primes = list(range(len(ctx.primes)))
    allp = ctx.primes
    x = np.stack([oracle_rand(P, 11 + i, allp[i]) for i in primes])
    x[0] = allp[0] - 1  # all (q-1)
    x[-1] = 0
    d = to_dev(x)
    out = empty_dev(x.shape)
    ctx.ntt(ptr(d), ptr(out), primes, inverse=False)
    ctx.sync()
    got = from_dev(out)
    want = np.stack([P.ntt(x[i:i + 1], first_prime=i if i < P.nq else i - P.nq, basis=0 if i < P.nq else 1)[0]
                     for i in primes])
    assert_same(got, want, "forward NTT")
    back = empty_dev(x.shape)
    ctx.ntt(ptr(out), ptr(back), primes, inverse=True)
    ctx.sync()
    assert_same(from_dev(back), x, "inverse NTT round trip")
    # inverse of arbitrary residues (not only NTT outputs)
    y = np.stack([oracle_rand(P, 91 + i, allp[i]) for i in primes])
    dy = to_dev(y)
    ctx.ntt(ptr(dy), ptr(dy), primes, inverse=True)
    ctx.sync()
    want = np.stack([P.ntt(y[i:i + 1], first_prime=i if i < P.nq else i - P.nq, inverse=True,
                           basis=0 if i < P.nq else 1)[0] for i in primes])
    assert_same(from_dev(dy), want, "inverse NTT in place")


def oracle_rand(P, seed, q):
    import oracle as O
    return O.random_poly(seed, [q], P.n)[0]


def test_pointwise(pair):
    P, ctx = pair
    L = P.max_level
    for i, level in enumerate(levels(L)):
        a = P.random_q(4500 + 10 * i, level)
        b = P.random_q(4501 + 10 * i, level)
        if i == 0:
            a[:] = np.asarray(P.q[: level + 1], np.uint64)[:, None] - 1
        da, db = to_dev(a), to_dev(b)
        out = empty_dev(a.shape)
        for op in range(3):
            ctx.poly_binary(op, ptr(da), ptr(db), ptr(out), 0, level + 1)
            ctx.sync()
            assert_same(from_dev(out), P.poly_op(op, a, b), f"op {op} level {level}")
        ctx.poly_negate(ptr(da), ptr(out), 0, level + 1)
        ctx.sync()
        assert_same(from_dev(out), P.poly_op(3, a), f"negate level {level}")
        scalar = (0xDEADBEEFCAFEF00D * (i + 1)) & 0xFFFFFFFFFFFFFFFF
        ctx.poly_mul_scalar(ptr(da), scalar, ptr(out), 0, level + 1)
        ctx.sync()
        assert_same(from_dev(out), P.poly_op(4, a, scalar=scalar), f"mul_scalar level {level}")


def test_automorphism(pair, oracle):
    P, ctx = pair
    L = P.max_level
    two_n = 2 * P.n
    elts = [oracle.galois_elt(P.n, s) for s in (1, -1, 2, 5)] + [two_n - 1]
    for i, g in enumerate(elts):
        a = P.random_q(600 + i, L)
        da = to_dev(a)
        out = empty_dev(a.shape)
        ctx.automorphism(ptr(da), ptr(out), L + 1, g)
        ctx.sync()
        assert_same(from_dev(out), P.automorphism(a, g), f"automorphism g={g}")


def test_rescale(pair):
    P, ctx = pair
    L = P.max_level
    for i, level in enumerate([l for l in levels(L) if l >= 1]):
        a = P.random_q(700 + i, level)
        if i == 0:
            a[-1] = P.q[level] - 1
        da = to_dev(a)
        out = empty_dev((level, P.n))
        ctx.rescale(ptr(da), level, ptr(out))
        ctx.sync()
        assert_same(from_dev(out), P.rescale(a), f"rescale level {level}")


def test_mod_up(pair):
    P, ctx = pair
    L = P.max_level
    for i, level in enumerate(levels(L)):
        x = P.random_q(5000 + i, level)
        dx = to_dev(x)
        for j in range(len(P.digit_ranges(level))):
            oq, op_ = empty_dev((level + 1, P.n)), empty_dev((P.np_, P.n))
            ctx.mod_up(ptr(dx), level, j, ptr(oq), ptr(op_))
            ctx.sync()
            wq, wp = P.mod_up(x, j)
            assert_same(from_dev(oq), wq, f"mod_up Q part level {level} digit {j}")
            assert_same(from_dev(op_), wp, f"mod_up P part level {level} digit {j}")


def test_mod_up_near_ties(pair):
    """Every digit's [x + h]_D next to 0 or Q_D (cases/mod.rs:334-345, 350-360)."""
    P, ctx = pair
    L = P.max_level
    for level in sorted({L, max(L - 1, 0), L // 2}):
        x = near_tie_limbs(P.q[: level + 1], P.n)
        x = P.ntt(x)
        dx = to_dev(x)
        for j in range(len(P.digit_ranges(level))):
            oq, op_ = empty_dev((level + 1, P.n)), empty_dev((P.np_, P.n))
            ctx.mod_up(ptr(dx), level, j, ptr(oq), ptr(op_))
            ctx.sync()
            wq, wp = P.mod_up(x, j)
            assert_same(from_dev(oq), wq, f"near-tie mod_up Q part level {level} digit {j}")
            assert_same(from_dev(op_), wp, f"near-tie mod_up P part level {level} digit {j}")


def test_mod_down(pair):
    P, ctx = pair
    L = P.max_level
    for i, level in enumerate(levels(L)):
        q = P.random_q(5100 + i, level)
        p = P.random_p(5200 + i)
        dq, dp = to_dev(q), to_dev(p)
        out = empty_dev(q.shape)
        ctx.mod_down(ptr(dq), level, ptr(dp), ptr(out))
        ctx.sync()
        assert_same(from_dev(out), P.mod_down(q, p), f"mod_down level {level}")


def test_mod_down_near_ties(pair):
    """P part with [X + h]_P next to 0 or P in every coefficient (cases/mod.rs:313-330)."""
    P, ctx = pair
    L = P.max_level
    for level in sorted({L, L // 2, 0}):
        q = P.ntt(P.random_q(5300 + level, level))
        p = P.ntt(near_tie_limbs(P.p, P.n), basis=1)
        dq, dp = to_dev(q), to_dev(p)
        out = empty_dev(q.shape)
        ctx.mod_down(ptr(dq), level, ptr(dp), ptr(out))
        ctx.sync()
        assert_same(from_dev(out), P.mod_down(q, p), f"near-tie mod_down level {level}")


def test_conversion_engines(pair):
    """ModUp and ModDown with the base conversions on the tensor cores (exact u8 x u8 -> s32
    products, FP64-quotient reduction) and on the integer kernels: both give the oracle's words,
    on random and near-tie inputs and on all-(q-1) limbs (largest partial sums)."""
    P, ctx = pair
    L = P.max_level
    default = ctx.bconv_tc
    engines = [0, 2] if default else [0]  # integer kernels; tensor cores at every source count
    try:
        for tc in engines:
            ctx.bconv_tc = tc
            for level in sorted({L, L // 2, 0}):
                for kind in ("random", "ties", "max"):
                    if kind == "random":
                        x = P.random_q(6000 + level, level)
                        p = P.random_p(6100 + level)
                    elif kind == "ties":
                        x = P.ntt(near_tie_limbs(P.q[: level + 1], P.n))
                        p = P.ntt(near_tie_limbs(P.p, P.n), basis=1)
                    else:
                        x = np.stack([np.full(P.n, q - 1, np.uint64) for q in P.q[: level + 1]])
                        p = np.stack([np.full(P.n, q - 1, np.uint64) for q in P.p])
                    dx, dp = to_dev(x), to_dev(p)
                    what = f"engine {'tc' if tc else 'int'} level {level} {kind}"
                    for j in range(len(P.digit_ranges(level))):
                        oq, op_ = empty_dev((level + 1, P.n)), empty_dev((P.np_, P.n))
                        ctx.mod_up(ptr(dx), level, j, ptr(oq), ptr(op_))
                        ctx.sync()
                        wq, wp = P.mod_up(x, j)
                        assert_same(from_dev(oq), wq, f"mod_up Q {what} digit {j}")
                        assert_same(from_dev(op_), wp, f"mod_up P {what} digit {j}")
                    out = empty_dev(x.shape)
                    ctx.mod_down(ptr(dx), level, ptr(dp), ptr(out))
                    ctx.sync()
                    assert_same(from_dev(out), P.mod_down(x, p), f"mod_down {what}")
        assert ctx.device_fault() == 0
    finally:
        ctx.bconv_tc = default


def test_ntt_tma_staging(pair):
    """The opt-in TMA-staged column passes (one tensor-map box per tile, two stages deep) give the
    per-tile kernels' words: forward and inverse over every prime, in place and out of place."""
    P, ctx = pair
    if P.n < (1 << 12):
        pytest.skip("two-pass transforms only")
    primes = list(range(len(ctx.primes)))
    allp = ctx.primes
    x = np.stack([oracle_rand(P, 211 + i, allp[i]) for i in primes])
    want_f = np.stack([P.ntt(x[i:i + 1], first_prime=i if i < P.nq else i - P.nq, basis=0 if i < P.nq else 1)[0]
                       for i in primes])
    try:
        ctx.ntt_tma = True
        d = to_dev(x)
        out = empty_dev(x.shape)
        ctx.ntt(ptr(d), ptr(out), primes, inverse=False)
        ctx.sync()
        assert_same(from_dev(out), want_f, "forward NTT, TMA-staged columns")
        ctx.ntt(ptr(out), ptr(out), primes, inverse=True)
        ctx.sync()
        assert_same(from_dev(out), x, "inverse NTT in place, TMA-staged columns")
        assert ctx.device_fault() == 0
    finally:
        ctx.ntt_tma = False
