"""The allocation-free key switch (ckg_key_switch_noalloc) against the regular one.

Callers that cannot allocate device memory while serving (a process that reserved its
whole HBM budget up front, or a runtime that owns every device allocation) use the entry
point whose working space is the library's fixed device array. This file is collected
last, and it passes both alone in a fresh process and after the other tests: the shared
array keeps the previous call's contents, and every call must still give the regular
entry point's result, bit for bit (integer arithmetic: the tolerance is zero).
"""

import numpy as np
import pytest

from gpu_util import assert_same, empty_dev, from_dev, make_pair, ptr, to_dev

pytestmark = pytest.mark.gpu


def _compare_two_calls(ckg, oracle, name, levels, seed):
    P, ctx = make_pair(ckg, oracle, name)
    kg = oracle.KeyGenerator(P, seed)
    key = ctx.upload_key(kg.relin_key().export())
    for call, level in enumerate(levels):
        d = P.random_q(1000 + 17 * call + level, level)
        dd = to_dev(d)
        rb, ra = empty_dev(d.shape), empty_dev(d.shape)
        nb, na = empty_dev(d.shape), empty_dev(d.shape)
        ctx.key_switch(key, ptr(dd), level, ptr(rb), ptr(ra))
        ctx.key_switch_noalloc(key, ptr(dd), level, ptr(nb), ptr(na))
        ctx.sync()
        assert_same(from_dev(nb), from_dev(rb), f"{name} call {call} level {level}: b")
        assert_same(from_dev(na), from_dev(ra), f"{name} call {call} level {level}: a")


def test_noalloc_matches_key_switch_small(ckg, oracle):
    """Two calls in a row (top level, then a lower one) on N = 2^12, 6 + 2 primes, dnum 3."""
    _compare_two_calls(ckg, oracle, "small", [5, 2], seed=3)


def test_noalloc_matches_key_switch_n16(ckg, oracle):
    """Two calls in a row at the largest supported size: N = 2^16, 24 + 8 primes, dnum 3,
    top level (112 MiB of the 128 MiB working space)."""
    _compare_two_calls(ckg, oracle, "cfg2", [23, 23], seed=4)


def test_noalloc_rejects_oversized(ckg, oracle):
    """N = 2^16 with 32 + 4 primes and 8 digits needs 216 MiB at its top level: rejected
    with a clear error before anything runs. A low level of the same context (level 3,
    about 22 MiB) fits, and gives the regular entry point's result."""
    P = oracle.Params.from_bits(16, [54] + [42] * 16 + [34] * 4 + [58] * 7 + [56] * 4, [60] * 4, 42, 8)
    ctx = ckg.Context(16, P.q, P.p, 8)
    n = 1 << 16
    dd = to_dev(np.zeros((32, n), np.uint64))
    out = empty_dev((32, n))
    with pytest.raises(ckg.InvalidParams, match="working space"):
        ctx.key_switch_noalloc(None, ptr(dd), 31, ptr(out), ptr(out))
    key = ctx.upload_key(oracle.KeyGenerator(P, 6).relin_key().export())
    d = to_dev(P.random_q(77, 3))
    rb, ra, nb, na = (empty_dev((4, n)) for _ in range(4))
    ctx.key_switch(key, ptr(d), 3, ptr(rb), ptr(ra))
    ctx.key_switch_noalloc(key, ptr(d), 3, ptr(nb), ptr(na))
    ctx.sync()
    assert_same(from_dev(nb), from_dev(rb), "n16_boot level 3: b")
    assert_same(from_dev(na), from_dev(ra), "n16_boot level 3: a")
