"""The reference's own CUDA kernels (crates/ckks-train-cuda/kernels, compiled unmodified into
oracle/_ref/libref_gpu.so and driven through the launch sequences of the reference's Rust host
code, oracle/ref_gpu/ref_ks.cu) against the oracle and this library, bit for bit: the batched NTT
and the hybrid key switch. This pins the replay that bench.py's reference arm times on the GPU,
so that timing measures the reference's real computation."""

import numpy as np
import pytest

from gpu_util import assert_same, empty_dev, from_dev, make_pair, ptr, to_dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref_gpu():
    import ref_gpu as R
    if not R.available():
        pytest.skip("oracle/_ref/libref_gpu.so not built (the reference tree was absent at build time)")
    return R


@pytest.mark.parametrize("name", ["small", "cfg2"])
def test_reference_kernels_match(ckg, oracle, ref_gpu, name):
    P, ctx = make_pair(ckg, oracle, name)
    import gpu_util
    R = ref_gpu.RefGpu(P.log_n, P.q, P.p, gpu_util.PARAM_SETS[name]["dnum"])
    # the batched NTT over every prime, forward then inverse
    primes = list(range(P.nq + P.np_))
    allp = list(P.q) + list(P.p)
    x = np.stack([oracle.random_poly(40 + i, [allp[i]], P.n)[0] for i in primes])
    d = to_dev(x)
    R.ntt(ptr(d), primes, False)
    R.sync()
    want = np.stack([P.ntt(x[i:i + 1], first_prime=i if i < P.nq else i - P.nq, basis=0 if i < P.nq else 1)[0]
                     for i in primes])
    assert_same(from_dev(d), want, f"{name}: reference forward NTT")
    R.ntt(ptr(d), primes, True)
    R.sync()
    assert_same(from_dev(d), x, f"{name}: reference inverse NTT")
    # the key switch at the top level and below
    kg = oracle.KeyGenerator(P, 17)
    rk = kg.relin_key()
    key_host = rk.export()
    key_dev = to_dev(key_host)
    d_rk = ctx.upload_key(key_host)
    for level in sorted({P.max_level, P.max_level // 2}):
        a = P.random_q(300 + level, level)
        da = to_dev(a)
        rb, ra = empty_dev(a.shape), empty_dev(a.shape)
        R.key_switch(ptr(da), level, ptr(key_dev), ptr(rb), ptr(ra))
        R.sync()
        ob, oa = empty_dev(a.shape), empty_dev(a.shape)
        ctx.key_switch(d_rk, ptr(da), level, ptr(ob), ptr(oa))
        ctx.sync()
        wb, wa = rk.key_switch(a)
        assert_same(from_dev(rb), wb, f"{name} level {level}: reference kernels, b")
        assert_same(from_dev(ra), wa, f"{name} level {level}: reference kernels, a")
        assert_same(from_dev(ob), wb, f"{name} level {level}: this library, b")
        assert_same(from_dev(oa), wa, f"{name} level {level}: this library, a")
