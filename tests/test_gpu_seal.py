"""SEAL 4.1 bytes through the device (include/ckg.h, "SEAL 4.1 wire format"): requests parsed
and uploaded (load_ciphertext / load_plaintext), evaluated, and written back
(save_ciphertext), bit-identical to the oracle's results serialized on the host."""

import numpy as np
import pytest

from gpu_util import PARAM_SETS, random_ct
from test_gpu_eval import Env

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(ckg, oracle):
    return Env(ckg, oracle, "small", [1, -1, 2])


def test_seal_bytes_through_the_evaluator(env):
    ckg, P, gpu, cpu = env.ckg, env.P, env.gpu, env.cpu
    log_n = PARAM_SETS["small"]["log_n"]
    a, b = random_ct(P, 1, P.max_level), random_ct(P, 2, P.max_level)
    wa = ckg.seal_encode(log_n, P.q, a, P.max_level, env.scale)
    wb = ckg.seal_encode(log_n, P.q, b, P.max_level, env.scale)
    ga, gb = gpu.ct_from_seal(wa), gpu.ct_from_seal(wb)
    assert ga.level() == P.max_level and ga.scale() == env.scale
    assert np.array_equal(gpu.download_ct(ga)[0], a)
    assert gpu.ct_to_seal(ga) == wa
    ca, cb = cpu.ct(a, env.scale), cpu.ct(b, env.scale)
    for want, got, what in [(cpu.rescale(cpu.mul(ca, cb)), gpu.rescale(gpu.mul(ga, gb)), "mul+relin+rescale"),
                            (cpu.rotate(ca, 1), gpu.rotate(ga, 1), "rotate")]:
        assert gpu.ct_to_seal(got) == ckg.seal_encode(log_n, P.q, want.data(), want.level, want.scale), what
    pt = P.random_q(3, P.max_level)
    gp = gpu.pt_from_seal(ckg.seal_encode(log_n, P.q, pt, P.max_level, env.scale, plaintext=True))
    assert gp.level() == P.max_level and gp.scale() == env.scale
    want = cpu.mul_plain(ca, pt, env.scale)
    assert gpu.ct_to_seal(gpu.mul_plain(ga, gp)) == ckg.seal_encode(log_n, P.q, want.data(), want.level, want.scale)


def test_seal_errors_before_upload(env):
    ckg, P, gpu = env.ckg, env.P, env.gpu
    log_n = PARAM_SETS["small"]["log_n"]
    good = ckg.seal_encode(log_n, P.q, random_ct(P, 4, 1), 1, env.scale)
    for bad in (good[:-8], good + b"\0", b"\x5e\xa1" + good[2:3] + bytes([3]) + good[4:]):
        with pytest.raises(ckg.InvalidParams):
            gpu.ct_from_seal(bad)
    with pytest.raises(ckg.InvalidParams):
        gpu.pt_from_seal(good)
    other = ckg.seal_encode(log_n + 1, ckg.primes_for_bits(log_n + 1, [60, 40], [60])[0],
                            np.zeros((2, 2, 1 << (log_n + 1)), np.uint64), 1, env.scale)
    with pytest.raises(ckg.InvalidParams):
        gpu.ct_from_seal(other)  # another ring degree's parms_id
