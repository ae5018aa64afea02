"""The benchmark configurations' exact workloads against the oracle, bit for bit:

* config 1 (N = 2^13, 4 x 45-bit q, one 60-bit p, dnum 4): 64 seeded ciphertext pairs,
  64 x (HMult + relinearization + rescale) and 64 x rotation by +1, through the per-op
  evaluator and through one batched launch sequence replayed from a CUDA graph;
* config 2's parameters (N = 2^16, 24 x 50-bit q, 8 x 60-bit p, dnum 3) through the per-op
  evaluator (the path the benchmark's `plain` line times): mul, rotate by +-2^k, hoisted
  rotations and matvec_enc, every coefficient, level, scale and OpCounter equal.
"""

import numpy as np
import pytest

from gpu_util import assert_same, random_ct
from test_gpu_eval import Env

pytestmark = pytest.mark.gpu


def _check(gpu, want, got, what):
    data, scale = gpu.download_ct(got)
    assert got.level() == want.level and scale == want.scale, f"{what}: level/scale"
    assert_same(data, want.data(), what)


def test_config1_workload(ckg, oracle):
    env = Env(ckg, oracle, "cfg1", [1], seed=12)
    P, cpu, gpu = env.P, env.cpu, env.gpu
    L = P.max_level
    pairs = [(random_ct(P, 2 * i + 1, L), random_ct(P, 2 * i + 2, L)) for i in range(64)]
    cpu.reset_counter()
    want_mul, want_rot = [], []
    for a, b in pairs:
        ca, cb = cpu.ct(a, env.scale), cpu.ct(b, env.scale)
        want_mul.append(cpu.rescale(cpu.mul(ca, cb)))
        want_rot.append(cpu.rotate(ca, 1))
    want_counter = cpu.counter()
    assert (want_counter["relins"], want_counter["rotations"], want_counter["rescales"]) == (64, 64, 64)
    # per op
    gpu.reset_counter()
    ups = [(gpu.upload_ct(a, env.scale), gpu.upload_ct(b, env.scale)) for a, b in pairs]
    for i, (ga, gb) in enumerate(ups):
        _check(gpu, want_mul[i], gpu.rescale(gpu.mul(ga, gb)), f"per-op HMult {i}")
        _check(gpu, want_rot[i], gpu.rotate(ga, 1), f"per-op rotation {i}")
    assert gpu.counter() == want_counter
    # batched, graph-replayed
    gpu.reset_counter()
    batch = ckg.Batch(gpu)
    got_mul = [batch.mul_relin_rescale(ga, gb) for ga, gb in ups]
    got_rot = [batch.rotate(ga, 1) for ga, _ in ups]
    batch.capture_graph()
    batch.launch_graph()
    for i in range(64):
        _check(gpu, want_mul[i], got_mul[i], f"batched HMult {i}")
        _check(gpu, want_rot[i], got_rot[i], f"batched rotation {i}")
    assert gpu.counter() == want_counter


@pytest.fixture(scope="module")
def cfg2(ckg, oracle):
    steps = [s * (1 << k) for k in range(15) for s in (1, -1)]
    return Env(ckg, oracle, "cfg2", steps, seed=21)


def test_cfg2_per_op_mul_rotate(cfg2):
    env = cfg2
    P = env.P
    env.cpu.reset_counter()
    env.gpu.reset_counter()
    for level in (23, 11):
        a_c, a_g = env.pair(random_ct(P, 60 + level, level))
        b_c, b_g = env.pair(random_ct(P, 61 + level, level))
        m_c, m_g = env.cpu.mul(a_c, b_c), env.gpu.mul(a_g, b_g)
        env.check(m_c, m_g, f"mul level {level}")
        env.check(env.cpu.rescale(m_c), env.gpu.rescale(m_g), f"rescale level {level}")
        for s in (1, -1, 1 << 7, -(1 << 14)):
            env.check(env.cpu.rotate(a_c, s), env.gpu.rotate(a_g, s), f"rotate {s} level {level}")


def test_cfg2_per_op_hoisted_and_matvec(cfg2):
    env = cfg2
    P = env.P
    env.cpu.reset_counter()
    env.gpu.reset_counter()
    x_c, x_g = env.pair(random_ct(P, 70, 23))
    steps = [1, 2, 4, -8, 1 << 10]
    for s, c, g in zip(steps, env.cpu.hoisted_rotate(x_c, steps), env.gpu.hoisted_rotate(x_g, steps)):
        env.check(c, g, f"hoisted_rotate {s}")
    d = 4
    cts = [env.pair(random_ct(P, 80 + i, 23)) for i in range(d)]
    env.check(env.cpu.matvec_enc(d, 1, [c for c, _ in cts], x_c),
              env.gpu.matvec_enc(d, 1, [g for _, g in cts], x_g), "matvec_enc d 4")
    pts = np.stack([P.random_q(90 + i, 23) for i in range(d)])
    env.check(env.cpu.matvec_plain(d, 1, pts, env.scale, x_c),
              env.gpu.matvec_plain(d, 1, [env.gpu.upload_pt(p, env.scale) for p in pts], x_g), "matvec_plain d 4")


def test_cfg2_matvec_enc_batch(cfg2):
    """matvec_enc_batch at N = 2^16, 24 + 8 primes, dnum 3: two jobs at two levels, each equal to
    the oracle's matvec_enc, with the counters of the jobs one by one."""
    env = cfg2
    P = env.P
    env.cpu.reset_counter()
    env.gpu.reset_counter()
    want, jobs = [], []
    for n, level in enumerate((23, 9)):
        x_c, x_g = env.pair(random_ct(P, 910 + n, level))
        ents = [env.pair(random_ct(P, 920 + 10 * n + i, level)) for i in range(4)]
        want.append(env.cpu.matvec_enc(4, 1, [c for c, _ in ents], x_c))
        jobs.append((4, 1, [g for _, g in ents], x_g))
    got = env.gpu.matvec_enc_batch(jobs)
    for n, (w, g) in enumerate(zip(want, got)):
        data, scale = env.gpu.download_ct(g)
        assert g.level() == w.level and scale == w.scale
        assert_same(data, w.data(), f"cfg2 matvec_enc_batch job {n}")
    assert env.gpu.counter() == env.cpu.counter()
