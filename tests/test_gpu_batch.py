"""Batched execution at uneven levels (one launch sequence for a whole op mix): every
result equals the same op run on its own through the evaluator and the oracle, bit for
bit, with the same OpCounter, whether run eagerly or replayed from a CUDA graph."""

import numpy as np
import pytest

from gpu_util import PARAM_SETS, assert_same, random_ct
from test_gpu_eval import Env

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["small", "cfg1", "tiny"])
def env(request, ckg, oracle):
    name = request.param
    slots = (1 << PARAM_SETS[name]["log_n"]) // 2
    return Env(ckg, oracle, name, [1, -1, 2, 4, 8, slots // 2])


def _mix(env, seed, count):
    """A seeded op mix (40% HMult+relin+rescale, 40% rotation, 20% PtMult+rescale) over
    ciphertexts at levels drawn uniformly from 1..L (0 for some rotations)."""
    rng = np.random.default_rng(seed)
    P = env.P
    L = P.max_level
    ops = []
    for i in range(count):
        r = rng.random()
        if r < 0.4:
            kind = "mul"
        elif r < 0.8:
            kind = "rot"
        else:
            kind = "pmul"
        level = int(rng.integers(1 if kind != "rot" else 0, L + 1)) if L >= 1 else 0
        if kind != "rot" and L < 1:
            kind = "rot"
        steps = int(rng.choice([1, -1, 2, 4, 8, 0]))
        ops.append((kind, level, steps, 1000 * seed + i))
    return ops


def _run_mix(env, ops, graph, chunk=None, tune=False):
    P, gpu, cpu = env.P, env.gpu, env.cpu
    batch = env.ckg.Batch(gpu)
    if chunk:
        batch.chunk_items = chunk
    want, got = [], []
    cpu.reset_counter()
    gpu.reset_counter()
    for kind, level, steps, s in ops:
        a = random_ct(P, s, level)
        a_c, a_g = env.pair(a)
        if kind == "mul":
            b = random_ct(P, s + 500, level)
            b_c, b_g = env.pair(b)
            want.append(cpu.rescale(cpu.mul(a_c, b_c)))
            got.append(batch.mul_relin_rescale(a_g, b_g))
        elif kind == "rot":
            want.append(cpu.rotate(a_c, steps))
            got.append(batch.rotate(a_g, steps))
        else:
            pt = P.random_q(s + 900, level)
            want.append(cpu.rescale(cpu.mul_plain(a_c, pt, env.scale)))
            got.append(batch.mul_plain_rescale(a_g, gpu.upload_pt(pt, env.scale)))
    if tune:
        before = gpu.counter()
        rep = batch.autotune(1)
        assert gpu.counter() == before, "tuning counted ops"
        assert len(rep["trials"]) == 15 and rep["ntt_wave"] in (0, 32, 64, 128, 256)
        assert rep["chunk_items"] in (64, 128, 256) and batch.chunk_items == rep["chunk_items"]
    if graph:
        batch.capture_graph()
        batch.launch_graph()
    else:
        batch.run()
    for i, (w, g) in enumerate(zip(want, got)):
        data, scale = gpu.download_ct(g)
        assert g.level() == w.level and scale == w.scale, f"op {i} {ops[i]}: level/scale"
        assert_same(data, w.data(), f"op {i} {ops[i]}")
    assert gpu.counter() == cpu.counter()
    return batch, got


@pytest.mark.parametrize("graph", [False, True])
def test_batch_matches_oracle(env, graph):
    _run_mix(env, _mix(env, 7, 24), graph)


def test_batch_graph_replay_is_stable(env):
    """Replaying the captured graph recomputes the same results (and counts again)."""
    batch, got = _run_mix(env, _mix(env, 11, 12), True)
    first = [env.gpu.download_ct(g)[0] for g in got]
    before = env.gpu.counter()
    batch.launch_graph()
    for i, g in enumerate(got):
        assert_same(env.gpu.download_ct(g)[0], first[i], f"replay op {i}")
    after = env.gpu.counter()
    assert after["relins"] - before["relins"] == sum(1 for k in _mix(env, 11, 12) if k[0] == "mul")


def test_same_alone_and_in_mix(env):
    """Each op gives the same ciphertext alone (a batch of one) and inside a large mix."""
    ops = _mix(env, 13, 20)
    _, mixed = _run_mix(env, ops, False)
    for i in (0, 5, 13):
        _, alone = _run_mix(env, [ops[i]], False)
        assert_same(env.gpu.download_ct(alone[0])[0], env.gpu.download_ct(mixed[i])[0], f"op {i} alone vs mix")


def test_batch_errors_before_work(env):
    P = env.P
    batch = env.ckg.Batch(env.gpu)
    a = env.gpu.upload_ct(random_ct(P, 1, P.max_level), env.scale)
    z = env.gpu.upload_ct(random_ct(P, 2, 0), env.scale)
    with pytest.raises(env.ckg.NoLevelsLeft):
        batch.mul_relin_rescale(z, z)
    with pytest.raises(env.ckg.InvalidParams, match="missing galois key"):
        batch.rotate(a, 3)
    if P.max_level >= 1:
        b = env.gpu.upload_ct(random_ct(P, 3, P.max_level - 1), env.scale)
        with pytest.raises(env.ckg.LevelMismatch):
            batch.mul_relin_rescale(a, b)
    assert batch.key_switches() == 0


def test_batch_tuning_is_bit_neutral(env):
    """Every NTT limb wave and chunk size computes the same words; the autotuner counts no ops
    and leaves its choice on the context and the batch (include/ckg.h, "tuning")."""
    ops = _mix(env, 17, 40)
    ctx = env.gpu.ctx
    wave0 = ctx.ntt_wave
    try:
        for wave, chunk in [(0, 128), (8, 3), (32, 7), (1, 1)]:
            ctx.ntt_wave = wave
            _run_mix(env, ops, wave % 2 == 0, chunk=chunk)
        _run_mix(env, ops, True, tune=True)
        with pytest.raises(env.ckg.InvalidParams):
            ctx.ntt_wave = -1
        with pytest.raises(env.ckg.InvalidParams):
            env.ckg.Batch(env.gpu).chunk_items = 0
    finally:
        ctx.ntt_wave = wave0


@pytest.fixture(scope="module")
def env_cfg2(ckg, oracle):
    """The benchmark's own parameters: N = 2^16, 24 x 50-bit + 8 x 60-bit primes, dnum 3."""
    return Env(ckg, oracle, "cfg2", [1, -1, 2, 4, 8])


def test_batch_matches_oracle_cfg2(env_cfg2):
    """A 48-op mix at random levels of the full-size parameters, replayed from a CUDA graph in
    chunks of 16 ops: every coefficient equals the oracle's, levels, scales and counters too."""
    _run_mix(env_cfg2, _mix(env_cfg2, 23, 48), True, chunk=16)
