"""The algorithmic-byte accounting behind bench.py's `roofline_stream` (stream_roofline), on CPU:
per op its inputs read once and outputs written once, and each distinct key read once per chunk
of the batch builder. At N = 2^16 with 24 + 8 primes and dnum 3 (digits of 8 primes) the top-level
figures are 334 limbs for HMult+relin+rescale and 288 limbs for a rotation, each with its key
(2 x 3 digits x 32 limbs = 192 limbs)."""

import importlib.util
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


N, K, ALPHA = 1 << 16, 8, 8
LIMB = 8 * N
PEAKS = {"hbm_gbs": 6549.4}


def alg_limbs(bench, ops):
    out = bench.stream_roofline(ops, N, K, ALPHA, 1.0, PEAKS)
    assert out["alg_bytes"] % LIMB == 0 and out["key_bytes"] % LIMB == 0
    return out["alg_bytes"] // LIMB, out["key_bytes"] // LIMB, out["chunks"]


def test_top_level_single_ops(bench):
    assert alg_limbs(bench, [("mul", 23, 1)]) == (334, 192, 1)
    assert alg_limbs(bench, [("rot", 23, 1)]) == (288, 192, 1)
    assert alg_limbs(bench, [("pmul", 23, 1)]) == (3 * 24 + 2 * 23, 0, 1)


def test_keys_read_once_per_chunk(bench):
    two_mul = alg_limbs(bench, [("mul", 23, 1), ("mul", 23, 1)])
    assert two_mul == (2 * 142 + 192, 192, 1)
    # two rotations by different steps use two keys; a trivial rotation (steps = 0) uses none
    assert alg_limbs(bench, [("rot", 23, 1), ("rot", 23, 2)]) == (2 * 96 + 2 * 192, 2 * 192, 1)
    assert alg_limbs(bench, [("rot", 23, 0)])[:2] == (96, 0)


def test_lower_levels_read_fewer_digits(bench):
    # 12 limbs: 2 digits, 12 + 8 limbs per key part and digit
    alg, key, _ = alg_limbs(bench, [("mul", 11, 1)])
    assert key == 2 * 2 * (12 + 8)
    assert alg == 4 * 12 + 2 * 11 + key


def test_chunks_of_at_most_128_ops(bench):
    ops = [("mul", 5, 1)] * 300
    alg, key, chunks = alg_limbs(bench, ops)
    assert chunks == 3 and key == 3 * 2 * 1 * (6 + 8)
