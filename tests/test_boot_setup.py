"""Host-side bootstrap setup, no GPU: the library's encoder, stage layouts, rotation steps
and EvalMod series against the oracle (which restates encoder.rs, bootstrap/linear.rs and
bootstrap/evalmod.rs), and both against the n16_boot layout and counts the reference
documents for its bootstrap (docs/bootstrap.md §9.2-9.3, §10.1, §11.2).
"""

import numpy as np
import pytest

MINI_Q = [54, 42, 42] + [34] * 4 + [58] * 7 + [56] * 4  # bootstrapper.rs `mini()`, N = 2^10
N16_Q = [54] + [42] * 16 + [34] * 4 + [58] * 7 + [56] * 4  # params.rs n16_boot


def _transform_cost(stages, slots, ctos):
    """sparse_transform_cost over stage layouts (linear.rs:679-755): (key switches,
    plaintext products), with CoeffToSlot's two conjugations."""
    rot = prod = 0
    for d, stride, offset, kept, kept2 in stages:
        log_d = d.bit_length() - 1
        baby = 1 << ((log_d + 1) // 2)
        giant = d // baby
        terms = [kept] + ([kept2] if kept2 is not None else [])
        for t in terms:
            prod += sum(t)
            for j in range(1, baby):
                if (j * stride) % slots and any(t[k * baby + j] for k in range(giant)):
                    rot += 1
        for k in range(giant):
            step = ((offset + baby * k) * stride) % slots
            if step and any(t[k * baby + j] for t in terms for j in range(baby)):
                rot += 1
        if ctos and kept2 is not None:
            rot += 1
    if ctos:
        rot += 1
    return rot, prod


def test_encoder_matches_oracle(ckg, oracle):
    rng = np.random.default_rng(3)
    for log_n, q_bits, p_bits, scale_bits, dnum in [(10, MINI_Q, [60, 60], 42, 9), (16, N16_Q, [60] * 4, 42, 8)]:
        P = oracle.Params.from_bits(log_n, q_bits, p_bits, scale_bits, dnum)
        enc = oracle.Encoder(P)
        slots = P.n // 2
        cases = [
            (rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots), 2.0 ** 42, P.max_level),
            (rng.uniform(-1, 1, slots // 3), 2.0 ** 34, 5),
            (rng.uniform(-1e3, 1e3, slots) + 1j * rng.uniform(-1e3, 1e3, slots), 2.0 ** 70, P.max_level),  # >= 2^63
        ]
        for vals, scale, level in cases:
            want = P.ntt(enc.encode(vals, scale, level), inverse=True)
            got = ckg.encode_complex_host(log_n, P.q, vals, scale, level)
            assert np.array_equal(got, want), f"encode N=2^{log_n} scale {scale} level {level}"
        with pytest.raises(ckg.InvalidParams):
            ckg.encode_complex_host(log_n, P.q, [1e30], 2.0 ** 60, 0)  # does not fit in Q/2


def test_mini_setup_matches_oracle(ckg, oracle):
    P = oracle.Params.from_bits(10, MINI_Q, [60, 60], 42, 9)
    bs = oracle.Bootstrapper(P, oracle.KeyGenerator(P, 7), oracle.Encoder(P), 9)
    bp = ckg.BootParams(log_slots=9)
    assert ckg.boot_rotation_steps(bp) == bs.rotation_steps()
    got = ckg.evalmod_coeffs(bp)
    assert got.tobytes() == bs.coeffs().tobytes()
    assert all(got[0::2] == 0.0)
    for direction in (0, 1):
        plan = ckg.boot_plan(bp, direction)
        assert plan == oracle.boot_plan(9, 4, 4, 13, direction)
        for (d, stride, offset, kept, kept2), (info, es, es2) in zip(plan, bs.stages(direction)):
            assert (d, stride, offset) == (info["d"], info["stride"], info["offset"])
            assert kept == [e is not None for e in es]
            assert (kept2 is None) == (es2 is None)
            if es2 is not None:
                assert kept2 == [e is not None for e in es2]


def test_n16_boot_layouts_and_counts(ckg, oracle):
    """docs/bootstrap.md §9.2-9.3: layouts (d, stride, offset) from distance 1 upward
    (16, 1, -8), (32, 8, -16), (32, 128, -16), (16, 2048, 0); 32 rotation steps;
    CoeffToSlot 34 key switches (2 conjugations) and 93 plaintext products, SlotToCoeff
    35 and 108; §10.1: the degree-127 series is odd."""
    bp = ckg.BootParams()
    slots = 1 << 15
    assert len(ckg.boot_rotation_steps(bp)) == 32
    stoc = ckg.boot_plan(bp, 1)
    ctos = ckg.boot_plan(bp, 0)
    assert stoc == oracle.boot_plan(15, 4, 4, 13, 1)
    assert ctos == oracle.boot_plan(15, 4, 4, 13, 0)
    layouts = [(16, 1, -8), (32, 8, -16), (32, 128, -16), (16, 2048, 0)]
    assert [s[:3] for s in stoc] == layouts
    assert [s[:3] for s in ctos] == layouts[::-1]
    assert _transform_cost(ctos, slots, True) == (34, 93)
    assert _transform_cost(stoc, slots, False) == (35, 108)
    c = ckg.evalmod_coeffs(bp)
    assert len(c) == 128 and all(c[0::2] == 0.0) and np.abs(c[1::2]).max() > 0.1
