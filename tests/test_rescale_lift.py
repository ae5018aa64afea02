"""The rescale's one-source conversion as the NTT column pass computes it on load (kernels.cu
centred_lift, used when a column pass's LimbRef::aux names a source prime), replayed exactly on
the CPU. The reference's rescale (crates/ckks-train-core/src/baseconv.rs:258-291) adds
h = (q_l - 1) / 2 to the last limb mod q_l, lifts it to every other prime and subtracts h there;
the column pass takes the centred representative of x (x or x - q_l) and reduces it mod q_i with
one Shoup product by 1 (floor(2^64 / q_i)) and a conditional subtraction, then negates. Both must
give the same residue for every value, on every (last prime, target) pair of the chains.
"""

import numpy as np
import pytest

CHAINS = {
    "cfg2": (16, [50] * 24, [60] * 8),
    "n16_train": (16, [58] + [42] * 31, [58] * 4),
    "n16_boot": (16, [54] + [42] * 16 + [34] * 4 + [58] * 7 + [56] * 4, [60] * 4),
    "cfg1": (13, [45] * 4, [60]),
}

M64 = (1 << 64) - 1


def reference_lift(x, ql, qi):
    h = (ql - 1) // 2
    return (((x + h) % ql) - h) % qi


def kernel_lift(x, ql, qi):
    """centred_lift with 64-bit wrap-around arithmetic, step by step."""
    one_s = (1 << 64) // qi  # Shoup companion of 1
    neg = x > (ql >> 1)
    m = ql - x if neg else x
    qh = (m * one_s) >> 64  # __umul64hi
    r = (m * 1 - qh * qi) & M64  # mul_shoup_lazy: in [0, 2 qi)
    assert r < 2 * qi
    r = r - qi if r >= qi else r  # csub
    return qi - r if (neg and r) else r


@pytest.mark.parametrize("name", sorted(CHAINS))
def test_centred_lift_equals_the_reference_conversion(ckg, name):
    log_n, qb, pb = CHAINS[name]
    q, _ = ckg.primes_for_bits(log_n, qb, pb)
    rng = np.random.default_rng(31)
    pairs = 0
    for l in range(1, len(q)):
        ql = q[l]
        h = (ql - 1) // 2
        xs = [0, 1, h - 1, h, h + 1, ql - 2, ql - 1] + [int(v) for v in rng.integers(0, ql, 24, dtype=np.uint64)]
        for i in range(l):
            qi = q[i]
            pairs += 1
            for x in xs:
                assert kernel_lift(x, ql, qi) == reference_lift(x, ql, qi), (name, l, i, x)
    assert pairs == len(q) * (len(q) - 1) // 2
