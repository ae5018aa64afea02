"""The FP64-assisted forms of exact base conversion (kernels.cu k_bconv, admitted per target by
engine.cu conv_f64_form) and of the key-switch inner product (k_inner_product, admitted per
prime by engine.cu ip_f64_offset), replayed in exact arithmetic on the CPU: FMA and every rounding
emulated with Fractions (float(Fraction) rounds to nearest even), on the prime chains of the
configurations and with the sources at their extremes. For every admitted target the residual
r = V - rint(A) t must stay within the admission bound, and the second rounded quotient plus
one conditional add must give exactly V mod t (crates/ckks-train-core/src/baseconv.rs:167-235
defines V mod t: sum_j y_j [S/s_j]_t - e [S]_t - [h]_t).
"""

import math
from fractions import Fraction

import numpy as np
import pytest

CHAINS = {
    "cfg2": (16, [50] * 24, [60] * 8, 3),
    "n16_train": (16, [58] + [42] * 31, [58] * 4, 8),
    "n16_boot": (16, [54] + [42] * 16 + [34] * 4 + [58] * 7 + [56] * 4, [60] * 4, 8),
    "cfg1": (13, [45] * 4, [60], 4),
}


def fl(x):
    return float(x)  # Fraction -> nearest double (ties to even)


def fma(a, b, c):
    return fl(Fraction(a) * Fraction(b) + Fraction(c))


def rint(x):
    return int(round(Fraction(x)))  # round half to even


def admitted(src, t):
    """conv_f64_form: (admitted, two_stage)."""
    if not src or len(src) > 8 or t < 2 ** 30:
        return False, False
    e2 = 3 if t >= 2 ** 53 else 1
    s = sum(src)
    rep = sum(v * (e2 + (1 if v > 2 ** 53 else 0)) for v in src)
    amax = (s + 17 + 64) * (1 + 2.0 ** -40)
    ulp = 2.0 ** (math.floor(math.log2(amax)) - 52)
    eta = rep * 2.0 ** -53 + (len(src) + 2) * ulp / 2 + 17 * 2.0 ** -52 + 2.0 ** -30
    return (eta + 0.5) * t <= 2.0 ** 62, eta >= 0.5, eta + 0.5


def conversions(q, p, dnum):
    """(sources, targets) of ModUp per (level, digit), ModDown and rescale per level."""
    alpha = len(q) // dnum
    for l in range(len(q)):
        for j in range((l + 1 + alpha - 1) // alpha):
            lo, hi = j * alpha, min((j + 1) * alpha, l + 1)
            yield "modup", q[lo:hi], [q[i] for i in range(l + 1) if not lo <= i < hi] + list(p)
        yield "moddown", list(p), q[:l + 1]
        if l >= 1:
            yield "rescale", [q[l]], q[:l]


def replay(src, t, ys):
    S = math.prod(src)
    h = (S - 1) // 2
    w = [(S // s) % t for s in src]
    e = int(sum(Fraction(y) / s for y, s in zip(ys, src))) if len(src) > 1 else 0
    V = sum(y * wj for y, wj in zip(ys, w)) + e * (t - S % t) + (t - h % t)
    A = 0.0
    for y, wj in zip(ys, w):
        A = fma(fl(y), fl(Fraction(fl(wj)) / Fraction(fl(t))), A)
    A = fma(float(e), fl(Fraction(fl(t - S % t)) / Fraction(fl(t))), A)
    A = fl(Fraction(A) + Fraction(fl(Fraction(fl(t - h % t)) / Fraction(fl(t)))))
    k = rint(A)
    r = V - k * t
    return V, r


@pytest.mark.parametrize("name", sorted(CHAINS))
def test_fp64_assisted_conversion_bound(ckg, name):
    log_n, qb, pb, dnum = CHAINS[name]
    q, p = ckg.primes_for_bits(log_n, qb, pb)
    rng = np.random.default_rng(7)
    seen = {"f64": 0, "exact": 0, "two_stage": 0}
    checked = set()
    for kind, src, dst in conversions(q, p, dnum):
        for t in dst:
            ok, two, bound = admitted(src, t)
            seen["f64" if ok else "exact"] += 1
            key = (tuple(src), t)
            if not ok or key in checked:
                continue
            checked.add(key)
            seen["two_stage"] += two
            trials = [[s - 1 for s in src], [s // 2 for s in src],
                      [int(x) for x in rng.integers(0, 2 ** 62, len(src)) % np.array(src, dtype=object)]]
            for ys in trials:
                V, r = replay(src, t, ys)
                assert abs(r) <= bound * t <= 2 ** 62, (kind, src, t)
                if two:
                    qinv = fl(Fraction(1) / Fraction(fl(t)))
                    r -= rint(fl(Fraction(fl(r)) * Fraction(qinv))) * t
                else:
                    assert abs(r) < t
                assert -t < r < t
                if r < 0:
                    r += t
                assert r == V % t, (kind, src, t)
    assert seen["f64"] > 0
    if name == "cfg2":  # data-prime targets of ModUp and the rescale are admitted, 60-bit ones not
        assert seen["exact"] > 0 and seen["two_stage"] > 0


def ip_offset(q, beta):
    """engine.cu ip_f64_offset."""
    if q >= 2 ** 50:
        return 0
    amax = beta * q * (1 + 2.0 ** -40) + 64
    if amax >= 2.0 ** 52:
        return 0
    ulp = 2.0 ** (math.floor(math.log2(amax)) - 52)
    delta = beta * q * 2.0 ** -52 + beta * ulp / 2 + 0.5 + 2.0 ** -30
    off = math.ceil(delta)
    return 0 if (off + delta) * q >= 2.0 ** 53 else off


@pytest.mark.parametrize("name", sorted(CHAINS))
def test_fp64_assisted_inner_product(ckg, name):
    """k_inner_product's FP64-assisted form (ip_finish_f64) replayed exactly: for every admitted
    prime and digit count up to dnum, extreme and random digits and key words give V mod q."""
    log_n, qb, pb, dnum = CHAINS[name]
    q, p = ckg.primes_for_bits(log_n, qb, pb)
    rng = np.random.default_rng(9)
    admitted_primes = 0
    for prime in sorted(set(q) | set(p)):
        off = ip_offset(prime, dnum)
        if not off:
            continue
        admitted_primes += 1
        qinv = fl(Fraction(1) / Fraction(prime))
        for beta in range(1, dnum + 1):
            trials = [([prime - 1] * beta, [prime - 1] * beta),
                      ([int(x) % prime for x in rng.integers(0, 2 ** 62, beta)],
                       [int(x) % prime for x in rng.integers(0, 2 ** 62, beta)])]
            for ds, ks in trials:
                V = sum(d * k for d, k in zip(ds, ks))
                A = 0.0
                for d, k in zip(ds, ks):
                    A = fma(float(d), fl(Fraction(float(k)) * Fraction(qinv)), A)
                assert 0 <= A < 2 ** 52
                x = V - rint(A) * prime + off * prime
                assert 0 <= x < 2 ** 53
                r = x - rint(fl(Fraction(float(x)) * Fraction(qinv))) * prime
                assert -prime < r < prime
                assert (r + prime if r < 0 else r) == V % prime
    assert admitted_primes > 0
