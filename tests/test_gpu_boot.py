"""Device bootstrapping against the oracle's CPU bootstrap: the bootstrap arithmetic
(bootstrap/poly.rs:453-486), ModRaise with SSE (modraise.rs), CoeffToSlot / SlotToCoeff
(linear.rs:776-859), the level-optimal Chebyshev evaluation (poly.rs:655-714), EvalMod
(evalmod.rs:147-189) and the assembled bootstrap (bootstrapper.rs:385-473) give every
coefficient, level, scale and OpCounter of the CPU code on the same inputs.

Parameters: the reference's N = 2^10 bootstrap chain (bootstrapper.rs `mini()`: q = 54,
42 x 2, 34 x 4, 58 x 7, 56 x 4 bits, P = 2 x 60, scale 2^42, dnum 9) with the n16_boot
constants at log_slots 9 (K = 13, degree 127, r = 0, SSE h' = 32); the oracle generates the
keys and encodes the stages, as the reference's Bootstrapper::new does on the host.
"""

import numpy as np
import pytest

from gpu_util import assert_same, random_ct

pytestmark = pytest.mark.gpu

Q_BITS = [54, 42, 42] + [34] * 4 + [58] * 7 + [56] * 4
DELTA = 2.0 ** 42


class Boot:
    """The mini chain with keys from KeyGenerator::new(rng(seed)); with `public_key` the
    generator first draws a public key, as the reference's `fixture` (bootstrapper.rs:485-508)
    does before the relinearization key and Bootstrapper::new."""

    def __init__(self, ckg, O, seed=7, public_key=False):
        self.ckg, self.O = ckg, O
        P = self.P = O.Params.from_bits(10, Q_BITS, [60, 60], 42, 9)
        self.kg = O.KeyGenerator(P, seed)
        self.enc = O.Encoder(P)
        self.pk = self.kg.public_key() if public_key else None
        self.rk = self.kg.relin_key()
        self.bs = O.Bootstrapper(P, self.kg, self.enc, 9)
        self.ctx = ckg.Context(10, P.q, P.p, 9, scale=DELTA)
        self.d_rk = self.ctx.upload_key(self.rk.export())
        gk = self.bs.galois_keys()
        self.d_gk = [self.ctx.upload_key(k.export(), e) for e, k in gk.items()]
        ts, td = self.bs.sse_keys()
        self.d_ts, self.d_td = self.ctx.upload_key(ts.export()), self.ctx.upload_key(td.export())
        self.gpu = ckg.CudaEvaluator(self.ctx, self.d_rk, self.d_gk)
        self.cpu_inner = self.bs.inner_evaluator(self.rk)

        def stages(direction):
            out = []
            for info, es, es2 in self.bs.stages(direction):
                up = lambda lst: [self.gpu.upload_pt(e, info["pt_scale"]) if e is not None else None for e in lst]
                out.append(ckg.LinearTransform(direction, info["level"], info["scale"], info["d"], info["stride"],
                                               info["offset"], up(es), up(es2) if es2 is not None else None))
            return out

        self.ctos, self.stoc = stages(0), stages(1)
        self.coeffs = self.bs.coeffs()
        self.bp = ckg.BootParams(log_slots=9)
        em, si = self.bs.scales()
        self.scales = (em, si, DELTA)
        self.dev_bs = ckg.Bootstrapper(self.ctx, self.bp, self.ctos, self.stoc, self.d_gk, self.d_ts, self.d_td,
                                       self.coeffs, self.scales)

    def pair(self, data, scale, ev=None):
        ev = ev or self.cpu_inner
        return ev.ct(data, scale), self.gpu.upload_ct(data, scale)

    def check(self, cpu_ct, gpu_ct, what):
        got, gscale = self.gpu.download_ct(gpu_ct)
        assert gpu_ct.level() == cpu_ct.level, f"{what}: level {gpu_ct.level()} != {cpu_ct.level}"
        assert gscale == cpu_ct.scale, f"{what}: scale {gscale!r} != {cpu_ct.scale!r}"
        assert_same(got, cpu_ct.data(), what)

    def counters_equal(self, what):
        assert self.gpu.counter() == self.cpu_inner.counter(), \
            f"{what}: counters {self.gpu.counter()} != {self.cpu_inner.counter()}"

    def reset(self):
        self.gpu.reset_counter()
        self.cpu_inner.reset_counter()


@pytest.fixture(scope="module")
def boot(ckg, oracle):
    return Boot(ckg, oracle)


def test_boot_arithmetic(boot):
    P, O = boot.P, boot.O
    b = boot
    b.reset()
    L = P.max_level
    c, g = b.pair(random_ct(P, 11, L), 2.0 ** 58)
    for value, scale in [(1.0, 2.0 ** 116), (-0.375, 2.0 ** 100), (3.25e-3, 2.0 ** 80)]:
        b.check(O.boot_mul_const(b.cpu_inner, c, value, scale), b.gpu.boot_mul_const(g, value, scale),
                f"boot_mul_const {value}")
    for value in (-1.0, 0.5, 1e-3, 12345.678):
        b.check(O.boot_add_const(b.cpu_inner, c, value), b.gpu.boot_add_const(g, value), f"boot_add_const {value}")
    b.check(O.mul_by_x_half(b.cpu_inner, c), b.gpu.mul_by_x_half(g), "mul_by_x_half")
    z = b.gpu.boot_zero(5, 2.0 ** 40)
    data, sc = b.gpu.download_ct(z)
    assert z.level() == 5 and sc == 2.0 ** 40 and not data.any()
    b.counters_equal("boot arithmetic")
    with pytest.raises(b.ckg.InvalidParams):
        b.gpu.boot_mul_const(g, 1.0, 2.0 ** 60)  # constant scale 2^2 < 2^20


def test_mod_raise(boot):
    P, b = boot.P, boot
    b.reset()
    c, g = b.pair(random_ct(P, 21, 0), DELTA)
    want = b.bs.mod_raise(b.cpu_inner, c)
    got = b.gpu.mod_raise(g, b.d_ts, b.d_td)
    b.check(want, got, "mod_raise")
    b.counters_equal("mod_raise")
    _, g1 = b.pair(random_ct(P, 22, 1), DELTA)
    with pytest.raises(b.ckg.LevelMismatch):
        b.gpu.mod_raise(g1, b.d_ts, b.d_td)
    with pytest.raises(b.ckg.InvalidParams):
        b.gpu.mod_raise(g, b.d_td, b.d_ts)  # keys swapped


def test_coeff_to_slot_eval_mod_slot_to_coeff(boot):
    P, b = boot.P, boot
    b.reset()
    q0 = float(P.q[0])
    c, g = b.pair(random_ct(P, 31, P.max_level), q0)
    cre, cim = b.bs.coeff_to_slot(b.cpu_inner, c)
    gre, gim = b.gpu.coeff_to_slot(g, b.ctos)
    b.check(cre, gre, "coeff_to_slot re")
    b.check(cim, gim, "coeff_to_slot im")
    b.counters_equal("coeff_to_slot")
    # EvalMod on the CtS output (same inputs on both sides)
    ere = b.bs.eval_mod(b.cpu_inner, cre)
    gere = b.gpu.eval_mod(gre, b.bp, b.coeffs)
    b.check(ere, gere, "eval_mod")
    b.counters_equal("eval_mod")
    # SlotToCoeff from the planned input scale
    em, si = b.bs.scales()
    start = b.stoc[0].level
    re_c = b.cpu_inner.relabel(b.cpu_inner.mod_switch_to_level(ere, start), si)
    re_g = b.gpu.relabel(b.gpu.mod_switch_to_level(gere, start), si)
    im_c = b.cpu_inner.relabel(b.cpu_inner.mod_switch_to_level(ere, start), si)
    im_g = b.gpu.relabel(b.gpu.mod_switch_to_level(gere, start), si)
    b.check(b.bs.slot_to_coeff(b.cpu_inner, re_c, im_c), b.gpu.slot_to_coeff(re_g, im_g, b.stoc), "slot_to_coeff")
    b.counters_equal("slot_to_coeff")
    with pytest.raises(b.ckg.ScaleMismatch):
        b.gpu.coeff_to_slot(b.gpu.relabel(g, q0 * 2), b.ctos)
    with pytest.raises(b.ckg.InvalidParams):
        b.gpu.coeff_to_slot(g, b.stoc)  # wrong direction


def test_eval_chebyshev_series(boot):
    """Random series of several degrees, on [-1, 1] and on an affine interval."""
    P, O, b = boot.P, boot.O, boot
    rng = np.random.default_rng(5)
    for degree, (lo, hi) in [(7, (-1.0, 1.0)), (31, (-1.0, 1.0)), (5, (-2.0, 3.0)), (63, (-1.0, 1.0))]:
        b.reset()
        coeffs = rng.uniform(-1, 1, degree + 1) / (1 + np.arange(degree + 1))
        c, g = b.pair(random_ct(P, 40 + degree, 13), 2.0 ** 58)
        want = O.eval_chebyshev(b.cpu_inner, c, coeffs, lo, hi, 2.0 ** 58)
        got = b.gpu.eval_chebyshev(g, coeffs, lo, hi, 2.0 ** 58)
        b.check(want, got, f"eval_chebyshev degree {degree} on [{lo}, {hi}]")
        b.counters_equal(f"eval_chebyshev degree {degree}")


def test_bootstrap_bit_exact_and_precision(boot):
    P, O, b = boot.P, boot.O, boot
    rng = np.random.default_rng(11)
    m = rng.uniform(-1, 1, P.n // 2)
    pt = b.enc.encode(m, DELTA, P.max_level)
    ev_cpu = O.Evaluator(P, b.rk)
    ct = O.encrypt_sk(ev_cpu, b.kg, 9, pt, DELTA)
    ct0 = ev_cpu.mod_switch_to_level(ct, 0)
    ev_gpu = b.ckg.CudaEvaluator(b.ctx, b.d_rk, [])
    g0 = ev_gpu.upload_ct(ct0.data(), DELTA)
    want = b.bs.bootstrap(ev_cpu, ct0)
    got = b.dev_bs.bootstrap(ev_gpu, g0)
    data, scale = ev_gpu.download_ct(got)
    assert got.level() == want.level == b.bs.output_level() == b.dev_bs.output_level()
    assert scale == want.scale == DELTA
    assert_same(data, want.data(), "bootstrap")
    assert ev_gpu.counter() == ev_cpu.counter()
    assert ev_gpu.counter()["bootstraps"] == 1 and ev_gpu.counter()["sse_switches"] == 2
    dec = b.enc.decode(O.decrypt(b.kg, want), want.scale)
    bits = -np.log2(np.abs(dec.real - m).max())
    assert bits > 24.0, f"precision {bits:.2f} bits"  # the reference measures 26.77 on this chain


def test_reference_seeded_mini_bootstrap(ckg, oracle):
    """The reference's `mini_bootstrap_precision_level_and_counts` (bootstrapper.rs:539-574) in its
    random-stream order: keys from rng(1) (public key, relinearization key, Bootstrapper::new),
    then rng(2) draws m (`uniform`, :446-450) and the public-key encryptions (encrypt.rs:68-90).
    The device bootstrap is bit-identical to the oracle's, with the reference's output level,
    scale and counts, for one bootstrap and for a second one of a bootstrapped output. The
    reference prints 26.77 and 26.18 bits on this run; the oracle gives 26.80 and 26.02 (the
    inputs differ from the reference's only through the host math library of its encoder, or
    not at all: the reference's raw outputs are not published), and the reference's own
    gates (>= 16 and >= 15 bits) are asserted."""
    b = Boot(ckg, oracle, seed=1, public_key=True)
    P, O = b.P, oracle
    assert b.bs.output_level() == b.dev_bs.output_level() == 2
    r = O.Rng(2)
    m = r.uniform(P.n // 2, 1.0)
    ev_cpu = O.Evaluator(P, b.rk)
    ev_gpu = ckg.CudaEvaluator(b.ctx, b.d_rk, [])

    def level0():
        ct = O.encrypt_pk(ev_cpu, b.pk, r, b.enc.encode(m, DELTA, P.max_level), DELTA)
        return ev_cpu.mod_switch_to_level(ct, 0)

    def both(c):
        want = b.bs.bootstrap(ev_cpu, c)
        got = b.dev_bs.bootstrap(ev_gpu, ev_gpu.upload_ct(c.data(), c.scale))
        data, scale = ev_gpu.download_ct(got)
        assert got.level() == want.level == 2 and scale == want.scale == DELTA
        assert_same(data, want.data(), "seeded bootstrap")
        assert ev_gpu.counter() == ev_cpu.counter()
        return want

    out = both(level0())
    c = ev_gpu.counter()
    assert (c["rotations"], c["relins"], c["sse_switches"], c["bootstraps"]) == (37, 40, 2, 1)
    bits = O.precision_bits(m, b.enc.decode(O.decrypt(b.kg, out), out.scale).real)
    out2 = both(level0())
    twice = both(ev_cpu.mod_switch_to_level(out2, 0))
    bits2 = O.precision_bits(m, b.enc.decode(O.decrypt(b.kg, twice), twice.scale).real)
    assert ev_gpu.counter()["bootstraps"] == 3
    print(f"seeded mini bootstrap: {bits:.2f} bits, twice {bits2:.2f} bits (reference: 26.77, 26.18)")
    assert bits >= 16.0 and bits2 >= 15.0
    assert abs(bits - 26.77) < 0.1 and abs(bits2 - 26.18) < 0.25


def test_bootstrap_errors(boot):
    P, b = boot.P, boot
    ev = b.ckg.CudaEvaluator(b.ctx, b.d_rk, [])
    g1 = ev.upload_ct(random_ct(P, 51, 1), DELTA)
    with pytest.raises(b.ckg.InvalidParams):
        b.dev_bs.bootstrap(ev, g1)  # not at level 0
    g0 = ev.upload_ct(random_ct(P, 52, 0), DELTA * 2)
    with pytest.raises(b.ckg.ScaleMismatch):
        b.dev_bs.bootstrap(ev, g0)
    no_rk = b.ckg.CudaEvaluator(b.ctx, None, [])
    with pytest.raises(b.ckg.InvalidParams):
        b.dev_bs.bootstrap(no_rk, no_rk.upload_ct(random_ct(P, 53, 0), DELTA))
    assert ev.counter()["bootstraps"] == 0


N16_Q = [54] + [42] * 16 + [34] * 4 + [58] * 7 + [56] * 4  # params.rs n16_boot


def test_n16_boot_bootstrap(ckg, oracle):
    """The reference's n16_boot precision gate (`n16_boot_keys_bootstrap`, bootstrapper.rs:860-905)
    in its random-stream order: keys from rng(38) (public key, relinearization key,
    Bootstrapper::new with BootParams::default_n16), then rng(39) draws m and the public-key
    encryption. The library encodes its own stages and EvalMod series; the bootstrap is
    bit-identical to the oracle's, performs the reference's 111 key switches (69 rotations,
    40 relinearizations, 2 SSE switches, docs/bootstrap.md §11.2) and gives the oracle's
    precision: 17.52 bits, against the 17.46 the reference prints for this run (gate 16)."""
    import time
    P = oracle.Params.from_bits(16, N16_Q, [60] * 4, 42, 8)
    kg = oracle.KeyGenerator(P, 38)
    enc = oracle.Encoder(P)
    pk = kg.public_key()
    rk = kg.relin_key()
    bs = oracle.Bootstrapper(P, kg, enc, 15)
    ctx = ckg.Context(16, P.q, P.p, 8, scale=DELTA)
    d_rk = ctx.upload_key(rk.export())
    d_gk = [ctx.upload_key(k.export(), e) for e, k in bs.galois_keys().items()]
    ts, td = bs.sse_keys()
    d_ts, d_td = ctx.upload_key(ts.export()), ctx.upload_key(td.export())
    ev_gpu = ckg.CudaEvaluator(ctx, d_rk, [])
    dev = ckg.Bootstrapper.encoded(ev_gpu, ckg.BootParams(), DELTA, d_gk, d_ts, d_td)
    assert dev.output_level() == bs.output_level() == 16
    r = oracle.Rng(39)
    m = r.uniform(P.n // 2, 1.0)
    ev_cpu = oracle.Evaluator(P, rk)
    ct = oracle.encrypt_pk(ev_cpu, pk, r, enc.encode(m, DELTA, P.max_level), DELTA)
    ct0 = ev_cpu.mod_switch_to_level(ct, 0)
    g0 = ev_gpu.upload_ct(ct0.data(), DELTA)
    got = dev.bootstrap(ev_gpu, g0)  # warm-up (Galois tables, pools)
    ev_gpu.reset_counter()
    ctx.sync()
    t = time.perf_counter()
    got = dev.bootstrap(ev_gpu, g0)
    ctx.sync()
    ms = (time.perf_counter() - t) * 1e3
    want = bs.bootstrap(ev_cpu, ct0)
    data, scale = ev_gpu.download_ct(got)
    assert scale == want.scale == DELTA and got.level() == want.level == 16
    assert_same(data, want.data(), "n16_boot bootstrap")
    c = ev_gpu.counter()
    assert c == ev_cpu.counter()
    assert (c["rotations"], c["relins"], c["sse_switches"], c["bootstraps"]) == (69, 40, 2, 1)
    bits = oracle.precision_bits(m, enc.decode(oracle.decrypt(kg, want), want.scale).real)
    print(f"n16_boot bootstrap on the GPU: {ms:.1f} ms wall (host-synchronised), precision {bits:.2f} bits "
          "(reference: 17.46)")
    assert bits >= 16.0 and abs(bits - 17.46) < 0.1
