"""GPU parity of key switching and of the HeOps evaluator against the oracle's CPU
Evaluator: every coefficient, the level, the f64 scale bits and the OpCounter must be
equal, and failures must raise the same error kind before any work is counted
(crates/ckks-train-cuda/tests/cases/{ks,eval}.rs, crates/ckks-train-ckks/src/evaluator.rs).
"""

import itertools

import numpy as np
import pytest

from gpu_util import PARAM_SETS, assert_same, empty_dev, from_dev, make_pair, ptr, random_ct, to_dev

pytestmark = pytest.mark.gpu


class Env:
    """Oracle and GPU evaluators with the same keys (Galois keys for `steps` + conjugation)."""

    def __init__(self, ckg, O, name, steps, seed=42, config=(True, True, True)):
        self.ckg, self.O = ckg, O
        self.P, self.ctx = make_pair(ckg, O, name)
        P = self.P
        self.scale = float(2.0 ** PARAM_SETS[name]["scale_bits"])
        kg = O.KeyGenerator(P, seed)
        self.rk = kg.relin_key()
        elts = sorted({O.galois_elt(P.n, s) for s in steps if O.galois_elt(P.n, s) != 1} | {2 * P.n - 1})
        self.gk = {e: kg.galois_key(e) for e in elts}
        self.d_rk = self.ctx.upload_key(self.rk.export())
        self.d_gk = [self.ctx.upload_key(self.gk[e].export(), e) for e in elts]
        self.set_config(*config)

    def set_config(self, hoist, bsgs, lazy):
        O, ckg = self.O, self.ckg
        self.cpu = O.Evaluator(self.P, self.rk, self.gk, hoist=hoist, bsgs=bsgs, lazy_relin=lazy)
        self.gpu = ckg.CudaEvaluator(self.ctx, self.d_rk, self.d_gk, ckg.EvalConfig(hoist, bsgs, lazy))

    def pair(self, data, scale=None):
        scale = self.scale if scale is None else scale
        return self.cpu.ct(data, scale), self.gpu.upload_ct(data, scale)

    def check(self, cpu_ct, gpu_ct, what):
        got, gscale = self.gpu.download_ct(gpu_ct)
        want = cpu_ct.data()
        assert gpu_ct.level() == cpu_ct.level, f"{what}: level"
        assert gscale == cpu_ct.scale, f"{what}: scale {gscale!r} != {cpu_ct.scale!r}"
        assert_same(got, want, what)
        assert self.gpu.counter() == self.cpu.counter(), f"{what}: counters {self.gpu.counter()} != {self.cpu.counter()}"


@pytest.fixture(scope="module", params=["tiny", "small", "cfg1"])
def env(request, ckg, oracle):
    name = request.param
    slots = (1 << PARAM_SETS[name]["log_n"]) // 2
    steps = [1, -1, 2, 3, 4, 8, 12, slots // 2]
    return Env(ckg, oracle, name, steps)


def test_key_switch_raw(env):
    P, ctx = env.P, env.ctx
    for i, level in enumerate(sorted({P.max_level, P.max_level // 2, 0})):
        d = P.random_q(800 + i, level)
        dd = to_dev(d)
        ob, oa = empty_dev(d.shape), empty_dev(d.shape)
        ctx.key_switch(env.d_rk, ptr(dd), level, ptr(ob), ptr(oa))
        ctx.sync()
        wb, wa = env.rk.key_switch(d)
        assert_same(from_dev(ob), wb, f"key_switch b level {level}")
        assert_same(from_dev(oa), wa, f"key_switch a level {level}")


def test_key_switch_raw_unaligned(env):
    """Caller buffers one word off a 16-byte boundary (tensor slices at odd offsets): the input's
    own-digit limbs take the word-pair loads of the inner product, and the outputs are written
    at odd word offsets, with the aligned call's result."""
    P, ctx = env.P, env.ctx
    level = P.max_level
    d = P.random_q(900, level)
    n_words = d.size
    dd = to_dev(np.concatenate([np.zeros(1, np.uint64), d.ravel()]))
    out = empty_dev((2 * n_words + 4,))
    assert ptr(dd) % 16 == 0 and ptr(out) % 16 == 0
    ob, oa = ptr(out) + 8, ptr(out) + 8 * (n_words + 3)
    ctx.key_switch(env.d_rk, ptr(dd) + 8, level, ob, oa)
    ctx.sync()
    got = from_dev(out)
    wb, wa = env.rk.key_switch(d)
    assert_same(got[1:1 + n_words].reshape(d.shape), wb, "unaligned key_switch b")
    assert_same(got[n_words + 3:2 * n_words + 3].reshape(d.shape), wa, "unaligned key_switch a")


def test_arithmetic_ops(env):
    P = env.P
    L = P.max_level
    env.cpu.reset_counter()
    env.gpu.reset_counter()
    a_cpu, a_gpu = env.pair(random_ct(P, 1, L))
    b_cpu, b_gpu = env.pair(random_ct(P, 2, L))
    env.check(env.cpu.add(a_cpu, b_cpu), env.gpu.add(a_gpu, b_gpu), "add")
    env.check(env.cpu.sub(a_cpu, b_cpu), env.gpu.sub(a_gpu, b_gpu), "sub")
    env.check(env.cpu.negate(a_cpu), env.gpu.negate(a_gpu), "negate")
    t_cpu, t_gpu = env.cpu.mul_no_relin(a_cpu, b_cpu), env.gpu.mul_no_relin(a_gpu, b_gpu)
    env.check(t_cpu, t_gpu, "mul_no_relin")
    # 3 + 2 component add / sub (lazy relinearization pattern), at the product's scale
    ar_cpu, ar_gpu = env.cpu.relabel(a_cpu, t_cpu.scale), env.gpu.relabel(a_gpu, t_gpu.scale())
    env.check(env.cpu.add(t_cpu, ar_cpu), env.gpu.add(t_gpu, ar_gpu), "add 3+2")
    env.check(env.cpu.sub(ar_cpu, t_cpu), env.gpu.sub(ar_gpu, t_gpu), "sub 2-3")
    r_cpu, r_gpu = env.cpu.relinearize(t_cpu), env.gpu.relinearize(t_gpu)
    env.check(r_cpu, r_gpu, "relinearize")
    m_cpu, m_gpu = env.cpu.mul(a_cpu, b_cpu), env.gpu.mul(a_gpu, b_gpu)
    env.check(m_cpu, m_gpu, "mul")
    env.check(env.cpu.rescale(m_cpu), env.gpu.rescale(m_gpu), "rescale")
    env.check(env.cpu.rescale(t_cpu), env.gpu.rescale(t_gpu), "rescale 3 components")
    env.check(env.cpu.mod_switch_to_level(a_cpu, L // 2), env.gpu.mod_switch_to_level(a_gpu, L // 2), "mod_switch")
    env.check(env.cpu.relabel(a_cpu, 3.5), env.gpu.relabel(a_gpu, 3.5), "relabel")
    pt = P.random_q(33, L)
    env.check(env.cpu.add_plain(a_cpu, pt, env.scale), env.gpu.add_plain(a_gpu, env.gpu.upload_pt(pt, env.scale)),
              "add_plain")
    env.check(env.cpu.mul_plain(a_cpu, pt, env.scale), env.gpu.mul_plain(a_gpu, env.gpu.upload_pt(pt, env.scale)),
              "mul_plain")
    if L >= 1:
        for value in (0.5, -0.3125, 0.0, -1.0):
            env.check(env.cpu.mul_scalar(a_cpu, value, env.scale), env.gpu.mul_scalar(a_gpu, value, env.scale),
                      f"mul_scalar {value}")
        sp = env.cpu.exact_product_scale(L, env.scale) / env.scale
        assert env.gpu.exact_product_scale(L, env.scale) == env.cpu.exact_product_scale(L, env.scale)
        env.check(env.cpu.mul_plain_to_scale(a_cpu, pt, sp, env.scale),
                  env.gpu.mul_plain_to_scale(a_gpu, env.gpu.upload_pt(pt, sp), env.scale), "mul_plain_to_scale")
    # lower-level operands
    low = max(L // 2, 1)
    c_cpu, c_gpu = env.pair(random_ct(P, 3, low))
    d_cpu, d_gpu = env.pair(random_ct(P, 4, low))
    e_cpu, e_gpu = env.cpu.mul(c_cpu, d_cpu), env.gpu.mul(c_gpu, d_gpu)
    env.check(e_cpu, e_gpu, f"mul level {low}")
    env.check(env.cpu.rescale(e_cpu), env.gpu.rescale(e_gpu), f"rescale level {low}")


def test_rotations(env):
    P = env.P
    L = P.max_level
    slots = P.n // 2
    env.cpu.reset_counter()
    env.gpu.reset_counter()
    for level in sorted({L, L // 2, 0}):
        a_cpu, a_gpu = env.pair(random_ct(P, 10 + level, level))
        for s in (1, -1, 2, 3, slots // 2, 0, slots):
            env.check(env.cpu.rotate(a_cpu, s), env.gpu.rotate(a_gpu, s), f"rotate {s} level {level}")
        env.check(env.cpu.conjugate(a_cpu), env.gpu.conjugate(a_gpu), f"conjugate level {level}")
        steps = [0, 1, 2, 3, -1, 8, 12, slots, 1]
        hc, hg = env.cpu.hoisted_rotate(a_cpu, steps), env.gpu.hoisted_rotate(a_gpu, steps)
        for s, c, g in zip(steps, hc, hg):
            env.check(c, g, f"hoisted_rotate step {s} level {level}")
        # hoisted == individual rotations, bit for bit
        for s, g in zip(steps, hg):
            want, _ = env.gpu.download_ct(env.gpu.rotate(a_gpu, s))
            got, _ = env.gpu.download_ct(g)
            assert_same(got, want, f"hoisted vs direct step {s}")
        env.cpu.reset_counter()
        env.gpu.reset_counter()


def _err(fn):
    try:
        fn()
    except Exception as e:  # noqa: BLE001
        return type(e).__name__.replace("OracleError", "")
    return None


def test_errors_match(env):
    """Same error kinds, checked before work, nothing counted (evaluator.rs:1-29)."""
    O, ckg = env.O, env.ckg
    P = env.P
    L = P.max_level
    a_cpu, a_gpu = env.pair(random_ct(P, 21, L))
    b_cpu, b_gpu = env.pair(random_ct(P, 22, max(L - 1, 0)))
    s_cpu, s_gpu = env.pair(random_ct(P, 23, L), env.scale * 3.0)
    z_cpu, z_gpu = env.pair(random_ct(P, 24, 0))
    t_cpu, t_gpu = env.cpu.mul_no_relin(a_cpu, a_cpu), env.gpu.mul_no_relin(a_gpu, a_gpu)
    env.cpu.reset_counter()
    env.gpu.reset_counter()
    cases = [
        ("add level", lambda e, a, b, s, z, t: e.add(a, b)),
        ("add scale", lambda e, a, b, s, z, t: e.add(a, s)),
        ("mul level", lambda e, a, b, s, z, t: e.mul(a, b)),
        ("mul level 0", lambda e, a, b, s, z, t: e.mul(z, z)),
        ("rescale level 0", lambda e, a, b, s, z, t: e.rescale(z)),
        ("mul 3 comps", lambda e, a, b, s, z, t: e.mul(t, a)),
        ("relin 2 comps", lambda e, a, b, s, z, t: e.relinearize(a)),
        ("rotate 3 comps", lambda e, a, b, s, z, t: e.rotate(t, 1)),
        ("missing key", lambda e, a, b, s, z, t: e.rotate(a, 5)),
        ("hoisted missing key", lambda e, a, b, s, z, t: e.hoisted_rotate(a, [1, 5])),
        ("mod switch up", lambda e, a, b, s, z, t: e.mod_switch_to_level(b, L)),
        ("relabel", lambda e, a, b, s, z, t: e.relabel(a, -1.0)),
        ("mul_scalar level 0", lambda e, a, b, s, z, t: e.mul_scalar(z, 0.5, 1.0)),
        ("mul_scalar nan", lambda e, a, b, s, z, t: e.mul_scalar(a, float("nan"), 1.0)),
        ("mul_scalar tiny", lambda e, a, b, s, z, t: e.mul_scalar(a, 0.5, 1e-30)),
    ]
    kinds = {"InvalidParams": "InvalidParams", "ScaleMismatch": "ScaleMismatch", "LevelMismatch": "LevelMismatch",
             "NoLevelsLeft": "NoLevelsLeft"}
    for name, fn in cases:
        ce = _err(lambda: fn(env.cpu, a_cpu, b_cpu, s_cpu, z_cpu, t_cpu))
        ge = _err(lambda: fn(env.gpu, a_gpu, b_gpu, s_gpu, z_gpu, t_gpu))
        if ce is None:
            assert ge is None, f"{name}: GPU raised {ge}, oracle succeeded"
            continue
        import oracle as OO
        try:
            fn(env.cpu, a_cpu, b_cpu, s_cpu, z_cpu, t_cpu)
        except OO.OracleError as e:
            want = e.kind
        assert ge == kinds.get(want, want), f"{name}: GPU {ge}, oracle {want}"
    assert env.gpu.counter() == env.cpu.counter()
    assert sum(env.gpu.counter().values()) == 0


@pytest.mark.parametrize("cfg", list(itertools.product([True, False], repeat=3)))
def test_matvec_configs(env, cfg):
    """matvec_plain / matvec_enc under every EvalConfig: same ciphertexts and counts
    (crates/ckks-train-ckks/src/ops.rs:136-161, linalg.rs:608-680)."""
    P = env.P
    env.set_config(*cfg)
    L = P.max_level
    if L < 1:
        pytest.skip("needs a level above 0")
    d = 4 if P.n // 2 < 64 else 16
    x_cpu, x_gpu = env.pair(random_ct(P, 31, L))
    pts = np.stack([P.random_q(300 + i, L) for i in range(d)])
    env.cpu.reset_counter()
    env.gpu.reset_counter()
    env.check(env.cpu.matvec_plain(d, 1, pts, env.scale, x_cpu),
              env.gpu.matvec_plain(d, 1, [env.gpu.upload_pt(p, env.scale) for p in pts], x_gpu), f"matvec_plain {cfg}")
    cts = [env.pair(random_ct(P, 400 + i, L)) for i in range(d)]
    env.check(env.cpu.matvec_enc(d, 1, [c for c, _ in cts], x_cpu),
              env.gpu.matvec_enc(d, 1, [g for _, g in cts], x_gpu), f"matvec_enc {cfg}")
    env.set_config(True, True, True)


def test_key_switch_cfg2(ckg, oracle):
    """Full-size key switch: N = 2^16, 24 data limbs, 8 special primes, dnum 3."""
    P, ctx = make_pair(ckg, oracle, "cfg2")
    kg = oracle.KeyGenerator(P, 7)
    rk = kg.relin_key()
    d_rk = ctx.upload_key(rk.export())
    assert d_rk.nbytes == 3 * 2 * 32 * (1 << 16) * 8
    for level in (23, 12):
        d = P.random_q(900 + level, level)
        dd = to_dev(d)
        ob, oa = empty_dev(d.shape), empty_dev(d.shape)
        ctx.key_switch(d_rk, ptr(dd), level, ptr(ob), ptr(oa))
        ctx.sync()
        wb, wa = rk.key_switch(d)
        assert_same(from_dev(ob), wb, f"cfg2 key_switch b level {level}")
        assert_same(from_dev(oa), wa, f"cfg2 key_switch a level {level}")


def test_matvec_batches(env):
    """matvec_enc_batch (crates/ckks-train-cuda/src/evaluator.rs:437-520) and its plaintext twin:
    jobs of several sizes, strides and levels give the oracle's matvec_enc / matvec_plain result
    for each job, bit for bit, and the counters of the jobs run one by one, under every
    EvalConfig; a failing job fails the whole call before any work, with nothing counted."""
    P = env.P
    L = P.max_level
    if L < 1:
        pytest.skip("needs a level above 0")
    big = 4 if P.n // 2 < 64 else 16
    specs = [(big, 1, L), (8, 1, max(L // 2, 1)), (4, 2, L), (4, 1, 1)]
    for cfg in itertools.product([True, False], repeat=3):
        env.set_config(*cfg)
        for kind in ("enc", "plain"):
            env.cpu.reset_counter()
            env.gpu.reset_counter()
            want, jobs = [], []
            for n, (d, stride, level) in enumerate(specs):
                x_c, x_g = env.pair(random_ct(P, 500 + n, level))
                if kind == "enc":
                    ents = [env.pair(random_ct(P, 600 + 20 * n + i, level)) for i in range(d)]
                    want.append(env.cpu.matvec_enc(d, stride, [c for c, _ in ents], x_c))
                    jobs.append((d, stride, [g for _, g in ents], x_g))
                else:
                    pts = np.stack([P.random_q(700 + 20 * n + i, level) for i in range(d)])
                    want.append(env.cpu.matvec_plain(d, stride, pts, env.scale, x_c))
                    jobs.append((d, stride, [env.gpu.upload_pt(p, env.scale) for p in pts], x_g))
            got = (env.gpu.matvec_enc_batch if kind == "enc" else env.gpu.matvec_plain_batch)(jobs)
            for n, (w, g) in enumerate(zip(want, got)):
                data, scale = env.gpu.download_ct(g)
                assert g.level() == w.level and scale == w.scale, f"job {n}"
                assert_same(data, w.data(), f"matvec_{kind}_batch job {n} {cfg}")
            assert env.gpu.counter() == env.cpu.counter(), f"matvec_{kind}_batch counters {cfg}"
    env.set_config(True, True, True)
    # the first failing job fails the call: nothing runs, nothing is counted
    env.gpu.reset_counter()
    x_hi = env.gpu.upload_ct(random_ct(P, 801, L), env.scale)
    x_lo = env.gpu.upload_ct(random_ct(P, 802, L - 1), env.scale)
    ents = [env.gpu.upload_ct(random_ct(P, 810 + i, L), env.scale) for i in range(4)]
    with pytest.raises(env.ckg.LevelMismatch):
        env.gpu.matvec_enc_batch([(4, 1, ents, x_hi), (4, 1, ents, x_lo)])
    assert sum(env.gpu.counter().values()) == 0
