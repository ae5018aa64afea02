"""Serving loop: requests from several key owners, admitted by HBM budget with LRU key
spill to pinned host memory and run with continuous batching, give every ciphertext
bit-identical to the oracle's CPU evaluator and to the same op run alone on the GPU, with
each owner's OpCounter equal to the CPU's for that owner's requests. Host-side failures
(missing key, operand errors, a failing key upload, a request that cannot fit, a
cancellation) fail only the request concerned.
"""

import random
import threading

import numpy as np
import pytest

from gpu_util import PARAM_SETS, assert_same, make_pair, random_ct

pytestmark = pytest.mark.gpu

STEPS = [1, -1, 2, 3]
D = 4  # mat-vec diagonals (baby 2, giant 2: keys for steps 1 and 2)


class Owners:
    """Per-owner oracle keys; oracle and per-op GPU evaluators for each owner."""

    def __init__(self, ckg, O, name, count):
        self.ckg, self.O = ckg, O
        self.P, self.ctx = make_pair(ckg, O, name)
        self.scale = float(2.0 ** PARAM_SETS[name]["scale_bits"])
        P = self.P
        self.keys = []
        for o in range(count):
            kg = O.KeyGenerator(P, 100 + o)
            rk = kg.relin_key()
            gk = {O.galois_elt(P.n, s): kg.galois_key(O.galois_elt(P.n, s)) for s in STEPS}
            self.keys.append((rk, gk))
        self.alone = []
        for rk, gk in self.keys:
            d_rk = self.ctx.upload_key(rk.export())
            d_gk = [self.ctx.upload_key(k.export(), e) for e, k in gk.items()]
            self.alone.append(ckg.CudaEvaluator(self.ctx, d_rk, d_gk))
        self.io = self.alone[0]

    def cpu(self, o):
        rk, gk = self.keys[o]
        return self.O.Evaluator(self.P, rk, gk)

    def server(self, budget, **kw):
        s = self.ckg.Server(self.ctx, budget, ev=self.io, **kw)
        for rk, gk in self.keys:
            o = s.add_owner()
            s.add_key(o, rk.export())
            for e, k in gk.items():
                s.add_key(o, k.export(), e)
        return s

    def key_bytes(self):
        P = self.P
        return P.dnum * 2 * (P.max_level + 1 + len(P.p)) * P.n * 8


def make_requests(env, count, seed):
    """A seeded mix: (owner, kind, args) with kind mul / rot / pmul / matvec."""
    P, rng = env.P, random.Random(seed)
    L = P.max_level
    reqs = []
    for i in range(count):
        o = rng.randrange(len(env.keys))
        kind = rng.choice(["mul", "mul", "rot", "rot", "pmul", "matvec"])
        level = rng.randint(1, L)
        a = random_ct(P, seed * 1000 + 4 * i, level)
        if kind == "mul":
            args = (a, random_ct(P, seed * 1000 + 4 * i + 1, level))
        elif kind == "rot":
            args = (a, rng.choice(STEPS))
        elif kind == "pmul":
            args = (a, P.random_q(seed * 1000 + 4 * i + 2, level))
        else:
            args = (a, np.stack([P.random_q(seed * 1000 + 4 * i + 3 + 7 * k, level) for k in range(D)]))
        reqs.append((o, kind, args))
    return reqs


def run_cpu(env, cpu, kind, args):
    s = env.scale
    a = cpu.ct(args[0], s)
    if kind == "mul":
        return cpu.rescale(cpu.mul(a, cpu.ct(args[1], s)))
    if kind == "rot":
        return cpu.rotate(a, args[1])
    if kind == "pmul":
        return cpu.rescale(cpu.mul_plain(a, args[1], s))
    return cpu.matvec_plain(D, 1, args[1], s, a)


def upload(env, kind, args):
    ev, s = env.io, env.scale
    a = ev.upload_ct(args[0], s)
    if kind == "mul":
        return a, ev.upload_ct(args[1], s)
    if kind == "rot":
        return a, args[1]
    if kind == "pmul":
        return a, ev.upload_pt(args[1], s)
    return a, [ev.upload_pt(p, s) for p in args[1]]


def submit(srv, o, kind, dev):
    if kind == "mul":
        return srv.submit_mul(o, *dev)
    if kind == "rot":
        return srv.submit_rotate(o, *dev)
    if kind == "pmul":
        return srv.submit_mul_plain(o, *dev)
    return srv.submit_matvec(o, D, 1, dev[1], dev[0])


def run_alone(ev, kind, dev):
    if kind == "mul":
        return ev.rescale(ev.mul(*dev))
    if kind == "rot":
        return ev.rotate(*dev)
    if kind == "pmul":
        return ev.rescale(ev.mul_plain(*dev))
    return ev.matvec_plain(D, 1, dev[1], dev[0])


@pytest.fixture(scope="module")
def owners(ckg, oracle):
    return Owners(ckg, oracle, "small", 3)


def serve_and_check(env, srv, reqs, threads=2):
    devs = [upload(env, k, a) for _, k, a in reqs]
    ids = [None] * len(reqs)

    def client(part):
        for i in part:
            o, kind, _ = reqs[i]
            ids[i] = submit(srv, o, kind, devs[i])

    parts = [list(range(t, len(reqs), threads)) for t in range(threads)]
    ts = [threading.Thread(target=client, args=(p,)) for p in parts]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    outs = []
    for i in range(len(reqs)):
        ct, times = srv.result(ids[i], timeout_ms=120000)
        assert times[0] <= times[1] <= times[2], f"request {i}: times {times}"
        outs.append(ct)
    cpus = [env.cpu(o) for o in range(len(env.keys))]
    for i, (o, kind, args) in enumerate(reqs):
        want = run_cpu(env, cpus[o], kind, args)
        got, gscale = env.io.download_ct(outs[i])
        assert outs[i].level() == want.level and gscale == want.scale, f"request {i} ({kind}): level/scale"
        assert_same(got, want.data(), f"request {i} ({kind}, owner {o}) vs oracle")
        alone, _ = env.io.download_ct(run_alone(env.alone[o], kind, devs[i]))
        assert np.array_equal(got, alone), f"request {i} ({kind}): served result differs from the op alone"
    for o in range(len(env.keys)):
        assert srv.owner_counter(o) == cpus[o].counter(), f"owner {o} counter"
    return srv.stats()


def test_serve_mixed_owners_roomy_budget(owners):
    """Everything resident: batches mix owners and ops; results equal alone and oracle."""
    srv = owners.server(256 << 20, max_batch_ks=64, max_inflight=2)
    st = serve_and_check(owners, srv, make_requests(owners, 48, 5))
    assert st["completed"] == 48 and st["failed"] == 0
    assert st["key_evictions"] == 0
    assert st["peak_device_bytes"] <= 256 << 20
    srv.close()


def test_serve_tight_budget_spills_keys(owners):
    """A budget near one owner's key set: keys are evicted to the host copy and uploaded
    again, the device bytes never exceed the budget, and every result is unchanged."""
    budget = 7 * owners.key_bytes() + (8 << 20)
    srv = owners.server(budget, max_batch_ks=16, max_inflight=2)
    st = serve_and_check(owners, srv, make_requests(owners, 40, 6))
    assert st["completed"] == 40 and st["failed"] == 0
    assert st["key_evictions"] > 0 and st["key_misses"] >= st["key_evictions"]
    assert st["key_upload_bytes"] == st["key_misses"] * owners.key_bytes()
    assert st["peak_device_bytes"] <= budget and st["peak_key_bytes"] <= budget
    srv.close()


def test_serve_errors_fail_only_their_request(owners, ckg):
    env, P, s = owners, owners.P, owners.scale
    srv = owners.server(256 << 20)
    L = P.max_level
    good = env.io.upload_ct(random_ct(P, 1, L), s)
    other = env.io.upload_ct(random_ct(P, 2, L - 1), s)
    missing = srv.submit_rotate(0, good, 5)          # no Galois key for step 5
    mismatch = srv.submit_mul(1, good, other)        # level mismatch
    ok = srv.submit_rotate(2, good, 1)
    with pytest.raises(ckg.InvalidParams, match="missing galois key"):
        srv.result(missing, 60000)
    with pytest.raises(ckg.LevelMismatch):
        srv.result(mismatch, 60000)
    ct, _ = srv.result(ok, 60000)
    want = run_cpu(env, env.cpu(2), "rot", (random_ct(P, 1, L), 1))
    assert_same(env.io.download_ct(ct)[0], want.data(), "rotation next to failing requests")
    with pytest.raises(ckg.InvalidParams):
        srv.result(ok, 0)                            # results are returned once
    with pytest.raises(ckg.InvalidParams):
        srv.submit_rotate(7, good, 1)                # unknown owner
    srv.close()


def test_serve_upload_failure_and_oom(owners, ckg):
    """An injected key-upload failure fails the requests that needed the key, the next
    upload succeeds; a request larger than the whole budget fails with OutOfMemory."""
    env, P, s = owners, owners.P, owners.scale
    L = P.max_level
    srv = owners.server(256 << 20)
    x = env.io.upload_ct(random_ct(P, 3, L), s)
    srv.inject_upload_failures(1)
    first = srv.submit_rotate(0, x, 1)
    with pytest.raises(ckg.OutOfMemory, match="injected"):
        srv.result(first, 60000)
    again = srv.submit_rotate(0, x, 1)
    ct, _ = srv.result(again, 60000)
    want = run_cpu(env, env.cpu(0), "rot", (random_ct(P, 3, L), 1))
    assert_same(env.io.download_ct(ct)[0], want.data(), "rotation after a failed upload")
    srv.close()
    tiny = owners.server(owners.key_bytes() - 1)  # no key fits; a plaintext product does
    big = tiny.submit_mul(0, x, x)
    with pytest.raises(ckg.OutOfMemory, match="budget"):
        tiny.result(big, 60000)
    plain = tiny.submit_mul_plain(1, x, env.io.upload_pt(P.random_q(4, L), s))  # needs no key
    tiny.result(plain, 60000)
    tiny.close()


def test_serve_cancel_and_drain(owners, ckg):
    env, P, s = owners, owners.P, owners.scale
    srv = owners.server(256 << 20, max_batch_ks=1, max_inflight=1)
    x = env.io.upload_ct(random_ct(P, 5, P.max_level), s)
    ids = [srv.submit_rotate(i % 3, x, 1) for i in range(12)]
    cancelled = srv.cancel(ids[-1])
    srv.drain(120000)
    for rid in ids[:-1]:
        srv.result(rid, 0)
    if cancelled:
        with pytest.raises(ckg.Cancelled):
            srv.result(ids[-1], 0)
    else:
        srv.result(ids[-1], 0)
    st = srv.stats()
    assert st["completed"] + st["cancelled"] == 12 and st["pending"] == 0
    assert srv.cancel(ids[0]) is False
    srv.close()


@pytest.mark.parametrize("boot_lanes", [0, 1, 2])
def test_serve_bootstrap_requests(ckg, oracle, boot_lanes):
    """Bootstrap requests from two owners (each with its own relinearization, rotation,
    conjugation and SSE keys) served beside rotations, on the reference's N = 2^10 bootstrap
    chain, on the context's stream and on compute lanes (one or two bootstrap lanes beside the
    lane of the rotations, overlapping them): every output equals the oracle's, each owner's OpCounter equals the CPU's, and
    outputs handed back from a lane are then used by the context's own stream."""
    O = oracle
    q_bits = [54, 42, 42] + [34] * 4 + [58] * 7 + [56] * 4
    delta = 2.0 ** 42
    P = O.Params.from_bits(10, q_bits, [60, 60], 42, 9)
    enc = O.Encoder(P)
    ctx = ckg.Context(10, P.q, P.p, 9, scale=delta)
    io = ckg.CudaEvaluator(ctx, None, [])
    srv = ckg.Server(ctx, 2 << 30, max_batch_ks=32, max_inflight=2, ev=io, boot_lanes=boot_lanes)
    srv.enable_bootstrap(ckg.BootParams(log_slots=9), delta)
    owners = []
    for o in range(2):
        kg = O.KeyGenerator(P, 60 + o)
        rk = kg.relin_key()
        bs = O.Bootstrapper(P, kg, enc, 9)
        oid = srv.add_owner()
        srv.add_key(oid, rk.export())
        for e, k in bs.galois_keys().items():
            srv.add_key(oid, k.export(), e)
        ts, td = bs.sse_keys()
        srv.add_sse_keys(oid, ts.export(), td.export())
        owners.append((kg, rk, bs, O.Evaluator(P, rk, bs.galois_keys())))
    rng = np.random.default_rng(3)
    reqs = []
    for i in range(6):
        o = i % 2
        kg, rk, bs, ev = owners[o]
        m = rng.uniform(-1, 1, P.n // 2)
        ct0 = ev.mod_switch_to_level(O.encrypt_sk(ev, kg, 20 + i, enc.encode(m, delta, P.max_level), delta), 0)
        g0 = io.upload_ct(ct0.data(), delta)
        reqs.append(("boot", o, ct0, srv.submit_bootstrap(o, g0)))
        x = random_ct(P, 200 + i, P.max_level - 2)
        reqs.append(("rot", o, x, srv.submit_rotate(o, io.upload_ct(x, delta), 1)))
    for kind, o, x, rid in reqs:
        ct, _ = srv.result(rid, 300000)
        kg, rk, bs, ev = owners[o]
        if kind == "boot":
            want = bs.bootstrap(ev, x)
        else:
            want = ev.rotate(ev.ct(x, delta), 1)
        got, scale = io.download_ct(ct)
        assert scale == want.scale and ct.level() == want.level
        assert_same(got, want.data(), f"served {kind} owner {o}")
        twice = io.add(ct, ct)  # the context's stream reads the output, then the handle goes
        del ct
        got2, _ = io.download_ct(twice)
        assert_same(got2, ev.add(want, want).data(), f"served {kind} owner {o}, used after completion")
    for o, (kg, rk, bs, ev) in enumerate(owners):
        assert srv.owner_counter(o) == ev.counter(), f"owner {o} counter"
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    srv.close()
