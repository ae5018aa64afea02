"""Key-switching throughput of the B200 RNS-CKKS evaluator path (one JSON line).

Beside it: `bootstrap` -- one full n16_boot bootstrap (ms, device events); `mlp_step` -- the
encrypted training step; `serving_one_lane` / `serving` / `serving_boot_spill` / `serving_spill`
-- the serving loop's throughput and p50/p99 latency under Poisson arrivals (one stream, a
bootstrap lane at the same offered load, bootstrap-key spill, key spill without bootstraps).

Parameters: N = 2^16, 24 x 50-bit data primes + 8 x 60-bit special primes, dnum = 3
(alpha = 8), 31 evaluation keys (relinearization + 30 Galois keys for +-2^k, k = 0..14).

Headline (`value`): the batched uneven-level stream. 512 ciphertexts with limb counts drawn
uniformly from {4..24}, a seeded op mix of 40% HMult+relin+rescale, 40% rotation by
+-2^k and 20% plaintext-multiply+rescale, executed as one CUDA-graph-captured batch (one
launch per stage for a chunk of ops); one step = one replay of the whole batch. The
metric is key switches per second (HMult and rotation one each).

Beside it (`plain`): the plain one-op-at-a-time path on the full-level workload, 128
ciphertexts at 24 limbs, 128 x (HMult+relin+rescale) and 128 rotations, each op an
individual evaluator call.

`e2e`: the batched stream through the C ABI with host buffers: every input uploaded from
pinned host memory, the batch built and run, every result downloaded to pinned host
memory, all inside the timed region. `--impl reference` times the reference's CPU path
(the oracle's restatement of crates/ckks-train-ckks with OpenMP over the units of its
`parallel` feature) on a bounded sample of the same op mix, cross-checks it against the
reference's published CPU time, and times the reference's own CUDA kernels on the same GPU
(`reference_gpu`).

Multi-GPU: each rank runs the same stream on its own GPU with its own keys and inputs
(independent ciphertexts shard with no exchange: weak scaling); time = max over ranks. Serving
on N GPUs places every key owner on one rank (ckks-train_b200/router.py) and pools the ranks'
latencies.
"""

import argparse
import gc
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "ckks-train_b200")

LOG_N = 16
Q_BITS = [50] * 24
P_BITS = [60] * 8
DNUM = 3
SCALE = 2.0 ** 50
ROT_STEPS = [s * (1 << k) for k in range(15) for s in (1, -1)]  # +-2^k, k = 0..14
MIX_OPS = 512
MIX_LIMBS = (4, 24)
PLAIN_CTS = 128
PLAIN_LEVEL = 23
BOOT_Q_BITS = [54] + [42] * 16 + [34] * 4 + [58] * 7 + [56] * 4  # n16_boot: 32 data primes
BOOT_P_BITS = [60] * 4
BOOT_DNUM = 8
BOOT_DELTA = 2.0 ** 42
SERVE_OWNERS = 32
SERVE_D = 64                 # BSGS mat-vec diagonals: baby 8, giant 8
SERVE_BUDGET = 24 << 30      # HBM bytes for cached keys + queued work: about half the owners
SERVE_REQUESTS = 1000
SERVE_LOAD = 0.7             # offered Poisson rate / measured capacity
SERVE_BOOT_OWNERS = 8        # n16_boot serving with bootstrap requests
SERVE_BOOT_BUDGET = 96 << 30
SERVE_BOOT_LANES = 1          # bootstrap lanes of the bootstrap-serving runs (0: one stream)
SERVE_BOOT_SPILL_OWNERS = 32  # the same with key spill: up to 32 owners within host memory
SERVE_BOOT_SPILL_BUDGET = 48 << 30
SERVE_BOOT_SPILL_REQUESTS = 400
SERVE_RESULT_DEADLINE_S = 600  # a serving run stops collecting (and counts the rest as failed) after this


def load_package():
    if "ckks_train_b200" in sys.modules:
        return sys.modules["ckks_train_b200"]
    spec = importlib.util.spec_from_file_location("ckks_train_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ckks_train_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def galois_elt(n, step):
    return pow(3, step % (n // 2), 2 * n)


def mix_ops(seed, count=MIX_OPS):
    """The seeded op stream: (kind, level, steps)."""
    rng = np.random.default_rng(seed)
    ops = []
    for _ in range(count):
        r = rng.random()
        kind = "mul" if r < 0.4 else ("rot" if r < 0.8 else "pmul")
        limbs = int(rng.integers(MIX_LIMBS[0], MIX_LIMBS[1] + 1))
        steps = ROT_STEPS[int(rng.integers(0, len(ROT_STEPS)))]
        ops.append((kind, limbs - 1, steps))
    return ops


# ---- clocks during the timed region -------------------------------------------------

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device, self.samples, self.proc = device, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ---- set-up: context, keys, evaluator ------------------------------------------------

class Setup:
    """Context, 31 keys (synthetic uniform key material: throughput does not depend on the
    key values) and the evaluator of one rank."""

    def __init__(self, ckg, torch, device):
        self.ckg, self.torch, self.device = ckg, torch, device
        self.ctx = ckg.Context.from_bits(LOG_N, Q_BITS, P_BITS, DNUM, device=device, scale_bits=50)
        ctx = self.ctx
        self.n = ctx.n
        self.gen = torch.Generator(device=f"cuda:{device}")
        self.gen.manual_seed(20261203 + device)
        self.q_all = torch.tensor(ctx.q + ctx.p, dtype=torch.int64, device=f"cuda:{device}")
        shape = (DNUM, 2, len(ctx.q) + ctx.k, self.n)

        def make_key(elt):
            t = self.uniform(shape, self.q_all.view(1, 1, -1, 1))
            k = ctx.upload_key_device(t.data_ptr(), shape, elt)
            del t
            return k

        self.relin = make_key(0)
        self.galois = {}
        for s in ROT_STEPS:
            e = galois_elt(self.n, s)
            if e not in self.galois:
                self.galois[e] = make_key(e)
        self.ev = ckg.CudaEvaluator(ctx, self.relin, list(self.galois.values()))

    def uniform(self, shape, qcol):
        t = self.torch.randint(0, 1 << 62, shape, generator=self.gen, device=self.q_all.device,
                               dtype=self.torch.int64) % qcol
        self.torch.cuda.synchronize()
        return t

    def ct(self, level, ncomp=2):
        t = self.uniform((ncomp, level + 1, self.n), self.q_all[: level + 1].view(1, -1, 1))
        c = self.ev.upload_ct_device(t.data_ptr(), ncomp, level, SCALE)
        self.ctx.sync()
        return c, t

    def pt(self, level):
        t = self.uniform((level + 1, self.n), self.q_all[: level + 1].view(-1, 1))
        p = self.ev.upload_pt_device(t.data_ptr(), level, SCALE)
        self.ctx.sync()
        return p, t


CFG1_LOG_N, CFG1_Q_BITS, CFG1_P_BITS, CFG1_DNUM, CFG1_SCALE_BITS = 13, [45] * 4, [60], 4, 45
CFG1_PAIRS = 64


class Config1:
    """The small-ring workload: N = 2^13, 4 x 45-bit q (descending prime search from 2^45), one
    60-bit p, dnum 4; 64 seeded uniform ciphertext pairs at the top level; 64 x (HMult + relin +
    rescale) and 64 x rotation by +1 per step (128 key switches), per op and as one batched
    CUDA-graph replay. Synthetic uniform key material (relinearization and the +1 Galois key)."""

    text = ("N=2^13, 4x45-bit q + 1x60-bit p, dnum 4; 64 ciphertext pairs; 64 x (HMult+relin+rescale) + "
            "64 x rotation by +1 per step")

    def __init__(self, ckg, torch, device):
        self.torch = torch
        self.ctx = ctx = ckg.Context.from_bits(CFG1_LOG_N, CFG1_Q_BITS, CFG1_P_BITS, CFG1_DNUM, device=device,
                                               scale_bits=CFG1_SCALE_BITS)
        n, L = ctx.n, len(ctx.q) - 1
        gen = torch.Generator(device=f"cuda:{device}")
        gen.manual_seed(13)
        qall = torch.tensor(ctx.q + ctx.p, dtype=torch.int64, device=f"cuda:{device}")

        def uniform(shape, qcol):
            t = torch.randint(0, 1 << 62, shape, generator=gen, device=qall.device, dtype=torch.int64) % qcol
            torch.cuda.synchronize()
            return t

        shape = (CFG1_DNUM, 2, len(ctx.q) + ctx.k, n)
        keys = [uniform(shape, qall.view(1, 1, -1, 1)) for _ in range(2)]
        self.relin = ctx.upload_key_device(keys[0].data_ptr(), shape, 0)
        self.gk = ctx.upload_key_device(keys[1].data_ptr(), shape, galois_elt(n, 1))
        self.ev = ev = ckg.CudaEvaluator(ctx, self.relin, [self.gk])
        scale = 2.0 ** CFG1_SCALE_BITS
        self.pairs = []
        for _ in range(CFG1_PAIRS):
            a, b = (uniform((2, L + 1, n), qall[: L + 1].view(1, -1, 1)) for _ in range(2))
            self.pairs.append((ev.upload_ct_device(a.data_ptr(), 2, L, scale),
                               ev.upload_ct_device(b.data_ptr(), 2, L, scale)))
        ctx.sync()
        self.batch = ckg.Batch(ev)
        self.outs = [self.batch.mul_relin_rescale(a, b) for a, b in self.pairs]
        self.outs += [self.batch.rotate(a, 1) for a, _ in self.pairs]
        self.batch.capture_graph()

    def step_per_op(self):
        ev = self.ev
        return [(ev.rescale(ev.mul(a, b)), ev.rotate(a, 1)) for a, b in self.pairs]

    def measure(self, steps=20, warmup=3):
        torch, ctx = self.torch, self.ctx
        ms_op = timed(torch, ctx, self.step_per_op, steps, warmup)[0]
        ms_b = timed(torch, ctx, self.batch.launch_graph, steps, warmup)[0]
        ks = 2 * CFG1_PAIRS
        return {"workload": self.text, "unit": "keyswitch/s",
                "per_op": round(ks * steps / (ms_op * 1e-3), 1), "per_op_ms_per_step": round(ms_op / steps, 3),
                "batched": round(ks * steps / (ms_b * 1e-3), 1), "batched_ms_per_step": round(ms_b / steps, 3),
                "data": "synthetic uniform ciphertexts and key material"}


def cpu_config1(threads, reps=3):
    """Config 1's workload on the CPU path (the oracle's evaluator) with keys from its key
    generator: key switches per second on `threads` OpenMP threads (the best of `reps` steps) and
    on one thread (one step)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.set_threads(threads)
    P = O.Params.from_bits(CFG1_LOG_N, CFG1_Q_BITS, CFG1_P_BITS, CFG1_SCALE_BITS, CFG1_DNUM)
    kg = O.KeyGenerator(P, 13)
    e1 = O.galois_elt(P.n, 1)
    ev = O.Evaluator(P, kg.relin_key(), {e1: kg.galois_key(e1)})
    L, scale = P.max_level, 2.0 ** CFG1_SCALE_BITS
    pairs = [(ev.ct(np.stack([P.random_q(4 * i + 1, L), P.random_q(4 * i + 2, L)]), scale),
              ev.ct(np.stack([P.random_q(4 * i + 3, L), P.random_q(4 * i + 4, L)]), scale))
             for i in range(CFG1_PAIRS)]
    def step():
        t0 = time.perf_counter()
        for a, b in pairs:
            ev.rescale(ev.mul(a, b))
            ev.rotate(a, 1)
        return time.perf_counter() - t0

    best = min(step() for _ in range(reps))
    O.set_threads(1)
    one = step()
    O.set_threads(threads)
    return {"value": round(2 * CFG1_PAIRS / best, 1), "unit": "keyswitch/s", "cores": threads,
            "one_thread": round(2 * CFG1_PAIRS / one, 1), "kind": "port",
            "sample": f"the whole workload: best of {reps} steps on {threads} threads {best * 1e3:.1f} ms, "
                      f"one step on 1 thread {one * 1e3:.1f} ms"}


class Mix:
    """The batched uneven-level stream."""

    def __init__(self, S, ops, keep_host=True):
        self.S, self.ops = S, ops
        self.inputs = []  # (kind, a, b_or_pt, steps)
        torch, n = S.torch, S.n
        # With keep_host, the inputs' host copies for the e2e step, each list in one pinned
        # allocation laid out in list order (a client's request buffer: ciphertexts a, b of each
        # op in op order; plaintexts in op order), filled straight from the device: no second
        # host copy, so N ranks on one host hold one copy of their inputs each.
        ct_words = sum(2 * (lv + 1) * n * (2 if kind == "mul" else 1) for kind, lv, _ in ops)
        pt_words = sum((lv + 1) * n for kind, lv, _ in ops if kind == "pmul")
        self.host_ct_flat = torch.empty(ct_words, dtype=torch.int64, pin_memory=True) if keep_host else None
        self.host_pt_flat = (torch.empty(pt_words, dtype=torch.int64, pin_memory=True)
                             if keep_host and pt_words else None)
        offs = [0, 0]

        def keep(t, flat, i):
            v = flat[offs[i]:offs[i] + t.numel()].view(t.shape)
            v.copy_(t)
            offs[i] += t.numel()
            return v

        host = []
        for kind, level, steps in ops:
            a, ta = S.ct(level)
            if kind == "mul":
                extra, tb = S.ct(level)
            elif kind == "pmul":
                extra, tb = S.pt(level)
            else:
                extra, tb = None, None
            self.inputs.append((kind, a, extra, steps))
            if keep_host:
                ha = keep(ta, self.host_ct_flat, 0)
                hb = None if tb is None else keep(tb, self.host_ct_flat, 0) if kind == "mul" else keep(
                    tb, self.host_pt_flat, 1)
                host.append((ha, hb))
            del ta, tb
        self.host = host
        self.chunk_items = None
        self.batch, self.outputs = self.make_batch(self.inputs)
        self.ks = self.batch.key_switches()

    def tune(self, ntt_wave=None, chunk_items=None, reps=3):
        """The library's autotuner on this stream (NTT limb wave x chunk size), or the given
        settings. Tuning replays run before any timed region."""
        if ntt_wave is None or chunk_items is None:
            out = self.batch.autotune(reps)
        else:
            self.S.ctx.ntt_wave = ntt_wave
            self.batch.chunk_items = chunk_items
            out = {"ntt_wave": ntt_wave, "chunk_items": chunk_items, "trials": []}
        self.chunk_items = out["chunk_items"]
        return out

    def make_batch(self, inputs):
        b = self.S.ckg.Batch(self.S.ev)
        if self.chunk_items:
            b.chunk_items = self.chunk_items
        outs = []
        for kind, a, extra, steps in inputs:
            if kind == "mul":
                outs.append(b.mul_relin_rescale(a, extra))
            elif kind == "rot":
                outs.append(b.rotate(a, steps))
            else:
                outs.append(b.mul_plain_rescale(a, extra))
        return b, outs

    def step_graph(self):
        self.batch.launch_graph()

    def prepare_e2e(self):
        """Result buffers of the e2e step: one pinned allocation laid out in list order (a client's
        reply buffer), so the list download moves the whole run with one copy. The inputs were
        packed the same way when the stream was built."""
        torch, n = self.S.torch, self.S.n
        shapes = [(2, (level if kind == "rot" else level - 1) + 1, n) for kind, level, _ in self.ops]
        self.out_flat = torch.empty(sum(int(np.prod(sh)) for sh in shapes), dtype=torch.int64, pin_memory=True)
        self.out_host, off = [], 0
        for sh in shapes:
            m = int(np.prod(sh))
            self.out_host.append(self.out_flat[off:off + m].view(sh))
            off += m
        self.out_ptrs = [t.data_ptr() for t in self.out_host]
        self.inflight, self.host_s, self.host_parts = [], 0.0, {}
        self.stream = torch.cuda.ExternalStream(self.S.ctx.stream)

    def step_e2e(self):
        """Upload every input from pinned host memory, build and run the batch, download every
        result to pinned host memory, through the C ABI's overlapped list transfers (one call
        per list): this step's uploads run beside the previous step's compute and downloads. The
        step's handles are dropped before its completion event is recorded, so that event also
        covers the frees of its buffers; the host waits for the event of the step before last, so
        at most two steps are in flight and each upload reuses memory whose free has completed."""
        torch, ev, clock = self.S.torch, self.S.ev, time.perf_counter
        if len(self.inflight) >= 2:
            self.inflight.pop(0).synchronize()
        t0 = clock()
        ct_items, pt_items, h2d = [], [], 0
        for (kind, level, steps), (ha, hb) in zip(self.ops, self.host):
            ct_items.append((ha.data_ptr(), 2, level, SCALE))
            h2d += ha.numel() * 8
            if kind == "mul":
                ct_items.append((hb.data_ptr(), 2, level, SCALE))
                h2d += hb.numel() * 8
            elif kind == "pmul":
                pt_items.append((hb.data_ptr(), level, SCALE))
                h2d += hb.numel() * 8
        cts = iter(ev.upload_ct_overlap_list(ct_items))
        pts = iter(ev.upload_pt_overlap_list(pt_items) if pt_items else [])
        ins = [(kind, next(cts), next(cts) if kind == "mul" else (next(pts) if kind == "pmul" else None), steps)
               for kind, level, steps in self.ops]
        t1 = clock()
        b, outs = self.make_batch(ins)
        t2 = clock()
        b.run()
        t3 = clock()
        ev.download_ct_overlap_list(outs, self.out_ptrs)
        t4 = clock()
        del b, outs, ins, cts, pts  # every handle of the step: its frees are queued here
        e = torch.cuda.Event()
        e.record(self.stream)
        self.inflight.append(e)
        t5 = clock()
        d2h = sum(t.numel() * 8 for t in self.out_host)
        for k, dt in zip(("upload", "batch_build", "run", "download", "release"),
                         (t1 - t0, t2 - t1, t3 - t2, t4 - t3, t5 - t4)):
            self.host_parts[k] = self.host_parts.get(k, 0.0) + dt
        self.host_s += t5 - t0
        return h2d, d2h


class PlainMix:
    """The same uneven-level stream, one evaluator call per op (no batching)."""

    def __init__(self, mix):
        self.mix = mix
        self.ks = mix.ks

    def step(self):
        ev, out = self.mix.S.ev, []
        for kind, a, extra, steps in self.mix.inputs:
            if kind == "mul":
                out.append(ev.rescale(ev.mul(a, extra)))
            elif kind == "rot":
                out.append(ev.rotate(a, steps))
            else:
                out.append(ev.rescale(ev.mul_plain(a, extra)))
        return out


class Plain:
    """The plain per-op path: 128 x (HMult+relin+rescale) + 128 rotations at 24 limbs."""

    def __init__(self, S):
        self.S = S
        self.cts = [S.ct(PLAIN_LEVEL)[0] for _ in range(PLAIN_CTS)]
        self.ks = 2 * PLAIN_CTS

    slowest = (0.0, None)  # (host seconds, op) of the slowest evaluator call so far

    def step(self):
        ev, cts = self.S.ev, self.cts
        out, clock = [], time.perf_counter
        for i in range(PLAIN_CTS):
            t0 = clock()
            out.append(ev.rescale(ev.mul(cts[i], cts[(i + 1) % PLAIN_CTS])))
            self.slowest = max(self.slowest, (clock() - t0, f"mul {i}"))
        for i in range(PLAIN_CTS):
            t0 = clock()
            out.append(ev.rotate(cts[i], ROT_STEPS[i % len(ROT_STEPS)]))
            self.slowest = max(self.slowest, (clock() - t0, f"rotate {i}"))
        return out


# ---- timing ---------------------------------------------------------------------------

class Serving:
    """The serving loop under Poisson arrivals from SERVE_OWNERS key owners. Each owner has
    its own relinearization key and the 14 Galois keys of a 64-diagonal BSGS mat-vec (steps
    1..7 and 8..56 by 8): 15 keys of 96 MiB (synthetic uniform key material), 45 GiB in all,
    registered into pinned host memory; the server caches device copies LRU within
    SERVE_BUDGET. Requests: 5/8 single ops (half HMult+relin+rescale, half rotation by one
    of the owner's steps) and 3/8 64x64 plaintext mat-vecs, on the owner's resident inputs
    (24, 18, 12 and 6 limbs; mat-vecs at 24 or 12 limbs against one shared 64-diagonal
    matrix per level)."""

    params_text = "N=2^16, 24x50-bit q + 8x60-bit p, dnum 3"
    mix_text = "5/8 single ops (HMult+relin+rescale | rotation), 3/8 64x64 BSGS plaintext mat-vec"

    def __init__(self, S, owners=SERVE_OWNERS, budget=SERVE_BUDGET, seed=7, router=None, rank=0):
        ckg, torch = S.ckg, S.torch
        self.S, self.owners = S, owners
        self.rng = np.random.default_rng(seed)
        ctx = S.ctx
        self.srv = ckg.Server(ctx, budget, max_batch_ks=256, max_inflight=2, ev=S.ev)
        bg = 8
        self.steps = [k for k in range(1, bg)] + [bg * k for k in range(1, SERVE_D // bg)]
        shape = (DNUM, 2, len(ctx.q) + ctx.k, ctx.n)
        qcol = S.q_all.view(1, 1, -1, 1)
        # On N GPUs every rank registers only the owners the router places on it.
        local = router.owners_of(rank) if router else list(range(owners))
        t0 = time.time()
        self.slot = {}  # owner -> the server's owner id on this rank
        for g in local:
            o = self.slot[g] = self.srv.add_owner()
            for e in [0] + [galois_elt(ctx.n, st) for st in self.steps]:
                t = S.uniform(shape, qcol)
                self.srv.add_key_device(o, t.data_ptr(), shape, e)
                del t
        self.register_s = time.time() - t0
        self.key_bytes = len(local) * (1 + len(self.steps)) * int(np.prod(shape)) * 8
        self.inputs = {g: [S.ct(l)[0] for l in (23, 17, 11, 5)] for g in local}
        self.diag = {l: [S.pt(l)[0] for _ in range(SERVE_D)] for l in (23, 11)}

    @staticmethod
    def key_bytes_per_owner():
        """Registered key bytes of one owner (15 keys at N=2^16, 24+8 primes, dnum 3)."""
        return 15 * DNUM * 2 * (len(Q_BITS) + len(P_BITS)) * (1 << LOG_N) * 8

    def request(self):
        """The next request of the one seeded stream every rank draws alike: a callable that
        submits it here, or None when its owner is placed on another rank."""
        g = int(self.rng.integers(self.owners))
        r = self.rng.random()
        if r < 5 / 16:
            which, st = int(self.rng.integers(4)), None
        elif r < 10 / 16:
            which = int(self.rng.integers(4))
            st = self.steps[int(self.rng.integers(len(self.steps)))]
        else:
            which, st = int(self.rng.integers(2)), None
        if g not in self.slot:
            return None
        o, ins = self.slot[g], self.inputs[g]
        if r < 5 / 16:
            a = ins[which]
            return lambda: self.srv.submit_mul(o, a, a)
        if r < 10 / 16:
            a = ins[which]
            return lambda: self.srv.submit_rotate(o, a, st)
        x, lvl = ins[0 if which == 0 else 2], (23, 11)[which]
        return lambda: self.srv.submit_matvec(o, SERVE_D, 1, self.diag[lvl], x)

    def run(self, count, rate=None):
        """Draws `count` requests of the stream and submits those placed here (all at once, or
        at the due times of Poisson arrivals at `rate` per second over the whole stream) while a
        collector takes the results; returns per-request (submitted, completed) in us."""
        reqs = [self.request() for _ in range(count)]
        gaps = self.rng.exponential(1.0 / rate, count) if rate else np.zeros(count)
        dues = np.cumsum(gaps)
        local = [(d, q) for d, q in zip(dues, reqs) if q is not None]
        ids, times, lag, failed, collected = [], [], [0.0], [], [0]
        submitted = threading.Event()  # every submit() has returned (or raised)
        done = threading.Event()
        deadline = time.perf_counter() + SERVE_RESULT_DEADLINE_S

        def collect():
            # Never dies silently: a failed request is recorded with its status, an exception or
            # the deadline ends the collection, and done is always set, so the submitter cannot
            # wait forever.
            try:
                while not (submitted.is_set() and collected[0] >= len(ids)):
                    if collected[0] >= len(ids):
                        time.sleep(0.0002)
                        continue
                    left_ms = int(np.ceil((deadline - time.perf_counter()) * 1e3))
                    code, _, t = self.srv.result_times(ids[collected[0]], max(1, left_ms))
                    collected[0] += 1
                    if code == 0:
                        times.append(t)
                        continue
                    failed.append(f"status {code}")
                    if time.perf_counter() >= deadline:
                        break
            except Exception as e:  # noqa: BLE001 -- counted and reported below
                failed.append(repr(e))
            finally:
                done.set()

        th = threading.Thread(target=collect, daemon=True)
        th.start()
        start = time.perf_counter()
        try:
            for due, submit in local:
                if done.is_set():
                    break
                now = time.perf_counter() - start
                if due > now:
                    time.sleep(due - now)
                lag[0] = max(lag[0], time.perf_counter() - start - due)
                ids.append(submit())
        finally:
            submitted.set()
            done.wait()
            th.join()
        lost = len(local) - len(times)
        if lost:
            print(f"serving: {lost} of {len(local)} requests not served, first failure: "
                  f"{failed[0] if failed else 'not submitted'}", file=sys.stderr)
        self.failed = getattr(self, "failed", 0) + lost
        return np.array([(t[0], t[2]) for t in times]).reshape(-1, 2), lag[0]

    def measure(self, requests=SERVE_REQUESTS, load=SERVE_LOAD, dist=None, rate=None):
        """Capacity (saturated), then `requests` Poisson arrivals at `load` x capacity, or at
        `rate` requests/s when given (to compare servers at one offered load). With `dist` (one
        rank per GPU, owners placed by the router) capacity is the sum over ranks, the latencies of
        all ranks are pooled and the span is the longest rank's."""
        self.failed = 0
        retries0 = self.alloc_retries()
        self.run(96)  # warm-up: Galois permutations, pools, first key uploads
        sat, _ = self.run(min(400, requests))
        capacity = len(sat) / ((sat[:, 1].max() - sat[:, 0].min()) * 1e-6) if len(sat) else 0.0
        if dist:
            capacity = sum(gather_objects(dist, capacity))
        st0 = self.srv.stats()
        rate = rate or load * capacity
        t, lag = self.run(requests, rate)
        st = self.srv.stats()
        lat = (t[:, 1] - t[:, 0]) * 1e-3
        span = (t[:, 1].max() - t[:, 0].min()) * 1e-6 if len(t) else 0.0
        d = {k: st[k] - st0[k] for k in ("batches", "multi_owner_batches", "key_hits", "key_misses",
                                          "key_evictions", "key_upload_bytes", "budget_waits")}
        peak_dev, key_bytes, failed = st["peak_device_bytes"], self.key_bytes, self.failed
        retries = self.alloc_retries()
        retries = None if retries is None or retries0 is None else retries - retries0
        if dist:
            parts = gather_objects(dist, (lat.tolist(), span, lag, d, peak_dev, key_bytes, failed))
            lat = np.array([x for p in parts for x in p[0]])
            span, lag = max(p[1] for p in parts), max(p[2] for p in parts)
            d = {k: sum(p[3][k] for p in parts) for k in d}
            peak_dev, key_bytes = max(p[4] for p in parts), sum(p[5] for p in parts)
            failed = sum(p[6] for p in parts)

        def pct(v):
            return round(float(np.percentile(lat, v)), 3) if len(lat) else None

        return {"requests": requests, "served": int(len(lat)), "failed": int(failed), "owners": self.owners,
                "params": self.params_text, "mix": self.mix_text,
                "capacity_req_s": round(capacity, 2), "offered_req_s": round(rate, 2),
                "throughput_req_s": round(len(lat) / span, 2) if span else 0.0,
                "p50_ms": pct(50), "p99_ms": pct(99),
                "mean_ms": round(float(lat.mean()), 3) if len(lat) else None,
                "max_submit_lag_ms": round(lag * 1e3, 3),
                "hbm_budget_gib": round(self.srv.stats()["hbm_budget"] / 2 ** 30, 2),
                "key_set_gib": round(key_bytes / 2 ** 30, 2),
                "peak_device_gib": round(peak_dev / 2 ** 30, 2),
                "key_hit_rate": round(d["key_hits"] / max(1, d["key_hits"] + d["key_misses"]), 3),
                "key_upload_gib": round(d["key_upload_bytes"] / 2 ** 30, 2),
                "batches": d["batches"], "multi_owner_batches": d["multi_owner_batches"],
                "key_evictions": d["key_evictions"], "budget_waits": d["budget_waits"],
                "register_s": round(self.register_s, 1),
                "alloc_retries": retries}

    def alloc_retries(self):
        """Device allocations of the serving context retried after out-of-memory (each hands
        every pool's cached memory back first): nonzero means the run was memory-bound."""
        try:
            ctx = getattr(self, "ctx", None) or self.S.ctx
            return ctx.transfer_stats()["alloc_retries"]
        except Exception:  # noqa: BLE001 -- a stand-in server in the CPU tests has no context
            return None

    def close(self):
        self.srv.close()


class BootServing(Serving):
    """The serving loop on the n16_boot chain with bootstrap requests in the mix:
    SERVE_BOOT_OWNERS owners, each with its own relinearization key, the 33 Galois keys of the
    bootstrap (32 rotations + conjugation), the 3 more a 64x64 BSGS mat-vec needs and the two
    SSE keys -- 38 keys of 288 MiB (about 11 GiB per owner, synthetic uniform key material) in
    pinned host memory, all resident once warm within SERVE_BOOT_BUDGET. Requests: 1/4 HMult
    +relin+rescale and 1/4 rotations at level 16 (the post-bootstrap level), 3/10 64x64 plaintext
    mat-vecs at level 16, 1/5 full bootstraps of a level-0 input; Poisson arrivals."""

    params_text = "n16_boot: N=2^16, 32 q primes + 4x60-bit p, dnum 8, BootParams::default_n16"
    mix_text = "1/4 HMult+relin+rescale, 1/4 rotation, 3/10 64x64 BSGS plaintext mat-vec, 1/5 full SSE bootstrap"

    def __init__(self, ckg, torch, device, owners=SERVE_BOOT_OWNERS, budget=SERVE_BOOT_BUDGET, seed=9,
                 boot_lanes=SERVE_BOOT_LANES, boot_priority=True):
        self.owners, self.lanes = owners, {"boot_lanes": boot_lanes, "boot_priority": boot_priority}
        self.rng = np.random.default_rng(seed)
        q, p = ckg.primes_for_bits(16, BOOT_Q_BITS, BOOT_P_BITS)
        self.ctx = ctx = ckg.Context(16, q, p, BOOT_DNUM, device=device)
        n, k, L = 1 << 16, len(p), len(q) - 1
        gen = torch.Generator(device=f"cuda:{device}")
        gen.manual_seed(777 + device)
        qall = torch.tensor(q + p, dtype=torch.int64, device=f"cuda:{device}")

        def uniform(shape, qcol):
            t = torch.randint(0, 1 << 62, shape, generator=gen, device=qall.device, dtype=torch.int64) % qcol
            torch.cuda.synchronize()
            return t

        def key_tensor(parts, qlimbs):
            shape = (parts, 2, qlimbs + k, n)
            return uniform(shape, torch.cat([qall[:qlimbs], qall[len(q):]]).view(1, 1, -1, 1)), shape

        self.ev = ckg.CudaEvaluator(ctx, None, [])
        self.srv = ckg.Server(ctx, budget, max_batch_ks=256, max_inflight=2, ev=self.ev, boot_lanes=boot_lanes,
                              boot_priority=boot_priority)
        bp = ckg.BootParams()
        self.srv.enable_bootstrap(bp, BOOT_DELTA)
        boot_steps = ckg.boot_rotation_steps(bp)
        self.steps = list(range(1, 8)) + [8 * j for j in range(1, 8)]
        elts = sorted({galois_elt(n, st) for st in boot_steps + self.steps} | {2 * n - 1})
        t0 = time.time()
        nkeys = 0
        for _ in range(owners):
            o = self.srv.add_owner()
            for e in [0] + elts:
                t, shape = key_tensor(BOOT_DNUM, L + 1)
                self.srv.add_key_device(o, t.data_ptr(), shape, e)
                del t
                nkeys += 1
            ts, _ = key_tensor(1, 1)
            td, _ = key_tensor(BOOT_DNUM, L + 1)
            self.srv.add_sse_keys_device(o, ts.data_ptr(), td.data_ptr())
            del ts, td
            nkeys += 1
        self.register_s = time.time() - t0
        self.key_bytes = nkeys * BOOT_DNUM * 2 * (L + 1 + k) * n * 8 + owners * 2 * (1 + k) * n * 8

        def ct(level):
            t = uniform((2, level + 1, n), qall[: level + 1].view(1, -1, 1))
            c = self.ev.upload_ct_device(t.data_ptr(), 2, level, BOOT_DELTA)
            ctx.sync()
            return c

        self.level0 = [ct(0) for _ in range(owners)]
        self.inputs = [[ct(16) for _ in range(2)] for _ in range(owners)]
        diag = []
        for _ in range(SERVE_D):
            t = uniform((17, n), qall[:17].view(-1, 1))
            diag.append(self.ev.upload_pt_device(t.data_ptr(), 16, BOOT_DELTA))
            ctx.sync()
        self.diag = diag

    def request(self):
        o = int(self.rng.integers(self.owners))
        r = self.rng.random()
        a = self.inputs[o][int(self.rng.integers(2))]
        if r < 0.25:
            return lambda: self.srv.submit_mul(o, a, a)
        if r < 0.5:
            st = self.steps[int(self.rng.integers(len(self.steps)))]
            return lambda: self.srv.submit_rotate(o, a, st)
        if r < 0.8:
            return lambda: self.srv.submit_matvec(o, SERVE_D, 1, self.diag, a)
        return lambda: self.srv.submit_bootstrap(o, self.level0[o])

    def measure(self, requests=SERVE_REQUESTS, load=SERVE_LOAD, rate=None):
        out = super().measure(requests, load, rate=rate)
        out["lanes"] = self.lanes
        return out

    def close(self):
        """Closes the server and drops every device object of this run's own context (its keys
        cache, inputs, matrix and the context itself), so the device memory is free for the next."""
        self.srv.close()
        self.srv = self.level0 = self.inputs = self.diag = self.ev = None
        ctx, self.ctx = self.ctx, None
        ctx.sync()
        del ctx
        gc.collect()

    @staticmethod
    def owner_bytes():
        """Pinned host bytes of one owner's keys: 38 switching keys at 32 + 4 limbs, dnum 8,
        and the level-0 SSE key."""
        limbs = len(BOOT_Q_BITS) + len(BOOT_P_BITS)
        return 38 * BOOT_DNUM * 2 * limbs * (1 << 16) * 8 + 2 * (1 + len(BOOT_P_BITS)) * (1 << 16) * 8

    @staticmethod
    def spill_owners(limit=SERVE_BOOT_SPILL_OWNERS):
        """Owners for the spill run: `limit`, or fewer so that their pinned keys take at most half
        of the host's available memory."""
        avail = 0
        try:
            with open("/proc/meminfo") as f:
                for line in f:
                    if line.startswith("MemAvailable:"):
                        avail = int(line.split()[1]) * 1024
        except OSError:
            pass
        return max(2, min(limit, int(avail / 2 // BootServing.owner_bytes())))


class BootBench:
    """One full bootstrap on the n16_boot chain (N = 2^16, 32 data primes of 54/42/34/58/56
    bits, 4 x 60-bit special primes, dnum 8) with BootParams::default_n16 (SSE h' = 32, K = 13,
    degree 127, CoeffToSlot 4 / EvalMod 7 / SlotToCoeff 4 levels): mod-raise, CoeffToSlot,
    two EvalMods, SlotToCoeff, 111 key switches. The library encodes the stages and the EvalMod
    series itself; the 35 keys (relinearization, 32 rotations, conjugation, the two SSE
    switches) are synthetic uniform key material, since a bootstrap's time does not depend on
    the key values, and the input is a uniform level-0 ciphertext."""

    def __init__(self, ckg, torch, device):
        self.ckg, self.torch = ckg, torch
        q, p = ckg.primes_for_bits(16, BOOT_Q_BITS, BOOT_P_BITS)
        self.ctx = ckg.Context(16, q, p, BOOT_DNUM, device=device)
        ctx, n = self.ctx, 1 << 16
        gen = torch.Generator(device=f"cuda:{device}")
        gen.manual_seed(424242 + device)
        qall = torch.tensor(q + p, dtype=torch.int64, device=f"cuda:{device}")
        k = len(p)

        def uniform(shape, qcol):
            t = torch.randint(0, 1 << 62, shape, generator=gen, device=qall.device, dtype=torch.int64) % qcol
            torch.cuda.synchronize()
            return t

        def key(parts, qlimbs, elt):
            shape = (parts, 2, qlimbs + k, n)
            qcol = torch.cat([qall[:qlimbs], qall[len(q):]]).view(1, 1, -1, 1)
            t = uniform(shape, qcol)
            kk = ctx.upload_key_device(t.data_ptr(), shape, elt)
            del t
            return kk

        bp = ckg.BootParams()
        relin = key(BOOT_DNUM, len(q), 0)
        self.galois = [key(BOOT_DNUM, len(q), galois_elt(n, s)) for s in ckg.boot_rotation_steps(bp)]
        self.galois.append(key(BOOT_DNUM, len(q), 2 * n - 1))
        self.to_sparse, self.to_dense = key(1, 1, 0), key(BOOT_DNUM, len(q), 0)
        self.key_bytes = sum(x.nbytes for x in self.galois) + relin.nbytes + self.to_sparse.nbytes + \
            self.to_dense.nbytes
        self.ev = ckg.CudaEvaluator(ctx, relin, [])
        t0 = time.time()
        l0 = ckg.launch_count()
        self.bs = ckg.Bootstrapper.encoded(self.ev, bp, BOOT_DELTA, self.galois, self.to_sparse, self.to_dense)
        ctx.sync()
        self.setup_s = time.time() - t0
        self.setup_launches = ckg.launch_count() - l0
        t = uniform((2, 1, n), qall[:1].view(1, 1, 1))
        self.ct = self.ev.upload_ct_device(t.data_ptr(), 2, 0, BOOT_DELTA)
        ctx.sync()
        del t
        self.out = None

    def step(self):
        self.out = self.bs.bootstrap(self.ev, self.ct)

    def measure(self, steps=8, warmup=4):
        ckg, torch = self.ckg, self.torch
        self.step()
        self.ctx.sync()
        l0 = ckg.launch_count()
        self.ev.reset_counter()
        self.step()
        self.ctx.sync()
        launches = ckg.launch_count() - l0
        c = self.ev.counter()
        ms, _ = timed(torch, self.ctx, self.step, steps, warmup)
        walls = []
        for _ in range(3):
            t0 = time.perf_counter()
            self.step()
            self.ctx.sync()
            walls.append((time.perf_counter() - t0) * 1e3)
        wall = float(np.median(walls))
        return {"ms": round(ms / steps, 3), "unit": "ms per bootstrap (device events, back-to-back)",
                "single_call_wall_ms": round(wall, 3), "single_call": "median of 3 host-synchronised calls",
                "target_ms": 150,
                "params": "n16_boot: N=2^16, 32 q primes (54, 42x16, 34x4, 58x7, 56x4 bits) + 4x60-bit P, "
                          "dnum 8; SSE h'=32, K=13, Chebyshev degree 127, CtS/EvalMod/StC 4/7/4 levels",
                "key_switches": c["rotations"] + c["relins"] + c["sse_switches"],
                "counts": c, "launches": int(launches), "setup_launches": int(self.setup_launches),
                "output_level": self.bs.output_level(),
                "setup_s": round(self.setup_s, 2), "key_gib": round(self.key_bytes / 2 ** 30, 2),
                "data": "synthetic uniform key material and level-0 input; stages encoded by the library"}


MLP_Q_BITS = [58] + [42] * 31   # n16_train (crates/ckks-train-ckks/src/params.rs:168-173)
MLP_P_BITS = [58] * 4
MLP_DNUM = 8
MLP_DIMS = [196, 64, 10]


class MlpBench:
    """One encrypted MLP training step (config 4): the interactive trainer's SGD step
    (crates/ckks-train-nn/src/trainer.rs) through the library's HeOps, on n16_train (N = 2^16,
    58 + 31 x 42-bit q, 4 x 58-bit p, dnum 8, scale 2^42), Layout(2^15, 256, 64), 196 -> 64 -> 10
    with Square, batch 64. The 53 keys (relinearization and 52 Galois keys, 288 MiB each) are
    uniform key material and the weights, biases and batch uniform ciphertexts at the levels and
    exact scales the client would encrypt them at: a step's time does not depend on the values.
    Each step starts from the same network (the trainer leaves updated weights 9 levels lower)."""

    def __init__(self, ckg, torch, device):
        self.ckg, self.torch = ckg, torch
        nn = ckg.nn
        q, p = ckg.primes_for_bits(16, MLP_Q_BITS, MLP_P_BITS)
        self.ctx = ctx = ckg.Context(16, q, p, MLP_DNUM, device=device, scale=2.0 ** 42)
        n = 1 << 16
        gen = torch.Generator(device=f"cuda:{device}")
        gen.manual_seed(515151 + device)
        qall = torch.tensor(q + p, dtype=torch.int64, device=f"cuda:{device}")

        def uniform(shape, qcol):
            t = torch.randint(0, 1 << 62, shape, generator=gen, device=qall.device, dtype=torch.int64) % qcol
            torch.cuda.synchronize()
            return t

        def key(elt):
            shape = (MLP_DNUM, 2, len(q) + len(p), n)
            t = uniform(shape, qall.view(1, 1, -1, 1))
            kk = ctx.upload_key_device(t.data_ptr(), shape, elt)
            del t
            return kk

        self.layout = layout = nn.Layout(n // 2, 256, 64)
        steps = nn.mlp_rotation_steps(MLP_DIMS, layout)
        self.keys = [key(0)] + [key(galois_elt(n, s)) for s in steps]
        self.ev = ev = ckg.CudaEvaluator(ctx, self.keys[0], self.keys[1:])
        top, delta = len(q) - 1, 2.0 ** 42
        self.cts = []

        def ct(level, scale):
            t = uniform((2, level + 1, n), qall[:level + 1].view(1, -1, 1))
            c = ev.upload_ct_device(t.data_ptr(), 2, level, scale)
            ctx.sync()
            del t
            self.cts.append(c)
            return c

        per_layer, (y_level, y_scale) = nn.Mlp.scales(ev, MLP_DIMS, top, delta)
        self.layers = []
        for i, (_, _, b_scale) in enumerate(per_layer):
            sh = nn.LayerShape(MLP_DIMS[i + 1], MLP_DIMS[i], layout)
            w = nn.EncWeights([ct(top, delta) for _ in range(sh.m)], MLP_DIMS[i + 1], MLP_DIMS[i], layout)
            self.layers.append((w, ct(top, b_scale)))
        self.x, self.y = ct(top, delta), ct(y_level, y_scale)
        self.trace = None

    def step(self):
        nn = self.ckg.nn
        mlp = nn.Mlp([(nn.Dense(w, b), nn.Square()) for w, b in self.layers])
        tr = nn.Trainer(self.ev, self.layout, [nn.Sgd(0.05) for _ in self.layers])
        tr.train_batch(mlp, self.x, self.y)
        self.trace = tr.trace

    def measure(self, steps=3, warmup=3):
        ckg, torch = self.ckg, self.torch
        self.step()
        self.ctx.sync()
        self.ev.reset_counter()
        l0 = ckg.launch_count()
        self.step()
        self.ctx.sync()
        launches = ckg.launch_count() - l0
        c = self.ev.counter()
        ms, _ = timed(torch, self.ctx, self.step, steps, warmup)
        ks = c["rotations"] + c["relins"]
        return {"ms": round(ms / steps, 3), "unit": "ms per training step (device events, back-to-back)",
                "key_switches": int(ks), "keyswitch_per_s": round(ks * steps / (ms * 1e-3), 1),
                "counts": c, "launches": int(launches),
                "params": "n16_train: N=2^16, 58 + 31x42-bit q, 4x58-bit p, dnum 8, scale 2^42",
                "network": "196 -> 64 -> 10, Square after each layer, SGD, batch 64, Layout(2^15, 256, 64)",
                "levels": dict(self.trace), "keys": len(self.keys),
                "data": "synthetic uniform key material and ciphertexts at the client's levels and scales"}


def max_over_ranks(dist, ms, device="cuda"):
    """The slowest rank's time: every rank's device-measured milliseconds, max-reduced."""
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_objects(dist, obj):
    """Every rank's `obj`, in rank order (a collective: every rank calls it)."""
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out


def rank_stream(rank, count=MIX_OPS):
    """The op stream of one rank: independent seeded ciphertexts per rank (weak scaling)."""
    return mix_ops(20261203 + rank, count)


def timed(torch, ctx, fn, steps, warmup, dist=None, tail=None):
    """Device time of `steps` calls of fn on the library's stream; `tail` queues what the end
    must wait for (e.g. the overlapped downloads) before the end event."""
    for _ in range(warmup):
        fn()
    if tail:
        tail()
    ctx.sync()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    stream = torch.cuda.ExternalStream(ctx.stream)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    extra = None
    for _ in range(steps):
        extra = fn()
    if tail:
        tail()
    end.record(stream)
    ctx.sync()
    torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    if dist:
        ms = max_over_ranks(dist, ms)
    return ms, extra


def stream_roofline(ops, n, k, alpha, ms_per_step, peaks):
    """HBM fraction of the whole batched stream. Algorithmic bytes per op, inputs read once
    and outputs written once (limbs of 8N bytes): HMult+relin+rescale 4(l+1) + 2l, rotation
    2(l+1) + 2(l+1), PtMult+rescale 3(l+1) + 2l; plus each distinct key read once per chunk
    (2 beta (l+1+k) limbs at the highest level that uses it there). Chunks follow the batch
    builder: key-switching ops sorted by key, then the plaintext products, at most 128 ops
    and 16 GiB of scratch per chunk (keys ordered here by Galois element, relinearization
    first; the builder orders them by address, which moves at most one key group per chunk
    boundary)."""
    limb = 8 * n

    def beta(l):
        return (l + 1 + alpha - 1) // alpha

    def conv_limbs(l):
        return sum((l + 1) - min(alpha, l + 1 - j * alpha) + k for j in range(beta(l)))

    def scratch_words(kind, l):
        if kind == "pmul":
            return 4 * (l + 1) * n
        w = (3 if kind == "mul" else 1) * (l + 1) + (l + 1) + conv_limbs(l) + 2 * (l + 1 + k) + 2 * (k + l + 1)
        return (w + (4 * (l + 1) if kind == "mul" else 0)) * n

    total, ks, pm = 0, [], []
    for kind, l, steps in ops:
        if kind == "mul":
            total += (4 * (l + 1) + 2 * l) * limb
            ks.append((0, kind, l))
        elif kind == "rot":
            total += 4 * (l + 1) * limb
            if steps % (n // 2):
                ks.append((galois_elt(n, steps), kind, l))
        else:
            total += (3 * (l + 1) + 2 * l) * limb
            pm.append((None, kind, l))
    ks.sort(key=lambda x: x[0])
    chunks, cur = [], 0
    for key, kind, l in ks + pm:
        w = scratch_words(kind, l)
        if not chunks or len(chunks[-1]) >= 128 or (cur + w) * 8 > (16 << 30):
            chunks.append([])
            cur = 0
        chunks[-1].append((key, l))
        cur += w
    key_bytes = 0
    for ch in chunks:
        top = {}
        for key, l in ch:
            if key is not None:
                top[key] = max(top.get(key, -1), l)
        key_bytes += sum(2 * beta(l) * (l + 1 + k) * limb for l in top.values())
    total += key_bytes
    peak = float(peaks.get("hbm_gbs") or 6650.0)
    gbs = total / (ms_per_step * 1e-3) / 1e9
    return {"scope": "whole batched stream, per step", "bound": "hbm", "alg_bytes": int(total),
            "key_bytes": int(key_bytes), "chunks": len(chunks), "achieved": round(gbs, 1), "peak": peak,
            "unit": "GB/s", "frac": round(gbs / peak, 4),
            "note": "bounded by the integer and FP64 pipes (NTT butterflies, base conversion), not by HBM"}


def pcie_ceiling(torch, h2d_bytes, d2h_bytes, ms_per_step, nbytes=1 << 30):
    """The host link's bound on the e2e step: 1 GiB pinned <-> device copies timed with CUDA
    events, each direction alone and both at once on two streams (as the e2e step overlaps
    them). bound_ms_per_step = the step's larger direction at the concurrent per-direction rate."""
    h_in = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    h_out = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d_in = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    d_out = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()

    def run(up, down, reps=3):
        best = None
        for _ in range(reps + 1):
            torch.cuda.synchronize()
            evs = []
            for on, st, fn in ((up, s_in, lambda: d_in.copy_(h_in, non_blocking=True)),
                               (down, s_out, lambda: h_out.copy_(d_out, non_blocking=True))):
                if on:
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(st)
                    with torch.cuda.stream(st):
                        fn()
                    b.record(st)
                    evs.append((a, b))
            torch.cuda.synchronize()
            ms = max(a.elapsed_time(b) for a, b in evs)
            best = ms if best is None else min(best, ms)
        return nbytes / (best * 1e-3) / 1e9

    h2d, d2h, both = run(True, False), run(False, True), run(True, True)
    bound = max(h2d_bytes, d2h_bytes) / (both * 1e9) * 1e3
    del h_in, h_out, d_in, d_out
    return {"h2d_gbs": round(h2d, 1), "d2h_gbs": round(d2h, 1), "concurrent_gbs_each_way": round(both, 1),
            "bound_ms_per_step": round(bound, 1), "frac": round(bound / ms_per_step, 3),
            "how": "1 GiB pinned copies, CUDA events, best of 3; both directions at once on two streams"}


# DRAM bytes (read + write) per 768-limb transform of ntt_roofline, from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum) of `bench.py --profile ntt`: its twelve
# launches (three 256-limb chunks, a column and a row pass each, forward then inverse) summed
# and halved.
NTT_TRAFFIC_PER_TRANSFORM = 1370446208


def ntt_pair(torch, ctx, n, limbs=768):
    """One forward and one inverse NTT over `limbs` limbs (24 data + 8 special primes cycled, as
    in a batched stage), in place; returns (buffer, primes) for more rounds."""
    buf = torch.randint(0, 1 << 40, (limbs, n), dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    nprimes = len(ctx.q) + ctx.k
    primes = [i % nprimes for i in range(limbs)]
    ctx.ntt(buf.data_ptr(), buf.data_ptr(), primes, False)
    ctx.ntt(buf.data_ptr(), buf.data_ptr(), primes, True)
    return buf, primes


def raw_keyswitch(torch, ks_call, stream_ptr, q_all, n, level=PLAIN_LEVEL, calls=128, distinct=16, seed=7):
    """Config 2's per-op key switch: `calls` single key switches of level-`level` polynomials
    (24 limbs at level 23), one call each (ks_call(in_ptr, out_b_ptr, out_a_ptr)), cycling over
    `distinct` seeded uniform inputs (more than L2 together), timed with CUDA events on the
    caller's stream after three warm-up calls."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    qcol = q_all[: level + 1].view(-1, 1)
    ins = [torch.randint(0, 1 << 62, (level + 1, n), generator=g, device="cuda", dtype=torch.int64) % qcol
           for _ in range(distinct)]
    ob = torch.empty((level + 1, n), dtype=torch.int64, device="cuda")
    oa = torch.empty_like(ob)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(stream_ptr)
    for i in range(3):
        ks_call(ins[i % distinct].data_ptr(), ob.data_ptr(), oa.data_ptr())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for i in range(calls):
        ks_call(ins[i % distinct].data_ptr(), ob.data_ptr(), oa.data_ptr())
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    return {"value": round(calls / (ms * 1e-3), 2), "unit": "keyswitch/s", "ms_per_keyswitch": round(ms / calls, 4),
            "workload": f"{calls} key switches of single polynomials at {level + 1} limbs (N=2^16, 24+8 primes, "
                        "dnum 3), one call each"}


def ntt_32_limbs(torch, ntt_call, stream_ptr, n, reps=20):
    """Config 2's standalone transform: forward + inverse NTT over 32 limbs (24 data + 8 special
    primes), in place, timed with CUDA events on the caller's stream."""
    buf = torch.randint(0, 1 << 40, (32, n), dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    primes = list(range(32))
    stream = torch.cuda.ExternalStream(stream_ptr)
    for _ in range(2):
        ntt_call(buf.data_ptr(), primes, False)
        ntt_call(buf.data_ptr(), primes, True)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps):
        ntt_call(buf.data_ptr(), primes, False)
        ntt_call(buf.data_ptr(), primes, True)
    b.record(stream)
    torch.cuda.synchronize()
    return {"us_per_pair": round(a.elapsed_time(b) * 1e3 / reps, 2), "limbs": 32}


def reference_gpu(torch):
    """The reference's own CUDA kernels (crates/ckks-train-cuda/kernels, unmodified, --fmad=false)
    through the launch sequences of its host code, on this device: the per-op key switch and the
    32-limb NTT pair of config 2 (oracle/ref_gpu)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import ref_gpu
    if not ref_gpu.available():
        return {"unavailable": "oracle/_ref/libref_gpu.so was not built (the reference tree was absent at build time)"}
    P = O.Params.from_bits(LOG_N, Q_BITS, P_BITS, 50, DNUM)
    R = ref_gpu.RefGpu(LOG_N, P.q, P.p, DNUM)
    n = P.n
    q_all = torch.tensor(P.q + P.p, dtype=torch.int64, device="cuda")
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    key = torch.randint(0, 1 << 62, (DNUM, 2, P.nq + P.np_, n), generator=g, device="cuda",
                        dtype=torch.int64) % q_all.view(1, 1, -1, 1)
    torch.cuda.synchronize()
    ks = raw_keyswitch(torch, lambda i, b, a: R.key_switch(i, PLAIN_LEVEL, key.data_ptr(), b, a), R.stream, q_all, n)
    ntt = ntt_32_limbs(torch, lambda buf, primes, inv: R.ntt(buf, primes, inv), R.stream, n)
    return {"kernels": "crates/ckks-train-cuda/kernels/{ntt,basis,keyswitch}.cu compiled unmodified (--fmad=false) "
                       "and driven through the launch sequences of src/ks.rs, src/basis.rs, src/device.rs "
                       "(oracle/ref_gpu/ref_ks.cu)",
            "keyswitch_raw": ks, "ntt_pair": ntt}


def ntt_roofline(torch, S, peaks, limbs=768):
    """Forward + inverse NTT over `limbs` limbs (24 data + 8 special primes cycled, as in a
    batched stage), timed alone with CUDA events on the library's stream. Algorithmic bytes
    per transform: every limb read and written once (both passes together)."""
    ctx = S.ctx
    buf, primes = ntt_pair(torch, ctx, S.n, limbs)
    stream = torch.cuda.ExternalStream(ctx.stream)
    for _ in range(2):
        ctx.ntt(buf.data_ptr(), buf.data_ptr(), primes, False)
        ctx.ntt(buf.data_ptr(), buf.data_ptr(), primes, True)
    ctx.sync()
    reps = 10
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        ctx.ntt(buf.data_ptr(), buf.data_ptr(), primes, False)
        ctx.ntt(buf.data_ptr(), buf.data_ptr(), primes, True)
    b.record(stream)
    ctx.sync()
    ms = a.elapsed_time(b) / (2 * reps)
    alg = limbs * S.n * 8 * 2
    achieved = alg / (ms * 1e-3) / 1e9
    peak = peaks.get("hbm_gbs", 6650.0)
    return {"kernel": f"ntt forward/inverse, {limbs} limbs of N=2^16 per transform (2 passes)", "bound": "hbm",
            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": NTT_TRAFFIC_PER_TRANSFORM if limbs == 768 else None,
            "ms_per_transform": round(ms, 4), "alg_bytes": alg,
            "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "fallback"}


# ---- CPU baseline / reference arm ------------------------------------------------------

class CpuPath:
    """The oracle's CPU evaluator (the reference's CPU path restated, OpenMP over the units
    of its `parallel` feature) with keys from its own key generator: the relinearization key
    and, generated on first use, the Galois key of every rotation step a sample draws."""

    def __init__(self, threads, seed=20261203):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        self.O, self.threads = O, threads
        O.set_threads(threads)
        self.P = O.Params.from_bits(LOG_N, Q_BITS, P_BITS, 50, DNUM)
        self.kg = O.KeyGenerator(self.P, 5)
        self.rk = self.kg.relin_key()
        self.ops = mix_ops(seed, 256)
        self.gk, self.ev, self.pos = {}, None, 0

    def take(self, key_switches):
        """The next ops of the mix, in order (wrapping), that hold `key_switches` key switches;
        every rotation among them gets its Galois key before it is timed."""
        out, ks = [], 0
        while ks < key_switches:
            op = self.ops[self.pos]
            self.pos = (self.pos + 1) % len(self.ops)
            out.append(op)
            ks += op[0] != "pmul"
        need = {self.O.galois_elt(self.P.n, s) for kind, _, s in out if kind == "rot"} - set(self.gk)
        for e in sorted(need):
            self.gk[e] = self.kg.galois_key(e)
        if need or self.ev is None:
            self.ev = self.O.Evaluator(self.P, self.rk, self.gk)
        return out


def cpu_host():
    """The host the CPU numbers were taken on: model name and logical CPUs."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "logical_cpus": os.cpu_count()}


def cpu_sample(path, key_switches=120):
    """Key switches per second of the CPU path on the next ops of the seeded mix, drawn in
    order with none skipped; only the ops themselves are timed (input generation and Galois
    key generation are not)."""
    O, P = path.O, path.P
    ops = path.take(key_switches)
    ev = path.ev
    load0 = os.getloadavg()[0]
    ks, dt, kinds = 0, 0.0, {"mul": 0, "rot": 0, "pmul": 0}
    for i, (kind, level, steps) in enumerate(ops):
        a = ev.ct(np.stack([P.random_q(2 * i + 1, level), P.random_q(2 * i + 2, level)]), SCALE)
        pt = P.random_q(7, level) if kind == "pmul" else None
        t0 = time.perf_counter()
        if kind == "mul":
            ev.rescale(ev.mul(a, a))
        elif kind == "rot":
            ev.rotate(a, steps)
        else:
            ev.rescale(ev.mul_plain(a, pt, SCALE))
        dt += time.perf_counter() - t0
        ks += kind != "pmul"
        kinds[kind] += 1
    load1 = os.getloadavg()[0]
    sample = (f"{ks} key switches of the seeded op mix in order, none skipped ({kinds['mul']} HMult+relin+rescale, "
              f"{kinds['rot']} rotations over {len(path.gk)} Galois keys, {kinds['pmul']} PtMult+rescale; "
              f"limbs 4..24) in {dt:.1f} s on {path.threads} threads; 1-min load {load0:.2f} -> {load1:.2f}")
    return ks / dt, sample


def cpu_crosscheck(threads):
    """The port against the reference's published CPU figure for the same op: relinearize at
    level 31 of n16_train (N = 2^16, 58 + 31 x 42-bit q, 4 x 58-bit p, dnum 8), median of 3,
    on 1 thread and on 12 (or all, if fewer) threads. The published medians are 639.6 ms and
    240.1 ms on an i9-13900KF (docs/m4-report.md, table 1.1, row relinearize)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    wide = min(12, threads)
    O.set_threads(threads)
    P = O.Params.from_bits(16, MLP_Q_BITS, MLP_P_BITS, 42, MLP_DNUM)
    kg = O.KeyGenerator(P, 5)
    ev = O.Evaluator(P, kg.relin_key(), {})
    a = ev.ct(np.stack([P.random_q(1, 31), P.random_q(2, 31)]), 2.0 ** 42)
    b = ev.ct(np.stack([P.random_q(3, 31), P.random_q(4, 31)]), 2.0 ** 42)
    c = ev.mul_no_relin(a, b)
    out = {"op": "relinearize, n16_train level 31", "published_ms": {"1": 639.6, "12": 240.1},
           "published_cpu": "i9-13900KF"}
    for th in (1, wide):
        O.set_threads(th)
        ev.relinearize(c)
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            ev.relinearize(c)
            ts.append(time.perf_counter() - t0)
        out[f"ms_{th}_threads"] = round(sorted(ts)[1] * 1e3, 1)
    O.set_threads(threads)
    return out


def main():
    t_start = time.time()
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--ops", type=int, default=MIX_OPS, help="ops of the batched stream (smaller for profiling)")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-boot", action="store_true")
    ap.add_argument("--boot-only", action="store_true", help="measure the n16_boot bootstrap only")
    ap.add_argument("--serve-only", action="store_true", help="set up and measure the serving loop only")
    ap.add_argument("--serve-lane-sweep", action="store_true",
                    help="measure bootstrap serving under each compute-lane layout at one offered load")
    ap.add_argument("--no-mlp", action="store_true")
    ap.add_argument("--ntt", default="plain", choices=["tma", "plain"],
                    help="NTT column passes: per-tile (plain, the default) or persistent TMA-staged (tma)")
    ap.add_argument("--bconv", default="auto", choices=["auto", "tc", "int"],
                    help="base conversion engine: tensor cores from 6 sources (auto, the default), tensor cores "
                         "at every source count (tc), integer kernels (int)")
    ap.add_argument("--ntt-wave", type=int, default=None, help="fixed NTT limb wave (with --chunk-items; default: autotune)")
    ap.add_argument("--chunk-items", type=int, default=None, help="fixed batch chunk size (with --ntt-wave)")
    ap.add_argument("--mlp-only", action="store_true", help="measure the encrypted MLP training step only")
    ap.add_argument("--config1-only", action="store_true", help="measure the N=2^13 small-ring workload only")
    ap.add_argument("--serve-owners", type=int, default=SERVE_OWNERS)
    ap.add_argument("--serve-requests", type=int, default=SERVE_REQUESTS)
    ap.add_argument("--profile", default=None, choices=["batch", "plain", "boot", "ntt"],
                    help="run the set-up and `warmup` + 1 step of one path, print nothing (for ncu)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    metric, unit = "keyswitch/s N=2^16 L=24 (24+8 primes, dnum 3), batched uneven-level stream", "keyswitch/s"
    config = {"workload": f"batched stream: {args.ops} ciphertexts, limbs uniform in 4..24, seeded mix 40% "
                          "HMult+relin+rescale / 40% rotation +-2^k / 20% PtMult+rescale; one CUDA-graph replay "
                          "per step",
              "params": "N=2^16, 24x50-bit q + 8x60-bit p, dnum 3, 31 keys",
              "l2": "inputs (~10 GB) and keys (3 GB) larger than L2"}

    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        vals, samples = [], []
        path = CpuPath(threads)
        per_step = -(-120 // max(args.steps, 1))
        for _ in range(args.warmup):
            cpu_sample(path, key_switches=2)
        for _ in range(max(args.steps, 1)):
            v, sample = cpu_sample(path, key_switches=per_step)
            vals.append(v)
            samples.append(sample)
        v = float(np.mean(vals))
        sample = f"{len(samples)} steps of: " + samples[-1]
        host = dict(cpu_host(), crosscheck=cpu_crosscheck(threads))
        ref_gpu_line = None
        try:
            import torch
            if torch.cuda.is_available():
                torch.cuda.set_device(local)
                ref_gpu_line = reference_gpu(torch)
        except Exception as e:  # noqa: BLE001 -- the CPU arm's line stands without it
            ref_gpu_line = {"unavailable": f"{type(e).__name__}: {e}"}
        print(json.dumps({"impl": "reference", "metric": metric, "value": round(v, 3), "unit": unit,
                          "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
                          "data": "synthetic", "config": config,
                          "cpu_baseline": dict({"value": round(v, 3), "unit": unit, "cores": threads,
                                                "kind": "port", "sample": sample}, **host),
                          "e2e": {"value": round(v, 3), "unit": unit, "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0},
                          "reference_gpu": ref_gpu_line}))
        return

    import torch
    dist = None
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist_mod
        dist_mod.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=300))
        dist = dist_mod
    ckg = load_package()
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass

    if args.profile == "ntt":  # the roofline's 768-limb forward + inverse transform pair, once
        ctx = ckg.Context.from_bits(LOG_N, Q_BITS, P_BITS, DNUM, device=local, scale_bits=50)
        ntt_pair(torch, ctx, ctx.n)
        ctx.sync()
        return
    if args.profile == "boot":
        B = BootBench(ckg, torch, local)
        for _ in range(args.warmup + 1):
            B.step()
        B.ctx.sync()
        return
    if args.mlp_only:
        out = MlpBench(ckg, torch, local).measure()
        if rank == 0:
            print(json.dumps({"mlp_step": out}))
        return
    if args.config1_only:
        out = Config1(ckg, torch, local).measure()
        if not args.no_cpu_baseline:
            out["cpu"] = cpu_config1(os.cpu_count() or 1)
        if rank == 0:
            print(json.dumps({"config1": out}))
        return
    if args.boot_only:
        out = BootBench(ckg, torch, local).measure()
        if rank == 0:
            print(json.dumps({"bootstrap": out}))
        return
    S = Setup(ckg, torch, local)
    S.ctx.bconv_tc = {"int": 0, "auto": 1, "tc": 2}[args.bconv]
    S.ctx.ntt_tma = args.ntt == "tma"
    if args.serve_lane_sweep:  # bootstrap serving under every lane layout, one offered load
        res, rate = {}, None
        for lanes, prio in ((0, True), (1, True), (1, False), (2, True), (2, False)):
            sv = BootServing(ckg, torch, local, boot_lanes=lanes, boot_priority=prio)
            out = sv.measure(args.serve_requests, rate=rate)
            rate = rate or out["offered_req_s"]
            res[f"lanes{lanes}_{'prio' if prio else 'equal'}"] = {
                k: out[k] for k in ("capacity_req_s", "offered_req_s", "throughput_req_s", "p50_ms", "p99_ms",
                                    "mean_ms", "key_hit_rate", "key_evictions", "batches")}
            sv.close()
            del sv
        if rank == 0:
            print(json.dumps({"serving_lane_sweep": res}))
        return
    if args.serve_only:
        res = {}
        for key, kw, count in (("serving_one_lane", {"boot_lanes": 0}, args.serve_requests),
                               ("serving", {}, args.serve_requests),
                               ("serving_boot_spill", {"owners": BootServing.spill_owners(),
                                                       "budget": SERVE_BOOT_SPILL_BUDGET}, SERVE_BOOT_SPILL_REQUESTS)):
            sv = BootServing(ckg, torch, local, **kw)
            rate = res["serving_one_lane"]["offered_req_s"] if key == "serving" else None
            res[key] = sv.measure(count, rate=rate)
            sv.close()
            del sv
        sv = Serving(S, owners=args.serve_owners)
        res["serving_spill"] = sv.measure(args.serve_requests)
        sv.close()
        if rank == 0:
            print(json.dumps(res))
        return
    if args.profile == "plain":
        P = Plain(S)
        for _ in range(args.warmup + 1):
            P.step()
        S.ctx.sync()
        return
    mix = Mix(S, rank_stream(rank, args.ops), keep_host=not args.no_e2e and args.profile is None)
    tuning = mix.tune(args.ntt_wave, args.chunk_items)
    l0 = ckg.launch_count()
    mix.batch.capture_graph()
    launches_per_step = ckg.launch_count() - l0
    if args.profile == "batch":
        for _ in range(args.warmup + 1):
            mix.step_graph()
        S.ctx.sync()
        return
    with ClockSampler(local) as clk:
        ms, _ = timed(torch, S.ctx, mix.step_graph, args.steps, args.warmup, dist)
    value = mix.ks * args.steps * world / (ms * 1e-3)
    e2e = None
    if not args.no_e2e:
        mix.batch = None  # the timed graph's batch is done with: its scratch goes back to the pool
        gc.collect()
        torch.cuda.empty_cache()
        mix.prepare_e2e()
        steps_e = max(8, args.steps)
        for _ in range(max(3, args.warmup)):  # warm-up: the transfer blocks reach their working set
            mix.step_e2e()
        mix.inflight.clear()
        mix.host_s, mix.host_parts = 0.0, {}
        ts0 = S.ctx.transfer_stats()
        ms_e, (h2d, d2h) = timed(torch, S.ctx, mix.step_e2e, steps_e, 0, dist, tail=S.ctx.join_transfers)
        ts1 = S.ctx.transfer_stats()
        e2e = {"value": round(mix.ks * steps_e * world / (ms_e * 1e-3), 2), "unit": unit,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": round(ms_e / steps_e, 3), "steps": steps_e,
               "host_ms_per_step": round(mix.host_s * 1e3 / steps_e, 2),
               "host_ms_per_step_by_phase": {k: round(v * 1e3 / steps_e, 2) for k, v in mix.host_parts.items()},
               "transfer_stats_per_step": {k: (ts1[k] if k == "upload_pool_bytes" else round((ts1[k] - ts0[k]) / steps_e, 1))
                                           for k in ts1}}
        if rank == 0:  # no collective inside: the other ranks skip it
            e2e["host_link"] = pcie_ceiling(torch, h2d, d2h, ms_e / steps_e)
    plain = None
    if not args.no_plain:
        P = Plain(S)
        # One timed run of 4 steps after 3 warm-up steps; the slowest evaluator call's host time is
        # reported beside it, so a host stall inside the run shows in the line.
        free0 = torch.cuda.mem_get_info()[0]
        ms_p = timed(torch, S.ctx, P.step, 4, 3, dist)[0]
        pv = P.ks * 4 * world / (ms_p * 1e-3)
        PM = PlainMix(mix)
        ms_m = timed(torch, S.ctx, PM.step, 2, 3, dist)[0]
        pm = PM.ks * 2 * world / (ms_m * 1e-3)
        plain = {"value": round(pv, 2), "unit": unit,
                 "workload": "128 ciphertexts at 24 limbs: 128 x (HMult+relin+rescale) + 128 rotations, "
                             "one evaluator call per op; 4 timed steps after 3 warm-up steps",
                 "ms_per_step": round(ms_p / 4, 3), "batched_over_plain": round(value / pv, 2),
                 "same_stream_one_op_at_a_time": round(pm, 2), "batched_over_same_stream_plain": round(value / pm, 2),
                 "slowest_host_call_ms": [round(P.slowest[0] * 1e3, 3), P.slowest[1]],
                 "device_free_gib_before": round(free0 / 2 ** 30, 1)}
    ks_raw = raw_keyswitch(torch, lambda i, b, a: S.ctx.key_switch(S.relin, i, PLAIN_LEVEL, b, a), S.ctx.stream,
                           S.q_all, S.n)
    ntt32 = ntt_32_limbs(torch, lambda buf, primes, inv: S.ctx.ntt(buf, buf, primes, inv), S.ctx.stream, S.n)
    roof = ntt_roofline(torch, S, peaks)
    roof_stream = stream_roofline(rank_stream(rank, args.ops), S.n, S.ctx.k, S.ctx.alpha, ms / args.steps, peaks)
    # The bootstrap, training-step and bootstrap-serving figures are single-GPU measurements: a run
    # on N > 1 GPUs (one replica per rank) reports the batched stream and the routed serving loop.
    single = world == 1

    def release():
        """Drops the batched stream's graph and the torch allocator's cached blocks between
        sections (untimed), so later sections' own pools find the device memory free."""
        mix.batch = None
        gc.collect()
        S.ctx.sync()
        torch.cuda.empty_cache()
        free, total = torch.cuda.mem_get_info(local)
        print(f"release at {time.time() - t_start:.0f} s: {free / 2 ** 30:.1f} of {total / 2 ** 30:.1f} GiB free",
              file=sys.stderr)

    boot = None
    if not args.no_boot and single:
        release()
        boot = BootBench(ckg, torch, local).measure()
    mlp_step = None
    if not args.no_mlp and single:
        release()
        mb = MlpBench(ckg, torch, local)
        mlp_step = mb.measure()
        del mb
    config1 = None
    if single:
        release()
        c1 = Config1(ckg, torch, local)
        config1 = c1.measure()
        del c1
    serving = serving_spill = serving_boot_spill = serving_one_lane = None
    if not args.no_serve and single:
        release()
        # each server is closed and its context released before the next one fills the device
        sv = BootServing(ckg, torch, local, boot_lanes=0)
        serving_one_lane = sv.measure(args.serve_requests)
        sv.close()
        del sv
        release()
        sv = BootServing(ckg, torch, local)  # two lanes, at the one-lane run's offered load
        serving = sv.measure(args.serve_requests, rate=serving_one_lane["offered_req_s"])
        sv.close()
        del sv
        release()
        sv = BootServing(ckg, torch, local, owners=BootServing.spill_owners(), budget=SERVE_BOOT_SPILL_BUDGET)
        serving_boot_spill = sv.measure(SERVE_BOOT_SPILL_REQUESTS)
        sv.close()
        del sv
        release()
        sv = Serving(S, owners=args.serve_owners)
        serving_spill = sv.measure(args.serve_requests)
        sv.close()
    elif not args.no_serve:  # N GPUs: owners placed on ranks by the router, one server per rank
        release()
        router = ckg.OwnerRouter([Serving.key_bytes_per_owner()] * args.serve_owners, world)
        sv = Serving(S, owners=args.serve_owners, router=router, rank=rank)
        serving_spill = dict(sv.measure(args.serve_requests, dist=dist), ranks=world,
                             owners_per_rank=[len(router.owners_of(r)) for r in range(world)])
        sv.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, sample = cpu_sample(CpuPath(threads))
        cpu = dict({"value": round(v, 3), "unit": unit, "cores": threads, "kind": "port", "sample": sample},
                   **cpu_host(), crosscheck=cpu_crosscheck(threads))
        if config1:
            config1["cpu"] = cpu_config1(threads)
    if rank == 0:
        line = {"metric": metric, "value": round(value, 2), "unit": unit, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u64",
                "data": "synthetic (seeded uniform ciphertexts and plaintexts, uniform key material)",
                "config": dict(config, key_switches_per_step=int(mix.ks), bconv=args.bconv, ntt=args.ntt,
                               autotune={"ntt_wave": tuning["ntt_wave"], "chunk_items": tuning["chunk_items"],
                                         "trials_ms": [[w, c, round(m, 3)] for w, c, m in tuning["trials"]]}),
                "e2e": e2e,
                "gpu_launches": int(launches_per_step * args.steps), "plain": plain,
                "keyswitch_raw": ks_raw, "ntt_pair_32_limbs": ntt32, "roofline": roof,
                "roofline_stream": roof_stream,
                "bootstrap": boot, "mlp_step": mlp_step, "config1": config1, "serving": serving, "serving_one_lane": serving_one_lane,
                "serving_boot_spill": serving_boot_spill, "serving_spill": serving_spill, "cpu_baseline": cpu,
                "clocks": clk.summary()}
        print(json.dumps(line))
    mix.batch = None
    S.ctx.sync()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
