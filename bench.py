"""Key-switching throughput of the B200 RNS-CKKS evaluator path (one JSON line).

Workload (one step): N = 2^16, 24 x 50-bit data primes + 8 x 60-bit special primes,
dnum = 3 (alpha = 8), 128 seeded uniform ciphertexts at 24 limbs (level 23):
128 x (HMult + relinearization + rescale) and 128 rotations by +-2^k (k = 0..14, 30 Galois
keys), i.e. 256 key switches. The metric is key switches per second.

`value` runs the inputs resident in HBM through the evaluator's C ABI; `e2e` runs the same
step with the inputs copied from pinned host memory and every result copied back inside
the timed region. `--impl reference` times the CPU path of the reference (the oracle's
restatement of crates/ckks-train-ckks, OpenMP over the same units as its `parallel`
feature) on a bounded sample of the same workload.

Multi-GPU: each rank runs the same step on its own GPU with its own keys (independent
ciphertexts shard with no exchange, weak scaling); the time is the max over ranks.
"""

import argparse
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
NCT = 128
LEVEL = 23
ROT_STEPS = [s * (1 << k) for k in range(15) for s in (1, -1)]  # +-2^k, k = 0..14


def load_package():
    if "ckks_train_b200" in sys.modules:
        return sys.modules["ckks_train_b200"]
    spec = importlib.util.spec_from_file_location("ckks_train_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ckks_train_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


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


# ---- the workload ---------------------------------------------------------------------

class Workload:
    """Keys, inputs and the evaluator of one rank (synthetic uniform key material)."""

    def __init__(self, ckg, torch, device, ncts=NCT):
        self.ckg, self.torch = ckg, torch
        self.ctx = ckg.Context.from_bits(LOG_N, Q_BITS, P_BITS, DNUM, device=device, scale_bits=50)
        ctx = self.ctx
        self.n = ctx.n
        self.ncts = ncts
        g = torch.Generator(device=f"cuda:{device}")
        g.manual_seed(20261203 + device)
        self.gen = g
        q_all = torch.tensor(ctx.q + ctx.p, dtype=torch.int64, device=f"cuda:{device}")
        self.q_all = q_all
        key_limbs = torch.cat([q_all[: LEVEL + 1], q_all[len(ctx.q):]])  # key Q limbs 0..L then P
        self.keys = []

        def make_key(elt):
            shape = (DNUM, 2, len(ctx.q) + ctx.k, self.n)
            qcol = torch.cat([q_all[: len(ctx.q)], q_all[len(ctx.q):]]).view(1, 1, -1, 1)
            t = torch.randint(0, 1 << 62, shape, generator=g, device=q_all.device, dtype=torch.int64) % qcol
            torch.cuda.synchronize()
            k = ctx.upload_key_device(t.data_ptr(), shape, elt)
            del t
            return k

        self.relin = make_key(0)
        self.galois = {}
        for s in ROT_STEPS:
            elt = galois_elt(self.n, s)
            if elt not in self.galois:
                self.galois[elt] = make_key(elt)
        self.ev = ckg.CudaEvaluator(ctx, self.relin, list(self.galois.values()))
        # inputs: NCT ciphertexts of 2 components at LEVEL (24 limbs), uniform residues
        shape = (ncts, 2, LEVEL + 1, self.n)
        qcol = q_all[: LEVEL + 1].view(1, 1, -1, 1)
        self.inputs = torch.randint(0, 1 << 62, shape, generator=g, device=q_all.device, dtype=torch.int64) % qcol
        torch.cuda.synchronize()
        self.host_in = torch.empty(shape, dtype=torch.int64, pin_memory=True)
        self.host_in.copy_(self.inputs.cpu())
        self.ct_words = 2 * (LEVEL + 1) * self.n
        self.cts = [self.ev.upload_ct_device(self.inputs[i].data_ptr(), 2, LEVEL, SCALE) for i in range(ncts)]
        self.ctx.sync()
        # pinned host staging of the results (largest result: 2 x 24 limbs)
        self.host_out = torch.empty((2 * ncts, 2, LEVEL + 1, self.n), dtype=torch.int64, pin_memory=True)

    def step_ops(self, cts):
        """128 x (mul + relin + rescale), 128 rotations by +-2^k; returns the results."""
        ev = self.ev
        out = []
        for i in range(self.ncts):
            out.append(ev.rescale(ev.mul(cts[i], cts[(i + 1) % self.ncts])))
        for i in range(self.ncts):
            out.append(ev.rotate(cts[i], ROT_STEPS[i % len(ROT_STEPS)]))
        return out

    def step_resident(self):
        return self.step_ops(self.cts)

    def step_e2e(self):
        """Through the C ABI with host buffers: upload_ct of the step's inputs from pinned
        host memory, the ops, and an asynchronous download of every result to pinned host
        memory; the caller's timing ends after the stream has drained."""
        ev = self.ev
        stride = self.ct_words * 8
        base_in = self.host_in.data_ptr()
        cts = [ev.upload_ct_host_ptr(base_in + i * stride, 2, LEVEL, SCALE) for i in range(self.ncts)]
        res = self.step_ops(cts)
        base_out = self.host_out.data_ptr()
        for i, r in enumerate(res):
            ev.download_ct_async(r, base_out + i * stride)
        h2d = self.ncts * self.ct_words * 8
        d2h = sum(2 * (r.level() + 1) * self.n * 8 for r in res)
        return h2d, d2h

    def close(self):
        self.ctx.sync()
        self.cts = None
        self.ev = None
        self.galois = None
        self.relin = None
        self.inputs = None
        self.host_in = None
        self.host_out = None


def galois_elt(n, step):
    m = 2 * n
    k = step % (n // 2)
    return pow(3, k, m)


# ---- timing ---------------------------------------------------------------------------

def timed(torch, ctx, fn, steps, warmup, dist=None):
    for _ in range(warmup):
        fn()
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
    end.record(stream)
    ctx.sync()
    torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    return ms, extra


def ntt_roofline(ckg, torch, w, peaks):
    """The forward + inverse NTT of 32 limbs (24 data + 8 special), timed alone with CUDA
    events on the library's stream; algorithmic bytes = every limb read and written once
    per transform."""
    ctx = w.ctx
    limbs = len(ctx.q) + ctx.k
    buf = torch.randint(0, 1 << 40, (limbs, w.n), dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    primes = list(range(limbs))
    stream = torch.cuda.ExternalStream(ctx.stream)
    for _ in range(3):
        ctx.ntt(buf.data_ptr(), buf.data_ptr(), primes, False)
        ctx.ntt(buf.data_ptr(), buf.data_ptr(), primes, True)
    ctx.sync()
    reps = 50
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        ctx.ntt(buf.data_ptr(), buf.data_ptr(), primes, False)
        ctx.ntt(buf.data_ptr(), buf.data_ptr(), primes, True)
    b.record(stream)
    ctx.sync()
    ms = a.elapsed_time(b) / (2 * reps)  # one transform over 32 limbs
    alg = limbs * w.n * 8 * 2
    achieved = alg / (ms * 1e-3) / 1e9
    peak = peaks.get("hbm_gbs", 6650.0)
    return {"kernel": "ntt (32 limbs, N=2^16, one transform = 2 passes)", "bound": "hbm",
            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": None, "ms_per_launch": round(ms, 5), "alg_bytes": alg,
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}


# ---- CPU baseline / reference arm ------------------------------------------------------

def cpu_sample(threads, budget_s=20.0):
    """The oracle's CPU evaluator on a bounded sample of the workload (mul+relin+rescale and
    rotations at level 23), keys generated by its own key generator."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.set_threads(threads)
    P = O.Params.from_bits(LOG_N, Q_BITS, P_BITS, 50, DNUM)
    kg = O.KeyGenerator(P, 5)
    rk = kg.relin_key()
    e1 = O.galois_elt(P.n, 1)
    gk = {e1: kg.galois_key(e1)}
    ev = O.Evaluator(P, rk, gk)
    a = ev.ct(np.stack([P.random_q(1, LEVEL), P.random_q(2, LEVEL)]), SCALE)
    b = ev.ct(np.stack([P.random_q(3, LEVEL), P.random_q(4, LEVEL)]), SCALE)
    done, t0 = 0, time.perf_counter()
    while True:
        ev.rescale(ev.mul(a, b))
        ev.rotate(a, 1)
        done += 2
        if time.perf_counter() - t0 > budget_s / 2 or done >= 8:
            break
    dt = time.perf_counter() - t0
    return done / dt, f"{done} key switches ({done // 2} mul+relin+rescale, {done // 2} rotations) at 24 limbs"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ncts", type=int, default=NCT, help="ciphertexts per step (smaller for profiling)")
    ap.add_argument("--profile", action="store_true", help="run `warmup` + one step and exit (for ncu)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    metric, unit = "keyswitch/s N=2^16 L=24 (24+8 primes, dnum 3)", "keyswitch/s"
    config = {"workload": "N=2^16, 24x50-bit q + 8x60-bit p, dnum 3; 128 uniform ciphertexts at 24 limbs; "
                          "128 x (HMult+relin+rescale) + 128 rotations by +-2^k (k=0..14)",
              "key_switches_per_step": 2 * NCT, "path": "plain per-op evaluator calls",
              "l2": "inputs (3.2 GB) and keys (3 GB) larger than L2"}

    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        vals = []
        for _ in range(args.warmup):
            pass
        for _ in range(max(args.steps, 1)):
            v, sample = cpu_sample(threads, budget_s=20.0 / max(args.steps, 1))
            vals.append(v)
        v = float(np.mean(vals))
        print(json.dumps({"impl": "reference", "metric": metric, "value": round(v, 3), "unit": unit,
                          "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                          "higher_is_better": True, "dtype": "u64", "data": "synthetic", "config": config,
                          "cpu_baseline": {"value": round(v, 3), "unit": unit, "cores": threads, "kind": "port",
                                           "sample": sample},
                          "e2e": {"value": round(v, 3), "unit": unit, "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))
        dist = dist_mod
    else:
        torch.cuda.set_device(local)
    ckg = load_package()
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass

    w = Workload(ckg, torch, local, args.ncts)
    if args.profile:
        for _ in range(args.warmup + 1):
            w.step_resident()
        w.close()
        return
    l0 = ckg.launch_count()
    with ClockSampler(local) as clk:
        ms, _ = timed(torch, w.ctx, w.step_resident, args.steps, args.warmup, dist)
    launches = (ckg.launch_count() - l0) // (args.steps + args.warmup) * args.steps
    ks = 2 * w.ncts * args.steps * world
    value = ks / (ms * 1e-3)
    ms_e2e, bytes_e2e = timed(torch, w.ctx, w.step_e2e, args.steps, max(args.warmup, 1), dist)
    e2e = 2 * w.ncts * args.steps * world / (ms_e2e * 1e-3)
    roof = ntt_roofline(ckg, torch, w, peaks)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, sample = cpu_sample(threads)
        cpu = {"value": round(v, 3), "unit": unit, "cores": threads, "kind": "port", "sample": sample}
    if rank == 0:
        line = {"metric": metric, "value": round(value, 2), "unit": unit, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded uniform "
                "ciphertexts and uniform key material)", "config": config,
                "e2e": {"value": round(e2e, 2), "unit": unit, "h2d_bytes_per_step": bytes_e2e[0],
                        "d2h_bytes_per_step": bytes_e2e[1]},
                "gpu_launches": int(launches), "roofline": roof, "cpu_baseline": cpu, "clocks": clk.summary()}
        print(json.dumps(line))
    w.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
