"""The multi-GPU path of bench.py on CPU with two gloo ranks: each rank runs its own
independent stream (no data-path collective), and the only exchange is the max-reduction
of the per-rank device times."""

import importlib.util
import os
import socket

import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    b = _bench()
    mx = b.max_over_ranks(dist, 10.0 * (rank + 1), device="cpu")
    stream = b.rank_stream(rank, 32)
    out[rank] = (mx, stream)
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_max_time_and_independent_streams():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
        r0, r1 = out[0], out[1]
    assert r0[0] == r1[0] == 20.0
    assert r0[1] != r1[1]
    assert r0[1] == _bench().rank_stream(0, 32)


class _FakeServer:
    """Stands in for the GPU server: records each submission's owner and completes it 0.5 ms
    after submission."""

    def __init__(self, fail_every=0):
        import time
        self.time, self.t0, self.times, self.seen = time, time.perf_counter(), [], []
        self.fail_every, self.failures = fail_every, 0

    def _submit(self, owner):
        t = (self.time.perf_counter() - self.t0) * 1e6
        self.seen.append(owner)
        self.times.append((t, t, t + 500.0))
        return len(self.times) - 1

    def submit_mul(self, o, a, b):
        return self._submit(o)

    def submit_rotate(self, o, a, steps):
        return self._submit(o)

    def submit_matvec(self, o, d, stride, diag, x):
        return self._submit(o)

    def result_times(self, i, timeout_ms):
        if self.fail_every and i % self.fail_every == self.fail_every - 1:
            self.failures += 1
            return 7, None, (0.0, 0.0, 0.0)  # an out-of-memory status
        return 0, None, self.times[i]

    def stats(self):
        keys = ("batches", "multi_owner_batches", "key_hits", "key_misses", "key_evictions", "key_upload_bytes",
                "budget_waits", "hbm_budget", "peak_device_bytes")
        return dict.fromkeys(keys, 0)


def _serving_worker(rank, world, port, owners, out, fail_every=(0, 0)):
    import numpy as np
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    b = _bench()
    router = b.load_package().OwnerRouter([b.Serving.key_bytes_per_owner()] * owners, world)
    sv = b.Serving.__new__(b.Serving)
    local = router.owners_of(rank)
    sv.rng, sv.owners, sv.srv = np.random.default_rng(7), owners, _FakeServer(fail_every[rank])
    sv.steps = list(range(1, 8)) + [8 * k for k in range(1, 8)]
    sv.slot = {g: i for i, g in enumerate(local)}
    sv.inputs = {g: [("ct", g, lv) for lv in (23, 17, 11, 5)] for g in local}
    sv.diag = {23: "diag23", 11: "diag11"}
    sv.key_bytes, sv.register_s = len(local) * b.Serving.key_bytes_per_owner(), 0.0
    res = sv.measure(requests=64, load=0.7, dist=dist)
    out[rank] = (res, sorted({local[o] for o in sv.srv.seen}), local, len(sv.srv.seen), sv.srv.failures)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_routed_serving():
    """bench.py's serving loop on 2 gloo ranks with the owner router: every rank draws the same
    request stream and submits exactly the requests of the owners placed on it, and the pooled
    result (all latencies, capacity summed, longest span) is the same on both ranks."""
    owners = 6
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_serving_worker, args=(2, _free_port(), owners, out), nprocs=2, join=True,
                           start_method="spawn")
        r0, r1 = out[0], out[1]
    assert r0[0] == r1[0]
    assert r0[0]["served"] == 64 and r0[0]["requests"] == 64
    assert set(r0[2]).isdisjoint(r1[2]) and sorted(r0[2] + r1[2]) == list(range(owners))
    assert set(r0[1]) <= set(r0[2]) and set(r1[1]) <= set(r1[2])
    assert r0[3] + r1[3] == 96 + 64 + 64  # warm-up, saturation and timed runs, split between ranks


def test_two_rank_routed_serving_counts_failures():
    """A rank whose server fails some requests: the pooled result counts every rank's failures,
    serves the rest, and both ranks report the same pooled figures (no rank hangs on a failure)."""
    owners = 6
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_serving_worker, args=(2, _free_port(), owners, out, (0, 5)), nprocs=2, join=True,
                           start_method="spawn")
        r0, r1 = out[0], out[1]
    assert r0[0] == r1[0]
    assert r0[4] == 0 and r1[4] > 0
    assert r0[0]["failed"] == r1[4]
    assert 0 < r0[0]["served"] < 64


def test_two_rank_routed_serving_with_an_idle_rank():
    """One owner on two ranks: the rank without owners submits nothing, and both still finish the
    same collective steps with the same pooled result."""
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_serving_worker, args=(2, _free_port(), 1, out), nprocs=2, join=True,
                           start_method="spawn")
        r0, r1 = out[0], out[1]
    assert r0[0] == r1[0]
    assert r0[2] == [0] and r1[2] == [] and r1[3] == 0
    assert r0[0]["served"] == 64 and r0[0]["failed"] == 0


def test_owner_router_balances_key_bytes():
    b = _bench()
    R = b.load_package().OwnerRouter
    r = R([5, 1, 1, 1, 1, 1], 2)
    assert r.load == [5, 5] and r.owners_of(0) == [0] and r.owners_of(1) == [1, 2, 3, 4, 5]
    r = R([1] * 7, 3)
    assert [len(r.owners_of(k)) for k in range(3)] == [3, 2, 2]
    assert r.split(list(range(7)), 1, lambda o: o) == r.owners_of(1)
    assert R([1] * 4, 1).owners_of(0) == [0, 1, 2, 3]
