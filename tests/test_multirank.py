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
