"""Overlapped host transfers (include/ckg.h, "overlapped host transfers"): uploads on the
context's upload stream, downloads on its download stream. Results equal the plain uploads and
downloads and the oracle's, work queued after an upload sees its data, and a ciphertext whose
handle is freed right after its download is not overwritten before the copy ends."""

import numpy as np
import pytest

from gpu_util import assert_same, random_ct, torch_dev
from test_gpu_eval import Env

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(ckg, oracle):
    return Env(ckg, oracle, "small", [1, 2])


def _pinned(arr):
    torch = torch_dev()
    return torch.from_numpy(np.ascontiguousarray(arr, np.uint64).view(np.int64)).pin_memory()


def _empty_pinned(shape):
    torch = torch_dev()
    return torch.empty(shape, dtype=torch.int64).pin_memory()


def test_overlapped_batch_matches_oracle(env):
    ckg, P, gpu, cpu = env.ckg, env.P, env.gpu, env.cpu
    L = P.max_level
    ins = [random_ct(P, 10 + i, L) for i in range(6)]
    host_in = [_pinned(a) for a in ins]
    pt = P.random_q(77, L)
    host_pt = _pinned(pt)
    outs_host = [_empty_pinned((2, L, P.n)), _empty_pinned((2, L + 1, P.n)), _empty_pinned((2, L, P.n))]
    for step in range(3):  # the same host buffers every step, as a pipelined client would use them
        g = [gpu.upload_ct_overlap(h.data_ptr(), 2, L, env.scale) for h in host_in]
        gp = gpu.upload_pt_overlap(host_pt.data_ptr(), L, env.scale)
        b = ckg.Batch(gpu)
        res = [b.mul_relin_rescale(g[0], g[1]), b.rotate(g[2], 1), b.mul_plain_rescale(g[3], gp)]
        b.run()
        for r, h in zip(res, outs_host):
            gpu.download_ct_overlap(r, h.data_ptr())
        del res, g, b  # handles go at once: the copies still read the right memory
    env.ctx.sync()
    c = [cpu.ct(a, env.scale) for a in ins]
    want = [cpu.rescale(cpu.mul(c[0], c[1])), cpu.rotate(c[2], 1), cpu.rescale(cpu.mul_plain(c[3], pt, env.scale))]
    for w, h, what in zip(want, outs_host, ("mul", "rotate", "mul_plain")):
        assert_same(h.numpy().view(np.uint64), w.data(), what)


def test_freed_handles_are_not_overwritten_early(env):
    """A result downloaded and dropped at once, then much more work allocating and writing
    device memory: the host copy still holds the result."""
    ckg, P, gpu = env.ckg, env.P, env.gpu
    L = P.max_level
    a = random_ct(P, 5, L)
    host = _empty_pinned((2, L + 1, P.n))
    ga = gpu.upload_ct(a, env.scale)
    r = gpu.rotate(ga, 2)
    want = gpu.download_ct(r)[0]
    gpu.download_ct_overlap(r, host.data_ptr())
    del r
    junk = [gpu.rotate(gpu.upload_ct(random_ct(P, 100 + i, L), env.scale), 1) for i in range(8)]
    env.ctx.join_transfers()
    env.ctx.sync()
    assert_same(host.numpy().view(np.uint64), want, "overlapped download")
    assert len(junk) == 8
    with pytest.raises(ckg.InvalidParams):
        gpu.upload_ct_overlap(0, 2, L, env.scale)
    with pytest.raises(ckg.InvalidParams):
        gpu.upload_ct_overlap(host.data_ptr(), 1, L, env.scale)


def test_overlapped_lists_match_oracle(env):
    """The list forms (one call per list, one shared allocation): uneven levels, the same
    results as the oracle, every entry checked before anything is queued."""
    ckg, P, gpu, cpu = env.ckg, env.P, env.gpu, env.cpu
    L = P.max_level
    levels = [L, L - 1, L, 1]
    ins = [random_ct(P, 30 + i, lv) for i, lv in enumerate(levels)]
    pts = [P.random_q(60 + i, lv) for i, lv in enumerate(levels)]
    host_in = [_pinned(a) for a in ins]
    host_pt = [_pinned(p) for p in pts]
    outs_host = [_empty_pinned((2, lv, P.n)) for lv in levels]
    for step in range(2):
        g = gpu.upload_ct_overlap_list([(h.data_ptr(), 2, lv, env.scale) for h, lv in zip(host_in, levels)])
        gp = gpu.upload_pt_overlap_list([(h.data_ptr(), lv, env.scale) for h, lv in zip(host_pt, levels)])
        b = ckg.Batch(gpu)
        res = [b.mul_plain_rescale(c, p) for c, p in zip(g, gp)]
        b.run()
        gpu.download_ct_overlap_list(res, [h.data_ptr() for h in outs_host])
        del res, g, gp, b
    env.ctx.join_transfers()
    env.ctx.sync()
    for i, (a, p) in enumerate(zip(ins, pts)):
        w = cpu.rescale(cpu.mul_plain(cpu.ct(a, env.scale), p, env.scale))
        assert_same(outs_host[i].numpy().view(np.uint64), w.data(), f"list entry {i}")
    # adjacent host buffers (one pinned allocation, list order): one copy per run, same words
    torch = torch_dev()
    flat_in = torch.from_numpy(np.concatenate([np.ascontiguousarray(a, np.uint64).ravel() for a in ins])
                               .view(np.int64)).pin_memory()
    offs = np.cumsum([0] + [a.size for a in ins])
    g = gpu.upload_ct_overlap_list([(flat_in.data_ptr() + 8 * int(offs[i]), 2, lv, env.scale)
                                    for i, lv in enumerate(levels)])
    flat_out = _empty_pinned((int(offs[-1]),))
    gpu.download_ct_overlap_list(g, [flat_out.data_ptr() + 8 * int(offs[i]) for i in range(len(levels))])
    del g
    env.ctx.join_transfers()
    env.ctx.sync()
    assert np.array_equal(flat_out.numpy(), flat_in.numpy()), "contiguous list round trip"
    with pytest.raises(ckg.InvalidParams):  # a bad entry late in the list: nothing is made
        gpu.upload_ct_overlap_list([(host_in[0].data_ptr(), 2, L, env.scale), (0, 2, L, env.scale)])
    with pytest.raises(ckg.InvalidParams):
        gpu.upload_pt_overlap_list([(host_pt[0].data_ptr(), L + 1, env.scale)])
    assert gpu.upload_ct_overlap_list([]) == []


def test_pinned_buffer_round_trip(env):
    """Host buffers from the library's own pinned allocation (ckg_host_alloc) carry a list
    round trip like any pinned memory."""
    ckg, P, gpu = env.ckg, env.P, env.gpu
    L = P.max_level
    ins = [random_ct(P, 70 + i, L) for i in range(3)]
    words = ins[0].size
    buf_in, buf_out = ckg.PinnedBuffer(8 * words * 3), ckg.PinnedBuffer(8 * words * 3)
    a_in = buf_in.array(np.uint64, (3,) + ins[0].shape)
    for i, a in enumerate(ins):
        a_in[i] = a
    g = gpu.upload_ct_overlap_list([(buf_in.ptr + 8 * words * i, 2, L, env.scale) for i in range(3)])
    gpu.download_ct_overlap_list(g, [buf_out.ptr + 8 * words * i for i in range(3)])
    del g
    env.ctx.join_transfers()
    env.ctx.sync()
    assert np.array_equal(buf_out.array(np.uint64, a_in.shape), a_in)
    with pytest.raises(ckg.InvalidParams):
        buf_in.array(np.uint64, (4,) + ins[0].shape)


def test_pipelined_steps_reuse_blocks_safely(env):
    """Six steps queued back to back with no host wait, each with its own inputs and its own
    host outputs: transfer blocks come back to the cache while the device still reads or copies
    them, and a block handed out again (completed, or still in use behind a device-side wait)
    never lets a later step's upload or pack overwrite an earlier step's data early."""
    ckg, P, gpu, cpu = env.ckg, env.P, env.gpu, env.cpu
    L = P.max_level
    steps = 6
    ins = [[random_ct(P, 100 + 4 * s + i, L) for i in range(4)] for s in range(steps)]
    host_in = [[_pinned(a) for a in step] for step in ins]
    outs_host = [[_empty_pinned((2, L, P.n)) for _ in range(2)] for _ in range(steps)]
    before = env.ctx.transfer_stats()
    for s in range(steps):
        g = gpu.upload_ct_overlap_list([(h.data_ptr(), 2, L, env.scale) for h in host_in[s]])
        b = ckg.Batch(gpu)
        res = [b.mul_relin_rescale(g[0], g[1]), b.mul_relin_rescale(g[2], g[3])]
        b.run()
        gpu.download_ct_overlap_list(res, [h.data_ptr() for h in outs_host[s]])
        del res, g, b
    env.ctx.join_transfers()
    env.ctx.sync()
    after = env.ctx.transfer_stats()
    assert after["upload_calls"] - before["upload_calls"] == steps
    for s in range(steps):
        c = [cpu.ct(a, env.scale) for a in ins[s]]
        for k in range(2):
            w = cpu.rescale(cpu.mul(c[2 * k], c[2 * k + 1]))
            assert_same(outs_host[s][k].numpy().view(np.uint64), w.data(), f"step {s} result {k}")
