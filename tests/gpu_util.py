"""Shared helpers of the GPU parity tests: parameter sets, device buffers (torch is only
used as device memory) and oracle-side key/ciphertext generation.

The parameter sets follow the reference's tests: ``small`` is the N = 2^12, 6 + 2 prime,
dnum 3 set of crates/ckks-train-ckks/src/keys.rs:742-746 (alpha > 1, k > 1, clipped
digits), ``tiny`` the N = 2^5 band layout of params.rs:203-209 (one prime per digit),
``cfg1`` the N = 2^13 small-ring configuration and ``cfg2`` the N = 2^16, 24 x 50-bit +
8 x 60-bit, dnum 3 configuration of the benchmark.
"""

import numpy as np

PARAM_SETS = {
    "tiny": dict(log_n=5, q_bits=[54, 42, 34, 34, 34, 34, 58, 58, 56, 56, 56, 56], p_bits=[60], scale_bits=42, dnum=12),
    "small": dict(log_n=12, q_bits=[60, 40, 40, 40, 40, 40], p_bits=[60, 60], scale_bits=40, dnum=3),
    "cfg1": dict(log_n=13, q_bits=[45] * 4, p_bits=[60], scale_bits=45, dnum=4),
    "n14": dict(log_n=14, q_bits=[50] * 6, p_bits=[60] * 3, scale_bits=50, dnum=2),
    "n15": dict(log_n=15, q_bits=[60] + [40] * 9, p_bits=[60], scale_bits=40, dnum=10),
    "cfg2": dict(log_n=16, q_bits=[50] * 24, p_bits=[60] * 8, scale_bits=50, dnum=3),
}


def torch_dev():
    import torch
    assert torch.cuda.is_available(), "GPU test without a GPU"
    return torch


def to_dev(arr):
    torch = torch_dev()
    a = np.ascontiguousarray(arr, np.uint64)
    t = torch.from_numpy(a.view(np.int64).copy()).cuda()
    torch.cuda.synchronize()
    return t


def empty_dev(shape):
    """Uninitialised device buffer (no fill kernel that could race with the library's stream)."""
    torch = torch_dev()
    t = torch.empty(tuple(shape), dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    return t


def from_dev(t):
    torch = torch_dev()
    torch.cuda.synchronize()
    return t.cpu().numpy().view(np.uint64)


def ptr(t):
    return t.data_ptr()


def make_pair(ckg, O, name):
    """(oracle Params, product Context) for one parameter set, with identical primes."""
    ps = PARAM_SETS[name]
    P = O.Params.from_bits(ps["log_n"], ps["q_bits"], ps["p_bits"], ps["scale_bits"], ps["dnum"])
    ctx = ckg.Context(ps["log_n"], P.q, P.p, ps["dnum"], scale=float(2.0 ** ps["scale_bits"]))
    return P, ctx


def random_ct(P, seed, level, ncomp=2):
    return np.stack([P.random_q(seed * 7919 + c, level) for c in range(ncomp)])


def assert_same(got, want, what):
    got = np.asarray(got, np.uint64)
    want = np.asarray(want, np.uint64)
    assert got.shape == want.shape, f"{what}: shape {got.shape} != {want.shape}"
    if not np.array_equal(got, want):
        idx = np.argwhere(got != want)[0]
        raise AssertionError(f"{what}: first mismatch at {tuple(idx)}: got {got[tuple(idx)]}, "
                             f"oracle {want[tuple(idx)]} ({int((got != want).sum())} words differ)")


def near_tie_residue(r, c):
    """Residue modulo r of a coefficient whose centered-conversion input [X + h]_D sits next
    to 0 or D (crates/ckks-train-cuda/tests/cases/mod.rs:277-290): m = c/2 + 1 for even c,
    D - m for odd c, shifted by -h."""
    m = c // 2 + 1
    s = m % r if c % 2 == 0 else (r - m % r) % r
    return (s + r - (r >> 1)) % r


def near_tie_limbs(primes, n):
    out = np.zeros((len(primes), n), np.uint64)
    for i, r in enumerate(primes):
        out[i] = [near_tie_residue(r, c) for c in range(n)]
    return out
