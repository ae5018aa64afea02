"""The encrypted MLP training step on the GPU (crates/ckks-train-nn through HeOps):

* ct-for-ct parity with the same step on the oracle's CPU evaluator (every forward value,
  delta, derivative factor, dz, transposed weight, backward delta, weight and bias gradient,
  and the updated network), with equal counters and level traces, on the N = 2^11 miniature
  of n16_train;
* config 4 at full size: N = 2^16 n16_train (58 + 31 x 42-bit q, 4 x 58-bit p, dnum 8, scale
  2^42), Layout(2^15, 256, 64), 196 -> 64 -> 10 with Square, B = 64: ct-for-ct against the
  oracle's run of the same step (digests of every ciphertext), the counter against the cost
  formula, and the decrypted update against the plaintext SGD step.
"""

import numpy as np
import pytest

from gpu_util import assert_same
from nn_backends import Client, OracleHeOps, ct_digest, deterministic_keys, plain_step, step_values
from test_nn import MINI, encrypt_network, make_problem

pytestmark = pytest.mark.gpu

N16_TRAIN = dict(log_n=16, q_bits=[58] + [42] * 31, p_bits=[58] * 4, scale_bits=42, dnum=8)


def _gpu_env(ckg, P, ps, rk, gk, ctx=None):
    ctx = ctx or ckg.Context(ps["log_n"], P.q, P.p, ps["dnum"], scale=float(2.0 ** ps["scale_bits"]))
    d_rk = ctx.upload_key(rk.export())
    d_gk = [ctx.upload_key(k.export(), e) for e, k in gk.items()]
    return ctx, ckg.CudaEvaluator(ctx, d_rk, d_gk)


def _check(gpu, cpu_ct, gpu_ct, what):
    got, scale = gpu.download_ct(gpu_ct)
    assert gpu_ct.level() == cpu_ct.level(), f"{what}: level"
    assert scale == cpu_ct.scale(), f"{what}: scale"
    assert_same(got, cpu_ct.ct.data(), what)


def test_training_step_parity(ckg, oracle):
    nn, O = ckg.nn, oracle
    P = O.Params.from_bits(MINI["log_n"], MINI["q_bits"], MINI["p_bits"], MINI["scale_bits"], MINI["dnum"])
    layout, dims = nn.Layout(P.n // 2, 16, 8), [12, 8, 3]
    kg, rk, gk = deterministic_keys(P, nn.mlp_rotation_steps(dims, layout), 21)
    cpu = OracleHeOps(P, rk, gk)
    _, gpu = _gpu_env(ckg, P, MINI, rk, gk)
    client = Client(P, kg)
    ws, bs, x, y = make_problem(nn, dims, layout, 31)
    top, delta = P.max_level, float(2.0 ** MINI["scale_bits"])
    cts = []  # client ciphertexts, encrypted once and given to both backends
    mlp_c, x_c, y_c = encrypt_network(nn, client, cpu.ev, cpu, layout, dims, ws, bs, x, y, top, delta,
                                      lambda c: (cts.append(c), cpu._w(c))[1])
    it = iter(cts)
    mlp_g, x_g, y_g = encrypt_network(nn, _Replay(it), None, gpu, layout, dims, ws, bs, x, y, top, delta,
                                      lambda c: gpu.upload_ct(c.data(), c.scale))
    lr = 0.5
    rec_c = nn.Trainer(cpu, layout, [nn.Sgd(lr) for _ in dims[1:]])
    rec_g = nn.Trainer(gpu, layout, [nn.Sgd(lr) for _ in dims[1:]])
    vc = rec_c.train_batch(mlp_c, x_c, y_c)
    vg = rec_g.train_batch(mlp_g, x_g, y_g)
    assert rec_c.trace == rec_g.trace
    assert gpu.counter() == cpu.counter() == dict(nn.step_counts(dims, layout), sse_switches=0, bootstraps=0)
    for name in ("z", "a", "delta", "s", "dz", "backward", "db"):
        for i in vc[name]:
            _check(gpu, vc[name][i], vg[name][i], f"{name}{i + 1}")
    for name in ("wt", "dw"):
        for i in vc[name]:
            ec = vc[name][i].entries if name == "wt" else vc[name][i]
            eg = vg[name][i].entries if name == "wt" else vg[name][i]
            for k, (a, b) in enumerate(zip(ec, eg)):
                _check(gpu, a, b, f"{name}{i + 1}[{k}]")
    for i, ((dc, _), (dg, _)) in enumerate(zip(mlp_c.layers, mlp_g.layers)):
        for k, (a, b) in enumerate(zip(dc.w.entries, dg.w.entries)):
            _check(gpu, a, b, f"W{i + 1}'[{k}]")
        _check(gpu, dc.b, dg.b, f"b{i + 1}'")
    # a second step from the updated network, and the errors before work
    x2, y2 = gpu.upload_ct(x_c.ct.data(), x_c.scale()), gpu.upload_ct(y_c.ct.data(), y_c.scale())
    dense = mlp_g.layers[0][0]
    with pytest.raises(ckg.LevelMismatch):
        dense.forward(gpu, x2, layout)  # the updated weights are below the top level
    before = gpu.counter()
    no_keys = ckg.CudaEvaluator(gpu.ctx, None, [])
    with pytest.raises(ckg.InvalidParams):
        mlp_g.layers[1][0].weight_grad_scaled(no_keys, y2, y2, layout, 0.1)
    assert gpu.counter() == before and no_keys.counter()["rotations"] == 0


class _Replay:
    """Hands out the ciphertexts the client encrypted for the CPU run, in the same order."""

    def __init__(self, it):
        self.it = it

    def encrypt(self, ev, values, scale, level):
        c = next(self.it)
        assert c.level == level and c.scale == scale
        return c


def test_config4_ct_for_ct(ckg, oracle):
    """Config 4 at full size: 196 -> 64 -> 10, Square, B = 64 on n16_train, Layout(2^15, 256, 64).
    Every ciphertext of the step (forward values, deltas, derivative factors, dz, transposed
    weights, backward deltas, weight and bias gradients, the updated network) has the digest
    of the oracle's ciphertext on the same seeded keys and inputs (tests/golden/config4_digests.json,
    made by tests/golden/make_config4_digests.py), with its level and scale; the counter and the
    level trace are the oracle's; and the decrypted update is the plaintext SGD step."""
    import json
    import os

    gold_path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "config4_digests.json")
    with open(gold_path) as f:
        gold = json.load(f)
    nn, O = ckg.nn, oracle
    ps = N16_TRAIN
    P = O.Params.from_bits(ps["log_n"], ps["q_bits"], ps["p_bits"], ps["scale_bits"], ps["dnum"])
    layout, dims = nn.Layout(P.n // 2, 256, 64), [196, 64, 10]
    kg, rk, gk = deterministic_keys(P, nn.mlp_rotation_steps(dims, layout), 41)
    ctx, gpu = _gpu_env(ckg, P, ps, rk, gk)
    del gk
    client = Client(P, kg)
    ws, bs, x, y = make_problem(nn, dims, layout, 43)
    top, delta = P.max_level, float(2.0 ** ps["scale_bits"])
    host = O.Evaluator(P)
    mlp, xc, yc = encrypt_network(nn, client, host, gpu, layout, dims, ws, bs, x, y, top, delta,
                                  lambda c: gpu.upload_ct(c.data(), c.scale))
    lr = 0.05
    tr = nn.Trainer(gpu, layout, [nn.Sgd(lr) for _ in dims[1:]])
    v = tr.train_batch(mlp, xc, yc)
    assert dict(tr.trace)["W1'"] == top - 9
    assert [list(t) for t in tr.trace] == gold["trace"]
    assert gpu.counter() == gold["counter"] == dict(nn.step_counts(dims, layout), sse_switches=0, bootstraps=0)
    got = step_values(v, mlp)
    assert [name for name, _ in got] == [g[0] for g in gold["values"]]
    for (name, ct), (_, level, scale, digest) in zip(got, gold["values"]):
        data, sc = gpu.download_ct(ct)
        assert ct.level() == level and sc == scale, f"{name}: level/scale"
        assert ct_digest(data, ct.level(), sc) == digest, f"{name}: words differ from the oracle's"
    new_w, new_b, _, _ = plain_step(ws, bs, x, y, lr)
    for i, (dense, _) in enumerate(mlp.layers):
        w = dense.w
        vals = [client.decrypt(gpu.download_ct(e)[0], e.level(), e.scale()) for e in w.entries]
        got_w = nn.unpack_weight_diagonals(vals, w.d_out, w.d_in, layout, 0)
        err = np.abs(got_w - new_w[i]).max()
        assert err < 1e-5, f"W{i + 1}: {err}"
        bv = client.decrypt(gpu.download_ct(dense.b)[0], dense.b.level(), dense.b.scale())
        assert np.abs(nn.unpack_activations(bv, layout, w.d_out)[0] - new_b[i]).max() < 1e-5, f"b{i + 1}"
