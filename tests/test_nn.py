"""The encrypted training step's host logic, no GPU (crates/ckks-train-nn):

* the slot layout and weight packing against their defining identities in plaintext, as the
  reference's layout and sim tests state them (layout.rs, sim.rs): the BSGS mat-vec over the
  packed diagonals plus the fold is W x, the rotation-only transpose gives exactly the packed
  W^T, unpacking inverts packing;
* the rotation key sets and the step's op counts (the per-op costs of dense.rs / trainer.rs);
* one full training step on the oracle's CPU evaluator through ckks_train_b200.nn: the trace of
  levels (9 levels for two Square layers, trainer.rs module docs), the counter against the cost
  formula, and the decrypted updated weights and biases against the plaintext SGD step.
"""

import numpy as np
import pytest

from nn_backends import Client, OracleHeOps, plain_step

MINI = dict(log_n=11, q_bits=[58] + [42] * 11, p_bits=[58, 58], scale_bits=42, dnum=6)


def _rot(v, k):
    """sim_rotate: out[i] = v[(i + k) mod n] (crates/ckks-train-nn/src/sim.rs:68-78)."""
    return np.roll(v, -k)


def _sim_matvec(diags, x, layout, nn):
    """sim_matvec (sim.rs:138-175): hoisted baby rotations of x, giant rotations of the sums."""
    baby, giant = nn.bsgs_split(len(diags))
    s = layout.batch
    xs = [_rot(x, k2 * s) for k2 in range(baby)]
    acc = np.zeros(layout.slots)
    for k1 in range(giant):
        inner = sum(diags[k1 * baby + k2] * xs[k2] for k2 in range(baby))
        acc = acc + _rot(inner, baby * k1 * s)
    return acc


SHAPES = [(8, 8), (8, 12), (3, 8), (12, 4), (16, 3), (1, 5), (7, 1)]


@pytest.mark.parametrize("d_out,d_in", SHAPES)
def test_pack_matvec_transpose(ckg, d_out, d_in):
    nn = ckg.nn
    layout = nn.Layout(512, 16, 8)
    rng = np.random.default_rng(d_out * 100 + d_in)
    w = rng.uniform(-1, 1, (d_out, d_in))
    x = rng.uniform(-1, 1, (layout.batch, d_in))
    diags = nn.pack_weight_diagonals(w, layout)
    sh = nn.LayerShape(d_out, d_in, layout)
    assert len(diags) == sh.m
    assert np.array_equal(nn.unpack_weight_diagonals(diags, d_out, d_in, layout, 3), w)
    # forward: matvec + fold is W x_b in canonical form with period n_out
    y = _sim_matvec(diags, nn.pack_activations(x, layout), layout, nn)
    for t in range(sh.fold_steps()):
        y = y + _rot(y, sh.n_out * (1 << t) * layout.batch)
    want = x @ w.T
    got = nn.unpack_activations(y, layout, d_out)
    assert np.allclose(got, want, atol=1e-12)
    # the rotation-only transpose is exactly the packed W^T (layout.rs:343-365)
    wt = [_rot(diags[c], a) for c, a in zip(nn.transpose_sources(d_out, d_in, layout),
                                            nn.rotations_for_transpose(d_out, d_in, layout))]
    assert all(np.array_equal(a, b) for a, b in zip(wt, nn.pack_weight_diagonals(w.T, layout)))
    assert sum(1 for a in nn.rotations_for_transpose(d_out, d_in, layout) if a != 0) == sh.m - 1


def test_layout_errors_and_steps(ckg):
    nn = ckg.nn
    with pytest.raises(ckg.InvalidParams):
        nn.Layout(512, 12, 8)
    with pytest.raises(ckg.InvalidParams):
        nn.Layout(512, 64, 16)
    L = nn.Layout(1 << 15, 256, 64)
    # config 4 (196 -> 64 -> 10, B = 64): layer splits 8 x 8 and 4 x 4 (linalg.rs:419-424)
    assert (nn.LayerShape(64, 196, L).baby, nn.LayerShape(64, 196, L).giant) == (8, 8)
    assert (nn.LayerShape(10, 64, L).baby, nn.LayerShape(10, 64, L).giant) == (4, 4)
    assert nn.forward_rotation_steps(64, 196, L) == sorted(
        [k * 64 for k in range(1, 8)] + [8 * k * 64 for k in range(1, 8)] + [64 * 64, 128 * 64])
    assert nn.bias_grad_rotation_steps(L) == [-32, -16, -8, -4, -2, -1, 1, 2, 4, 8, 16, 32]
    assert nn.grad_reduced_rotation_steps(10, 64, L) == sorted(
        [64, 128, 192, -256, -512, -768, 1, 2, 4, 8, 16, 32])
    c = nn.step_counts([196, 64, 10], L)
    assert c["rotations"] == 1049 and c["relins"] == 100


@pytest.fixture(scope="module")
def mini(ckg, oracle):
    """N = 2^11 with the n16_train band shape in miniature (58 + 11 x 42-bit q, 2 x 58-bit p,
    scale 2^42, dnum 6), a 12 -> 8 -> 3 Square MLP in Layout(1024, 16, 8), all keys."""
    nn, O = ckg.nn, oracle
    P = O.Params.from_bits(MINI["log_n"], MINI["q_bits"], MINI["p_bits"], MINI["scale_bits"], MINI["dnum"])
    layout = nn.Layout(P.n // 2, 16, 8)
    dims = [12, 8, 3]
    kg = O.KeyGenerator(P, 5)
    steps = nn.mlp_rotation_steps(dims, layout)
    elts = sorted({O.galois_elt(P.n, s) for s in steps} - {1})
    rk, gk = kg.relin_key(), {e: kg.galois_key(e) for e in elts}
    return dict(P=P, layout=layout, dims=dims, kg=kg, rk=rk, gk=gk, steps=steps)


def make_problem(nn, dims, layout, seed, batch=None):
    rng = np.random.default_rng(seed)
    batch = layout.batch if batch is None else batch
    ws = [rng.uniform(-0.1, 0.1, (dims[i + 1], dims[i])) for i in range(len(dims) - 1)]
    bs = [rng.uniform(-0.1, 0.1, dims[i + 1]) for i in range(len(dims) - 1)]
    x = rng.uniform(0, 1, (batch, dims[0]))
    y = rng.uniform(0, 1, (batch, dims[-1]))
    return ws, bs, x, y


def encrypt_network(nn, client, ev_ct, ev, layout, dims, ws, bs, x, y, level, delta, upload):
    """Client-side encryption (Mlp::encrypt_at, BatchSpec::encrypt): weights at delta, biases at
    the product scale, x at (level, delta), y at the output's exact (level, scale)."""
    per_layer, (y_level, y_scale) = nn.Mlp.scales(ev, dims, level, delta)
    layers = []
    for (w, b), (_, x_scale, b_scale) in zip(zip(ws, bs), per_layer):
        entries = [upload(client.encrypt(ev_ct, v, delta, level)) for v in nn.pack_weight_diagonals(w, layout)]
        bias = upload(client.encrypt(ev_ct, nn.pack_bias(b, layout), b_scale, level))
        layers.append((nn.Dense(nn.EncWeights(entries, w.shape[0], w.shape[1], layout), bias), nn.Square()))
    xc = upload(client.encrypt(ev_ct, nn.pack_activations(x, layout), delta, level))
    yc = upload(client.encrypt(ev_ct, nn.pack_activations(y, layout), y_scale, y_level))
    return nn.Mlp(layers), xc, yc


def test_oracle_training_step(ckg, oracle, mini):
    """One step on the CPU evaluator: levels, counts, and the decrypted update."""
    nn, O = ckg.nn, oracle
    P, layout, dims = mini["P"], mini["layout"], mini["dims"]
    ev = OracleHeOps(P, mini["rk"], mini["gk"])
    client = Client(P, mini["kg"])
    ws, bs, x, y = make_problem(nn, dims, layout, 11)
    top, delta = P.max_level, float(2.0 ** MINI["scale_bits"])
    mlp, xc, yc = encrypt_network(nn, client, ev.ev, ev, layout, dims, ws, bs, x, y, top, delta,
                                  lambda c: ev._w(c))
    lr = 0.5
    tr = nn.Trainer(ev, layout, [nn.Sgd(lr) for _ in dims[1:]])
    tr.train_batch(mlp, xc, yc)
    levels = dict(tr.trace)
    assert levels["z1"] == top - 1 and levels["a2"] == top - 4
    assert levels["W1'"] == top - 9, tr.trace  # the 9 levels of two Square layers
    assert ev.counter() == dict(nn.step_counts(dims, layout), sse_switches=0, bootstraps=0)
    new_w, new_b, _, _ = plain_step(ws, bs, x, y, lr)
    for i, (dense, _) in enumerate(mlp.layers):
        w = dense.w
        vals = [client.decrypt(e.ct.data(), e.level(), e.scale()) for e in w.entries]
        got = nn.unpack_weight_diagonals(vals, w.d_out, w.d_in, layout, 0)
        assert np.abs(got - new_w[i]).max() < 1e-6, f"W{i + 1}"
        bv = client.decrypt(dense.b.ct.data(), dense.b.level(), dense.b.scale())
        assert np.abs(nn.unpack_activations(bv, layout, w.d_out)[0] - new_b[i]).max() < 1e-6, f"b{i + 1}"
        assert dense.b.scale() == mlp.layers[i][0].b.scale()


def test_oracle_partial_batch_and_errors(ckg, oracle, mini):
    """n_valid < batch masks the padded lanes out of the gradients; errors come before work."""
    nn = ckg.nn
    P, layout, dims = mini["P"], mini["layout"], mini["dims"]
    ev = OracleHeOps(P, mini["rk"], mini["gk"])
    client = Client(P, mini["kg"], seed=50)
    ws, bs, x, y = make_problem(nn, dims, layout, 12)
    top, delta = P.max_level, float(2.0 ** MINI["scale_bits"])
    mlp, xc, yc = encrypt_network(nn, client, ev.ev, ev, layout, dims, ws, bs, x, y, top, delta,
                                  lambda c: ev._w(c))
    tr = nn.Trainer(ev, layout, [nn.Sgd(0.25) for _ in dims[1:]])
    with pytest.raises(ckg.InvalidParams):
        tr.train_batch_valid(mlp, xc, yc, 0)
    with pytest.raises(ckg.InvalidParams):
        nn.Trainer(ev, layout, [nn.Sgd(0.25)]).train_batch(mlp, xc, yc)
    dense = mlp.layers[0][0]
    bad = nn.Dense(dense.w, ev.mod_switch_to_level(dense.b, top))
    bad.b = ev._w(ev.ev.relabel(dense.b.ct, dense.b.scale() * 2))
    with pytest.raises(ckg.ScaleMismatch):
        bad.forward(ev, xc, layout)
    no_keys = OracleHeOps(P, mini["rk"], {})
    with pytest.raises(ckg.InvalidParams):
        dense.forward(no_keys, xc, layout)
    assert ev.counter()["rotations"] == 0 and no_keys.counter()["rotations"] == 0
    tr.train_batch_valid(mlp, xc, yc, 5)
    new_w, new_b, _, _ = plain_step(ws, bs, x, y, 0.25, n_valid=5)
    w = mlp.layers[1][0].w
    vals = [client.decrypt(e.ct.data(), e.level(), e.scale()) for e in w.entries]
    assert np.abs(nn.unpack_weight_diagonals(vals, w.d_out, w.d_in, layout, 0) - new_w[1]).max() < 1e-6
