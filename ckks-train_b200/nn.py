"""The encrypted MLP training step of ckks-train-nn, over any evaluator with the HeOps methods.

This is the caller side of the evaluator path: the reference's `ckks-train-nn` layers and
interactive trainer are generic over `E: HeOps` and issue only evaluator ops, so the same op
sequence runs on the device through `CudaEvaluator` (the C ABI) and, in the tests, on a CPU
restatement of the reference evaluator. Every function follows its reference counterpart op for op and check
for check (file:line in each docstring), so both backends see the same ciphertexts:

* slot layout and weight packing (crates/ckks-train-nn/src/layout.rs);
* `Dense::forward`, `fold`, the rotation-only transpose, `Dense::backward_input`, the weight and
  bias gradients, interactive and reduce-only (crates/ckks-train-nn/src/dense.rs);
* the `Square` activation (crates/ckks-train-nn/src/activation.rs), `Mse::grad`
  (crates/ckks-train-nn/src/loss.rs), `Sgd` (crates/ckks-train-nn/src/optim.rs);
* `Trainer::train_batch_valid` with SGD, one micro-batch, without the refresh
  (crates/ckks-train-nn/src/trainer.rs:1014-1366).

Encryption and decryption stay with the client: weights, biases and batches arrive as
ciphertexts; plaintext masks are encoded by the evaluator (`ev.encode`).

The evaluator needs: `params()` (with `q`, `n`), `add`, `sub`, `mul`, `mul_lazy`, `relin_lazy`,
`rescale`, `rotate`, `hoisted_rotate`, `mod_switch_to_level`, `mul_plain`, `mul_plain_to_scale`,
`matvec_enc(d, stride, entries, x)`, `exact_product_scale`, `target_plain_scale`,
`encode(values, scale, level)`, `has_galois_key`, `has_relin_key`, `owns`; ciphertexts need
`level()`, `scale()`, `size()`. Where the reference loops over independent ciphertexts (the m
diagonals of a weight gradient, the transpose's entries), an evaluator that also offers
`rotate_many` / `mul_rescale_many` (CudaEvaluator: one batched launch sequence) gets each round
at once; every ciphertext still sees its reference op sequence, so results and counts are the same.
"""

import math

import numpy as np

from .heops import InvalidParams, LevelMismatch, NoLevelsLeft, ScaleMismatch

# ---------------------------------------------------------------------------------------------
# Layout (crates/ckks-train-nn/src/layout.rs)
# ---------------------------------------------------------------------------------------------


def _pow2(x):
    return x > 0 and (x & (x - 1)) == 0


def _next_pow2(x):
    return 1 << (x - 1).bit_length()


def bsgs_split(d):
    """(baby, giant) = (2^ceil(log2(d) / 2), d / baby) (crates/ckks-train-ckks/src/linalg.rs:419-424)."""
    assert _pow2(d), f"d = {d} must be a power of two"
    baby = 1 << ((d.bit_length() - 1 + 1) // 2)
    return baby, d // baby


def bsgs_rotation_steps(d, stride):
    """Baby steps k2 stride (k2 < baby), then giant steps baby k1 stride (linalg.rs:426-435)."""
    baby, giant = bsgs_split(d)
    return [k2 * stride for k2 in range(1, baby)] + [baby * k1 * stride for k1 in range(1, giant)]


class Layout:
    """`slot(j, b) = j * batch + b` for feature j < d and lane b < batch (layout.rs:50-100)."""

    def __init__(self, slots, d, batch):
        if not (_pow2(d) and _pow2(batch) and slots > 0 and slots % (d * batch) == 0):
            raise InvalidParams(f"layout needs powers of two d = {d}, batch = {batch} with d * batch dividing "
                                f"slots = {slots}")
        self.slots, self.d, self.batch = slots, d, batch

    def slot(self, j, b):
        return j * self.batch + b

    def block(self):
        return self.d * self.batch

    def features(self):
        return self.slots // self.batch

    def log_batch(self):
        return self.batch.bit_length() - 1

    def __eq__(self, o):
        return isinstance(o, Layout) and (self.slots, self.d, self.batch) == (o.slots, o.d, o.batch)

    def __repr__(self):
        return f"Layout(slots={self.slots}, d={self.d}, batch={self.batch})"


class LayerShape:
    """Geometry of a d_out x d_in layer: padded sizes, l = max, m = min, BSGS split of m
    (layout.rs:102-175)."""

    def __init__(self, d_out, d_in, layout):
        assert d_out > 0 and d_in > 0, "layer dimensions must be positive"
        n_out, n_in = _next_pow2(d_out), _next_pow2(d_in)
        assert n_out <= layout.d and n_in <= layout.d, \
            f"layer {d_out} x {d_in} (padded {n_out} x {n_in}) exceeds layout d = {layout.d}"
        self.d_out, self.d_in, self.n_out, self.n_in = d_out, d_in, n_out, n_in
        self.l, self.m = max(n_out, n_in), min(n_out, n_in)
        self.baby, self.giant = bsgs_split(self.m)

    def fold_steps(self):
        """log2(n_in / n_out) for a wide layer, else 0 (layout.rs:166-172)."""
        return (self.n_in // self.n_out).bit_length() - 1 if self.n_in > self.n_out else 0


def checked_shape(d_out, d_in, layout):
    """LayerShape, as InvalidParams instead of a panic (dense.rs:64-76)."""
    fits = lambda n: n > 0 and _next_pow2(n) <= layout.d
    if not (fits(d_out) and fits(d_in)):
        raise InvalidParams(f"layer {d_out} x {d_in} does not fit layout d = {layout.d}")
    return LayerShape(d_out, d_in, layout)


def _check_slots(layout, ev):
    """dense.rs:78-87."""
    slots = ev.params().n // 2
    if layout.slots != slots:
        raise InvalidParams(f"layout of {layout.slots} slots for parameters with {slots} slots")


def pack_activations(x, layout):
    """Canonical form: slot j batch + b holds x[b][j mod n_in], 0 for padded features and unused
    lanes (layout.rs:177-199). `x` is rows x d_in, rows <= batch."""
    x = np.asarray(x, np.float64)
    rows, cols = x.shape
    assert rows <= layout.batch, f"{rows} samples exceed batch {layout.batch}"
    n = _next_pow2(cols)
    assert cols > 0 and n <= layout.d, f"dimension {cols} exceeds d = {layout.d}"
    s = np.arange(layout.slots)
    j, b = (s // layout.batch) % n, s % layout.batch
    ok = (b < rows) & (j < cols)
    out = np.zeros(layout.slots)
    out[ok] = x[b[ok], j[ok]]
    return out


def pack_bias(bias, layout):
    """A per-feature vector in canonical form, the same in every lane (layout.rs:204-207)."""
    bias = np.asarray(bias, np.float64)
    return pack_activations(np.tile(bias, (layout.batch, 1)), layout)


def unpack_activations(v, layout, d_valid):
    """batch x d_valid from slot j batch + b (layout.rs:209-226)."""
    v = np.asarray(v)
    assert len(v) == layout.slots and d_valid <= layout.d
    b, j = np.meshgrid(np.arange(layout.batch), np.arange(d_valid), indexing="ij")
    return v[j * layout.batch + b]


def _padded(w, r, c):
    out = np.zeros(r.shape)
    ok = (r < w.shape[0]) & (c < w.shape[1])
    out[ok] = w[r[ok], c[ok]]
    return out


def pack_weight_diagonals(w, layout):
    """The m generalised diagonals of w (d_out x d_in), BSGS order, pre-rotated and replicated:
    entries[k1 baby + k2][j batch + b] = D_c[j - g k1], c = g k1 + k2, g = baby,
    D_c[j] = W~[j mod n_out][(j + c) mod n_in] (layout.rs:228-264)."""
    w = np.asarray(w, np.float64)
    sh = LayerShape(w.shape[0], w.shape[1], layout)
    f = layout.features()
    s = np.arange(layout.slots)
    out = []
    for c in range(sh.m):
        shift = sh.baby * (c // sh.baby)
        j = (s // layout.batch + f - shift) % f
        out.append(_padded(w, j % sh.n_out, (j + c) % sh.n_in))
    return out


def unpack_weight_diagonals(diags, d_out, d_in, layout, lane=0):
    """Inverse of pack_weight_diagonals, reading lane `lane` (layout.rs:266-298)."""
    sh = LayerShape(d_out, d_in, layout)
    assert len(diags) == sh.m and lane < layout.batch
    f = layout.features()
    w = np.zeros((sh.n_out, sh.n_in))
    j = np.arange(sh.l)
    for c, v in enumerate(diags):
        v = np.asarray(v)
        shift = sh.baby * (c // sh.baby)
        w[j % sh.n_out, (j + c) % sh.n_in] = v[((j + shift) % f) * layout.batch + lane]
    return w[:d_out, :d_in]


def transpose_sources(d_out, d_in, layout):
    """Entry c(i) of W that output entry i of W^T is rotated from (layout.rs:300-306)."""
    m = LayerShape(d_out, d_in, layout).m
    return [(m - i % m) % m for i in range(m)]


def rotations_for_transpose(d_out, d_in, layout):
    """a_i batch, a_i = (t - g floor(i/g) + g floor(c/g)) mod l, t = -c (wide or square) or i (tall)
    (layout.rs:308-328)."""
    sh = LayerShape(d_out, d_in, layout)
    g, l = sh.baby, sh.l
    out = []
    for i, c in enumerate(transpose_sources(d_out, d_in, layout)):
        t = -c if sh.n_in >= sh.n_out else i
        out.append(((t - g * (i // g) + g * (c // g)) % l) * layout.batch)
    return out


def valid_lane_mask(layout, n_valid):
    """1 on lanes below n_valid, 0 elsewhere (crates/ckks-train-nn/src/sim.rs:266-275)."""
    assert n_valid <= layout.batch, f"n_valid {n_valid} > batch {layout.batch}"
    return np.where(np.arange(layout.slots) % layout.batch < n_valid, 1.0, 0.0)


# ---------------------------------------------------------------------------------------------
# Rotation steps (dense.rs)
# ---------------------------------------------------------------------------------------------


def _fold_rotation_steps(sh, layout):
    """n_out 2^t batch for t < fold_steps (dense.rs:89-94)."""
    return [sh.n_out * (1 << t) * layout.batch for t in range(sh.fold_steps())]


def forward_rotation_steps(d_out, d_in, layout):
    """The matvec's BSGS steps and the fold steps, sorted and distinct (dense.rs:96-113)."""
    sh = LayerShape(d_out, d_in, layout)
    return sorted(set(bsgs_rotation_steps(sh.m, layout.batch) + _fold_rotation_steps(sh, layout)))


def backward_rotation_steps(d_out, d_in, layout):
    """The forward steps of W^T (dense.rs:533-541)."""
    return forward_rotation_steps(d_in, d_out, layout)


def transpose_rotation_steps(d_out, d_in, layout):
    """The distinct nonzero transpose rotations (dense.rs:645-668, layout.rs:330-341)."""
    return sorted({s for s in rotations_for_transpose(d_out, d_in, layout) if s != 0})


def _lane_steps(layout):
    """Reduce 2^t and replicate -2^t, t < log2(batch) (dense.rs:862-868)."""
    reduce = [1 << t for t in range(layout.log_batch())]
    return reduce, [-s for s in reduce]


def bias_grad_rotation_steps(layout):
    """dense.rs:870-877."""
    reduce, rep = _lane_steps(layout)
    return sorted(reduce + rep)


def grad_rotation_steps(d_out, d_in, layout):
    """Baby k2 batch, giant -g k1 batch and the bias steps (dense.rs:879-895)."""
    sh = LayerShape(d_out, d_in, layout)
    b = layout.batch
    steps = [k2 * b for k2 in range(1, sh.baby)] + [-(sh.baby * k1 * b) for k1 in range(1, sh.giant)]
    return sorted(set(steps + bias_grad_rotation_steps(layout)))


def grad_reduced_rotation_steps(d_out, d_in, layout):
    """Baby, giant and batch-reduce steps, no replication (dense.rs:1141-1160)."""
    sh = LayerShape(d_out, d_in, layout)
    b = layout.batch
    steps = [k2 * b for k2 in range(1, sh.baby)] + [-(sh.baby * k1 * b) for k1 in range(1, sh.giant)]
    return sorted(set(steps + _lane_steps(layout)[0]))


def mlp_rotation_steps(dims, layout):
    """The key set of one training step of an MLP with layer widths `dims`: forward and gradient
    steps of every layer, backward and transpose steps of every layer but the first
    (crates/ckks-train-nn/src/trainer.rs module docs, "Galois keys")."""
    steps = set()
    for i in range(len(dims) - 1):
        d_in, d_out = dims[i], dims[i + 1]
        steps |= set(forward_rotation_steps(d_out, d_in, layout))
        steps |= set(grad_rotation_steps(d_out, d_in, layout))
        if i > 0:
            steps |= set(backward_rotation_steps(d_out, d_in, layout))
            steps |= set(transpose_rotation_steps(d_out, d_in, layout))
    return sorted(steps)


def _check_keys(ev, steps):
    """InvalidParams("missing galois key") unless every step has a key (dense.rs:136-145)."""
    for s in steps:
        if not ev.has_galois_key(s):
            raise InvalidParams(f"missing galois key for step {s}")


def _check_input(ev, ct):
    """A 2-component ciphertext over the evaluator's basis (dense.rs:844-860)."""
    if not ev.owns(ct) or ct.size() != 2:
        raise InvalidParams("gradient inputs must be 2-component ciphertexts over the evaluator's basis")


# ---------------------------------------------------------------------------------------------
# Weights and the dense layer (dense.rs)
# ---------------------------------------------------------------------------------------------


def _check_uniform(entries):
    """LevelMismatch / ScaleMismatch unless all entries share one level and one scale (dense.rs:812-824)."""
    l0, s0 = entries[0].level(), entries[0].scale()
    for e in entries:
        if e.level() != l0:
            raise LevelMismatch("diagonals at different levels")
        if e.scale() != s0:
            raise ScaleMismatch("diagonals at different scales")


class EncWeights:
    """The encrypted pre-rotated diagonals of a d_out x d_in layer, d = m, stride = batch
    (dense.rs:180-361): `EncWeights::from_diagonals`."""

    def __init__(self, entries, d_out, d_in, layout):
        sh = checked_shape(d_out, d_in, layout)
        entries = list(entries)
        if len(entries) != sh.m:
            raise InvalidParams(f"{len(entries)} diagonals for a {d_out} x {d_in} layer need d = {sh.m}")
        _check_uniform(entries)
        self.entries, self.d_out, self.d_in, self.stride = entries, d_out, d_in, layout.batch

    @staticmethod
    def pack(w, layout):
        """The slot vectors the client encrypts (pack_weight_diagonals)."""
        return pack_weight_diagonals(w, layout)

    def level(self):
        return self.entries[0].level()

    def scale(self):
        return self.entries[0].scale()

    def product_scale(self, x_scale):
        return x_scale * self.scale()

    def shape(self, layout):
        return checked_shape(self.d_out, self.d_in, layout)

    def check_batch(self, layout):
        if self.stride != layout.batch:
            raise InvalidParams(f"weights packed for batch {self.stride}, layout batch {layout.batch}")

    def mod_switch_to_level(self, ev, level):
        """Diagonals::mod_switch_to_level (crates/ckks-train-ckks/src/linalg.rs:406-412)."""
        return [ev.mod_switch_to_level(e, level) for e in self.entries]

    def transpose(self, ev, layout):
        """W^T (d_in x d_out) by rotations only, TransposeKeys::Dedicated: entry i is entry
        transpose_sources[i] rotated by rotations_for_transpose[i] (dense.rs:672-757)."""
        self.shape(layout)
        _check_slots(layout, ev)
        self.check_batch(layout)
        _check_keys(ev, transpose_rotation_steps(self.d_out, self.d_in, layout))
        plan = zip(transpose_sources(self.d_out, self.d_in, layout),
                   rotations_for_transpose(self.d_out, self.d_in, layout))
        plan = list(plan)
        moved = iter(_rotate_all(ev, [(self.entries[c], a) for c, a in plan if a != 0]))
        entries = [self.entries[c] if a == 0 else next(moved) for c, a in plan]
        return EncWeights(entries, self.d_in, self.d_out, layout)


def fold(ev, y, d_out, d_in, layout):
    """y = y + rot(y, n_out 2^t batch) for t < log2(n_in / n_out) (dense.rs:115-134)."""
    sh = checked_shape(d_out, d_in, layout)
    steps = _fold_rotation_steps(sh, layout)
    _check_keys(ev, steps)
    for step in steps:
        r = ev.rotate(y, step)
        y = ev.add(y, r)
    return y


def _lane0_plaintext(ev, layout, c, scale, level):
    """c on lane 0 of every feature, encoded at scale and level (dense.rs:949-967)."""
    if not math.isfinite(c):
        raise InvalidParams(f"gradient constant {c} must be finite")
    mask = np.where(np.arange(layout.slots) % layout.batch == 0, c, 0.0)
    return ev.encode(mask, scale, level)


def _first_period_plaintext(ev, layout, period, c, scale, level):
    """c on lane 0 of the first `period` features (dense.rs:1162-1190)."""
    if not math.isfinite(c):
        raise InvalidParams(f"gradient constant {c} must be finite")
    s = np.arange(layout.slots)
    mask = np.where((s < period * layout.batch) & (s % layout.batch == 0), c, 0.0)
    return ev.encode(mask, scale, level)


def _rotate_all(ev, items):
    """rotate(ct, steps) for every (ct, steps) pair. An evaluator with `rotate_many` runs the
    independent rotations as one batched launch sequence; the results and counts are those of
    the single rotations."""
    if hasattr(ev, "rotate_many"):
        return ev.rotate_many(items)
    return [ev.rotate(c, s) for c, s in items]


def _mul_rescale_all(ev, pairs):
    """rescale(mul(a, b)) for every pair, batched where the evaluator offers `mul_rescale_many`."""
    if hasattr(ev, "mul_rescale_many"):
        return ev.mul_rescale_many(pairs)
    return [ev.rescale(ev.mul(a, b)) for a, b in pairs]


def _batch_sum_consts_all(ev, vs, masks, target, layout):
    """_batch_sum_consts for several independent ciphertexts, each rotation round batched over
    them (every ciphertext sees the op sequence of _batch_sum_consts)."""
    reduce, replicate = _lane_steps(layout)
    for s in reduce:
        rs = _rotate_all(ev, [(v, s) for v in vs])
        vs = [ev.add(v, r) for v, r in zip(vs, rs)]
    outs = []
    for mask in masks:
        os_ = [ev.rescale(ev.mul_plain_to_scale(v, mask, target)) for v in vs]
        for s in replicate:
            rs = _rotate_all(ev, [(o, s) for o in os_])
            os_ = [ev.add(o, r) for o, r in zip(os_, rs)]
        outs.append(os_)
    return outs


def _batch_sum_consts(ev, v, masks, target, layout):
    """Reduce (log2 B rotations), per mask a ct-pt product landing on `target` and a rescale,
    then replicate (log2 B rotations) (dense.rs:917-947)."""
    return [out[0] for out in _batch_sum_consts_all(ev, [v], masks, target, layout)]


class Dense:
    """An encrypted dense layer z = x W^T + b (dense.rs:363-531). `b` is in canonical form at the
    exact scale of the unrescaled matvec output."""

    def __init__(self, w, b):
        self.w, self.b = w, b

    def forward(self, ev, x, layout):
        """rescale(fold(matvec_enc(W, x)) + b) (dense.rs:467-504)."""
        sh = self.w.shape(layout)
        _check_slots(layout, ev)
        self.w.check_batch(layout)
        _check_keys(ev, forward_rotation_steps(sh.d_out, sh.d_in, layout))
        level = x.level()
        if self.w.level() < level or self.b.level() < level:
            raise LevelMismatch("weights or bias below the input level")
        if self.b.scale() != self.w.product_scale(x.scale()):
            raise ScaleMismatch("bias scale is not the product scale")
        diags = self.w.mod_switch_to_level(ev, level) if self.w.level() > level else self.w.entries
        b = ev.mod_switch_to_level(self.b, level) if self.b.level() > level else self.b
        y = ev.matvec_enc(sh.m, layout.batch, diags, x)
        y = fold(ev, y, sh.d_out, sh.d_in, layout)
        y = ev.add(y, b)
        return ev.rescale(y)

    def backward_input(self, ev, delta, wt, layout):
        """rescale(fold_{W^T}(matvec_enc(W^T, delta))) (dense.rs:761-796)."""
        d_out, d_in = self.w.d_out, self.w.d_in
        if (wt.d_out, wt.d_in) != (d_in, d_out):
            raise InvalidParams(f"backward of a {d_out} x {d_in} layer needs {d_in} x {d_out} weights, "
                                f"got {wt.d_out} x {wt.d_in}")
        sh = wt.shape(layout)
        _check_slots(layout, ev)
        wt.check_batch(layout)
        _check_keys(ev, backward_rotation_steps(d_out, d_in, layout))
        level = delta.level()
        if wt.level() < level:
            raise LevelMismatch("transposed weights below delta's level")
        diags = wt.mod_switch_to_level(ev, level) if wt.level() > level else wt.entries
        y = ev.matvec_enc(sh.m, layout.batch, diags, delta)
        y = fold(ev, y, d_in, d_out, layout)
        return ev.rescale(y)

    def weight_grad_scaled(self, ev, delta, a_prev, layout, c):
        """c delta^T A summed over the lanes, as replicated pre-rotated diagonals at level l - 2
        and exactly the weights' scale (dense.rs:1014-1098)."""
        return self.weight_grad_scaled_consts(ev, delta, a_prev, layout, [c])[0]

    def weight_grad_scaled_consts(self, ev, delta, a_prev, layout, cs):
        """dense.rs:1035-1098: hoisted rotations of A (baby) and delta (giant), per diagonal one
        mul + rescale, then the batch sum with one lane-0 mask per constant."""
        if not cs:
            raise InvalidParams("no gradient constant")
        sh = self.w.shape(layout)
        _check_slots(layout, ev)
        self.w.check_batch(layout)
        _check_keys(ev, grad_rotation_steps(sh.d_out, sh.d_in, layout))
        if not ev.has_relin_key():
            raise InvalidParams("evaluator has no relinearization key")
        for ct in (delta, a_prev):
            _check_input(ev, ct)
        level = min(delta.level(), a_prev.level())
        if level < 2:
            raise NoLevelsLeft("gradient needs two levels")
        prod_scale = delta.scale() * a_prev.scale() / float(ev.params().q[level])
        target = self.w.scale()
        mask_scale = ev.exact_product_scale(level - 1, target) / prod_scale
        masks = [_lane0_plaintext(ev, layout, c, mask_scale, level - 1) for c in cs]
        b = layout.batch
        delta = ev.mod_switch_to_level(delta, level)
        a = ev.mod_switch_to_level(a_prev, level)
        a_rot = ev.hoisted_rotate(a, [k2 * b for k2 in range(sh.baby)])
        d_rot = ev.hoisted_rotate(delta, [-(sh.baby * k1 * b) for k1 in range(sh.giant)])
        # the m diagonals are independent: each takes dense.rs's sequence, the rounds batched
        ps = _mul_rescale_all(ev, [(d_rot[e // sh.baby], a_rot[e % sh.baby]) for e in range(sh.m)])
        return _batch_sum_consts_all(ev, ps, masks, target, layout)

    def bias_grad_scaled(self, ev, delta, layout, c):
        """c sum_b delta_b in canonical form at exactly the bias scale, one level below delta
        (dense.rs:1118-1139)."""
        self.w.shape(layout)
        _check_slots(layout, ev)
        self.w.check_batch(layout)
        _check_keys(ev, bias_grad_rotation_steps(layout))
        _check_input(ev, delta)
        target = self.b.scale()
        mask_scale = ev.target_plain_scale(delta, target)
        mask = _lane0_plaintext(ev, layout, c, mask_scale, delta.level())
        return _batch_sum_consts(ev, delta, [mask], target, layout)[0]

    def weight_grad_reduced(self, ev, deltas, a_prevs, layout, c):
        """The compact update's gradient: products summed over micro-batches before one relin per
        diagonal, the batch reduce only and the first-period lane-0 mask (dense.rs:1233-1345)."""
        return self.weight_grad_reduced_consts(ev, deltas, a_prevs, layout, [c])[-1]

    def weight_grad_reduced_consts(self, ev, deltas, a_prevs, layout, cs):
        """dense.rs:1252-1345."""
        if not cs:
            raise InvalidParams("no gradient constant")
        sh = self.w.shape(layout)
        _check_slots(layout, ev)
        self.w.check_batch(layout)
        if len(deltas) != len(a_prevs):
            raise InvalidParams(f"{len(deltas)} delta and {len(a_prevs)} input micro-batches")
        _check_micro(deltas, "delta")
        _check_micro(a_prevs, "layer input")
        _check_keys(ev, grad_reduced_rotation_steps(sh.d_out, sh.d_in, layout))
        if not ev.has_relin_key():
            raise InvalidParams("evaluator has no relinearization key")
        for ct in list(deltas) + list(a_prevs):
            _check_input(ev, ct)
        level = min(deltas[0].level(), a_prevs[0].level())
        if level < 2:
            raise NoLevelsLeft("gradient needs two levels")
        prod_scale = deltas[0].scale() * a_prevs[0].scale() / float(ev.params().q[level])
        target = self.w.scale()
        mask_scale = ev.exact_product_scale(level - 1, target) / prod_scale
        masks = [_first_period_plaintext(ev, layout, sh.l, c, mask_scale, level - 1) for c in cs]
        b = layout.batch
        a_steps = [k2 * b for k2 in range(sh.baby)]
        d_steps = [-(sh.baby * k1 * b) for k1 in range(sh.giant)]
        rots = []
        for d, a in zip(deltas, a_prevs):
            d = ev.mod_switch_to_level(d, level)
            a = ev.mod_switch_to_level(a, level)
            rots.append((ev.hoisted_rotate(d, d_steps), ev.hoisted_rotate(a, a_steps)))
        reduce = _lane_steps(layout)[0]
        out = [[] for _ in cs]
        for e in range(sh.m):
            acc = None
            for d_rot, a_rot in rots:
                p = ev.mul_lazy(d_rot[e // sh.baby], a_rot[e % sh.baby])
                acc = p if acc is None else ev.add(acc, p)
            v = ev.rescale(ev.relin_lazy(acc))
            for s in reduce:
                r = ev.rotate(v, s)
                v = ev.add(v, r)
            for o, mask in zip(out, masks):
                o.append(ev.rescale(ev.mul_plain_to_scale(v, mask, target)))
        return out

    def bias_grad_reduced(self, ev, dzs, layout, c, period, target_scale):
        """c sum_mb sum_b dz on lane 0 of the first `period` features, exactly `target_scale`
        (dense.rs:1347-1385)."""
        sh = self.w.shape(layout)
        _check_slots(layout, ev)
        self.w.check_batch(layout)
        _check_micro(dzs, "dz")
        reduce = _lane_steps(layout)[0]
        _check_keys(ev, reduce)
        if not (_pow2(period) and sh.n_out <= period <= layout.d):
            raise InvalidParams(f"bias period {period} for {sh.n_out} outputs in layout d = {layout.d}")
        for ct in dzs:
            _check_input(ev, ct)
        mask_scale = ev.target_plain_scale(dzs[0], target_scale)
        mask = _first_period_plaintext(ev, layout, period, c, mask_scale, dzs[0].level())
        v = dzs[0]
        for d in dzs[1:]:
            v = ev.add(v, d)
        for s in reduce:
            r = ev.rotate(v, s)
            v = ev.add(v, r)
        return ev.rescale(ev.mul_plain_to_scale(v, mask, target_scale))


def _check_micro(xs, what):
    """Nonempty, one level and one scale (dense.rs:1192-1206)."""
    if not xs:
        raise InvalidParams(f"no {what} ciphertexts")
    l0, s0 = xs[0].level(), xs[0].scale()
    if any(x.level() != l0 or x.scale() != s0 for x in xs):
        raise InvalidParams(f"the {what} micro-batches must share one level and one scale")


# ---------------------------------------------------------------------------------------------
# Activation, loss, optimizer
# ---------------------------------------------------------------------------------------------


class Square:
    """z^2; derivative 2z (crates/ckks-train-nn/src/activation.rs:119-121, 386-432)."""

    depth = 1
    derivative_depth = 1

    @staticmethod
    def eval_plain(z):
        return z * z

    def constant_derivative(self):
        return None

    def forward(self, ev, z):
        """rescale(z * z) (activation.rs:409-412, 238-240)."""
        if z.level() < 1:
            raise NoLevelsLeft("square needs a level")
        return ev.rescale(ev.mul(z, z))

    def derivative_factor_at(self, ev, z, scale_const, mask=None, target_scale=None):
        """scale_const * mask * 2z with the constants folded into one plaintext multiply
        (activation.rs:414-430): eval_poly with coefficients [None, 2 km] is `mul_to`, the plaintext
        encoded at target q_l / z.scale (activation.rs:178-196, 252-256)."""
        slots = ev.params().n // 2
        if not math.isfinite(scale_const):
            raise InvalidParams("non-finite scale_const")
        if mask is None:
            km = np.full(slots, scale_const)
        else:
            mask = np.asarray(mask, np.float64)
            if len(mask) > slots:
                raise InvalidParams(f"mask has {len(mask)} entries, {slots} slots")
            km = mask * scale_const
        if not np.any(km != 0.0):
            raise InvalidParams("derivative factor is identically zero")
        c1 = km * 2.0
        if z.level() < 1:
            raise NoLevelsLeft("derivative needs a level")
        t = z.scale() if target_scale is None else target_scale
        lvl = z.level()
        q = float(ev.params().q[lvl])
        pt = ev.encode(c1, t * q / z.scale(), lvl)
        return ev.rescale(ev.mul_plain(z, pt))


_SAME_SCALE = 1e-12


class Mse:
    """delta = pred - target, scales equal to 1e-12 relative (crates/ckks-train-nn/src/loss.rs:20-44)."""

    @staticmethod
    def grad(ev, pred, target):
        a, b = pred.scale(), target.scale()
        if abs(a - b) > _SAME_SCALE * min(a, b):
            raise ScaleMismatch("prediction and target scales differ")
        level = min(pred.level(), target.level())
        return ev.sub(ev.mod_switch_to_level(pred, level), ev.mod_switch_to_level(target, level))


class Sgd:
    """W' = W - dW with lr folded into the gradient (crates/ckks-train-nn/src/optim.rs:136-179)."""

    def __init__(self, lr):
        if not (math.isfinite(lr) and lr > 0):
            raise InvalidParams(f"learning rate {lr} must be finite and positive")
        self.lr = lr

    def grad_scale(self):
        return self.lr

    def bias_grad_scale(self):
        return self.lr

    def step(self, ev, w, dw, layout):
        """optim.rs:110-124, 171-179: dw uniform, w at or above its level with exactly its scale."""
        if len(dw) != len(w.entries):
            raise InvalidParams("gradient and weights differ in shape")
        _check_uniform(dw)
        level = dw[0].level()
        if w.level() < level:
            raise LevelMismatch("weights below the gradient's level")
        if w.scale() != dw[0].scale():
            raise ScaleMismatch("gradient scale is not the weights' scale")
        entries = [ev.sub(we, g) for we, g in zip(w.mod_switch_to_level(ev, level), dw)]
        return EncWeights(entries, w.d_out, w.d_in, layout)


# ---------------------------------------------------------------------------------------------
# The network and the interactive training step (trainer.rs)
# ---------------------------------------------------------------------------------------------


def dense_out(ev, level, x_scale, w_scale):
    """(level - 1, x_scale w_scale / q_level) (trainer.rs:343-356)."""
    if level == 0:
        raise NoLevelsLeft("dense layer needs a level")
    return level - 1, (x_scale * w_scale) / float(ev.params().q[level])


def square_out(ev, level, scale):
    """Square's output (level, scale): the labels of rescale(mul(z, z))."""
    if level == 0:
        raise NoLevelsLeft("square needs a level")
    return level - 1, (scale * scale) / float(ev.params().q[level])


class Mlp:
    """Dense layers, each followed by its activation (trainer.rs:446-455)."""

    def __init__(self, layers):
        if not layers:
            raise InvalidParams("empty network")
        self.layers = list(layers)

    def dims(self):
        return [self.layers[0][0].w.d_in] + [d.w.d_out for d, _ in self.layers]

    @staticmethod
    def scales(ev, dims, level, delta, w_scale=None):
        """For inputs at (level, delta) and weights at `w_scale` (default delta): per layer the
        (level, scale) of its input and the bias scale, and the output (level, scale) where the
        client encrypts y (Mlp::encrypt_at / batch_spec_at, trainer.rs:480-548, 566-600, with the
        Square activation's labels in place of the zero-ciphertext probe)."""
        w_scale = delta if w_scale is None else w_scale
        out, scale = [], delta
        for _ in range(len(dims) - 1):
            bias_scale = scale * w_scale
            out.append((level, scale, bias_scale))
            level, scale = dense_out(ev, level, scale, w_scale)
            level, scale = square_out(ev, level, scale)
        return out, (level, scale)


class Trainer:
    """The interactive trainer's step with per-layer SGD (trainer.rs:780-1366), one micro-batch,
    without the refresh: afterwards every weight and bias is at its old exact scale, on the level
    the step left it (a refresher or a bootstrap brings it back up)."""

    def __init__(self, ev, layout, optims, frozen_biases=False):
        self.ev, self.layout, self.optims = ev, layout, list(optims)
        self.frozen_biases = frozen_biases
        self.trace = []

    def train_batch(self, mlp, x, y):
        return self.train_batch_valid(mlp, x, y, self.layout.batch)

    def train_batch_valid(self, mlp, x, y, n_valid):
        """trainer.rs:1014-1366 for one micro-batch. Returns the step's values by name
        ("z", "a", "delta", "s", "dz", "wt", "backward", "dw", "db") for inspection; the network
        is updated in place."""
        ev, layout = self.ev, self.layout
        n_layers = len(mlp.layers)
        if n_layers == 0 or len(self.optims) != n_layers:
            raise InvalidParams(f"{n_layers} layers and {len(self.optims)} optimizers")
        if n_valid == 0 or n_valid > layout.batch:
            raise InvalidParams(f"{n_valid} valid samples for a batch of {layout.batch}")
        for p, q in zip(mlp.layers, mlp.layers[1:]):
            if q[0].w.d_in != p[0].w.d_out:
                raise InvalidParams("layer shapes do not chain")
        coeffs = []
        for opt in self.optims:
            cur = opt.grad_scale() / n_valid
            bias = 0.0 if self.frozen_biases else opt.bias_grad_scale() / n_valid
            if not (math.isfinite(cur) and math.isfinite(bias)):
                raise InvalidParams("nonfinite folded gradient coefficient")
            coeffs.append((cur, bias))
        trace, rec = [], {k: {} for k in ("z", "a", "delta", "s", "dz", "wt", "backward", "dw", "db")}
        # 1. forward: acts[i] is the input of layer i
        acts, zs = [x], []
        for i, (dense, act) in enumerate(mlp.layers):
            z = dense.forward(ev, acts[i], layout)
            trace.append((f"z{i + 1}", z.level()))
            a = act.forward(ev, z)
            trace.append((f"a{i + 1}", a.level()))
            zs.append(z)
            acts.append(a)
            rec["z"][i], rec["a"][i] = z, a
        # 2. loss gradient
        delta = Mse.grad(ev, acts[n_layers], y)
        trace.append((f"delta{n_layers}", delta.level()))
        rec["delta"][n_layers - 1] = delta
        # 3. backward and gradients, top down
        mask = valid_lane_mask(layout, n_valid)
        grads, new_biases = [], []
        for i in reversed(range(n_layers)):
            ln = i + 1
            dense, act = mlp.layers[i]
            if act.constant_derivative() is not None:
                raise InvalidParams("activations with a constant derivative are not supported")
            s = act.derivative_factor_at(ev, zs[i], 1.0, mask, None)
            trace.append((f"s{ln}", s.level()))
            lv = min(s.level(), delta.level())
            dz = ev.rescale(ev.mul(ev.mod_switch_to_level(delta, lv), ev.mod_switch_to_level(s, lv)))
            trace.append((f"dz{ln}", dz.level()))
            rec["s"][i], rec["dz"][i] = s, dz
            nxt = None
            if i > 0:
                low = EncWeights(dense.w.mod_switch_to_level(ev, dz.level()), dense.w.d_out, dense.w.d_in, layout)
                wt = low.transpose(ev, layout)
                nxt = dense.backward_input(ev, dz, wt, layout)
                trace.append((f"delta{i}", nxt.level()))
                rec["wt"][i], rec["backward"][i] = wt, nxt
            c, c_b = coeffs[i]
            dw = dense.weight_grad_scaled(ev, dz, acts[i], layout, c)
            db = self._bias_grad(dense, dz, c_b)
            rec["dw"][i], rec["db"][i] = dw, db
            new_biases.append(ev.sub(ev.mod_switch_to_level(dense.b, db.level()), db))
            grads.append((i, dw))
            if nxt is not None:
                delta = nxt
        # 4. optimizer steps, then commit
        new_layers = []
        for (i, dw), b_new in zip(grads, new_biases):
            w = self.optims[i].step(ev, mlp.layers[i][0].w, dw, layout)
            trace.append((f"W{i + 1}'", w.level()))
            trace.append((f"b{i + 1}'", b_new.level()))
            new_layers.append((i, w, b_new))
        for i, w, b in new_layers:
            mlp.layers[i][0].w = w
            mlp.layers[i][0].b = b
        self.trace = trace
        return rec

    def _bias_grad(self, dense, dz, c):
        """bias_grad_scaled, retried one level lower on ScaleMismatch (trainer.rs:764-785)."""
        try:
            return dense.bias_grad_scaled(self.ev, dz, self.layout, c)
        except ScaleMismatch:
            if dz.level() < 2:
                raise
            lower = self.ev.mod_switch_to_level(dz, dz.level() - 1)
            return dense.bias_grad_scaled(self.ev, lower, self.layout, c)


def step_counts(dims, layout):
    """Evaluator counts of one training step (Trainer::train_batch, SGD, Square everywhere, full
    batch), from the per-op costs documented in dense.rs and trainer.rs: forward
    baby + giant - 2 + fold rotations, m tensors, giant relins, 1 rescale; Square 1 tensor, 1 relin,
    1 rescale; derivative 1 ct-pt, 1 rescale; dz 1 tensor, 1 relin, 1 rescale; transpose m - 1
    rotations; backward as the forward of W^T; weight gradient (baby - 1) + (giant - 1) +
    2 m log2 B rotations, m tensors, m relins, m ct-pt, 2 m rescales; bias gradient 2 log2 B
    rotations, 1 ct-pt, 1 rescale."""
    lb = layout.log_batch()
    c = dict(rotations=0, relins=0, ct_ct_tensor=0, ct_pt_mults=0, rescales=0)
    for i in range(len(dims) - 1):
        sh = LayerShape(dims[i + 1], dims[i], layout)
        # forward and the activation
        c["rotations"] += sh.baby + sh.giant - 2 + sh.fold_steps()
        c["ct_ct_tensor"] += sh.m + 1
        c["relins"] += sh.giant + 1
        c["rescales"] += 2
        # derivative factor and dz
        c["ct_pt_mults"] += 1
        c["ct_ct_tensor"] += 1
        c["relins"] += 1
        c["rescales"] += 2
        if i > 0:
            st = LayerShape(dims[i], dims[i + 1], layout)
            c["rotations"] += (sh.m - 1) + st.baby + st.giant - 2 + st.fold_steps()
            c["ct_ct_tensor"] += st.m
            c["relins"] += st.giant
            c["rescales"] += 1
        c["rotations"] += (sh.baby - 1) + (sh.giant - 1) + 2 * sh.m * lb + 2 * lb
        c["ct_ct_tensor"] += sh.m
        c["relins"] += sh.m
        c["ct_pt_mults"] += sh.m + 1
        c["rescales"] += 2 * sh.m + 1
    return c
