"""Test helpers for the encrypted training step: the oracle's CPU evaluator behind the same
HeOps methods as CudaEvaluator (so `ckks_train_b200.nn` runs unchanged on both, as the
reference's generic trainer does on its CPU and CUDA backends), the client side (encryption,
decryption) and the plaintext training step the decrypted results are held against.
"""

import numpy as np

import oracle as O


class OracleCt:
    def __init__(self, ct):
        self.ct = ct

    def level(self):
        return self.ct.level

    def scale(self):
        return self.ct.scale

    def size(self):
        return self.ct.ncomp


class OraclePt:
    def __init__(self, data, scale, level):
        self.data, self._scale, self._level = data, scale, level

    def level(self):
        return self._level

    def scale(self):
        return self._scale


class _Params:
    def __init__(self, P):
        self.q = [int(x) for x in P.q]
        self.n = P.n


class OracleHeOps:
    """The oracle Evaluator (crates/ckks-train-ckks/src/evaluator.rs restated) with HeOps method
    names and argument order; `steps` are the rotations the Galois keys cover."""

    def __init__(self, P, relin, galois, lazy_relin=True):
        self.P, self._params = P, _Params(P)
        self.ev = O.Evaluator(P, relin, galois, lazy_relin=lazy_relin)
        self.enc = O.Encoder(P)
        self._relin, self._elts, self.lazy = relin is not None, set(galois), lazy_relin

    def params(self):
        return self._params

    def counter(self):
        return self.ev.counter()

    def has_relin_key(self):
        return self._relin

    def has_galois_key(self, step):
        slots = self.P.n // 2
        return step % slots == 0 or O.galois_elt(self.P.n, step) in self._elts

    def owns(self, ct):
        return isinstance(ct, OracleCt)

    def _w(self, ct):
        return OracleCt(ct)

    def add(self, a, b):
        return self._w(self.ev.add(a.ct, b.ct))

    def sub(self, a, b):
        return self._w(self.ev.sub(a.ct, b.ct))

    def mul(self, a, b):
        return self._w(self.ev.mul(a.ct, b.ct))

    def mul_no_relin(self, a, b):
        return self._w(self.ev.mul_no_relin(a.ct, b.ct))

    def relinearize(self, a):
        return self._w(self.ev.relinearize(a.ct))

    def mul_lazy(self, a, b):
        return self.mul_no_relin(a, b) if self.lazy else self.mul(a, b)

    def relin_lazy(self, s):
        return self.relinearize(s) if self.lazy else s

    def rescale(self, a):
        return self._w(self.ev.rescale(a.ct))

    def rotate(self, a, steps):
        return self._w(self.ev.rotate(a.ct, steps))

    def hoisted_rotate(self, a, steps):
        return [self._w(c) for c in self.ev.hoisted_rotate(a.ct, list(steps))]

    def mod_switch_to_level(self, a, level):
        return self._w(self.ev.mod_switch_to_level(a.ct, level))

    def mul_plain(self, a, pt):
        return self._w(self.ev.mul_plain(a.ct, pt.data, pt.scale()))

    def mul_plain_to_scale(self, a, pt, target):
        return self._w(self.ev.mul_plain_to_scale(a.ct, pt.data, pt.scale(), target))

    def matvec_enc(self, d, stride, entries, x):
        return self._w(self.ev.matvec_enc(d, stride, [e.ct for e in entries], x.ct))

    def exact_product_scale(self, level, target):
        return self.ev.exact_product_scale(level, target)

    def target_plain_scale(self, ct, target):
        from ckks_train_b200 import InvalidParams
        sp = self.exact_product_scale(ct.level(), target) / ct.scale()
        if sp < 1048576.0:
            raise InvalidParams("plaintext scale is below 2^20")
        return sp

    def encode(self, values, scale, level):
        return OraclePt(self.enc.encode(np.asarray(values, np.float64), scale, level), scale, level)


class Client:
    """The key owner: secret key, symmetric encryption, decryption and decoding."""

    def __init__(self, P, kg, seed=1):
        self.P, self.kg, self.enc = P, kg, O.Encoder(P)
        self.seed = seed

    def encrypt(self, ev, values, scale, level):
        self.seed += 1
        pt = self.enc.encode(np.asarray(values, np.float64), scale, level)
        return O.encrypt_sk(ev, self.kg, self.seed.to_bytes(4, "little") * 8, pt, scale)

    def decrypt(self, data, level, scale):
        """Decoded real slots of a ciphertext given as (components, limbs, N) words."""
        ct = O.Evaluator(self.P).ct(np.asarray(data, np.uint64), scale)
        return self.enc.decode(O.decrypt(self.kg, ct), scale).real


def plain_step(ws, bs, x, y, lr, n_valid=None):
    """The SGD step of trainer.rs in plaintext fp64 (Square after every layer, MSE gradient
    a_L - y, gradients summed over the valid samples and scaled by lr / n): the updated
    weights and biases and the forward values."""
    n = x.shape[0] if n_valid is None else n_valid
    acts, zs = [x[:n]], []
    for w, b in zip(ws, bs):
        z = acts[-1] @ w.T + b
        zs.append(z)
        acts.append(z * z)
    delta = acts[-1] - y[:n]
    new_w, new_b = [None] * len(ws), [None] * len(ws)
    for i in reversed(range(len(ws))):
        dz = delta * 2.0 * zs[i]
        c = lr / n
        new_w[i] = ws[i] - c * dz.T @ acts[i]
        new_b[i] = bs[i] - c * dz.sum(axis=0)
        delta = dz @ ws[i]
    return new_w, new_b, zs, acts


def deterministic_keys(P, steps, seed, threads=8):
    """Relinearization key and the Galois keys of `steps` from `threads` key generators of the
    same seed: generator t makes the keys of elements t, t + threads, ... one after another in
    its own task, then generator 0 the relinearization key. The keys depend on the seed and
    `threads` only (not on the host's core count or on scheduling)."""
    from concurrent.futures import ThreadPoolExecutor

    elts = sorted({O.galois_elt(P.n, s) for s in steps} - {1})
    kgs = [O.KeyGenerator(P, seed) for _ in range(threads)]

    def task(t):
        return [(e, kgs[t].galois_key(e)) for e in elts[t::threads]]

    with ThreadPoolExecutor(threads) as ex:
        parts = list(ex.map(task, range(threads)))
    gk = dict(kv for part in parts for kv in part)
    return kgs[0], kgs[0].relin_key(), {e: gk[e] for e in elts}


def step_values(v, mlp):
    """Every ciphertext of one training step in a fixed order, as (name, ciphertext): the
    forward values, deltas, derivative factors, dz, backward deltas and bias gradients, the
    transposed weights and weight gradients, then the updated network."""
    out = []
    for name in ("z", "a", "delta", "s", "dz", "backward", "db"):
        for i in sorted(v[name]):
            out.append((f"{name}{i + 1}", v[name][i]))
    for name in ("wt", "dw"):
        for i in sorted(v[name]):
            es = v[name][i].entries if name == "wt" else v[name][i]
            out.extend((f"{name}{i + 1}[{k}]", e) for k, e in enumerate(es))
    for i, (dense, _) in enumerate(mlp.layers):
        out.extend((f"W{i + 1}'[{k}]", e) for k, e in enumerate(dense.w.entries))
        out.append((f"b{i + 1}'", dense.b))
    return out


def ct_digest(data, level, scale):
    """SHA-256 of a ciphertext's words (little-endian u64, components x limbs x N), its level
    and the bits of its f64 scale."""
    import hashlib
    import struct

    h = hashlib.sha256(np.ascontiguousarray(data, "<u8").tobytes())
    h.update(struct.pack("<Qd", int(level), float(scale)))
    return h.hexdigest()
