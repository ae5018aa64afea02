"""ctypes wrapper of the CPU oracle (test infrastructure only).

The oracle (``oracle_ckks.cpp``) restates the reference's CPU path of the RNS-CKKS
evaluator: crates/ckks-train-core/src/{modulus,ntt,rns,primes,poly,baseconv,sampler}.rs
and crates/ckks-train-ckks/src/{params,keys,keyswitch,evaluator,linalg,counter}.rs.
Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this
module; the product never does.
"""

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "libckks_oracle.so")

U64P = C.POINTER(C.c_uint64)
U32P = C.POINTER(C.c_uint32)
I32P = C.POINTER(C.c_int32)

ERR_NAMES = {1: "InvalidParams", 2: "ScaleMismatch", 3: "LevelMismatch", 4: "NoLevelsLeft", 5: "Decode",
             6: "Device", 100: "Panic"}


class OracleError(Exception):
    """A reference-side error (HekitError kind + message)."""

    def __init__(self, code, msg):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code
        self.kind = ERR_NAMES.get(code, str(code))


def build():
    """Compiles the oracle with its Makefile (g++, OpenMP, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    vp = C.c_void_p
    L.orc_last_error.restype = C.c_char_p
    L.orc_is_prime.argtypes = [C.c_uint64]
    L.orc_ntt_primes_skip.argtypes = [C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64, U64P]
    L.orc_min_root.argtypes = [C.c_uint64, C.c_uint64, U64P]
    L.orc_barrett.argtypes = [C.c_uint64, U64P, U64P]
    L.orc_mulmod.argtypes = [C.c_uint64] * 3
    L.orc_mulmod.restype = C.c_uint64
    L.orc_mul_shoup.argtypes = [C.c_uint64] * 3
    L.orc_mul_shoup.restype = C.c_uint64
    L.orc_galois_elt.argtypes = [C.c_uint64, C.c_int32]
    L.orc_galois_elt.restype = C.c_uint64
    L.orc_galois_perm.argtypes = [C.c_uint64, C.c_uint64, U32P]
    L.orc_chacha_words.argtypes = [C.c_char_p, C.c_uint64, U64P]
    L.orc_seed_from_u64.argtypes = [C.c_uint64, C.c_char_p]
    L.orc_bsgs_split.argtypes = [C.c_uint64, U64P, U64P]
    L.orc_bsgs_steps.argtypes = [C.c_uint64, C.c_uint64, C.c_int64, I32P]
    L.orc_cdt_table.argtypes = [C.c_double, U64P, U64P]
    L.orc_params_from_bits.argtypes = [C.c_uint32, U32P, C.c_uint64, U32P, C.c_uint64, C.c_uint32, C.c_uint64,
                                       C.POINTER(vp)]
    L.orc_params_from_primes.argtypes = [C.c_uint32, U64P, C.c_uint64, U64P, C.c_uint64, C.c_double, C.c_uint64,
                                         C.POINTER(vp)]
    L.orc_params_free.argtypes = [vp]
    L.orc_params_primes.argtypes = [vp, U64P, U64P]
    L.orc_params_log_pq.argtypes = [vp]
    L.orc_params_log_pq.restype = C.c_double
    L.orc_params_scale_at.argtypes = [vp, C.c_uint64]
    L.orc_params_scale_at.restype = C.c_double
    L.orc_digit_ranges.argtypes = [vp, C.c_uint64, U64P]
    L.orc_ntt.argtypes = [vp, C.c_int, C.c_uint64, C.c_uint64, U64P, C.c_int]
    L.orc_poly_op.argtypes = [vp, C.c_int, C.c_uint64, C.c_int, U64P, U64P, C.c_uint64]
    L.orc_automorphism.argtypes = [vp, C.c_int, C.c_uint64, U64P, C.c_uint64, C.c_int, U64P]
    L.orc_rescale.argtypes = [vp, U64P, C.c_uint64, C.c_int, U64P]
    L.orc_mod_up.argtypes = [vp, U64P, C.c_uint64, C.c_uint64, U64P, U64P]
    L.orc_mod_down.argtypes = [vp, U64P, C.c_uint64, U64P, C.c_int, U64P]
    L.orc_raise_from_level0.argtypes = [vp, U64P, C.c_uint64, C.c_int, U64P]
    L.orc_random_poly.argtypes = [C.c_uint64, U64P, C.c_uint64, C.c_uint64, U64P]
    L.orc_keygen_new.argtypes = [vp, C.c_char_p, C.POINTER(vp)]
    L.orc_keygen_free.argtypes = [vp]
    L.orc_keygen_secret.argtypes = [vp, U64P]
    L.orc_keygen_relin.argtypes = [vp, C.POINTER(vp)]
    L.orc_keygen_galois.argtypes = [vp, C.c_uint64, C.POINTER(vp)]
    L.orc_key_free.argtypes = [vp]
    L.orc_key_parts.argtypes = [vp]
    L.orc_key_parts.restype = C.c_uint64
    L.orc_key_qlimbs.argtypes = [vp]
    L.orc_key_qlimbs.restype = C.c_uint64
    L.orc_key_export.argtypes = [vp, U64P]
    L.orc_key_import.argtypes = [vp, U64P, C.c_uint64, C.c_uint64, C.POINTER(vp)]
    L.orc_key_switch.argtypes = [vp, vp, U64P, C.c_uint64, U64P, U64P]
    L.orc_eval_new.argtypes = [vp, vp, C.POINTER(vp), U64P, C.c_uint64, C.c_int, C.c_int, C.c_int, C.POINTER(vp)]
    L.orc_eval_free.argtypes = [vp]
    L.orc_eval_counter.argtypes = [vp, U64P]
    L.orc_eval_reset_counter.argtypes = [vp]
    L.orc_ct_new.argtypes = [vp, C.c_uint64, C.c_uint64, C.c_double, U64P, C.POINTER(vp)]
    L.orc_ct_free.argtypes = [vp]
    L.orc_ct_info.argtypes = [vp, U64P, U64P, C.POINTER(C.c_double)]
    L.orc_ct_data.argtypes = [vp, U64P]
    L.orc_ct_op.argtypes = [vp, C.c_int, vp, vp, C.POINTER(vp)]
    L.orc_ct_rotate.argtypes = [vp, vp, C.c_int32, C.POINTER(vp)]
    L.orc_ct_hoisted_rotate.argtypes = [vp, vp, I32P, C.c_uint64, C.POINTER(vp)]
    L.orc_ct_mod_switch.argtypes = [vp, vp, C.c_uint64, C.POINTER(vp)]
    L.orc_ct_relabel.argtypes = [vp, vp, C.c_double, C.POINTER(vp)]
    L.orc_ct_mul_scalar.argtypes = [vp, vp, C.c_double, C.c_double, C.POINTER(vp)]
    L.orc_ct_plain_op.argtypes = [vp, C.c_int, vp, U64P, C.c_uint64, C.c_double, C.c_double, C.POINTER(vp)]
    L.orc_exact_product_scale.argtypes = [vp, C.c_uint64, C.c_double, C.POINTER(C.c_int)]
    L.orc_exact_product_scale.restype = C.c_double
    L.orc_matvec_plain.argtypes = [vp, C.c_uint64, C.c_uint64, U64P, C.c_uint64, C.c_double, vp, C.POINTER(vp)]
    L.orc_matvec_enc.argtypes = [vp, C.c_uint64, C.c_uint64, C.POINTER(vp), vp, C.POINTER(vp)]
    L.orc_set_threads.argtypes = [C.c_int]
    L.orc_get_threads.restype = C.c_int
    # bootstrapping (oracle_boot.inc)
    DP = C.POINTER(C.c_double)
    L.orc_encoder_new.argtypes = [vp, C.POINTER(vp)]
    L.orc_encoder_free.argtypes = [vp]
    L.orc_encode_complex.argtypes = [vp, DP, C.c_uint64, C.c_double, C.c_uint64, U64P]
    L.orc_decode_complex.argtypes = [vp, U64P, C.c_uint64, C.c_double, DP]
    L.orc_encrypt_sk.argtypes = [vp, C.c_char_p, U64P, C.c_uint64, C.c_double, C.POINTER(vp)]
    L.orc_decrypt.argtypes = [vp, vp, U64P]
    L.orc_rng_new.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.orc_rng_free.argtypes = [vp]
    L.orc_rng_next_u64.argtypes = [vp, C.c_uint64, U64P]
    L.orc_keygen_public.argtypes = [vp, C.POINTER(vp)]
    L.orc_pk_free.argtypes = [vp]
    L.orc_encrypt_sk_rng.argtypes = [vp, vp, U64P, C.c_uint64, C.c_double, C.POINTER(vp)]
    L.orc_encrypt_pk.argtypes = [vp, vp, vp, U64P, C.c_uint64, C.c_double, C.POINTER(vp)]
    L.orc_boot_new.argtypes = [vp, vp, vp, C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64,
                               C.c_uint64, C.c_int64, C.POINTER(vp)]
    L.orc_boot_free.argtypes = [vp]
    L.orc_boot_output_level.argtypes = [vp]
    L.orc_boot_output_level.restype = C.c_uint64
    L.orc_boot_scales.argtypes = [vp, DP, DP]
    L.orc_boot_coeffs.argtypes = [vp, DP]
    L.orc_boot_coeffs.restype = C.c_uint64
    L.orc_boot_num_stages.argtypes = [vp, C.c_int]
    L.orc_boot_num_stages.restype = C.c_uint64
    L.orc_boot_stage_info.argtypes = [vp, C.c_int, C.c_uint64, U64P, C.POINTER(C.c_int64), DP]
    L.orc_boot_stage_entry.argtypes = [vp, C.c_int, C.c_uint64, C.c_int, C.c_uint64, U64P]
    L.orc_boot_num_galois.argtypes = [vp]
    L.orc_boot_num_galois.restype = C.c_uint64
    L.orc_boot_galois.argtypes = [vp, C.c_uint64, U64P, C.POINTER(vp)]
    L.orc_boot_num_steps.argtypes = [vp, I32P]
    L.orc_boot_num_steps.restype = C.c_uint64
    L.orc_boot_sse.argtypes = [vp, C.POINTER(vp), C.POINTER(vp)]
    L.orc_boot_eval.argtypes = [vp, vp, C.POINTER(vp)]
    L.orc_bootstrap.argtypes = [vp, vp, vp, C.POINTER(vp)]
    L.orc_boot_mod_raise.argtypes = [vp, vp, vp, C.POINTER(vp)]
    L.orc_boot_coeff_to_slot.argtypes = [vp, vp, vp, C.POINTER(vp), C.POINTER(vp)]
    L.orc_boot_eval_mod.argtypes = [vp, vp, vp, C.POINTER(vp)]
    L.orc_boot_slot_to_coeff.argtypes = [vp, vp, vp, vp, C.POINTER(vp)]
    L.orc_eval_chebyshev.argtypes = [vp, vp, DP, C.c_uint64, C.c_double, C.c_double, C.c_double, C.POINTER(vp)]
    L.orc_boot_mul_const.argtypes = [vp, vp, C.c_double, C.c_double, C.POINTER(vp)]
    L.orc_boot_add_const.argtypes = [vp, vp, C.c_double, C.POINTER(vp)]
    L.orc_mul_by_x_half.argtypes = [vp, vp, C.POINTER(vp)]
    L.orc_boot_plan.argtypes = [C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64, C.c_int, C.c_uint64,
                                C.POINTER(C.c_int64), C.POINTER(C.c_uint8)]


def _p64(a):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(U64P)


def _check(code):
    if code != 0:
        raise OracleError(code, lib().orc_last_error().decode())


def set_threads(t):
    lib().orc_set_threads(int(t))


def get_threads():
    return lib().orc_get_threads()


# ---- scalar helpers ------------------------------------------------------------------

def is_prime(n):
    return bool(lib().orc_is_prime(int(n)))


def ntt_primes_skip(bits, n, skip, count):
    out = np.zeros(max(count, 1), np.uint64)
    _check(lib().orc_ntt_primes_skip(bits, n, skip, count, _p64(out)))
    return [int(x) for x in out[:count]]


def min_root(n, q):
    v = C.c_uint64()
    _check(lib().orc_min_root(n, q, C.byref(v)))
    return v.value


def barrett(q):
    lo, hi = C.c_uint64(), C.c_uint64()
    _check(lib().orc_barrett(q, C.byref(lo), C.byref(hi)))
    return lo.value | (hi.value << 64)


def mulmod(q, a, b):
    return lib().orc_mulmod(q, a, b)


def mul_shoup(q, a, w):
    return lib().orc_mul_shoup(q, a, w)


def galois_elt(n, step):
    return lib().orc_galois_elt(n, step)


def galois_perm(n, g):
    out = np.zeros(n, np.uint32)
    lib().orc_galois_perm(n, g, out.ctypes.data_as(U32P))
    return out


def chacha_u64(seed32, count):
    out = np.zeros(count, np.uint64)
    lib().orc_chacha_words(bytes(seed32), count, _p64(out))
    return out


def seed_from_u64(s):
    buf = C.create_string_buffer(32)
    lib().orc_seed_from_u64(s, buf)
    return bytes(buf.raw)


def bsgs_split(d):
    b, g = C.c_uint64(), C.c_uint64()
    lib().orc_bsgs_split(d, C.byref(b), C.byref(g))
    return b.value, g.value


def bsgs_steps(d, stride=1, offset=0):
    out = (C.c_int32 * (2 * d + 2))()
    k = lib().orc_bsgs_steps(d, stride, offset, out)
    return list(out[:k])


def cdt_table(sigma):
    n = C.c_uint64()
    lib().orc_cdt_table(sigma, None, C.byref(n))
    out = np.zeros(n.value, np.uint64)
    lib().orc_cdt_table(sigma, _p64(out), C.byref(n))
    return out


def random_poly(seed, primes, n):
    primes = np.asarray(primes, np.uint64)
    out = np.zeros((len(primes), n), np.uint64)
    lib().orc_random_poly(seed, _p64(primes), len(primes), n, _p64(out))
    return out


# ---- parameters and polynomial primitives --------------------------------------------

class Params:
    """CkksParams (crates/ckks-train-ckks/src/params.rs)."""

    @classmethod
    def from_bits(cls, log_n, q_bits, p_bits, scale_bits, dnum):
        qb = (C.c_uint32 * len(q_bits))(*q_bits)
        pb = (C.c_uint32 * len(p_bits))(*p_bits)
        h = C.c_void_p()
        _check(lib().orc_params_from_bits(log_n, qb, len(q_bits), pb, len(p_bits), scale_bits, dnum, C.byref(h)))
        p = cls.__new__(cls)
        p.h = h
        p.log_n, p.dnum = log_n, dnum
        p.nq, p.np_ = len(q_bits), len(p_bits)
        p._load()
        return p

    @classmethod
    def from_primes(cls, log_n, q, p, scale, dnum):
        qa = np.asarray(q, np.uint64)
        pa = np.asarray(p, np.uint64)
        h = C.c_void_p()
        _check(lib().orc_params_from_primes(log_n, _p64(qa), len(qa), _p64(pa), len(pa), scale, dnum, C.byref(h)))
        r = cls.__new__(cls)
        r.h = h
        r.log_n, r.dnum, r.nq, r.np_ = log_n, dnum, len(qa), len(pa)
        r._load()
        return r

    def _load(self):
        q = np.zeros(self.nq, np.uint64)
        p = np.zeros(self.np_, np.uint64)
        lib().orc_params_primes(self.h, _p64(q), _p64(p))
        self.q = [int(x) for x in q]
        self.p = [int(x) for x in p]
        self.n = 1 << self.log_n
        self.alpha = self.nq // self.dnum
        self.max_level = self.nq - 1

    def __del__(self):
        try:
            lib().orc_params_free(self.h)
        except Exception:
            pass

    def log_pq(self):
        return lib().orc_params_log_pq(self.h)

    def scale_at(self, level):
        return lib().orc_params_scale_at(self.h, level)

    def digit_ranges(self, level):
        out = np.zeros(2 * self.dnum, np.uint64)
        k = lib().orc_digit_ranges(self.h, level, _p64(out))
        return [(int(out[2 * i]), int(out[2 * i + 1])) for i in range(k)]

    # primitives (arrays are (limbs, N) uint64, modified copies are returned)
    def ntt(self, data, first_prime=0, inverse=False, basis=0):
        a = np.ascontiguousarray(data, np.uint64).copy()
        _check(lib().orc_ntt(self.h, basis, first_prime, a.shape[0], _p64(a), int(inverse)))
        return a

    def poly_op(self, op, a, b=None, scalar=0, basis=0):
        x = np.ascontiguousarray(a, np.uint64).copy()
        y = np.ascontiguousarray(b if b is not None else a, np.uint64)
        _check(lib().orc_poly_op(self.h, basis, x.shape[0], op, _p64(x), _p64(y), scalar))
        return x

    def automorphism(self, a, g, ntt=True, basis=0):
        x = np.ascontiguousarray(a, np.uint64)
        out = np.zeros_like(x)
        _check(lib().orc_automorphism(self.h, basis, x.shape[0], _p64(x), g, int(ntt), _p64(out)))
        return out

    def rescale(self, a, ntt=True):
        x = np.ascontiguousarray(a, np.uint64)
        level = x.shape[0] - 1
        out = np.zeros((level, self.n), np.uint64)
        _check(lib().orc_rescale(self.h, _p64(x), level, int(ntt), _p64(out)))
        return out

    def mod_up(self, a, digit):
        x = np.ascontiguousarray(a, np.uint64)
        level = x.shape[0] - 1
        oq = np.zeros((level + 1, self.n), np.uint64)
        op = np.zeros((self.np_, self.n), np.uint64)
        _check(lib().orc_mod_up(self.h, _p64(x), level, digit, _p64(oq), _p64(op)))
        return oq, op

    def mod_down(self, q_part, p_part, ntt=True):
        x = np.ascontiguousarray(q_part, np.uint64)
        y = np.ascontiguousarray(p_part, np.uint64)
        level = x.shape[0] - 1
        out = np.zeros_like(x)
        _check(lib().orc_mod_down(self.h, _p64(x), level, _p64(y), int(ntt), _p64(out)))
        return out

    def raise_from_level0(self, a, level, ntt=True):
        x = np.ascontiguousarray(a, np.uint64)
        out = np.zeros((level + 1, self.n), np.uint64)
        _check(lib().orc_raise_from_level0(self.h, _p64(x), level, int(ntt), _p64(out)))
        return out

    def random_q(self, seed, level):
        return random_poly(seed, self.q[: level + 1], self.n)

    def random_p(self, seed):
        return random_poly(seed, self.p, self.n)


# ---- keys ----------------------------------------------------------------------------

class Key:
    """A KskKey (dnum parts (b_j, a_j) over Q*P, NTT form)."""

    def __init__(self, params, handle):
        self.params, self.h = params, handle

    def __del__(self):
        try:
            lib().orc_key_free(self.h)
        except Exception:
            pass

    @property
    def parts(self):
        return lib().orc_key_parts(self.h)

    @property
    def qlimbs(self):
        return lib().orc_key_qlimbs(self.h)

    def export(self):
        """Flat (parts, 2, qlimbs + k, N): per part b then a, each Q limbs then P limbs."""
        P = self.params
        out = np.zeros((self.parts, 2, self.qlimbs + P.np_, P.n), np.uint64)
        lib().orc_key_export(self.h, _p64(out))
        return out

    @classmethod
    def from_array(cls, params, arr):
        arr = np.ascontiguousarray(arr, np.uint64)
        h = C.c_void_p()
        _check(lib().orc_key_import(params.h, _p64(arr), arr.shape[0], arr.shape[2] - params.np_, C.byref(h)))
        return cls(params, h)

    def key_switch(self, d):
        P = self.params
        x = np.ascontiguousarray(d, np.uint64)
        level = x.shape[0] - 1
        ob = np.zeros_like(x)
        oa = np.zeros_like(x)
        _check(lib().orc_key_switch(P.h, self.h, _p64(x), level, _p64(ob), _p64(oa)))
        return ob, oa


class KeyGenerator:
    def __init__(self, params, seed):
        if isinstance(seed, int):
            seed = bytes([seed]) * 32
        self.params = params
        self.h = C.c_void_p()
        _check(lib().orc_keygen_new(params.h, seed, C.byref(self.h)))

    def __del__(self):
        try:
            lib().orc_keygen_free(self.h)
        except Exception:
            pass

    def secret(self):
        P = self.params
        out = np.zeros((P.nq + P.np_, P.n), np.uint64)
        lib().orc_keygen_secret(self.h, _p64(out))
        return out[: P.nq], out[P.nq:]

    def relin_key(self):
        h = C.c_void_p()
        _check(lib().orc_keygen_relin(self.h, C.byref(h)))
        return Key(self.params, h)

    def galois_key(self, elt):
        h = C.c_void_p()
        _check(lib().orc_keygen_galois(self.h, elt, C.byref(h)))
        return Key(self.params, h)

    def public_key(self):
        return PublicKey(self)


# ---- evaluator -----------------------------------------------------------------------

COUNTER_FIELDS = ("rotations", "relins", "ct_ct_tensor", "ct_pt_mults", "rescales", "sse_switches", "bootstraps")


class Ct:
    def __init__(self, ev, h):
        self.ev, self.h = ev, h

    def __del__(self):
        try:
            lib().orc_ct_free(self.h)
        except Exception:
            pass

    def info(self):
        n, l, s = C.c_uint64(), C.c_uint64(), C.c_double()
        lib().orc_ct_info(self.h, C.byref(n), C.byref(l), C.byref(s))
        return n.value, l.value, s.value

    @property
    def level(self):
        return self.info()[1]

    @property
    def scale(self):
        return self.info()[2]

    @property
    def ncomp(self):
        return self.info()[0]

    def data(self):
        n, l, _ = self.info()
        out = np.zeros((n, l + 1, self.ev.params.n), np.uint64)
        lib().orc_ct_data(self.h, _p64(out))
        return out


class Evaluator:
    """The reference CPU Evaluator (crates/ckks-train-ckks/src/evaluator.rs)."""

    def __init__(self, params, relin=None, galois=None, hoist=True, bsgs=True, lazy_relin=True):
        self.params = params
        galois = galois or {}
        elts = np.asarray(sorted(galois), np.uint64)
        arr = (C.c_void_p * max(len(elts), 1))(*[galois[int(e)].h for e in elts])
        self._keep = (relin, galois)
        self.h = C.c_void_p()
        _check(lib().orc_eval_new(params.h, relin.h if relin else None, arr, _p64(elts) if len(elts) else None,
                                  len(elts), int(hoist), int(bsgs), int(lazy_relin), C.byref(self.h)))

    def __del__(self):
        try:
            lib().orc_eval_free(self.h)
        except Exception:
            pass

    def counter(self):
        out = np.zeros(7, np.uint64)
        lib().orc_eval_counter(self.h, _p64(out))
        return dict(zip(COUNTER_FIELDS, (int(x) for x in out)))

    def reset_counter(self):
        lib().orc_eval_reset_counter(self.h)

    def ct(self, data, scale):
        d = np.ascontiguousarray(data, np.uint64)
        h = C.c_void_p()
        _check(lib().orc_ct_new(self.h, d.shape[0], d.shape[1] - 1, scale, _p64(d), C.byref(h)))
        return Ct(self, h)

    def _op(self, code, a, b=None):
        h = C.c_void_p()
        _check(lib().orc_ct_op(self.h, code, a.h, b.h if b is not None else None, C.byref(h)))
        return Ct(self, h)

    def add(self, a, b):
        return self._op(0, a, b)

    def sub(self, a, b):
        return self._op(1, a, b)

    def negate(self, a):
        return self._op(2, a)

    def mul_no_relin(self, a, b):
        return self._op(3, a, b)

    def relinearize(self, a):
        return self._op(4, a)

    def mul(self, a, b):
        return self._op(5, a, b)

    def rescale(self, a):
        return self._op(6, a)

    def conjugate(self, a):
        return self._op(7, a)

    def rotate(self, a, steps):
        h = C.c_void_p()
        _check(lib().orc_ct_rotate(self.h, a.h, steps, C.byref(h)))
        return Ct(self, h)

    def hoisted_rotate(self, a, steps):
        st = (C.c_int32 * len(steps))(*steps)
        outs = (C.c_void_p * len(steps))()
        _check(lib().orc_ct_hoisted_rotate(self.h, a.h, st, len(steps), outs))
        return [Ct(self, C.c_void_p(o)) for o in outs]

    def mod_switch_to_level(self, a, level):
        h = C.c_void_p()
        _check(lib().orc_ct_mod_switch(self.h, a.h, level, C.byref(h)))
        return Ct(self, h)

    def relabel(self, a, scale):
        h = C.c_void_p()
        _check(lib().orc_ct_relabel(self.h, a.h, scale, C.byref(h)))
        return Ct(self, h)

    def mul_scalar(self, a, value, target):
        h = C.c_void_p()
        _check(lib().orc_ct_mul_scalar(self.h, a.h, value, target, C.byref(h)))
        return Ct(self, h)

    def _plain(self, op, a, pt, pt_scale, target=0.0):
        p = np.ascontiguousarray(pt, np.uint64)
        h = C.c_void_p()
        _check(lib().orc_ct_plain_op(self.h, op, a.h, _p64(p), p.shape[0] - 1, pt_scale, target, C.byref(h)))
        return Ct(self, h)

    def add_plain(self, a, pt, pt_scale):
        return self._plain(0, a, pt, pt_scale)

    def mul_plain(self, a, pt, pt_scale):
        return self._plain(1, a, pt, pt_scale)

    def mul_plain_to_scale(self, a, pt, pt_scale, target):
        return self._plain(2, a, pt, pt_scale, target)

    def exact_product_scale(self, level, target):
        err = C.c_int()
        v = lib().orc_exact_product_scale(self.h, level, target, C.byref(err))
        _check(err.value)
        return v

    def matvec_plain(self, d, stride, pts, pt_scale, x):
        p = np.ascontiguousarray(pts, np.uint64)
        h = C.c_void_p()
        _check(lib().orc_matvec_plain(self.h, d, stride, _p64(p), p.shape[1] - 1, pt_scale, x.h, C.byref(h)))
        return Ct(self, h)

    def matvec_enc(self, d, stride, cts, x):
        arr = (C.c_void_p * len(cts))(*[c.h for c in cts])
        h = C.c_void_p()
        _check(lib().orc_matvec_enc(self.h, d, stride, arr, x.h, C.byref(h)))
        return Ct(self, h)


# ---- bootstrapping (oracle_boot.inc) ----------------------------------------------------

def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Encoder:
    """The reference Encoder (crates/ckks-train-ckks/src/encoder.rs)."""

    def __init__(self, params):
        self.params = params
        self.h = C.c_void_p()
        _check(lib().orc_encoder_new(params.h, C.byref(self.h)))

    def __del__(self):
        try:
            lib().orc_encoder_free(self.h)
        except Exception:
            pass

    def encode(self, values, scale, level):
        """values: complex (or real) array of at most `slots` entries -> (level+1, N) NTT form."""
        z = np.asarray(values, np.complex128)
        flat = np.ascontiguousarray(np.stack([z.real, z.imag], axis=-1).reshape(-1), np.float64)
        out = np.zeros((level + 1, self.params.n), np.uint64)
        _check(lib().orc_encode_complex(self.h, _dp(flat), len(z), scale, level, _p64(out)))
        return out

    def decode(self, pt, scale):
        p = np.ascontiguousarray(pt, np.uint64)
        out = np.zeros(2 * (self.params.n // 2), np.float64)
        _check(lib().orc_decode_complex(self.h, _p64(p), p.shape[0] - 1, scale, _dp(out)))
        return out[0::2] + 1j * out[1::2]


def encrypt_sk(ev, kg, seed, pt, scale):
    """Symmetric encryption of the NTT-form plaintext `pt` under kg's secret (encrypt.rs)."""
    if isinstance(seed, int):
        seed = bytes([seed]) * 32
    p = np.ascontiguousarray(pt, np.uint64)
    h = C.c_void_p()
    _check(lib().orc_encrypt_sk(kg.h, seed, _p64(p), p.shape[0] - 1, scale, C.byref(h)))
    return Ct(ev, h)


class Rng:
    """One `Rng::from_seed([seed; 32])` stream (crates/ckks-train-core/src/sampler.rs:35-37) that
    successive calls consume in turn, as the reference's tests pass one `&mut Rng` first to
    the input sampler and then to the encryptor."""

    def __init__(self, seed):
        if isinstance(seed, int):
            seed = bytes([seed]) * 32
        self.h = C.c_void_p()
        _check(lib().orc_rng_new(seed, C.byref(self.h)))

    def __del__(self):
        try:
            lib().orc_rng_free(self.h)
        except Exception:
            pass

    def next_u64(self, count):
        out = np.zeros(count, np.uint64)
        lib().orc_rng_next_u64(self.h, count, _p64(out))
        return out

    def uniform(self, count, a):
        """`a * (2 u - 1)` with `u = (next_u64() >> 11) * 2^-53`, in order: the `uniform` helper
        of the reference's bootstrap tests (bootstrap/bootstrapper.rs:446-450)."""
        u = (self.next_u64(count) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
        return a * (2.0 * u - 1.0)


class PublicKey:
    """KeyGenerator::public_key (crates/ckks-train-ckks/src/keys.rs:365-369)."""

    def __init__(self, kg):
        self.kg = kg
        self.h = C.c_void_p()
        _check(lib().orc_keygen_public(kg.h, C.byref(self.h)))

    def __del__(self):
        try:
            lib().orc_pk_free(self.h)
        except Exception:
            pass


def encrypt_pk(ev, pk, rng, pt, scale):
    """Public-key encryption of the NTT-form plaintext `pt` (crates/ckks-train-ckks/src/encrypt.rs:68-90)
    with randomness drawn from the stream `rng` (u, then e0, then e1)."""
    p = np.ascontiguousarray(pt, np.uint64)
    h = C.c_void_p()
    _check(lib().orc_encrypt_pk(pk.kg.h, pk.h, rng.h, _p64(p), p.shape[0] - 1, scale, C.byref(h)))
    return Ct(ev, h)


def encrypt_sk_stream(ev, kg, rng, pt, scale):
    """Symmetric encryption of `pt` (encrypt.rs:91-101) with randomness drawn from the stream `rng`."""
    p = np.ascontiguousarray(pt, np.uint64)
    h = C.c_void_p()
    _check(lib().orc_encrypt_sk_rng(kg.h, rng.h, _p64(p), p.shape[0] - 1, scale, C.byref(h)))
    return Ct(ev, h)


def precision_bits(expected, actual):
    """-log2 of the largest absolute error (crates/ckks-train-ckks/src/precision.rs:39-58)."""
    err = float(np.max(np.abs(np.asarray(expected) - np.asarray(actual))))
    return float("inf") if err == 0.0 else -np.log2(err)


def decrypt(kg, ct):
    """c_0 + c_1 s (+ c_2 s^2 ...) in NTT form, (level+1, N)."""
    out = np.zeros((ct.level + 1, kg.params.n), np.uint64)
    _check(lib().orc_decrypt(kg.h, ct.h, _p64(out)))
    return out


class Bootstrapper:
    """Bootstrapper::new and its pieces (crates/ckks-train-ckks/src/bootstrap/bootstrapper.rs):
    encoded CoeffToSlot / SlotToCoeff stages, Galois and SSE keys, EvalMod coefficients."""

    def __init__(self, params, kg, encoder, log_slots, ctos=4, evalmod=7, stoc=4, k_intervals=13, degree=127,
                 double_angle=0, ephemeral_hw=32):
        self.params = params
        self._keep = (kg, encoder)
        self.h = C.c_void_p()
        _check(lib().orc_boot_new(params.h, kg.h, encoder.h, log_slots, ctos, evalmod, stoc, k_intervals, degree,
                                  double_angle, -1 if ephemeral_hw is None else ephemeral_hw, C.byref(self.h)))

    def __del__(self):
        try:
            lib().orc_boot_free(self.h)
        except Exception:
            pass

    def output_level(self):
        return lib().orc_boot_output_level(self.h)

    def scales(self):
        a, b = C.c_double(), C.c_double()
        lib().orc_boot_scales(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def coeffs(self):
        n = lib().orc_boot_coeffs(self.h, None)
        out = np.zeros(n, np.float64)
        lib().orc_boot_coeffs(self.h, _dp(out))
        return out

    def stages(self, direction):
        """[(info dict, entries, second entries)] with entries a list of (level+1, N) arrays
        or None for skipped all-zero diagonals; direction 0 = CoeffToSlot, 1 = SlotToCoeff."""
        out = []
        n = self.params.n
        for k in range(lib().orc_boot_num_stages(self.h, direction)):
            info = np.zeros(4, np.uint64)
            off = C.c_int64()
            sc = np.zeros(2, np.float64)
            lib().orc_boot_stage_info(self.h, direction, k, _p64(info), C.byref(off), _dp(sc))
            level, d, stride, has2 = (int(x) for x in info)

            def entries(second):
                es = []
                for i in range(d):
                    buf = np.zeros((level + 1, n), np.uint64)
                    es.append(buf if lib().orc_boot_stage_entry(self.h, direction, k, second, i, _p64(buf)) else None)
                return es

            out.append((dict(level=level, d=d, stride=stride, offset=off.value, scale=float(sc[0]),
                             pt_scale=float(sc[1]), direction=direction), entries(0), entries(1) if has2 else None))
        return out

    def galois_keys(self):
        keys = {}
        for i in range(lib().orc_boot_num_galois(self.h)):
            e = C.c_uint64()
            h = C.c_void_p()
            lib().orc_boot_galois(self.h, i, C.byref(e), C.byref(h))
            keys[e.value] = Key(self.params, h)
        return keys

    def rotation_steps(self):
        n = lib().orc_boot_num_steps(self.h, None)
        out = (C.c_int32 * max(n, 1))()
        lib().orc_boot_num_steps(self.h, out)
        return list(out[:n])

    def sse_keys(self):
        a, b = C.c_void_p(), C.c_void_p()
        _check(lib().orc_boot_sse(self.h, C.byref(a), C.byref(b)))
        return Key(self.params, a), Key(self.params, b)

    def inner_evaluator(self, relin):
        ev = Evaluator.__new__(Evaluator)
        ev.params = self.params
        ev._keep = (relin, self)
        ev.h = C.c_void_p()
        _check(lib().orc_boot_eval(self.h, relin.h if relin else None, C.byref(ev.h)))
        return ev

    def _one(self, fn, ev, *args):
        h = C.c_void_p()
        _check(fn(self.h, ev.h, *args, C.byref(h)))
        return Ct(ev, h)

    def bootstrap(self, ev, ct):
        return self._one(lib().orc_bootstrap, ev, ct.h)

    def mod_raise(self, inner, ct):
        return self._one(lib().orc_boot_mod_raise, inner, ct.h)

    def coeff_to_slot(self, inner, ct):
        a, b = C.c_void_p(), C.c_void_p()
        _check(lib().orc_boot_coeff_to_slot(self.h, inner.h, ct.h, C.byref(a), C.byref(b)))
        return Ct(inner, a), Ct(inner, b)

    def eval_mod(self, inner, ct):
        return self._one(lib().orc_boot_eval_mod, inner, ct.h)

    def slot_to_coeff(self, inner, re, im):
        return self._one(lib().orc_boot_slot_to_coeff, inner, re.h, im.h)


def eval_chebyshev(ev, ct, coeffs, a, b, target):
    c = np.ascontiguousarray(coeffs, np.float64)
    h = C.c_void_p()
    _check(lib().orc_eval_chebyshev(ev.h, ct.h, _dp(c), len(c), a, b, target, C.byref(h)))
    return Ct(ev, h)


def boot_mul_const(ev, ct, value, scale):
    h = C.c_void_p()
    _check(lib().orc_boot_mul_const(ev.h, ct.h, value, scale, C.byref(h)))
    return Ct(ev, h)


def boot_add_const(ev, ct, value):
    h = C.c_void_p()
    _check(lib().orc_boot_add_const(ev.h, ct.h, value, C.byref(h)))
    return Ct(ev, h)


def mul_by_x_half(ev, ct):
    h = C.c_void_p()
    _check(lib().orc_mul_by_x_half(ev.h, ct.h, C.byref(h)))
    return Ct(ev, h)


def boot_plan(log_slots, ctos_levels, stoc_levels, k_intervals, direction):
    """[(d, stride, offset, kept, kept_second or None)] per stage (no keys, no encoding)."""
    out = []
    k = 0
    while True:
        info = (C.c_int64 * 5)()
        _check(lib().orc_boot_plan(log_slots, ctos_levels, stoc_levels, k_intervals, direction, k, info, None))
        d = info[0]
        kept = (C.c_uint8 * (2 * d))()
        _check(lib().orc_boot_plan(log_slots, ctos_levels, stoc_levels, k_intervals, direction, k, info, kept))
        out.append((d, info[1], info[2], [bool(x) for x in kept[:d]], [bool(x) for x in kept[d:]] if info[3] else None))
        k += 1
        if k >= info[4]:
            return out
