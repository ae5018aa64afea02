"""TEST AND BASELINE INFRASTRUCTURE ONLY: ctypes binding of oracle/_ref/libref_gpu.so, the
reference's own CUDA kernels (crates/ckks-train-cuda/kernels) driven through the launch sequences
of its Rust host code (oracle/ref_gpu/ref_ks.cu). Used by the GPU tests (its key switch against
the library's and the oracle's) and by bench.py's reference arm (the reference's GPU key switch
timed on the same device). Built by oracle/ref_gpu/Makefile where the reference tree is present;
the built library travels with the repository snapshot.
"""

import ctypes as C
import os

_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libref_gpu.so")
_lib = None


def available():
    return os.path.exists(_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(_PATH)
        vp, u64p, u32p = C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)
        L.ref_last_error.restype = C.c_char_p
        L.ref_ctx_create.argtypes = [C.c_uint32, u64p, C.c_uint32, u64p, C.c_uint32, C.c_uint32, C.POINTER(vp)]
        L.ref_ctx_destroy.argtypes = [vp]
        L.ref_ctx_stream.argtypes = [vp]
        L.ref_ctx_stream.restype = vp
        L.ref_ntt.argtypes = [vp, vp, u32p, C.c_uint32, C.c_int]
        L.ref_key_switch.argtypes = [vp, vp, C.c_uint32, vp, C.c_uint32, vp, vp]
        L.ref_sync.argtypes = [vp]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().ref_last_error().decode())


class RefGpu:
    """The reference's device tables for primes q (data) and p (special) at N = 2^log_n."""

    def __init__(self, log_n, q, p, dnum):
        qa = (C.c_uint64 * len(q))(*[int(x) for x in q])
        pa = (C.c_uint64 * len(p))(*[int(x) for x in p])
        self.h = C.c_void_p()
        _check(lib().ref_ctx_create(log_n, qa, len(q), pa, len(p), dnum, C.byref(self.h)))
        self.nq = len(q)

    def __del__(self):
        try:
            lib().ref_ctx_destroy(self.h)
        except Exception:
            pass

    @property
    def stream(self):
        return lib().ref_ctx_stream(self.h)

    def ntt(self, buf_ptr, primes, inverse):
        arr = (C.c_uint32 * len(primes))(*primes)
        _check(lib().ref_ntt(self.h, buf_ptr, arr, len(primes), int(inverse)))

    def key_switch(self, in_ptr, level, key_ptr, out_b_ptr, out_a_ptr):
        """Ks::key_switch of a level-`level` NTT-form polynomial with a full key (L + 1 data limbs)."""
        _check(lib().ref_key_switch(self.h, in_ptr, level, key_ptr, self.nq, out_b_ptr, out_a_ptr))

    def sync(self):
        _check(lib().ref_sync(self.h))
