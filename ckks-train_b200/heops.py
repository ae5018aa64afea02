"""Python mirror of the reference's ``HeOps`` evaluator interface over ``libckg.so``.

The names, argument meanings and errors follow ``crates/ckks-train-ckks/src/ops.rs:198-356``
(``HeOps``) and the CPU ``Evaluator`` it documents (``crates/ckks-train-ckks/src/evaluator.rs``):
every method returns a new ciphertext, failures raise the ``HekitError`` kind the
reference returns, and the ``OpCounter`` is kept exactly. All arithmetic runs in the
sm_100a kernels of the C ABI (``include/ckg.h``); there is no CPU fallback: loading fails
loudly when the library is missing.
"""

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libckg.so")

U64P = C.POINTER(C.c_uint64)
U32P = C.POINTER(C.c_uint32)
I32P = C.POINTER(C.c_int32)
VP = C.c_void_p

HOIST, BSGS, LAZY_RELIN = 1, 2, 4


# ---- errors (crates/ckks-train-core/src/error.rs:7-21) ---------------------------------

class HekitError(Exception):
    code = -1


class InvalidParams(HekitError):
    code = 1


class ScaleMismatch(HekitError):
    code = 2


class LevelMismatch(HekitError):
    code = 3


class NoLevelsLeft(HekitError):
    code = 4


class Decode(HekitError):
    code = 5


class Device(HekitError):
    code = 6


class OutOfMemory(Device):
    code = 7


class Timeout(Device):
    code = 8


class Cancelled(HekitError):
    """A served request was cancelled before it was admitted (no reference counterpart)."""
    code = 9


_ERRORS = {c.code: c for c in (InvalidParams, ScaleMismatch, LevelMismatch, NoLevelsLeft, Decode, Device,
                               OutOfMemory, Timeout, Cancelled)}

_lib = None


def build():
    """Compiles libckg.so for sm_100a (nvcc, in-tree)."""
    subprocess.run(["make", "-s", "-j8", "-C", os.path.join(_HERE, "csrc")], check=True)


def lib():
    """The loaded C ABI. Raises if libckg.so has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with ckks_train_b200.build() (no CPU fallback)")
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    L.ckg_last_error.restype = C.c_char_p
    L.ckg_abi_version.restype = C.c_uint32
    L.ckg_launch_count.restype = C.c_uint64
    L.ckg_primes_for_bits.argtypes = [C.c_uint32, U32P, C.c_uint32, U32P, C.c_uint32, U64P, U64P]
    L.ckg_ctx_create.argtypes = [C.c_uint32, U64P, C.c_uint32, U64P, C.c_uint32, C.c_uint32, C.c_int, VP,
                                 C.POINTER(VP)]
    L.ckg_ctx_destroy.argtypes = [VP]
    L.ckg_ctx_sync.argtypes = [VP]
    L.ckg_ctx_stream.argtypes = [VP]
    L.ckg_ctx_stream.restype = VP
    L.ckg_ntt.argtypes = [VP, VP, VP, U32P, C.c_uint32, C.c_int]
    L.ckg_poly_binary.argtypes = [VP, C.c_int, VP, VP, VP, C.c_uint32, C.c_uint32]
    L.ckg_poly_negate.argtypes = [VP, VP, VP, C.c_uint32, C.c_uint32]
    L.ckg_poly_mul_scalar.argtypes = [VP, VP, C.c_uint64, VP, C.c_uint32, C.c_uint32]
    L.ckg_automorphism.argtypes = [VP, VP, VP, C.c_uint32, C.c_uint64]
    L.ckg_rescale.argtypes = [VP, VP, C.c_uint32, VP]
    L.ckg_mod_up.argtypes = [VP, VP, C.c_uint32, C.c_uint32, VP, VP]
    L.ckg_mod_down.argtypes = [VP, VP, C.c_uint32, VP, VP]
    L.ckg_key_upload.argtypes = [VP, U64P, C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(VP)]
    L.ckg_key_upload_device.argtypes = [VP, VP, C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(VP)]
    L.ckg_key_free.argtypes = [VP]
    L.ckg_key_bytes.argtypes = [VP]
    L.ckg_key_bytes.restype = C.c_uint64
    L.ckg_key_switch.argtypes = [VP, VP, VP, C.c_uint32, VP, VP]
    L.ckg_key_switch_noalloc.argtypes = [VP, VP, VP, C.c_uint32, VP, VP]
    L.ckg_eval_create.argtypes = [VP, VP, C.POINTER(VP), C.c_uint32, C.c_uint32, C.POINTER(VP)]
    L.ckg_eval_destroy.argtypes = [VP]
    L.ckg_eval_fork.argtypes = [VP, C.POINTER(VP)]
    L.ckg_eval_config.argtypes = [VP]
    L.ckg_eval_config.restype = C.c_uint32
    L.ckg_eval_counter.argtypes = [VP, U64P]
    L.ckg_eval_reset_counter.argtypes = [VP]
    L.ckg_eval_add_counts.argtypes = [VP, U64P]
    L.ckg_eval_has_relin_key.argtypes = [VP]
    L.ckg_eval_has_galois_key.argtypes = [VP, C.c_int32]
    L.ckg_ct_upload.argtypes = [VP, U64P, C.c_uint32, C.c_uint32, C.c_double, C.POINTER(VP)]
    L.ckg_ct_upload_device.argtypes = [VP, VP, C.c_uint32, C.c_uint32, C.c_double, C.POINTER(VP)]
    L.ckg_ct_download.argtypes = [VP, U64P]
    L.ckg_ct_download_device.argtypes = [VP, VP]
    L.ckg_ct_download_async.argtypes = [VP, VP]
    L.ckg_ct_info.argtypes = [VP, U32P, U32P, C.POINTER(C.c_double)]
    L.ckg_ct_clone.argtypes = [VP]
    L.ckg_ct_clone.restype = VP
    L.ckg_ct_free.argtypes = [VP]
    L.ckg_eval_owns.argtypes = [VP, VP]
    L.ckg_pt_upload.argtypes = [VP, U64P, C.c_uint32, C.c_double, C.POINTER(VP)]
    L.ckg_pt_upload_device.argtypes = [VP, VP, C.c_uint32, C.c_double, C.POINTER(VP)]
    L.ckg_pt_clone.argtypes = [VP]
    L.ckg_pt_clone.restype = VP
    L.ckg_pt_free.argtypes = [VP]
    for name in ("ckg_add", "ckg_sub", "ckg_mul_no_relin", "ckg_mul"):
        getattr(L, name).argtypes = [VP, VP, VP, C.POINTER(VP)]
    for name in ("ckg_negate", "ckg_relinearize", "ckg_rescale_ct", "ckg_conjugate"):
        getattr(L, name).argtypes = [VP, VP, C.POINTER(VP)]
    L.ckg_add_plain.argtypes = [VP, VP, VP, C.POINTER(VP)]
    L.ckg_mul_plain.argtypes = [VP, VP, VP, C.POINTER(VP)]
    L.ckg_mul_scalar.argtypes = [VP, VP, C.c_double, C.c_double, C.POINTER(VP)]
    L.ckg_mul_plain_to_scale.argtypes = [VP, VP, VP, C.c_double, C.POINTER(VP)]
    L.ckg_mod_switch_to_level.argtypes = [VP, VP, C.c_uint32, C.POINTER(VP)]
    L.ckg_relabel.argtypes = [VP, VP, C.c_double, C.POINTER(VP)]
    L.ckg_rotate.argtypes = [VP, VP, C.c_int32, C.POINTER(VP)]
    L.ckg_hoisted_rotate.argtypes = [VP, VP, I32P, C.c_uint32, C.POINTER(VP)]
    L.ckg_exact_product_scale.argtypes = [VP, C.c_uint32, C.c_double, C.POINTER(C.c_double)]
    L.ckg_matvec_plain.argtypes = [VP, C.c_uint32, C.c_uint32, C.POINTER(VP), VP, C.POINTER(VP)]
    L.ckg_matvec_enc.argtypes = [VP, C.c_uint32, C.c_uint32, C.POINTER(VP), VP, C.POINTER(VP)]
    for name in ("ckg_matvec_enc_batch", "ckg_matvec_plain_batch"):
        getattr(L, name).argtypes = [VP, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(VP),
                                     C.POINTER(VP), C.POINTER(VP)]
    L.ckg_batch_create.argtypes = [VP, C.POINTER(VP)]
    L.ckg_batch_destroy.argtypes = [VP]
    L.ckg_batch_mul_relin_rescale.argtypes = [VP, VP, VP, C.POINTER(VP)]
    L.ckg_batch_rotate.argtypes = [VP, VP, C.c_int32, C.POINTER(VP)]
    L.ckg_batch_mul_plain_rescale.argtypes = [VP, VP, VP, C.POINTER(VP)]
    for name in ("ckg_batch_run", "ckg_batch_capture_graph", "ckg_batch_launch_graph"):
        getattr(L, name).argtypes = [VP]
    L.ckg_batch_key_switches.argtypes = [VP]
    L.ckg_batch_key_switches.restype = C.c_uint64
    L.ckg_ctx_set_ntt_wave.argtypes = [VP, C.c_int32]
    L.ckg_ctx_ntt_wave.argtypes = [VP]
    L.ckg_ctx_ntt_wave.restype = C.c_int32
    L.ckg_ctx_set_bconv_tc.argtypes = [VP, C.c_int32]
    L.ckg_ctx_bconv_tc.argtypes = [VP]
    L.ckg_ctx_bconv_tc.restype = C.c_int32
    L.ckg_device_fault.argtypes = [VP, C.POINTER(C.c_int32)]
    L.ckg_ctx_set_ntt_tma.argtypes = [VP, C.c_int32]
    L.ckg_ctx_ntt_tma.argtypes = [VP]
    L.ckg_ctx_ntt_tma.restype = C.c_int32
    L.ckg_batch_set_chunk_items.argtypes = [VP, C.c_int32]
    L.ckg_batch_chunk_items.argtypes = [VP]
    L.ckg_batch_chunk_items.restype = C.c_int32
    L.ckg_batch_autotune.argtypes = [VP, C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_int32)]
    U8P = C.POINTER(C.c_uint8)
    L.ckg_seal_parms_id.argtypes = [C.c_uint32, U64P, C.c_uint32, U64P]
    L.ckg_seal_bytes.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
    L.ckg_seal_bytes.restype = C.c_uint64
    L.ckg_seal_encode.argtypes = [C.c_uint32, U64P, C.c_uint32, U64P, C.c_uint32, C.c_uint32, C.c_double, U8P,
                                  C.c_uint64, C.POINTER(C.c_uint64)]
    L.ckg_seal_decode.argtypes = [C.c_uint32, U64P, C.c_uint32, U64P, C.c_uint32, U8P, C.c_uint64, C.c_int, U64P,
                                  C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                  C.POINTER(C.c_double)]
    L.ckg_ct_from_seal.argtypes = [VP, U8P, C.c_uint64, C.POINTER(VP)]
    L.ckg_pt_from_seal.argtypes = [VP, U8P, C.c_uint64, C.POINTER(VP)]
    L.ckg_ct_to_seal.argtypes = [VP, U8P, C.c_uint64, C.POINTER(C.c_uint64)]
    L.ckg_pt_info.argtypes = [VP, C.POINTER(C.c_uint32), C.POINTER(C.c_double)]
    L.ckg_pt_info.restype = None
    L.ckg_ct_upload_overlap.argtypes = [VP, U64P, C.c_uint32, C.c_uint32, C.c_double, C.POINTER(VP)]
    L.ckg_pt_upload_overlap.argtypes = [VP, U64P, C.c_uint32, C.c_double, C.POINTER(VP)]
    L.ckg_ct_download_overlap.argtypes = [VP, VP]
    L.ckg_ctx_transfer_stats.argtypes = [VP, C.POINTER(C.c_uint64), C.c_uint32]
    L.ckg_ctx_trim.argtypes = [VP]
    L.ckg_debug_bounds.argtypes = [C.c_int, C.c_uint64, C.c_uint64]
    L.ckg_host_alloc.argtypes = [C.c_uint64, C.POINTER(VP)]
    L.ckg_host_free.argtypes = [VP]
    L.ckg_host_free.restype = None
    L.ckg_ct_upload_overlap_list.argtypes = [VP, C.c_uint32, C.POINTER(VP), C.POINTER(C.c_uint32),
                                             C.POINTER(C.c_uint32), C.POINTER(C.c_double), C.POINTER(VP)]
    L.ckg_pt_upload_overlap_list.argtypes = [VP, C.c_uint32, C.POINTER(VP), C.POINTER(C.c_uint32),
                                             C.POINTER(C.c_double), C.POINTER(VP)]
    L.ckg_ct_download_overlap_list.argtypes = [C.c_uint32, C.POINTER(VP), C.POINTER(VP)]
    L.ckg_ctx_join_transfers.argtypes = [VP]
    DP = C.POINTER(C.c_double)
    L.ckg_boot_mul_const.argtypes = [VP, VP, C.c_double, C.c_double, C.POINTER(VP)]
    L.ckg_boot_add_const.argtypes = [VP, VP, C.c_double, C.POINTER(VP)]
    L.ckg_boot_zero.argtypes = [VP, C.c_uint32, C.c_double, C.POINTER(VP)]
    L.ckg_boot_relabel.argtypes = [VP, VP, C.c_double, C.POINTER(VP)]
    L.ckg_mul_by_x_half.argtypes = [VP, VP, C.POINTER(VP)]
    L.ckg_mod_raise.argtypes = [VP, VP, VP, VP, C.POINTER(VP)]
    L.ckg_lt_create.argtypes = [C.c_int, C.c_uint32, C.c_double, C.c_uint32, C.c_uint32, C.c_int64, C.POINTER(VP),
                                C.POINTER(VP), C.POINTER(VP)]
    L.ckg_lt_free.argtypes = [VP]
    L.ckg_coeff_to_slot.argtypes = [VP, VP, C.POINTER(VP), C.c_uint32, C.POINTER(VP), C.POINTER(VP)]
    L.ckg_slot_to_coeff.argtypes = [VP, VP, VP, C.POINTER(VP), C.c_uint32, C.POINTER(VP)]
    L.ckg_eval_chebyshev.argtypes = [VP, VP, DP, C.c_uint32, C.c_double, C.c_double, C.c_double, C.POINTER(VP)]
    L.ckg_eval_mod.argtypes = [VP, VP, U32P, DP, C.c_uint32, C.POINTER(VP)]
    L.ckg_boot_create.argtypes = [VP, U32P, C.POINTER(VP), C.c_uint32, C.POINTER(VP), C.c_uint32, C.POINTER(VP),
                                  C.c_uint32, VP, VP, DP, C.c_uint32, DP, C.POINTER(VP)]
    L.ckg_boot_destroy.argtypes = [VP]
    L.ckg_bootstrap.argtypes = [VP, VP, VP, C.POINTER(VP)]
    L.ckg_boot_output_level.argtypes = [VP]
    L.ckg_boot_output_level.restype = C.c_uint32
    L.ckg_encode_complex.argtypes = [VP, DP, C.c_uint32, C.c_double, C.c_uint32, C.POINTER(VP)]
    L.ckg_encode_complex_host.argtypes = [C.c_uint32, U64P, C.c_uint32, DP, C.c_uint32, C.c_double, C.c_uint32, U64P]
    L.ckg_boot_rotation_steps.argtypes = [U32P, I32P, C.c_uint32, U32P]
    L.ckg_evalmod_coeffs.argtypes = [U32P, DP, C.c_uint32]
    L.ckg_boot_plan.argtypes = [U32P, C.c_int, C.c_uint32, C.POINTER(C.c_int64), C.POINTER(C.c_uint8)]
    L.ckg_boot_stage_scales.argtypes = [VP, U32P, C.c_double, DP]
    L.ckg_boot_encode_stages.argtypes = [VP, U32P, C.c_int, C.c_double, C.POINTER(VP), C.c_uint32]
    L.ckg_boot_create_encoded.argtypes = [VP, U32P, C.c_double, C.POINTER(VP), C.c_uint32, VP, VP, C.POINTER(VP)]
    L.ckg_server_create.argtypes = [VP, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(VP)]
    L.ckg_server_destroy.argtypes = [VP]
    L.ckg_server_add_owner.argtypes = [VP, U32P]
    L.ckg_server_add_key.argtypes = [VP, C.c_uint32, VP, C.c_int, C.c_uint32, C.c_uint32, C.c_uint64]
    L.ckg_server_add_sse_keys.argtypes = [VP, C.c_uint32, VP, VP, C.c_int]
    L.ckg_server_enable_bootstrap.argtypes = [VP, U32P, C.c_double]
    L.ckg_server_submit_bootstrap.argtypes = [VP, C.c_uint32, VP, U64P]
    L.ckg_server_submit_mul.argtypes = [VP, C.c_uint32, VP, VP, U64P]
    L.ckg_server_submit_rotate.argtypes = [VP, C.c_uint32, VP, C.c_int32, U64P]
    L.ckg_server_submit_mul_plain.argtypes = [VP, C.c_uint32, VP, VP, U64P]
    L.ckg_server_submit_matvec.argtypes = [VP, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(VP), VP, U64P]
    L.ckg_server_result.argtypes = [VP, C.c_uint64, C.c_int64, C.POINTER(VP), C.POINTER(C.c_double)]
    L.ckg_server_cancel.argtypes = [VP, C.c_uint64, C.POINTER(C.c_int)]
    L.ckg_server_drain.argtypes = [VP, C.c_int64]
    L.ckg_server_stats.argtypes = [VP, U64P, C.c_uint32]
    L.ckg_server_owner_counter.argtypes = [VP, C.c_uint32, U64P]
    L.ckg_server_inject_upload_failures.argtypes = [VP, C.c_uint32]


def _check(code):
    if code != 0:
        msg = lib().ckg_last_error().decode()
        raise _ERRORS.get(code, Device)(msg)


def _p64(a):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"], "expected a C-contiguous uint64 array"
    return a.ctypes.data_as(U64P)


def launch_count():
    """Kernel launches issued by libckg.so so far."""
    return lib().ckg_launch_count()


def set_bounds_checking(on):
    """Turns the library's host-side bounds checking of kernel work lists on or off (ckg_debug_bounds;
    the CKG_CHECK_BOUNDS environment variable sets the initial state). Only allocations made while
    it is on are known to it."""
    _check(lib().ckg_debug_bounds(0, 0, 1 if on else 0))


def primes_for_bits(log_n, q_bits, p_bits):
    """The data and special primes CkksParams::new hands out (params.rs:87-157)."""
    qb = (C.c_uint32 * len(q_bits))(*q_bits)
    pb = (C.c_uint32 * len(p_bits))(*p_bits)
    q = np.zeros(len(q_bits), np.uint64)
    p = np.zeros(len(p_bits), np.uint64)
    _check(lib().ckg_primes_for_bits(log_n, qb, len(q_bits), pb, len(p_bits), _p64(q), _p64(p)))
    return [int(x) for x in q], [int(x) for x in p]


class Context:
    """Parameters resident on one GPU: primes, NTT and base-conversion tables, a stream."""

    def __init__(self, log_n, q, p, dnum, device=0, stream=None, scale=None):
        self.log_n, self.n = log_n, 1 << log_n
        self.q, self.p, self.dnum = [int(x) for x in q], [int(x) for x in p], dnum
        self.alpha = len(self.q) // dnum
        self.max_level = len(self.q) - 1
        self.k = len(self.p)
        self.scale = scale
        qa, pa = np.asarray(self.q, np.uint64), np.asarray(self.p, np.uint64)
        h = VP()
        _check(lib().ckg_ctx_create(log_n, _p64(qa), len(qa), _p64(pa), len(pa), dnum, device,
                                    VP(stream) if stream else None, C.byref(h)))
        self.h = h

    @classmethod
    def from_bits(cls, log_n, q_bits, p_bits, dnum, device=0, stream=None, scale_bits=None):
        q, p = primes_for_bits(log_n, q_bits, p_bits)
        return cls(log_n, q, p, dnum, device, stream, None if scale_bits is None else float(2.0 ** scale_bits))

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().ckg_ctx_destroy(self.h)
                self.h = None
        except Exception:
            pass

    @property
    def primes(self):
        return self.q + self.p

    @property
    def stream(self):
        return lib().ckg_ctx_stream(self.h)

    def sync(self):
        _check(lib().ckg_ctx_sync(self.h))

    TRANSFER_STATS = ("upload_calls", "upload_bytes", "upload_alloc_ns", "upload_copy_ns", "upload_pool_bytes",
                      "download_calls", "download_ns", "alloc_retries", "reused_in_use")

    def trim(self):
        """Hands the device memory this context keeps cached back to the driver (ckg_ctx_trim)."""
        _check(lib().ckg_ctx_trim(self.h))

    def transfer_stats(self):
        """Host-side accounting of the overlapped transfers (include/ckg.h, ckg_ctx_transfer_stats)."""
        out = (C.c_uint64 * len(self.TRANSFER_STATS))()
        _check(lib().ckg_ctx_transfer_stats(self.h, out, len(self.TRANSFER_STATS)))
        return dict(zip(self.TRANSFER_STATS, [int(x) for x in out]))

    def join_transfers(self):
        """The context's stream waits for every overlapped transfer queued so far."""
        _check(lib().ckg_ctx_join_transfers(self.h))

    @property
    def ntt_wave(self):
        """Limbs per column + row launch pair of the batched transforms (0: all at once)."""
        return lib().ckg_ctx_ntt_wave(self.h)

    @ntt_wave.setter
    def ntt_wave(self, limbs):
        _check(lib().ckg_ctx_set_ntt_wave(self.h, int(limbs)))

    @property
    def bconv_tc(self):
        """Base conversion engine (bit-neutral): 0 integer kernels, 1 tensor cores from 6 sources
        on (the default where the context qualifies), 2 tensor cores for every source count."""
        return lib().ckg_ctx_bconv_tc(self.h)

    @bconv_tc.setter
    def bconv_tc(self, mode):
        _check(lib().ckg_ctx_set_bconv_tc(self.h, int(mode)))

    @property
    def ntt_tma(self):
        """True when NTT column passes run persistent with TMA-staged tiles (bit-neutral; off by
        default, measured slower than the per-tile passes at N = 2^16)."""
        return lib().ckg_ctx_ntt_tma(self.h) == 1

    @ntt_tma.setter
    def ntt_tma(self, on):
        _check(lib().ckg_ctx_set_ntt_tma(self.h, 1 if on else 0))

    def device_fault(self):
        """Reads and clears the device fault word (0: none)."""
        v = C.c_int32()
        _check(lib().ckg_device_fault(self.h, C.byref(v)))
        return v.value

    def digit_ranges(self, level):
        """keyswitch::digit_ranges (crates/ckks-train-ckks/src/keyswitch.rs:68-74)."""
        out = []
        for j in range(self.dnum):
            s, e = j * self.alpha, min((j + 1) * self.alpha, level + 1)
            if s > level:
                break
            out.append((s, e))
        return out

    # -- device-buffer primitives (integer device addresses) --
    def ntt(self, src, dst, primes, inverse=False):
        pr = (C.c_uint32 * len(primes))(*primes)
        _check(lib().ckg_ntt(self.h, VP(src), VP(dst), pr, len(primes), int(inverse)))

    def poly_binary(self, op, a, b, out, first_prime, nlimbs):
        _check(lib().ckg_poly_binary(self.h, op, VP(a), VP(b), VP(out), first_prime, nlimbs))

    def poly_negate(self, a, out, first_prime, nlimbs):
        _check(lib().ckg_poly_negate(self.h, VP(a), VP(out), first_prime, nlimbs))

    def poly_mul_scalar(self, a, scalar, out, first_prime, nlimbs):
        _check(lib().ckg_poly_mul_scalar(self.h, VP(a), scalar, VP(out), first_prime, nlimbs))

    def automorphism(self, src, dst, nlimbs, galois_elt):
        _check(lib().ckg_automorphism(self.h, VP(src), VP(dst), nlimbs, galois_elt))

    def rescale(self, src, level, dst):
        _check(lib().ckg_rescale(self.h, VP(src), level, VP(dst)))

    def mod_up(self, src, level, digit, out_q, out_p):
        _check(lib().ckg_mod_up(self.h, VP(src), level, digit, VP(out_q), VP(out_p)))

    def mod_down(self, q_part, level, p_part, out):
        _check(lib().ckg_mod_down(self.h, VP(q_part), level, VP(p_part), VP(out)))

    def upload_key(self, key, galois_elt=0):
        """key: uint64 array (parts, 2, q_limbs + k, N) in the reference device layout."""
        return Key(self, key, galois_elt)

    def upload_key_device(self, ptr, shape, galois_elt=0):
        """The same from a device buffer of that shape."""
        return Key(self, None, galois_elt, device_ptr=ptr, shape=shape)

    def key_switch(self, key, src, level, out_b, out_a):
        _check(lib().ckg_key_switch(self.h, key.h, VP(src), level, VP(out_b), VP(out_a)))

    def key_switch_noalloc(self, key, src, level, out_b, out_a):
        """key_switch that allocates no device memory: its working space is the library's
        fixed 128 MiB device array (for callers that cannot allocate while serving)."""
        _check(lib().ckg_key_switch_noalloc(self.h, key.h if key else None, VP(src), level, VP(out_b), VP(out_a)))


class Key:
    """A key-switching key resident in HBM (relinearization key when galois_elt is 0)."""

    def __init__(self, ctx, arr, galois_elt=0, device_ptr=None, shape=None):
        self.ctx, self.elt = ctx, galois_elt
        h = VP()
        if device_ptr is not None:
            parts, two, limbs, n = shape
            assert two == 2 and n == ctx.n and limbs > ctx.k
            _check(lib().ckg_key_upload_device(ctx.h, VP(device_ptr), parts, limbs - ctx.k, galois_elt, C.byref(h)))
        else:
            arr = np.ascontiguousarray(arr, np.uint64)
            parts, two, limbs, n = arr.shape
            assert two == 2 and n == ctx.n and limbs > ctx.k
            _check(lib().ckg_key_upload(ctx.h, _p64(arr), parts, limbs - ctx.k, galois_elt, C.byref(h)))
        self.h = h

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().ckg_key_free(self.h)
                self.h = None
        except Exception:
            pass

    @property
    def nbytes(self):
        return lib().ckg_key_bytes(self.h)


class EvalConfig:
    """The ablation flags (crates/ckks-train-ckks/src/ops.rs:111-178)."""

    def __init__(self, hoist=True, bsgs=True, lazy_relin=True):
        self.hoist, self.bsgs, self.lazy_relin = hoist, bsgs, lazy_relin

    @property
    def flags(self):
        return (HOIST if self.hoist else 0) | (BSGS if self.bsgs else 0) | (LAZY_RELIN if self.lazy_relin else 0)

    @classmethod
    def from_flags(cls, f):
        return cls(bool(f & HOIST), bool(f & BSGS), bool(f & LAZY_RELIN))

    def __eq__(self, o):
        return self.flags == o.flags

    def __repr__(self):
        return f"EvalConfig(hoist={self.hoist}, bsgs={self.bsgs}, lazy_relin={self.lazy_relin})"


COUNTER_FIELDS = ("rotations", "relins", "ct_ct_tensor", "ct_pt_mults", "rescales", "sse_switches", "bootstraps")


class Ciphertext:
    """A device ciphertext handle. Copies share the device buffer (no allocation)."""

    def __init__(self, ev, h):
        self.ev, self.h = ev, h

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().ckg_ct_free(self.h)
                self.h = None
        except Exception:
            pass

    def info(self):
        n, l, s = C.c_uint32(), C.c_uint32(), C.c_double()
        lib().ckg_ct_info(self.h, C.byref(n), C.byref(l), C.byref(s))
        return n.value, l.value, s.value

    def size(self):
        return self.info()[0]

    def level(self):
        return self.info()[1]

    def scale(self):
        return self.info()[2]

    def slots(self):
        return self.ev.ctx.n // 2

    def clone(self):
        return Ciphertext(self.ev, VP(lib().ckg_ct_clone(self.h)))

    __copy__ = clone


class Plaintext:
    def __init__(self, ev, h, level, scale):
        self.ev, self.h, self._level, self._scale = ev, h, level, scale

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().ckg_pt_free(self.h)
                self.h = None
        except Exception:
            pass

    def level(self):
        return self._level

    def scale(self):
        return self._scale

    def slots(self):
        return self.ev.ctx.n // 2


class CudaEvaluator:
    """HeOps on the GPU (crates/ckks-train-ckks/src/ops.rs:198-356)."""

    def __init__(self, ctx, relin_key=None, galois_keys=(), config=None, _handle=None):
        self.ctx = ctx
        self._keys = (relin_key, tuple(galois_keys))
        if _handle is not None:
            self.h = _handle
            return
        config = config or EvalConfig()
        gal = list(galois_keys)
        arr = (VP * max(len(gal), 1))(*[k.h for k in gal])
        h = VP()
        _check(lib().ckg_eval_create(ctx.h, relin_key.h if relin_key else None, arr, len(gal), config.flags,
                                     C.byref(h)))
        self.h = h

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().ckg_eval_destroy(self.h)
                self.h = None
        except Exception:
            pass

    # -- bookkeeping --
    def params(self):
        return self.ctx

    def config(self):
        return EvalConfig.from_flags(lib().ckg_eval_config(self.h))

    def counter(self):
        out = np.zeros(7, np.uint64)
        lib().ckg_eval_counter(self.h, _p64(out))
        return dict(zip(COUNTER_FIELDS, (int(x) for x in out)))

    def key_switches(self):
        """OpCounter::key_switches (counter.rs:76-78)."""
        c = self.counter()
        return c["rotations"] + c["relins"] + c["sse_switches"]

    def reset_counter(self):
        lib().ckg_eval_reset_counter(self.h)

    def add_counts(self, counts):
        arr = np.asarray([counts.get(f, 0) for f in COUNTER_FIELDS], np.uint64)
        lib().ckg_eval_add_counts(self.h, _p64(arr))

    def fork(self):
        h = VP()
        _check(lib().ckg_eval_fork(self.h, C.byref(h)))
        return CudaEvaluator(self.ctx, *self._keys, _handle=h)

    def has_relin_key(self):
        return bool(lib().ckg_eval_has_relin_key(self.h))

    def has_galois_key(self, step):
        return bool(lib().ckg_eval_has_galois_key(self.h, step))

    def owns(self, ct):
        return bool(lib().ckg_eval_owns(self.h, ct.h))

    # -- transfers --
    def upload_ct(self, data, scale):
        """data: uint64 (ncomp, level+1, N), NTT form, reduced."""
        d = np.ascontiguousarray(data, np.uint64)
        h = VP()
        _check(lib().ckg_ct_upload(self.h, _p64(d), d.shape[0], d.shape[1] - 1, scale, C.byref(h)))
        return Ciphertext(self, h)

    upload_ct_owned = upload_ct

    def upload_ct_device(self, ptr, ncomp, level, scale):
        h = VP()
        _check(lib().ckg_ct_upload_device(self.h, VP(ptr), ncomp, level, scale, C.byref(h)))
        return Ciphertext(self, h)

    def download_ct(self, ct):
        n, l, s = ct.info()
        out = np.zeros((n, l + 1, self.ctx.n), np.uint64)
        _check(lib().ckg_ct_download(ct.h, _p64(out)))
        return out, s

    def download_ct_device(self, ct, ptr):
        _check(lib().ckg_ct_download_device(ct.h, VP(ptr)))

    def upload_ct_host_ptr(self, ptr, ncomp, level, scale):
        """upload_ct from a raw host address (pinned memory makes the copy asynchronous)."""
        h = VP()
        _check(lib().ckg_ct_upload(self.h, C.cast(VP(ptr), U64P), ncomp, level, scale, C.byref(h)))
        return Ciphertext(self, h)

    def upload_pt_host_ptr(self, ptr, level, scale):
        """upload_pt from a raw host address."""
        h = VP()
        _check(lib().ckg_pt_upload(self.h, C.cast(VP(ptr), U64P), level, scale, C.byref(h)))
        return Plaintext(self, h, level, scale)

    def upload_ct_overlap(self, ptr, ncomp, level, scale):
        """upload_ct from a pinned host address on the context's upload stream (include/ckg.h,
        "overlapped host transfers")."""
        h = VP()
        _check(lib().ckg_ct_upload_overlap(self.h, C.cast(VP(ptr), U64P), ncomp, level, scale, C.byref(h)))
        return Ciphertext(self, h)

    def upload_pt_overlap(self, ptr, level, scale):
        h = VP()
        _check(lib().ckg_pt_upload_overlap(self.h, C.cast(VP(ptr), U64P), level, scale, C.byref(h)))
        return Plaintext(self, h, level, scale)

    def download_ct_overlap(self, ct, ptr):
        """Queues the copy of `ct` to the pinned host address `ptr` on the download stream;
        complete after ctx.sync()."""
        _check(lib().ckg_ct_download_overlap(ct.h, VP(ptr)))

    def upload_ct_overlap_list(self, items):
        """upload_ct_overlap of every (ptr, ncomp, level, scale) in `items` in one call (one device
        allocation, one stream dependency)."""
        n = len(items)
        hosts = (VP * n)(*[VP(p) for p, _, _, _ in items])
        out = (VP * n)()
        _check(lib().ckg_ct_upload_overlap_list(self.h, n, hosts, (C.c_uint32 * n)(*[c for _, c, _, _ in items]),
                                                (C.c_uint32 * n)(*[lv for _, _, lv, _ in items]),
                                                (C.c_double * n)(*[sc for _, _, _, sc in items]), out))
        return [Ciphertext(self, VP(h)) for h in out]

    def upload_pt_overlap_list(self, items):
        """upload_pt_overlap of every (ptr, level, scale) in `items` in one call."""
        n = len(items)
        hosts = (VP * n)(*[VP(p) for p, _, _ in items])
        out = (VP * n)()
        _check(lib().ckg_pt_upload_overlap_list(self.h, n, hosts, (C.c_uint32 * n)(*[lv for _, lv, _ in items]),
                                                (C.c_double * n)(*[sc for _, _, sc in items]), out))
        return [Plaintext(self, VP(h), lv, sc) for h, (_, lv, sc) in zip(out, items)]

    def download_ct_overlap_list(self, cts, ptrs):
        """download_ct_overlap of every ciphertext in `cts` to the matching pinned host address."""
        n = len(cts)
        _check(lib().ckg_ct_download_overlap_list(n, (VP * n)(*[c.h for c in cts]),
                                                  (VP * n)(*[VP(p) for p in ptrs])))

    def download_ct_async(self, ct, ptr):
        """Queues the copy of `ct` to the host address `ptr`; complete after ctx.sync()."""
        _check(lib().ckg_ct_download_async(ct.h, VP(ptr)))

    def upload_pt(self, data, scale):
        d = np.ascontiguousarray(data, np.uint64)
        h = VP()
        _check(lib().ckg_pt_upload(self.h, _p64(d), d.shape[0] - 1, scale, C.byref(h)))
        return Plaintext(self, h, d.shape[0] - 1, scale)

    upload_pt_owned = upload_pt

    def ct_from_seal(self, data):
        """Parse SEAL 4.1 ciphertext bytes and upload them (load_ciphertext)."""
        buf, bp = _u8(data)
        return self._ct(lib().ckg_ct_from_seal, bp, len(buf))

    def pt_from_seal(self, data):
        """Parse SEAL 4.1 plaintext bytes and upload them (load_plaintext)."""
        buf, bp = _u8(data)
        h = VP()
        _check(lib().ckg_pt_from_seal(self.h, bp, len(buf), C.byref(h)))
        lv, sc = C.c_uint32(), C.c_double()
        lib().ckg_pt_info(h, C.byref(lv), C.byref(sc))
        return Plaintext(self, h, lv.value, sc.value)

    def ct_to_seal(self, ct):
        """SEAL 4.1 bytes of a device ciphertext (save_ciphertext)."""
        n, l, _ = ct.info()
        size = lib().ckg_seal_bytes(self.ctx.log_n, n, l)
        out = np.zeros(size, np.uint8)
        ln = C.c_uint64()
        _check(lib().ckg_ct_to_seal(ct.h, out.ctypes.data_as(C.POINTER(C.c_uint8)), size, C.byref(ln)))
        return out.tobytes()

    def upload_pt_device(self, ptr, level, scale):
        h = VP()
        _check(lib().ckg_pt_upload_device(self.h, VP(ptr), level, scale, C.byref(h)))
        return Plaintext(self, h, level, scale)

    # -- arithmetic --
    def _ct(self, fn, *args):
        h = VP()
        _check(fn(self.h, *args, C.byref(h)))
        return Ciphertext(self, h)

    def add(self, a, b):
        return self._ct(lib().ckg_add, a.h, b.h)

    def sub(self, a, b):
        return self._ct(lib().ckg_sub, a.h, b.h)

    def negate(self, a):
        return self._ct(lib().ckg_negate, a.h)

    def add_plain(self, a, p):
        return self._ct(lib().ckg_add_plain, a.h, p.h)

    def mul_plain(self, a, p):
        return self._ct(lib().ckg_mul_plain, a.h, p.h)

    def mul_scalar(self, ct, value, target_scale):
        return self._ct(lib().ckg_mul_scalar, ct.h, value, target_scale)

    def mul_plain_to_scale(self, a, p, target_scale):
        return self._ct(lib().ckg_mul_plain_to_scale, a.h, p.h, target_scale)

    def mul_no_relin(self, a, b):
        return self._ct(lib().ckg_mul_no_relin, a.h, b.h)

    def relinearize(self, ct):
        return self._ct(lib().ckg_relinearize, ct.h)

    def mul(self, a, b):
        return self._ct(lib().ckg_mul, a.h, b.h)

    def rescale(self, ct):
        return self._ct(lib().ckg_rescale_ct, ct.h)

    def mod_switch_to_level(self, ct, level):
        return self._ct(lib().ckg_mod_switch_to_level, ct.h, level)

    def relabel(self, ct, scale):
        return self._ct(lib().ckg_relabel, ct.h, scale)

    def rotate(self, ct, steps):
        return self._ct(lib().ckg_rotate, ct.h, steps)

    def conjugate(self, ct):
        return self._ct(lib().ckg_conjugate, ct.h)

    def hoisted_rotate(self, ct, steps):
        st = (C.c_int32 * max(len(steps), 1))(*steps)
        outs = (VP * max(len(steps), 1))()
        _check(lib().ckg_hoisted_rotate(self.h, ct.h, st, len(steps), outs))
        return [Ciphertext(self, VP(outs[i])) for i in range(len(steps))]

    def rotate_many(self, items):
        """rotate(ct, steps) for independent (ct, steps) pairs, as one batched launch sequence
        (results and OpCounter those of the single calls)."""
        if len(items) < 2:
            return [self.rotate(c, s) for c, s in items]
        b = Batch(self)
        outs = [b.rotate(c, s) for c, s in items]
        b.run()
        return outs

    def mul_rescale_many(self, pairs):
        """rescale(mul(a, b)) for independent pairs, as one batched launch sequence."""
        if len(pairs) < 2:
            return [self.rescale(self.mul(a, b)) for a, b in pairs]
        bt = Batch(self)
        outs = [bt.mul_relin_rescale(a, b) for a, b in pairs]
        bt.run()
        return outs

    def matvec_plain(self, d, stride, entries, x):
        arr = (VP * len(entries))(*[e.h for e in entries])
        return self._ct(lib().ckg_matvec_plain, d, stride, arr, x.h)

    def matvec_enc(self, d, stride, entries, x):
        arr = (VP * len(entries))(*[e.h for e in entries])
        return self._ct(lib().ckg_matvec_enc, d, stride, arr, x.h)

    def _matvec_batch(self, fn, jobs):
        n = len(jobs)
        ds = (C.c_uint32 * max(n, 1))(*[j[0] for j in jobs])
        ss = (C.c_uint32 * max(n, 1))(*[j[1] for j in jobs])
        flat = [e for j in jobs for e in j[2]]
        es = (VP * max(len(flat), 1))(*[e.h for e in flat])
        xs = (VP * max(n, 1))(*[j[3].h for j in jobs])
        outs = (VP * max(n, 1))()
        _check(fn(self.h, n, ds, ss, es, xs, outs))
        return [Ciphertext(self, VP(outs[i])) for i in range(n)]

    def matvec_enc_batch(self, jobs):
        """CudaEvaluator::matvec_enc_batch (evaluator.rs:437-520): jobs of (d, stride, entries, x)."""
        return self._matvec_batch(lib().ckg_matvec_enc_batch, jobs)

    def matvec_plain_batch(self, jobs):
        """matvec_plain for every job of (d, stride, entries, x), batched stage by stage."""
        return self._matvec_batch(lib().ckg_matvec_plain_batch, jobs)

    # ---- bootstrapping (include/ckg.h, "bootstrapping") ----

    def boot_mul_const(self, a, value, scale):
        """Integer multiple round(value * scale / a.scale) of a, labelled `scale` (poly.rs:380-400)."""
        return self._ct(lib().ckg_boot_mul_const, a.h, value, scale)

    def boot_add_const(self, a, value):
        return self._ct(lib().ckg_boot_add_const, a.h, value)

    def boot_zero(self, level, scale):
        h = VP()
        _check(lib().ckg_boot_zero(self.h, level, scale, C.byref(h)))
        return Ciphertext(self, h)

    def boot_relabel(self, a, scale):
        return self._ct(lib().ckg_boot_relabel, a.h, scale)

    def mul_by_x_half(self, a):
        return self._ct(lib().ckg_mul_by_x_half, a.h)

    def mod_raise(self, a, to_sparse, to_dense):
        return self._ct(lib().ckg_mod_raise, a.h, to_sparse.h, to_dense.h)

    def coeff_to_slot(self, a, stages):
        arr = (VP * len(stages))(*[s.h for s in stages])
        re, im = VP(), VP()
        _check(lib().ckg_coeff_to_slot(self.h, a.h, arr, len(stages), C.byref(re), C.byref(im)))
        return Ciphertext(self, re), Ciphertext(self, im)

    def slot_to_coeff(self, re, im, stages):
        arr = (VP * len(stages))(*[s.h for s in stages])
        return self._ct(lib().ckg_slot_to_coeff, re.h, im.h, arr, len(stages))

    def eval_chebyshev(self, a, coeffs, lo=-1.0, hi=1.0, target_scale=None):
        c = np.ascontiguousarray(coeffs, np.float64)
        t = a.scale() if target_scale is None else target_scale
        return self._ct(lib().ckg_eval_chebyshev, a.h, c.ctypes.data_as(C.POINTER(C.c_double)), len(c), lo, hi, t)

    def encode(self, values, scale, level):
        """Encoder::encode_complex (encoder.rs:215-283) into a device plaintext."""
        flat = _complex_pairs(values)
        h = VP()
        _check(lib().ckg_encode_complex(self.h, flat.ctypes.data_as(C.POINTER(C.c_double)), len(flat) // 2, scale,
                                        level, C.byref(h)))
        return Plaintext(self, h, level, scale)

    def eval_mod(self, a, bp, coeffs):
        b = (C.c_uint32 * 7)(*bp.words())
        c = np.ascontiguousarray(coeffs, np.float64)
        return self._ct(lib().ckg_eval_mod, a.h, b, c.ctypes.data_as(C.POINTER(C.c_double)), len(c))

    def exact_product_scale(self, level, target_scale):
        out = C.c_double()
        _check(lib().ckg_exact_product_scale(self.h, level, target_scale, C.byref(out)))
        return out.value

    def target_plain_scale(self, ct, target_scale):
        """HeOps::target_plain_scale (ops.rs:334-338)."""
        sp = self.exact_product_scale(ct.level(), target_scale) / ct.scale()
        if sp < 1048576.0:
            raise InvalidParams("plaintext scale is below 2^20")
        return sp

    def mul_lazy(self, a, b):
        """HeOps::mul_lazy (ops.rs:340-347)."""
        return self.mul_no_relin(a, b) if self.config().lazy_relin else self.mul(a, b)

    def relin_lazy(self, s):
        """HeOps::relin_lazy (ops.rs:349-355)."""
        return self.relinearize(s) if self.config().lazy_relin else s


class Batch:
    """Many evaluator ops at uneven levels run as one launch sequence (include/ckg.h,
    "batched execution"); results are returned at enqueue and valid after run()."""

    def __init__(self, ev):
        self.ev = ev
        h = VP()
        _check(lib().ckg_batch_create(ev.h, C.byref(h)))
        self.h = h
        self._keep = []

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().ckg_batch_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def _out(self, fn, *args):
        h = VP()
        _check(fn(self.h, *args, C.byref(h)))
        return Ciphertext(self.ev, h)

    def mul_relin_rescale(self, a, b):
        self._keep += [a, b]
        return self._out(lib().ckg_batch_mul_relin_rescale, a.h, b.h)

    def rotate(self, a, steps):
        self._keep.append(a)
        return self._out(lib().ckg_batch_rotate, a.h, steps)

    def mul_plain_rescale(self, a, p):
        self._keep += [a, p]
        return self._out(lib().ckg_batch_mul_plain_rescale, a.h, p.h)

    def run(self):
        _check(lib().ckg_batch_run(self.h))

    def capture_graph(self):
        _check(lib().ckg_batch_capture_graph(self.h))

    def launch_graph(self):
        _check(lib().ckg_batch_launch_graph(self.h))

    def key_switches(self):
        return lib().ckg_batch_key_switches(self.h)

    @property
    def chunk_items(self):
        return lib().ckg_batch_chunk_items(self.h)

    @chunk_items.setter
    def chunk_items(self, items):
        _check(lib().ckg_batch_set_chunk_items(self.h, int(items)))

    def autotune(self, reps=3):
        """Times the (NTT limb wave, chunk size) grid on this batch's ops and keeps the fastest
        (include/ckg.h, "tuning"). Returns {"ntt_wave", "chunk_items", "trials": [(wave,
        chunk, ms per replay)]}."""
        buf = (C.c_int32 * 96)()
        n = C.c_int32()
        _check(lib().ckg_batch_autotune(self.h, int(reps), buf, 32, C.byref(n)))
        trials = [(buf[3 * i], buf[3 * i + 1], buf[3 * i + 2] / 1000.0) for i in range(min(n.value, 32))]
        return {"ntt_wave": self.ev.ctx.ntt_wave, "chunk_items": self.chunk_items, "trials": trials}


SERVER_STATS = ("submitted", "completed", "failed", "cancelled", "batches", "multi_owner_batches",
                "max_batch_requests", "key_hits", "key_misses", "key_evictions", "key_upload_bytes", "key_bytes",
                "peak_key_bytes", "peak_device_bytes", "budget_waits", "pending", "hbm_budget")


class PinnedBuffer:
    """Pinned host memory from the library's CUDA runtime (ckg_host_alloc), for the overlapped
    transfers; `array(dtype, shape)` views it as a numpy array. Freed when the object goes."""

    def __init__(self, nbytes):
        h = VP()
        _check(lib().ckg_host_alloc(int(nbytes), C.byref(h)))
        self.ptr, self.nbytes = h.value, int(nbytes)

    def array(self, dtype=np.int64, shape=None, offset=0):
        dt = np.dtype(dtype)
        count = (self.nbytes - offset) // dt.itemsize if shape is None else int(np.prod(shape))
        if offset + count * dt.itemsize > self.nbytes:
            raise InvalidParams("view beyond the buffer")
        buf = (C.c_char * (count * dt.itemsize)).from_address(self.ptr + offset)
        a = np.frombuffer(buf, dtype=dt, count=count)
        return a if shape is None else a.reshape(shape)

    def __del__(self):
        try:
            if getattr(self, "ptr", None):
                lib().ckg_host_free(VP(self.ptr))
                self.ptr = None
        except Exception:
            pass


SERVE_BOOT_LANE = 256  # CKG_SERVE_BOOT_LANE
SERVE_BOOT_LANES_2 = 512  # CKG_SERVE_BOOT_LANES_2
SERVE_LANES_EQUAL_PRIORITY = 1024  # CKG_SERVE_LANES_EQUAL_PRIORITY


class Server:
    """Serving loop over one context (include/ckg.h, "serving loop"): requests from many key
    owners, admitted by HBM budget with LRU key spill to pinned host memory and run with
    continuous batching. `ev` is any evaluator of the context; results are wrapped with it."""

    def __init__(self, ctx, hbm_budget, max_batch_ks=128, max_inflight=2, config=None, ev=None, boot_lanes=0,
                 boot_priority=True):
        self.ctx, self.ev = ctx, ev
        if boot_lanes not in (0, 1, 2):
            raise InvalidParams("boot_lanes must be 0, 1 or 2")
        flags = (config or EvalConfig()).flags | {0: 0, 1: SERVE_BOOT_LANE, 2: SERVE_BOOT_LANES_2}[boot_lanes]
        flags |= 0 if boot_priority else SERVE_LANES_EQUAL_PRIORITY
        h = VP()
        _check(lib().ckg_server_create(ctx.h, int(hbm_budget), max_batch_ks, max_inflight, flags, C.byref(h)))
        self.h = h
        self._keep = {}

    def close(self):
        if getattr(self, "h", None):
            lib().ckg_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_owner(self):
        o = C.c_uint32()
        _check(lib().ckg_server_add_owner(self.h, C.byref(o)))
        return o.value

    def add_key(self, owner, key, galois_elt=0):
        """key: uint64 array (parts, 2, q_limbs + k, N), the layout Context.upload_key takes."""
        key = np.ascontiguousarray(key, dtype=np.uint64)
        parts, two, limbs, n = key.shape
        assert two == 2 and n == self.ctx.n
        _check(lib().ckg_server_add_key(self.h, owner, key.ctypes.data_as(VP), 0, parts, limbs - self.ctx.k,
                                        galois_elt))

    def add_key_device(self, owner, ptr, shape, galois_elt=0):
        parts, two, limbs, n = shape
        assert two == 2 and n == self.ctx.n
        _check(lib().ckg_server_add_key(self.h, owner, VP(ptr), 1, parts, limbs - self.ctx.k, galois_elt))

    def add_sse_keys(self, owner, to_sparse, to_dense):
        """The owner's SSE keys (to_sparse (1, 2, 1 + k, N), to_dense (dnum, 2, L + 1 + k, N))."""
        a = np.ascontiguousarray(to_sparse, np.uint64)
        b = np.ascontiguousarray(to_dense, np.uint64)
        _check(lib().ckg_server_add_sse_keys(self.h, owner, a.ctypes.data_as(VP), b.ctypes.data_as(VP), 0))

    def add_sse_keys_device(self, owner, ptr_sparse, ptr_dense):
        _check(lib().ckg_server_add_sse_keys(self.h, owner, VP(ptr_sparse), VP(ptr_dense), 1))

    def enable_bootstrap(self, bp, delta):
        _check(lib().ckg_server_enable_bootstrap(self.h, _bp(bp), delta))

    def submit_bootstrap(self, owner, a):
        return self._submit(lib().ckg_server_submit_bootstrap, owner, a.h, keep=(a,))

    def _submit(self, fn, owner, *args, keep=()):
        i = C.c_uint64()
        _check(fn(self.h, owner, *args, C.byref(i)))
        self._keep[i.value] = keep
        return i.value

    def submit_mul(self, owner, a, b):
        return self._submit(lib().ckg_server_submit_mul, owner, a.h, b.h, keep=(a, b))

    def submit_rotate(self, owner, a, steps):
        return self._submit(lib().ckg_server_submit_rotate, owner, a.h, steps, keep=(a,))

    def submit_mul_plain(self, owner, a, p):
        return self._submit(lib().ckg_server_submit_mul_plain, owner, a.h, p.h, keep=(a, p))

    def submit_matvec(self, owner, d, stride, diag, x):
        arr = (VP * len(diag))(*[p.h for p in diag])
        return self._submit(lib().ckg_server_submit_matvec, owner, d, stride, arr, x.h, keep=(x, *diag))

    def result(self, rid, timeout_ms=-1):
        """(ciphertext, (submitted, admitted, completed) in microseconds); raises the op's
        error, or Timeout (the request stays pending) when timeout_ms runs out."""
        h = VP()
        t = (C.c_double * 3)()
        code = lib().ckg_server_result(self.h, rid, int(timeout_ms), C.byref(h), t)
        if code != Timeout.code:
            self._keep.pop(rid, None)
        _check(code)
        return Ciphertext(self.ev, h), (t[0], t[1], t[2])

    def result_times(self, rid, timeout_ms=-1):
        """Like result(), but also returns the status code instead of raising."""
        h = VP()
        t = (C.c_double * 3)()
        code = lib().ckg_server_result(self.h, rid, int(timeout_ms), C.byref(h), t)
        if code != Timeout.code:
            self._keep.pop(rid, None)
        ct = Ciphertext(self.ev, h) if code == 0 else None
        return code, ct, (t[0], t[1], t[2])

    def cancel(self, rid):
        c = C.c_int()
        _check(lib().ckg_server_cancel(self.h, rid, C.byref(c)))
        return bool(c.value)

    def drain(self, timeout_ms=-1):
        _check(lib().ckg_server_drain(self.h, int(timeout_ms)))

    def stats(self):
        out = np.zeros(len(SERVER_STATS), np.uint64)
        _check(lib().ckg_server_stats(self.h, _p64(out), len(SERVER_STATS)))
        return {k: int(v) for k, v in zip(SERVER_STATS, out)}

    def owner_counter(self, owner):
        out = np.zeros(7, np.uint64)
        _check(lib().ckg_server_owner_counter(self.h, owner, _p64(out)))
        return dict(zip(COUNTER_FIELDS, (int(x) for x in out)))

    def inject_upload_failures(self, count):
        _check(lib().ckg_server_inject_upload_failures(self.h, count))


class BootParams:
    """Bootstrapping parameters (crates/ckks-train-ckks/src/bootstrap/params.rs:35-66)."""

    def __init__(self, log_slots=15, ctos_levels=4, evalmod_levels=7, stoc_levels=4, k_intervals=13,
                 cheb_degree=127, double_angle=0):
        self.log_slots, self.ctos_levels, self.evalmod_levels = log_slots, ctos_levels, evalmod_levels
        self.stoc_levels, self.k_intervals = stoc_levels, k_intervals
        self.cheb_degree, self.double_angle = cheb_degree, double_angle

    def words(self):
        return (self.log_slots, self.ctos_levels, self.evalmod_levels, self.stoc_levels, self.k_intervals,
                self.cheb_degree, self.double_angle)


def _complex_pairs(values):
    z = np.asarray(values, np.complex128).reshape(-1)
    return np.ascontiguousarray(np.stack([z.real, z.imag], axis=-1).reshape(-1), np.float64)


def _bp(bp):
    return (C.c_uint32 * 7)(*bp.words())


def encode_complex_host(log_n, q, values, scale, level):
    """Host encoding over the data primes `q` (coefficient form, (level+1, 2^log_n))."""
    flat = _complex_pairs(values)
    qa = np.ascontiguousarray(q, np.uint64)
    out = np.zeros((level + 1, 1 << log_n), np.uint64)
    _check(lib().ckg_encode_complex_host(log_n, _p64(qa), len(qa), flat.ctypes.data_as(C.POINTER(C.c_double)),
                                         len(flat) // 2, scale, level, _p64(out)))
    return out


def _u8(data):
    buf = np.frombuffer(bytes(data), np.uint8)
    return buf, buf.ctypes.data_as(C.POINTER(C.c_uint8))


def seal_parms_id(log_n, moduli):
    """SEAL's parms_id of the moduli at ring degree 2^log_n (include/ckg.h, "SEAL 4.1 wire format")."""
    m = np.ascontiguousarray(moduli, np.uint64)
    out = np.zeros(4, np.uint64)
    _check(lib().ckg_seal_parms_id(log_n, _p64(m), len(m), _p64(out)))
    return [int(x) for x in out]


def seal_encode(log_n, q, words, level, scale, plaintext=False):
    """SEAL 4.1 bytes of NTT-form words over q[0..level] (ncomp x (level+1) x N for a
    ciphertext, (level+1) x N for a plaintext)."""
    qa = np.ascontiguousarray(q, np.uint64)
    w = np.ascontiguousarray(words, np.uint64)
    ncomp = 0 if plaintext else w.shape[0]
    n = C.c_uint64()
    size = lib().ckg_seal_bytes(log_n, ncomp, level)
    out = np.zeros(size, np.uint8)
    _check(lib().ckg_seal_encode(log_n, _p64(qa), len(qa), _p64(w), ncomp, level, scale,
                                 out.ctypes.data_as(C.POINTER(C.c_uint8)), size, C.byref(n)))
    return out.tobytes()


def seal_decode(log_n, q, p, data, plaintext=False):
    """Parse SEAL 4.1 bytes against the primes: (words, level, scale), words shaped like
    seal_encode's input. Raises InvalidParams for anything malformed."""
    qa, pa = np.ascontiguousarray(q, np.uint64), np.ascontiguousarray(p, np.uint64)
    buf, bp = _u8(data)
    cap = max(len(buf) // 8, 1)
    words = np.zeros(cap, np.uint64)
    nw, nc, lv, sc = C.c_uint64(), C.c_uint32(), C.c_uint32(), C.c_double()
    _check(lib().ckg_seal_decode(log_n, _p64(qa), len(qa), _p64(pa), len(pa), bp, len(buf), int(plaintext),
                                 _p64(words), cap, C.byref(nw), C.byref(nc), C.byref(lv), C.byref(sc)))
    w = words[:nw.value].reshape((-1, lv.value + 1, 1 << log_n))
    return (w[0] if plaintext else w), lv.value, sc.value


def boot_rotation_steps(bp):
    n = C.c_uint32()
    _check(lib().ckg_boot_rotation_steps(_bp(bp), None, 0, C.byref(n)))
    out = (C.c_int32 * max(n.value, 1))()
    _check(lib().ckg_boot_rotation_steps(_bp(bp), out, n.value, C.byref(n)))
    return list(out[:n.value])


def evalmod_coeffs(bp):
    out = np.zeros(bp.cheb_degree + 1, np.float64)
    _check(lib().ckg_evalmod_coeffs(_bp(bp), out.ctypes.data_as(C.POINTER(C.c_double)), len(out)))
    return out


def boot_plan(bp, direction):
    """[(d, stride, offset, kept, kept_second or None)] for each stage of a direction."""
    out = []
    k = 0
    while True:
        info = (C.c_int64 * 5)()
        _check(lib().ckg_boot_plan(_bp(bp), direction, k, info, None))
        d = info[0]
        kept = (C.c_uint8 * (2 * d))()
        _check(lib().ckg_boot_plan(_bp(bp), direction, k, info, kept))
        out.append((d, info[1], info[2], [bool(x) for x in kept[:d]], [bool(x) for x in kept[d:]] if info[3] else None))
        k += 1
        if k >= info[4]:
            return out


def boot_encode_stages(ev, bp, direction, delta):
    n = bp.ctos_levels if direction == 0 else bp.stoc_levels
    arr = (VP * n)()
    _check(lib().ckg_boot_encode_stages(ev.h, _bp(bp), direction, delta, arr, n))
    stages = []
    for i in range(n):
        lt = LinearTransform.__new__(LinearTransform)
        lt.h, lt._keep, lt.direction = VP(arr[i]), (), direction
        stages.append(lt)
    return stages


class LinearTransform:
    """One CoeffToSlot (direction 0) or SlotToCoeff (1) stage of encoded diagonals
    (bootstrap/linear.rs:482-497); entries / second: d Plaintexts or None (zero diagonal)."""

    def __init__(self, direction, level, scale, d, stride, offset, entries, second=None):
        self._keep = (list(entries), list(second or []))
        arr = (VP * d)(*[e.h if e is not None else None for e in entries])
        arr2 = (VP * d)(*[e.h if e is not None else None for e in second]) if second is not None else None
        self.h = VP()
        _check(lib().ckg_lt_create(direction, level, scale, d, stride, offset, arr, arr2, C.byref(self.h)))
        self.direction, self.level, self.scale = direction, level, scale

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().ckg_lt_free(self.h)
                self.h = None
        except Exception:
            pass


class Bootstrapper:
    """The device bootstrap (bootstrap/bootstrapper.rs:385-473) over encoded stages, the
    Galois keys of the stages plus the conjugation key, optional SSE keys and the EvalMod
    series; scales = (evalmod_scale, stoc_input_scale, delta)."""

    def __init__(self, ctx, bp, ctos, stoc, galois_keys, to_sparse, to_dense, coeffs, scales):
        self.ctx, self.bp = ctx, bp
        self._keep = (list(ctos), list(stoc), list(galois_keys), to_sparse, to_dense)
        b = (C.c_uint32 * 7)(*bp.words())
        a1 = (VP * len(ctos))(*[s.h for s in ctos])
        a2 = (VP * len(stoc))(*[s.h for s in stoc])
        g = (VP * max(len(galois_keys), 1))(*[k.h for k in galois_keys])
        c = np.ascontiguousarray(coeffs, np.float64)
        sc = (C.c_double * 3)(*scales)
        self.h = VP()
        _check(lib().ckg_boot_create(ctx.h, b, a1, len(ctos), a2, len(stoc), g, len(galois_keys),
                                     to_sparse.h if to_sparse else None, to_dense.h if to_dense else None,
                                     c.ctypes.data_as(C.POINTER(C.c_double)), len(c), sc, C.byref(self.h)))

    @classmethod
    def encoded(cls, ev, bp, delta, galois_keys, to_sparse=None, to_dense=None):
        """Stages and EvalMod series encoded by the library itself (ckg_boot_create_encoded)."""
        self = cls.__new__(cls)
        self.ctx, self.bp = ev.ctx, bp
        self._keep = (list(galois_keys), to_sparse, to_dense)
        g = (VP * max(len(galois_keys), 1))(*[k.h for k in galois_keys])
        self.h = VP()
        _check(lib().ckg_boot_create_encoded(ev.h, _bp(bp), delta, g, len(galois_keys),
                                             to_sparse.h if to_sparse else None, to_dense.h if to_dense else None,
                                             C.byref(self.h)))
        return self

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().ckg_boot_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def output_level(self):
        return lib().ckg_boot_output_level(self.h)

    def bootstrap(self, ev, ct):
        h = VP()
        _check(lib().ckg_bootstrap(self.h, ev.h, ct.h, C.byref(h)))
        return Ciphertext(ev, h)
