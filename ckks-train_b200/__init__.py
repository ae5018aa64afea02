"""B200-native RNS-CKKS evaluator path (sm_100a kernels behind a C ABI, include/ckg.h).

This directory is imported under the module name ``ckks_train_b200`` (its name has a
hyphen, so loaders register it by path; see ``load_package`` in bench.py).
"""

from .heops import (  # noqa: F401
    BSGS,
    Batch,
    BootParams,
    Bootstrapper,
    Cancelled,
    HOIST,
    LAZY_RELIN,
    COUNTER_FIELDS,
    Ciphertext,
    Context,
    CudaEvaluator,
    Decode,
    Device,
    EvalConfig,
    HekitError,
    InvalidParams,
    Key,
    LevelMismatch,
    LinearTransform,
    LIB_PATH,
    NoLevelsLeft,
    OutOfMemory,
    Plaintext,
    PinnedBuffer,
    SERVER_STATS,
    ScaleMismatch,
    Server,
    Timeout,
    boot_encode_stages,
    boot_plan,
    boot_rotation_steps,
    build,
    encode_complex_host,
    evalmod_coeffs,
    launch_count,
    lib,
    primes_for_bits,
    seal_decode,
    seal_encode,
    seal_parms_id,
    set_bounds_checking,
)
from . import nn  # noqa: F401,E402
from .router import OwnerRouter  # noqa: F401,E402
