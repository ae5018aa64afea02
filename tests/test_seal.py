"""The SEAL 4.1 wire format on the host (include/ckg.h, "SEAL 4.1 wire format";
crates/ckks-train-ckks/src/seal_compat.rs), no GPU:

* parms_id pinned to the values SEAL 4.1.2 printed for seal_2020 and to the n16_train key-level
  value the reference pins (seal_compat.rs:580-625), and to Python's hashlib.blake2b, including
  inputs of exactly one block and of several blocks;
* serialization byte-identical to an independent writer (struct + hashlib) of the layout at
  seal_compat.rs:11-33, with the length and header of seal_compat.rs's round-trip test;
* round trips of ciphertexts and plaintexts, and every rejection of seal_compat.rs's
  malformed-input test (seal_compat.rs:665-720), each an InvalidParams.
"""

import hashlib
import math
import struct

import numpy as np
import pytest

SEAL_2020 = (15, [60] + [40] * 9, [60])  # CoeffModulus::Create(32768, {60, 40 x 9, 60})
N16_TRAIN = (16, [58] + [42] * 31, [58] * 4)
SMALL = (6, [60, 40, 40], [60])  # the parameters of seal_compat.rs's own round-trip tests


def _ref_parms_id(n, moduli):
    data = b"".join(struct.pack("<Q", w) for w in [2, n] + list(moduli) + [0])
    return list(struct.unpack("<4Q", hashlib.blake2b(data, digest_size=32).digest()))


def _ref_ct_bytes(n, q, words, level, scale):
    """An independent writer of a SEAL 4.1 Ciphertext (compr_mode_type::none)."""
    count = words.size
    total = 16 + 73 + 24 + 8 * count
    head = lambda size: struct.pack("<HBBBBHQ", 0xA15E, 16, 4, 1, 0, 0, size)
    body = struct.pack("<4Q", *_ref_parms_id(n, q[:level + 1]))
    body += struct.pack("<BQQQdQ", 1, words.shape[0], n, level + 1, scale, 1)
    return head(total) + body + head(24 + 8 * count) + struct.pack("<Q", count) + words.astype("<u8").tobytes()


def _params(ckg, spec):
    log_n, qb, pb = spec
    q, p = ckg.primes_for_bits(log_n, qb, pb)
    return log_n, q, p


def _random_words(q, n, ncomp, level, seed):
    rng = np.random.default_rng(seed)
    w = np.zeros((ncomp, level + 1, n), np.uint64)
    for c in range(ncomp):
        for i in range(level + 1):
            w[c, i] = rng.integers(0, q[i], n, dtype=np.uint64)
    return w


def test_parms_id_pinned(ckg):
    log_n, q, p = _params(ckg, SEAL_2020)
    assert ckg.seal_parms_id(log_n, q + p) == [7191370043490053719, 62418774019697152, 17097305126088585189,
                                              18375298844209535223]
    assert ckg.seal_parms_id(log_n, q[:1]) == [1256757360063172209, 3701657226246155154, 6506013794352499262,
                                               1216675072159714914]
    assert ckg.seal_parms_id(log_n, q[:10]) == [16169145876469523575, 11660861062887149260, 12362353866312426611,
                                                17077531305736521100]
    log_n, q, p = _params(ckg, N16_TRAIN)
    assert ckg.seal_parms_id(log_n, q + p) == [6651339613328061365, 2299678865699252732, 1912788140720359349,
                                              5768396979508793702]
    rng = np.random.default_rng(1)
    for count in (0, 1, 13, 14, 29, 36, 61):  # 13 moduli: exactly 128 bytes; 29: exactly 256
        m = [int(x) for x in rng.integers(1, 2 ** 62, count)]
        assert ckg.seal_parms_id(12, m) == _ref_parms_id(4096, m), count


def test_ciphertext_layout_and_round_trip(ckg):
    log_n, q, p = _params(ckg, SMALL)
    n = 1 << log_n
    w = _random_words(q, n, 2, 2, 5)
    data = ckg.seal_encode(log_n, q, w, 2, 2.0 ** 40)
    assert len(data) == 16 + 73 + 24 + 8 * 2 * 3 * 64
    assert data[:8] == bytes([0x5E, 0xA1, 16, 4, 1, 0, 0, 0])
    assert data == _ref_ct_bytes(n, q, w, 2, 2.0 ** 40)
    back, level, scale = ckg.seal_decode(log_n, q, p, data)
    assert level == 2 and scale == 2.0 ** 40 and np.array_equal(back, w)
    assert ckg.seal_encode(log_n, q, back, level, scale) == data
    # a 3-component ciphertext at level 0, and a plaintext
    w3 = _random_words(q, n, 3, 0, 6)
    back, level, _ = ckg.seal_decode(log_n, q, p, ckg.seal_encode(log_n, q, w3, 0, 3.5))
    assert level == 0 and np.array_equal(back, w3)
    pt = _random_words(q, n, 1, 1, 7)[0]
    pdata = ckg.seal_encode(log_n, q, pt, 1, 2.0 ** 30, plaintext=True)
    assert len(pdata) == 16 + 48 + 24 + 8 * 2 * 64
    back, level, scale = ckg.seal_decode(log_n, q, p, pdata, plaintext=True)
    assert level == 1 and scale == 2.0 ** 30 and np.array_equal(back, pt)
    with pytest.raises(ckg.InvalidParams):
        ckg.seal_decode(log_n, q, p, pdata)  # a plaintext is not a ciphertext
    with pytest.raises(ckg.InvalidParams):
        ckg.seal_decode(log_n, q, p, data, plaintext=True)


def test_rejects_malformed_ciphertexts(ckg):
    """seal_compat.rs:665-720: every malformed variant is InvalidParams."""
    log_n, q, p = _params(ckg, SMALL)
    n = 1 << log_n
    good = ckg.seal_encode(log_n, q, _random_words(q, n, 2, 2, 8), 2, 2.0 ** 40)
    ckg.seal_decode(log_n, q, p, good)

    def patched(at, b):
        v = bytearray(good)
        v[at:at + len(b)] = b
        return bytes(v)

    u64 = lambda x: struct.pack("<Q", x)
    f64 = lambda x: struct.pack("<d", x)
    cases = [(b"", "empty"), (good[:-1], "truncated"), (good + b"\0", "trailing byte"),
             (patched(0, b"\0\0"), "magic"), (patched(2, bytes([17])), "header size"),
             (patched(3, bytes([3])), "version 3"), (patched(5, bytes([2])), "zstd"),
             (patched(8, u64(2 ** 64 - 1)), "outer size"), (patched(16, b"\xff"), "parms_id"),
             (patched(48, b"\0"), "coefficient form"), (patched(49, u64(1)), "size 1"),
             (patched(49, u64(17)), "size 17"), (patched(49, u64(2 ** 64 - 1)), "size huge"),
             (patched(57, u64(128)), "N"), (patched(65, u64(2)), "coeff_modulus_size"),
             (patched(73, f64(0.0)), "scale 0"), (patched(73, f64(math.nan)), "scale NaN"),
             (patched(81, u64(2)), "correction factor"), (patched(89, b"\0\0"), "inner magic"),
             (patched(97, u64(2 ** 64 - 1)), "inner size"), (patched(105, u64(3 * 64)), "seeded count"),
             (patched(105, u64(2 ** 64 - 1)), "huge count"), (patched(113, u64(q[0])), "unreduced residue")]
    other = _ref_parms_id(n, [q[0] - 2 * n, q[1], q[2]])
    cases.append((patched(16, struct.pack("<4Q", *other)), "other moduli"))
    cases.append((patched(16, struct.pack("<4Q", *_ref_parms_id(n, q + p))), "key level"))
    for data, what in cases:
        with pytest.raises(ckg.InvalidParams):
            ckg.seal_decode(log_n, q, p, data)
            pytest.fail(what)
    q7, p7 = ckg.primes_for_bits(7, [60, 40, 40], [60])
    with pytest.raises(ckg.InvalidParams):
        ckg.seal_decode(7, q7, p7, good)  # another ring degree
