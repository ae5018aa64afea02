// Microsoft SEAL 4.1 serialization of CKKS ciphertexts and plaintexts (compr_mode_type::none),
// the wire format of crates/ckks-train-ckks/src/seal_compat.rs: requests that arrive as SEAL
// bytes are parsed and checked on the host, then uploaded; results go back the same way.
// Host code only.
#pragma once
#include <array>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace ckg {
namespace seal {

// Unkeyed BLAKE2b (RFC 7693) with an out_len-byte digest, 1 <= out_len <= 64.
void blake2b(const uint8_t* data, size_t len, uint8_t* out, size_t out_len);

// SEAL's parms_id of CKKS parameters with ring degree n and coefficient moduli `moduli` (in
// SEAL's order): BLAKE2b-256 of the little-endian words [2 (CKKS), n, moduli..., 0].
std::array<uint64_t, 4> parms_id(uint64_t n, const uint64_t* moduli, size_t count);

// Byte lengths of a serialized ciphertext (ncomp components) and plaintext at `limbs` limbs.
uint64_t ct_bytes(uint64_t n, uint32_t ncomp, uint32_t limbs);
uint64_t pt_bytes(uint64_t n, uint32_t limbs);

// Serialization of NTT-form data at `level` over the data primes q (words: component-major,
// then limb, then coefficient). `out` holds ct_bytes / pt_bytes bytes.
void encode_ct(uint64_t n, const uint64_t* q, const uint64_t* words, uint32_t ncomp, uint32_t level, double scale,
               uint8_t* out);
void encode_pt(uint64_t n, const uint64_t* q, const uint64_t* words, uint32_t level, double scale, uint8_t* out);

// Parsing of untrusted bytes against the parameters (data primes q[0..nq), special primes
// p[0..np)): every length is checked against the bytes present, the parms_id must name a data
// level, every residue must be reduced and nothing may trail. Errors are ST_INVALID_PARAMS.
struct Parsed {
  uint32_t ncomp = 0, level = 0;
  double scale = 0;
  std::vector<uint64_t> words;
};
Parsed decode_ct(uint64_t n, const uint64_t* q, uint32_t nq, const uint64_t* p, uint32_t np, const uint8_t* bytes,
                 uint64_t len);
Parsed decode_pt(uint64_t n, const uint64_t* q, uint32_t nq, const uint64_t* p, uint32_t np, const uint8_t* bytes,
                 uint64_t len);

}  // namespace seal
}  // namespace ckg
