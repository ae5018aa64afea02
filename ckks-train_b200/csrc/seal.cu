// SEAL 4.1 wire format (crates/ckks-train-ckks/src/seal_compat.rs:11-42 for the layout,
// :226-258 for writing, :313-455 for the checks on reading). The byte layout, the parms_id
// construction and the BLAKE2b constants are fixed by SEAL and RFC 7693.
#include <cmath>
#include <cstring>
#include <string>

#include "engine.hpp"
#include "seal.hpp"

static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "SEAL objects are little-endian");

namespace ckg {
namespace seal {
namespace {

constexpr uint16_t kMagic = 0xA15E;
constexpr uint8_t kHeaderSize = 16, kMajor = 4, kMinor = 1;
constexpr uint64_t kSchemeCkks = 2;
constexpr uint64_t kMaxComponents = 16;     // SEAL_CIPHERTEXT_SIZE_MAX
constexpr uint64_t kCtMeta = 32 + 1 + 5 * 8;  // parms_id, is_ntt_form, size, N, L, scale, correction
constexpr uint64_t kPtMeta = 32 + 8 + 8;      // parms_id, coeff_count, scale
constexpr uint64_t kArrayMeta = kHeaderSize + 8;  // DynArray header and element count

// ---- BLAKE2b (RFC 7693) ----------------------------------------------------------------

const uint64_t kIv[8] = {0x6a09e667f3bcc908ULL, 0xbb67ae8584caa73bULL, 0x3c6ef372fe94f82bULL,
                         0xa54ff53a5f1d36f1ULL, 0x510e527fade682d1ULL, 0x9b05688c2b3e6c1fULL,
                         0x1f83d9abfb41bd6bULL, 0x5be0cd19137e2179ULL};
const uint8_t kSigma[10][16] = {
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}, {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3},
    {11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4}, {7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8},
    {9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13}, {2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9},
    {12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11}, {13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10},
    {6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5}, {10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0}};

inline uint64_t rotr(uint64_t x, int r) { return (x >> r) | (x << (64 - r)); }

struct Blake2b {
  uint64_t h[8];
  explicit Blake2b(size_t out_len) {
    memcpy(h, kIv, sizeof h);
    h[0] ^= 0x01010000ULL ^ (uint64_t)out_len;  // digest length, no key, fanout and depth 1
  }
  // One 128-byte block; `bytes` counts every input byte up to the end of this block.
  void compress(const uint8_t* block, uint64_t bytes, bool last) {
    uint64_t m[16], v[16];
    memcpy(m, block, 128);
    for (int i = 0; i < 8; ++i) v[i] = h[i], v[i + 8] = kIv[i];
    v[12] ^= bytes;  // inputs stay below 2^64 bytes: the high counter word is 0
    if (last) v[14] = ~v[14];
    auto mix = [&](int a, int b, int c, int d, uint64_t x, uint64_t y) {
      v[a] += v[b] + x;
      v[d] = rotr(v[d] ^ v[a], 32);
      v[c] += v[d];
      v[b] = rotr(v[b] ^ v[c], 24);
      v[a] += v[b] + y;
      v[d] = rotr(v[d] ^ v[a], 16);
      v[c] += v[d];
      v[b] = rotr(v[b] ^ v[c], 63);
    };
    for (int r = 0; r < 12; ++r) {
      const uint8_t* s = kSigma[r % 10];
      mix(0, 4, 8, 12, m[s[0]], m[s[1]]);
      mix(1, 5, 9, 13, m[s[2]], m[s[3]]);
      mix(2, 6, 10, 14, m[s[4]], m[s[5]]);
      mix(3, 7, 11, 15, m[s[6]], m[s[7]]);
      mix(0, 5, 10, 15, m[s[8]], m[s[9]]);
      mix(1, 6, 11, 12, m[s[10]], m[s[11]]);
      mix(2, 7, 8, 13, m[s[12]], m[s[13]]);
      mix(3, 4, 9, 14, m[s[14]], m[s[15]]);
    }
    for (int i = 0; i < 8; ++i) h[i] ^= v[i] ^ v[i + 8];
  }
};

// ---- little-endian writer and bounds-checked reader -------------------------------------

struct Writer {
  uint8_t* p;
  template <class T>
  void put(T v) {
    memcpy(p, &v, sizeof v);
    p += sizeof v;
  }
  void header(uint64_t size) {
    put<uint16_t>(kMagic);
    put<uint8_t>(kHeaderSize);
    put<uint8_t>(kMajor);
    put<uint8_t>(kMinor);
    put<uint8_t>(0);  // compr_mode_type::none
    put<uint16_t>(0);
    put<uint64_t>(size);
  }
  void parms(const std::array<uint64_t, 4>& id) {
    for (uint64_t w : id) put(w);
  }
};

[[noreturn]] void bad(const std::string& msg) { throw Error(ST_INVALID_PARAMS, "SEAL object: " + msg); }

struct Reader {
  const uint8_t* p;
  uint64_t left;
  template <class T>
  T get() {
    if (left < sizeof(T)) bad("truncated");
    T v;
    memcpy(&v, p, sizeof v);
    p += sizeof v;
    left -= sizeof v;
    return v;
  }
  // A SEALHeader; returns its size field.
  uint64_t header() {
    if (get<uint16_t>() != kMagic) bad("bad magic (not a SEAL object)");
    if (get<uint8_t>() != kHeaderSize) bad("unsupported header size");
    const uint8_t major = get<uint8_t>();
    get<uint8_t>();
    if (major != kMajor) bad("SEAL " + std::to_string(major) + ".x serialization is not supported (need 4.x)");
    const uint8_t compr = get<uint8_t>();
    if (compr == 1 || compr == 2) bad("compressed objects are not supported (save with compr_mode_type::none)");
    if (compr != 0) bad("unknown compression mode " + std::to_string(compr));
    get<uint16_t>();
    return get<uint64_t>();
  }
  std::array<uint64_t, 4> parms() {
    std::array<uint64_t, 4> id;
    for (auto& w : id) w = get<uint64_t>();
    return id;
  }
  // A DynArray<u64> of exactly `count` words, each reduced modulo its limb's prime.
  void words(uint64_t count, uint64_t n, const uint64_t* q, uint32_t limbs, std::vector<uint64_t>& out) {
    const uint64_t size = header();
    const uint64_t have = get<uint64_t>();
    if (have != count)
      bad("holds " + std::to_string(have) + " data words, expected " + std::to_string(count) +
          " (seeded ciphertexts are not supported)");
    if (size != kArrayMeta + 8 * count) bad("data header size does not match its count");
    if (left < 8 * count) bad("truncated");
    out.resize(count);
    memcpy(out.data(), p, 8 * count);
    p += 8 * count;
    left -= 8 * count;
    for (uint64_t i = 0; i < count; ++i)
      if (out[i] >= q[(i / n) % limbs]) bad("residue " + std::to_string(i) + " is not reduced");
  }
};

// The outer header must span exactly the given bytes.
Reader open(const uint8_t* bytes, uint64_t len) {
  if (!bytes && len) bad("null bytes");
  Reader r{bytes, len};
  const uint64_t size = r.header();
  if (size != len) bad("header size " + std::to_string(size) + " != object length " + std::to_string(len));
  return r;
}

// The data level whose parms_id is `id`, -1 for the key level (all primes), else an error.
int level_of(const std::array<uint64_t, 4>& id, uint64_t n, const uint64_t* q, uint32_t nq, const uint64_t* p,
             uint32_t np) {
  for (uint32_t l = 0; l < nq; ++l)
    if (parms_id(n, q, l + 1) == id) return (int)l;
  std::vector<uint64_t> all(q, q + nq);
  all.insert(all.end(), p, p + np);
  if (parms_id(n, all.data(), all.size()) == id) return -1;
  bad("parms_id matches no level of these parameters (different N or moduli)");
}

}  // namespace

void blake2b(const uint8_t* data, size_t len, uint8_t* out, size_t out_len) {
  if (out_len < 1 || out_len > 64) throw Error(ST_INVALID_PARAMS, "BLAKE2b digest length outside 1..=64");
  Blake2b b(out_len);
  uint8_t block[128];
  size_t done = 0;
  while (len - done > 128) {  // every block but the last
    memcpy(block, data + done, 128);
    done += 128;
    b.compress(block, done, false);
  }
  memset(block, 0, sizeof block);
  if (len > done) memcpy(block, data + done, len - done);
  b.compress(block, len, true);
  memcpy(out, b.h, out_len);
}

std::array<uint64_t, 4> parms_id(uint64_t n, const uint64_t* moduli, size_t count) {
  std::vector<uint64_t> words;
  words.reserve(count + 3);
  words.push_back(kSchemeCkks);
  words.push_back(n);
  words.insert(words.end(), moduli, moduli + count);
  words.push_back(0);  // plain_modulus (none for CKKS)
  std::array<uint64_t, 4> id;
  blake2b((const uint8_t*)words.data(), words.size() * 8, (uint8_t*)id.data(), 32);
  return id;
}

uint64_t ct_bytes(uint64_t n, uint32_t ncomp, uint32_t limbs) {
  return kHeaderSize + kCtMeta + kArrayMeta + 8 * (uint64_t)ncomp * limbs * n;
}

uint64_t pt_bytes(uint64_t n, uint32_t limbs) { return kHeaderSize + kPtMeta + kArrayMeta + 8 * (uint64_t)limbs * n; }

void encode_ct(uint64_t n, const uint64_t* q, const uint64_t* words, uint32_t ncomp, uint32_t level, double scale,
               uint8_t* out) {
  const uint64_t count = (uint64_t)ncomp * (level + 1) * n;
  Writer w{out};
  w.header(ct_bytes(n, ncomp, level + 1));
  w.parms(parms_id(n, q, level + 1));
  w.put<uint8_t>(1);  // is_ntt_form
  w.put<uint64_t>(ncomp);
  w.put<uint64_t>(n);
  w.put<uint64_t>(level + 1);
  w.put<double>(scale);
  w.put<uint64_t>(1);  // correction_factor (1 for CKKS)
  w.header(kArrayMeta + 8 * count);
  w.put<uint64_t>(count);
  memcpy(w.p, words, 8 * count);
}

void encode_pt(uint64_t n, const uint64_t* q, const uint64_t* words, uint32_t level, double scale, uint8_t* out) {
  const uint64_t count = (uint64_t)(level + 1) * n;
  Writer w{out};
  w.header(pt_bytes(n, level + 1));
  w.parms(parms_id(n, q, level + 1));
  w.put<uint64_t>(count);
  w.put<double>(scale);
  w.header(kArrayMeta + 8 * count);
  w.put<uint64_t>(count);
  memcpy(w.p, words, 8 * count);
}

Parsed decode_ct(uint64_t n, const uint64_t* q, uint32_t nq, const uint64_t* p, uint32_t np, const uint8_t* bytes,
                 uint64_t len) {
  Reader r = open(bytes, len);
  const auto id = r.parms();
  const uint8_t ntt = r.get<uint8_t>();
  const uint64_t size = r.get<uint64_t>(), degree = r.get<uint64_t>(), limbs = r.get<uint64_t>();
  const double scale = r.get<double>();
  const uint64_t correction = r.get<uint64_t>();
  const int level = level_of(id, n, q, nq, p, np);
  if (level < 0) bad("parms_id is the key level, not a ciphertext level");
  if (degree != n || limbs != (uint64_t)level + 1) bad("ring degree or modulus count does not match the parms_id");
  if (ntt != 1) bad("ciphertext is not in NTT form");
  if (size < 2 || size > kMaxComponents) bad("ciphertext size " + std::to_string(size) + " outside 2..=16");
  if (correction != 1) bad("CKKS ciphertexts have correction_factor 1");
  if (!(std::isfinite(scale) && scale > 0)) bad("scale must be positive and finite");
  Parsed out;
  out.ncomp = (uint32_t)size;
  out.level = (uint32_t)level;
  out.scale = scale;
  r.words(size * limbs * n, n, q, (uint32_t)limbs, out.words);
  if (r.left) bad(std::to_string(r.left) + " trailing bytes");
  return out;
}

Parsed decode_pt(uint64_t n, const uint64_t* q, uint32_t nq, const uint64_t* p, uint32_t np, const uint8_t* bytes,
                 uint64_t len) {
  Reader r = open(bytes, len);
  const auto id = r.parms();
  const uint64_t coeffs = r.get<uint64_t>();
  const double scale = r.get<double>();
  if (id == std::array<uint64_t, 4>{}) bad("coefficient-form plaintexts are not supported (CKKS uses NTT form)");
  const int level = level_of(id, n, q, nq, p, np);
  if (level < 0) bad("parms_id is the key level, not a plaintext level");
  if (coeffs != ((uint64_t)level + 1) * n) bad("coeff_count does not match the level");
  if (!(std::isfinite(scale) && scale > 0)) bad("scale must be positive and finite");
  Parsed out;
  out.ncomp = 1;
  out.level = (uint32_t)level;
  out.scale = scale;
  r.words(coeffs, n, q, (uint32_t)level + 1, out.words);
  if (r.left) bad(std::to_string(r.left) + " trailing bytes");
  return out;
}

}  // namespace seal
}  // namespace ckg
