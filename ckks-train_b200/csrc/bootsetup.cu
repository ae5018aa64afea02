// Host-side bootstrap setup (bootsetup.hpp): encoder, special-DFT stages, stage encoding,
// EvalMod series. Host code only; the encoded diagonals are uploaded and moved to NTT form
// on the device.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <thread>

#include "bootsetup.hpp"

namespace ckg {

namespace {

// ---- complex numbers with num-complex 0.4's formulas ----------------------------------

struct Cx {
  double re = 0, im = 0;
};
inline Cx operator+(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }
inline Cx operator-(Cx a, Cx b) { return {a.re - b.re, a.im - b.im}; }
inline Cx operator-(Cx a) { return {-a.re, -a.im}; }
inline Cx operator*(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline Cx operator*(Cx a, double s) { return {a.re * s, a.im * s}; }
inline Cx operator/(Cx a, double s) { return {a.re / s, a.im / s}; }
inline Cx operator/(Cx a, Cx b) {
  const double n = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / n, (a.im * b.re - a.re * b.im) / n};
}
inline Cx conj(Cx a) { return {a.re, -a.im}; }
inline bool is_zero(Cx a) { return a.re == 0.0 && a.im == 0.0; }
const Cx kZero{0.0, 0.0}, kOne{1.0, 0.0};

// ---- encoder tables (encoder.rs:14-190) ------------------------------------------------

size_t rev_bits(size_t i, uint32_t bits) {
  if (!bits) return 0;
  uint64_t r = 0;
  for (uint32_t b = 0; b < 64; ++b) r |= (((uint64_t)i >> b) & 1ULL) << (63 - b);
  return (size_t)(r >> (64 - bits));
}

Cx complex_root(const std::vector<Cx>& t, size_t m, size_t index) {  // encoder.rs:31-46
  index &= m - 1;
  if (index <= m / 8) return t[index];
  if (index <= m / 4) {
    const Cx a = t[m / 4 - index];
    return {a.im, a.re};
  }
  if (index <= m / 2) return -conj(complex_root(t, m, m / 2 - index));
  if (index <= 3 * m / 4) return -complex_root(t, m, index - m / 2);
  return conj(complex_root(t, m, m - index));
}

struct EncTables {
  std::vector<size_t> index_map;
  std::vector<Cx> inv_roots;
};

const EncTables& enc_tables(uint32_t log_n) {
  static std::mutex mu;
  static std::map<uint32_t, EncTables> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(log_n);
  if (it != cache.end()) return it->second;
  EncTables t;
  const size_t n = (size_t)1 << log_n, slots = n / 2, m = 2 * n;
  t.index_map.assign(n, 0);
  size_t pos = 1;
  for (size_t i = 0; i < slots; ++i) {
    t.index_map[i] = rev_bits((pos - 1) >> 1, log_n);
    t.index_map[slots | i] = rev_bits((m - pos - 1) >> 1, log_n);
    pos = (pos * 3) & (m - 1);
  }
  t.inv_roots.assign(n, kZero);
  if (m >= 8) {
    std::vector<Cx> table;
    for (size_t i = 0; i <= m / 8; ++i) {
      const double th = 2.0 * M_PI * (double)i / (double)m;
      table.push_back({1.0 * std::cos(th), 1.0 * std::sin(th)});
    }
    for (size_t i = 1; i < n; ++i) t.inv_roots[i] = conj(complex_root(table, m, rev_bits(i - 1, log_n) + 1));
  } else {
    t.inv_roots[1] = {0.0, -1.0};
  }
  return cache.emplace(log_n, std::move(t)).first->second;
}

void transform_from_rev(std::vector<Cx>& v, const std::vector<Cx>& roots, double scalar) {  // encoder.rs:75-105
  size_t n = v.size(), ri = 0, gap = 1, m = n >> 1;
  while (m > 1) {
    size_t offset = 0;
    for (size_t b = 0; b < m; ++b) {
      ri += 1;
      const Cx r = roots[ri];
      for (size_t x = offset; x < offset + gap; ++x) {
        const Cx u = v[x], w = v[x + gap];
        v[x] = u + w;
        v[x + gap] = (u - w) * r;
      }
      offset += gap << 1;
    }
    gap <<= 1;
    m >>= 1;
  }
  ri += 1;
  const Cx scaled_r = roots[ri] * scalar;
  for (size_t x = 0; x < gap; ++x) {
    const Cx u = v[x], w = v[x + gap];
    v[x] = (u + w) * scalar;
    v[x + gap] = (u - w) * scaled_r;
  }
}

// The data primes and their moduli, all a host encode needs.
struct Chain {
  uint32_t log_n = 0;
  std::vector<uint64_t> q;
  std::vector<HostMod> mods;
  explicit Chain(const Context& c) : log_n(c.log_n), q(c.primes.begin(), c.primes.begin() + c.L + 1) {
    for (auto v : q) mods.emplace_back(v);
  }
  Chain(uint32_t ln, const uint64_t* primes, uint32_t nq) : log_n(ln), q(primes, primes + nq) {
    for (auto v : q) mods.emplace_back(v);
  }
};

std::vector<uint64_t> encode_cx(const Chain& c, const std::vector<Cx>& values, double scale, uint32_t level) {
  const size_t n = (size_t)1 << c.log_n, slots = n / 2;  // encoder.rs:215-283
  if (values.size() > slots) throw Error(ST_INVALID_PARAMS, "more values than slots");
  if (level + 1 > c.q.size()) throw Error(ST_INVALID_PARAMS, "level exceeds max_level");
  if (!(std::isfinite(scale) && scale > 0.0)) throw Error(ST_INVALID_PARAMS, "scale must be positive and finite");
  for (auto& z : values)
    if (!(std::isfinite(z.re) && std::isfinite(z.im))) throw Error(ST_INVALID_PARAMS, "non-finite value");
  const EncTables& t = enc_tables(c.log_n);
  std::vector<Cx> cv(n, kZero);
  for (size_t i = 0; i < values.size(); ++i) {
    cv[t.index_map[i]] = values[i];
    cv[t.index_map[slots + i]] = conj(values[i]);
  }
  transform_from_rev(cv, t.inv_roots, scale / (double)n);
  double log_q = -0.0;
  for (uint32_t i = 0; i <= level; ++i) log_q += std::log2((double)c.q[i]);
  const double limit = std::exp2(log_q - 1.0);
  std::vector<double> coeffs(n);
  for (size_t i = 0; i < n; ++i) {
    coeffs[i] = std::round(cv[i].re);
    if (std::isnan(coeffs[i]) || std::fabs(coeffs[i]) >= limit)
      throw Error(ST_INVALID_PARAMS, "encoded coefficient does not fit in Q/2 at this level");
  }
  std::vector<uint64_t> out((size_t)(level + 1) * n);
  for (uint32_t k = 0; k <= level; ++k) {
    const HostMod& m = c.mods[k];
    uint64_t* limb = out.data() + (size_t)k * n;
    for (size_t i = 0; i < n; ++i) {
      const double a = std::fabs(coeffs[i]);
      uint64_t r;
      if (a < 9223372036854775808.0) {
        r = (uint64_t)a % m.q;
      } else {  // a = mantissa * 2^exponent exactly
        uint64_t bits;
        memcpy(&bits, &a, 8);
        const uint64_t exponent = ((bits >> 52) & 0x7ff) - 1075;
        const uint64_t mantissa = (bits & ((1ULL << 52) - 1)) | (1ULL << 52);
        r = m.mul(mantissa % m.q, m.pow(2, exponent));
      }
      limb[i] = (coeffs[i] < 0.0 && r != 0) ? m.q - r : r;
    }
  }
  return out;
}

Pt upload_coeffs(Evaluator& ev, const std::vector<uint64_t>& coeffs, double scale, uint32_t level) {
  Context& c = *ev.ctx();
  Pt p = ev.upload_pt(coeffs.data(), false, level, scale);
  std::vector<LimbRef> refs;
  for (uint32_t i = 0; i <= level; ++i) refs.push_back(LimbRef{p->buf->p + (size_t)i * c.n, p->buf->p + (size_t)i * c.n, i, 0});
  ntt_limbs(c, refs, false);
  return p;
}

// ---- special-DFT stages (linear.rs:78-455) ---------------------------------------------

struct Shape {
  uint32_t d = 1, stride = 1;
  int64_t offset = 0;
};

struct DiagMatrix {
  size_t n = 0;
  std::map<size_t, std::vector<Cx>> diags;

  static DiagMatrix identity(size_t n) {
    DiagMatrix m;
    m.n = n;
    m.diags[0] = std::vector<Cx>(n, kOne);
    return m;
  }
  std::vector<Cx>& diag_at(size_t o) {
    auto it = diags.find(o);
    if (it == diags.end()) it = diags.emplace(o, std::vector<Cx>(n, kZero)).first;
    return it->second;
  }
  void add_entry(size_t row, size_t col, Cx v) {
    auto& d = diag_at((col + n - row) % n);
    d[row] = d[row] + v;
  }
  DiagMatrix mul(const DiagMatrix& rhs) const {  // (A B)[t][t+o1+o2] += A[t][t+o1] B[t+o1][t+o1+o2]
    DiagMatrix out;
    out.n = n;
    for (auto& a : diags)
      for (auto& b : rhs.diags) {
        auto& c = out.diag_at((a.first + b.first) % n);
        for (size_t t = 0; t < n; ++t) c[t] = c[t] + a.second[t] * b.second[(t + a.first) % n];
      }
    return out;
  }
  template <class F>
  DiagMatrix map_entries(F f) const {
    DiagMatrix out;
    out.n = n;
    for (auto& d : diags) {
      std::vector<Cx> w(n);
      for (size_t t = 0; t < n; ++t) w[t] = f(t, (t + d.first) % n, d.second[t]);
      out.diags.emplace(d.first, std::move(w));
    }
    return out;
  }
  DiagMatrix scaled(Cx c) const {
    return map_entries([&](size_t, size_t, Cx v) { return v * c; });
  }
  DiagMatrix rho() const {
    return map_entries([](size_t r, size_t, Cx v) { return r % 2 == 1 ? conj(v) : v; });
  }
  std::pair<DiagMatrix, DiagMatrix> conj_sandwich() const {
    auto part = [&](bool same) {
      return map_entries([&](size_t r, size_t c, Cx v) {
        if ((r % 2 == c % 2) != same) return kZero;
        return r % 2 == 1 ? conj(v) : v;
      });
    };
    return {part(true), part(false)};
  }
  bool parity_preserving() const {
    for (auto& d : diags)
      if (d.first % 2) return false;
    return true;
  }
  Shape shape() const;
  std::vector<std::vector<Cx>> window(Shape s) const {
    const int64_t nn = (int64_t)n;
    std::vector<size_t> idx;
    for (int64_t i = 0; i < (int64_t)s.d; ++i) {
      const int64_t v = ((s.offset + i) * (int64_t)s.stride) % nn;
      idx.push_back((size_t)(v < 0 ? v + nn : v));
    }
    for (auto& d : diags)
      if (std::find(idx.begin(), idx.end(), d.first) == idx.end())
        throw Error(ST_INVALID_PARAMS, "diagonal outside the stage layout");
    std::vector<std::vector<Cx>> out;
    for (size_t o : idx) {
      auto it = diags.find(o);
      out.push_back(it == diags.end() ? std::vector<Cx>(n, kZero) : it->second);
    }
    return out;
  }
};

Shape shape_from_offsets(size_t n, const std::vector<size_t>& offsets) {  // linear.rs:283-321
  uint32_t tz = 64;
  for (size_t o : offsets)
    if (o) tz = std::min<uint32_t>(tz, (uint32_t)__builtin_ctzll(o));
  if (tz == 64) return Shape{};
  const size_t stride = (size_t)1 << tz;
  const int64_t m = (int64_t)(n / stride);
  int64_t kmin = INT64_MAX, kmax = INT64_MIN;
  for (size_t o : offsets) {
    int64_t k = (int64_t)(o / stride);
    if (k > m / 2) k -= m;
    kmin = std::min(kmin, k);
    kmax = std::max(kmax, k);
  }
  size_t d = 1;
  while (d < (size_t)(kmax - kmin + 1)) d <<= 1;
  while ((int64_t)d < m) {
    const int64_t g = (int64_t)bsgs_split((uint32_t)d).first;
    const int64_t fl = kmin >= 0 ? kmin / g : -((-kmin + g - 1) / g);
    const int64_t offset = std::min<int64_t>(fl * g, 0);
    if (offset > -(int64_t)d && offset + (int64_t)d > kmax) return Shape{(uint32_t)d, (uint32_t)stride, offset};
    d *= 2;
  }
  return Shape{(uint32_t)m, (uint32_t)stride, 0};
}

Shape DiagMatrix::shape() const {
  std::vector<size_t> offs;
  for (auto& d : diags) offs.push_back(d.first);
  return shape_from_offsets(n, offs);
}

size_t pow_mod_sz(size_t b, size_t e, size_t m) {  // linear.rs:329-340
  size_t base = b % m, acc = 1 % m;
  for (; e; e >>= 1) {
    if (e & 1) acc = acc * base % m;
    base = base * base % m;
  }
  return acc;
}

DiagMatrix butterfly(size_t n, size_t len, bool inverse) {  // linear.rs:345-375
  const size_t h = len / 2, m4 = 4 * len;
  DiagMatrix s;
  s.n = n;
  for (size_t i = 0; i < n; i += len)
    for (size_t j = 0; j < h; ++j) {
      const double a = 2.0 * M_PI * (double)pow_mod_sz(m4 - 3, j, m4) / (double)m4;
      const Cx w{std::cos(a), std::sin(a)};
      const size_t top = i + j, bot = i + j + h;
      if (inverse) {
        const Cx half{0.5, 0.0}, wi = half / w;
        s.add_entry(top, top, half);
        s.add_entry(top, bot, half);
        s.add_entry(bot, top, wi);
        s.add_entry(bot, bot, -wi);
      } else {
        s.add_entry(top, top, kOne);
        s.add_entry(top, bot, w);
        s.add_entry(bot, top, kOne);
        s.add_entry(bot, bot, -w);
      }
    }
  return s;
}

std::vector<DiagMatrix> dft_stages(uint32_t log_slots, uint32_t levels, bool inverse) {  // linear.rs:377-430
  if (log_slots < 1 || log_slots > 16 || levels < 1 || levels > log_slots)
    throw Error(ST_INVALID_PARAMS, "dft_stages: log_slots outside 1..=16 or levels outside 1..=log_slots");
  const size_t n = (size_t)1 << log_slots;
  const uint32_t base = log_slots / levels, extra = log_slots % levels;
  std::vector<DiagMatrix> groups;
  uint32_t k = 1;
  for (uint32_t g = 0; g < levels; ++g) {
    const uint32_t r = base + (g >= levels - extra ? 1 : 0);
    DiagMatrix m = DiagMatrix::identity(n);
    for (uint32_t s = k; s < k + r; ++s) {
      DiagMatrix b = butterfly(n, (size_t)1 << s, inverse);
      m = inverse ? m.mul(b) : b.mul(m);
    }
    groups.push_back(std::move(m));
    k += r;
  }
  if (inverse) std::reverse(groups.begin(), groups.end());
  return groups;
}

std::pair<Cx, Cx> folded_factors(Cx f, size_t l) {  // linear.rs:559-570
  const double nrm = std::hypot(f.re, f.im);
  if (!(std::isfinite(f.re) && std::isfinite(f.im) && nrm > 0.0))
    throw Error(ST_INVALID_PARAMS, "factor must be finite and nonzero");
  return {Cx{std::pow(nrm, 1.0 / (double)l), 0.0}, f / nrm};
}

struct Adapted {
  DiagMatrix main;
  bool has_second = false;
  DiagMatrix second;
};

std::vector<Adapted> adapt(const std::vector<DiagMatrix>& st, int dir, Cx factor) {  // linear.rs:512-557
  const size_t l = st.size();
  if (!l) throw Error(ST_INVALID_PARAMS, "no stages");
  auto mp = folded_factors(factor, l);
  const Cx mag = mp.first, phase = mp.second;
  const size_t lo = dir == DIR_COEFF_TO_SLOT ? 0 : 1, hi = dir == DIR_COEFF_TO_SLOT ? l - 1 : l;
  for (size_t i = lo; i < hi; ++i)
    if (!st[i].parity_preserving())
      throw Error(ST_INVALID_PARAMS, "only the distance-1 group may mix even and odd slots");
  std::vector<Adapted> out;
  if (dir == DIR_COEFF_TO_SLOT) {
    for (size_t i = lo; i < hi; ++i) out.push_back(Adapted{st[i].rho().scaled(mag), false, DiagMatrix{}});
    auto ab = st[l - 1].scaled(phase * mag * 0.5).conj_sandwich();
    out.push_back(Adapted{ab.first, true, ab.second});
  } else {
    const Cx c = phase * mag;
    out.push_back(Adapted{st[0].rho().scaled(c), true, st[0].scaled(Cx{0.0, 1.0}).rho().scaled(c)});
    for (size_t i = lo; i < hi; ++i) out.push_back(Adapted{st[i].rho().scaled(mag), false, DiagMatrix{}});
  }
  return out;
}

// Pre-rotation of a window by the giant steps (linalg.rs:561-592): entry k1 * baby + k2 is
// diagonal k1 * baby + k2 rotated by -(offset + baby k1) stride; `zero` marks all-zero entries.
void prerotate(const std::vector<std::vector<Cx>>& diagonals, Shape sh, size_t slots,
               std::vector<std::vector<Cx>>& pre, std::vector<bool>& zero) {
  const size_t d = diagonals.size();
  if (!(sh.offset <= 0 && sh.offset > -(int64_t)d))
    throw Error(ST_INVALID_PARAMS, "diagonal offset outside -d < offset <= 0");
  if (!slots || slots % ((size_t)d * sh.stride)) throw Error(ST_INVALID_PARAMS, "d * stride must divide the slot count");
  auto bg = bsgs_split((uint32_t)d);
  pre.assign(d, {});
  zero.assign(d, true);
  for (uint32_t k1 = 0; k1 < bg.second; ++k1) {
    int64_t s = ((sh.offset + (int64_t)bg.first * k1) * (int64_t)sh.stride) % (int64_t)slots;
    const size_t shift = (size_t)(s < 0 ? s + (int64_t)slots : s);
    for (uint32_t k2 = 0; k2 < bg.first; ++k2) {
      const size_t e = (size_t)bg.first * k1 + k2;
      const auto& v = diagonals[e];
      pre[e].resize(slots);
      for (size_t j = 0; j < slots; ++j) {
        pre[e][j] = v[(j + slots - shift) % slots];
        if (!is_zero(pre[e][j])) zero[e] = false;
      }
    }
  }
}

// Encoding of the non-zero pre-rotated entries (linalg.rs:334-369); host encodes run on
// worker threads, uploads in entry order.
SparseDiag encode_window(Evaluator& ev, const std::vector<std::vector<Cx>>& diagonals, Shape sh, double scale,
                         uint32_t level) {
  const Chain c(*ev.ctx());
  const size_t d = diagonals.size(), slots = ev.ctx()->n / 2;
  std::vector<std::vector<Cx>> pre;
  std::vector<bool> zero;
  prerotate(diagonals, sh, slots, pre, zero);
  auto bg = bsgs_split((uint32_t)d);
  SparseDiag out;
  out.d = (uint32_t)d;
  out.baby = bg.first;
  out.giant = bg.second;
  out.stride = sh.stride;
  out.offset = sh.offset;
  std::vector<std::vector<uint64_t>> coeffs(d);
  std::vector<std::string> errs(d);
  std::vector<int> codes(d, 0);
  const size_t workers = std::max<size_t>(1, std::min<size_t>(d, std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  for (size_t w = 0; w < workers; ++w)
    pool.emplace_back([&, w] {
      for (size_t e = w; e < d; e += workers) {
        if (zero[e]) continue;
        try {
          coeffs[e] = encode_cx(c, pre[e], scale, level);
        } catch (const Error& x) {
          errs[e] = x.what();
          codes[e] = x.code;
        }
      }
    });
  for (auto& t : pool) t.join();
  for (size_t e = 0; e < d; ++e)
    if (codes[e]) throw Error(codes[e], errs[e]);
  bool any = false;
  for (size_t e = 0; e < d; ++e) {
    out.entries.push_back(zero[e] ? Pt() : upload_coeffs(ev, coeffs[e], scale, level));
    any = any || !zero[e];
  }
  if (!any) throw Error(ST_INVALID_PARAMS, "every diagonal is zero (nothing to encode)");
  return out;
}

std::vector<double> chebyshev_coeffs(double (*f)(double, const BootParams&), const BootParams& bp, double a, double b,
                                     size_t degree) {  // poly.rs:90-140
  const size_t n = degree + 1;
  std::vector<double> theta(n), fx(n), out(n);
  for (size_t k = 0; k < n; ++k) theta[k] = M_PI * ((double)k + 0.5) / (double)n;
  for (size_t k = 0; k < n; ++k) fx[k] = f(0.5 * (b - a) * std::cos(theta[k]) + 0.5 * (a + b), bp);
  for (size_t j = 0; j < n; ++j) {
    double s = -0.0;
    for (size_t k = 0; k < n; ++k) s += fx[k] * std::cos((double)j * theta[k]);
    const double value = 2.0 * s / (double)n;
    out[j] = j == 0 ? value / 2.0 : value;
  }
  return out;
}

double evalmod_function(double y, const BootParams& bp) {  // evalmod.rs:73-83
  const double k = (double)bp.k_intervals;
  if (bp.double_angle == 0) return std::sin(2.0 * M_PI * k * y);
  const double div = (double)(1ULL << bp.double_angle);
  return std::cos(2.0 * M_PI * (k * y - 0.25) / div);
}

double nominal_scale(const Context& c, uint32_t level, double delta) {  // params.rs:282-289
  return level == 0 ? delta : std::exp2((double)bit_length(c.primes[level]));
}

}  // namespace

std::vector<uint64_t> encode_complex_coeffs(uint32_t log_n, const uint64_t* primes, uint32_t nq, const double* values,
                                           size_t count, double scale, uint32_t level) {
  std::vector<Cx> z(count);
  for (size_t i = 0; i < count; ++i) z[i] = Cx{values[2 * i], values[2 * i + 1]};
  return encode_cx(Chain(log_n, primes, nq), z, scale, level);
}

Pt encode_plaintext(Evaluator& ev, const double* values, size_t count, double scale, uint32_t level) {
  std::vector<Cx> z(count);
  for (size_t i = 0; i < count; ++i) z[i] = Cx{values[2 * i], values[2 * i + 1]};
  return upload_coeffs(ev, encode_cx(Chain(*ev.ctx()), z, scale, level), scale, level);
}

std::vector<StagePlan> plan_boot_stages(const BootParams& bp, int direction) {
  const bool ctos = direction == DIR_COEFF_TO_SLOT;
  auto stages = dft_stages(bp.log_slots, ctos ? bp.ctos_levels : bp.stoc_levels, ctos);
  auto adapted = adapt(stages, direction, ctos ? Cx{1.0 / (double)bp.k_intervals, 0.0} : Cx{1.0 / (2.0 * M_PI), 0.0});
  std::vector<StagePlan> out;
  for (size_t k = 0; k < stages.size(); ++k) {
    Shape sh = stages[k].shape();
    StagePlan p;
    p.d = sh.d;
    p.stride = sh.stride;
    p.offset = sh.offset;
    std::vector<std::vector<Cx>> pre;
    std::vector<bool> zero;
    prerotate(adapted[k].main.window(sh), sh, stages[k].n, pre, zero);
    for (bool z : zero) p.kept.push_back(!z);
    if (adapted[k].has_second) {
      p.has_second = true;
      prerotate(adapted[k].second.window(sh), sh, stages[k].n, pre, zero);
      for (bool z : zero) p.kept2.push_back(!z);
    }
    out.push_back(std::move(p));
  }
  return out;
}

std::vector<int32_t> boot_rotation_steps(const BootParams& bp) {  // linear.rs:432-450, bootstrapper.rs:60-77
  std::set<int32_t> steps;
  for (int inv = 1; inv >= 0; --inv) {
    auto st = dft_stages(bp.log_slots, inv ? bp.ctos_levels : bp.stoc_levels, inv != 0);
    for (auto& s : st) {
      Shape sh = s.shape();
      const int64_t n = (int64_t)s.n;
      for (int32_t v : bsgs_rotation_steps_with_offset(sh.d, sh.stride, sh.offset)) {
        const int64_t r = (((int64_t)v % n) + n) % n;
        if (r) steps.insert((int32_t)r);
      }
    }
  }
  return std::vector<int32_t>(steps.begin(), steps.end());
}

std::vector<double> evalmod_coeffs(const BootParams& bp) {  // evalmod.rs:58-96
  if (!bp.k_intervals || !bp.cheb_degree) throw Error(ST_INVALID_PARAMS, "k_intervals and cheb_degree must be positive");
  auto c = chebyshev_coeffs(evalmod_function, bp, -1.0, 1.0, bp.cheb_degree);
  if (bp.double_angle == 0)
    for (size_t i = 0; i < c.size(); i += 2) c[i] = 0.0;
  return c;
}

std::pair<double, double> boot_stage_scales(const Context& c, const BootParams& bp, double delta) {
  const double q0 = (double)c.primes[0];  // bootstrapper.rs:207-230
  const double evalmod_scale = nominal_scale(c, c.L - bp.ctos_levels, delta);
  return {evalmod_scale, evalmod_scale * delta / q0};
}

std::vector<LtPtr> encode_boot_stages(Evaluator& ev, const BootParams& bp, int direction, double delta) {
  const Context& c = *ev.ctx();
  if (bp.log_slots + 1 != c.log_n) throw Error(ST_INVALID_PARAMS, "bootstrapping needs full packing");
  const uint32_t used = bp.ctos_levels + bp.evalmod_levels + bp.stoc_levels;
  if (used >= c.L) throw Error(ST_INVALID_PARAMS, "the bootstrap bands leave no compute level");
  const bool ctos = direction == DIR_COEFF_TO_SLOT;
  auto stages = dft_stages(bp.log_slots, ctos ? bp.ctos_levels : bp.stoc_levels, ctos);
  auto sc = boot_stage_scales(c, bp, delta);
  const uint32_t start = ctos ? c.L : c.L - used + bp.stoc_levels;
  const double in_scale = ctos ? (double)c.primes[0] : sc.second, out_scale = ctos ? sc.first : delta;
  const Cx factor = ctos ? Cx{1.0 / (double)bp.k_intervals, 0.0} : Cx{1.0 / (2.0 * M_PI), 0.0};
  const size_t l = stages.size();
  if (start < l) throw Error(ST_INVALID_PARAMS, "start level cannot hold the stages");  // linear.rs:595-652
  auto adapted = adapt(stages, direction, factor);
  // diagonal_scales (linear.rs:654-677) over the scale path (linear.rs:572-582)
  const double la = std::log2(in_scale), lb = std::log2(out_scale);
  double s_in = in_scale;
  std::vector<LtPtr> out;
  for (size_t k = 0; k < l; ++k) {
    const double target = k + 1 == l ? out_scale : std::exp2(std::round(la + (lb - la) * (double)(k + 1) / (double)l));
    const uint32_t level = start - (uint32_t)k;
    const double sp = ev.exact_product_scale(level, target) / s_in;
    if (sp < 1048576.0) throw Error(ST_INVALID_PARAMS, "diagonal scale below 2^20");
    Shape sh = stages[k].shape();
    auto lt = std::make_shared<LinearTransform>();
    lt->direction = direction;
    lt->level = level;
    lt->scale = target;
    lt->diags = encode_window(ev, adapted[k].main.window(sh), sh, sp, level);
    if (adapted[k].has_second) {
      lt->has_second = true;
      lt->second = encode_window(ev, adapted[k].second.window(sh), sh, sp, level);
    }
    out.push_back(lt);
    s_in = target;
  }
  return out;
}

}  // namespace ckg
