// Bounds checks of the kernels' work-list entries (bounds.hpp): each entry's buffers with the
// extent its kernel touches, in words of N coefficients per limb. No-ops unless checking is on.
#pragma once
#include "bounds.hpp"
#include "kernels.cuh"

namespace ckg {
namespace bounds {

inline void limb(const void* p, size_t n, const char* what) { check(p, n * 8, what); }
inline void perm(const uint32_t* p, size_t n, const char* what) { check(p, n * 4, what); }

inline void refs(const LimbRef* r, size_t count, size_t n, const char* what) {
  if (!enabled()) return;
  for (size_t i = 0; i < count; ++i) {
    limb(r[i].src, n, what);
    limb(r[i].dst, n, what);
  }
}

inline void refs(const BinRef* r, size_t count, size_t n, const char* what) {
  if (!enabled()) return;
  for (size_t i = 0; i < count; ++i) {
    limb(r[i].a, n, what);
    limb(r[i].b, n, what);
    limb(r[i].out, n, what);
  }
}

inline void refs(const FinRef* r, size_t count, size_t n, const char* what) {
  if (!enabled()) return;
  for (size_t i = 0; i < count; ++i) {
    limb(r[i].x, n, what);
    limb(r[i].t, n, what);
    limb(r[i].add, n, what);
    perm(r[i].add_perm, n, what);
    limb(r[i].out, n, what);
  }
}

inline void refs(const TensorRef* r, size_t count, size_t n, const char* what) {
  if (!enabled()) return;
  for (size_t i = 0; i < count; ++i)
    for (const void* p : {(const void*)r[i].a0, (const void*)r[i].a1, (const void*)r[i].b0, (const void*)r[i].b1,
                          (const void*)r[i].d0, (const void*)r[i].d1, (const void*)r[i].d2})
      limb(p, n, what);
}

inline void refs(const GatherRef* r, size_t count, size_t n, const char* what) {
  if (!enabled()) return;
  for (size_t i = 0; i < count; ++i) {
    limb(r[i].src, n, what);
    limb(r[i].dst, n, what);
    perm(r[i].perm, n, what);
  }
}

// Conversion jobs from n_src sources: source limb j at src + j * src_stride, target t at
// dst + t * dst_stride.
inline void refs(const ConvJob* r, size_t count, int n_src, size_t n, const char* what) {
  if (!enabled()) return;
  for (size_t i = 0; i < count; ++i) {
    if (n_src > 0) check(r[i].src, ((size_t)(n_src - 1) * r[i].src_stride + n) * 8, what);
    if (r[i].n_dst > 0) check(r[i].dst, ((size_t)(r[i].n_dst - 1) * r[i].dst_stride + n) * 8, what);
  }
}

// Inner-product jobs: the input's l+1 limbs, each digit's converted limbs (the primes of Q_l * P
// outside the digit), the key's ndig parts of b and a, the two accumulators of l+1+k limbs.
inline void refs(const IpJob* r, size_t count, int alpha, int k, size_t n, const char* what) {
  if (!enabled()) return;
  for (size_t i = 0; i < count; ++i) {
    const IpJob& j = r[i];
    const size_t l1 = (size_t)j.level + 1, ext = l1 + (size_t)k;
    check(j.in, l1 * n * 8, what);
    for (int d = 0; d < j.ndig && d < kMaxDigits; ++d) {
      const size_t start = (size_t)d * alpha, end = start + alpha < l1 ? start + alpha : l1;
      check(j.conv[d], (ext - (end - start)) * n * 8, what);
    }
    check(j.key, (size_t)2 * j.ndig * ((size_t)j.key_q + k) * n * 8, what);
    check(j.out_b, ext * n * 8, what);
    check(j.out_a, ext * n * 8, what);
    perm(j.perm, n, what);
  }
}

}  // namespace bounds
}  // namespace ckg
