// Key switching without any device allocation, for callers that cannot allocate device
// memory at request time: a serving process that reserved its whole HBM budget up front
// and must not have a request fail or stall on an allocation, or an embedding runtime that
// owns every device allocation and forbids a library from allocating behind its back.
//
// The working space of the key switch (the coefficient copy of the input, the converted
// digits, both accumulators and the ModDown temporaries) lives in one file-scope device
// array of fixed size, shared by every call in the process. Its device address is looked
// up with the device current on every call made outside stream capture, so a context that
// was reset and re-created (the module loaded again, possibly at another address) gets the
// new address. A call made while its stream is capturing uses the address found by the
// last call outside capture on that device, so the first call on a device must come before
// any capture.
#include <mutex>

#include "../../include/ckg.h"
#include "handles.hpp"

namespace {

// 16 Mi words = 128 MiB: enough for N = 2^16 with 24 data + 8 special primes and 3 digits
// at the top level (112 MiB). Every GPU that loads this library holds it until exit.
constexpr size_t kScratchWords = (size_t)1 << 24;

static __device__ __align__(256) uint64_t g_ks_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint64_t* g_scratch_addr[kMaxDevices] = {};

// Device address of g_ks_scratch on the current device (host code may not use the symbol
// itself as an address: it names a host-side stand-in).
uint64_t* scratch_on(int device, cudaStream_t st) {
  std::lock_guard<std::mutex> lk(g_mu);
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) cs = cudaStreamCaptureStatusNone;
  if (cs == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_ks_scratch);
    if (e != cudaSuccess) ckg::throw_cuda(e, "cudaGetSymbolAddress(g_ks_scratch)");
    g_scratch_addr[device] = (uint64_t*)p;
  } else if (!g_scratch_addr[device]) {
    throw ckg::Error(CKG_INVALID_PARAMS,
                     "the first allocation-free key switch on a device must come before any stream capture");
  }
  return g_scratch_addr[device];
}

}  // namespace

extern "C" int ckg_key_switch_noalloc(ckg_ctx* ctx, const ckg_key* key, const uint64_t* in, uint32_t level,
                                      uint64_t* out_b, uint64_t* out_a) {
  try {
    if (!ctx || !ctx->c) throw ckg::Error(CKG_INVALID_PARAMS, "null context");
    ckg::Context& c = *ctx->c;
    if (level > c.L) throw ckg::Error(CKG_INVALID_PARAMS, "level above max_level");
    const size_t need = ckg::key_switch_scratch_words(c, level);
    if (need > kScratchWords)
      throw ckg::Error(CKG_INVALID_PARAMS, "key switch at this level needs " + std::to_string(need * 8) +
                                               " bytes of working space; the fixed scratch holds " +
                                               std::to_string(kScratchWords * 8));
    if (!key || !key->k) throw ckg::Error(CKG_INVALID_PARAMS, "null key");
    if (c.device < 0 || c.device >= kMaxDevices) throw ckg::Error(CKG_INVALID_PARAMS, "device ordinal out of range");
    c.activate();
    uint64_t* scratch = scratch_on(c.device, c.stream);
    ckg::KsJob j;
    j.in = in;
    j.key = key->k.get();
    j.out_b = out_b;
    j.out_a = out_a;
    ckg::key_switch_with_scratch(c, j, level, scratch);
    CKG_CUDA(cudaGetLastError());
    return CKG_OK;
  } catch (const ckg::Error& e) {
    ckg_set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    ckg_set_last_error(e.what());
    return CKG_DEVICE;
  }
}
