// Opt-in bounds checking of kernel work lists: the allocation registry (bounds.hpp).
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <iterator>
#include <map>
#include <mutex>
#include <string>

#include "bounds.hpp"
#include "engine.hpp"

namespace ckg {
namespace bounds {
namespace {

std::atomic<bool> g_on{[] {
  const char* v = std::getenv("CKG_CHECK_BOUNDS");
  return v && v[0] && v[0] != '0';
}()};

constexpr size_t kFreedKept = 4096;  // freed ranges remembered for use-after-free reports

struct Registry {
  std::mutex mu;
  std::map<uintptr_t, size_t> live;                    // start -> bytes
  std::map<uintptr_t, size_t> freed;                    // start -> bytes (recent frees)
  std::deque<uintptr_t> freed_order;                    // oldest first
};

Registry& reg() {
  static Registry r;
  return r;
}

// The range of `m` that contains address a, or m.end().
std::map<uintptr_t, size_t>::const_iterator containing(const std::map<uintptr_t, size_t>& m, uintptr_t a) {
  auto it = m.upper_bound(a);
  if (it == m.begin()) return m.end();
  --it;
  return a < it->first + it->second ? it : m.end();
}

std::string hex(uintptr_t a) {
  char b[32];
  std::snprintf(b, sizeof b, "0x%llx", (unsigned long long)a);
  return b;
}

}  // namespace

bool enabled() { return g_on.load(std::memory_order_relaxed); }

void set_enabled(bool on) { g_on.store(on); }

void track(const void* p, size_t bytes) {
  if (!enabled() || !p || !bytes) return;
  Registry& r = reg();
  std::lock_guard<std::mutex> lk(r.mu);
  const uintptr_t a = (uintptr_t)p;
  r.live[a] = bytes;
  // a new allocation over a remembered free: that memory is live again
  for (auto it = r.freed.lower_bound(a); it != r.freed.end() && it->first < a + bytes;) it = r.freed.erase(it);
  auto before = containing(r.freed, a);
  if (before != r.freed.end()) r.freed.erase(before->first);
}

void untrack(const void* p) {
  if (!enabled() || !p) return;
  Registry& r = reg();
  std::lock_guard<std::mutex> lk(r.mu);
  const uintptr_t a = (uintptr_t)p;
  auto it = r.live.find(a);
  if (it == r.live.end()) return;
  r.freed[a] = it->second;
  r.freed_order.push_back(a);
  r.live.erase(it);
  while (r.freed_order.size() > kFreedKept) {
    r.freed.erase(r.freed_order.front());
    r.freed_order.pop_front();
  }
}

void check(const void* p, size_t bytes, const char* what) {
  if (!enabled() || !p) return;
  Registry& r = reg();
  std::lock_guard<std::mutex> lk(r.mu);
  const uintptr_t a = (uintptr_t)p;
  auto it = containing(r.live, a);
  if (it != r.live.end()) {
    if (a + bytes > it->first + it->second)
      throw Error(ST_DEVICE, std::string("bounds check: ") + what + " [" + hex(a) + ", +" + std::to_string(bytes) +
                                 ") runs past its allocation [" + hex(it->first) + ", +" +
                                 std::to_string(it->second) + ")");
    return;
  }
  auto f = containing(r.freed, a);
  if (f != r.freed.end())
    throw Error(ST_DEVICE, std::string("bounds check: ") + what + " at " + hex(a) + " lies in freed memory [" +
                               hex(f->first) + ", +" + std::to_string(f->second) + ")");
}

}  // namespace bounds
}  // namespace ckg
