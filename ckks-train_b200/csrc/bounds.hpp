// Opt-in host-side bounds checking of kernel work lists (CKG_CHECK_BOUNDS=1 in the environment).
//
// The library records every device allocation it makes (context scratch, transfer blocks, served
// key copies) and, for a while, the ones it has freed. Before a launch (or before a batch uploads
// its work lists) each buffer a kernel will read or write is checked on the host: a range that
// starts inside a live allocation must end inside it, and a range that starts inside a freed one
// (and no live one) is a use after free. A violation throws before anything is queued. Pointers
// the library did not allocate (a caller's device buffers, the context's tables) pass unchecked.
// Off by default: every check is then one predictable branch.
#pragma once
#include <cstddef>
#include <cstdint>

namespace ckg {
namespace bounds {

bool enabled();
void set_enabled(bool on);  // test hook; the environment variable sets the initial state
void track(const void* p, size_t bytes);
void untrack(const void* p);
// Throws Error(ST_DEVICE, ...) naming `what` when [p, p + bytes) leaves the live allocation it
// starts in, or starts in freed memory.
void check(const void* p, size_t bytes, const char* what);

}  // namespace bounds
}  // namespace ckg
