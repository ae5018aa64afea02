// Definitions of the opaque C ABI handles (include/ckg.h), shared by the C ABI sources.
#pragma once
#include <memory>

#include "batch.hpp"
#include "boot.hpp"
#include "evaluator.hpp"
#include "serve.hpp"

struct ckg_ctx {
  std::unique_ptr<ckg::Context> c;
};
struct ckg_key {
  ckg::KeyPtr k;
};
struct ckg_eval {
  std::unique_ptr<ckg::Evaluator> e;
};
struct ckg_ct {
  ckg::Ct c;
};
struct ckg_pt {
  ckg::Pt p;
};
struct ckg_batch {
  std::unique_ptr<ckg::Batch> b;
  ckg_eval* ev;
};
struct ckg_lt {
  ckg::LtPtr lt;
};
struct ckg_boot {
  std::unique_ptr<ckg::Bootstrapper> b;
};
struct ckg_server {
  std::unique_ptr<ckg::Server> s;
  uint64_t budget = 0;
};

// Sets the calling thread's message returned by ckg_last_error().
void ckg_set_last_error(const char* msg);
