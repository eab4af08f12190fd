// Layout of the opaque C ABI handles (include/nedy.h), shared by the files that
// implement entry points.
#pragma once
#include "../../include/nedy.h"
#include "engine.cuh"
#include <functional>

struct nedy_ctx {
  nedy::Ctx c;
};
// Green's functions and buffers remember their device, so that they can be
// destroyed after their context.
struct nedy_gf {
  nedy_ctx *ctx;
  int device;
  nedy::DevGF g;
};
struct nedy_buf {
  nedy_ctx *ctx;
  int device;
  void *p;
  long long bytes;
};

struct nedy_predictor {
  nedy_ctx *ctx;
  nedy::Predictor *p;
};

namespace nedy {
// Runs f, maps its exceptions to a nedy_status and records the message for
// nedy_last_error (the same mapping every entry point uses).
int run_guarded(const std::function<void()> &f);
}  // namespace nedy
