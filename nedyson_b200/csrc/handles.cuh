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
  bool host_tri = false;  // les / ret in mapped pinned host memory (cudaFreeHost)
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

// Whole-step bodies shared by the entry points (h_t: device pointers to the nao x nao
// one-body Hamiltonian at tstp).  They throw; callers map the exceptions.
// DecompSimulation::do_tstp (src/molNEsim_decomp_impl.h:85-104): corr_steps iterations.
void decomp_step_fixed(nedy_ctx *ctx, int tstp, nedy_gf *G, nedy_gf *S, nedy_buf *hmf, const double2 *h_t,
                       double mu, int corr_steps, double *err);
// The same with the residual exit, one or two spins.
void step_tol(nedy_ctx *ctx, int tstp, int nspin, nedy_gf *const *G, nedy_gf *const *S, nedy_buf *const *hmf,
              const double2 *const *h_t, const double *mu, int max_corr, double tol, int *iters, double *err_hist);
}  // namespace nedy
