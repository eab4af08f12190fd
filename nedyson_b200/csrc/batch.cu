// Batched time stepping of independent density-fitted GF2 simulations of uneven size.
//
// Every instance keeps its own context (CUDA stream, workspace, cached inverses and
// mixing kernel), Green's functions, mean field and one-body Hamiltonians.  One batched
// step runs DecompSimulation::do_tstp (reference src/molNEsim_decomp_impl.h:85-104) of
// every instance; a pool of native worker threads takes the instances largest first and
// issues each one's step on that instance's stream.  Kernels of different instances then
// run concurrently on the GPU: the many small launches of the small instances fill the
// SMs that the large instances leave idle, and the host round trips inside one instance's
// step (residual norms, pivot status) stall only its own worker.
#include "handles.cuh"
#include <algorithm>
#include <atomic>
#include <exception>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

struct nedy_batch {
  std::vector<nedy_batch_instance> inst;
  std::vector<int> order;  // instances by decreasing cost
  int workers = 1;
};

using namespace nedy;

extern "C" {

int nedy_batch_create(const nedy_batch_instance *inst, int n, int workers, nedy_batch **out) {
  return run_guarded([&] {
    NEDY_REQUIRE(inst && n > 0 && out, "bad argument");
    auto *b = new nedy_batch;
    b->inst.assign(inst, inst + n);
    for (int i = 0; i < n; i++) {
      const nedy_batch_instance &x = inst[i];
      if (!(x.ctx && x.G && x.Sigma && x.hmf && x.h_all)) {
        delete b;
        throw ArgError("nedy_batch_create: instance " + std::to_string(i) + " has a null handle");
      }
      const i64 es = x.G->g.es, rows = (i64)x.G->g.nt + 1;
      if (x.h_all->bytes < rows * es * 16 || x.hmf->bytes < rows * es * 16 || x.Sigma->g.nao != x.G->g.nao) {
        delete b;
        throw ArgError("nedy_batch_create: instance " + std::to_string(i) +
                       " has buffers smaller than (nt+1) x nao x nao or mismatched sizes");
      }
    }
    b->order.resize(n);
    std::iota(b->order.begin(), b->order.end(), 0);
    // cost of a step grows like nao^5 (the exchange contraction): largest first
    std::stable_sort(b->order.begin(), b->order.end(),
                     [&](int a, int c) { return inst[a].G->g.nao > inst[c].G->g.nao; });
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    b->workers = workers > 0 ? std::min(workers, n) : std::min({n, hw, 16});
    *out = b;
  });
}

int nedy_batch_destroy(nedy_batch *b) {
  return run_guarded([&] { delete b; });
}

int nedy_batch_tstp(nedy_batch *b, int tstp, int corr_steps, double tol, int *iters) {
  return run_guarded([&] {
    NEDY_REQUIRE(b, "null batch");
    NEDY_REQUIRE(corr_steps >= 1 && tol >= 0.0, "corr_steps must be >= 1 and tol >= 0");
    const int n = (int)b->inst.size();
    for (const auto &x : b->inst)
      NEDY_REQUIRE(tstp > x.ctx->c.k && tstp <= x.G->g.nt, "nedy_batch_tstp: tstp outside (k, nt]");
    std::atomic<int> next{0};
    std::mutex emu;
    std::exception_ptr first;
    int first_idx = -1;
    auto work = [&]() {
      for (;;) {
        const int q = next.fetch_add(1);
        if (q >= n) return;
        const int i = b->order[q];
        const nedy_batch_instance &x = b->inst[i];
        try {
          const double2 *h = (const double2 *)x.h_all->p + (i64)tstp * x.G->g.es;
          int it = corr_steps;
          if (tol > 0.0) {
            nedy_gf *G[1] = {x.G}, *S[1] = {x.Sigma};
            nedy_buf *hm[1] = {x.hmf};
            const double2 *ht[1] = {h};
            step_tol(x.ctx, tstp, 1, G, S, hm, ht, &x.mu, corr_steps, tol, &it, nullptr);
          } else {
            decomp_step_fixed(x.ctx, tstp, x.G, x.Sigma, x.hmf, h, x.mu, corr_steps, nullptr);
          }
          if (iters) iters[i] = it;
        } catch (...) {
          std::lock_guard<std::mutex> lk(emu);
          if (!first) {
            first = std::current_exception();
            first_idx = i;
          }
          next.store(n);  // stop handing out further instances
        }
      }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < b->workers; w++) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    if (first) {
      try {
        std::rethrow_exception(first);
      } catch (const ArgError &e) {
        throw ArgError("instance " + std::to_string(first_idx) + ": " + e.what());
      } catch (const CudaError &e) {
        throw CudaError("instance " + std::to_string(first_idx) + ": " + e.what());
      }
    }
  });
}

}  // extern "C"
