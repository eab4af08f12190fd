// C ABI (include/nedy.h): handles, memory, and the public entry points.
#include "handles.cuh"
#include "sigma.cuh"
#include "split_gemm.cuh"
#include "predictor.cuh"
#include <cstring>
#include <cstdlib>
#include <string>
#include <vector>

using namespace nedy;

namespace nedy {

std::atomic<unsigned long long> g_launches{0};

// Optional per-phase device timing of the whole-step entry points (CUDA events
// on the engine stream): predictor, mean field, self-energy, Dyson step.
struct PhaseTimer {
  Ctx &c;
  std::vector<std::pair<int, cudaEvent_t>> marks;
  explicit PhaseTimer(Ctx &cx) : c(cx) {}
  void mark(int phase) {
    if (!c.timing) return;
    cudaEvent_t e;
    NEDY_CUDA(cudaEventCreate(&e));
    NEDY_CUDA(cudaEventRecord(e, c.stream));
    marks.push_back({phase, e});
  }
  // phase p runs from its mark to the next mark
  void collect() {
    if (!c.timing || marks.empty()) return;
    NEDY_CUDA(cudaEventSynchronize(marks.back().second));
    for (size_t i = 0; i + 1 < marks.size(); i++) {
      float ms = 0;
      NEDY_CUDA(cudaEventElapsedTime(&ms, marks[i].second, marks[i + 1].second));
      if (marks[i].first >= 0 && marks[i].first < 4) c.phase_ms[marks[i].first] += ms;
    }
    for (auto &m : marks) cudaEventDestroy(m.second);
    marks.clear();
  }
};

Arena::~Arena() {
  for (auto &b : blocks_) cudaFree(b.p);
}
size_t Arena::capacity() const {
  size_t s = 0;
  for (auto &b : blocks_) s += b.cap;
  return s;
}
char *Arena::alloc_block(size_t bytes) {
  char *p = nullptr;
  cudaError_t e = stream_ ? cudaMallocAsync((void **)&p, bytes, stream_) : cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw CudaError("workspace allocation of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
  }
  return p;
}
void Arena::reset() {
  if (blocks_.size() > 1) {
    // the blocks were used by work queued on stream_ only: free and reallocate in its order
    const size_t total = capacity() + capacity() / 2;
    for (auto &b : blocks_) {
      if (stream_)
        NEDY_CUDA(cudaFreeAsync(b.p, stream_));
      else
        cudaFree(b.p);
    }
    blocks_.clear();
    char *p = alloc_block(total);
    blocks_.push_back({p, total, 0});
  }
  for (auto &b : blocks_) b.top = 0;
}
void *Arena::get(size_t bytes) {
  size_t need = ((bytes + 255) / 256) * 256;
  if (need == 0) need = 256;
  if (!blocks_.empty() && blocks_.back().top + need <= blocks_.back().cap) {
    Block &b = blocks_.back();
    void *p = b.p + b.top;
    b.top += need;
    return p;
  }
  const size_t cap = std::max(need, (size_t)64 << 20);
  char *p = alloc_block(cap);
  blocks_.push_back({p, cap, need});
  return p;
}

Ctx::~Ctx() {
  auto f = [](void *p) { if (p) cudaFree(p); };
  f(Vija); f(Viaj); f(Vaij); f(Vmbq); f(Vp); f(Vanj_p); f(Vjkb_p); f(Vila_p); f(rowcopy); f(d_maxdiff); f(pred_corr); f(U); f(Uexch); f(mixK); f(mixK_alt); f(Minv); f(greg); f(small);
  if (stream) cudaStreamDestroy(stream);
  delete aux;
}

// full-U Hartree-Fock (molHFSolver.cpp:35-56): hmf_ij += sum_kl rho_kl (2 U_ijkl - U_ilkj)
__global__ void hf_full_kernel(int N, const double *U, const double2 *rho, double2 *h) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= N * N) return;
  const int i = e / N, j = e - (e / N) * N;
  double2 acc = czero();
  for (int k = 0; k < N; k++)
    for (int l = 0; l < N; l++) {
      const double u = 2.0 * U[((i64)(i * N + j) * N + k) * N + l] - U[((i64)(i * N + l) * N + k) * N + j];
      acc = cadd(acc, cscale(rho[k * N + l], u));
    }
  h[e] = cadd(h[e], acc);
}
void hf_full(Ctx &c, double2 *hmf_T, const double2 *rho) {
  NEDY_REQUIRE(c.U, "hf_full: U not set");
  int N = c.u_nao;
  hf_full_kernel<<<(N * N + 127) / 128, 128, 0, c.stream>>>(N, c.U, rho, hmf_T);
  NEDY_CHECK_LAUNCH();
}

// max |a - b| over n complex values (non-negative doubles order like their bit patterns)
__global__ void maxdiff_kernel(i64 n, const double2 *a, const double2 *b, unsigned long long *out) {
  double m = 0.0;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    const double2 x = a[i], y = b[i];
    m = fmax(m, hypot(x.x - y.x, x.y - y.y));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// The new row of step T (les column, ret row, tv row) as three contiguous block ranges.
struct RowRanges {
  double2 *p[3];
  i64 n[3];
};
static RowRanges row_ranges(const DevGF &g, int T) {
  const i64 es = (i64)g.nao * g.nao;
  return RowRanges{{g.lesptr(0, T), g.retptr(T, 0), g.tvptr(T, 0)}, {(T + 1) * es, (T + 1) * es, (g.ntau + 1) * es}};
}
// the copy of spin `slot` (0 or 1) starts at slot * (elements of one row)
static i64 row_len(const DevGF &g, int T) {
  RowRanges r = row_ranges(g, T);
  return r.n[0] + r.n[1] + r.n[2];
}
static void save_row(Ctx &c, const DevGF &g, int T, int slot = 0) {
  RowRanges r = row_ranges(g, T);
  const i64 tot = r.n[0] + r.n[1] + r.n[2];
  if (c.rowcopy_cap < 2 * tot) {
    // rows grow with T: size the copy for the longest row of the run, so that it is
    // allocated once (a cudaFree per step would synchronise the whole device)
    const i64 cap = std::max<i64>(2 * tot, 2 * row_len(g, g.nt));
    if (c.rowcopy) cudaFree(c.rowcopy);
    c.rowcopy = nullptr;
    NEDY_CUDA(cudaMalloc(&c.rowcopy, sizeof(double2) * cap));
    c.rowcopy_cap = cap;
  }
  i64 o = slot * tot;
  for (int k = 0; k < 3; k++) {
    NEDY_CUDA(cudaMemcpyAsync(c.rowcopy + o, r.p[k], sizeof(double2) * r.n[k], cudaMemcpyDefault, c.stream));
    o += r.n[k];
  }
}
static double row_change(Ctx &c, const DevGF &g, int T, int slot = 0) {
  if (!c.d_maxdiff) NEDY_CUDA(cudaMalloc(&c.d_maxdiff, sizeof(unsigned long long)));
  NEDY_CUDA(cudaMemsetAsync(c.d_maxdiff, 0, sizeof(unsigned long long), c.stream));
  RowRanges r = row_ranges(g, T);
  i64 o = slot * (r.n[0] + r.n[1] + r.n[2]);
  for (int k = 0; k < 3; k++) {
    const unsigned blocks = (unsigned)std::min<i64>((r.n[k] + 255) / 256, 148 * 8);
    maxdiff_kernel<<<blocks, 256, 0, c.stream>>>(r.n[k], r.p[k], c.rowcopy + o, c.d_maxdiff);
    NEDY_CHECK_LAUNCH();
    o += r.n[k];
  }
  unsigned long long h = 0;
  NEDY_CUDA(cudaMemcpyAsync(&h, c.d_maxdiff, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
  NEDY_CUDA(cudaStreamSynchronize(c.stream));
  return __builtin_bit_cast(double, h);
}

} // namespace nedy

namespace {
thread_local std::string g_err;

template <class F>
int guard(F &&f) {
  try {
    f();
    return NEDY_OK;
  } catch (const ArgError &e) {
    g_err = e.what();
    if (g_err.find("singular") != std::string::npos) return NEDY_ERR_SINGULAR;
    return NEDY_ERR_ARG;
  } catch (const CudaError &e) {
    g_err = e.what();
    if (g_err.find("timed out") != std::string::npos) return NEDY_ERR_TIMEOUT;
    if (g_err.find("out of memory") != std::string::npos || g_err.find("allocation") != std::string::npos)
      return NEDY_ERR_OOM;
    return NEDY_ERR_CUDA;
  } catch (const std::exception &e) {
    g_err = e.what();
    return NEDY_ERR_STATE;
  } catch (...) {
    g_err = "unknown error";
    return NEDY_ERR_STATE;
  }
}

void set_dev(nedy_ctx *ctx) { NEDY_CUDA(cudaSetDevice(ctx->c.device)); }
} // namespace

int nedy::run_guarded(const std::function<void()> &f) { return guard(f); }

namespace {

double2 *comp_ptr(const nedy_gf *g, int comp, i64 &nblocks) {
  const DevGF &d = g->g;
  NEDY_REQUIRE(!d.win || (comp != NEDY_LES && comp != NEDY_RET),
               "windowed green_func: lesser and retarded blocks are addressed a time step at a time");
  switch (comp) {
    case NEDY_LES: nblocks = d.nt >= 0 ? d.ntri() : 0; return d.les;
    case NEDY_RET: nblocks = d.nt >= 0 ? d.ntri() : 0; return d.ret;
    case NEDY_TV: nblocks = (i64)(d.nt + 1) * (d.ntau + 1); return d.tv;
    case NEDY_MAT: nblocks = d.ntau + 1; return d.mat;
  }
  throw ArgError("unknown component");
}

double2 *hmf_row(const nedy_buf *b, const nedy_ctx *ctx, int tstp, int nao) {
  const i64 es = (i64)nao * nao;
  NEDY_REQUIRE(b && b->bytes >= (i64)(tstp + 1) * es * 16, "hmf buffer too small for tstp");
  return (double2 *)b->p + (i64)tstp * es;
}
} // namespace

extern "C" {

int nedy_abi_version(void) { return NEDY_ABI_VERSION; }

const char *nedy_status_string(int s) {
  switch (s) {
    case NEDY_OK: return "ok";
    case NEDY_ERR_ARG: return "bad argument";
    case NEDY_ERR_CUDA: return "CUDA error";
    case NEDY_ERR_NOCONV: return "not converged";
    case NEDY_ERR_TIMEOUT: return "device wait timed out";
    case NEDY_ERR_OOM: return "out of device memory";
    case NEDY_ERR_STATE: return "call out of order";
    case NEDY_ERR_SINGULAR: return "singular matrix";
  }
  return "unknown status";
}

const char *nedy_last_error(void) { return g_err.c_str(); }

int nedy_ctx_create(const nedy_config *cfg, nedy_ctx **out) {
  return guard([&] {
    NEDY_REQUIRE(cfg && out, "null argument");
    NEDY_REQUIRE(cfg->nt >= cfg->k && cfg->k >= 1 && cfg->ntau >= 2 && cfg->nao >= 1, "bad sizes in nedy_config");
    NEDY_REQUIRE(cfg->beta > 0 && cfg->dt > 0, "beta and dt must be positive");
    int ndev = 0;
    NEDY_CUDA(cudaGetDeviceCount(&ndev));
    NEDY_REQUIRE(cfg->device >= 0 && cfg->device < ndev, "no such CUDA device");
    auto *h = new nedy_ctx;
    Ctx &c = h->c;
    c.device = cfg->device;
    c.nt = cfg->nt; c.ntau = cfg->ntau; c.nao = cfg->nao; c.k = cfg->k;
    c.beta = cfg->beta; c.dt = cfg->dt;
    if (cfg->workspace_bytes > 0) c.ws_budget = cfg->workspace_bytes;
    try {
      NEDY_CUDA(cudaSetDevice(c.device));
      NEDY_CUDA(cudaStreamCreate(&c.stream));
      c.ws.set_stream(c.stream);
      c.W = make_weights(c.k);
      c.col = make_colloc(c.ntau);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

int nedy_ctx_destroy(nedy_ctx *ctx) {
  return guard([&] {
    if (!ctx) return;
    cudaSetDevice(ctx->c.device);
    cudaStreamSynchronize(ctx->c.stream);
    delete ctx;
  });
}

int nedy_ctx_synchronize(nedy_ctx *ctx) {
  return guard([&] {
    NEDY_REQUIRE(ctx, "null context");
    NEDY_CUDA(cudaStreamSynchronize(ctx->c.stream));
  });
}

int nedy_ctx_stream(nedy_ctx *ctx, void **stream) {
  return guard([&] {
    NEDY_REQUIRE(ctx && stream, "null argument");
    *stream = (void *)ctx->c.stream;
  });
}

int nedy_ctx_set_precision(nedy_ctx *ctx, int mode) {
  return guard([&] {
    NEDY_REQUIRE(ctx, "null context");
    NEDY_REQUIRE(mode == NEDY_PREC_FP64 || mode == NEDY_PREC_SPLIT_BF16X3 || mode == NEDY_PREC_SPLIT_BF16X2,
                 "unknown precision mode");
    ctx->c.precision = mode;
  });
}

int nedy_split_autotune(int on) {
  return guard([&] { split_autotune(on != 0); });
}

int nedy_split_tune_pending(int *classes) {
  return guard([&] {
    NEDY_REQUIRE(classes, "null argument");
    *classes = split_tune_pending();
  });
}

int nedy_split_tune_report(char *buf, int len) {
  return guard([&] {
    NEDY_REQUIRE(buf && len > 0, "bad argument");
    const std::string r = split_tune_report();
    const size_t n = std::min<size_t>(r.size(), (size_t)len - 1);
    memcpy(buf, r.data(), n);
    buf[n] = 0;
  });
}

int nedy_sigma_chunk_plan(int nao, int naux, long long budget, int precision, int real_symmetric, int sms, int *chunk,
                          int *sub) {
  return guard([&] {
    NEDY_REQUIRE(chunk && sub, "null argument");
    NEDY_REQUIRE(nao > 0 && naux > 0 && budget > 0 && sms > 0, "bad sizes");
    NEDY_REQUIRE(precision == NEDY_PREC_FP64 || precision == NEDY_PREC_SPLIT_BF16X3 ||
                     precision == NEDY_PREC_SPLIT_BF16X2,
                 "unknown precision mode");
    chunk_plan(nao, naux, budget, precision != NEDY_PREC_FP64, real_symmetric != 0,
               precision == NEDY_PREC_SPLIT_BF16X2 ? 2 : 3, sms, *chunk, *sub);
  });
}

int nedy_split_gemm_check(int device, int M, int N, int K, int nb, int a_cplx, int b_cplx, int conj_a, int conj_b,
                          int npieces, int out_pieces, int accumulate, int tile_n, int stages, int k_block, int kdiv,
                          int persistent, unsigned long long seed, double *rel_err) {
  return guard([&] {
    NEDY_REQUIRE(rel_err, "null argument");
    NEDY_CUDA(cudaSetDevice(device));
    SplitCheck k;
    k.M = M; k.N = N; k.K = K; k.nb = nb;
    k.a_cplx = a_cplx; k.b_cplx = b_cplx; k.conjA = conj_a; k.conjB = conj_b; k.np = npieces;
    k.out_pieces = out_pieces; k.accumulate = accumulate;
    k.bn = tile_n; k.stages = stages; k.bk = k_block; k.kdiv = kdiv; k.persist = persistent;
    k.seed = seed;
    k.alpha = 0.75;
    cudaStream_t st = nullptr;
    NEDY_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    try {
      *rel_err = split_gemm_check(k, st);
    } catch (...) {
      cudaStreamDestroy(st);
      throw;
    }
    cudaStreamDestroy(st);
  });
}

int nedy_split_stats(int on, double *pipe_flops, double *ms) {
  return guard([&] { split_stats(on != 0, pipe_flops, ms); });
}

int nedy_ctx_set_timing(nedy_ctx *ctx, int on) {
  return guard([&] {
    NEDY_REQUIRE(ctx, "null context");
    ctx->c.timing = on != 0;
    for (double &v : ctx->c.phase_ms) v = 0;
  });
}

int nedy_dense_solve(nedy_ctx *ctx, int n, int nrhs, int nb, const double *A, double *B) {
  return guard([&] {
    NEDY_REQUIRE(ctx && A && B, "null argument");
    NEDY_REQUIRE(n > 0 && nrhs > 0 && nb > 0, "sizes must be positive");
    set_dev(ctx);
    Ctx &c = ctx->c;
    c.ws.reset();
    const i64 sa = (i64)n * n, sb = (i64)n * nrhs;
    double2 *dA = c.ws.alloc<double2>(sa * nb), *dB = c.ws.alloc<double2>(sb * nb);
    NEDY_CUDA(cudaMemcpyAsync(dA, A, sizeof(double2) * sa * nb, cudaMemcpyHostToDevice, c.stream));
    NEDY_CUDA(cudaMemcpyAsync(dB, B, sizeof(double2) * sb * nb, cudaMemcpyHostToDevice, c.stream));
    gj_public(c, n, nrhs, nb, dA, sa, dB, sb);
    check_status(c);
    NEDY_CUDA(cudaMemcpyAsync(B, dB, sizeof(double2) * sb * nb, cudaMemcpyDeviceToHost, c.stream));
    NEDY_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int nedy_ctx_inject_split_error(nedy_ctx *ctx, int code) {
  return guard([&] {
    NEDY_REQUIRE(ctx && code != 0, "null context or zero code");
    set_dev(ctx);
    split_gemm_set_error(ctx->c.stream, code);
  });
}

int nedy_ctx_phase_times(const nedy_ctx *ctx, double *ms4) {
  return guard([&] {
    NEDY_REQUIRE(ctx && ms4, "null argument");
    for (int i = 0; i < 4; i++) ms4[i] = ctx->c.phase_ms[i];
  });
}

unsigned long long nedy_launch_count(void) { return g_launches.load(); }

int nedy_collocation_nodes(const nedy_ctx *ctx, double *x, double *w) {
  return guard([&] {
    NEDY_REQUIRE(ctx, "null context");
    if (x) std::memcpy(x, ctx->c.col.x.data(), sizeof(double) * ctx->c.col.x.size());
    if (w) std::memcpy(w, ctx->c.col.w.data(), sizeof(double) * ctx->c.col.w.size());
  });
}

static int gf_create(nedy_ctx *ctx, int nt, int ntau, int nao, int sig, int window, nedy_gf **out,
                     bool host_tri = false) {
  return guard([&] {
    NEDY_REQUIRE(ctx && out, "null argument");
    NEDY_REQUIRE(nao > 0 && nt >= -1 && ntau >= 0 && sig * sig == 1, "green_func: bad sizes (greens.cpp:35)");
    NEDY_REQUIRE(window == 0 || (window >= NEDY_GF_MIN_WINDOW && nt >= 0),
                 "green_func: a window holds at least NEDY_GF_MIN_WINDOW time steps");
    set_dev(ctx);
    auto *g = new nedy_gf;
    g->ctx = ctx;
    g->device = ctx->c.device;
    DevGF &d = g->g;
    d.nt = nt; d.ntau = ntau; d.nao = nao; d.sig = sig; d.es = (i64)nao * nao;
    d.win = window > nt ? 0 : window;  // a window as long as the run is the full triangle
    g->host_tri = host_tri;
    // triangle in pinned host memory mapped into the device's address space (unified
    // addressing: the device pointer is the host pointer); cleared by the device
    auto alloc_host = [&](double2 *&p, i64 nblk) {
      if (nblk <= 0) { p = nullptr; return; }
      void *h = nullptr;
      cudaError_t e = cudaHostAlloc(&h, sizeof(double2) * nblk * d.es, cudaHostAllocMapped | cudaHostAllocPortable);
      if (e != cudaSuccess) {
        cudaGetLastError();
        throw CudaError(std::string("green_func host history allocation failed: ") + cudaGetErrorString(e));
      }
      void *dp = nullptr;
      e = cudaHostGetDevicePointer(&dp, h, 0);
      if (e != cudaSuccess || dp != h) {
        cudaGetLastError();
        cudaFreeHost(h);
        throw CudaError("green_func host history: the mapped pointer differs from the host pointer (no unified addressing)");
      }
      p = (double2 *)dp;
      memset_sync(p, sizeof(double2) * nblk * d.es, ctx->c.stream);
    };
    auto alloc = [&](double2 *&p, i64 nblk) {
      if (nblk <= 0) { p = nullptr; return; }
      cudaError_t e = cudaMalloc(&p, sizeof(double2) * nblk * d.es);
      if (e != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        throw CudaError(std::string("green_func allocation failed: ") + cudaGetErrorString(e));
      }
      memset_sync(p, sizeof(double2) * nblk * d.es, ctx->c.stream);
    };
    try {
      alloc(d.mat, ntau + 1);
      if (nt >= 0) {
        if (host_tri) {
          alloc_host(d.les, d.nstore());
          alloc_host(d.ret, d.nstore());
        } else {
          alloc(d.les, d.nstore());
          alloc(d.ret, d.nstore());
        }
        alloc(d.tv, (i64)(nt + 1) * (ntau + 1));
      }
    } catch (...) {
      auto tri_free = [&](double2 *p) { if (p) { if (host_tri) cudaFreeHost(p); else cudaFree(p); } };
      if (d.mat) cudaFree(d.mat);
      tri_free(d.les);
      tri_free(d.ret);
      if (d.tv) cudaFree(d.tv);
      delete g;
      throw;
    }
    *out = g;
  });
}

int nedy_gf_create(nedy_ctx *ctx, int nt, int ntau, int nao, int sig, nedy_gf **out) {
  return gf_create(ctx, nt, ntau, nao, sig, 0, out);
}

int nedy_gf_create_windowed(nedy_ctx *ctx, int nt, int ntau, int nao, int sig, int window, nedy_gf **out) {
  return gf_create(ctx, nt, ntau, nao, sig, window, out);
}

int nedy_gf_create_host_history(nedy_ctx *ctx, int nt, int ntau, int nao, int sig, nedy_gf **out) {
  return gf_create(ctx, nt, ntau, nao, sig, 0, out, true);
}

int nedy_gf_host_history(const nedy_gf *g, int *host) {
  return guard([&] {
    NEDY_REQUIRE(g && host, "null argument");
    *host = g->host_tri ? 1 : 0;
  });
}

int nedy_gf_window(const nedy_gf *g, int *window) {
  return guard([&] {
    NEDY_REQUIRE(g && window, "null argument");
    *window = g->g.win;
  });
}

int nedy_gf_destroy(nedy_gf *g) {
  return guard([&] {
    if (!g) return;
    // cudaFree waits for the device; the context may already be gone
    cudaSetDevice(g->device);
    if (g->g.mat) cudaFree(g->g.mat);
    if (g->host_tri) {
      if (g->g.les) cudaFreeHost(g->g.les);
      if (g->g.ret) cudaFreeHost(g->g.ret);
    } else {
      if (g->g.les) cudaFree(g->g.les);
      if (g->g.ret) cudaFree(g->g.ret);
    }
    if (g->g.tv) cudaFree(g->g.tv);
    delete g;
  });
}

// Windowed lesser / retarded storage: the block range [first, first + nb) of the packed
// triangle must lie in one retarded row / lesser column t, which must be in the window.
double2 *window_range(const nedy_gf *g, int comp, i64 first, i64 nb) {
  const DevGF &d = g->g;
  i64 t = (i64)((std::sqrt(8.0 * (double)first + 1.0) - 1.0) / 2.0);
  while (t * (t + 1) / 2 > first) t--;
  while ((t + 1) * (t + 2) / 2 <= first) t++;
  const i64 j = first - t * (t + 1) / 2;
  NEDY_REQUIRE(t <= d.nt && j + nb <= t + 1,
               "windowed green_func: the block range must lie in one time step's row (column)");
  return comp == NEDY_RET ? d.retptr(t, j) : d.lesptr(j, t);
}

double2 *range_ptr(const nedy_gf *g, int comp, i64 first, i64 nb) {
  if (g->g.win && (comp == NEDY_LES || comp == NEDY_RET)) return window_range(g, comp, first, nb);
  i64 tot;
  double2 *p = comp_ptr(g, comp, tot);
  NEDY_REQUIRE(first >= 0 && nb >= 0 && first + nb <= tot, "block range out of bounds");
  return p + first * g->g.es;
}

int nedy_gf_upload(nedy_gf *g, int comp, long long first, long long nb, const void *host) {
  return guard([&] {
    NEDY_REQUIRE(g && host, "null argument");
    set_dev(g->ctx);
    NEDY_REQUIRE(first >= 0 && nb >= 0, "block range out of bounds");
    double2 *dst = range_ptr(g, comp, first, nb);
    NEDY_CUDA(cudaMemcpyAsync(dst, host, sizeof(double2) * nb * g->g.es, cudaMemcpyDefault, g->ctx->c.stream));
    NEDY_CUDA(cudaStreamSynchronize(g->ctx->c.stream));
    if (comp == NEDY_MAT) g->g.mat_version++;
  });
}

int nedy_gf_download(const nedy_gf *g, int comp, long long first, long long nb, void *host) {
  return guard([&] {
    NEDY_REQUIRE(g && host, "null argument");
    set_dev(g->ctx);
    NEDY_REQUIRE(first >= 0 && nb >= 0, "block range out of bounds");
    const double2 *src = range_ptr(g, comp, first, nb);
    NEDY_CUDA(cudaMemcpyAsync(host, src, sizeof(double2) * nb * g->g.es, cudaMemcpyDefault,
                              g->ctx->c.stream));
    NEDY_CUDA(cudaStreamSynchronize(g->ctx->c.stream));
  });
}

int nedy_gf_device_pointer(const nedy_gf *g, int comp, void **dev) {
  return guard([&] {
    NEDY_REQUIRE(g && dev, "null argument");
    i64 tot;
    *dev = comp_ptr(g, comp, tot);
  });
}

int nedy_gf_set_tstp_zero(nedy_gf *g, int tstp) {
  return guard([&] {
    NEDY_REQUIRE(g, "null argument");
    const DevGF &d = g->g;
    NEDY_REQUIRE(tstp >= -1 && tstp <= d.nt, "tstp out of range");
    set_dev(g->ctx);
    cudaStream_t s = g->ctx->c.stream;
    if (tstp == -1) {
      NEDY_CUDA(cudaMemsetAsync(d.mat, 0, sizeof(double2) * (d.ntau + 1) * d.es, s));
      g->g.mat_version++;
    } else {
      NEDY_CUDA(cudaMemsetAsync(d.retptr(tstp, 0), 0, sizeof(double2) * (tstp + 1) * d.es, s));
      NEDY_CUDA(cudaMemsetAsync(d.lesptr(0, tstp), 0, sizeof(double2) * (tstp + 1) * d.es, s));
      NEDY_CUDA(cudaMemsetAsync(d.tvptr(tstp, 0), 0, sizeof(double2) * (d.ntau + 1) * d.es, s));
    }
  });
}

int nedy_buf_create(nedy_ctx *ctx, long long bytes, nedy_buf **out) {
  return guard([&] {
    NEDY_REQUIRE(ctx && out && bytes > 0, "bad argument");
    set_dev(ctx);
    auto *b = new nedy_buf;
    b->ctx = ctx;
    b->device = ctx->c.device;
    b->bytes = bytes;
    cudaError_t e = cudaMalloc(&b->p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      delete b;
      throw CudaError(std::string("buffer allocation failed: ") + cudaGetErrorString(e));
    }
    memset_sync(b->p, bytes, ctx->c.stream);
    *out = b;
  });
}

int nedy_buf_destroy(nedy_buf *b) {
  return guard([&] {
    if (!b) return;
    cudaSetDevice(b->device);
    cudaFree(b->p);
    delete b;
  });
}

int nedy_buf_upload(nedy_buf *b, long long off, long long bytes, const void *host) {
  return guard([&] {
    NEDY_REQUIRE(b && host && off >= 0 && bytes >= 0 && off + bytes <= b->bytes, "buffer range out of bounds");
    set_dev(b->ctx);
    NEDY_CUDA(cudaMemcpyAsync((char *)b->p + off, host, bytes, cudaMemcpyHostToDevice, b->ctx->c.stream));
    NEDY_CUDA(cudaStreamSynchronize(b->ctx->c.stream));
  });
}

int nedy_buf_download(const nedy_buf *b, long long off, long long bytes, void *host) {
  return guard([&] {
    NEDY_REQUIRE(b && host && off >= 0 && bytes >= 0 && off + bytes <= b->bytes, "buffer range out of bounds");
    set_dev(b->ctx);
    NEDY_CUDA(cudaMemcpyAsync(host, (char *)b->p + off, bytes, cudaMemcpyDeviceToHost, b->ctx->c.stream));
    NEDY_CUDA(cudaStreamSynchronize(b->ctx->c.stream));
  });
}

int nedy_buf_device_pointer(const nedy_buf *b, void **dev) {
  return guard([&] {
    NEDY_REQUIRE(b && dev, "null argument");
    *dev = b->p;
  });
}

int nedy_set_df_tensor(nedy_ctx *ctx, const double *Vija, int nao, int naux) {
  return guard([&] {
    NEDY_REQUIRE(ctx && Vija && nao > 0 && naux > 0, "bad argument");
    set_dev(ctx);
    Ctx &c = ctx->c;
    const size_t n = (size_t)nao * nao * naux;
    std::vector<double> viaj(n), vaij(n), vmbq(n);
    for (int i = 0; i < nao; i++)
      for (int j = 0; j < nao; j++)
        for (int a = 0; a < naux; a++) {
          const double v = Vija[((size_t)i * nao + j) * naux + a];
          viaj[((size_t)i * naux + a) * nao + j] = v;   // Viaj(i,a,j) = Vija(i,j,a)
          vaij[((size_t)a * nao + i) * nao + j] = v;    // Vaij(a,i,j)
          vmbq[((size_t)j * naux + a) * nao + i] = v;   // Vmbq(m=j, b=a, q=i) = V^b_qm
        }
    auto put = [&](double *&d, const double *h) {
      if (d) cudaFree(d);
      NEDY_CUDA(cudaMalloc(&d, sizeof(double) * n));
      h2d_sync(d, h, sizeof(double) * n, c.stream);
    };
    put(c.Vija, Vija);
    put(c.Viaj, viaj.data());
    put(c.Vaij, vaij.data());
    put(c.Vmbq, vmbq.data());
    for (void **q : {&c.Vp, &c.Vanj_p, &c.Vjkb_p, &c.Vila_p}) {  // pieces of the previous tensor
      if (*q) cudaFree(*q);
      *q = nullptr;
    }
    c.Vp_np = 0;
    c.df_nao = nao;
    c.df_naux = naux;
    bool sym = true;
    for (int i = 0; i < nao && sym; i++)
      for (int j = 0; j < i && sym; j++)
        for (int q = 0; q < naux; q++)
          if (Vija[((size_t)i * nao + j) * naux + q] != Vija[((size_t)j * nao + i) * naux + q]) { sym = false; break; }
    c.V_sym = sym;
  });
}

int nedy_set_full_tensor(nedy_ctx *ctx, const double *U, const double *Uexch, int nao) {
  return guard([&] {
    NEDY_REQUIRE(ctx && U && Uexch && nao > 0, "bad argument");
    set_dev(ctx);
    Ctx &c = ctx->c;
    const size_t n = (size_t)nao * nao * nao * nao;
    if (c.U) cudaFree(c.U);
    if (c.Uexch) cudaFree(c.Uexch);
    NEDY_CUDA(cudaMalloc(&c.U, sizeof(double) * n));
    NEDY_CUDA(cudaMalloc(&c.Uexch, sizeof(double) * n));
    h2d_sync(c.U, U, sizeof(double) * n, c.stream);
    h2d_sync(c.Uexch, Uexch, sizeof(double) * n, c.stream);
    c.u_nao = nao;
  });
}

int nedy_gf2_decomp_solve(nedy_ctx *ctx, int tstp, nedy_gf *Sigma, const nedy_gf *G) {
  return guard([&] {
    NEDY_REQUIRE(ctx && Sigma && G, "null argument");
    set_dev(ctx);
    DevGF *S[1] = {&Sigma->g};
    const DevGF *Gs[1] = {&G->g};
    sigma_df(ctx->c, tstp, 1, S, Gs);
    NEDY_CUDA(cudaStreamSynchronize(ctx->c.stream));
  });
}

int nedy_gf2_spin_decomp_solve(nedy_ctx *ctx, int tstp, nedy_gf *Su, nedy_gf *Sd, const nedy_gf *Gu,
                               const nedy_gf *Gd) {
  return guard([&] {
    NEDY_REQUIRE(ctx && Su && Sd && Gu && Gd, "null argument");
    set_dev(ctx);
    DevGF *S[2] = {&Su->g, &Sd->g};
    const DevGF *Gs[2] = {&Gu->g, &Gd->g};
    sigma_df(ctx->c, tstp, 2, S, Gs);
    NEDY_CUDA(cudaStreamSynchronize(ctx->c.stream));
  });
}

int nedy_gf2_full_solve(nedy_ctx *ctx, int tstp, nedy_gf *Sigma, const nedy_gf *G) {
  return guard([&] {
    NEDY_REQUIRE(ctx && Sigma && G, "null argument");
    set_dev(ctx);
    sigma_full(ctx->c, tstp, Sigma->g, G->g);
    NEDY_CUDA(cudaStreamSynchronize(ctx->c.stream));
  });
}

int nedy_get_dm(nedy_ctx *ctx, const nedy_gf *G, int tstp, nedy_buf *rho, long long off) {
  return guard([&] {
    NEDY_REQUIRE(ctx && G && rho, "null argument");
    NEDY_REQUIRE(tstp >= 0 && tstp <= G->g.nt, "tstp out of range");
    const i64 es = G->g.es;
    NEDY_REQUIRE(off >= 0 && off % 16 == 0 && off + es * 16 <= rho->bytes, "rho buffer too small");
    set_dev(ctx);
    get_dm(ctx->c, G->g, tstp, (double2 *)((char *)rho->p + off));
  });
}

int nedy_hf_decomp(nedy_ctx *ctx, int tstp, nedy_buf *hmf, const nedy_buf *rho) {
  return guard([&] {
    NEDY_REQUIRE(ctx && hmf && rho, "null argument");
    set_dev(ctx);
    Ctx &c = ctx->c;
    c.ws.reset();
    double2 *h[1] = {hmf_row(hmf, ctx, tstp, c.df_nao)};
    NEDY_REQUIRE(rho->bytes >= (i64)c.df_nao * c.df_nao * 16, "rho buffer too small");
    hf_decomp(c, 1, h, (const double2 *)rho->p);
    NEDY_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int nedy_hf_spin_decomp(nedy_ctx *ctx, int tstp, nedy_buf *hu, nedy_buf *hd, const nedy_buf *rho2) {
  return guard([&] {
    NEDY_REQUIRE(ctx && hu && hd && rho2, "null argument");
    set_dev(ctx);
    Ctx &c = ctx->c;
    c.ws.reset();
    double2 *h[2] = {hmf_row(hu, ctx, tstp, c.df_nao), hmf_row(hd, ctx, tstp, c.df_nao)};
    NEDY_REQUIRE(rho2->bytes >= 2LL * c.df_nao * c.df_nao * 16, "rho buffer too small");
    hf_decomp(c, 2, h, (const double2 *)rho2->p);
    NEDY_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int nedy_hf_full(nedy_ctx *ctx, int tstp, nedy_buf *hmf, const nedy_buf *rho) {
  return guard([&] {
    NEDY_REQUIRE(ctx && hmf && rho, "null argument");
    set_dev(ctx);
    hf_full(ctx->c, hmf_row(hmf, ctx, tstp, ctx->c.u_nao), (const double2 *)rho->p);
    NEDY_CUDA(cudaStreamSynchronize(ctx->c.stream));
  });
}

int nedy_extrapolate(nedy_ctx *ctx, int tstp, nedy_gf *G) {
  return guard([&] {
    NEDY_REQUIRE(ctx && G, "null argument");
    set_dev(ctx);
    extrapolate(ctx->c, tstp, G->g);
    NEDY_CUDA(cudaStreamSynchronize(ctx->c.stream));
  });
}

int nedy_dyson_step(nedy_ctx *ctx, int tstp, nedy_gf *G, const nedy_gf *Sigma, const nedy_buf *hmf, double mu,
                    double *err3) {
  return guard([&] {
    NEDY_REQUIRE(ctx && G && Sigma && hmf, "null argument");
    set_dev(ctx);
    hmf_row(hmf, ctx, G->g.nt, G->g.nao);
    double e[3];
    dyson_step(ctx->c, tstp, G->g, Sigma->g, (const double2 *)hmf->p, mu, e);
    NEDY_CUDA(cudaStreamSynchronize(ctx->c.stream));
    if (err3) { err3[0] = e[0]; err3[1] = e[1]; err3[2] = e[2]; }
  });
}

int nedy_dyson_start(nedy_ctx *ctx, nedy_gf *G, const nedy_gf *Sigma, const nedy_buf *hmf, double mu, double *err) {
  return guard([&] {
    NEDY_REQUIRE(ctx && G && Sigma && hmf, "null argument");
    set_dev(ctx);
    hmf_row(hmf, ctx, ctx->c.k, G->g.nao);
    double e = dyson_start(ctx->c, G->g, Sigma->g, (const double2 *)hmf->p, mu);
    if (err) *err = e;
  });
}

int nedy_energy_conv(nedy_ctx *ctx, int tstp, const nedy_gf *Sigma, const nedy_gf *G, double *energy) {
  return guard([&] {
    NEDY_REQUIRE(ctx && Sigma && G && energy, "null argument");
    set_dev(ctx);
    *energy = energy_conv(ctx->c, tstp, Sigma->g, G->g);
  });
}

int nedy_decomp_tstp(nedy_ctx *ctx, int tstp, nedy_gf *G, nedy_gf *S, nedy_buf *hmf, const nedy_buf *h_t,
                     double mu, int corr_steps, double *err) {
  return guard([&] {
    NEDY_REQUIRE(ctx && G && S && hmf && h_t, "null argument");
    NEDY_REQUIRE(h_t->bytes >= G->g.es * 16, "h_t buffer too small");
    decomp_step_fixed(ctx, tstp, G, S, hmf, (const double2 *)h_t->p, mu, corr_steps, err);
  });
}

} // extern "C"

// DecompSimulation::do_tstp (src/molNEsim_decomp_impl.h:85-104) with h_t a device pointer.
void nedy::decomp_step_fixed(nedy_ctx *ctx, int tstp, nedy_gf *G, nedy_gf *S, nedy_buf *hmf, const double2 *h_t,
                             double mu, int corr_steps, double *err) {
  {
    NEDY_REQUIRE(ctx && G && S && hmf && h_t, "null argument");
    NEDY_REQUIRE(corr_steps >= 1, "corr_steps must be >= 1");
    set_dev(ctx);
    Ctx &c = ctx->c;
    const int N = G->g.nao;
    const i64 es = (i64)N * N;
    double2 *hT = hmf_row(hmf, ctx, tstp, N);
    hmf_row(hmf, ctx, G->g.nt, N);
    PhaseTimer pt(c);
    pt.mark(0);
    extrapolate(c, tstp, G->g);
    double e[3] = {0, 0, 0};
    for (int it = 0; it < corr_steps; it++) {
      c.ws.reset();
      pt.mark(1);
      double2 *rho = c.ws.alloc<double2>(es);
      get_dm(c, G->g, tstp, rho);
      NEDY_CUDA(cudaMemcpyAsync(hT, h_t, sizeof(double2) * es, cudaMemcpyDeviceToDevice, c.stream));
      double2 *h[1] = {hT};
      hf_decomp(c, 1, h, rho);
      DevGF *Ss[1] = {&S->g};
      const DevGF *Gs[1] = {&G->g};
      pt.mark(2);
      sigma_df(c, tstp, 1, Ss, Gs);
      pt.mark(3);
      dyson_step(c, tstp, G->g, S->g, (const double2 *)hmf->p, mu, e);
    }
    pt.mark(-1);
    NEDY_CUDA(cudaStreamSynchronize(c.stream));
    pt.collect();
    if (err) *err = e[0] + e[1] + e[2];
  }
}

extern "C" {

int nedy_full_tstp(nedy_ctx *ctx, int tstp, nedy_gf *G, nedy_gf *S, nedy_buf *hmf, const nedy_buf *h_t, double mu,
                   int corr_steps, double *err) {
  return guard([&] {
    NEDY_REQUIRE(ctx && G && S && hmf && h_t, "null argument");
    NEDY_REQUIRE(corr_steps >= 1, "corr_steps must be >= 1");
    set_dev(ctx);
    Ctx &c = ctx->c;
    NEDY_REQUIRE(c.U && c.u_nao == G->g.nao, "nedy_full_tstp: full U tensor not set for this nao");
    const int N = G->g.nao;
    const i64 es = (i64)N * N;
    NEDY_REQUIRE(h_t->bytes >= es * 16, "h_t buffer too small");
    double2 *hT = hmf_row(hmf, ctx, tstp, N);
    hmf_row(hmf, ctx, G->g.nt, N);
    PhaseTimer pt(c);
    pt.mark(0);
    extrapolate(c, tstp, G->g);
    double e[3] = {0, 0, 0};
    for (int it = 0; it < corr_steps; it++) {
      c.ws.reset();
      pt.mark(1);
      double2 *rho = c.ws.alloc<double2>(es);
      get_dm(c, G->g, tstp, rho);
      NEDY_CUDA(cudaMemcpyAsync(hT, h_t->p, sizeof(double2) * es, cudaMemcpyDeviceToDevice, c.stream));
      hf_full(c, hT, rho);
      pt.mark(2);
      sigma_full(c, tstp, S->g, G->g);
      pt.mark(3);
      dyson_step(c, tstp, G->g, S->g, (const double2 *)hmf->p, mu, e);
    }
    pt.mark(-1);
    NEDY_CUDA(cudaStreamSynchronize(c.stream));
    pt.collect();
    if (err) *err = e[0] + e[1] + e[2];
  });
}

} // extern "C"

namespace nedy {
// One time step with the residual exit for one (restricted) or two (unrestricted) spins.
// After iteration k the change d_k = max over the spins' new rows of |G_k - G_{k-1}| is
// measured; the step stops once d_k times the corrector's contraction is <= tol.  The
// contraction is measured (4 x the ratio of successive changes) on steps that run two or
// more iterations: the first step of a context, and every 8th after, run at least two.
// h_t[s]: device pointer to the nao x nao one-body Hamiltonian of spin s at tstp.
void step_tol(nedy_ctx *ctx, int tstp, int nspin, nedy_gf *const *G, nedy_gf *const *S, nedy_buf *const *hmf,
              const double2 *const *h_t, const double *mu, int max_corr, double tol, int *iters, double *err_hist) {
  NEDY_REQUIRE(max_corr >= 1 && tol >= 0.0, "max_corr must be >= 1 and tol >= 0");
  for (int s = 0; s < nspin; s++) NEDY_REQUIRE(G[s] && S[s] && hmf[s] && h_t[s], "null argument");
  set_dev(ctx);
  Ctx &c = ctx->c;
  const int N = G[0]->g.nao;
  const i64 es = (i64)N * N;
  double2 *hT[2];
  for (int s = 0; s < nspin; s++) {
    NEDY_REQUIRE(G[s]->g.nao == N, "nao mismatch between the spins");
    hT[s] = hmf_row(hmf[s], ctx, tstp, N);
    hmf_row(hmf[s], ctx, G[s]->g.nt, N);
  }
  PhaseTimer pt(c);
  pt.mark(0);
  for (int s = 0; s < nspin; s++) extrapolate(c, tstp, G[s]->g);
  const i64 npred = c.pred ? Predictor::row_elements(G[0]->g, tstp) : 0;
  const bool learned = c.pred && c.pred_active && npred > 0;
  if (learned) {
    if (c.pred_corr_cap < nspin * npred) {  // sized for the longest row of the run (allocated once)
      const i64 cap = std::max<i64>(nspin * npred, nspin * Predictor::row_elements(G[0]->g, G[0]->g.nt));
      if (c.pred_corr) cudaFree(c.pred_corr);
      c.pred_corr = nullptr;
      NEDY_CUDA(cudaMalloc(&c.pred_corr, sizeof(double2) * cap));
      c.pred_corr_cap = cap;
    }
    for (int s = 0; s < nspin; s++) c.pred->apply(G[s]->g, tstp, c.pred_corr + s * npred);
  }
  const bool refresh = c.contraction >= 1.0 || c.steps_since_measure >= 8;
  const i64 rl = row_len(G[0]->g, tstp);
  int it = 0;
  double prev = 0.0, ratio = 0.0;
  for (; it < max_corr;) {
    for (int s = 0; s < nspin; s++) save_row(c, G[s]->g, tstp, s);
    c.ws.reset();
    pt.mark(1);
    double2 *rho = c.ws.alloc<double2>(nspin * es);
    for (int s = 0; s < nspin; s++) {
      get_dm(c, G[s]->g, tstp, rho + s * es);
      NEDY_CUDA(cudaMemcpyAsync(hT[s], h_t[s], sizeof(double2) * es, cudaMemcpyDeviceToDevice, c.stream));
    }
    hf_decomp(c, nspin, hT, rho);
    DevGF *Ss[2] = {&S[0]->g, nspin > 1 ? &S[1]->g : nullptr};
    const DevGF *Gs[2] = {&G[0]->g, nspin > 1 ? &G[1]->g : nullptr};
    pt.mark(2);
    sigma_df(c, tstp, nspin, Ss, Gs);
    pt.mark(3);
    double d = 0.0;
    {
      double e[2][3] = {{0, 0, 0}, {0, 0, 0}};
      if (nspin == 2)
        dyson_step_spins(c, tstp, G[0]->g, S[0]->g, (const double2 *)hmf[0]->p, mu[0], e[0], G[1]->g, S[1]->g,
                         (const double2 *)hmf[1]->p, mu[1], e[1]);
      else
        dyson_step(c, tstp, G[0]->g, S[0]->g, (const double2 *)hmf[0]->p, mu[0], e[0]);
      for (int s = 0; s < nspin; s++) d = std::max(d, row_change(c, G[s]->g, tstp, s));
    }
    if (err_hist) err_hist[it] = d;
    if (learned && it == 0) {
      // the first iteration judges the learned prediction against the polynomial one;
      // once 8 steps are judged, fewer than 3 wins among the last 8 switch back to the
      // polynomial predictor
      double dl = 0, dp = 0;
      for (int s = 0; s < nspin; s++) {
        double a = 0, b = 0;
        c.pred->judge(G[s]->g, tstp, c.rowcopy + s * rl, c.pred_corr + s * npred, a, b);
        dl = std::max(dl, a);
        dp = std::max(dp, b);
      }
      c.pred_last[0] = dl;
      c.pred_last[1] = dp;
      c.pred_judged++;
      const bool won = dl <= dp;
      if (won) c.pred_better++;
      c.pred_window = (c.pred_window << 1) | (won ? 1u : 0u);
      if (c.pred_judged >= 8 && __builtin_popcount(c.pred_window & 0xFFu) < 3) c.pred_active = false;
    }
    if (it > 0 && prev > 0.0) ratio = std::max(ratio, d / prev);
    prev = d;
    it++;
    if (refresh && it < 2) continue;
    if (d * std::min(1.0, c.contraction) <= tol || (ratio > 0.0 && d * std::min(1.0, 4.0 * ratio) <= tol)) break;
  }
  if (ratio > 0.0) {
    c.contraction = std::min(1.0, 4.0 * ratio);
    c.steps_since_measure = 0;
  } else {
    c.steps_since_measure++;
  }
  pt.mark(-1);
  NEDY_CUDA(cudaStreamSynchronize(c.stream));
  pt.collect();
  if (iters) *iters = it;
}
}  // namespace nedy

extern "C" {

int nedy_decomp_tstp_tol(nedy_ctx *ctx, int tstp, nedy_gf *G, nedy_gf *S, nedy_buf *hmf, const nedy_buf *h_t,
                         double mu, int max_corr, double tol, int *iters, double *err_hist) {
  return guard([&] {
    NEDY_REQUIRE(ctx, "null argument");
    NEDY_REQUIRE(G && h_t && h_t->bytes >= G->g.es * 16, "null argument or h_t buffer too small");
    nedy_gf *Gs[1] = {G}, *Ss[1] = {S};
    nedy_buf *hs[1] = {hmf};
    const double2 *hts[1] = {(const double2 *)h_t->p};
    step_tol(ctx, tstp, 1, Gs, Ss, hs, hts, &mu, max_corr, tol, iters, err_hist);
  });
}

int nedy_decomp_spin_tstp_tol(nedy_ctx *ctx, int tstp, nedy_gf *G_up, nedy_gf *G_dn, nedy_gf *S_up, nedy_gf *S_dn,
                              nedy_buf *hmf_up, nedy_buf *hmf_dn, const nedy_buf *h_t_up, const nedy_buf *h_t_dn,
                              double mu_up, double mu_dn, int max_corr, double tol, int *iters, double *err_hist) {
  return guard([&] {
    NEDY_REQUIRE(ctx, "null argument");
    NEDY_REQUIRE(G_up && G_dn && h_t_up && h_t_dn, "null argument");
    NEDY_REQUIRE(h_t_up->bytes >= G_up->g.es * 16 && h_t_dn->bytes >= G_dn->g.es * 16, "h_t buffer too small");
    nedy_gf *Gs[2] = {G_up, G_dn}, *Ss[2] = {S_up, S_dn};
    nedy_buf *hs[2] = {hmf_up, hmf_dn};
    const double2 *hts[2] = {(const double2 *)h_t_up->p, (const double2 *)h_t_dn->p};
    const double mus[2] = {mu_up, mu_dn};
    step_tol(ctx, tstp, 2, Gs, Ss, hs, hts, mus, max_corr, tol, iters, err_hist);
  });
}

int nedy_predictor_create(nedy_ctx *ctx, long long capacity, unsigned long long seed, nedy_predictor **out) {
  return guard([&] {
    NEDY_REQUIRE(ctx && out && capacity > 0, "bad argument");
    set_dev(ctx);
    NEDY_REQUIRE(ctx->c.k == 5, "the learned predictor corrects the k = 5 extrapolation");
    ensure_tables(ctx->c);
    auto *h = new nedy_predictor;
    h->ctx = ctx;
    try {
      h->p = new Predictor(ctx->c, capacity, seed);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

int nedy_predictor_destroy(nedy_predictor *p) {
  return guard([&] {
    if (!p) return;
    cudaSetDevice(p->p->ctx.device);
    if (p->ctx->c.pred == p->p) {
      p->ctx->c.pred = nullptr;
      p->ctx->c.pred_active = false;
    }
    delete p->p;
    delete p;
  });
}

int nedy_predictor_collect(nedy_predictor *p, const nedy_gf *G, int tstp, int stride) {
  return guard([&] {
    NEDY_REQUIRE(p && G && tstp >= 0 && tstp <= G->g.nt, "bad argument");
    set_dev(p->ctx);
    p->p->collect(G->g, tstp, stride);
  });
}

int nedy_predictor_samples(nedy_predictor *p, long long *n) {
  return guard([&] {
    NEDY_REQUIRE(p && n, "null argument");
    set_dev(p->ctx);
    *n = p->p->samples();
  });
}

int nedy_predictor_clear(nedy_predictor *p) {
  return guard([&] {
    NEDY_REQUIRE(p, "null argument");
    set_dev(p->ctx);
    p->p->clear_samples();
  });
}

int nedy_predictor_train(nedy_predictor *p, int iters, int batch, double lr, double *loss) {
  return guard([&] {
    NEDY_REQUIRE(p, "null argument");
    set_dev(p->ctx);
    const double l = p->p->train(iters, batch, lr);
    if (loss) *loss = l;
  });
}

long long nedy_predictor_nparams(void) { return PRED_NPARAM; }

int nedy_predictor_params(nedy_predictor *p, float *host, int get) {
  return guard([&] {
    NEDY_REQUIRE(p && host, "null argument");
    set_dev(p->ctx);
    if (get)
      p->p->get_params(host);
    else
      p->p->set_params(host);
  });
}

int nedy_predictor_infer(nedy_predictor *p, const float *x, int n, float *y) {
  return guard([&] {
    NEDY_REQUIRE(p && x && y && n > 0, "bad argument");
    set_dev(p->ctx);
    Ctx &c = p->ctx->c;
    float *d = nullptr;
    NEDY_CUDA(cudaMalloc(&d, sizeof(float) * (size_t)n * (PRED_IN + 2)));
    float *yd = d + (i64)n * PRED_IN;
    cudaError_t e = cudaMemcpyAsync(d, x, sizeof(float) * n * PRED_IN, cudaMemcpyHostToDevice, c.stream);
    if (e == cudaSuccess) {
      try {
        p->p->infer(n, d, yd);
      } catch (...) {
        cudaFree(d);
        throw;
      }
      e = cudaMemcpyAsync(y, yd, sizeof(float) * n * 2, cudaMemcpyDeviceToHost, c.stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    cudaFree(d);
    NEDY_CUDA(e);
  });
}

int nedy_predictor_forward(nedy_predictor *p, const float *x, int n, float *y) {
  return guard([&] {
    NEDY_REQUIRE(p && x && y && n > 0, "bad argument");
    set_dev(p->ctx);
    Ctx &c = p->ctx->c;
    float *d = nullptr;
    NEDY_CUDA(cudaMalloc(&d, sizeof(float) * (size_t)n * (PRED_IN + 2 * PRED_W + 2)));
    float *h1 = d + (i64)n * PRED_IN, *h2 = h1 + (i64)n * PRED_W, *yd = h2 + (i64)n * PRED_W;
    cudaError_t e = cudaMemcpyAsync(d, x, sizeof(float) * n * PRED_IN, cudaMemcpyHostToDevice, c.stream);
    if (e == cudaSuccess) {
      try {
        p->p->forward(n, d, h1, h2, yd);
      } catch (...) {
        cudaFree(d);
        throw;
      }
      e = cudaMemcpyAsync(y, yd, sizeof(float) * n * 2, cudaMemcpyDeviceToHost, c.stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    cudaFree(d);
    NEDY_CUDA(e);
  });
}

int nedy_predictor_loss_grad(nedy_predictor *p, const float *x, const float *t, int n, double *loss, float *grad) {
  return guard([&] {
    NEDY_REQUIRE(p && x && t && n > 0, "bad argument");
    set_dev(p->ctx);
    Ctx &c = p->ctx->c;
    float *d = nullptr;
    NEDY_CUDA(cudaMalloc(&d, sizeof(float) * (size_t)n * (PRED_IN + 2)));
    cudaError_t e = cudaMemcpyAsync(d, x, sizeof(float) * n * PRED_IN, cudaMemcpyHostToDevice, c.stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d + (i64)n * PRED_IN, t, sizeof(float) * n * 2, cudaMemcpyHostToDevice, c.stream);
    double l = 0;
    if (e == cudaSuccess) {
      try {
        l = p->p->loss_grad(n, d, d + (i64)n * PRED_IN, true);
      } catch (...) {
        cudaFree(d);
        throw;
      }
      if (grad) e = cudaMemcpyAsync(grad, p->p->grad(), sizeof(float) * PRED_NPARAM, cudaMemcpyDeviceToHost, c.stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    cudaFree(d);
    NEDY_CUDA(e);
    if (loss) *loss = l;
  });
}

int nedy_predict(nedy_ctx *ctx, int tstp, nedy_gf *G, int learned) {
  return guard([&] {
    NEDY_REQUIRE(ctx && G, "null argument");
    set_dev(ctx);
    Ctx &c = ctx->c;
    extrapolate(c, tstp, G->g);
    if (learned) {
      NEDY_REQUIRE(c.pred, "nedy_predict: no learned predictor set on this context");
      c.pred->apply(G->g, tstp, nullptr);
    }
    NEDY_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int nedy_ctx_set_predictor(nedy_ctx *ctx, nedy_predictor *p) {
  return guard([&] {
    NEDY_REQUIRE(ctx, "null context");
    NEDY_REQUIRE(!p || p->ctx == ctx, "predictor belongs to another context");
    Ctx &c = ctx->c;
    c.pred = p ? p->p : nullptr;
    c.pred_active = p != nullptr;
    c.pred_window = 0;
    c.pred_judged = c.pred_better = 0;
  });
}

int nedy_ctx_predictor_stats(const nedy_ctx *ctx, int *active, long long *judged, long long *better, double *last2) {
  return guard([&] {
    NEDY_REQUIRE(ctx, "null context");
    const Ctx &c = ctx->c;
    if (active) *active = c.pred && c.pred_active ? 1 : 0;
    if (judged) *judged = c.pred_judged;
    if (better) *better = c.pred_better;
    if (last2) {
      last2[0] = c.pred_last[0];
      last2[1] = c.pred_last[1];
    }
  });
}

int nedy_decomp_spin_tstp(nedy_ctx *ctx, int tstp, nedy_gf *Gu, nedy_gf *Gd, nedy_gf *Su, nedy_gf *Sd,
                          nedy_buf *hu, nedy_buf *hd, const nedy_buf *htu, const nedy_buf *htd, double mu_up,
                          double mu_dn, int corr_steps, double *err) {
  return guard([&] {
    NEDY_REQUIRE(ctx && Gu && Gd && Su && Sd && hu && hd && htu && htd, "null argument");
    NEDY_REQUIRE(corr_steps >= 1, "corr_steps must be >= 1");
    set_dev(ctx);
    Ctx &c = ctx->c;
    const int N = Gu->g.nao;
    const i64 es = (i64)N * N;
    double2 *hT[2] = {hmf_row(hu, ctx, tstp, N), hmf_row(hd, ctx, tstp, N)};
    PhaseTimer pt(c);
    pt.mark(0);
    extrapolate(c, tstp, Gu->g);
    extrapolate(c, tstp, Gd->g);
    double eu[3] = {0, 0, 0}, ed[3] = {0, 0, 0};
    for (int it = 0; it < corr_steps; it++) {
      c.ws.reset();
      pt.mark(1);
      double2 *rho = c.ws.alloc<double2>(2 * es);
      get_dm(c, Gu->g, tstp, rho);
      get_dm(c, Gd->g, tstp, rho + es);
      NEDY_CUDA(cudaMemcpyAsync(hT[0], htu->p, sizeof(double2) * es, cudaMemcpyDeviceToDevice, c.stream));
      NEDY_CUDA(cudaMemcpyAsync(hT[1], htd->p, sizeof(double2) * es, cudaMemcpyDeviceToDevice, c.stream));
      hf_decomp(c, 2, hT, rho);
      DevGF *Ss[2] = {&Su->g, &Sd->g};
      const DevGF *Gs[2] = {&Gu->g, &Gd->g};
      pt.mark(2);
      sigma_df(c, tstp, 2, Ss, Gs);
      pt.mark(3);
      dyson_step_spins(c, tstp, Gu->g, Su->g, (const double2 *)hu->p, mu_up, eu, Gd->g, Sd->g,
                       (const double2 *)hd->p, mu_dn, ed);
    }
    pt.mark(-1);
    NEDY_CUDA(cudaStreamSynchronize(c.stream));
    pt.collect();
    if (err) *err = eu[0] + eu[1] + eu[2] + ed[0] + ed[1] + ed[2];
  });
}

} // extern "C"
