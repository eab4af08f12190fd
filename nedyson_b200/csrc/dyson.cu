// Dyson time step, its history integrals, the predictor, the bootstrap, the HF
// mean field and the energy -- device side.
//
//   dyson_step_ret : reference src/dyson_step.h:7-127
//   dyson_step_tv  : reference src/dyson_step.h:130-169 (+ Ctv_tstp / CTV1, dyson_integrals.h:80-116, 254-324)
//   dyson_step_les : reference src/dyson_step.h:171-326 (+ Cles2 / Cles3, dyson_integrals.h:336-461)
//   Extrapolate    : reference src/dyson.cpp:47-117
//   dyson_start    : reference src/dyson_boot.h:6-230
//   energy_conv    : reference src/dyson_integrals.h:24-70
//   HF             : reference src/molHFSolver.cpp:81-110, 203-239, 35-56
//
// Layout: every history sum is one (grouped) FP64 GEMM over packed blocks.  The
// sequential Volterra sweeps use the cached inverses of the time-local matrices
// M(t') = (i bd0/dt + mu) - hmf(t') - dt*w0*Sig^R(t',t'): for t' < T they no longer
// change, so each step is a single block product instead of an LU solve.
#include "sigma.cuh"
#include <cooperative_groups.h>
#include <exception>
#include <thread>
#include <atomic>
#include <cmath>
#include <algorithm>

namespace nedy {
namespace {

constexpr int TPB = 256;

inline unsigned nblk(i64 n, int tpb = TPB) { return (unsigned)std::min<i64>((n + tpb - 1) / tpb, 65535LL * 16); }

#define GRID_STRIDE(i, n) for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < (n); i += (i64)gridDim.x * blockDim.x)

// ---------------------------------------------------------------------------------
// Gauss-Jordan with partial pivoting, one CTA per system, in global memory.
// A: n x n (destroyed), B: n x nrhs (overwritten by X = A^-1 B).  status[b] = 1 on a zero pivot.
__global__ void gj_kernel(int n, int nrhs, double2 *A, i64 sA, double2 *B, i64 sB, int *status) {
  double2 *a = A + blockIdx.x * sA;
  double2 *b = B + blockIdx.x * sB;
  __shared__ double sval[TPB];
  __shared__ int sidx[TPB];
  __shared__ double2 fac[1024];
  const int tid = threadIdx.x;
  for (int c = 0; c < n; c++) {
    // pivot search
    double best = -1.0;
    int bi = c;
    for (int r = c + tid; r < n; r += blockDim.x) {
      double v = hypot(a[(i64)r * n + c].x, a[(i64)r * n + c].y);
      if (v > best) { best = v; bi = r; }
    }
    sval[tid] = best;
    sidx[tid] = bi;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (tid < s && sval[tid + s] > sval[tid]) { sval[tid] = sval[tid + s]; sidx[tid] = sidx[tid + s]; }
      __syncthreads();
    }
    const int p = sidx[0];
    if (sval[0] == 0.0) {
      if (tid == 0 && status) status[blockIdx.x] = 1;
      return;
    }
    if (p != c) {
      for (int j = tid; j < n; j += blockDim.x) {
        double2 t = a[(i64)c * n + j]; a[(i64)c * n + j] = a[(i64)p * n + j]; a[(i64)p * n + j] = t;
      }
      for (int j = tid; j < nrhs; j += blockDim.x) {
        double2 t = b[(i64)c * nrhs + j]; b[(i64)c * nrhs + j] = b[(i64)p * nrhs + j]; b[(i64)p * nrhs + j] = t;
      }
    }
    __syncthreads();
    const double2 piv = a[(i64)c * n + c];
    const double dd = piv.x * piv.x + piv.y * piv.y;
    const double2 inv = make_double2(piv.x / dd, -piv.y / dd);
    __syncthreads();
    for (int j = tid; j < n; j += blockDim.x) a[(i64)c * n + j] = cmul(a[(i64)c * n + j], inv);
    for (int j = tid; j < nrhs; j += blockDim.x) b[(i64)c * nrhs + j] = cmul(b[(i64)c * nrhs + j], inv);
    __syncthreads();
    // elimination factors (column c of the other rows), processed in slabs of 1024 rows
    for (int r0 = 0; r0 < n; r0 += 1024) {
      const int rn = min(1024, n - r0);
      for (int r = tid; r < rn; r += blockDim.x) fac[r] = (r0 + r == c) ? czero() : a[(i64)(r0 + r) * n + c];
      __syncthreads();
      const int w = n + nrhs;
      for (i64 idx = tid; idx < (i64)rn * w; idx += blockDim.x) {
        const int r = (int)(idx / w), j = (int)(idx - (i64)r * w);
        const double2 f = fac[r];
        if (f.x == 0.0 && f.y == 0.0) continue;
        if (j < n) {
          if (j == c) continue;
          a[(i64)(r0 + r) * n + j] = csub(a[(i64)(r0 + r) * n + j], cmul(f, a[(i64)c * n + j]));
        } else {
          const int jj = j - n;
          b[(i64)(r0 + r) * nrhs + jj] = csub(b[(i64)(r0 + r) * nrhs + jj], cmul(f, b[(i64)c * nrhs + jj]));
        }
      }
      __syncthreads();
      for (int r = tid; r < rn; r += blockDim.x)
        if (r0 + r != c) a[(i64)(r0 + r) * n + c] = czero();
      __syncthreads();
    }
  }
}

// Gauss-Jordan with partial pivoting for ONE large system, spread over many CTAs:
// CTA g owns the augmented columns [g*cw, (g+1)*cw) of [A | B].  One launch per
// elimination step c; the pivot index and the pivot column of step c are produced
// by the launch of step c-1 (by the CTA that owns column c) into buffer c & 1.
__device__ __forceinline__ double2 &aug(double2 *A, double2 *B, int n, int nrhs, int r, int j) {
  return j < n ? A[(i64)r * n + j] : B[(i64)r * nrhs + (j - n)];
}

__device__ void gj_pivot_block(int n, int nrhs, double2 *A, double2 *B, int c, int *piv, double2 *fac) {
  __shared__ double sval[TPB];
  __shared__ int sidx[TPB];
  const int tid = threadIdx.x;
  double best = -1.0;
  int bi = c;
  for (int r = c + tid; r < n; r += blockDim.x) {
    const double2 v = A[(i64)r * n + c];
    const double a = hypot(v.x, v.y);
    if (a > best) { best = a; bi = r; }
  }
  sval[tid] = best;
  sidx[tid] = bi;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (tid < s && sval[tid + s] > sval[tid]) { sval[tid] = sval[tid + s]; sidx[tid] = sidx[tid + s]; }
    __syncthreads();
  }
  if (tid == 0) piv[c & 1] = sidx[0];
  for (int r = tid; r < n; r += blockDim.x) fac[(i64)(c & 1) * n + r] = A[(i64)r * n + c];
}

__global__ void gj_first_pivot_kernel(int n, int nrhs, double2 *A, double2 *B, int *piv, double2 *fac) {
  gj_pivot_block(n, nrhs, A, B, 0, piv, fac);
}

// One elimination step c on this CTA's column slab.  COOP: inside the cooperative kernel,
// where the pivot index and column come from another CTA in the same launch, so they are
// read through L2 (ld.global.cg) rather than a possibly stale L1 line.
template <bool COOP>
__device__ void gj_step_body(int n, int nrhs, double2 *A, double2 *B, int c, int cw, int *piv, double2 *fac,
                             int *status, double2 *rowc) {
  const int j0 = blockIdx.x * cw, W = n + nrhs;
  const int jn = min(cw, W - j0);
  if (jn <= 0) return;
  const int p = COOP ? __ldcg(piv + (c & 1)) : piv[c & 1];
  const double2 *f = fac + (i64)(c & 1) * n;
  auto fget = [&](int r) { return COOP ? __ldcg(f + r) : f[r]; };
  double2 pv = fget(p);
  if (pv.x == 0.0 && pv.y == 0.0) {
    if (threadIdx.x == 0) *status = 1;
    pv = make_double2(1.0, 0.0);
  }
  const double dd = pv.x * pv.x + pv.y * pv.y;
  const double2 inv = make_double2(pv.x / dd, -pv.y / dd);
  // phase 1: swap rows c and p, scale the pivot row
  for (int jj = threadIdx.x; jj < jn; jj += blockDim.x) {
    const int j = j0 + jj;
    const double2 ac = aug(A, B, n, nrhs, c, j), ap = aug(A, B, n, nrhs, p, j);
    const double2 rc = cmul(ap, inv);
    rowc[jj] = rc;
    aug(A, B, n, nrhs, c, j) = rc;
    if (p != c) aug(A, B, n, nrhs, p, j) = csub(ac, cmul(fget(c), rc));
  }
  __syncthreads();
  // phase 2: eliminate the other rows (the factors are the pivot column after the swap)
  for (i64 idx = threadIdx.x; idx < (i64)n * jn; idx += blockDim.x) {
    const int r = (int)(idx / jn), jj = (int)(idx - (i64)r * jn);
    if (r == c || r == p) continue;
    double2 &x = aug(A, B, n, nrhs, r, j0 + jj);
    x = csub(x, cmul(fget(r), rowc[jj]));
  }
  __syncthreads();
  // the owner of column c+1 prepares the next step
  const int c1 = c + 1;
  if (c1 < n && c1 >= j0 && c1 < j0 + jn) gj_pivot_block(n, nrhs, A, B, c1, piv, fac);
}

__global__ void gj_step_kernel(int n, int nrhs, double2 *A, double2 *B, int c, int cw, int *piv, double2 *fac,
                               int *status) {
  __shared__ double2 rowc[64];
  gj_step_body<false>(n, nrhs, A, B, c, cw, piv, fac, status, rowc);
}

__device__ __forceinline__ unsigned long long gj_gtime() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Barrier over all CTAs of a cooperative launch (every CTA is resident).  bar[0] counts
// arrivals, bar[1] is the generation.  The wait is bounded (2 s of %globaltimer, or an
// error another CTA reported): on give-up it sets *status = 2 and returns false, and the
// caller returns, so the launch always ends.
__device__ bool gj_grid_barrier(unsigned *bar, int *status) {
  __syncthreads();
  __shared__ int ok;
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned *gen = bar + 1;
    const unsigned g = *gen;  // read the generation before arriving
    __threadfence();
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      bar[0] = 0;  // nobody arrives again before the generation moves on
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const unsigned long long t0 = gj_gtime();
      for (unsigned it = 1; *gen == g; it++) {
        if ((it & 1023) == 0 && (gj_gtime() - t0 > 2000000000ULL || *(volatile int *)status == 2)) {
          atomicExch(status, 2);
          ok = 0;
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

// All n elimination steps of gj_step_kernel in one cooperative launch, a grid barrier
// between steps (the pivot of step c+1 is produced by the owner of column c+1 during step c).
__global__ void gj_coop_kernel(int n, int nrhs, double2 *A, double2 *B, int cw, int *piv, double2 *fac, int *status,
                               unsigned *bar) {
  __shared__ double2 rowc[64];
  if (blockIdx.x == 0) gj_pivot_block(n, nrhs, A, B, 0, piv, fac);
  if (!gj_grid_barrier(bar, status)) return;
  for (int c = 0; c < n; c++) {
    gj_step_body<true>(n, nrhs, A, B, c, cw, piv, fac, status, rowc);
    if (!gj_grid_barrier(bar, status)) return;
  }
}

// ---------------------------------------------------------------------------------
// Gauss-Jordan with partial pivoting on [A | B] held in shared memory: one thread-block
// cluster of CL CTAs per system (system b = blockIdx.x / CL), CTA r of the cluster owns the
// augmented columns [r cw, (r + 1) cw) of its system.  Step c: every CTA holds pivot column c
// and the pivot row index p in its own shared memory (buffer c & 1, written there by the owner
// of column c); it swaps rows c and p of its columns, scales the pivot row and eliminates the
// other rows.  The owner of column c + 1 then picks the next pivot (largest |.|, first row on
// ties) and stores column c + 1 and the pivot index into buffer (c + 1) & 1 of every CTA of
// the cluster (distributed shared memory); the cluster barrier (release / acquire) orders
// those stores before step c + 1, and the two buffers keep them clear of the reads of step c.
// Columns of A at or left of the pivot are not updated any more (they are unit columns and
// no longer read), and A in global memory is left as it was; B is overwritten by A^-1 B.
// Every CTA runs the same n steps (a zero pivot is seen by all of them and ends all loops
// together), so every barrier is reached by the whole cluster.
constexpr int GJS_THREADS = 512;
constexpr int GJS_SMEM_MAX = 225 * 1024;

inline i64 gjs_smem_bytes(int n, int cw) { return ((i64)n * cw + 2 * (i64)n + cw) * 16 + 16; }

__global__ void __launch_bounds__(GJS_THREADS, 1)
    gj_smem_kernel(int n, int nrhs, const double2 *A, i64 sA, double2 *B, i64 sB, int cw, int *status) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int CL = (int)cl.num_blocks(), rank = (int)cl.block_rank();
  const int sys = blockIdx.x / CL;
  A += sys * sA;
  B += sys * sB;
  extern __shared__ double2 gsm[];
  double2 *slab = gsm;                    // [n][cw]
  double2 *facb = slab + (i64)n * cw;     // [2][n]: pivot column of the step, pre-swap
  double2 *rowc = facb + 2 * (i64)n;      // [cw]: scaled pivot row, this CTA's columns
  int *spiv = (int *)(rowc + cw);         // [2]: pivot row index of the step
  __shared__ double rv[GJS_THREADS / 32];
  __shared__ int ri[GJS_THREADS / 32];
  const int W = n + nrhs, j0 = rank * cw, jn = max(0, min(cw, W - j0));
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (i64 idx = tid; idx < (i64)n * jn; idx += blockDim.x) {
    const int r = (int)(idx / jn), jj = (int)(idx - (i64)r * jn), j = j0 + jj;
    slab[(i64)r * cw + jj] = j < n ? A[(i64)r * n + j] : B[(i64)r * nrhs + (j - n)];
  }
  cl.sync();  // every CTA of the cluster has started before any stores into its shared memory
  // the owner of column c picks the pivot among rows >= c and hands column c to every CTA
  auto publish = [&](int c) {
    const int lc = c - j0;
    double best = -1.0;
    int bi = n;
    for (int r = c + tid; r < n; r += blockDim.x) {
      const double2 v = slab[(i64)r * cw + lc];
      const double a = v.x * v.x + v.y * v.y;
      if (a > best) { best = a; bi = r; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_down_sync(0xffffffffu, best, o);
      const int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    if (lane == 0) { rv[wid] = best; ri[wid] = bi; }
    __syncthreads();
    if (wid == 0) {
      best = lane < (int)(blockDim.x >> 5) ? rv[lane] : -1.0;
      bi = lane < (int)(blockDim.x >> 5) ? ri[lane] : n;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, o);
        const int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      if (lane == 0) ri[0] = bi < n ? bi : c;
    }
    __syncthreads();
    const int p = ri[0], buf = c & 1;
    for (int t = 0; t < CL; t++) {
      double2 *dst = cl.map_shared_rank(facb + (i64)buf * n, t);
      for (int r = tid; r < n; r += blockDim.x) dst[r] = slab[(i64)r * cw + lc];
      if (tid == 0) *cl.map_shared_rank(spiv + buf, t) = p;
    }
  };
  if (j0 == 0 && jn > 0) publish(0);
  cl.sync();
  for (int c = 0; c < n; c++) {
    const int buf = c & 1, p = spiv[buf];
    const double2 *f = facb + (i64)buf * n;
    const double2 pv = f[p];
    if (pv.x == 0.0 && pv.y == 0.0) {  // the same in every CTA of the cluster
      if (rank == 0 && tid == 0 && status) status[sys] = 1;
      break;
    }
    const double dd = pv.x * pv.x + pv.y * pv.y;
    const double2 inv = make_double2(pv.x / dd, -pv.y / dd);
    const int jlo = min(jn, max(0, c + 1 - j0)), wl = jn - jlo;
    const double2 fc = f[c];
    for (int jj = jlo + tid; jj < jn; jj += blockDim.x) {
      const double2 ac = slab[(i64)c * cw + jj], ap = slab[(i64)p * cw + jj];
      const double2 rc = cmul(ap, inv);
      rowc[jj] = rc;
      slab[(i64)c * cw + jj] = rc;
      if (p != c) slab[(i64)p * cw + jj] = csub(ac, cmul(fc, rc));
    }
    __syncthreads();
    for (int idx = tid; idx < n * wl; idx += blockDim.x) {
      const int r = idx / wl, jj = jlo + (idx - r * wl);
      if (r == c || r == p) continue;
      double2 &x = slab[(i64)r * cw + jj];
      x = csub(x, cmul(f[r], rowc[jj]));
    }
    __syncthreads();
    if (c + 1 < n && c + 1 >= j0 && c + 1 < j0 + jn) publish(c + 1);
    cl.sync();
  }
  for (i64 idx = tid; idx < (i64)n * jn; idx += blockDim.x) {
    const int r = (int)(idx / jn), jj = (int)(idx - (i64)r * jn), j = j0 + jj;
    if (j >= n) B[(i64)r * nrhs + (j - n)] = slab[(i64)r * cw + jj];
  }
}

// Cluster size for gj_smem_kernel (0: the system does not fit in the shared memory of
// 16 CTAs, or no such cluster can be resident).  A single system is spread until each CTA
// holds at most 32 columns; a batch keeps one CTA per system where it fits.
int gjs_cluster(int n, int nrhs, int nb, int &cw) {
  static std::atomic<int> ok[64][5];  // per device and cluster size: 0 unknown, 1 yes, -1 no
  int dev = 0;
  NEDY_CUDA(cudaGetDevice(&dev));
  if (dev >= 64) return 0;
  const int W = n + nrhs;
  for (int li = 0; li < 5; li++) {
    const int CL = 1 << li;
    cw = (W + CL - 1) / CL;
    const i64 bytes = gjs_smem_bytes(n, cw);
    if (bytes > GJS_SMEM_MAX) continue;
    if (nb == 1 && cw > 32 && CL < 16) continue;
    if (ok[dev][li].load() == 0) {
      NEDY_CUDA(cudaFuncSetAttribute(gj_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, GJS_SMEM_MAX));
      NEDY_CUDA(cudaFuncSetAttribute(gj_smem_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = CL;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3(CL);
      cfg.blockDim = dim3(GJS_THREADS);
      cfg.dynamicSmemBytes = GJS_SMEM_MAX;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      int nclusters = 0;
      const cudaError_t e = cudaOccupancyMaxActiveClusters(&nclusters, gj_smem_kernel, &cfg);
      if (e != cudaSuccess) (void)cudaGetLastError();
      ok[dev][li].store(e == cudaSuccess && nclusters > 0 ? 1 : -1);
    }
    if (ok[dev][li].load() > 0) return CL;
  }
  return 0;
}

void gj(Ctx &c, int n, int nrhs, int nb, double2 *A, i64 sA, double2 *B, i64 sB) {
  int *st = c.ws.alloc<int>(nb);
  NEDY_CUDA(cudaMemsetAsync(st, 0, sizeof(int) * nb, c.stream));
  int cw = 0;
  const int CL = gjs_cluster(n, nrhs, nb, cw);
  if (CL > 0) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)(nb * CL));
    cfg.blockDim = dim3(GJS_THREADS);
    cfg.dynamicSmemBytes = (size_t)gjs_smem_bytes(n, cw);
    cfg.stream = c.stream;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    NEDY_CUDA(cudaLaunchKernelEx(&cfg, gj_smem_kernel, n, nrhs, (const double2 *)A, sA, B, sB, cw, st));
    NEDY_CHECK_LAUNCH();
  } else if (nb == 1 && n >= 128) {
    const int W = n + nrhs;
    const int cw = std::min(64, std::max(2, (W + 147) / 148));
    const int G = (W + cw - 1) / cw;
    int *piv = c.ws.alloc<int>(2);
    double2 *fac = c.ws.alloc<double2>(2 * (i64)n);
    // one cooperative launch when every CTA fits on the device at once, else one launch per step
    static std::atomic<int> coop_ok[64];  // per device: 0 unknown, 1 yes, -1 no (host threads may race here)
    int dev = 0;
    NEDY_CUDA(cudaGetDevice(&dev));
    NEDY_REQUIRE(dev < 64, "device index out of range");
    if (coop_ok[dev].load() == 0) {
      int coop = 0, sms = 0, per_sm = 0;
      NEDY_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
      NEDY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      NEDY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gj_coop_kernel, TPB, 0));
      coop_ok[dev].store(coop && (i64)per_sm * sms >= 148 ? 1 : -1);
    }
    int sms = 0, per_sm = 0;
    NEDY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    NEDY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gj_coop_kernel, TPB, 0));
    if (coop_ok[dev].load() > 0 && G <= per_sm * sms) {
      unsigned *bar = c.ws.alloc<unsigned>(2);
      NEDY_CUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), c.stream));
      int nn = n, nr = nrhs, cww = cw;
      void *args[] = {&nn, &nr, &A, &B, &cww, &piv, &fac, &st, &bar};
      NEDY_CUDA(cudaLaunchCooperativeKernel((const void *)gj_coop_kernel, dim3(G), dim3(TPB), args, 0, c.stream));
      NEDY_CHECK_LAUNCH();
    } else {
      gj_first_pivot_kernel<<<1, TPB, 0, c.stream>>>(n, nrhs, A, B, piv, fac);
      NEDY_CHECK_LAUNCH();
      for (int col = 0; col < n; col++) {
        gj_step_kernel<<<G, TPB, 0, c.stream>>>(n, nrhs, A, B, col, cw, piv, fac, st);
        NEDY_CHECK_LAUNCH();
      }
    }
  } else {
    gj_kernel<<<nb, TPB, 0, c.stream>>>(n, nrhs, A, sA, B, sB, st);
    NEDY_CHECK_LAUNCH();
  }
  c.pending_status.push_back({st, nb});
}

// ---------------------------------------------------------------------------------
// M(t') = (i bd0/dt + mu) I - hmf(t') - dt w0 Sig^R(t',t')  for t' = t0 + b; B = I
__global__ void build_M_kernel(int N, int nb, int t0, const double2 *hmf, DevGF S, double bd0, double mu, double dt,
                               double w0, double2 *Mout, double2 *Iout) {
  const i64 es = (i64)N * N;
  GRID_STRIDE(idx, es * nb) {
    const int b = (int)(idx / es), e = (int)(idx - (i64)b * es);
    const int i = e / N, j = e - (e / N) * N;
    const int t = t0 + b;
    const double2 h = hmf[(i64)t * es + e];
    const double2 s = S.retptr(t, t)[e];
    double2 m = make_double2(-h.x - dt * w0 * s.x, -h.y - dt * w0 * s.y);
    if (i == j) { m.x += mu; m.y += bd0 / dt; }
    Mout[idx] = m;
    Iout[idx] = make_double2(i == j ? 1.0 : 0.0, 0.0);
  }
}

// ---------------------------------------------------------------------------------
// Retarded start block (dyson_step.h:26-71): M (kN x kN) and Q (kN x N)
__global__ void ret_start_kernel(int N, int k, int T, DevGF G, DevGF S, const double2 *hmf, const double *pdiff,
                                 const double *greg, int greg_ld, double mu, double dt, double2 *M, double2 *Q) {
  const i64 es = (i64)N * N;
  const int kn = k * N;
  // M: element (r, c) with r = (n-1)*N + i, c = (l-1)*N + j for n, l in 1..k
  GRID_STRIDE(idx, (i64)kn * kn + (i64)kn * N) {
    if (idx < (i64)kn * kn) {
      const int r = (int)(idx / kn), cc = (int)(idx - (i64)r * kn);
      const int n = r / N + 1, i = r % N, l = cc / N + 1, j = cc % N;
      // derivative: -(-i/dt) pdiff(n,l) I  = +(i/dt) pdiff
      double2 m = make_double2(0.0, 0.0);
      if (i == j) m.y += pdiff[n * (k + 1) + l] / dt;
      if (l == n) {
        const double2 h = hmf[(i64)(T - n) * es + (i64)j * N + i];  // hmf^T
        m.x -= h.x; m.y -= h.y;
        if (i == j) m.x += mu;
      }
      const double w = dt * greg[n * greg_ld + l];
      if (T - l >= T - n) {  // l <= n: -dt w Sig^R(T-l, T-n)^T
        const double2 s = S.retptr(T - l, T - n)[(i64)j * N + i];
        m.x -= w * s.x; m.y -= w * s.y;
      } else {  // +dt w conj(Sig^R(T-n, T-l))
        const double2 s = S.retptr(T - n, T - l)[(i64)i * N + j];
        m.x += w * s.x; m.y -= w * s.y;
      }
      M[idx] = m;
    } else {
      const i64 q = idx - (i64)kn * kn;
      const int r = (int)(q / N), j = (int)(q - (i64)r * N);
      const int n = r / N + 1, i = r % N;
      // Q_n = (-i/dt) pdiff(n,0) G^R(T,T)^T + dt w(n,0) (G^R(T,T) Sig^R(T,T-n))^T
      const double2 *g = G.retptr(T, T);
      double2 v = make_double2(0.0, 0.0);
      const double2 gt = g[(i64)j * N + i];
      const double pd = pdiff[n * (k + 1)] / dt;
      v.x += pd * gt.y;  // (-i) * gt * pd
      v.y -= pd * gt.x;
      double2 acc = czero();  // (G S)^T[i][j] = (G S)[j][i] = sum_c G[j][c] S[c][i]
      const double2 *s = S.retptr(T, T - n);
      for (int c2 = 0; c2 < N; c2++) acc = cadd(acc, cmul(g[(i64)j * N + c2], s[(i64)c2 * N + i]));
      const double w = dt * greg[n * greg_ld];
      v.x += w * acc.x; v.y += w * acc.y;
      Q[q] = v;
    }
  }
}

// G^R(T, T-l-1) = X_l^T for l < k, and the error norm contribution
__global__ void ret_start_store(int N, int k, int T, DevGF G, const double2 *X, double *err) {
  const i64 es = (i64)N * N;
  GRID_STRIDE(idx, es * k) {
    const int l = (int)(idx / es), e = (int)(idx - (i64)l * es);
    const int i = e / N, j = e - (e / N) * N;
    double2 *dst = G.retptr(T, T - l - 1) + e;
    const double2 v = X[(i64)l * es + (i64)j * N + i];
    const double2 d = csub(*dst, v);
    add_warp(&err[l], d.x * d.x + d.y * d.y);
    *dst = v;
  }
}

// One retarded Volterra step (dyson_step.h:88-106): Qh = dt Q_n + sum_l bd(l)(-i/dt) G^R(T,T-n+l);
// G^R(T,T-n) = Qh * Minv(T-n).  One CTA per output row.
__global__ void ret_step_kernel(int N, int k, int T, int n, DevGF G, const double2 *Q, const double2 *Minv,
                                const double *bd, double dt, double *err) {
  extern __shared__ double2 row[];
  const i64 es = (i64)N * N;
  const int i = blockIdx.x;
  for (int c = threadIdx.x; c < N; c += blockDim.x) {
    double2 v = cscale(Q[(i64)n * es + (i64)i * N + c], dt);
    for (int l = 1; l <= k + 1; l++) {
      const double2 g = G.retptr(T, T - n + l)[(i64)i * N + c];
      const double f = bd[l] / dt;
      v.x += f * g.y;  // (-i) f g
      v.y -= f * g.x;
    }
    row[c] = v;
  }
  __syncthreads();
  const double2 *Mi = Minv + (i64)(T - n) * es;
  for (int j = threadIdx.x; j < N; j += blockDim.x) {
    double2 acc = czero();
    for (int c = 0; c < N; c++) acc = cadd(acc, cmul(row[c], Mi[(i64)c * N + j]));
    double2 *dst = G.retptr(T, T - n) + (i64)i * N + j;
    const double2 d = csub(*dst, acc);
    add_warp(&err[n], d.x * d.x + d.y * d.y);
    *dst = acc;
  }
}

// ---------------------------------------------------------------------------------
// History pushes of the sequential sweeps: C_b += s_b A_b B_b + g_b Y for nb blocks of
// nao x nao (nao <= 64), b = 0..nb-1, one CTA per (block, 32-column half).  Both operands are
// staged whole by cp.async (A 64 x 64, B 64 x 32) and multiplied on the FP64 tensor path (DMMA
// m8n8k4), eight warps of 16 x 16 outputs; no K loop, no atomics (every block has its own C).
// Y is the pushed block and g_b = -i bd(m - a) dscale the derivative weight of target
// m = m0 + b when 1 <= m - a <= k + 1 and m <= m_dmax, so that the step itself needs only Q_m:
//   PUSH_RET (dyson_step.h:89-92, 103-106): A = Y = G^R(T, T-a), B_b = Sig^R(T-a, T-m0-b),
//            C_b = Q_{m0+b}, s_b = gregT[a ld + m0 + b], dscale = 1 / dt^2
//   PUSH_LES (dyson_step.h:266-274, the sum over l pushed from l = a): A_b = Sig^R(m0+b, a),
//            B = Y = X_a, C_b = Q_{m0+b}, s_b = dt greg[(m0+b) ld + a], dscale = 1 / dt
enum PushMode { PUSH_RET = 0, PUSH_LES = 1 };
constexpr int PB_LDA = 68, PB_LDB = 34;  // padded strides: conflict-free quarter-warp fragment reads
constexpr int PB_SMEM = (64 * PB_LDA + 64 * PB_LDB) * 16;

__device__ __forceinline__ void pb_cp16(void *dst, const void *src, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(src), "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void pb_dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// this warp's 16 x 16 outputs of the 64 x 32 half-tile: acc = As (64 x 64) * Bs (64 x 32)
__device__ __forceinline__ void pb_product(const double2 *As, const double2 *Bs, int N, double (&cr)[2][2][2],
                                           double (&ci)[2][2][2]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = (warp >> 1) * 16, wn = (warp & 1) * 16;
  const int kmax = (N + 3) >> 2;
  for (int kk = 0; kk < kmax; kk++) {
    const int k = kk * 4 + (lane & 3);
    double ar[2], ai[2], br[2], bi[2];
#pragma unroll
    for (int i = 0; i < 2; i++) {
      const double2 v = As[(wm + i * 8 + (lane >> 2)) * PB_LDA + k];
      ar[i] = v.x;
      ai[i] = v.y;
    }
#pragma unroll
    for (int j = 0; j < 2; j++) {
      const double2 v = Bs[k * PB_LDB + wn + j * 8 + (lane >> 2)];
      br[j] = v.x;
      bi[j] = v.y;
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 2; j++) {
        pb_dmma(cr[i][j][0], cr[i][j][1], ar[i], br[j]);
        pb_dmma(cr[i][j][0], cr[i][j][1], -ai[i], bi[j]);
        pb_dmma(ci[i][j][0], ci[i][j][1], ar[i], bi[j]);
        pb_dmma(ci[i][j][0], ci[i][j][1], ai[i], br[j]);
      }
  }
}

// Stages the 64 x 64 block A and the 32 columns [n0, n0 + 32) of the block B (nao x nao,
// row-major; zero outside) by cp.async; the caller waits.
__device__ __forceinline__ void pb_stage(double2 *dst, int ld, const double2 *src, int N, int rows, int cols,
                                         int c0) {
  const int sh = cols == 64 ? 6 : 5;
  for (int i = threadIdx.x; i < rows * cols; i += blockDim.x) {
    const int r = i >> sh, c = i & (cols - 1);
    const bool v = r < N && c0 + c < N;
    pb_cp16(dst + r * ld + c, v ? src + (i64)r * N + c0 + c : src, v);
  }
}

// Shared memory of push_blocks_kernel: the operand shared by all blocks once, the varying
// one double-buffered (PUSH_RET: A shared, B_b varies; PUSH_LES: B shared, A_b varies).
constexpr int PB_ABYTES = 64 * PB_LDA * 16, PB_BBYTES = 64 * PB_LDB * 16;
inline int push_smem(int mode) { return mode == PUSH_RET ? PB_ABYTES + 2 * PB_BBYTES : PB_BBYTES + 2 * PB_ABYTES; }

__global__ void __launch_bounds__(256, 1)
    push_blocks_kernel(int mode, int N, int T, int a, int m0, int nb, DevGF G, DevGF S, const double2 *X,
                       double2 *Q, const double *w, i64 w_stride, double alpha, const double *bd, double dscale,
                       int k, int m_dmax) {
  extern __shared__ double2 pbs[];
  const bool ret = mode == PUSH_RET;
  const int n0 = blockIdx.y * 32;
  const i64 es = (i64)N * N;
  // shared operand, then the two buffers of the varying one
  double2 *sh = pbs, *v0 = pbs + (ret ? 64 * PB_LDA : 64 * PB_LDB);
  const int vstride = ret ? 64 * PB_LDB : 64 * PB_LDA;
  auto stage_var = [&](int b, double2 *dst) {
    if (ret)
      pb_stage(dst, PB_LDB, S.retptr(T - a, T - m0 - b), N, 64, 32, n0);
    else
      pb_stage(dst, PB_LDA, S.retptr(m0 + b, a), N, 64, 64, 0);
  };
  if (ret)
    pb_stage(sh, PB_LDA, G.retptr(T, T - a), N, 64, 64, 0);
  else
    pb_stage(sh, PB_LDB, X + (i64)a * es, N, 64, 32, n0);
  if ((int)blockIdx.x < nb) stage_var(blockIdx.x, v0);
  asm volatile("cp.async.commit_group;\n" ::);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = (warp >> 1) * 16, wn = (warp & 1) * 16;
  int it = 0;
  for (int b = blockIdx.x; b < nb; b += gridDim.x, it++) {
    double2 *cur = v0 + (it & 1) * vstride, *nxt = v0 + ((it + 1) & 1) * vstride;
    if (b + (int)gridDim.x < nb) stage_var(b + gridDim.x, nxt);  // overlaps this block's product
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 1;\n" ::);
    __syncthreads();
    const double2 *As = ret ? sh : cur, *Bs = ret ? cur : sh;
    double cr[2][2][2] = {}, ci[2][2][2] = {};
    pb_product(As, Bs, N, cr, ci);
    double2 *C = Q + (i64)(m0 + b) * es;
    const double s = alpha * w[(i64)b * w_stride];
    const int dl = m0 + b - a;
    const double g = (dl >= 1 && dl <= k + 1 && m0 + b <= m_dmax) ? bd[dl] * dscale : 0.0;
#pragma unroll
    for (int i = 0; i < 2; i++) {
      const int r = wm + i * 8 + (lane >> 2);
      if (r >= N) continue;
#pragma unroll
      for (int j = 0; j < 2; j++)
#pragma unroll
        for (int c = 0; c < 2; c++) {
          const int col = n0 + wn + j * 8 + (lane & 3) * 2 + c;
          if (col >= N) continue;
          // the pushed block Y (derivative term) is the shared operand
          const double2 y = ret ? sh[r * PB_LDA + col] : sh[r * PB_LDB + col - n0];
          double2 &o = C[(i64)r * N + col];
          o.x += s * cr[i][j][c] + g * y.y;  // -i g y
          o.y += s * ci[i][j][c] - g * y.x;
        }
    }
    __syncthreads();  // every thread is done with `cur` before the next prefetch reuses it
  }
  asm volatile("cp.async.wait_group 0;\n" ::);
}

// One step of a sequential sweep as a block product on the FP64 tensor path (nao <= 64), one
// CTA per 32-column half; the derivative terms are already in Q (pushed with the history):
//   STEP_RET (dyson_step.h:88-101): G^R(T, T-a) = dt Q_a Minv(T-a), and err[a] += |change|^2
//   STEP_LES (dyson_step.h:271-279): X_a = Minv(a) Q_a
enum StepMode { STEP_RET = 0, STEP_LES = 1 };
__global__ void __launch_bounds__(256, 1)
    step_block_kernel(int mode, int N, int T, int a, DevGF G, const double2 *Q, double2 *X, const double2 *Minv,
                      double dt, double *err) {
  extern __shared__ double2 pbs[];
  double2 *As = pbs, *Bs = pbs + 64 * PB_LDA;
  const int n0 = blockIdx.y * 32;
  const i64 es = (i64)N * N;
  const bool ret = mode == STEP_RET;
  pb_stage(As, PB_LDA, ret ? Q + (i64)a * es : Minv + (i64)a * es, N, 64, 64, 0);
  pb_stage(Bs, PB_LDB, ret ? Minv + (i64)(T - a) * es : Q + (i64)a * es, N, 64, 32, n0);
  asm volatile("cp.async.commit_group;\n" ::);
  asm volatile("cp.async.wait_group 0;\n" ::);
  __syncthreads();
  double cr[2][2][2] = {}, ci[2][2][2] = {};
  pb_product(As, Bs, N, cr, ci);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = (warp >> 1) * 16, wn = (warp & 1) * 16;
  double2 *C = ret ? G.retptr(T, T - a) : X + (i64)a * es;
  const double sc = ret ? dt : 1.0;
#pragma unroll
  for (int i = 0; i < 2; i++) {
    const int r = wm + i * 8 + (lane >> 2);
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const int col = n0 + wn + j * 8 + (lane & 3) * 2 + c;
        const bool ok = r < N && col < N;
        double d2 = 0.0;
        if (ok) {
          double2 &o = C[(i64)r * N + col];
          const double2 v = make_double2(sc * cr[i][j][c], sc * ci[i][j][c]);
          const double2 d = csub(o, v);
          d2 = d.x * d.x + d.y * d.y;
          o = v;
        }
        if (ret) add_warp(&err[a], d2);
      }
  }
}

// Launches push_blocks_kernel for nb blocks (nao <= 64); false when nao is larger.  One CTA
// per SM and column half, each looping over its blocks.
bool push_blocks(Ctx &c, int mode, int N, int T, int a, int m0, int nb, const DevGF &G, const DevGF &S,
                 const double2 *X, double2 *Q, const double *w, i64 w_stride, double alpha, double dscale,
                 int m_dmax) {
  if (N > 64) return false;
  if (nb <= 0) return true;
  static std::atomic<bool> attr_set[64];  // per device (host threads may race here)
  static std::atomic<int> sms_of[64];
  int dev = 0;
  NEDY_CUDA(cudaGetDevice(&dev));
  NEDY_REQUIRE(dev < 64, "device index out of range");
  if (!attr_set[dev].load()) {
    NEDY_CUDA(cudaFuncSetAttribute(push_blocks_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   std::max(push_smem(PUSH_RET), push_smem(PUSH_LES))));
    int sms = 0;
    NEDY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    sms_of[dev].store(sms);
    attr_set[dev].store(true);
  }
  const int halves = N > 32 ? 2 : 1;
  const int gx = std::max(1, std::min(nb, sms_of[dev].load() / halves));
  push_blocks_kernel<<<dim3((unsigned)gx, halves), 256, push_smem(mode), c.stream>>>(
      mode, N, T, a, m0, nb, G, S, X, Q, w, w_stride, alpha, c.d_bd, dscale, c.k, m_dmax);
  NEDY_CHECK_LAUNCH();
  return true;
}

// Launches step_block_kernel (nao <= 64); false when nao is larger.
bool step_block(Ctx &c, int mode, int N, int T, int a, const DevGF &G, const double2 *Q, double2 *X, double *err) {
  if (N > 64) return false;
  static std::atomic<bool> attr_set[64];  // per device (host threads may race here)
  int dev = 0;
  NEDY_CUDA(cudaGetDevice(&dev));
  NEDY_REQUIRE(dev < 64, "device index out of range");
  if (!attr_set[dev].load()) {
    NEDY_CUDA(cudaFuncSetAttribute(step_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, PB_SMEM));
    attr_set[dev].store(true);
  }
  step_block_kernel<<<dim3(1, N > 32 ? 2 : 1), 256, PB_SMEM, c.stream>>>(mode, N, T, a, G, Q, X, c.Minv, c.dt,
                                                                        err);
  NEDY_CHECK_LAUNCH();
  return true;
}

// ---------------------------------------------------------------------------------
// tv: derivative history terms  out += -(i/dt) bd(l) G^tv(T-l, .)
__global__ void tv_bd_kernel(i64 n, int k, int T, DevGF G, const double *bd, double dt, double2 *out) {
  GRID_STRIDE(idx, n) {
    double2 v = out[idx];
    for (int l = 1; l <= k + 1; l++) {
      const double2 g = G.tvptr(T - l, 0)[idx];
      const double f = bd[l] / dt;
      v.x += f * g.y;
      v.y -= f * g.x;
    }
    out[idx] = v;
  }
}

// per-block squared difference norms: err[b] = ||A_b - B_b||^2 (accumulated)
__global__ void diffnorm_kernel(int N, int nb, const double2 *A, const double2 *B, double *err) {
  const i64 es = (i64)N * N;
  GRID_STRIDE(idx, es * nb) {
    const int b = (int)(idx / es);
    const double2 d = csub(A[idx], B[idx]);
    add_warp(&err[b], d.x * d.x + d.y * d.y);
  }
}

// ---------------------------------------------------------------------------------
// les helpers
// G^<(0,n) = -G^tv(n,0)^+ ; err
__global__ void les_init_kernel(int N, int n, DevGF G, double2 *X0, double *err) {
  const i64 es = (i64)N * N;
  GRID_STRIDE(e, es) {
    const int i = (int)(e / N), j = (int)(e - (e / N) * N);
    const double2 t = G.tvptr(n, 0)[(i64)j * N + i];
    const double2 v = make_double2(-t.x, t.y);
    double2 *dst = G.lesptr(0, n) + e;
    const double2 d = csub(*dst, v);
    add_warp(err, d.x * d.x + d.y * d.y);
    *dst = v;
    X0[e] = v;
  }
}

// NTT_j = sig * i * G^tv(n, ntau-j)^+   (dyson_integrals.h:424-425) ; UB = sum_j u_j NTT_j
__global__ void ntt_kernel(int N, int ntau, int n, DevGF G, int sig, double2 *ntt) {
  const i64 es = (i64)N * N;
  GRID_STRIDE(idx, es * (ntau + 1)) {
    const int j = (int)(idx / es), e = (int)(idx - (i64)j * es);
    const int a = e / N, b = e - (e / N) * N;
    const double2 g = G.tvptr(n, ntau - j)[(i64)b * N + a];  // conj transpose
    // sig * i * conj(g)
    ntt[idx] = make_double2(sig * g.y, sig * g.x);
  }
}
// B''_j = (beta/2) (w_j NTT_j + ctop u_j UB),  UB = sum_i u_i NTT_i (one CTA per element column chunk)
__global__ void lesser_weights_kernel(int N, int ntau, const double2 *ntt, const double *w, const double *u,
                                      double ctop, double beta, double2 *out) {
  const i64 es = (i64)N * N;
  GRID_STRIDE(e, es) {
    double2 ub = czero();
    for (int i = 0; i <= ntau; i++) ub = cadd(ub, cscale(ntt[(i64)i * es + e], u[i]));
    for (int j = 0; j <= ntau; j++) {
      double2 v = cadd(cscale(ntt[(i64)j * es + e], w[j]), cscale(ub, ctop * u[j]));
      out[(i64)j * es + e] = cscale(v, 0.5 * beta);
    }
  }
}
// X_j = dt w(n,j) G^R(n,j)^+  (dyson_integrals.h:355-362, m = n >= j)
__global__ void cles2_x_kernel(int N, int n, DevGF G, const double *gregrow, double dt, double2 *X) {
  const i64 es = (i64)N * N;
  GRID_STRIDE(idx, es * (n + 1)) {
    const int j = (int)(idx / es), e = (int)(idx - (i64)j * es);
    const int a = e / N, b = e - (e / N) * N;
    const double2 g = G.retptr(n, j)[(i64)b * N + a];
    const double f = dt * gregrow[j];
    X[idx] = make_double2(f * g.x, -f * g.y);
  }
}

// Lesser start block (dyson_step.h:217-252): M (kN x kN); Q_m (m=1..k) gets the G^<(0,n) terms.
__global__ void les_start_kernel(int N, int k, int n, DevGF G, DevGF S, const double2 *hmf, const double *pdiff,
                                 const double *greg, int greg_ld, double mu, double dt, const double2 *Qmain,
                                 double2 *M, double2 *Q) {
  const i64 es = (i64)N * N;
  const int kn = k * N;
  GRID_STRIDE(idx, (i64)kn * kn + (i64)kn * N) {
    if (idx < (i64)kn * kn) {
      const int r = (int)(idx / kn), cc = (int)(idx - (i64)r * kn);
      const int m = r / N + 1, i = r % N, l = cc / N + 1, j = cc % N;
      double2 v = czero();
      if (i == j) v.y += pdiff[m * (k + 1) + l] / dt;  // (i/dt) pdiff
      if (m == l) {
        const double2 h = hmf[(i64)l * es + (i64)i * N + j];
        v.x -= h.x; v.y -= h.y;
        if (i == j) v.x += mu;
      }
      const double w = dt * greg[m * greg_ld + l];
      if (m >= l) {
        const double2 s = S.retptr(m, l)[(i64)i * N + j];
        v.x -= w * s.x; v.y -= w * s.y;
      } else {
        const double2 s = S.retptr(l, m)[(i64)j * N + i];  // adjoint
        v.x += w * s.x; v.y -= w * s.y;
      }
      M[idx] = v;
    } else {
      const i64 q = idx - (i64)kn * kn;
      const int r = (int)(q / N), j = (int)(q - (i64)r * N);
      const int m = r / N + 1, i = r % N;
      // Q_m -= (i/dt) pdiff(m,0) G^<(0,n) ; Q_m += dt w(m,0) Sig^R(m,0) G^<(0,n)
      const double2 *g0 = G.lesptr(0, n);
      double2 v = Qmain[(i64)m * es + (i64)i * N + j];
      const double pd = pdiff[m * (k + 1)] / dt;
      const double2 gij = g0[(i64)i * N + j];
      v.x += pd * gij.y;  // -(i pd) g
      v.y -= pd * gij.x;
      double2 acc = czero();
      const double2 *s = S.retptr(m, 0);
      for (int c2 = 0; c2 < N; c2++) acc = cadd(acc, cmul(s[(i64)i * N + c2], g0[(i64)c2 * N + j]));
      const double w = dt * greg[m * greg_ld];
      v.x += w * acc.x; v.y += w * acc.y;
      Q[q] = v;  // packed (kN x N) right-hand side for rows m = 1..k
    }
  }
}

// One lesser Volterra step (dyson_step.h:257-280): Qh = Q_m - sum_l (i/dt) bd(l) X_{m-l}; X_m = Minv(m) Qh
__global__ void les_step_kernel(int N, int k, int m, const double2 *Q, double2 *X, const double2 *Minv,
                                const double *bd, double dt) {
  extern __shared__ double2 col[];
  const i64 es = (i64)N * N;
  const int j = blockIdx.x;  // output column
  for (int c = threadIdx.x; c < N; c += blockDim.x) {
    double2 v = Q[(i64)m * es + (i64)c * N + j];
    for (int l = 1; l <= k + 1; l++) {
      const double2 x = X[(i64)(m - l) * es + (i64)c * N + j];
      const double f = bd[l] / dt;
      v.x += f * x.y;  // -(i f) x
      v.y -= f * x.x;
    }
    col[c] = v;
  }
  __syncthreads();
  const double2 *Mi = Minv + (i64)m * es;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    double2 acc = czero();
    for (int c = 0; c < N; c++) acc = cadd(acc, cmul(Mi[(i64)i * N + c], col[c]));
    X[(i64)m * es + (i64)i * N + j] = acc;
  }
}

// Diagonal G^<(n,n) (dyson_step.h:284-310), one CTA.
__global__ void les_diag_kernel(int N, int k, int n, DevGF G, DevGF S, const double2 *hmf, const double *ex,
                                const double *bd, double wnn, double mu, double dt, const double2 *Q, double2 *X) {
  extern __shared__ double2 sm[];
  const i64 es = (i64)N * N;
  double2 *xn = sm, *qn = sm + es;
  for (int e = threadIdx.x; e < es; e += blockDim.x) {
    double2 v = czero();
    for (int jj = 0; jj <= k; jj++) v = cadd(v, cscale(G.lesptr(n - jj - 1, n - jj - 1)[e], ex[jj]));
    xn[e] = v;
  }
  __syncthreads();
  const double2 *sr = S.retptr(n, n);
  const double2 *h = hmf + (i64)n * es;
  for (int e = threadIdx.x; e < es; e += blockDim.x) {
    const int i = e / N, j = e - (e / N) * N;
    double2 acc = Q[(i64)n * es + e];
    double2 a1 = czero(), a2 = czero();
    for (int c = 0; c < N; c++) {
      a1 = cadd(a1, cmul(sr[(i64)i * N + c], xn[(i64)c * N + j]));
      double2 hm = h[(i64)i * N + c];
      if (c == i) hm.x -= mu;
      a2 = cadd(a2, cmul(hm, xn[(i64)c * N + j]));
    }
    acc = cadd(acc, cadd(cscale(a1, dt * wnn), a2));
    qn[e] = acc;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < es; e += blockDim.x) {
    const int i = e / N, j = e - (e / N) * N;
    const double2 a = qn[e], b = qn[(i64)j * N + i];
    // -i (Q + Q^+)
    const double2 s = make_double2(a.x + b.x, a.y - b.y);
    double2 v = make_double2(s.y, -s.x);
    for (int l = 1; l <= k + 1; l++) v = csub(v, cscale(G.lesptr(n - l, n - l)[e], bd[l] / dt));
    X[(i64)n * es + e] = cscale(v, dt / bd[0]);
  }
}

// ---------------------------------------------------------------------------------
// Extrapolate (dyson.cpp:47-117)
__global__ void extrap_tv_kernel(int N, int k, int n, DevGF G, const double *exw) {
  const i64 tot = (i64)N * N * (G.ntau + 1);
  GRID_STRIDE(idx, tot) {
    double2 v = czero();
    for (int j = 0; j <= k; j++) v = cadd(v, cscale(G.tvptr(n - j - 1, 0)[idx], exw[j]));
    G.tvptr(n, 0)[idx] = v;
  }
}
__global__ void extrap_ret_kernel(int N, int k, int n, DevGF G, const double *exw) {
  const i64 es = (i64)N * N;
  GRID_STRIDE(idx, es * (n + 1)) {
    const int col = (int)(idx / es), e = (int)(idx - (i64)col * es);  // G^R(n, col)
    const int i = e / N, j = e - (e / N) * N;
    double2 v = czero();
    if (col > k) {  // col = n - l with l < n - k
      const int l = n - col;
      for (int jj = 0; jj <= k; jj++) v = cadd(v, cscale(G.retptr(n - jj - 1, n - l - jj - 1)[e], exw[jj]));
    } else {
      const int l = col;
      const int jcut = (l <= n - k - 1) ? k : (n - l - 1);
      for (int jj = 0; jj <= jcut; jj++) v = cadd(v, cscale(G.retptr(n - jj - 1, l)[e], exw[jj]));
      for (int jj = jcut + 1; jj <= k; jj++) {
        const double2 a = G.retptr(l, n - jj - 1)[(i64)j * N + i];
        v.x -= exw[jj] * a.x;
        v.y += exw[jj] * a.y;
      }
    }
    G.retptr(n, col)[e] = v;
  }
}
__global__ void extrap_les_kernel(int N, int k, int n, DevGF G, const double *exw) {
  const i64 es = (i64)N * N;
  GRID_STRIDE(idx, es * (n + 1)) {
    const int l = (int)(idx / es), e = (int)(idx - (i64)l * es);  // G^<(l, n)
    const int i = e / N, j = e - (e / N) * N;
    double2 v = czero();
    if (l == 0) {
      const double2 t = G.tvptr(n, 0)[(i64)j * N + i];
      v = make_double2(-t.x, t.y);
    } else if (l <= k) {
      const int jcut = (k > n - l - 1) ? (n - l - 1) : k;
      for (int jj = 0; jj <= jcut; jj++) v = cadd(v, cscale(G.lesptr(l, n - 1 - jj)[e], exw[jj]));
      for (int jj = jcut + 1; jj <= k; jj++) {
        const double2 a = G.lesptr(n - 1 - jj, l)[(i64)j * N + i];
        v.x -= exw[jj] * a.x;
        v.y += exw[jj] * a.y;
      }
    } else {
      for (int jj = 0; jj <= k; jj++) v = cadd(v, cscale(G.lesptr(l - jj - 1, n - jj - 1)[e], exw[jj]));
    }
    G.lesptr(l, n)[e] = v;
  }
}

// rho = i sig G^<(T,T)
__global__ void dm_kernel(int N, int T, DevGF G, double2 *rho) {
  GRID_STRIDE(e, (i64)N * N) {
    const double2 g = G.lesptr(T, T)[e];
    rho[e] = make_double2(-G.sig * g.y, G.sig * g.x);
  }
}

__global__ void set_diag_kernel(int N, double2 *blk, double2 v) {
  GRID_STRIDE(e, (i64)N * N) {
    const int i = (int)(e / N), j = (int)(e - (e / N) * N);
    blk[e] = i == j ? v : czero();
  }
}

__global__ void add_kernel(i64 n, const double2 *a, double2 *out) {
  GRID_STRIDE(i, n) out[i] = cadd(out[i], a[i]);
}

[[maybe_unused]] double *dev_table(Ctx &c, const std::vector<double> &h) {
  double *d = c.ws.alloc<double>((i64)h.size());
  NEDY_CUDA(cudaMemcpyAsync(d, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, c.stream));
  return d;
}

double sum_dev(Ctx &c, const double *d, int n, bool sqrt_each) {
  std::vector<double> h(n);
  NEDY_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream));
  NEDY_CUDA(cudaStreamSynchronize(c.stream));
  double s = 0;
  for (double v : h) s += sqrt_each ? std::sqrt(v) : v;
  return s;
}

} // namespace

// ===================================================================================
void gj_public(Ctx &c, int n, int nrhs, int nb, double2 *A, i64 sA, double2 *B, i64 sB) { gj(c, n, nrhs, nb, A, sA, B, sB); }

void check_status(Ctx &c) {
  for (auto &p : c.pending_status) {
    std::vector<int> h(p.second);
    NEDY_CUDA(cudaMemcpyAsync(h.data(), p.first, sizeof(int) * p.second, cudaMemcpyDeviceToHost, c.stream));
    NEDY_CUDA(cudaStreamSynchronize(c.stream));
    for (int v : h)
      if (v) {
        c.pending_status.clear();
        if (v == 2) throw CudaError("Dyson solve: a bounded grid barrier timed out");
        throw ArgError("singular matrix in a Dyson solve");
      }
  }
  c.pending_status.clear();
}

void ensure_tables(Ctx &c) {
  if (c.greg && c.greg_n == c.nt) return;
  int n = c.nt + 1;
  std::vector<double> g((size_t)n * n, 0.0), gt((size_t)n * n, 0.0);
  for (int a = 0; a < n; a++) {
    int top = std::max(a, c.k);
    for (int j = 0; j <= top && j < n; j++) {
      double w = c.W.gregory(a, j);
      g[(size_t)a * n + j] = w;
      gt[(size_t)j * n + a] = w;
    }
  }
  if (c.greg) { NEDY_CUDA(cudaStreamSynchronize(c.stream)); cudaFree(c.greg); }
  NEDY_CUDA(cudaMalloc(&c.greg, sizeof(double) * 2 * (size_t)n * n));
  c.gregT = c.greg + (size_t)n * n;
  h2d_sync(c.greg, g.data(), sizeof(double) * g.size(), c.stream);
  h2d_sync(c.gregT, gt.data(), sizeof(double) * gt.size(), c.stream);
  std::vector<double> small;
  small.insert(small.end(), c.W.poly_diff.begin(), c.W.poly_diff.end());
  small.insert(small.end(), c.W.bd.begin(), c.W.bd.end());
  small.insert(small.end(), c.W.ex.begin(), c.W.ex.end());
  small.insert(small.end(), c.col.w.begin(), c.col.w.end());
  small.insert(small.end(), c.col.u.begin(), c.col.u.end());
  if (c.small) cudaFree(c.small);
  NEDY_CUDA(cudaMalloc(&c.small, sizeof(double) * small.size()));
  h2d_sync(c.small, small.data(), sizeof(double) * small.size(), c.stream);
  c.d_pdiff = c.small;
  c.d_bd = c.d_pdiff + c.W.poly_diff.size();
  c.d_ex = c.d_bd + c.W.bd.size();
  c.d_w = c.d_ex + c.W.ex.size();
  c.d_u = c.d_w + c.col.w.size();
  c.greg_n = c.nt;
}

void update_minv(Ctx &c, const DevGF &Sig, const double2 *hmf, double mu, int t0, int t1) {
  int N = Sig.nao, nb = t1 - t0 + 1;
  if (nb <= 0) return;
  i64 es = (i64)N * N;
  double2 *M = c.ws.alloc<double2>(es * nb);
  double2 *Mi = c.Minv + (i64)t0 * es;
  build_M_kernel<<<nblk(es * nb), TPB, 0, c.stream>>>(N, nb, t0, hmf, Sig, c.W.bd[0], mu, c.dt, c.W.omega(0), M, Mi);
  NEDY_CHECK_LAUNCH();
  gj(c, N, N, nb, M, es, Mi, es);
}

void ensure_minv(Ctx &c, int N) {
  if (c.Minv && c.Minv_cap >= (c.nt + 1) && c.Minv_nao == N) return;
  if (c.Minv) cudaFree(c.Minv);
  NEDY_CUDA(cudaMalloc(&c.Minv, sizeof(double2) * (size_t)(c.nt + 1) * N * N));
  c.Minv_cap = c.nt + 1;
  c.Minv_nao = N;
}

void ensure_mixing_kernel(Ctx &c, const DevGF &G) {
  const int N = G.nao, np = G.ntau + 1;
  const i64 es = (i64)N * N;
  if (c.mixK && c.mixK_src == G.mat && c.mixK_ver == G.mat_version && c.mixK_nao == N) return;
  // two cached kernels: swap in the other one if it matches, else rebuild the older one
  std::swap(c.mixK, c.mixK_alt);
  std::swap(c.mixK_src, c.mixK_alt_src);
  std::swap(c.mixK_ver, c.mixK_alt_ver);
  std::swap(c.mixK_nao, c.mixK_alt_nao);
  if (c.mixK && c.mixK_src == G.mat && c.mixK_ver == G.mat_version && c.mixK_nao == N) return;
  if (c.mixK && c.mixK_nao != N) { cudaFree(c.mixK); c.mixK = nullptr; }
  if (!c.mixK) NEDY_CUDA(cudaMalloc(&c.mixK, sizeof(double2) * (size_t)np * np * es));
  build_tau_kernel(c, G.mat, N, (double)G.sig, c.mixK);
  c.mixK_src = G.mat;
  c.mixK_ver = G.mat_version;
  c.mixK_nao = N;
}

// K[m][i] = int_0^beta L_i(tau') B(tau' - tau_m) dtau' for the degree-ntau interpolant B of
// the np nodal blocks Bn (extended to negative arguments by B(x) = sig B(x + beta)), L_i the
// Lagrange polynomial of node i: then int_0^beta f(tau') B(tau' - tau_m) dtau' = sum_i f_i K[m][i]
// for any degree-ntau f.  The quadrature tables split the integral at tau_m (collocation.cpp).
void build_tau_kernel(Ctx &c, const double2 *Bn, int N, double sig, double2 *K) {
  const int np = c.ntau + 1;
  const i64 es = (i64)N * N;
  build_mixing_eval(c.col);
  const int Q2 = 2 * c.col.Q;
  // sign of the antiperiodic extension folded into the first half of EB
  std::vector<double> EBs(c.col.EB);
  for (int m = 0; m < np; m++)
    for (int q = 0; q < c.col.Q; q++)
      for (int j = 0; j < np; j++) EBs[((size_t)m * Q2 + q) * np + j] *= sig;
  const int chunk = std::max(1, (int)std::min<i64>(np, (i64)(2LL << 30) / (sizeof(double2) * Q2 * es)));
  double *dEA = nullptr, *dEB = nullptr;
  double2 *BB = nullptr;
  NEDY_CUDA(cudaMalloc(&dEA, sizeof(double) * c.col.EA.size()));
  NEDY_CUDA(cudaMalloc(&dEB, sizeof(double) * EBs.size()));
  NEDY_CUDA(cudaMalloc(&BB, sizeof(double2) * (size_t)chunk * Q2 * es));
  h2d_sync(dEA, c.col.EA.data(), sizeof(double) * c.col.EA.size(), c.stream);
  h2d_sync(dEB, EBs.data(), sizeof(double) * EBs.size(), c.stream);
  for (int m0 = 0; m0 < np; m0 += chunk) {
    int nm = std::min(chunk, np - m0);
    {  // BB[m] = EB[m] (2Q x np) * Bn (np x N^2)
      GemmArgs g;
      g.M = Q2; g.N = (int)es; g.K = np; g.nb1 = nm;
      g.A = rowmajor(dEB + (size_t)m0 * Q2 * np, np); g.A.bs1 = (i64)Q2 * np; g.a_cplx = false;
      g.B = rowmajor(Bn, es);
      g.C = rowmajor(BB, es); g.C.bs1 = (i64)Q2 * es;
      gemm(g, c.stream);
    }
    {  // K[m] = (beta/2) EA[m] (np x 2Q) * BB[m]
      GemmArgs g;
      g.M = np; g.N = (int)es; g.K = Q2; g.nb1 = nm;
      g.A = rowmajor(dEA + (size_t)m0 * np * Q2, Q2); g.A.bs1 = (i64)np * Q2; g.a_cplx = false;
      g.B = rowmajor(BB, es); g.B.bs1 = (i64)Q2 * es;
      g.C = rowmajor(K + (size_t)m0 * np * es, es); g.C.bs1 = (i64)np * es;
      g.alpha = make_double2(0.5 * c.beta, 0.0);
      gemm(g, c.stream);
    }
  }
  NEDY_CUDA(cudaStreamSynchronize(c.stream));
  cudaFree(dEA);
  cudaFree(dEB);
  cudaFree(BB);
}

// out[m] (+)= sum_i A_i K[m][i]   (A_i = tv blocks of one time row), out in [m][a][b] layout
static void mixing_gemm(Ctx &c, int N, int np, const double2 *Arow, const double2 *K, double2 *out, bool real_only,
                        double2 beta) {
  const i64 es = (i64)N * N;
  GemmArgs g;
  g.M = N; g.N = (int)(np * N); g.K = (int)(np * N);
  g.A.p = Arow; g.A.rs_lo = N; g.A.cdiv = N; g.A.cs_hi = es; g.A.cs_lo = 1;
  g.B.p = K; g.B.rdiv = N; g.B.rs_hi = es; g.B.rs_lo = N; g.B.cdiv = N; g.B.cs_hi = (i64)np * es; g.B.cs_lo = 1;
  g.C.p = out; g.C.rs_lo = N; g.C.cdiv = N; g.C.cs_hi = es; g.C.cs_lo = 1;
  g.beta = beta;
  (void)real_only;
  gemm(g, c.stream);
}

// ===================================================================================
void extrapolate(Ctx &c, int n, DevGF &G) {
  NEDY_REQUIRE(n > c.k && n <= G.nt, "extrapolate: need k < n <= nt");
  ensure_tables(c);
  const int N = G.nao, k = c.k;
  const i64 es = (i64)N * N;
  extrap_tv_kernel<<<nblk(es * (G.ntau + 1)), TPB, 0, c.stream>>>(N, k, n, G, c.d_ex);
  NEDY_CHECK_LAUNCH();
  extrap_ret_kernel<<<nblk(es * (n + 1)), TPB, 0, c.stream>>>(N, k, n, G, c.d_ex);
  NEDY_CHECK_LAUNCH();
  extrap_les_kernel<<<nblk(es * (n + 1)), TPB, 0, c.stream>>>(N, k, n, G, c.d_ex);
  NEDY_CHECK_LAUNCH();
}

void get_dm(Ctx &c, const DevGF &G, int T, double2 *rho) {
  dm_kernel<<<nblk((i64)G.nao * G.nao), TPB, 0, c.stream>>>(G.nao, T, G, rho);
  NEDY_CHECK_LAUNCH();
}

void hf_decomp(Ctx &c, int nspin, double2 *const *hmf_T, const double2 *rho) {
  NEDY_REQUIRE(c.Vija, "hf: density-fitted tensor not set");
  const int N = c.df_nao, A = c.df_naux;
  const i64 es = (i64)N * N;
  double2 *rt = c.ws.alloc<double2>(es);
  double2 *Xa = c.ws.alloc<double2>(A);
  double2 *T1 = c.ws.alloc<double2>(es * A);
  // total density for the Hartree term
  NEDY_CUDA(cudaMemcpyAsync(rt, rho, sizeof(double2) * es, cudaMemcpyDeviceToDevice, c.stream));
  if (nspin == 2) {
    add_kernel<<<nblk(es), TPB, 0, c.stream>>>(es, rho + es, rt);
    NEDY_CHECK_LAUNCH();
  }
  {  // Xa = rho_flat (1 x N^2) * Vija (N^2 x A)
    GemmArgs g;
    g.M = 1; g.N = A; g.K = (int)es;
    g.A = rowmajor(rt, es);
    g.B = rowmajor(c.Vija, A); g.b_cplx = false;
    g.C = rowmajor(Xa, A);
    gemm(g, c.stream);
  }
  for (int s = 0; s < nspin; s++) {
    {  // hmf_flat += f * Vija (N^2 x A) * Xa (A x 1)
      GemmArgs g;
      g.M = (int)es; g.N = 1; g.K = A;
      g.A = rowmajor(c.Vija, A); g.a_cplx = false;
      g.B = rowmajor(Xa, 1);
      g.C = rowmajor(hmf_T[s], 1);
      g.alpha = make_double2(nspin == 1 ? 2.0 : 1.0, 0.0);
      g.beta = make_double2(1.0, 0.0);
      gemm(g, c.stream);
    }
    const double2 *rs = rho + (nspin == 2 ? s * es : 0);
    {  // T1[(i,a)][k] = sum_l Viaj[(i,a)][l] rho[k][l]
      GemmArgs g;
      g.M = N * A; g.N = N; g.K = N;
      g.A = rowmajor(c.Viaj, N); g.a_cplx = false;
      g.B = transposed(rs, N);
      g.C = rowmajor(T1, N);
      gemm(g, c.stream);
    }
    {  // hmf -= T1 (N x (a,k)) * Vaij ((a,k) x j)
      GemmArgs g;
      g.M = N; g.N = N; g.K = N * A;
      g.A = rowmajor(T1, (i64)N * A);
      g.B = rowmajor(c.Vaij, N); g.b_cplx = false;
      g.C = rowmajor(hmf_T[s], N);
      g.alpha = make_double2(-1.0, 0.0);
      g.beta = make_double2(1.0, 0.0);
      gemm(g, c.stream);
    }
  }
}

// ===================================================================================
static double dyson_ret(Ctx &c, int T, DevGF &G, const DevGF &S, const double2 *hmf, double mu) {
  const int N = G.nao, k = c.k, kn = k * N, ld = c.nt + 1;
  const i64 es = (i64)N * N;
  const double dt = c.dt;
  double *err = c.ws.alloc<double>(T + 1);
  NEDY_CUDA(cudaMemsetAsync(err, 0, sizeof(double) * (T + 1), c.stream));
  set_diag_kernel<<<nblk(es), TPB, 0, c.stream>>>(N, G.retptr(T, T), make_double2(0.0, -1.0));
  NEDY_CHECK_LAUNCH();
  double2 *M = c.ws.alloc<double2>((i64)kn * kn);
  double2 *Qs = c.ws.alloc<double2>((i64)kn * N);
  ret_start_kernel<<<nblk((i64)kn * kn + (i64)kn * N), TPB, 0, c.stream>>>(N, k, T, G, S, hmf, c.d_pdiff, c.greg, ld,
                                                                             mu, dt, M, Qs);
  NEDY_CHECK_LAUNCH();
  gj(c, kn, N, 1, M, 0, Qs, 0);
  ret_start_store<<<nblk(es * k), TPB, 0, c.stream>>>(N, k, T, G, Qs, err + 1);
  NEDY_CHECK_LAUNCH();
  if (T <= k) return sum_dev(c, err, T + 1, true);
  double2 *Q = c.ws.alloc<double2>((i64)(T + 1) * es);
  NEDY_CUDA(cudaMemsetAsync(Q, 0, sizeof(double2) * (T + 1) * es, c.stream));
  // Q_n = sum_{l<=k} w(n,l) G^R(T,T-l) Sig^R(T-l,T-n),  n = k+1..T.  For nao <= 64 the block
  // kernels also push the derivative terms -i bd(n-l)/dt^2 G^R(T,T-l) into Q_n, and the step is
  // the single product dt Q_n Minv(T-n).
  const bool fused = N <= 64;
  for (int l = 0; l <= k; l++) {
    if (fused) {
      push_blocks(c, PUSH_RET, N, T, l, k + 1, T - k, G, S, nullptr, Q, c.gregT + (i64)l * ld + (k + 1), 1, 1.0,
                  1.0 / (dt * dt), T);
      continue;
    }
    GemmArgs g;
    g.M = N; g.N = N; g.K = N; g.nb1 = T - k;
    g.A = rowmajor(G.retptr(T, T - l), N);
    g.B = rowmajor(S.retptr(T - l, T - (k + 1)), N); g.B.bs1 = -es;
    g.C = rowmajor(Q + (i64)(k + 1) * es, N); g.C.bs1 = es;
    g.bscale = c.gregT + (i64)l * ld + (k + 1);
    g.beta = make_double2(1.0, 0.0);
    gemm(g, c.stream);
  }
  const int smem = N * sizeof(double2);
  for (int n = k + 1; n <= T; n++) {
    if (fused) {
      step_block(c, STEP_RET, N, T, n, G, Q, nullptr, err);
      if (n < T)
        push_blocks(c, PUSH_RET, N, T, n, n + 1, T - n, G, S, nullptr, Q, c.gregT + (i64)n * ld + (n + 1), 1, 1.0,
                    1.0 / (dt * dt), T);
      continue;
    }
    ret_step_kernel<<<N, std::min(N, 256), smem, c.stream>>>(N, k, T, n, G, Q, c.Minv, c.d_bd, dt, err);
    NEDY_CHECK_LAUNCH();
    if (n < T) {  // push G^R(T,T-n) into Q_m, m = n+1..T
      GemmArgs g;
      g.M = N; g.N = N; g.K = N; g.nb1 = T - n;
      g.A = rowmajor(G.retptr(T, T - n), N);
      g.B = rowmajor(S.retptr(T - n, T - n - 1), N); g.B.bs1 = -es;
      g.C = rowmajor(Q + (i64)(n + 1) * es, N); g.C.bs1 = es;
      g.bscale = c.gregT + (i64)n * ld + (n + 1);
      g.beta = make_double2(1.0, 0.0);
      gemm(g, c.stream);
    }
  }
  return sum_dev(c, err, T + 1, true);
}

static double dyson_tv(Ctx &c, int T, DevGF &G, const DevGF &S, const double2 *hmf, double mu) {
  const int N = G.nao, np = G.ntau + 1, ld = c.nt + 1;
  const i64 es = (i64)N * N, row = (i64)np * es;
  double2 *old = c.ws.alloc<double2>(row);
  double2 *ctv = c.ws.alloc<double2>(row);
  NEDY_CUDA(cudaMemcpyAsync(old, G.tvptr(T, 0), sizeof(double2) * row, cudaMemcpyDeviceToDevice, c.stream));
  // mixing: int_0^beta Sig^tv(T,tau') G^M(tau' - tau_m)
  mixing_gemm(c, N, np, S.tvptr(T, 0), c.mixK, ctv, false, czero());
  // CTV1: sum_{j<T} dt w(T,j) Sig^R(T,j) G^tv(j, .)   (the j = T term multiplies G^tv(T,.) = 0),
  // computed transposed, ctv^T ((m,q) x i) = G^tv^T ((m,q) x (j,c)) Sig^R^T ((j,c) x i), so that
  // the long dimension (np N) is the GEMM's M: 128-row tiles instead of 64-wide column tiles
  if (T > 0) {
    GemmArgs g;
    g.M = (int)(np * N); g.N = N; g.K = T * N;
    g.A.p = G.tvptr(0, 0); g.A.rdiv = N; g.A.rs_hi = es; g.A.rs_lo = 1; g.A.cdiv = N; g.A.cs_hi = row; g.A.cs_lo = N;
    g.B.p = S.retptr(T, 0); g.B.rdiv = N; g.B.rs_hi = es; g.B.rs_lo = 1; g.B.cs_lo = N;
    g.C.p = ctv; g.C.rdiv = N; g.C.rs_hi = es; g.C.rs_lo = 1; g.C.cs_lo = N;
    g.kscale = c.greg + (i64)T * ld; g.kdiv = N;
    g.alpha = make_double2(c.dt, 0.0);
    g.beta = make_double2(1.0, 0.0);
    gemm(g, c.stream);
  }
  tv_bd_kernel<<<nblk(row), TPB, 0, c.stream>>>(row, c.k, T, G, c.d_bd, c.dt, ctv);
  NEDY_CHECK_LAUNCH();
  // M(T) and its inverse
  update_minv(c, S, hmf, mu, T, T);
  {  // G^tv(T, m) = Minv(T) ctv_m
    GemmArgs g;
    g.M = N; g.N = (int)(np * N); g.K = N;
    g.A = rowmajor(c.Minv + (i64)T * es, N);
    g.B.p = ctv; g.B.rs_lo = N; g.B.cdiv = N; g.B.cs_hi = es; g.B.cs_lo = 1;
    g.C.p = G.tvptr(T, 0); g.C.rs_lo = N; g.C.cdiv = N; g.C.cs_hi = es; g.C.cs_lo = 1;
    gemm(g, c.stream);
  }
  double *err = c.ws.alloc<double>(np);
  NEDY_CUDA(cudaMemsetAsync(err, 0, sizeof(double) * np, c.stream));
  diffnorm_kernel<<<nblk(row), TPB, 0, c.stream>>>(N, np, old, G.tvptr(T, 0), err);
  NEDY_CHECK_LAUNCH();
  return sum_dev(c, err, np, true);
}

static double dyson_les(Ctx &c, int n, DevGF &G, const DevGF &S, const double2 *hmf, double mu) {
  const int N = G.nao, k = c.k, kn = k * N, np = G.ntau + 1, ld = c.nt + 1;
  const i64 es = (i64)N * N;
  const double dt = c.dt;
  double *err = c.ws.alloc<double>(n + 2);
  NEDY_CUDA(cudaMemsetAsync(err, 0, sizeof(double) * (n + 2), c.stream));
  double2 *X = c.ws.alloc<double2>((i64)(n + 1) * es);
  double2 *Q = c.ws.alloc<double2>((i64)(n + 1) * es);
  NEDY_CUDA(cudaMemsetAsync(X, 0, sizeof(double2) * (n + 1) * es, c.stream));
  NEDY_CUDA(cudaMemsetAsync(Q, 0, sizeof(double2) * (n + 1) * es, c.stream));
  les_init_kernel<<<nblk(es), TPB, 0, c.stream>>>(N, n, G, X, err + n + 1);
  NEDY_CHECK_LAUNCH();
  // Cles3: Q_p += int Sig^tv(p,tau) [sig i G^tv(n,beta-tau)^+] dtau   (p = 0..n)
  {
    double2 *ntt = c.ws.alloc<double2>((i64)np * es);
    double2 *Bw = c.ws.alloc<double2>((i64)np * es);
    ntt_kernel<<<nblk(es * np), TPB, 0, c.stream>>>(N, G.ntau, n, G, G.sig, ntt);
    NEDY_CHECK_LAUNCH();
    lesser_weights_kernel<<<nblk(es), TPB, 0, c.stream>>>(N, G.ntau, ntt, c.d_w, c.d_u, c.col.ctop, c.beta, Bw);
    NEDY_CHECK_LAUNCH();
    GemmArgs g;
    g.M = (n + 1) * N; g.N = N; g.K = np * N;
    g.A.p = S.tvptr(0, 0); g.A.rdiv = N; g.A.rs_hi = (i64)np * es; g.A.rs_lo = N;
    g.A.cdiv = N; g.A.cs_hi = es; g.A.cs_lo = 1;
    g.B = rowmajor(Bw, N);
    g.C = rowmajor(Q, N);
    g.beta = make_double2(1.0, 0.0);
    gemm(g, c.stream);
  }
  // Cles2 with X_j = dt w(n,j) G^R(n,j)^+
  {
    double2 *Xc = c.ws.alloc<double2>((i64)(n + 1) * es);
    cles2_x_kernel<<<nblk(es * (n + 1)), TPB, 0, c.stream>>>(N, n, G, c.greg + (i64)n * ld, dt, Xc);
    NEDY_CHECK_LAUNCH();
    std::vector<i64> offA(n + 1), offC(n + 1), offB(n + 1);
    std::vector<int> Mv(n + 1), Kv(n + 1);
    for (int p = 0; p <= n; p++) {
      offA[p] = les_idx(0, p) * es;
      offC[p] = (i64)p * es;
      offB[p] = (i64)p * es;
      Mv[p] = (p + 1) * N;
      Kv[p] = p * N;
    }
    // part 1 in groups (p, chunk of at most PC blocks j): the groups' K no longer grows with p,
    // so the longest CTA does PC blocks instead of n (the chunks of one p accumulate atomically)
    constexpr int PC = 8;
    std::vector<i64> cA, cB, cC;
    std::vector<int> cK;
    for (int p = 1; p <= n; p++)
      for (int j0 = 0; j0 < p; j0 += PC) {
        cA.push_back(offA[p] + (i64)j0 * es);
        cB.push_back((i64)j0 * es);
        cC.push_back((i64)p * es);
        cK.push_back(std::min(PC, p - j0) * N);
      }
    const int ng = (int)cK.size();
    i64 *dOffA = c.ws.alloc<i64>(n + 1), *dOffB = c.ws.alloc<i64>(n + 1);
    int *dM = c.ws.alloc<int>(n + 1);
    i64 *dcA = c.ws.alloc<i64>(ng), *dcB = c.ws.alloc<i64>(ng), *dcC = c.ws.alloc<i64>(ng);
    int *dcK = c.ws.alloc<int>(ng);
    NEDY_CUDA(cudaMemcpyAsync(dOffA, offA.data(), sizeof(i64) * (n + 1), cudaMemcpyHostToDevice, c.stream));
    NEDY_CUDA(cudaMemcpyAsync(dOffB, offB.data(), sizeof(i64) * (n + 1), cudaMemcpyHostToDevice, c.stream));
    NEDY_CUDA(cudaMemcpyAsync(dM, Mv.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, c.stream));
    NEDY_CUDA(cudaMemcpyAsync(dcA, cA.data(), sizeof(i64) * ng, cudaMemcpyHostToDevice, c.stream));
    NEDY_CUDA(cudaMemcpyAsync(dcB, cB.data(), sizeof(i64) * ng, cudaMemcpyHostToDevice, c.stream));
    NEDY_CUDA(cudaMemcpyAsync(dcC, cC.data(), sizeof(i64) * ng, cudaMemcpyHostToDevice, c.stream));
    NEDY_CUDA(cudaMemcpyAsync(dcK, cK.data(), sizeof(int) * ng, cudaMemcpyHostToDevice, c.stream));
    if (ng > 0) {  // part 1: Q_p -= sum_{j<p} Sig^<(j,p)^+ X_j
      GemmArgs g;
      g.M = N; g.N = N; g.K = PC * N; g.nb1 = ng;
      g.A.p = S.les; g.A.rs_lo = 1; g.A.cdiv = N; g.A.cs_hi = es; g.A.cs_lo = N;
      g.conjA = true;
      g.B = rowmajor(Xc, N);
      g.C = rowmajor(Q, N);
      g.goffA = dcA; g.goffB = dcB; g.goffC = dcC; g.gK = dcK;
      g.alpha = make_double2(-1.0, 0.0);
      g.atomic = true;
      gemm(g, c.stream);
    }
    {  // part 2: Q_p += sum_{j>=p} Sig^<(p,j) X_j        (group j: rows (p,a), p <= j)
      GemmArgs g;
      g.M = (n + 1) * N; g.N = N; g.K = N; g.nb1 = n + 1;
      g.A = rowmajor(S.les, N);
      g.B = rowmajor(Xc, N);
      g.C = rowmajor(Q, N);
      g.goffA = dOffA; g.goffB = dOffB; g.gM = dM;
      g.atomic = true;
      gemm(g, c.stream);
    }
  }
  // start block m = 1..k
  {
    double2 *M = c.ws.alloc<double2>((i64)kn * kn);
    double2 *Qs = c.ws.alloc<double2>((i64)kn * N);
    les_start_kernel<<<nblk((i64)kn * kn + (i64)kn * N), TPB, 0, c.stream>>>(N, k, n, G, S, hmf, c.d_pdiff, c.greg,
                                                                              ld, mu, dt, Q, M, Qs);
    NEDY_CHECK_LAUNCH();
    gj(c, kn, N, 1, M, 0, Qs, 0);
    NEDY_CUDA(cudaMemcpyAsync(X + es, Qs, sizeof(double2) * kn * N, cudaMemcpyDeviceToDevice, c.stream));
  }
  // sequential m = k+1 .. n-1, then the diagonal.  Q_m += sum_{l<m} dt w(m,l) Sig^R(m,l) X_l:
  // for nao <= 64 each X_l is pushed into Q_{l+1..n} once it is known (the start block's
  // X_0..X_k into Q_{k+1..n} first), one block product per target and no atomics
  if (N <= 64) {
    // the derivative terms -i bd(m-l)/dt X_l go into Q_m with the pushes (targets m < n: the
    // diagonal takes its own, dyson_step.h:303-306), and the step is the product Minv(m) Q_m
    for (int l = 0; l <= k; l++)
      push_blocks(c, PUSH_LES, N, 0, l, k + 1, n - k, G, S, X, Q, c.greg + (i64)(k + 1) * ld + l, ld, dt, 1.0 / dt,
                  n - 1);
    for (int m = k + 1; m < n; m++) {
      step_block(c, STEP_LES, N, 0, m, G, Q, X, nullptr);
      push_blocks(c, PUSH_LES, N, 0, m, m + 1, n - m, G, S, X, Q, c.greg + (i64)(m + 1) * ld + m, ld, dt, 1.0 / dt,
                  n - 1);
    }
  } else {
    // blocks per split-K chunk of the pull sums: one block per CTA, so the sequential
    // step m runs m CTAs (each 64x64x64 at nao=64) instead of m/8 long ones
    const int LC = 1;
    for (int m = k + 1; m <= n; m++) {
      // Q_m += sum_{l<m} dt w(m,l) Sig^R(m,l) X_l   (split-K over l in chunks of LC blocks, atomics)
      for (int part = 0; part < 2; part++) {
        const int nfull = m / LC, rem = m - nfull * LC;
        const int nb = part == 0 ? nfull : (rem > 0 ? 1 : 0);
        if (nb == 0) continue;
        const int l0 = part == 0 ? 0 : nfull * LC;
        GemmArgs g;
        g.M = N; g.N = N; g.K = (part == 0 ? LC : rem) * N; g.nb1 = nb;
        g.A.p = S.retptr(m, l0); g.A.rs_lo = N; g.A.cdiv = N; g.A.cs_hi = es; g.A.cs_lo = 1; g.A.bs1 = LC * es;
        g.B = rowmajor(X + (i64)l0 * es, N); g.B.bs1 = LC * es;
        g.C = rowmajor(Q + (i64)m * es, N);
        g.kscale = c.greg + (i64)m * ld + l0; g.kdiv = N; g.kscale_bs1 = LC;
        g.alpha = make_double2(dt, 0.0);
        g.atomic = true;
        gemm(g, c.stream);
      }
      if (m < n) {
        les_step_kernel<<<N, std::min(N, 256), N * sizeof(double2), c.stream>>>(N, k, m, Q, X, c.Minv, c.d_bd, dt);
        NEDY_CHECK_LAUNCH();
      }
    }
  }
  {
    const double wnn = c.W.gregory(n, n);
    static std::atomic<bool> attr_set[64];  // per device (host threads may race here)
    int dev = 0;
    NEDY_CUDA(cudaGetDevice(&dev));
    NEDY_REQUIRE(dev < 64, "device index out of range");
    if (!attr_set[dev].load()) {
      NEDY_CUDA(cudaFuncSetAttribute(les_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
      attr_set[dev].store(true);
    }
    NEDY_REQUIRE(2 * es * (i64)sizeof(double2) <= 200 * 1024, "dyson_step: nao too large for the diagonal kernel");
    les_diag_kernel<<<1, 256, 2 * es * sizeof(double2), c.stream>>>(N, k, n, G, S, hmf, c.d_ex, c.d_bd, wnn, mu, dt,
                                                                   Q, X);
    NEDY_CHECK_LAUNCH();
  }
  diffnorm_kernel<<<nblk((i64)(n + 1) * es), TPB, 0, c.stream>>>(N, n + 1, G.lesptr(0, n), X, err);
  NEDY_CHECK_LAUNCH();
  NEDY_CUDA(cudaMemcpyAsync(G.lesptr(1, n), X + es, sizeof(double2) * n * es, cudaMemcpyDefault, c.stream));
  return sum_dev(c, err, n + 2, true);
}

void dyson_step(Ctx &c, int n, DevGF &G, const DevGF &Sig, const double2 *hmf, double mu, double *err) {
  NEDY_REQUIRE(n > c.k && n <= G.nt, "dyson_step: need k < n <= nt");
  NEDY_REQUIRE(G.nao == Sig.nao && G.ntau == Sig.ntau && G.nt == Sig.nt && G.sig == Sig.sig,
               "dyson_step: G and Sigma shapes differ");
  NEDY_REQUIRE(G.nt == c.nt && G.ntau == c.ntau, "dyson_step: G does not match the context sizes");
  NEDY_REQUIRE(Sig.win == 0, "dyson_step: Sigma must hold its whole history (the integrals read every time)");
  ensure_tables(c);
  ensure_mixing_kernel(c, G);
  ensure_minv(c, G.nao);
  c.ws.reset();
  // time-local inverses for t' < n (final) -- recomputed each call, they are cheap and batched
  update_minv(c, Sig, hmf, mu, 0, n - 1);
  double e1 = dyson_ret(c, n, G, Sig, hmf, mu);
  double e2 = dyson_tv(c, n, G, Sig, hmf, mu);
  double e3 = dyson_les(c, n, G, Sig, hmf, mu);
  check_status(c);
  if (err) { err[0] = e1; err[1] = e2; err[2] = e3; }
}

// Second context of c, created on first use: the same sizes, weights and collocation, its
// own stream (ordered after c's by events), workspace, inverses and mixing kernel.
static Ctx &aux_ctx(Ctx &c) {
  if (!c.aux) {
    Ctx *a = new Ctx;
    a->device = c.device;
    a->nt = c.nt; a->ntau = c.ntau; a->nao = c.nao; a->k = c.k;
    a->beta = c.beta; a->dt = c.dt;
    a->ws_budget = c.ws_budget;
    a->W = c.W;
    a->col = c.col;
    const cudaError_t e = cudaStreamCreate(&a->stream);
    if (e != cudaSuccess) {
      delete a;
      NEDY_CUDA(e);
    }
    a->ws.set_stream(a->stream);
    c.aux = a;
  }
  return *c.aux;
}

// A mixing kernel that `from` holds for G's G^M moves to `to` (no second 16 ntau^2 nao^2
// bytes for the same kernel).  Work already queued on from's stream that reads it comes
// before to's stream by the event order of the caller.
static void hand_over_mixing_kernel(Ctx &from, Ctx &to, const DevGF &G) {
  const int N = G.nao;
  if (to.mixK && to.mixK_src == G.mat && to.mixK_ver == G.mat_version && to.mixK_nao == N) return;
  double2 **p = nullptr;
  const double2 **src = nullptr;
  unsigned long long *ver = nullptr;
  int *nao = nullptr;
  if (from.mixK && from.mixK_src == G.mat && from.mixK_ver == G.mat_version && from.mixK_nao == N) {
    p = &from.mixK; src = &from.mixK_src; ver = &from.mixK_ver; nao = &from.mixK_nao;
  } else if (from.mixK_alt && from.mixK_alt_src == G.mat && from.mixK_alt_ver == G.mat_version &&
             from.mixK_alt_nao == N) {
    p = &from.mixK_alt; src = &from.mixK_alt_src; ver = &from.mixK_alt_ver; nao = &from.mixK_alt_nao;
  }
  if (!p) return;
  if (to.mixK) NEDY_CUDA(cudaFree(to.mixK));
  to.mixK = *p; to.mixK_src = *src; to.mixK_ver = *ver; to.mixK_nao = *nao;
  *p = nullptr; *src = nullptr; *ver = ~0ULL; *nao = 0;
}

void dyson_step_spins(Ctx &c, int n, DevGF &G0, const DevGF &S0, const double2 *h0, double mu0, double *e0,
                      DevGF &G1, const DevGF &S1, const double2 *h1, double mu1, double *e1) {
  // The two steps are independent; each is a chain of small dependent kernels (sequential
  // sweeps, the pivot steps of the start blocks) with host round trips, which leaves most
  // of the GPU idle, so they run side by side.
  Ctx &a = aux_ctx(c);
  hand_over_mixing_kernel(c, a, G1);
  cudaEvent_t ev[2] = {nullptr, nullptr};
  NEDY_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
  const cudaError_t ce = cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
  if (ce != cudaSuccess) {
    cudaEventDestroy(ev[0]);
    NEDY_CUDA(ce);
  }
  std::exception_ptr ex0, ex1;
  try {
    NEDY_CUDA(cudaEventRecord(ev[0], c.stream));  // a's stream after everything queued on c's
    NEDY_CUDA(cudaStreamWaitEvent(a.stream, ev[0], 0));
    std::thread th([&] {
      try {
        NEDY_CUDA(cudaSetDevice(a.device));
        dyson_step(a, n, G1, S1, h1, mu1, e1);
      } catch (...) {
        ex1 = std::current_exception();
      }
    });
    try {
      dyson_step(c, n, G0, S0, h0, mu0, e0);
    } catch (...) {
      ex0 = std::current_exception();
    }
    th.join();
    NEDY_CUDA(cudaEventRecord(ev[1], a.stream));  // c's stream continues after spin 1's step
    NEDY_CUDA(cudaStreamWaitEvent(c.stream, ev[1], 0));
  } catch (...) {
    if (!ex0) ex0 = std::current_exception();
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (ex0) std::rethrow_exception(ex0);
  if (ex1) std::rethrow_exception(ex1);
}

} // namespace nedy
