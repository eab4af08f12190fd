// Batched FP64 / complex128 GEMM on DMMA (mma.sync.aligned.m8n8k4 .f64).  See gemm_f64.cuh.
//
// CTA tile BM x 64 x 16 (BM = 128 with 8 warps, or 64 with 4 warps for short M),
// each warp owning a 32 x 32 tile = 4 x 4 DMMA fragments.  Operands are copied to
// shared memory with cp.async in a three-stage pipeline, complex values kept
// interleaved (one 16-byte copy per element, one 16-byte shared load per fragment
// element); a complex product is four real DMMAs (re*re - im*im, re*im + im*re).
// Row offsets of the A tile are computed once per CTA; the two-level index split of
// the views costs one division per element per k-tile only for the split dimension.
#include "gemm_f64.cuh"
#include <cmath>

namespace nedy {
namespace {

constexpr int BN = 64, BK = 16, STAGES = 3;

struct DView {
  const char *p;
  i64 rs_hi, rs_lo, cs_hi, cs_lo, bs1, bs2;
  int rdiv, cdiv;
};

struct Params {
  int M, N, K, nb1, nb2;
  DView A, B, C;
  int conjA, conjB;
  double2 alpha, beta;
  const double *kscale;
  int kdiv;
  i64 kscale_bs1;
  const i64 *goffA, *goffB, *goffC;
  const int *gM, *gK;
  const double *bscale;
  int atomic;
  int ksplit, kchunk;  // split-K: z index = batch * ksplit + split, each split covers kchunk of K
  int a_kcontig, b_ncontig;
};

__device__ __forceinline__ i64 off2(int idx, int div, i64 hi, i64 lo) {
  if (div == 0) return (i64)idx * lo;
  int q = idx / div;
  return (i64)q * hi + (i64)(idx - q * div) * lo;
}

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <int BYTES>
__device__ __forceinline__ void cp_async(void *dst, const void *src, bool valid) {
  unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  int n = valid ? BYTES : 0;
  if (BYTES == 16)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(src), "r"(n));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(src), "r"(n));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// shared-memory geometry (units: elements of the operand type)
template <bool C>
struct Lay {
  // complex: 16-byte elements, stride = 2 (mod 8) -> conflict-free quarter-warp fragment reads
  // real:     8-byte elements, stride = 4 (mod 16) -> conflict-free half-warp fragment reads
  static constexpr int pad = C ? 2 : 4;
  static constexpr int esz = C ? 16 : 8;
};

template <int BM, bool AC, bool BC>
struct Smem {
  static constexpr int LDA = BM + Lay<AC>::pad;
  static constexpr int LDB = BN + Lay<BC>::pad;
  static constexpr int ABYTES = BK * LDA * Lay<AC>::esz;
  static constexpr int BBYTES = BK * LDB * Lay<BC>::esz;
  static constexpr int STAGE = ABYTES + BBYTES;
  static constexpr int TOTAL = STAGES * STAGE;
};

template <int BM, bool AC, bool BC>
__global__ void __launch_bounds__(BM * 2, (BM == 128 ? 1 : 2)) gemm_kernel(const Params P) {
  using SM = Smem<BM, AC, BC>;
  constexpr int NT = BM * 2;            // threads: (BM/32) x 2 warps
  constexpr int A_PER = BM * BK / NT;   // = 8
  constexpr int B_PER = BK * BN / NT;   // 8 (BM=64) or 4 (BM=128)
  extern __shared__ __align__(16) char smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int nb = P.nb1 * P.nb2 * P.ksplit;
  const double sA = P.conjA ? -1.0 : 1.0, sB = P.conjB ? -1.0 : 1.0;
  const int esA = AC ? 16 : 8, esB = BC ? 16 : 8;

  for (int bzs = blockIdx.z; bzs < nb; bzs += gridDim.z) {
    const int bz = bzs / P.ksplit, ks = bzs - bz * P.ksplit;
    const int b1 = bz / P.nb2, b2 = bz - b1 * P.nb2;
    const int Mg = P.gM ? P.gM[b1] : P.M;
    const int Kfull = P.gK ? P.gK[b1] : P.K;
    if (m0 >= Mg) continue;
    // this split covers k in [kb, kb + Kg) of the full K range
    const int kb = ks * P.kchunk;
    const int Kg = max(0, min(Kfull - kb, P.kchunk));
    if (Kg == 0 && P.ksplit > 1) continue;
    const int ntiles = (Kg + BK - 1) / BK;
    const i64 oA = b1 * P.A.bs1 + b2 * P.A.bs2 + (P.goffA ? P.goffA[b1] : 0);
    const i64 oB = b1 * P.B.bs1 + b2 * P.B.bs2 + (P.goffB ? P.goffB[b1] : 0);
    const char *Ab = P.A.p + oA * esA;
    const char *Bb = P.B.p + oB * esB;
    const double *ksc = P.kscale ? P.kscale + b1 * P.kscale_bs1 : nullptr;

    // fixed per-thread load coordinates; row (A) / column (B) offsets precomputed
    const int akc = P.a_kcontig, bnc = P.b_ncontig;
    auto a_m = [&](int i) { return akc ? (tid / BK) + (NT / BK) * i : tid % BM; };
    auto a_k = [&](int i) { return akc ? (tid & (BK - 1)) : (tid / BM) + (NT / BM) * i; };
    auto b_n = [&](int i) { return bnc ? tid % BN : (tid / BK) + (NT / BK) * i; };
    auto b_k = [&](int i) { return bnc ? (tid / BN) + (NT / BN) * i : (tid & (BK - 1)); };
    i64 aro[A_PER], bco[B_PER];
#pragma unroll
    for (int i = 0; i < A_PER; i++) {
      const int gm = m0 + a_m(i);
      aro[i] = gm < Mg ? off2(gm, P.A.rdiv, P.A.rs_hi, P.A.rs_lo) : -1;
    }
#pragma unroll
    for (int i = 0; i < B_PER; i++) {
      const int gn = n0 + b_n(i);
      bco[i] = gn < P.N ? off2(gn, P.B.cdiv, P.B.cs_hi, P.B.cs_lo) : -1;
    }

    auto load = [&](int t, int stage) {
      char *st = smem + stage * SM::STAGE;
      char *As = st, *Bs = st + SM::ABYTES;
      const int k0 = t * BK;
      const int kg0 = kb + k0;  // absolute k of this tile
#pragma unroll
      for (int i = 0; i < A_PER; i++) {
        const int kk = a_k(i), gk = k0 + kk;
        const bool v = aro[i] >= 0 && gk < Kg;
        const char *src = v ? Ab + (aro[i] + off2(kg0 + kk, P.A.cdiv, P.A.cs_hi, P.A.cs_lo)) * esA : Ab;
        cp_async<AC ? 16 : 8>(As + (kk * SM::LDA + a_m(i)) * esA, src, v);
      }
#pragma unroll
      for (int i = 0; i < B_PER; i++) {
        const int kk = b_k(i), gk = k0 + kk;
        const bool v = bco[i] >= 0 && gk < Kg;
        const char *src = v ? Bb + (off2(kg0 + kk, P.B.rdiv, P.B.rs_hi, P.B.rs_lo) + bco[i]) * esB : Bb;
        cp_async<BC ? 16 : 8>(Bs + (kk * SM::LDB + b_n(i)) * esB, src, v);
      }
    };

    double acc_re[4][4][2], acc_im[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) {
        acc_re[i][j][0] = acc_re[i][j][1] = 0.0;
        acc_im[i][j][0] = acc_im[i][j][1] = 0.0;
      }

#pragma unroll
    for (int s = 0; s < STAGES - 1; s++) {
      if (s < ntiles) load(s, s);
      cp_commit();
    }
    for (int t = 0; t < ntiles; t++) {
      cp_wait<STAGES - 2>();
      __syncthreads();
      // prefetch tile t + STAGES - 1 into the stage freed at iteration t - 1
      {
        const int tn = t + STAGES - 1;
        if (tn < ntiles) load(tn, tn % STAGES);
        cp_commit();
      }
      const char *st = smem + (t % STAGES) * SM::STAGE;
      const char *As = st, *Bs = st + SM::ABYTES;
#pragma unroll
      for (int kk = 0; kk < BK / 4; kk++) {
        const int kr = kk * 4 + (lane & 3);
        double ksv = 1.0;
        if (ksc) {
          const int gk = t * BK + kr;
          ksv = gk < Kg ? ksc[(kb + gk) / P.kdiv] : 0.0;
        }
        double ar[4], ai[4], br[4], bi[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const int mm = wm * 32 + i * 8 + (lane >> 2);
          if (AC) {
            const double2 v = ((const double2 *)As)[kr * SM::LDA + mm];
            ar[i] = v.x * ksv;
            ai[i] = v.y * ksv * sA;
          } else {
            ar[i] = ((const double *)As)[kr * SM::LDA + mm] * ksv;
            ai[i] = 0.0;
          }
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int nn = wn * 32 + j * 8 + (lane >> 2);
          if (BC) {
            const double2 v = ((const double2 *)Bs)[kr * SM::LDB + nn];
            br[j] = v.x;
            bi[j] = v.y * sB;
          } else {
            br[j] = ((const double *)Bs)[kr * SM::LDB + nn];
            bi[j] = 0.0;
          }
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const double nai = -ai[i];
#pragma unroll
          for (int j = 0; j < 4; j++) {
            dmma(acc_re[i][j][0], acc_re[i][j][1], ar[i], br[j]);
            if (AC && BC) dmma(acc_re[i][j][0], acc_re[i][j][1], nai, bi[j]);
            if (BC) dmma(acc_im[i][j][0], acc_im[i][j][1], ar[i], bi[j]);
            if (AC) dmma(acc_im[i][j][0], acc_im[i][j][1], ai[i], br[j]);
          }
        }
      }
    }
    cp_wait<0>();
    __syncthreads();

    // epilogue: C = alpha * acc + beta * C   (or C += alpha * acc with atomics)
    double2 *Cb = (double2 *)(P.C.p) + (b1 * P.C.bs1 + b2 * P.C.bs2 + (P.goffC ? P.goffC[b1] : 0));
    const bool useb = (P.beta.x != 0.0 || P.beta.y != 0.0);
    const double2 alpha = P.bscale ? cscale(P.alpha, P.bscale[b1]) : P.alpha;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int row = m0 + wm * 32 + i * 8 + (lane >> 2);
      if (row >= Mg) continue;
      const i64 ro = off2(row, P.C.rdiv, P.C.rs_hi, P.C.rs_lo);
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
        for (int c = 0; c < 2; c++) {
          const int col = n0 + wn * 32 + j * 8 + (lane & 3) * 2 + c;
          if (col >= P.N) continue;
          double2 *dst = Cb + ro + off2(col, P.C.cdiv, P.C.cs_hi, P.C.cs_lo);
          double2 v = make_double2(acc_re[i][j][c], acc_im[i][j][c]);
          double2 o = cmul(alpha, v);
          if (P.atomic || P.ksplit > 1) {
            atomicAdd(&dst->x, o.x);
            atomicAdd(&dst->y, o.y);
          } else {
            if (useb) o = cadd(o, cmul(P.beta, *dst));
            *dst = o;
          }
        }
    }
  }
}

// C(view) = beta * C  (prologue of a split-K launch, whose splits accumulate with atomics)
__global__ void scale_c_kernel(int M, int N, int nb1, int nb2, DView C, const i64 *goffC, const int *gM, double2 beta) {
  const i64 tot = (i64)M * N * nb1 * nb2;
  for (i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x; idx < tot; idx += (i64)gridDim.x * blockDim.x) {
    const i64 b = idx / ((i64)M * N);
    const int e = (int)(idx - b * M * N);
    const int r = e / N, c = e - (e / N) * N;
    const int b1 = (int)(b / nb2), b2 = (int)(b - (i64)b1 * nb2);
    if (gM && r >= gM[b1]) continue;
    double2 *dst = (double2 *)C.p + b1 * C.bs1 + b2 * C.bs2 + (goffC ? goffC[b1] : 0) +
                   off2(r, C.rdiv, C.rs_hi, C.rs_lo) + off2(c, C.cdiv, C.cs_hi, C.cs_lo);
    *dst = (beta.x == 0.0 && beta.y == 0.0) ? make_double2(0.0, 0.0) : cmul(beta, *dst);
  }
}

DView dv(const View &v) {
  DView d;
  d.p = (const char *)v.p;
  d.rs_hi = v.rs_hi; d.rs_lo = v.rs_lo; d.rdiv = v.rdiv;
  d.cs_hi = v.cs_hi; d.cs_lo = v.cs_lo; d.cdiv = v.cdiv;
  d.bs1 = v.bs1; d.bs2 = v.bs2;
  return d;
}

template <int BM, bool AC, bool BC>
void launch(const Params &P, cudaStream_t s) {
  using SM = Smem<BM, AC, BC>;
  static std::atomic<bool> attr[64];  // per device: shared-memory attribute set (host threads may race here)
  int dev = 0;
  NEDY_CUDA(cudaGetDevice(&dev));
  NEDY_REQUIRE(dev < 64, "device index out of range");
  if (!attr[dev].load()) {
    NEDY_CUDA(cudaFuncSetAttribute(gemm_kernel<BM, AC, BC>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM::TOTAL));
    attr[dev].store(true);
  }
  int nb = P.nb1 * P.nb2 * P.ksplit;
  dim3 grid(cdiv(P.N, BN), cdiv(P.M, BM), (unsigned)(nb < 65535 ? nb : 65535));
  NEDY_REQUIRE(grid.y <= 65535, "gemm: M too large");
  gemm_kernel<BM, AC, BC><<<grid, BM * 2, SM::TOTAL, s>>>(P);
  NEDY_CHECK_LAUNCH();
}

template <bool AC, bool BC>
void launch_bm(const Params &P, cudaStream_t s) {
  if (P.M >= 128) launch<128, AC, BC>(P, s);
  else launch<64, AC, BC>(P, s);
}

} // namespace

void gemm(const GemmArgs &g, cudaStream_t stream) {
  if (g.M <= 0 || g.N <= 0 || g.nb1 <= 0 || g.nb2 <= 0) return;
  NEDY_REQUIRE(g.K >= 0, "gemm: negative K");
  NEDY_REQUIRE(g.C.p != nullptr, "gemm: null C");
  Params P;
  P.M = g.M; P.N = g.N; P.K = g.K; P.nb1 = g.nb1; P.nb2 = g.nb2;
  P.A = dv(g.A); P.B = dv(g.B); P.C = dv(g.C);
  P.conjA = g.conjA; P.conjB = g.conjB;
  P.alpha = g.alpha; P.beta = g.beta;
  P.kscale = g.kscale; P.kdiv = g.kdiv > 0 ? g.kdiv : 1; P.kscale_bs1 = g.kscale_bs1;
  P.goffA = g.goffA; P.goffB = g.goffB; P.goffC = g.goffC;
  P.gM = g.gM; P.gK = g.gK; P.bscale = g.bscale; P.atomic = g.atomic ? 1 : 0;
  NEDY_REQUIRE(!g.atomic || (g.beta.x == 0.0 && g.beta.y == 0.0), "gemm: atomic epilogue needs beta = 0");
  // loader mapping: walk consecutive threads along the unit-stride direction
  P.a_kcontig = (g.A.cs_lo == 1) ? 1 : 0;
  P.b_ncontig = (g.B.cs_lo == 1) ? 1 : 0;
  // split-K when the output grid is too small to fill the GPU and K is long
  P.ksplit = 1;
  P.kchunk = g.K;
  {
    // resident CTAs: two per SM with 64-row tiles, one with 128-row tiles (148 SMs).  The split
    // fills the device once (at least 256 of K per split); a somewhat larger one is taken when
    // its last wave is clearly fuller (wave quantisation).
    const int bm = g.M >= 128 ? 128 : 64;
    const i64 ctas = (i64)cdiv(g.N, BN) * cdiv(g.M, bm) * g.nb1 * g.nb2;
    const i64 slots = (bm == 128 ? 1 : 2) * 148;
    if (!g.gK && ctas < slots && g.K >= 1024) {
      const int kmax = (int)(g.K / 256);
      auto eff = [&](int s) {
        const double w = (double)(ctas * s) / (double)slots;
        return w / std::ceil(w);
      };
      int ks = (int)std::min<i64>((slots + ctas - 1) / ctas, kmax);
      for (int s2 = ks + 1, s_hi = std::min(kmax, 2 * ks + 8); s2 <= s_hi; s2++)
        if (eff(s2) > eff(ks) + 0.03) ks = s2;
      if (ks > 1) {
        int kc = (g.K + ks - 1) / ks;
        kc = ((kc + BK - 1) / BK) * BK;
        ks = (g.K + kc - 1) / kc;
        P.ksplit = ks;
        P.kchunk = kc;
      }
    }
  }
  if (P.ksplit > 1 && !g.atomic) {
    const i64 tot = (i64)g.M * g.N * g.nb1 * g.nb2;
    scale_c_kernel<<<(unsigned)std::min<i64>((tot + 255) / 256, 65535LL * 8), 256, 0, stream>>>(
        g.M, g.N, g.nb1, g.nb2, P.C, P.goffC, P.gM, g.beta);
    NEDY_CHECK_LAUNCH();
  }
  if (g.a_cplx && g.b_cplx) launch_bm<true, true>(P, stream);
  else if (g.a_cplx) launch_bm<true, false>(P, stream);
  else if (g.b_cplx) launch_bm<false, true>(P, stream);
  else launch_bm<false, false>(P, stream);
}

} // namespace nedy
