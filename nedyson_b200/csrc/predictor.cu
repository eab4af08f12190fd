// Learned next-step predictor: a correction to the polynomial extrapolation of
// dyson::Extrapolate (reference src/dyson.cpp:47-117) for the new row T.
//
// Every element of the new row is the next value z_0 of a time series z_1..z_9
// (z_l its value l steps back): G^tv(T-l, tau) for the mixed row, G^R(T-l, c-l) along
// the diagonals of the retarded row and G^<(r-l, T-l) along those of the lesser
// column (elements with fewer than 9 history points keep the plain prediction).  The
// k = 5 extrapolation p = sum_j w_j z_{j+1} misses z_0 by a sixth difference; the
// network sees the three previous sixth differences a = D6 z_1, b = D6 z_2, c = D6 z_3
// scaled by s6 = max(|a|, |b|, |c|) (for one oscillation e^{-i w t}, z_0 - p = a^2 / b)
// and returns (z_0 - p) / s6.  Only series whose three magnitudes agree within a factor
// 4 are corrected or trained on: next to a kink of the drive (the switch-on at t = k dt)
// the sixth differences follow the binomial pattern C(5, i) of a derivative jump, whose
// outer positions (ratios 5 and 10) are left to the plain prediction.
//
// Network: 12 inputs [a/s6, b/s6, c/s6, one-hot component, log10(s6/|z_1|)/16,
// a^2/(b s6)] -> 256 tanh -> 256 tanh -> 2, BF16 operands with FP32 accumulation in the
// forward and the backward pass, FP32 master weights updated by Adam.  Training data are
// the rows the engine itself converged (collect); training runs on the GPU in these kernels.
// Inference corrects the elements whose sixth-difference scale is within a factor
// PRED_SELECT of the row's largest (the others keep the polynomial prediction).
#include "predictor.cuh"
#include "tcgen05.cuh"
#include <random>

namespace nedy {
namespace {

constexpr int TPB = 256;
constexpr double CLIP = 8.0;
constexpr int HIST = 9;

__device__ __forceinline__ float bfr(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// element idx of row T in the learned layout: [tv (ntau+1) | ret cols 9..T | les rows 9..T] x N^2
struct Series {
  int comp;                    // 0 tv, 1 ret, 2 les
  const double2 *z[HIST + 1];  // z[0]: the row value, z[1..9]: history
};

__device__ bool series_of(const DevGF &G, int T, i64 idx, Series &s) {
  const i64 es = G.es;
  const i64 blk = idx / es;
  const int e = (int)(idx - blk * es);
  const i64 ntv = G.ntau + 1;
  if (T < HIST) return false;
  if (blk < ntv) {
    s.comp = 0;
    for (int l = 0; l <= HIST; l++) s.z[l] = G.tvptr(T - l, blk) + e;
    return true;
  }
  const i64 nd = T - HIST + 1;  // diagonal entries with 9 history points: col / row 9..T
  i64 b = blk - ntv;
  if (b < nd) {
    const int col = (int)(HIST + b);
    s.comp = 1;
    for (int l = 0; l <= HIST; l++) s.z[l] = G.retptr(T - l, col - l) + e;
    return true;
  }
  b -= nd;
  if (b < nd) {
    const int row = (int)(HIST + b);
    s.comp = 2;
    for (int l = 0; l <= HIST; l++) s.z[l] = G.lesptr(row - l, T - l) + e;
    return true;
  }
  return false;
}

// features of one element; false when the sixth differences are at the rounding level
// or outside the oscillatory regime
__device__ bool features(const Series &s, const double *exw, float *x, double2 &p, double &s6) {
  double2 z[HIST + 1];
  for (int l = 1; l <= HIST; l++) z[l] = *s.z[l];
  const double C6[7] = {1, -6, 15, -20, 15, -6, 1};
  double2 d[3];
  for (int q = 0; q < 3; q++) {
    d[q] = make_double2(0, 0);
    for (int i = 0; i < 7; i++) {
      d[q].x += C6[i] * z[1 + q + i].x;
      d[q].y += C6[i] * z[1 + q + i].y;
    }
  }
  p = make_double2(0, 0);
  for (int j = 0; j < 6; j++) {
    p.x += exw[j] * z[j + 1].x;
    p.y += exw[j] * z[j + 1].y;
  }
  const double m0 = hypot(d[0].x, d[0].y), m1 = hypot(d[1].x, d[1].y), m2 = hypot(d[2].x, d[2].y);
  s6 = fmax(m0, fmax(m1, m2));
  const double lo = fmin(m0, fmin(m1, m2));
  const double ref = hypot(z[1].x, z[1].y);
  if (!(s6 > 1e-13 * ref) || !(s6 > 1e-300) || !(lo * 4.0 >= s6)) return false;
  for (int q = 0; q < 3; q++) {
    x[2 * q] = (float)(d[q].x / s6);
    x[2 * q + 1] = (float)(d[q].y / s6);
  }
  x[6] = s.comp == 0;
  x[7] = s.comp == 1;
  x[8] = s.comp == 2;
  x[9] = (float)(log10(s6 / ref) / 16.0);
  // the single-oscillation continuation a^2 / b (normalised), clipped
  const double ar = d[0].x / s6, ai = d[0].y / s6, br = d[1].x / s6, bi = d[1].y / s6;
  const double nr = ar * ar - ai * ai, ni = 2 * ar * ai, den = br * br + bi * bi;
  double qr = (nr * br + ni * bi) / den, qi = (ni * br - nr * bi) / den;
  const double qm = hypot(qr, qi);
  if (qm > CLIP) {
    qr *= CLIP / qm;
    qi *= CLIP / qm;
  }
  x[10] = (float)qr;
  x[11] = (float)qi;
  return true;
}

__device__ __forceinline__ unsigned hash32(unsigned long long v) {
  v ^= v >> 33;
  v *= 0xff51afd7ed558ccdULL;
  v ^= v >> 33;
  v *= 0xc4ceb9fe1a85ec53ULL;
  v ^= v >> 33;
  return (unsigned)v;
}

__global__ void collect_kernel(DevGF G, int T, i64 total, const double *exw, int stride, unsigned long long salt,
                               float *X, float *Y, unsigned long long *count, i64 cap) {
  for (i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x; idx < total; idx += (i64)gridDim.x * blockDim.x) {
    if (stride > 1 && hash32(salt * 1000003ULL + (unsigned long long)idx) % stride) continue;
    Series s;
    if (!series_of(G, T, idx, s)) continue;
    float x[PRED_IN];
    double2 p;
    double s6;
    if (!features(s, exw, x, p, s6)) continue;
    const double2 z0 = *s.z[0];
    const double yr = fmin(CLIP, fmax(-CLIP, (z0.x - p.x) / s6)), yi = fmin(CLIP, fmax(-CLIP, (z0.y - p.y) / s6));
    const unsigned long long slot = atomicAdd(count, 1ULL);
    if ((i64)slot >= cap) continue;
    for (int i = 0; i < PRED_IN; i++) X[slot * PRED_IN + i] = x[i];
    Y[slot * 2] = (float)yr;
    Y[slot * 2 + 1] = (float)yi;
  }
}

// Learned correction of the new row (after the polynomial extrapolation wrote p into it),
// on the 5th-generation tensor cores: one CTA of 128 threads per 128-element tile, thread t
// owns element t (TMEM lane t).  Layer 1 (K = 16: the 12 inputs, zero-padded) and layer 2
// (K = 256) are tcgen05.mma M128 N256 with BF16 operands K-major in shared memory (64-wide
// K blocks, 128-byte swizzle) and the FP32 accumulator in TMEM (256 columns, reused by
// both layers); W1 and W2 (BF16) stay in shared memory for all tiles of the CTA, h1 is
// written back into the A tile by the layer-1 epilogue.  The output layer (2 x 256) runs in
// registers in the layer-2 epilogue.  Operand rounding is that of the training forward
// (BF16 inputs, weights and hidden activations, FP32 accumulation).
// xin != nullptr: the network on given inputs (n rows of PRED_IN), raw outputs (with b3)
// to yout; else the elements sel[0 .. nsel[1]) of row T of G.
constexpr int MLP_T = 128;
constexpr int MLP_W2 = 4 * PRED_W * 128;     // 4 K blocks x 256 rows x 128 B
constexpr int MLP_W1 = PRED_W * 128;         // 1 K block x 256 rows
constexpr int MLP_H = 4 * MLP_T * 128;       // 4 K blocks x 128 rows (X in block 0 first)
constexpr int MLP_SMEM = MLP_W2 + MLP_W1 + MLP_H + 64 + 1024;

__global__ void __launch_bounds__(MLP_T, 1)
    mlp_tc_kernel(DevGF G, int T, const i64 *sel, const unsigned long long *nsel, const double *exw, const float *W,
                  double2 *corr_out, const float *xin, int nin, float *yout, int *err) {
  using namespace tc;
  extern __shared__ uint8_t mraw[];
  uint8_t *sm = (uint8_t *)(((uintptr_t)mraw + 1023) & ~(uintptr_t)1023);
  uint8_t *w2s = sm, *w1s = sm + MLP_W2, *hs = w1s + MLP_W1;
  uint64_t *bar = (uint64_t *)(hs + MLP_H);
  uint32_t *tslot = (uint32_t *)(bar + 1);
  const float *W1 = W, *b1 = W1 + PRED_W * PRED_IN, *W2 = b1 + PRED_W, *b2 = W2 + PRED_W * PRED_W;
  const float *W3 = b2 + PRED_W, *b3 = W3 + 2 * PRED_W;
  const int tid = threadIdx.x, warp = tid >> 5;
  const i64 total = xin ? (i64)nin : (i64)nsel[1];
  // weights into the K-major swizzled tiles: W2 row = output unit, K = input unit
  for (int q = tid; q < PRED_W * PRED_W / 8; q += MLP_T) {
    const int n = q / (PRED_W / 8), k0 = (q % (PRED_W / 8)) * 8;
    uint32_t w[4];
    for (int j = 0; j < 4; j++) {
      const __nv_bfloat162 h = __floats2bfloat162_rn(W2[n * PRED_W + k0 + 2 * j], W2[n * PRED_W + k0 + 2 * j + 1]);
      w[j] = *(const uint32_t *)&h;
    }
    *(uint4 *)(w2s + sw128_offset(PRED_W, n, k0)) = make_uint4(w[0], w[1], w[2], w[3]);
  }
  for (int q = tid; q < PRED_W * 2; q += MLP_T) {  // W1: K 0..15 (inputs 12..15 are zero)
    const int n = q >> 1, k0 = (q & 1) * 8;
    uint32_t w[4];
    for (int j = 0; j < 4; j++) {
      const int k = k0 + 2 * j;
      const float a = k < PRED_IN ? W1[n * PRED_IN + k] : 0.f, b = k + 1 < PRED_IN ? W1[n * PRED_IN + k + 1] : 0.f;
      const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
      w[j] = *(const uint32_t *)&h;
    }
    *(uint4 *)(w1s + sw128_offset(PRED_W, n, k0)) = make_uint4(w[0], w[1], w[2], w[3]);
  }
  if (tid == 0) {
    mbar_init(smem_u32(bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(PRED_W));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot, trow = tmem + ((uint32_t)(warp * 32) << 16);
  const uint32_t IDESC = idesc_bf16(MLP_T, PRED_W), mb = smem_u32(bar);
  uint32_t phase = 0;
  bool ok = true;
  for (i64 base = (i64)blockIdx.x * MLP_T; base < total && ok; base += (i64)gridDim.x * MLP_T) {
    // inputs of this thread's element into the A tile (K block 0, chunks 0 and 1)
    const i64 slot = base + tid;
    float x[PRED_IN] = {};
    double s6 = 0.0;
    i64 idx = -1;
    Series s;
    if (slot < total) {
      if (xin) {
        for (int i = 0; i < PRED_IN; i++) x[i] = xin[slot * PRED_IN + i];
        s6 = 1.0;
      } else {
        idx = sel[slot];
        double2 p;
        if (!(series_of(G, T, idx, s) && features(s, exw, x, p, s6))) s6 = 0.0;
      }
    }
    for (int c = 0; c < 2; c++) {
      uint32_t w[4];
      for (int j = 0; j < 4; j++) {
        const int k = c * 8 + 2 * j;
        const __nv_bfloat162 h = __floats2bfloat162_rn(k < PRED_IN ? x[k] : 0.f, k + 1 < PRED_IN ? x[k + 1] : 0.f);
        w[j] = *(const uint32_t *)&h;
      }
      *(uint4 *)(hs + sw128_offset(MLP_T, tid, c * 8)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {  // layer 1: one K = 16 step
      mma_bf16(tmem, sw128_desc(smem_u32(hs)), sw128_desc(smem_u32(w1s)), IDESC, 0u);
      mma_commit(mb);
    }
    ok = __syncthreads_and(mbar_wait_drain(mb, phase, err, 6)) != 0;  // one decision for the whole CTA
    phase ^= 1u;
    if (!ok) break;
    tc_fence_after();
    // layer-1 epilogue: h1 = bf(tanh(acc + b1)) into the A tile, K = hidden unit
    for (int c0 = 0; c0 < PRED_W; c0 += 64) {
      float v[64];
      tmem_ld64(trow + (uint32_t)c0, v);
#pragma unroll
      for (int c = 0; c < 8; c++) {
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int u = c0 + c * 8 + 2 * j;
          const __nv_bfloat162 h = __floats2bfloat162_rn(tanhf(v[c * 8 + 2 * j] + b1[u]),
                                                         tanhf(v[c * 8 + 2 * j + 1] + b1[u + 1]));
          w[j] = *(const uint32_t *)&h;
        }
        *(uint4 *)(hs + sw128_offset(MLP_T, tid, c0 + c * 8)) = make_uint4(w[0], w[1], w[2], w[3]);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {  // layer 2: 4 K blocks x 4 K = 16 steps
      for (int kb = 0; kb < 4; kb++)
#pragma unroll
        for (int kk = 0; kk < 4; kk++)
          mma_bf16(tmem, sw128_desc(smem_u32(hs + kb * MLP_T * 128 + kk * 32)),
                   sw128_desc(smem_u32(w2s + kb * PRED_W * 128 + kk * 32)), IDESC, (kb | kk) ? 1u : 0u);
      mma_commit(mb);
    }
    ok = __syncthreads_and(mbar_wait_drain(mb, phase, err, 7)) != 0;
    phase ^= 1u;
    if (!ok) break;
    tc_fence_after();
    // layer-2 epilogue and the output layer
    float y0 = 0.f, y1 = 0.f;
    for (int c0 = 0; c0 < PRED_W; c0 += 64) {
      float v[64];
      tmem_ld64(trow + (uint32_t)c0, v);
#pragma unroll
      for (int j = 0; j < 64; j++) {
        const int u = c0 + j;
        const float h2 = bfr(tanhf(v[j] + b2[u]));
        y0 = fmaf(h2, bfr(W3[u]), y0);
        y1 = fmaf(h2, bfr(W3[PRED_W + u]), y1);
      }
    }
    if (slot < total) {
      if (xin) {
        yout[slot * 2] = y0 + b3[0];
        yout[slot * 2 + 1] = y1 + b3[1];
      } else {
        double2 cr = make_double2(0, 0);
        if (s6 > 0.0) {
          const double yr = fmin(CLIP, fmax(-CLIP, (double)(y0 + b3[0])));
          const double yi = fmin(CLIP, fmax(-CLIP, (double)(y1 + b3[1])));
          cr = make_double2(s6 * yr, s6 * yi);
          double2 *dst = (double2 *)s.z[0];
          dst->x += cr.x;
          dst->y += cr.y;
        }
        if (corr_out) corr_out[idx] = cr;
      }
    }
    // the next tile's inputs overwrite the A tile only after every thread read its TMEM lanes
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(PRED_W));
  }
}

// Selection of the elements the network corrects: the scale s6 of every element of row T
// (0 where no correction applies) and the row maximum; then the elements with
// s6 >= max / PRED_SELECT go into a list and every other element's correction is zero.
// An element left out keeps the polynomial prediction, whose error there is of order s6,
// i.e. far below the row's largest error, which is what the corrector's residual sees.
constexpr double PRED_SELECT = 32.0;
__global__ void s6_kernel(DevGF G, int T, i64 total, const double *exw, double *s6buf, unsigned long long *mx) {
  double m = 0.0;
  for (i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x; idx < total; idx += (i64)gridDim.x * blockDim.x) {
    Series s;
    float x[PRED_IN];
    double2 p;
    double s6 = 0.0;
    if (!(series_of(G, T, idx, s) && features(s, exw, x, p, s6))) s6 = 0.0;
    s6buf[idx] = s6;
    m = fmax(m, s6);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(mx, (unsigned long long)__double_as_longlong(m));
}

__global__ void select_kernel(i64 total, const double *s6buf, unsigned long long *w, i64 *sel, double2 *corr_out) {
  const double lim = __longlong_as_double((long long)w[0]) / PRED_SELECT;
  for (i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x; idx < total; idx += (i64)gridDim.x * blockDim.x) {
    const double s6 = s6buf[idx];
    if (s6 > 0.0 && s6 >= lim) {
      sel[atomicAdd(w + 1, 1ULL)] = idx;
    } else if (corr_out) {
      corr_out[idx] = make_double2(0.0, 0.0);
    }
  }
}

// Judge the two predictions after the first corrector iteration, on the corrected
// elements: out[0] = max |G_1 - P_learned|, out[1] = max |G_1 - P_plain| with
// P_learned the saved row (les column | ret row | tv row) and P_plain = P_learned - corr.
__global__ void judge_kernel(DevGF G, int T, i64 total, const double2 *saved, const double2 *corr,
                             unsigned long long *out) {
  double ml = 0.0, mp = 0.0;
  const i64 es = G.es, ntv = G.ntau + 1, nd = T - HIST + 1;
  for (i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x; idx < total; idx += (i64)gridDim.x * blockDim.x) {
    const double2 c = corr[idx];
    if (c.x == 0.0 && c.y == 0.0) continue;
    const i64 blk = idx / es, e = idx - blk * es;
    const double2 *g;
    i64 off;
    if (blk < ntv) {
      g = G.tvptr(T, blk) + e;
      off = (2 * (i64)(T + 1) + blk) * es + e;
    } else if (blk - ntv < nd) {
      const i64 col = HIST + blk - ntv;
      g = G.retptr(T, col) + e;
      off = ((i64)(T + 1) + col) * es + e;
    } else {
      const i64 row = HIST + blk - ntv - nd;
      g = G.lesptr(row, T) + e;
      off = row * es + e;
    }
    const double2 v = *g, s = saved[off];
    ml = fmax(ml, hypot(v.x - s.x, v.y - s.y));
    mp = fmax(mp, hypot(v.x - s.x + c.x, v.y - s.y + c.y));
  }
  for (int o = 16; o > 0; o >>= 1) {
    ml = fmax(ml, __shfl_xor_sync(0xffffffffu, ml, o));
    mp = fmax(mp, __shfl_xor_sync(0xffffffffu, mp, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, (unsigned long long)__double_as_longlong(ml));
    atomicMax(out + 1, (unsigned long long)__double_as_longlong(mp));
  }
}

// ---- training kernels -------------------------------------------------------------
// C[m][n] (+)= sum_k bf(A(m,k)) bf(B(k,n)); A(m,k) = A[m*sam + k*sak], B(k,n) = B[k*sbk + n*sbn]
__global__ void mm_kernel(int M, int Nn, int K, const float *A, i64 sam, i64 sak, const float *B, i64 sbk, i64 sbn,
                          float *C, i64 ldc, int accumulate) {
  __shared__ float As[64][17], Bs[16][65];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += 16) {
    for (int i = threadIdx.x; i < 64 * 16; i += TPB) {
      const int r = i / 16, k = i % 16;
      As[r][k] = (m0 + r < M && k0 + k < K) ? bfr(A[(i64)(m0 + r) * sam + (i64)(k0 + k) * sak]) : 0.f;
      const int kk = i / 64, c = i % 64;
      Bs[kk][c] = (k0 + kk < K && n0 + c < Nn) ? bfr(B[(i64)(k0 + kk) * sbk + (i64)(n0 + c) * sbn]) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 16; k++) {
      float a[4], b[4];
      for (int i = 0; i < 4; i++) a[i] = As[ty * 4 + i][k];
      for (int j = 0; j < 4; j++) b[j] = Bs[k][tx * 4 + j];
      for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      const int m = m0 + ty * 4 + i, n = n0 + tx * 4 + j;
      if (m < M && n < Nn) C[(i64)m * ldc + n] = accumulate ? C[(i64)m * ldc + n] + acc[i][j] : acc[i][j];
    }
}

__global__ void bias_tanh_kernel(int B, int W, float *Z, const float *b, int act) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B * W; i += gridDim.x * blockDim.x) {
    const float v = Z[i] + b[i % W];
    Z[i] = act ? bfr(tanhf(v)) : v;
  }
}
// dZ = dH * (1 - H^2)
__global__ void tanh_back_kernel(int n, const float *H, float *dH) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dH[i] *= 1.f - H[i] * H[i];
}
// column sums of dZ (B x W) into db
__global__ void colsum_kernel(int B, int W, const float *dZ, float *db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= W) return;
  float s = 0.f;
  for (int r = 0; r < B; r++) s += dZ[(i64)r * W + c];
  db[c] = s;
}
// dY = (Y - T) / B and the loss 0.5 sum |Y - T|^2 / B
__global__ void loss_kernel(int n, const float *Y, const float *T, float scale, float *dY, double *loss) {
  double l = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float d = Y[i] - T[i];
    dY[i] = d * scale;
    l += 0.5 * (double)d * d;
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, l * scale);
}
__global__ void gather_kernel(int B, const float *X, const float *Y, i64 n, unsigned long long seed, float *xb,
                              float *yb) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < B; r += gridDim.x * blockDim.x) {
    const unsigned long long h = ((unsigned long long)hash32(seed * 7919ULL + (unsigned long long)r) << 32) |
                                 hash32(seed + 31ULL * (unsigned long long)r + 17ULL);
    const i64 src = (i64)(h % (unsigned long long)n);
    for (int i = 0; i < PRED_IN; i++) xb[r * PRED_IN + i] = X[src * PRED_IN + i];
    yb[r * 2] = Y[src * 2];
    yb[r * 2 + 1] = Y[src * 2 + 1];
  }
}
__global__ void adam_kernel(int n, float *w, const float *g, float *m, float *v, float lr, float b1, float b2,
                            float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    m[i] = b1 * m[i] + (1.f - b1) * gi;
    v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
    w[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + 1e-8f);
  }
}

void mm(cudaStream_t s, int M, int N, int K, const float *A, i64 sam, i64 sak, const float *B, i64 sbk, i64 sbn,
        float *C, i64 ldc, bool acc) {
  dim3 grid((N + 63) / 64, (M + 63) / 64);
  mm_kernel<<<grid, TPB, 0, s>>>(M, N, K, A, sam, sak, B, sbk, sbn, C, ldc, acc ? 1 : 0);
  NEDY_CHECK_LAUNCH();
}
unsigned gblocks(i64 n) { return (unsigned)std::min<i64>((n + TPB - 1) / TPB, 148LL * 8); }

}  // namespace

// parameter offsets
static constexpr i64 OW1 = 0, OB1 = OW1 + PRED_W * PRED_IN, OW2 = OB1 + PRED_W, OB2 = OW2 + PRED_W * PRED_W;
static constexpr i64 OW3 = OB2 + PRED_W, OB3 = OW3 + 2 * PRED_W;
static_assert(OB3 + 2 == PRED_NPARAM, "parameter layout");

Predictor::Predictor(Ctx &c, i64 capacity, unsigned long long seed_) : ctx(c), cap(capacity), seed(seed_) {
  NEDY_REQUIRE(capacity > 0, "predictor: capacity must be positive");
  NEDY_CUDA(cudaMalloc(&W, sizeof(float) * PRED_NPARAM * 4));  // weights, gradient, Adam m, v
  G = W + PRED_NPARAM;
  Mo = G + PRED_NPARAM;
  Vo = Mo + PRED_NPARAM;
  NEDY_CUDA(cudaMalloc(&X, sizeof(float) * cap * (PRED_IN + 2)));
  Y = X + cap * PRED_IN;
  NEDY_CUDA(cudaMalloc(&count, 4 * sizeof(unsigned long long)));
  dloss = (double *)(count + 1);
  NEDY_CUDA(cudaMemsetAsync(count, 0, 4 * sizeof(unsigned long long), c.stream));
  init(seed);
}

Predictor::~Predictor() {
  if (s6buf) cudaFree(s6buf);
  if (sel) cudaFree(sel);
  if (selw) cudaFree(selw);
  cudaFree(W);
  cudaFree(X);
  cudaFree(count);
  if (work) cudaFree(work);
}

void Predictor::init(unsigned long long sd) {
  std::vector<float> h(PRED_NPARAM, 0.f);
  std::mt19937_64 rng(sd);
  auto fill = [&](i64 off, int out, int in, float gain) {
    std::uniform_real_distribution<float> u(-gain / std::sqrt((float)in), gain / std::sqrt((float)in));
    for (i64 i = 0; i < (i64)out * in; i++) h[off + i] = u(rng);
  };
  fill(OW1, PRED_W, PRED_IN, 1.0f);
  fill(OW2, PRED_W, PRED_W, 1.0f);
  fill(OW3, 2, PRED_W, 0.1f);
  set_params(h.data());
  NEDY_CUDA(cudaMemsetAsync(Mo, 0, sizeof(float) * PRED_NPARAM * 2, ctx.stream));
  adam_t = 0;
}

void Predictor::set_params(const float *host) {
  NEDY_CUDA(cudaMemcpyAsync(W, host, sizeof(float) * PRED_NPARAM, cudaMemcpyHostToDevice, ctx.stream));
  NEDY_CUDA(cudaStreamSynchronize(ctx.stream));
}
void Predictor::get_params(float *host) {
  NEDY_CUDA(cudaMemcpyAsync(host, W, sizeof(float) * PRED_NPARAM, cudaMemcpyDeviceToHost, ctx.stream));
  NEDY_CUDA(cudaStreamSynchronize(ctx.stream));
}

i64 Predictor::row_elements(const DevGF &g, int T) {
  return T < HIST ? 0 : ((i64)(g.ntau + 1) + 2 * (i64)(T - HIST + 1)) * g.es;
}

void Predictor::collect(const DevGF &g, int T, int stride) {
  const i64 tot = row_elements(g, T);
  if (tot == 0) return;
  NEDY_REQUIRE(ctx.k == 5, "predictor: needs the k = 5 extrapolation");
  collect_kernel<<<gblocks(tot), TPB, 0, ctx.stream>>>(g, T, tot, ctx.d_ex, std::max(1, stride),
                                                       seed * 131ULL + (unsigned long long)T * 977ULL + ncollect++, X,
                                                       Y, count, cap);
  NEDY_CHECK_LAUNCH();
}

void Predictor::clear_samples() { NEDY_CUDA(cudaMemsetAsync(count, 0, sizeof(unsigned long long), ctx.stream)); }

i64 Predictor::samples() {
  unsigned long long h = 0;
  NEDY_CUDA(cudaMemcpyAsync(&h, count, sizeof(h), cudaMemcpyDeviceToHost, ctx.stream));
  NEDY_CUDA(cudaStreamSynchronize(ctx.stream));
  return std::min<i64>((i64)h, cap);
}

void Predictor::ensure_work(int B) {
  const i64 need = (i64)B * (3 * PRED_W + 4);
  if (work_cap >= need) return;
  if (work) cudaFree(work);
  work = nullptr;
  NEDY_CUDA(cudaMalloc(&work, sizeof(float) * need));
  work_cap = need;
}

// forward on B rows of xb (B x PRED_IN) -> y (B x 2); keeps h1, h2 for the backward pass
void Predictor::forward(int B, const float *xb, float *h1, float *h2, float *y) {
  cudaStream_t s = ctx.stream;
  mm(s, B, PRED_W, PRED_IN, xb, PRED_IN, 1, W + OW1, 1, PRED_IN, h1, PRED_W, false);
  bias_tanh_kernel<<<gblocks((i64)B * PRED_W), TPB, 0, s>>>(B, PRED_W, h1, W + OB1, 1);
  NEDY_CHECK_LAUNCH();
  mm(s, B, PRED_W, PRED_W, h1, PRED_W, 1, W + OW2, 1, PRED_W, h2, PRED_W, false);
  bias_tanh_kernel<<<gblocks((i64)B * PRED_W), TPB, 0, s>>>(B, PRED_W, h2, W + OB2, 1);
  NEDY_CHECK_LAUNCH();
  mm(s, B, 2, PRED_W, h2, PRED_W, 1, W + OW3, 1, PRED_W, y, 2, false);
  bias_tanh_kernel<<<gblocks((i64)B * 2), TPB, 0, s>>>(B, 2, y, W + OB3, 0);
  NEDY_CHECK_LAUNCH();
}

// loss = sum 0.5 |y - t|^2 / B and its gradient into G
double Predictor::loss_grad(int B, const float *xb, const float *tb, bool want_loss) {
  cudaStream_t s = ctx.stream;
  ensure_work(B);
  float *h1 = work, *h2 = h1 + (i64)B * PRED_W, *y = h2 + (i64)B * PRED_W, *dy = y + 2 * B;
  float *dh2 = dy + 2 * B;
  forward(B, xb, h1, h2, y);
  NEDY_CUDA(cudaMemsetAsync(dloss, 0, sizeof(double), s));
  loss_kernel<<<gblocks(2 * B), TPB, 0, s>>>(2 * B, y, tb, 1.f / B, dy, dloss);
  NEDY_CHECK_LAUNCH();
  // output layer: dW3 = dy^T h2 (2 x 256), db3
  mm(s, 2, PRED_W, B, dy, 1, 2, h2, PRED_W, 1, G + OW3, PRED_W, false);
  colsum_kernel<<<1, 32, 0, s>>>(B, 2, dy, G + OB3);
  NEDY_CHECK_LAUNCH();
  // dh2 = dy W3 (B x 256), through tanh
  mm(s, B, PRED_W, 2, dy, 2, 1, W + OW3, PRED_W, 1, dh2, PRED_W, false);
  tanh_back_kernel<<<gblocks((i64)B * PRED_W), TPB, 0, s>>>(B * PRED_W, h2, dh2);
  NEDY_CHECK_LAUNCH();
  mm(s, PRED_W, PRED_W, B, dh2, 1, PRED_W, h1, PRED_W, 1, G + OW2, PRED_W, false);
  colsum_kernel<<<1, PRED_W, 0, s>>>(B, PRED_W, dh2, G + OB2);
  NEDY_CHECK_LAUNCH();
  // dh1 = dh2 W2 (into the h2 buffer, no longer needed), through tanh
  float *dh1 = h2;
  mm(s, B, PRED_W, PRED_W, dh2, PRED_W, 1, W + OW2, PRED_W, 1, dh1, PRED_W, false);
  tanh_back_kernel<<<gblocks((i64)B * PRED_W), TPB, 0, s>>>(B * PRED_W, h1, dh1);
  NEDY_CHECK_LAUNCH();
  mm(s, PRED_W, PRED_IN, B, dh1, 1, PRED_W, xb, PRED_IN, 1, G + OW1, PRED_IN, false);
  colsum_kernel<<<1, PRED_W, 0, s>>>(B, PRED_W, dh1, G + OB1);
  NEDY_CHECK_LAUNCH();
  double l = 0.0;
  if (want_loss) {
    NEDY_CUDA(cudaMemcpyAsync(&l, dloss, sizeof(double), cudaMemcpyDeviceToHost, s));
    NEDY_CUDA(cudaStreamSynchronize(s));
  }
  return l;
}

double Predictor::train(int iters, int B, double lr) {
  const i64 n = samples();
  NEDY_REQUIRE(n > 0, "predictor: no training samples collected");
  NEDY_REQUIRE(iters >= 0 && B > 0 && lr > 0, "predictor: bad training arguments");
  ensure_work(B);
  float *xb = nullptr;
  NEDY_CUDA(cudaMalloc(&xb, sizeof(float) * B * (PRED_IN + 2)));
  float *tb = xb + (i64)B * PRED_IN;
  double l = 0.0;
  const float b1 = 0.9f, b2 = 0.999f;
  for (int it = 0; it < iters; it++) {
    gather_kernel<<<gblocks(B), TPB, 0, ctx.stream>>>(B, X, Y, n, seed * 65537ULL + (unsigned long long)adam_t, xb, tb);
    NEDY_CHECK_LAUNCH();
    l = loss_grad(B, xb, tb, it == iters - 1);
    adam_t++;
    const float c1 = 1.f - powf(b1, (float)adam_t), c2 = 1.f - powf(b2, (float)adam_t);
    adam_kernel<<<gblocks(PRED_NPARAM), TPB, 0, ctx.stream>>>((int)PRED_NPARAM, W, G, Mo, Vo, (float)lr, b1, b2, c1,
                                                               c2);
    NEDY_CHECK_LAUNCH();
  }
  NEDY_CUDA(cudaStreamSynchronize(ctx.stream));
  cudaFree(xb);
  return l;
}

void Predictor::ensure_mlp() {
  static std::atomic<bool> attr[64];  // per device (host threads may race here)
  NEDY_REQUIRE(ctx.device < 64, "device index out of range");
  if (!attr[ctx.device].load()) {
    NEDY_CUDA(cudaFuncSetAttribute(mlp_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, MLP_SMEM));
    attr[ctx.device].store(true);
  }
  if (!selw) {
    NEDY_CUDA(cudaMalloc(&selw, 2 * sizeof(unsigned long long) + sizeof(int)));
    NEDY_CUDA(cudaMemsetAsync(selw, 0, 2 * sizeof(unsigned long long) + sizeof(int), ctx.stream));
  }
}

int *Predictor::err_word() const { return (int *)(selw + 2); }

void Predictor::check_err() {
  int e = 0;
  NEDY_CUDA(cudaMemcpyAsync(&e, err_word(), sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
  NEDY_CUDA(cudaStreamSynchronize(ctx.stream));
  if (e) {
    NEDY_CUDA(cudaMemsetAsync(err_word(), 0, sizeof(int), ctx.stream));
    throw CudaError("learned predictor: a bounded tensor-core wait timed out");
  }
}

void Predictor::apply(const DevGF &g, int T, double2 *corr_out) {
  const i64 tot = row_elements(g, T);
  if (tot == 0) return;
  ensure_mlp();
  if (sel_cap < tot) {  // grown geometrically, so that a run reallocates a few times at most
    const i64 cap2 = std::max<i64>(tot, sel_cap + sel_cap / 2);
    NEDY_CUDA(cudaStreamSynchronize(ctx.stream));
    cudaFree(s6buf);
    cudaFree(sel);
    s6buf = nullptr;
    sel = nullptr;
    sel_cap = 0;
    NEDY_CUDA(cudaMalloc(&s6buf, sizeof(double) * cap2));
    NEDY_CUDA(cudaMalloc(&sel, sizeof(i64) * cap2));
    sel_cap = cap2;
  }
  NEDY_CUDA(cudaMemsetAsync(selw, 0, 2 * sizeof(unsigned long long), ctx.stream));
  const unsigned gb = (unsigned)std::min<i64>((tot + TPB - 1) / TPB, 148LL * 8);
  s6_kernel<<<gb, TPB, 0, ctx.stream>>>(g, T, tot, ctx.d_ex, s6buf, selw);
  NEDY_CHECK_LAUNCH();
  select_kernel<<<gb, TPB, 0, ctx.stream>>>(tot, s6buf, selw, sel, corr_out);
  NEDY_CHECK_LAUNCH();
  // the selected count is read by the kernel; the grid covers every element in the worst case
  const unsigned blocks = (unsigned)std::min<i64>((tot + MLP_T - 1) / MLP_T, 148LL);
  mlp_tc_kernel<<<blocks, MLP_T, MLP_SMEM, ctx.stream>>>(g, T, sel, selw, ctx.d_ex, W, corr_out, nullptr, 0, nullptr,
                                                         err_word());
  NEDY_CHECK_LAUNCH();
}

void Predictor::infer(int n, const float *x, float *y) {
  ensure_mlp();
  const unsigned blocks = (unsigned)std::min<i64>((n + MLP_T - 1) / MLP_T, 148LL);
  mlp_tc_kernel<<<blocks, MLP_T, MLP_SMEM, ctx.stream>>>(DevGF{}, 0, nullptr, nullptr, nullptr, W, nullptr, x, n, y,
                                                         err_word());
  NEDY_CHECK_LAUNCH();
  check_err();
}

void Predictor::judge(const DevGF &g, int T, const double2 *saved, const double2 *corr, double &d_learned,
                      double &d_plain) {
  const i64 tot = row_elements(g, T);
  d_learned = d_plain = 0.0;
  if (tot == 0) return;
  unsigned long long *o = count + 2;  // the two judge words after the sample count and the loss
  NEDY_CUDA(cudaMemsetAsync(o, 0, 2 * sizeof(unsigned long long), ctx.stream));
  judge_kernel<<<gblocks(tot), TPB, 0, ctx.stream>>>(g, T, tot, saved, corr, o);
  NEDY_CHECK_LAUNCH();
  unsigned long long h[2];
  NEDY_CUDA(cudaMemcpyAsync(h, o, sizeof(h), cudaMemcpyDeviceToHost, ctx.stream));
  NEDY_CUDA(cudaStreamSynchronize(ctx.stream));
  d_learned = __builtin_bit_cast(double, h[0]);
  d_plain = __builtin_bit_cast(double, h[1]);
  if (selw) check_err();
}

}  // namespace nedy
