// Split-precision GEMM: BF16 piece products on tcgen05 with FP32 accumulation in
// tensor memory, operands brought into shared memory by TMA (see split_gemm.cuh).
//
// One CTA computes a 128 x BN tile of both output parts: the real part accumulates in
// TMEM columns [0, BN), the imaginary part in [BN, 2 BN).
//   warp 4      TMA producer (one thread): per stage the A tiles (128 x 64; real and
//               imaginary plane of a complex operand) and B tiles (BN x 64) of one
//               piece product and K block, mbarrier transaction counts;
//   warp 5      MMA issuer (one thread): per stage 2 (complex x real) or 4 (complex x
//               complex) tile products, each 4 x tcgen05.mma (M128 N BN K16) into the
//               accumulator of its part, the instruction's negate bit giving the minus
//               of Re = Ar Br - Ai Bi; tcgen05.commit frees the stage; owns the TMEM;
//   warps 0-3   epilogue: tcgen05.ld of their 32 TMEM lanes of both parts, FP64 complex
//               or BF16-piece stores through the output View.
// Every mbarrier wait is bounded (2 s); a wait that gives up sets the error word and
// the CTA drains and returns, so no launch can hang.
#include "split_gemm.cuh"
#include "tcgen05.cuh"
#include <cuda.h>
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

namespace nedy {
namespace {
using namespace tc;

constexpr int BM = 128, BK = 64, THREADS = 192;
constexpr int A_BYTES = BM * BK * 2;
constexpr int SMEM_LIMIT = 196608;  // operand stages per CTA (the rest: alignment, barriers)
// one tile product of a stage: A slot, B slot, accumulator (0 real, 1 imaginary), negate A
struct Mma {
  signed char sa, sb, acc, neg;
};

struct Params {
  int M, N, kblocks, kb_per_split, ksplit, nb;
  int a_nb, b_nb;  // batches stored in the A / B maps (1: shared)
  int a_b0, b_b0;  // first stored batch used
  int nA, nB, nmma, nprod, np, stage_bytes;
  int fuse;  // one-load kernel, real x complex: one N = 2 BN product covers both parts
  int a_comp[2], b_comp[2];  // plane group (0 real, 1 imaginary) of each A / B slot
  Mma mma[4];
  int pa[6], pb[6];  // piece products
  // epilogue
  int out_pieces, out_np, accumulate, atomic;
  double alpha;
  void *out;
  i64 rs_hi, rs_lo, cs_hi, cs_lo, bs, plane;
  int rdiv, cdiv;
  int *err;
};

constexpr int smem_bytes(int stage_bytes, int stages) { return stages * stage_bytes + 1024 + 256; }

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, uint32_t mbar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::
          "r"(dst),
      "l"(map), "r"(mbar), "r"(x), "r"(y), "r"(z)
      : "memory");
}

template <int BKT>
__device__ __forceinline__ uint64_t op_desc(uint32_t saddr) {
  static_assert(BKT == 64 || BKT == 32, "K block of 32 or 64");
  return BKT == 64 ? sw128_desc(saddr) : sw64_desc(saddr);
}

// kind::f16 instruction descriptor: BF16 x BF16 -> F32, both K-major, M = 128, N = bn.
constexpr uint32_t idesc_for(int bn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(bn >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

// column offsets of a 16-column chunk: one division when the chunk stays inside one cdiv
// segment (fast), then base + j * cs_lo
__device__ __forceinline__ bool chunk_base(const Params &P, int nf, i64 &cbase) {
  bool fast = nf + 16 <= P.N;
  cbase = 0;
  if (fast) {
    if (P.cdiv) {
      const int qd = nf / P.cdiv, rm = nf - qd * P.cdiv;
      fast = rm + 16 <= P.cdiv;
      cbase = (i64)qd * P.cs_hi + (i64)rm * P.cs_lo;
    } else {
      cbase = (i64)nf * P.cs_lo;
    }
  }
  return fast;
}
__device__ __forceinline__ i64 col_off(const Params &P, int n) {
  return P.cdiv ? (i64)(n / P.cdiv) * P.cs_hi + (i64)(n % P.cdiv) * P.cs_lo : (i64)n * P.cs_lo;
}

// BF16 pieces of 16 values into the np planes of one part
__device__ __forceinline__ void store_pieces16(const Params &P, __nv_bfloat16 *o, i64 roff, i64 cbase, bool fast,
                                               int nf, const float (&v)[16]) {
  const float al = (float)P.alpha;
  if (fast && P.cs_lo == 1 && ((roff + cbase) & 7) == 0) {
    float x[16];
#pragma unroll
    for (int j = 0; j < 16; j++) x[j] = al * v[j];
    for (int p = 0; p < P.out_np; p++) {
      uint32_t w[8];
#pragma unroll
      for (int j = 0; j < 8; j++) {  // two values per conversion instruction
        const __nv_bfloat162 h = __floats2bfloat162_rn(x[2 * j], x[2 * j + 1]);
        const float2 f = __bfloat1622float2(h);
        x[2 * j] -= f.x;
        x[2 * j + 1] -= f.y;
        w[j] = *(const uint32_t *)&h;
      }
      uint4 *dst = (uint4 *)(o + (i64)p * P.plane + roff + cbase);
      dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
      dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
    }
    return;
  }
#pragma unroll
  for (int j = 0; j < 16; j++) {
    const int n = nf + j;
    if (n >= P.N) break;
    const i64 off = roff + (fast ? cbase + (i64)j * P.cs_lo : col_off(P, n));
    float x = al * v[j];
    for (int p = 0; p < P.out_np; p++) {
      const __nv_bfloat16 h = __float2bfloat16_rn(x);
      o[(i64)p * P.plane + off] = h;
      x -= __bfloat162float(h);
    }
  }
}

// BF16 pieces of a 32-row x 16-column chunk whose 32 rows are contiguous in the output
// (one warp, lane = row): staged through a warp-private 1 KB shared buffer so that every
// lane stores two 16-byte runs of 8 consecutive rows instead of 16 scattered elements.
__device__ __forceinline__ void store_pieces16_rows(const Params &P, __nv_bfloat16 *o, i64 roff0, i64 cbase, int nf,
                                                    const float (&v)[16], __nv_bfloat16 *sbuf, int lane) {
  const float al = (float)P.alpha;
  float x[16];
#pragma unroll
  for (int j = 0; j < 16; j++) x[j] = al * v[j];
  for (int p = 0; p < P.out_np; p++) {
#pragma unroll
    for (int j = 0; j < 16; j += 2) {  // two values per conversion instruction
      const __nv_bfloat162 h = __floats2bfloat162_rn(x[j], x[j + 1]);
      const float2 f = __bfloat1622float2(h);
      x[j] -= f.x;
      x[j + 1] -= f.y;
      sbuf[j * 32 + lane] = h.x;
      sbuf[(j + 1) * 32 + lane] = h.y;
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 2; i++) {
      const int w = lane + 32 * i, c = w >> 2, r8 = (w & 3) * 8;
      if (nf + c < P.N)
        *(uint4 *)(o + (i64)p * P.plane + roff0 + r8 + cbase + (i64)c * P.cs_lo) = *(const uint4 *)(sbuf + c * 32 + r8);
    }
    __syncwarp();
  }
}

// Staged epilogue stores.  A lane owns one output row; rows of a warp are generally far
// apart in memory, so per-lane stores send 32 scattered requests per instruction.  These
// helpers stage the warp's 32 rows in a warp-private shared buffer and write them back
// so that each store instruction covers whole row segments (4 x 128 B of BF16 pieces,
// or 2 x 256 B of FP64 complex).
// BF16 rows of 64 are staged unpadded (128 B) with the 16-byte chunks of row r at chunk
// position j ^ (r & 7), so that both the row-wise writes and the column-wise reads of a warp
// touch every bank once per 128 bytes.
constexpr int STAGE_LD64 = 64;        // BF16 elements per staged row of 64 (swizzled, 128 B)
constexpr int STAGE_LD16 = 17;        // double2 per staged row of 16 (padded, 272 B)
constexpr int STAGE_WARP_BYTES = 32 * STAGE_LD16 * 16;   // FP64 outputs; >= PIECE_WARP_BYTES
constexpr int PIECE_WARP_BYTES = 32 * STAGE_LD64 * 2;    // BF16 piece outputs only

// BF16 pieces of 64 contiguous columns (x: this lane's row, scaled; consumed)
__device__ __forceinline__ void store_pieces64_staged(const Params &P, __nv_bfloat16 *o, i64 roff, int mok,
                                                      i64 cbase, float (&x)[64], __nv_bfloat16 *sbuf, int lane) {
  for (int p = 0; p < P.out_np; p++) {
#pragma unroll
    for (int j = 0; j < 64; j += 8) {
      uint32_t w[4];
#pragma unroll
      for (int t = 0; t < 4; t++) {  // two values per conversion instruction
        const __nv_bfloat162 h = __floats2bfloat162_rn(x[j + 2 * t], x[j + 2 * t + 1]);
        const float2 f = __bfloat1622float2(h);
        x[j + 2 * t] -= f.x;
        x[j + 2 * t + 1] -= f.y;
        w[t] = *(const uint32_t *)&h;
      }
      *(uint4 *)(sbuf + lane * STAGE_LD64 + (((j >> 3) ^ (lane & 7)) << 3)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int idx = i * 32 + lane, r = idx >> 3, c8 = (idx & 7) * 8, sw = ((idx & 7) ^ (r & 7)) * 8;
      const i64 ro = __shfl_sync(0xffffffffu, roff, r);
      const int okr = __shfl_sync(0xffffffffu, mok, r);
      if (okr)
        *(uint4 *)(o + (i64)p * P.plane + ro + cbase + c8) = *(const uint4 *)(sbuf + r * STAGE_LD64 + sw);
    }
    __syncwarp();
  }
}

// BF16 pieces of 64 columns of any alignment (the columns may cross index segments of the
// output View, e.g. (l, n) with n < nao for nao not a multiple of 16): one piece at a time
// staged through the warp's buffer (values re-read from TMEM 16 columns at a time, so that
// few registers stay live), then written a row at a time, lane i storing columns i and
// i + 32 of the row, so that each store instruction covers consecutive columns of one row
// instead of one scattered element in each of 32 rows.
__device__ __noinline__ void store_pieces64_generic(const Params &P, __nv_bfloat16 *o, i64 roff, int mok, int nf,
                                                    uint32_t taddr, bool zero, __nv_bfloat16 *sbuf, int lane) {
  i64 coff[2];
  bool cok[2];
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int c = nf + lane + 32 * h;
    cok[h] = c < P.N;
    coff[h] = cok[h] ? col_off(P, c) : 0;
  }
  const float al = (float)P.alpha;
  for (int p = 0; p < P.out_np; p++) {
    for (int q = 0; q < 4; q++) {
      float x[16];
      tmem_ld16(taddr + (uint32_t)(16 * q), x);
#pragma unroll
      for (int j = 0; j < 16; j++) x[j] = zero ? 0.f : al * x[j];
      for (int pp = 0; pp < p; pp++)  // the residual after the earlier pieces
#pragma unroll
        for (int j = 0; j < 16; j++) x[j] -= __bfloat162float(__float2bfloat16_rn(x[j]));
#pragma unroll
      for (int j = 0; j < 16; j += 8) {
        uint32_t w[4];
#pragma unroll
        for (int t = 0; t < 4; t++) {
          const __nv_bfloat162 h = __floats2bfloat162_rn(x[j + 2 * t], x[j + 2 * t + 1]);
          w[t] = *(const uint32_t *)&h;
        }
        const int ch = (16 * q + j) >> 3;
        *(uint4 *)(sbuf + lane * STAGE_LD64 + ((ch ^ (lane & 7)) << 3)) = make_uint4(w[0], w[1], w[2], w[3]);
      }
    }
    __syncwarp();
    __nv_bfloat16 *op = o + (i64)p * P.plane;
    for (int r = 0; r < 32; r++) {
      const i64 ro = __shfl_sync(0xffffffffu, roff, r);
      const int okr = __shfl_sync(0xffffffffu, mok, r);
      if (!okr) continue;  // uniform across the warp
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int c = lane + 32 * h;
        const __nv_bfloat16 v = sbuf[r * STAGE_LD64 + ((((c >> 3) ^ (r & 7)) << 3) | (c & 7))];
        if (cok[h]) op[ro + coff[h]] = v;
      }
    }
    __syncwarp();
  }
}

// FP64 complex outputs of 16 contiguous columns (store, accumulate or atomic add)
__device__ __forceinline__ void store_fp64_16_staged(const Params &P, i64 roff, int mok, i64 cbase,
                                                     const float (&vr)[16], const float (&vi)[16], double2 *sb,
                                                     int lane) {
#pragma unroll
  for (int j = 0; j < 16; j++) sb[lane * STAGE_LD16 + j] = make_double2(P.alpha * (double)vr[j], P.alpha * (double)vi[j]);
  __syncwarp();
#pragma unroll 4
  for (int i = 0; i < 16; i++) {
    const int idx = i * 32 + lane, r = idx >> 4, j = idx & 15;
    const i64 ro = __shfl_sync(0xffffffffu, roff, r);
    const int okr = __shfl_sync(0xffffffffu, mok, r);
    if (!okr) continue;
    double2 *o = (double2 *)P.out + ro + cbase + j;
    const double2 v = sb[r * STAGE_LD16 + j];
    if (P.atomic) {
      atomicAdd(&o->x, v.x);
      atomicAdd(&o->y, v.y);
    } else if (P.accumulate) {
      double2 t = *o;
      t.x += v.x;
      t.y += v.y;
      *o = t;
    } else {
      *o = v;
    }
  }
  __syncwarp();
}

// Epilogue of one 128 x BN output tile: the 32 TMEM lanes of lane quarter `warp` (rows
// m0 + 32 warp ...) of both parts (columns [0, BN) real, [BN, 2 BN) imaginary from tmem),
// output columns [c_lo, c_hi) of the tile, to the output View.  zero: the tile had no K
// blocks (store zeros).  wbuf: this warp's staging buffer in shared memory.
template <int BN>
__device__ __forceinline__ void epilogue_tile(const Params &P, int m0, int n0, int b, int warp, int lane,
                                              uint32_t tmem, bool zero, uint8_t *wbuf, int c_lo = 0, int c_hi = BN) {
    const int m = m0 + warp * 32 + lane;
    const bool mok = m < P.M;
    const i64 roff =
        (P.rdiv ? (i64)(m / P.rdiv) * P.rs_hi + (i64)(m % P.rdiv) * P.rs_lo : (i64)m * P.rs_lo) + (i64)b * P.bs;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    // piece outputs whose 32 rows of this warp are contiguous use the row-staged store
    const int r0 = m0 + warp * 32;
    bool rows_contig = P.out_pieces && P.rs_lo == 1 && r0 + 32 <= P.M;
    if (rows_contig && P.rdiv) rows_contig = (r0 % P.rdiv) + 32 <= P.rdiv;
    const i64 roff0 = __shfl_sync(0xffffffffu, roff, 0);
    rows_contig = rows_contig && (roff0 & 7) == 0;
    // every row offset a multiple of 8 elements (16-byte stores of BF16 pieces)
    const bool rows_al8 = __all_sync(0xffffffffu, (roff & 7) == 0);
    __nv_bfloat16 *sbuf = (__nv_bfloat16 *)wbuf;
    const int imok = mok ? 1 : 0;
    {
      for (int c0 = c_lo; c0 < c_hi;) {
        if (n0 + c0 >= P.N) break;  // uniform across the warp
        const int nf = n0 + c0;
        if (P.out_pieces && !rows_contig && rows_al8 && c0 + 64 <= c_hi && nf + 64 <= P.N && P.cs_lo == 1 &&
            (P.cdiv == 0 || (nf % P.cdiv) + 64 <= P.cdiv)) {
          // 64 contiguous columns of each part, staged
          const i64 cbase = P.cdiv ? (i64)(nf / P.cdiv) * P.cs_hi + (i64)(nf % P.cdiv) : (i64)nf;
          if ((cbase & 7) == 0) {
            __nv_bfloat16 *o = (__nv_bfloat16 *)P.out;
            const float al = (float)P.alpha;
            for (int part = 0; part < 2; part++) {
              float x[64];
              tmem_ld64(trow + (uint32_t)(part * BN + c0), x);
#pragma unroll
              for (int j = 0; j < 64; j++) x[j] = zero ? 0.f : al * x[j];
              store_pieces64_staged(P, o + (i64)part * P.out_np * P.plane, roff, imok, cbase, x, sbuf, lane);
            }
            c0 += 64;
            continue;
          }
        }
        if (P.out_pieces && !rows_contig && c0 + 64 <= c_hi && P.cs_lo == 1 && nf + 16 < P.N &&
            (!rows_al8 || (P.cdiv != 0 && ((nf % P.cdiv) + 16 > P.cdiv || (P.cdiv & 15) != 0)))) {
          // 64 columns that the aligned paths would store element by element
          __nv_bfloat16 *o = (__nv_bfloat16 *)P.out;
          for (int part = 0; part < 2; part++)
            store_pieces64_generic(P, o + (i64)part * P.out_np * P.plane, roff, imok, nf,
                                   trow + (uint32_t)(part * BN + c0), zero, sbuf, lane);
          c0 += 64;
          continue;
        }
        float vr[16], vi[16];
        tmem_ld16(trow + (uint32_t)c0, vr);
        tmem_ld16(trow + (uint32_t)(BN + c0), vi);
        if (zero) {
#pragma unroll
          for (int j = 0; j < 16; j++) vr[j] = vi[j] = 0.f;
        }
        c0 += 16;
        i64 cbase;
        const bool fast = chunk_base(P, nf, cbase);
        if (!P.out_pieces && fast && P.cs_lo == 1) {  // warp-uniform
          store_fp64_16_staged(P, roff, imok, cbase, vr, vi, (double2 *)wbuf, lane);
          continue;
        }
        if (!mok) continue;
        if (P.out_pieces) {
          __nv_bfloat16 *o = (__nv_bfloat16 *)P.out;
          if (rows_contig && fast && (cbase & 7) == 0 && (P.cs_lo & 7) == 0) {
            store_pieces16_rows(P, o, roff0, cbase, nf, vr, sbuf, lane);
            store_pieces16_rows(P, o + (i64)P.out_np * P.plane, roff0, cbase, nf, vi, sbuf, lane);
          } else {
            store_pieces16(P, o, roff, cbase, fast, nf, vr);
            store_pieces16(P, o + (i64)P.out_np * P.plane, roff, cbase, fast, nf, vi);
          }
        } else {
#pragma unroll
          for (int j = 0; j < 16; j++) {
            const int n = nf + j;
            if (n >= P.N) break;
            const i64 off = roff + (fast ? cbase + (i64)j * P.cs_lo : col_off(P, n));
            double2 *o = (double2 *)P.out + off;
            const double xr = P.alpha * (double)vr[j], xi = P.alpha * (double)vi[j];
            if (P.atomic) {
              atomicAdd(&o->x, xr);
              atomicAdd(&o->y, xi);
            } else if (P.accumulate) {
              double2 t = *o;
              t.x += xr;
              t.y += xi;
              *o = t;
            } else {
              *o = make_double2(xr, xi);
            }
          }
        }
      }
    }
}

// OL = false: one stage holds one piece product of one K block (the A and B tiles of that
//   product), BKT = 64;
// OL = true ("one load"): one stage holds every piece of one K block (BKT = 32 or 64), and
//   the MMA warp issues all piece products from it, so each piece tile crosses L2 -> SM
//   once per K block instead of once per product it takes part in.  A slots are ordered
//   piece-major (slot p nA + component), B slots likewise, so the real and imaginary B
//   tiles of one piece are adjacent: for real x complex products one MMA with N = 2 BN
//   writes both parts (TMEM columns [0, BN) real, [BN, 2 BN) imaginary).
template <int BN, int STAGES, int BKT, bool OL>
__global__ void __launch_bounds__(THREADS, (BN == 128 || (BN == 64 && STAGES <= 2)) ? 2 : 1)
    split_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const __grid_constant__ Params P) {
  static_assert(OL || BKT == BK, "the per-product kernel uses 64-wide K blocks");
  constexpr int A_TILE = BM * BKT * 2;
  constexpr int B_BYTES = BN * BKT * 2;
  constexpr uint32_t TCOLS = 2 * BN;
  constexpr uint32_t IDESC = idesc_for(BN);
  constexpr uint32_t IDESC2 = idesc_for(BN * 2 <= 256 ? BN * 2 : BN);
  extern __shared__ uint8_t sraw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)sraw + 1023) & ~(uintptr_t)1023);
  uint64_t *bar = (uint64_t *)(smem + STAGES * P.stage_bytes);  // full[STAGES], empty[STAGES], done
  uint32_t *tmem_slot = (uint32_t *)(bar + 2 * STAGES + 1);
  __shared__ int s_skip;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.z / P.ksplit, ks = blockIdx.z - (blockIdx.z / P.ksplit) * P.ksplit;
  const int n0 = blockIdx.x * BN, m0 = blockIdx.y * BM;
  const int kb0 = ks * P.kb_per_split;
  const int nkb = max(0, min(P.kblocks, kb0 + P.kb_per_split) - kb0);
  int iters = OL ? nkb : nkb * P.nprod;
  const uint32_t full0 = smem_u32(bar), empty0 = smem_u32(bar + STAGES), done = smem_u32(bar + 2 * STAGES);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_skip = *(volatile int *)P.err != 0;  // an earlier CTA gave up: do nothing
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const bool skip = s_skip != 0;
  if (skip) iters = 0;

  if (warp == 4 && lane == 0) {
    // ---- TMA producer
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmB) : "memory");
    int issued = 0;
    for (int it = 0; it < iters; it++) {
      const int s = it % STAGES;
      const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
      if (it >= STAGES && !mbar_wait(empty0 + 8 * s, ph ^ 1u, P.err, 1)) break;
      const uint32_t base = smem_u32(smem + s * P.stage_bytes);
      mbar_expect_tx(full0 + 8 * s, P.stage_bytes);
      issued = it + 1;
      const int ab = P.a_nb > 1 ? P.a_b0 + b : 0, bb = P.b_nb > 1 ? P.b_b0 + b : 0;
      if (OL) {
        const int kb = kb0 + it;
        const uint32_t bbase = base + P.np * P.nA * A_TILE;
        for (int p = 0; p < P.np; p++) {
          for (int i = 0; i < P.nA; i++)
            tma_load_3d(base + (p * P.nA + i) * A_TILE, &tmA, full0 + 8 * s, kb * BKT, m0,
                        (P.a_comp[i] * P.np + p) * P.a_nb + ab);
          for (int j = 0; j < P.nB; j++)
            tma_load_3d(bbase + (p * P.nB + j) * B_BYTES, &tmB, full0 + 8 * s, kb * BKT, n0,
                        (P.b_comp[j] * P.np + p) * P.b_nb + bb);
        }
      } else {
        const int pr = it / nkb, kb = kb0 + it % nkb;
        for (int i = 0; i < P.nA; i++)
          tma_load_3d(base + i * A_TILE, &tmA, full0 + 8 * s, kb * BKT, m0,
                      (P.a_comp[i] * P.np + P.pa[pr]) * P.a_nb + ab);
        for (int j = 0; j < P.nB; j++)
          tma_load_3d(base + P.nA * A_TILE + j * B_BYTES, &tmB, full0 + 8 * s, kb * BKT, n0,
                      (P.b_comp[j] * P.np + P.pb[pr]) * P.b_nb + bb);
      }
    }
    // The loads of the last STAGES issued stages may still be in flight (the MMA warp may
    // have given up before consuming them): wait until each has landed, so that no TMA
    // write reaches this CTA's shared memory after it exits.  Earlier stages were
    // consumed, which their empty barriers showed.
    for (int j = max(0, issued - STAGES); j < issued; j++)
      mbar_wait_drain(full0 + 8 * (j % STAGES), (uint32_t)(j / STAGES) & 1u, P.err, 4);
  } else if (warp == 5 && lane == 0) {
    // ---- MMA issuer
    bool started0 = false, started1 = false;  // accumulator written once (then accumulate)
    for (int it = 0; it < iters; it++) {
      const int s = it % STAGES;
      const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
      if (!mbar_wait(full0 + 8 * s, ph, P.err, 2)) break;
      tc_fence_after();
      const uint32_t base = smem_u32(smem + s * P.stage_bytes);
      const int nprod = OL ? P.nprod : 1;
      for (int pr = 0; pr < nprod; pr++) {
        // slots of this product's A / B tiles inside the stage
        const int sa0 = OL ? P.pa[pr] * P.nA : 0, sb0 = OL ? P.pb[pr] * P.nB : 0;
        const uint32_t bbase = base + (OL ? P.np : 1) * P.nA * A_TILE;
        if (OL && BN * 2 <= 256 && P.fuse) {
          const uint64_t da = op_desc<BKT>(base + sa0 * A_TILE);
          const uint64_t db = op_desc<BKT>(bbase + sb0 * B_BYTES);
#pragma unroll
          for (int k = 0; k < BKT / 16; k++)
            mma_bf16(tmem, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), IDESC2, (started0 || k > 0) ? 1u : 0u);
          started0 = started1 = true;
          continue;
        }
        for (int q = 0; q < P.nmma; q++) {
          const Mma mq = P.mma[q];
          const uint64_t da = op_desc<BKT>(base + (sa0 + mq.sa) * A_TILE);
          const uint64_t db = op_desc<BKT>(bbase + (sb0 + mq.sb) * B_BYTES);
          const uint32_t idesc = IDESC | (mq.neg ? (1u << 13) : 0u);
          const uint32_t tacc = tmem + (uint32_t)(mq.acc * BN);
#pragma unroll
          for (int k = 0; k < BKT / 16; k++)  // K = 16 per instruction: +32 bytes inside the swizzle atom
            mma_bf16(tacc, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), idesc,
                     ((mq.acc ? started1 : started0) || k > 0) ? 1u : 0u);
          if (mq.acc)
            started1 = true;
          else
            started0 = true;
        }
      }
      mma_commit(empty0 + 8 * s);
    }
    mma_commit(done);
  } else if (warp < 4) {
    // ---- epilogue
    // lane 0 waits and tells the warp, so the .sync.aligned TMEM loads stay convergent
    // `done` tracks every MMA the issuer started, also when it gave up early, so this
    // wait ends once they have finished and TMEM can be read and released.  Accumulators
    // of a CTA whose producer or issuer gave up are incomplete: nothing is stored then.
    int okl = 0;
    if (lane == 0) okl = (mbar_wait_drain(done, 0, P.err, 3) && *(volatile int *)P.err == 0) ? 1 : 0;
    __syncwarp();
    const bool ok = __shfl_sync(0xffffffffu, okl, 0) != 0 && !skip;
    tc_fence_after();
    if (ok) epilogue_tile<BN>(P, m0, n0, b, warp, lane, tmem, iters == 0, smem + warp * STAGE_WARP_BYTES);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 5) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS));
  }
}

// ---- CTA-pair variant of the one-load kernel (tcgen05.mma.cta_group::2)
// A cluster of two CTAs (adjacent row tiles, the same column tile) computes one 256 x BN
// tile: each CTA stages its own 128 rows of A and half of the BN rows of B (rows
// n0 + r BN/2 for pair rank r), so per K block a CTA moves A + B/2 instead of A + B, and
// its TMEM holds its 128 rows x BN columns of both parts.  Rank 0 issues the MMAs
// (M = 256, each operand read from the same shared-memory offset in both CTAs).
// Barriers: every CTA's TMA loads complete on its own full barrier; the MMA warp of rank 1
// (idle otherwise) waits for each of its stages and arrives remotely on rank 0's full
// barrier, which therefore expects two arrivals (rank 0's expect_tx and rank 1's); the MMA
// issuer's tcgen05.commit multicasts stage release (empty) and completion (done) to both
// CTAs.  Both CTAs take the same path (a skip decided by either is taken by both), every
// wait is bounded, every CTA drains the loads it issued itself, and a cluster barrier
// before TMEM is released keeps each CTA's shared memory alive while the other still uses it.
namespace pr {
__device__ __forceinline__ uint32_t cta_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t map_to(uint32_t saddr, uint32_t rank) {
  uint32_t a;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(saddr), "r"(rank));
  return a;
}
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ int ld_cluster(uint32_t caddr) {
  int v;
  asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(caddr) : "memory");
  return v;
}
__device__ __forceinline__ void arrive_remote(uint32_t caddr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(caddr) : "memory");
}
__device__ __forceinline__ void mma2(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}
// arrive on the barrier at this shared-memory offset in every CTA of `mask` once the MMAs
// this thread issued have finished
__device__ __forceinline__ void commit2(uint32_t mbar, uint16_t mask) {
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::
                   "r"(mbar), "h"(mask)
               : "memory");
}
}  // namespace pr

template <int BN, int STAGES, int BKT>
__global__ void __launch_bounds__(THREADS, 1)
    split_gemm_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                           const __grid_constant__ Params P) {
  constexpr int A_TILE = BM * BKT * 2;
  constexpr int BH = BN / 2;               // rows of B this CTA stages
  constexpr int B_BYTES = BH * BKT * 2;
  constexpr uint32_t TCOLS = 2 * BN;
  constexpr uint32_t IDESC = idesc_bf16(2 * BM, BN);
  extern __shared__ uint8_t sraw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)sraw + 1023) & ~(uintptr_t)1023);
  uint64_t *bar = (uint64_t *)(smem + STAGES * P.stage_bytes);  // full[STAGES], empty[STAGES], done
  uint32_t *tmem_slot = (uint32_t *)(bar + 2 * STAGES + 1);
  __shared__ int s_skip, s_skip_pair;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = pr::cta_rank(), peer = rank ^ 1u, lead = rank & ~1u;
  const bool leader = (rank & 1u) == 0;
  const uint16_t mask = (uint16_t)(3u << lead);
  // grid: x row tiles (pairs of consecutive x form the clusters), y column tiles, z batch x K split
  const int b = blockIdx.z / P.ksplit, ks = blockIdx.z - (blockIdx.z / P.ksplit) * P.ksplit;
  const int n0 = blockIdx.y * BN, m0 = blockIdx.x * BM;
  const int kb0 = ks * P.kb_per_split;
  const int nkb = max(0, min(P.kblocks, kb0 + P.kb_per_split) - kb0);
  int iters = nkb;
  const uint32_t full0 = smem_u32(bar), empty0 = smem_u32(bar + STAGES), done = smem_u32(bar + 2 * STAGES);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(full0 + 8 * s, leader ? 2 : 1);  // rank 0: its own expect_tx + rank 1's forward
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_skip = *(volatile int *)P.err != 0;  // an earlier CTA gave up: do nothing
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
  }
  tc_fence_before();
  pr::cluster_sync();  // barriers of both CTAs initialised, both skip flags written
  tc_fence_after();
  if (threadIdx.x == 0) s_skip_pair = s_skip | pr::ld_cluster(pr::map_to(smem_u32(&s_skip), peer));
  __syncthreads();
  const uint32_t tmem = *tmem_slot;
  const bool skip = s_skip_pair != 0;
  if (skip) iters = 0;

  if (warp == 4 && lane == 0) {
    // ---- TMA producer (both CTAs): own A rows, own half of the B rows, own full barrier
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmB) : "memory");
    int issued = 0;
    const int ab = P.a_nb > 1 ? P.a_b0 + b : 0, bb = P.b_nb > 1 ? P.b_b0 + b : 0;
    const int nb0 = n0 + (int)(rank & 1u) * BH;
    for (int it = 0; it < iters; it++) {
      const int s = it % STAGES;
      const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
      if (it >= STAGES && !mbar_wait(empty0 + 8 * s, ph ^ 1u, P.err, 1)) break;
      const uint32_t base = smem_u32(smem + s * P.stage_bytes);
      mbar_expect_tx(full0 + 8 * s, P.stage_bytes);
      issued = it + 1;
      const int kb = kb0 + it;
      const uint32_t bbase = base + P.np * P.nA * A_TILE;
      for (int p = 0; p < P.np; p++) {
        for (int i = 0; i < P.nA; i++)
          tma_load_3d(base + (p * P.nA + i) * A_TILE, &tmA, full0 + 8 * s, kb * BKT, m0,
                      (P.a_comp[i] * P.np + p) * P.a_nb + ab);
        for (int j = 0; j < P.nB; j++)
          tma_load_3d(bbase + (p * P.nB + j) * B_BYTES, &tmB, full0 + 8 * s, kb * BKT, nb0,
                      (P.b_comp[j] * P.np + p) * P.b_nb + bb);
      }
    }
    // loads of the last STAGES issued stages may still be in flight (the consumer may have
    // given up): wait until each has landed, so that none reaches shared memory after exit
    for (int j = max(0, issued - STAGES); j < issued; j++)
      mbar_wait_drain(full0 + 8 * (j % STAGES), (uint32_t)(j / STAGES) & 1u, P.err, 4);
  } else if (warp == 5 && lane == 0 && !leader) {
    // ---- rank 1: tell rank 0 when each of its stages has landed
    const uint32_t lfull0 = pr::map_to(full0, lead);
    for (int it = 0; it < iters; it++) {
      const int s = it % STAGES;
      if (!mbar_wait(full0 + 8 * s, (uint32_t)(it / STAGES) & 1u, P.err, 2)) break;
      pr::arrive_remote(lfull0 + 8 * s);
    }
  } else if (warp == 5 && lane == 0) {
    // ---- rank 0: MMA issuer for the pair
    bool started0 = false, started1 = false;
    for (int it = 0; it < iters; it++) {
      const int s = it % STAGES;
      const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
      if (!mbar_wait(full0 + 8 * s, ph, P.err, 2)) break;
      tc_fence_after();
      const uint32_t base = smem_u32(smem + s * P.stage_bytes);
      const uint32_t bbase = base + P.np * P.nA * A_TILE;
      for (int pr_ = 0; pr_ < P.nprod; pr_++) {
        const int sa0 = P.pa[pr_] * P.nA, sb0 = P.pb[pr_] * P.nB;
        for (int q = 0; q < P.nmma; q++) {
          const Mma mq = P.mma[q];
          const uint64_t da = op_desc<BKT>(base + (sa0 + mq.sa) * A_TILE);
          const uint64_t db = op_desc<BKT>(bbase + (sb0 + mq.sb) * B_BYTES);
          const uint32_t idesc = IDESC | (mq.neg ? (1u << 13) : 0u);
          const uint32_t tacc = tmem + (uint32_t)(mq.acc * BN);
#pragma unroll
          for (int k = 0; k < BKT / 16; k++)
            pr::mma2(tacc, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), idesc,
                     ((mq.acc ? started1 : started0) || k > 0) ? 1u : 0u);
          if (mq.acc)
            started1 = true;
          else
            started0 = true;
        }
      }
      pr::commit2(empty0 + 8 * s, mask);
    }
    pr::commit2(done, mask);
  } else if (warp < 4) {
    // ---- epilogue (both CTAs): this CTA's 128 rows from its own TMEM.  `done` follows
    // every MMA rank 0 started, also when it gave up; incomplete accumulators are not stored.
    int okl = 0;
    if (lane == 0) okl = (mbar_wait_drain(done, 0, P.err, 3) && *(volatile int *)P.err == 0) ? 1 : 0;
    __syncwarp();
    const bool ok = __shfl_sync(0xffffffffu, okl, 0) != 0 && !skip;
    tc_fence_after();
    if (ok) epilogue_tile<BN>(P, m0, n0, b, warp, lane, tmem, iters == 0, smem + warp * STAGE_WARP_BYTES);
  }
  tc_fence_before();
  __syncthreads();
  pr::cluster_sync();  // neither CTA releases TMEM or exits while the other still works
  if (warp == 5) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS));
  }
}

// Persistent variant of the one-load kernel: one CTA per SM walks a static list of tiles
// (tile t, t + gridDim.x, ...), and TMEM holds two accumulators, so that the epilogue warps
// store tile i while the MMA warp accumulates tile i+1 and the TMA warp loads ahead across
// tile boundaries.  Eight epilogue warps, two per TMEM lane quarter (warps w and w + 4 read
// the same 32 lanes and store half of the columns each): the epilogue is a long chain of
// dependent conversions and stores, and a second warp per SM sub-partition hides its latency.
// Warp 8 is the TMA producer, warp 9 the MMA issuer.  Barriers: full / empty per stage
// (TMA -> MMA -> TMA), tfull per accumulator (MMA -> epilogue, tcgen05.commit), tempty per
// accumulator (the eight epilogue warps -> MMA).  Every wait is bounded; on give-up the roles stop, the TMA warp waits for
// the loads it issued and the MMA warp for the MMAs it issued before TMEM is released.
constexpr int P_EPI_WARPS = 8;                      // two per TMEM lane quarter, each half the columns
constexpr int P_THREADS = 32 * (P_EPI_WARPS + 2);   // + TMA warp + MMA warp
constexpr int P_EPI_BYTES = P_EPI_WARPS * PIECE_WARP_BYTES;  // epilogue staging (piece outputs), apart from the stages
// stages + staging; the rest of the 232448-byte opt-in limit: alignment, barriers, static shared memory
constexpr int P_SMEM_LIMIT = 232448 - 1024 - 256 - 128;
constexpr int psmem_bytes(int stage_bytes, int stages) { return stages * stage_bytes + P_EPI_BYTES + 1024 + 256; }

__device__ __forceinline__ void mbar_arrive(uint32_t a) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}

template <int BN, int STAGES, int BKT>
__global__ void __launch_bounds__(P_THREADS, 1)
    split_gemm_persist_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                              const __grid_constant__ Params P, int ntn, int ntm, int ntiles) {
  static_assert(BN <= 128, "two accumulators of 2 BN TMEM columns must fit in 512 columns");
  constexpr int A_TILE = BM * BKT * 2;
  constexpr int B_BYTES = BN * BKT * 2;
  constexpr uint32_t TCOLS = 2 * BN;     // one accumulator: real [0, BN), imaginary [BN, 2 BN)
  constexpr uint32_t TALLOC = 2 * TCOLS;
  constexpr uint32_t IDESC = idesc_for(BN);
  constexpr uint32_t IDESC2 = idesc_for(BN * 2);
  extern __shared__ uint8_t sraw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)sraw + 1023) & ~(uintptr_t)1023);
  uint8_t *epi = smem + STAGES * P.stage_bytes;
  uint64_t *bar = (uint64_t *)(epi + P_EPI_BYTES);  // full[ST], empty[ST], tfull[2], tempty[2], done
  uint32_t *tmem_slot = (uint32_t *)(bar + 2 * STAGES + 5);
  __shared__ int s_skip;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t full0 = smem_u32(bar), empty0 = smem_u32(bar + STAGES), tfull0 = smem_u32(bar + 2 * STAGES),
                 tempty0 = smem_u32(bar + 2 * STAGES + 2), done = smem_u32(bar + 2 * STAGES + 4);
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int i = 0; i < 2; i++) {
      mbar_init(tfull0 + 8 * i, 1);
      mbar_init(tempty0 + 8 * i, P_EPI_WARPS);  // one arrival per epilogue warp
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_skip = *(volatile int *)P.err != 0;
  }
  if (warp == P_EPI_WARPS + 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TALLOC));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int first = s_skip ? ntiles : (int)blockIdx.x;
  // tile t: column tile fastest, then row tile, then batch x K split (the grid order of the
  // non-persistent kernel)
  auto decode = [&](int t, int &n0, int &m0, int &b, int &kb0, int &nkb) {
    const int nt = t % ntn, r = t / ntn, mt = r % ntm, z = r / ntm;
    b = z / P.ksplit;
    const int ks = z - b * P.ksplit;
    n0 = nt * BN;
    m0 = mt * BM;
    kb0 = ks * P.kb_per_split;
    nkb = max(0, min(P.kblocks, kb0 + P.kb_per_split) - kb0);
  };

  if (warp == P_EPI_WARPS && lane == 0) {
    // ---- TMA producer
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmB) : "memory");
    int g = 0;
    bool stop = false;
    for (int t = first; t < ntiles && !stop; t += gridDim.x) {
      int n0, m0, b, kb0, nkb;
      decode(t, n0, m0, b, kb0, nkb);
      const int ab = P.a_nb > 1 ? P.a_b0 + b : 0, bb = P.b_nb > 1 ? P.b_b0 + b : 0;
      for (int it = 0; it < nkb; it++) {
        const int s = g % STAGES;
        const uint32_t ph = (uint32_t)(g / STAGES) & 1u;
        if (g >= STAGES && !mbar_wait(empty0 + 8 * s, ph ^ 1u, P.err, 1)) {
          stop = true;
          break;
        }
        const uint32_t base = smem_u32(smem + s * P.stage_bytes);
        mbar_expect_tx(full0 + 8 * s, P.stage_bytes);
        const int kb = kb0 + it;
        const uint32_t bbase = base + P.np * P.nA * A_TILE;
        for (int p = 0; p < P.np; p++) {
          for (int i = 0; i < P.nA; i++)
            tma_load_3d(base + (p * P.nA + i) * A_TILE, &tmA, full0 + 8 * s, kb * BKT, m0,
                        (P.a_comp[i] * P.np + p) * P.a_nb + ab);
          for (int j = 0; j < P.nB; j++)
            tma_load_3d(bbase + (p * P.nB + j) * B_BYTES, &tmB, full0 + 8 * s, kb * BKT, n0,
                        (P.b_comp[j] * P.np + p) * P.b_nb + bb);
        }
        g++;
      }
    }
    // the loads of the last STAGES issued stages may still be in flight: wait for them
    for (int j = max(0, g - STAGES); j < g; j++)
      mbar_wait_drain(full0 + 8 * (j % STAGES), (uint32_t)(j / STAGES) & 1u, P.err, 4);
  } else if (warp == P_EPI_WARPS + 1 && lane == 0) {
    // ---- MMA issuer
    int g = 0, lt = 0;
    bool stop = false;
    for (int t = first; t < ntiles && !stop; t += gridDim.x, lt++) {
      int n0, m0, b, kb0, nkb;
      decode(t, n0, m0, b, kb0, nkb);
      const int bi = lt & 1;
      const uint32_t tacc = tmem + (uint32_t)bi * TCOLS;
      // accumulator bi is free once the epilogue has stored tile lt - 2
      if (lt >= 2 && !mbar_wait(tempty0 + 8 * bi, (uint32_t)((lt >> 1) - 1) & 1u, P.err, 5)) break;
      tc_fence_after();
      bool started0 = false, started1 = false;
      for (int it = 0; it < nkb; it++) {
        const int s = g % STAGES;
        const uint32_t ph = (uint32_t)(g / STAGES) & 1u;
        if (!mbar_wait(full0 + 8 * s, ph, P.err, 2)) {
          stop = true;
          break;
        }
        tc_fence_after();
        const uint32_t base = smem_u32(smem + s * P.stage_bytes);
        const uint32_t bbase = base + P.np * P.nA * A_TILE;
        for (int pr = 0; pr < P.nprod; pr++) {
          const int sa0 = P.pa[pr] * P.nA, sb0 = P.pb[pr] * P.nB;
          if (P.fuse) {
            const uint64_t da = op_desc<BKT>(base + sa0 * A_TILE);
            const uint64_t db = op_desc<BKT>(bbase + sb0 * B_BYTES);
#pragma unroll
            for (int k = 0; k < BKT / 16; k++)
              mma_bf16(tacc, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), IDESC2, (started0 || k > 0) ? 1u : 0u);
            started0 = started1 = true;
            continue;
          }
          for (int q = 0; q < P.nmma; q++) {
            const Mma mq = P.mma[q];
            const uint64_t da = op_desc<BKT>(base + (sa0 + mq.sa) * A_TILE);
            const uint64_t db = op_desc<BKT>(bbase + (sb0 + mq.sb) * B_BYTES);
            const uint32_t idesc = IDESC | (mq.neg ? (1u << 13) : 0u);
            const uint32_t ta = tacc + (uint32_t)(mq.acc * BN);
#pragma unroll
            for (int k = 0; k < BKT / 16; k++)
              mma_bf16(ta, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), idesc,
                       ((mq.acc ? started1 : started0) || k > 0) ? 1u : 0u);
            if (mq.acc)
              started1 = true;
            else
              started0 = true;
          }
        }
        mma_commit(empty0 + 8 * s);
        g++;
      }
      if (stop) break;
      mma_commit(tfull0 + 8 * bi);
    }
    // every MMA this thread issued has finished before TMEM is released
    mma_commit(done);
    mbar_wait_drain(done, 0, P.err, 3);
  } else if (warp < P_EPI_WARPS) {
    // ---- epilogue: tile lt from accumulator lt & 1, then hand the accumulator back; warp w
    // reads lane quarter w & 3 and stores columns [(w >> 2) BN / 2, (w >> 2 + 1) BN / 2)
    const int q = warp & 3, c_lo = (warp >> 2) * (BN / 2);
    int lt = 0;
    for (int t = first; t < ntiles; t += gridDim.x, lt++) {
      int n0, m0, b, kb0, nkb;
      decode(t, n0, m0, b, kb0, nkb);
      const int bi = lt & 1;
      int okl = 0;
      if (lane == 0) okl = mbar_wait(tfull0 + 8 * bi, (uint32_t)(lt >> 1) & 1u, P.err, 3) ? 1 : 0;
      __syncwarp();
      if (!__shfl_sync(0xffffffffu, okl, 0)) break;
      tc_fence_after();
      epilogue_tile<BN>(P, m0, n0, b, q, lane, tmem + (uint32_t)bi * TCOLS, nkb == 0, epi + warp * PIECE_WARP_BYTES,
                        c_lo, c_lo + BN / 2);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(tempty0 + 8 * bi);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == P_EPI_WARPS + 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TALLOC));
  }
}

// Persistent CTA-pair kernel (BF16 piece outputs): clusters of two CTAs walk a static list of
// 256 x BN pair tiles (cluster c takes tiles c, c + clusters, ...), each CTA with two TMEM
// accumulators of its 128 rows, so the epilogue of one tile runs beside the MMAs of the next
// as in the persistent kernel, while each CTA stages only its own A rows and half of B as in
// the pair kernel.  Real x complex products (P.fuse): one MMA with N = 2 BN whose B rows are
// the real plane tile (staged by rank 0) followed by the imaginary one (rank 1).
// Barriers: full / empty per stage (rank 1's landings forwarded to rank 0's full barrier),
// tfull per accumulator (multicast commit to both CTAs), tempty per accumulator on rank 0
// with one arrival per epilogue warp of both CTAs (rank 1's remote).
template <int BN, int STAGES, int BKT>
__global__ void __launch_bounds__(P_THREADS, 1)
    split_gemm_persist_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                                   const __grid_constant__ Params P, int ntn, int ntmp, int ntiles) {
  static_assert(BN <= 128, "two accumulators of 2 BN TMEM columns must fit in 512 columns");
  constexpr int A_TILE = BM * BKT * 2;
  constexpr uint32_t TCOLS = 2 * BN;
  constexpr uint32_t TALLOC = 2 * TCOLS;
  constexpr uint32_t IDESC = idesc_bf16(2 * BM, BN);
  constexpr uint32_t IDESC2 = idesc_bf16(2 * BM, 2 * BN);
  extern __shared__ uint8_t sraw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)sraw + 1023) & ~(uintptr_t)1023);
  uint8_t *epi = smem + STAGES * P.stage_bytes;
  uint64_t *bar = (uint64_t *)(epi + P_EPI_BYTES);  // full[ST], empty[ST], tfull[2], tempty[2], done
  uint32_t *tmem_slot = (uint32_t *)(bar + 2 * STAGES + 5);
  __shared__ int s_skip, s_skip_pair;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = pr::cta_rank(), peer = rank ^ 1u, lead = rank & ~1u;
  const bool leader = (rank & 1u) == 0;
  const uint16_t mask = (uint16_t)(3u << lead);
  // B rows this CTA stages per piece: fused, one plane tile of BN rows (rank r: plane r);
  // else BN / 2 rows of every plane (rows n0 + r BN / 2)
  const int brows = P.fuse ? BN : BN / 2;
  const int b_bytes = brows * BKT * 2;
  const uint32_t full0 = smem_u32(bar), empty0 = smem_u32(bar + STAGES), tfull0 = smem_u32(bar + 2 * STAGES),
                 tempty0 = smem_u32(bar + 2 * STAGES + 2), done = smem_u32(bar + 2 * STAGES + 4);
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(full0 + 8 * s, leader ? 2 : 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int i = 0; i < 2; i++) {
      mbar_init(tfull0 + 8 * i, 1);
      mbar_init(tempty0 + 8 * i, 2 * P_EPI_WARPS);  // on rank 0: every epilogue warp of the pair
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_skip = *(volatile int *)P.err != 0;
  }
  if (warp == P_EPI_WARPS + 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TALLOC));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
  }
  tc_fence_before();
  pr::cluster_sync();
  tc_fence_after();
  if (threadIdx.x == 0) s_skip_pair = s_skip | pr::ld_cluster(pr::map_to(smem_u32(&s_skip), peer));
  __syncthreads();
  const uint32_t tmem = *tmem_slot;
  const int cid = (int)(blockIdx.x >> 1), ncl = (int)(gridDim.x >> 1);
  const int first = s_skip_pair ? ntiles : cid;
  // pair tile t: column tile fastest, then pair of row tiles, then batch x K split
  auto decode = [&](int t, int &n0, int &m0, int &b, int &kb0, int &nkb) {
    const int nt = t % ntn, r = t / ntn, mp = r % ntmp, z = r / ntmp;
    b = z / P.ksplit;
    const int ks = z - b * P.ksplit;
    n0 = nt * BN;
    m0 = (2 * mp + (int)(rank & 1u)) * BM;
    kb0 = ks * P.kb_per_split;
    nkb = max(0, min(P.kblocks, kb0 + P.kb_per_split) - kb0);
  };

  if (warp == P_EPI_WARPS && lane == 0) {
    // ---- TMA producer (both CTAs)
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmB) : "memory");
    int g = 0;
    bool stop = false;
    for (int t = first; t < ntiles && !stop; t += ncl) {
      int n0, m0, b, kb0, nkb;
      decode(t, n0, m0, b, kb0, nkb);
      const int ab = P.a_nb > 1 ? P.a_b0 + b : 0, bb = P.b_nb > 1 ? P.b_b0 + b : 0;
      const int nb0 = P.fuse ? n0 : n0 + (int)(rank & 1u) * (BN / 2);
      for (int it = 0; it < nkb; it++) {
        const int s = g % STAGES;
        const uint32_t ph = (uint32_t)(g / STAGES) & 1u;
        if (g >= STAGES && !mbar_wait(empty0 + 8 * s, ph ^ 1u, P.err, 1)) {
          stop = true;
          break;
        }
        const uint32_t base = smem_u32(smem + s * P.stage_bytes);
        mbar_expect_tx(full0 + 8 * s, P.stage_bytes);
        const int kb = kb0 + it;
        const uint32_t bbase = base + P.np * P.nA * A_TILE;
        for (int p = 0; p < P.np; p++) {
          for (int i = 0; i < P.nA; i++)
            tma_load_3d(base + (p * P.nA + i) * A_TILE, &tmA, full0 + 8 * s, kb * BKT, m0,
                        (P.a_comp[i] * P.np + p) * P.a_nb + ab);
          if (P.fuse) {
            tma_load_3d(bbase + p * b_bytes, &tmB, full0 + 8 * s, kb * BKT, nb0,
                        (P.b_comp[rank & 1u] * P.np + p) * P.b_nb + bb);
          } else {
            for (int j = 0; j < P.nB; j++)
              tma_load_3d(bbase + (p * P.nB + j) * b_bytes, &tmB, full0 + 8 * s, kb * BKT, nb0,
                          (P.b_comp[j] * P.np + p) * P.b_nb + bb);
          }
        }
        g++;
      }
    }
    for (int j = max(0, g - STAGES); j < g; j++)
      mbar_wait_drain(full0 + 8 * (j % STAGES), (uint32_t)(j / STAGES) & 1u, P.err, 4);
  } else if (warp == P_EPI_WARPS + 1 && lane == 0 && !leader) {
    // ---- rank 1: forward each landed stage to rank 0
    const uint32_t lfull0 = pr::map_to(full0, lead);
    int g = 0;
    bool stop = false;
    for (int t = first; t < ntiles && !stop; t += ncl) {
      int n0, m0, b, kb0, nkb;
      decode(t, n0, m0, b, kb0, nkb);
      for (int it = 0; it < nkb; it++, g++) {
        const int s = g % STAGES;
        if (!mbar_wait(full0 + 8 * s, (uint32_t)(g / STAGES) & 1u, P.err, 2)) {
          stop = true;
          break;
        }
        pr::arrive_remote(lfull0 + 8 * s);
      }
    }
  } else if (warp == P_EPI_WARPS + 1 && lane == 0) {
    // ---- rank 0: MMA issuer for the pair
    int g = 0, lt = 0;
    bool stop = false;
    for (int t = first; t < ntiles && !stop; t += ncl, lt++) {
      int n0, m0, b, kb0, nkb;
      decode(t, n0, m0, b, kb0, nkb);
      const int bi = lt & 1;
      const uint32_t tacc = tmem + (uint32_t)bi * TCOLS;
      if (lt >= 2 && !mbar_wait(tempty0 + 8 * bi, (uint32_t)((lt >> 1) - 1) & 1u, P.err, 5)) break;
      tc_fence_after();
      bool started0 = false, started1 = false;
      for (int it = 0; it < nkb; it++) {
        const int s = g % STAGES;
        const uint32_t ph = (uint32_t)(g / STAGES) & 1u;
        if (!mbar_wait(full0 + 8 * s, ph, P.err, 2)) {
          stop = true;
          break;
        }
        tc_fence_after();
        const uint32_t base = smem_u32(smem + s * P.stage_bytes);
        const uint32_t bbase = base + P.np * P.nA * A_TILE;
        for (int pr_ = 0; pr_ < P.nprod; pr_++) {
          const int sa0 = P.pa[pr_] * P.nA;
          if (P.fuse) {
            const uint64_t da = op_desc<BKT>(base + sa0 * A_TILE);
            const uint64_t db = op_desc<BKT>(bbase + P.pb[pr_] * b_bytes);
#pragma unroll
            for (int k = 0; k < BKT / 16; k++)
              pr::mma2(tacc, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), IDESC2, (started0 || k > 0) ? 1u : 0u);
            started0 = started1 = true;
            continue;
          }
          const int sb0 = P.pb[pr_] * P.nB;
          for (int q = 0; q < P.nmma; q++) {
            const Mma mq = P.mma[q];
            const uint64_t da = op_desc<BKT>(base + (sa0 + mq.sa) * A_TILE);
            const uint64_t db = op_desc<BKT>(bbase + (sb0 + mq.sb) * b_bytes);
            const uint32_t idesc = IDESC | (mq.neg ? (1u << 13) : 0u);
            const uint32_t ta = tacc + (uint32_t)(mq.acc * BN);
#pragma unroll
            for (int k = 0; k < BKT / 16; k++)
              pr::mma2(ta, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), idesc,
                       ((mq.acc ? started1 : started0) || k > 0) ? 1u : 0u);
            if (mq.acc)
              started1 = true;
            else
              started0 = true;
          }
        }
        pr::commit2(empty0 + 8 * s, mask);
        g++;
      }
      if (stop) break;
      pr::commit2(tfull0 + 8 * bi, mask);
    }
    // every MMA issued has finished before either CTA releases TMEM or shared memory
    pr::commit2(done, mask);
    mbar_wait_drain(done, 0, P.err, 3);
  } else if (warp < P_EPI_WARPS) {
    // ---- epilogue (both CTAs): this CTA's 128 rows of tile lt from accumulator lt & 1,
    // then release the accumulator on rank 0
    const int q = warp & 3, c_lo = (warp >> 2) * (BN / 2);
    const uint32_t tempty_l = pr::map_to(tempty0, lead);
    int lt = 0;
    for (int t = first; t < ntiles; t += ncl, lt++) {
      int n0, m0, b, kb0, nkb;
      decode(t, n0, m0, b, kb0, nkb);
      const int bi = lt & 1;
      int okl = 0;
      if (lane == 0) okl = mbar_wait(tfull0 + 8 * bi, (uint32_t)(lt >> 1) & 1u, P.err, 3) ? 1 : 0;
      __syncwarp();
      if (!__shfl_sync(0xffffffffu, okl, 0)) break;
      tc_fence_after();
      epilogue_tile<BN>(P, m0, n0, b, q, lane, tmem + (uint32_t)bi * TCOLS, nkb == 0, epi + warp * PIECE_WARP_BYTES,
                        c_lo, c_lo + BN / 2);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) pr::arrive_remote(tempty_l + 8 * bi);
    }
  }
  tc_fence_before();
  __syncthreads();
  pr::cluster_sync();  // neither CTA releases TMEM or exits while the other still works
  if (warp == P_EPI_WARPS + 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TALLOC));
  }
}

// ---------------------------------------------------------------------------------
__global__ void split_pieces_kernel(int rows, int K, int kpad, int nb, int cplx, int np, const double *in, View v,
                                    double conj_sign, __nv_bfloat16 *out, i64 plane) {
  const i64 tot = (i64)nb * rows * kpad;
  for (i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x; idx < tot; idx += (i64)gridDim.x * blockDim.x) {
    const int k = (int)(idx % kpad);
    const i64 rb = idx / kpad;
    const int r = (int)(rb % rows), b = (int)(rb / rows);
    double x[2] = {0.0, 0.0};
    if (k < K) {
      const i64 off = (v.rdiv ? (i64)(r / v.rdiv) * v.rs_hi + (i64)(r % v.rdiv) * v.rs_lo : (i64)r * v.rs_lo) +
                      (v.cdiv ? (i64)(k / v.cdiv) * v.cs_hi + (i64)(k % v.cdiv) * v.cs_lo : (i64)k * v.cs_lo) +
                      (i64)b * v.bs1;
      if (cplx) {
        const double2 z = ((const double2 *)in)[off];
        x[0] = z.x;
        x[1] = conj_sign * z.y;
      } else {
        x[0] = in[off];
      }
    }
    for (int c = 0; c < (cplx ? 2 : 1); c++) {
      double r0 = x[c];
      for (int p = 0; p < np; p++) {
        const __nv_bfloat16 h = __double2bfloat16(r0);
        out[(i64)(c * np + p) * plane + idx] = h;
        r0 -= (double)__bfloat162float(h);
      }
    }
  }
}

typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    NEDY_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    NEDY_REQUIRE(q == cudaDriverEntryPointSuccess && p, "cuTensorMapEncodeTiled is not available");
    fn = (EncodeTiled)p;
  }
  return fn;
}

CUtensorMap make_map(const Pieces &x, int box_rows, int bk) {
  NEDY_REQUIRE(x.p && x.kpad % 64 == 0 && x.rows > 0, "split gemm: bad piece planes");
  NEDY_REQUIRE(((uintptr_t)x.p & 15) == 0, "split gemm: piece planes not 16-byte aligned");
  CUtensorMap m;
  const cuuint64_t dims[3] = {(cuuint64_t)x.kpad, (cuuint64_t)x.rows, (cuuint64_t)x.ncomp * x.np * x.nb};
  const cuuint64_t strides[2] = {(cuuint64_t)x.kpad * 2, (cuuint64_t)x.kpad * 2 * x.rows};
  NEDY_REQUIRE(bk == 64 || bk == 32, "split gemm: K block of 32 or 64");
  const cuuint32_t box[3] = {(cuuint32_t)bk, (cuuint32_t)box_rows, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, (void *)x.p, dims, strides, box, es,
                                 CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 bk == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  NEDY_REQUIRE(r == CUDA_SUCCESS, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return m;
}

// Error word of the split kernels launched on one stream (one per engine context), so
// that a wait that gives up in one context does not stop the work of another.  The word
// is cleared when split_gemm_error reports it.
int *err_word(cudaStream_t s) {
  static std::map<std::pair<int, cudaStream_t>, int *> words;
  static std::mutex mu;
  int dev = 0;
  NEDY_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  int *&w = words[{dev, s}];
  if (!w) {
    NEDY_CUDA(cudaMalloc(&w, sizeof(int)));
    NEDY_CUDA(cudaMemsetAsync(w, 0, sizeof(int), s));
    NEDY_CUDA(cudaStreamSynchronize(s));
  }
  return w;
}

void products(int np, int (&pa)[6], int (&pb)[6], int &n) {
  static const int A3[6] = {0, 0, 1, 0, 1, 2}, B3[6] = {0, 1, 0, 2, 1, 0};
  n = np == 3 ? 6 : np == 2 ? 3 : 1;
  for (int i = 0; i < n; i++) {
    pa[i] = A3[i];
    pb[i] = B3[i];
  }
}

}  // namespace

void split_pieces(const View &v, bool cplx, bool conj, int K, Pieces &out, cudaStream_t s) {
  NEDY_REQUIRE(out.p && out.ncomp == (cplx ? 2 : 1) && out.kpad >= K && out.np >= 1 && out.np <= 3,
               "split_pieces: bad output planes");
  const i64 tot = out.plane();
  const unsigned blocks = (unsigned)std::min<i64>((tot + 255) / 256, 148LL * 16);
  split_pieces_kernel<<<blocks, 256, 0, s>>>(out.rows, K, out.kpad, out.nb, cplx ? 1 : 0, out.np,
                                              (const double *)v.p, v, conj ? -1.0 : 1.0, out.p, out.plane());
  NEDY_CHECK_LAUNCH();
}

// Optional accounting of the split kernels: algorithmic BF16 tensor-pipe FLOPs
// (2 M N K per piece-product term) and device time from events around each launch.
namespace {
std::mutex g_stats_mu;
bool g_stats_on = false;
double g_stats_flops = 0.0;
struct StatEv {
  cudaEvent_t e0, e1;
  std::string cls;  // problem class of the launch
};
std::vector<StatEv> g_stats_ev;
std::map<std::string, std::pair<int, double>> g_class_ms;  // last window: launches, ms per class
}  // namespace

void split_stats(bool on, double *flops, double *ms) {
  std::lock_guard<std::mutex> lk(g_stats_mu);
  double t = 0.0;
  if (!g_stats_ev.empty()) g_class_ms.clear();
  for (auto &e : g_stats_ev) {
    NEDY_CUDA(cudaEventSynchronize(e.e1));
    float x = 0.f;
    NEDY_CUDA(cudaEventElapsedTime(&x, e.e0, e.e1));
    t += x;
    auto &c = g_class_ms[e.cls];
    c.first++;
    c.second += x;
    cudaEventDestroy(e.e0);
    cudaEventDestroy(e.e1);
  }
  g_stats_ev.clear();
  if (flops) *flops = g_stats_flops;
  if (ms) *ms = t;
  g_stats_flops = 0.0;
  g_stats_on = on;
}

template <int BN, int STAGES, int BKT = BK, bool OL = false>
void launch(const Params &P, const CUtensorMap &ma, const CUtensorMap &mb, dim3 grid, cudaStream_t s) {
  static std::atomic<bool> attr[64];  // per device (host threads may race here)
  int dev = 0;
  NEDY_CUDA(cudaGetDevice(&dev));
  NEDY_REQUIRE(dev < 64, "device index out of range");
  const int bytes = smem_bytes(P.stage_bytes, STAGES);
  NEDY_REQUIRE(STAGES * P.stage_bytes <= SMEM_LIMIT, "split_gemm: stages exceed shared memory");
  if (!attr[dev].load()) {
    NEDY_CUDA(cudaFuncSetAttribute(split_gemm_kernel<BN, STAGES, BKT, OL>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes(SMEM_LIMIT / STAGES, STAGES)));
    attr[dev].store(true);
  }
  split_gemm_kernel<BN, STAGES, BKT, OL><<<grid, THREADS, bytes, s>>>(ma, mb, P);
  NEDY_CHECK_LAUNCH();
}

// persistent kernel: one CTA per SM (TMEM holds its two accumulators), at most one per tile
template <int BN, int STAGES, int BKT>
void launch_persist(const Params &P, const CUtensorMap &ma, const CUtensorMap &mb, dim3 grid, cudaStream_t s) {
  static std::atomic<bool> attr[64];  // per device (host threads may race here)
  static std::atomic<int> sms_of[64];
  int dev = 0;
  NEDY_CUDA(cudaGetDevice(&dev));
  NEDY_REQUIRE(dev < 64, "device index out of range");
  const int bytes = psmem_bytes(P.stage_bytes, STAGES);
  NEDY_REQUIRE(STAGES * P.stage_bytes + P_EPI_BYTES <= P_SMEM_LIMIT, "split_gemm: stages exceed shared memory");
  NEDY_REQUIRE(P.out_pieces, "split_gemm: the persistent kernel writes BF16 piece outputs only");
  if (!attr[dev].load()) {
    int sms = 0;
    NEDY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    sms_of[dev].store(sms);
    NEDY_CUDA(cudaFuncSetAttribute(split_gemm_persist_kernel<BN, STAGES, BKT>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, P_SMEM_LIMIT + 1024 + 256));
    attr[dev].store(true);
  }
  const long long ntiles = (long long)grid.x * grid.y * grid.z;
  NEDY_REQUIRE(ntiles < (1LL << 31), "split_gemm: too many tiles");
  const int nct = (int)std::min<long long>(ntiles, std::max(1, sms_of[dev].load()));
  split_gemm_persist_kernel<BN, STAGES, BKT><<<nct, P_THREADS, bytes, s>>>(ma, mb, P, (int)grid.x, (int)grid.y,
                                                                         (int)ntiles);
  NEDY_CHECK_LAUNCH();
}

// persistent CTA-pair kernel: clusters of two CTAs (one per SM), at most one cluster per pair tile
template <int BN, int STAGES, int BKT>
void launch_persist_pair(const Params &P, const CUtensorMap &ma, const CUtensorMap &mb, dim3 grid, cudaStream_t s) {
  static std::atomic<bool> attr[64];  // per device (host threads may race here)
  static std::atomic<int> sms_of[64];
  int dev = 0;
  NEDY_CUDA(cudaGetDevice(&dev));
  NEDY_REQUIRE(dev < 64, "device index out of range");
  NEDY_REQUIRE(grid.y % 2 == 0, "split_gemm: the pair kernel needs an even number of row tiles");
  NEDY_REQUIRE(STAGES * P.stage_bytes + P_EPI_BYTES <= P_SMEM_LIMIT, "split_gemm: stages exceed shared memory");
  NEDY_REQUIRE(P.out_pieces, "split_gemm: the persistent kernels write BF16 piece outputs only");
  if (!attr[dev].load()) {
    int sms = 0;
    NEDY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    sms_of[dev].store(sms);
    NEDY_CUDA(cudaFuncSetAttribute(split_gemm_persist_pair_kernel<BN, STAGES, BKT>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, P_SMEM_LIMIT + 1024 + 256));
    attr[dev].store(true);
  }
  const int ntmp = (int)grid.y / 2;
  const long long ntiles = (long long)grid.x * ntmp * grid.z;
  NEDY_REQUIRE(ntiles < (1LL << 31), "split_gemm: too many tiles");
  const int ncl = (int)std::min<long long>(ntiles, std::max(1, sms_of[dev].load() / 2));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2 * ncl);
  cfg.blockDim = dim3(P_THREADS);
  cfg.dynamicSmemBytes = (size_t)psmem_bytes(P.stage_bytes, STAGES);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  NEDY_CUDA(cudaLaunchKernelEx(&cfg, split_gemm_persist_pair_kernel<BN, STAGES, BKT>, ma, mb, P, (int)grid.x, ntmp,
                               (int)ntiles));
  NEDY_CHECK_LAUNCH();
}

// CTA-pair kernel: grid (column tiles, row tiles, z) of the other kernels launched as
// (row tiles, column tiles, z), clusters of two consecutive row tiles along x (an even count)
template <int BN, int STAGES, int BKT>
void launch_pair(const Params &P, const CUtensorMap &ma, const CUtensorMap &mb, dim3 grid, cudaStream_t s) {
  static std::atomic<bool> attr[64];  // per device (host threads may race here)
  int dev = 0;
  NEDY_CUDA(cudaGetDevice(&dev));
  NEDY_REQUIRE(dev < 64, "device index out of range");
  NEDY_REQUIRE(grid.y % 2 == 0, "split_gemm: the pair kernel needs an even number of row tiles");
  NEDY_REQUIRE(STAGES * P.stage_bytes <= SMEM_LIMIT, "split_gemm: stages exceed shared memory");
  if (!attr[dev].load()) {
    NEDY_CUDA(cudaFuncSetAttribute(split_gemm_pair_kernel<BN, STAGES, BKT>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes(SMEM_LIMIT / STAGES, STAGES)));
    attr[dev].store(true);
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid.y, grid.x, grid.z);
  cfg.blockDim = dim3(THREADS);
  cfg.dynamicSmemBytes = (size_t)smem_bytes(P.stage_bytes, STAGES);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, split_gemm_pair_kernel<BN, STAGES, BKT>, ma, mb, P);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    int nclusters = -1;
    if (cudaOccupancyMaxActiveClusters(&nclusters, split_gemm_pair_kernel<BN, STAGES, BKT>, &cfg) != cudaSuccess)
      (void)cudaGetLastError();
    throw CudaError(std::string("split_gemm pair launch: ") + cudaGetErrorString(e) + " (grid " +
                    std::to_string(cfg.gridDim.x) + "x" + std::to_string(cfg.gridDim.y) + "x" +
                    std::to_string(cfg.gridDim.z) + ", " + std::to_string(cfg.dynamicSmemBytes) +
                    " bytes of shared memory, at most " + std::to_string(nclusters) + " active clusters)");
  }
  NEDY_CHECK_LAUNCH();
}

// ---- autotuner: the tile shape (BN, stages) of each problem class is chosen by timing
// the candidates on the live launches.  Every candidate computes the same result; the
// first launches of a class cycle through the candidates with CUDA events around them,
// and once each has TUNE_TRIALS timings the fastest (device time per batch) is kept.
namespace {
struct Cand {
  int bn, stages, kdiv;  // kdiv: divide the automatic K split by this (FP64-accumulating outputs)
  int bk;                // 0: per-product kernel (64-wide K blocks); 32 / 64: one-load kernel
  int persist = 0;       // 1: persistent one-load kernel (two TMEM accumulators)
  int pair = 0;          // 1: CTA-pair one-load kernel (cta_group::2, 256-row tiles)
};
struct TuneKey {
  int dev, np, nA, nB, out_pieces, acc, M, N, kpad;
  bool operator<(const TuneKey &o) const {
    return std::tie(dev, np, nA, nB, out_pieces, acc, M, N, kpad) <
           std::tie(o.dev, o.np, o.nA, o.nB, o.out_pieces, o.acc, o.M, o.N, o.kpad);
  }
};
struct Pending {
  int c, nb;
  cudaEvent_t e0, e1;
};
struct TuneEntry {
  std::vector<Cand> cands;
  std::vector<double> best;  // ms per batch, min over trials
  std::vector<int> trials, inflight;
  std::vector<Pending> pend;
  int chosen = -1;
};
constexpr int TUNE_TRIALS = 2;
std::mutex g_tune_mu;
std::map<TuneKey, TuneEntry> g_tune;
bool g_tune_on = true;

// shared memory of one stage (a CTA of the pair kernel stages half of the B rows)
int stage_bytes_for(int nA, int nB, int np, int bn, int bk, int pair = 0) {
  if (pair) return np * (nA * BM * bk * 2 + nB * (bn / 2) * bk * 2);
  return bk == 0 ? nA * A_BYTES + nB * bn * BK * 2 : np * (nA * BM * bk * 2 + nB * bn * bk * 2);
}

std::vector<Cand> candidates(int nA, int nB, int np, int N, bool acc, bool pieces) {
  std::vector<Cand> c;
  if (N <= 64 && acc) {  // one output tile per batch: the K split is what there is to tune
    for (int kd : {1, 2, 4, 8}) c.push_back({64, 4, kd, 0});
    for (int kd : {1, 2}) c.push_back({64, 2, kd, 0});  // two CTAs per SM
    return c;
  }
  for (int bn : {64, 128, 256}) {
    if (bn > 64 && N <= 64) continue;    // one 64-wide tile covers the output
    if (bn == 256 && N <= 128) continue;
    const int sb = stage_bytes_for(nA, nB, np, bn, 0);
    const int st = std::min(4, SMEM_LIMIT / sb);
    if (st < 2) continue;
    if (bn == 64) {
      if (st >= 4) c.push_back({64, 4, 1, 0});
      c.push_back({64, 2, 1, 0});  // two CTAs per SM: one's epilogue beside the other's main loop
    } else if (bn == 128) {
      c.push_back({128, 2, 1, 0});
      if (st >= 3) c.push_back({128, std::min(st, 4), 1, 0});
    } else {
      c.push_back({256, std::min(st, 3), 1, 0});
      if (acc) c.push_back({256, std::min(st, 3), 2, 0});
    }
  }
  // one-load kernel: every piece of a K block per stage
  for (int bn : {128, 256}) {
    if (N <= 64 || (bn == 256 && N <= 128)) continue;
    for (int bk : {32, 64}) {
      const int sb = stage_bytes_for(nA, nB, np, bn, bk);
      const int st = std::min(4, SMEM_LIMIT / sb);
      if (st < 2) continue;
      c.push_back({bn, 2, 1, bk});
      if (st >= 3) c.push_back({bn, std::min(st, 4), 1, bk});
      if (acc && bn == 256) c.push_back({bn, 2, 2, bk});
      if (bn == 128 && pieces) {  // persistent: the epilogue of one tile beside the MMAs of the next
        const int pst = std::min(bk == 32 ? 4 : 2, (P_SMEM_LIMIT - P_EPI_BYTES) / sb);
        if (pst >= 2) c.push_back({bn, pst, 1, bk, 1});
        if (pst >= 4) c.push_back({bn, 3, 1, bk, 1});
        // persistent CTA pairs: each CTA stages half of B (instances: 3-4 stages of 32, 2-3 of 64)
        const int ppst = std::min(bk == 32 ? 4 : 3, (P_SMEM_LIMIT - P_EPI_BYTES) / stage_bytes_for(nA, nB, np, bn, bk, 1));
        if (ppst >= (bk == 32 ? 3 : 2)) c.push_back({bn, ppst, 1, bk, 1, 1});
      }
    }
  }
  // persistent 64-wide tiles for narrow piece outputs: with K often one block, the loads and
  // MMAs of one tile overlap the stores of the previous one only in the persistent kernel
  if (pieces && N <= 64) {
    for (int bk : {32, 64}) {
      const int pst = std::min(bk == 32 ? 4 : 3, (P_SMEM_LIMIT - P_EPI_BYTES) / stage_bytes_for(nA, nB, np, 64, bk));
      if (pst >= (bk == 32 ? 4 : 2)) c.push_back({64, pst, 1, bk, 1});
    }
  }
  // CTA pairs (complex x complex): 256-row tiles, each CTA staging half of B
  if (nA == 2 && nB == 2) {
    for (int bn : {128, 256}) {
      if (N <= 64 || (bn == 256 && N <= 128)) continue;
      for (int bk : {32, 64}) {
        const int sb = stage_bytes_for(nA, nB, np, bn, bk, 1);
        // instances: 128-wide tiles 2-4 stages (K block 32) or 2 (64); 256-wide 2-3 (32)
        const int st = std::min(bn == 256 ? 3 : bk == 64 ? 2 : 4, SMEM_LIMIT / sb);
        if (st < 2 || (bn == 256 && bk == 64)) continue;
        c.push_back({bn, st, 1, bk, 0, 1});
        if (acc && bn == 256) c.push_back({bn, st, 2, bk, 0, 1});
      }
    }
  }
  return c;
}

void poll(TuneEntry &e) {
  for (size_t i = 0; i < e.pend.size();) {
    Pending &q = e.pend[i];
    if (cudaEventQuery(q.e1) != cudaSuccess) {
      cudaGetLastError();  // cudaErrorNotReady is not an error here
      i++;
      continue;
    }
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, q.e0, q.e1) == cudaSuccess) {
      e.best[q.c] = std::min(e.best[q.c], (double)ms / std::max(1, q.nb));
      e.trials[q.c]++;
    } else {
      cudaGetLastError();
    }
    e.inflight[q.c]--;
    cudaEventDestroy(q.e0);
    cudaEventDestroy(q.e1);
    e.pend.erase(e.pend.begin() + i);
  }
  if (e.chosen < 0) {
    bool all = true;
    for (int t : e.trials) all = all && t >= TUNE_TRIALS;
    if (all) e.chosen = (int)(std::min_element(e.best.begin(), e.best.end()) - e.best.begin());
  }
}
}  // namespace

void split_autotune(bool on) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_on = on;
}

int split_tune_pending() {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  int n = 0;
  for (auto &kv : g_tune) {
    poll(kv.second);
    if (kv.second.chosen == -1) n++;
  }
  return n;
}

std::string split_tune_report() {
  std::string r;
  {
    std::lock_guard<std::mutex> lk(g_stats_mu);
    for (auto &kv : g_class_ms) {
      char buf[160];
      snprintf(buf, sizeof(buf), "time %s: %d launches %.2f ms;", kv.first.c_str(), kv.second.first,
               kv.second.second);
      r += buf;
    }
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (auto &kv : g_tune) {
    TuneEntry &e = kv.second;
    poll(e);
    const TuneKey &k = kv.first;
    r += "M=" + std::to_string(k.M) + " N=" + std::to_string(k.N) + " K=" + std::to_string(k.kpad) +
         (k.nA == 2 ? (k.nB == 2 ? " cxc" : " cxr") : " rxc") + (k.out_pieces ? " pieces" : " fp64") + " np=" + std::to_string(k.np) + ":";
    for (size_t i = 0; i < e.cands.size(); i++) {
      char buf[96];
      char ol[16] = "";
      if (e.cands[i].bk)
        snprintf(ol, sizeof(ol), "/ol%d%s%s", e.cands[i].bk, e.cands[i].persist ? "p" : "", e.cands[i].pair ? "x2" : "");
      snprintf(buf, sizeof(buf), " %d/%d/k%d%s=%.1fus%s", e.cands[i].bn, e.cands[i].stages, e.cands[i].kdiv, ol,
               e.trials[i] ? e.best[i] * 1e3 : -1.0, (int)i == e.chosen ? "*" : "");
      r += buf;
    }
    r += ";";
  }
  return r;
}

void split_gemm(const SplitGemmArgs &g, cudaStream_t s) {
  const bool ac = g.A.ncomp == 2, bc = g.B.ncomp == 2;
  NEDY_REQUIRE(ac || bc, "split_gemm: at least one operand must be complex");
  NEDY_REQUIRE(g.A.rows >= g.M && g.B.rows >= g.N && g.A.kpad == g.B.kpad && g.A.kpad >= g.K,
               "split_gemm: operand planes do not match the sizes");
  NEDY_REQUIRE(g.A.np == g.B.np, "split_gemm: operands split into different piece counts");
  NEDY_REQUIRE((g.A.nb == 1 || (g.A.b0 >= 0 && g.A.b0 + g.nb <= g.A.nb)) &&
                   (g.B.nb == 1 || (g.B.b0 >= 0 && g.B.b0 + g.nb <= g.B.nb)),
               "split_gemm: batch range outside the operand planes");
  if (g.M == 0 || g.N == 0 || g.nb == 0) return;
  Params P;
  memset(&P, 0, sizeof(P));
  P.M = g.M;
  P.N = g.N;
  P.nb = g.nb;
  P.a_nb = g.A.nb;
  P.b_nb = g.B.nb;
  P.a_b0 = g.A.b0;
  P.b_b0 = g.B.b0;
  P.np = g.A.np;
  products(g.A.np, P.pa, P.pb, P.nprod);
  const signed char cA = g.conjA ? 1 : 0, cB = g.conjB ? 1 : 0;  // negate the imaginary part
  // tile products of a stage (slots: A re/im, B re/im)
  if (ac && bc) {  // Re = Ar Br - Ai Bi, Im = Ar Bi + Ai Br (with the conjugation signs)
    P.nA = 2; P.nB = 2;
    P.a_comp[0] = 0; P.a_comp[1] = 1; P.b_comp[0] = 0; P.b_comp[1] = 1;
    P.nmma = 4;
    P.mma[0] = Mma{0, 0, 0, 0};
    P.mma[1] = Mma{1, 1, 0, (signed char)(1 ^ cA ^ cB)};
    P.mma[2] = Mma{0, 1, 1, cB};
    P.mma[3] = Mma{1, 0, 1, cA};
  } else if (ac) {  // Re = Ar B, Im = Ai B
    P.nA = 2; P.nB = 1;
    P.a_comp[0] = 0; P.a_comp[1] = 1; P.b_comp[0] = 0;
    P.nmma = 2;
    P.mma[0] = Mma{0, 0, 0, 0};
    P.mma[1] = Mma{1, 0, 1, cA};
  } else {  // Re = A Br, Im = A Bi
    P.nA = 1; P.nB = 2;
    P.a_comp[0] = 0; P.b_comp[0] = 0; P.b_comp[1] = 1;
    P.nmma = 2;
    P.mma[0] = Mma{0, 0, 0, 0};
    P.mma[1] = Mma{0, 1, 1, cB};  // negating A negates the product
  }
  // instance without the autotuner: outputs at most 64 wide use 64-wide tiles; piece
  // outputs 128-wide tiles (two CTAs per SM overlap one CTA's store-heavy epilogue with
  // the other's main loop); FP64 outputs 256-wide tiles; wider tiles take the one-load
  // kernel with 32-wide K blocks and two stages when those fit (the usual choice of the
  // autotuner), else the per-product kernel with as many stages as fit
  int BNsel = g.N <= 64 ? 64 : g.out_pieces ? 128 : 256;
  int STsel = 0;  // 0: as many stages as fit
  int KDsel = 1;
  int BKsel = 0;  // per-product kernel
  int PSsel = 0;  // persistent kernel
  int PRsel = 0;  // CTA-pair kernel
  if (BNsel >= 128 && 2 * stage_bytes_for(P.nA, P.nB, P.np, BNsel, 32) <= SMEM_LIMIT) {
    BKsel = 32;
    STsel = 2;
  }
  int tune_c = -1;
  TuneEntry *te = nullptr;
  int dev = 0;
  NEDY_CUDA(cudaGetDevice(&dev));
  if (g.force_bn > 0) {  // a given instance (the candidate checks of the test suite)
    NEDY_REQUIRE(g.force_bn == 64 || g.force_bn == 128 || g.force_bn == 256, "split_gemm: bad forced tile width");
    NEDY_REQUIRE(g.force_bk == 0 || g.force_bk == 32 || g.force_bk == 64, "split_gemm: bad forced K block");
    NEDY_REQUIRE(g.force_bk == 0 || g.force_bn >= 128 || (g.force_bn == 64 && g.force_persist && !g.force_pair),
                 "split_gemm: the one-load kernel has 128 or 256 wide tiles (64 persistent)");
    NEDY_REQUIRE(g.force_stages >= 2 && g.force_stages <= 4 && g.force_kdiv >= 1, "split_gemm: bad forced stages");
    NEDY_REQUIRE(g.force_bk != 0 || g.force_bn != 64 || g.force_stages == 4 || g.force_stages == 2,
                 "split_gemm: 64-wide tiles use 2 or 4 stages");
    NEDY_REQUIRE(g.force_bk != 0 || g.force_bn != 256 || g.force_stages <= 3, "split_gemm: 256-wide tiles use <= 3 stages");
    NEDY_REQUIRE(!g.force_persist || (g.force_bk != 0 && (g.force_bn == 128 || (g.force_bn == 64 && !g.force_pair)) &&
                                      g.out_pieces),
                 "split_gemm: the persistent kernel is the one-load kernel with 64- or 128-wide tiles and piece outputs");
    NEDY_REQUIRE(!g.force_pair || (g.force_bk != 0 && (g.force_persist ? g.out_pieces : (ac && bc))),
                 "split_gemm: the pair kernels are one-load kernels (complex x complex, or persistent with piece outputs)");
    BNsel = g.force_bn;
    STsel = g.force_stages;
    KDsel = g.force_kdiv;
    BKsel = g.force_bk;
    PSsel = g.force_persist ? 1 : 0;
    PRsel = g.force_pair ? 1 : 0;
  } else {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (g_tune_on) {
      const TuneKey key{dev, P.np, P.nA, P.nB, g.out_pieces ? 1 : 0, g.accumulate ? 1 : g.overwrite ? 2 : 0,
                        g.M, g.N, g.A.kpad};
      auto it = g_tune.find(key);
      if (it == g_tune.end()) {
        TuneEntry e;
        e.cands = candidates(P.nA, P.nB, P.np, g.N, (g.accumulate || g.overwrite) && g.ksplit <= 0, g.out_pieces);
        e.best.assign(e.cands.size(), 1e30);
        e.trials.assign(e.cands.size(), 0);
        e.inflight.assign(e.cands.size(), 0);
        if (e.cands.size() <= 1) e.chosen = e.cands.empty() ? -2 : 0;
        it = g_tune.emplace(key, std::move(e)).first;
      }
      TuneEntry &e = it->second;
      poll(e);
      int c = e.chosen;
      if (c == -1) {  // still tuning: the candidate with the fewest timings so far
        c = 0;
        for (size_t i = 1; i < e.cands.size(); i++)
          if (e.trials[i] + e.inflight[i] < e.trials[c] + e.inflight[c]) c = (int)i;
        tune_c = c;
        te = &e;
      }
      if (c >= 0) {
        BNsel = e.cands[c].bn;
        STsel = e.cands[c].stages;
        KDsel = e.cands[c].kdiv;
        BKsel = e.cands[c].bk;
        PSsel = e.cands[c].persist;
        PRsel = e.cands[c].pair;
      }
    }
  }
  const int bkt = BKsel ? BKsel : BK;
  P.stage_bytes = stage_bytes_for(P.nA, P.nB, P.np, BNsel, BKsel, PRsel);
  // real x complex without conjugation: one N = 2 BN product writes both parts
  P.fuse = (BKsel && !(PRsel && !PSsel) && !ac && bc && !g.conjB && 2 * BNsel <= 256) ? 1 : 0;
  P.kblocks = g.A.kpad / 64;  // 64-wide blocks while the K split is chosen
  // row tiles: an even number for CTA pairs (the rows of a last odd tile are out of range:
  // loaded as zeros, not stored)
  const int ntn = (g.N + BNsel - 1) / BNsel, ntm = (g.M + BM - 1) / BM + (PRsel ? ((g.M + BM - 1) / BM) & 1 : 0);
  // K split: bounded FP32 accumulation length, and enough CTAs for the GPU
  int ksplit = g.ksplit;
  const i64 tiles = (i64)ntm * ntn * g.nb;
  if (ksplit <= 0) {
    ksplit = 1;
    if (g.accumulate || g.overwrite) {
      while (tiles * ksplit < 2 * 148 && P.kblocks / (ksplit * 2) >= 4) ksplit *= 2;
      ksplit = std::max(1, ksplit / KDsel);
      if (g.max_kblocks > 0)
        while ((P.kblocks + ksplit - 1) / ksplit > g.max_kblocks) ksplit++;
    }
  }
  NEDY_REQUIRE(!(g.accumulate && g.overwrite), "split_gemm: accumulate and overwrite exclude each other");
  NEDY_REQUIRE(ksplit == 1 || ((g.accumulate || g.overwrite) && !g.out_pieces),
               "split_gemm: K split needs an accumulating or overwritten FP64 output");
  NEDY_REQUIRE(!g.overwrite || ksplit == 1 || g.zero_elems > 0, "split_gemm: overwrite with a K split needs zero_elems");
  P.ksplit = ksplit;
  // in units of the kernel's K block
  P.kb_per_split = (P.kblocks + ksplit - 1) / ksplit * (64 / bkt);
  P.kblocks *= 64 / bkt;
  NEDY_REQUIRE((i64)g.nb * ksplit <= 65535 && ntm <= 65535, "split_gemm: grid too large");
  P.out_pieces = g.out_pieces ? 1 : 0;
  P.accumulate = g.accumulate ? 1 : 0;  // overwrite without a K split: plain stores
  P.atomic = ksplit > 1 ? 1 : 0;
  P.alpha = g.alpha;
  if (g.out_pieces) {
    NEDY_REQUIRE(g.Cp.p && g.Cp.ncomp == 2 && !g.accumulate && !g.overwrite, "split_gemm: bad piece output");
    P.out = g.Cp.p;
    P.out_np = g.Cp.np;
    P.plane = g.Cp.plane();
  } else {
    NEDY_REQUIRE(g.C.p, "split_gemm: no output");
    P.out = (void *)g.C.p;
  }
  P.rs_hi = g.C.rs_hi;
  P.rs_lo = g.C.rs_lo;
  P.rdiv = g.C.rdiv;
  P.cs_hi = g.C.cs_hi;
  P.cs_lo = g.C.cs_lo;
  P.cdiv = g.C.cdiv;
  P.bs = g.C.bs1;
  P.err = err_word(s);
  // B rows per CTA: half of a tile in CTA pairs, except a fused real x complex product, where
  // each CTA of the pair stages one whole plane tile
  const CUtensorMap ma = make_map(g.A, BM, bkt), mb = make_map(g.B, PRsel && !P.fuse ? BNsel / 2 : BNsel, bkt);
  dim3 grid(ntn, ntm, g.nb * ksplit);
  cudaEvent_t ev[2] = {nullptr, nullptr};
  {
    std::lock_guard<std::mutex> lk(g_stats_mu);
    if (g_stats_on) {
      g_stats_flops += 2.0 * g.M * (double)g.N * g.K * g.nb * P.nprod * P.nmma;
      NEDY_CUDA(cudaEventCreate(&ev[0]));
      NEDY_CUDA(cudaEventCreate(&ev[1]));
      NEDY_CUDA(cudaEventRecord(ev[0], s));
    }
  }
  const int stages = STsel ? STsel : BNsel == 128 ? 2 : std::min(4, SMEM_LIMIT / P.stage_bytes);
  NEDY_REQUIRE(stages >= 2 && (PSsel ? stages * P.stage_bytes + P_EPI_BYTES <= P_SMEM_LIMIT
                                      : stages * P.stage_bytes <= SMEM_LIMIT),
               "split_gemm: stages exceed shared memory");
  cudaEvent_t tev[2] = {nullptr, nullptr};
  if (te) {
    NEDY_CUDA(cudaEventCreate(&tev[0]));
    NEDY_CUDA(cudaEventCreate(&tev[1]));
    NEDY_CUDA(cudaEventRecord(tev[0], s));
  }
  using LaunchFn = void (*)(const Params &, const CUtensorMap &, const CUtensorMap &, dim3, cudaStream_t);
  struct Inst {
    int bk, bn, st;
    LaunchFn fn;
    int persist;
    int pair = 0;
  };
  static const Inst insts[] = {
      {0, 64, 4, launch<64, 4>, 0},       {0, 64, 2, launch<64, 2>, 0},       {0, 128, 2, launch<128, 2>, 0},
      {0, 128, 3, launch<128, 3>, 0},     {0, 128, 4, launch<128, 4>, 0},     {0, 256, 2, launch<256, 2>, 0},
      {0, 256, 3, launch<256, 3>, 0},
      {32, 128, 2, launch<128, 2, 32, true>, 0}, {32, 128, 3, launch<128, 3, 32, true>, 0},
      {32, 128, 4, launch<128, 4, 32, true>, 0}, {32, 256, 2, launch<256, 2, 32, true>, 0},
      {32, 256, 3, launch<256, 3, 32, true>, 0}, {64, 128, 2, launch<128, 2, 64, true>, 0},
      {64, 128, 3, launch<128, 3, 64, true>, 0},
      {32, 128, 2, launch_persist<128, 2, 32>, 1}, {32, 128, 3, launch_persist<128, 3, 32>, 1},
      {32, 128, 4, launch_persist<128, 4, 32>, 1}, {64, 128, 2, launch_persist<128, 2, 64>, 1},
      {32, 64, 4, launch_persist<64, 4, 32>, 1}, {64, 64, 2, launch_persist<64, 2, 64>, 1},
      {64, 64, 3, launch_persist<64, 3, 64>, 1},
      {32, 256, 2, launch_pair<256, 2, 32>, 0, 1}, {32, 256, 3, launch_pair<256, 3, 32>, 0, 1},
      {32, 128, 2, launch_pair<128, 2, 32>, 0, 1}, {32, 128, 3, launch_pair<128, 3, 32>, 0, 1},
      {32, 128, 4, launch_pair<128, 4, 32>, 0, 1},
      {64, 128, 2, launch_pair<128, 2, 64>, 0, 1},
      {32, 128, 3, launch_persist_pair<128, 3, 32>, 1, 1}, {32, 128, 4, launch_persist_pair<128, 4, 32>, 1, 1},
      {64, 128, 2, launch_persist_pair<128, 2, 64>, 1, 1}, {64, 128, 3, launch_persist_pair<128, 3, 64>, 1, 1}};
  int st_run = stages;
  if (BKsel == 0) {  // per-product kernel: the instance nearest to the requested stages
    st_run = BNsel == 64 ? (stages <= 2 ? 2 : 4)
                         : BNsel == 128 ? std::min(std::max(stages, 2), 4) : std::min(std::max(stages, 2), 3);
  }
  LaunchFn fn = nullptr;
  for (const Inst &x : insts)
    if (x.bk == BKsel && x.bn == BNsel && x.st == st_run && x.persist == PSsel && x.pair == PRsel) fn = x.fn;
  NEDY_REQUIRE(fn != nullptr, "split_gemm: no kernel instance for this tile shape");
  if (g.overwrite && ksplit > 1)  // inside the timed region: part of what a K split costs
    NEDY_CUDA(cudaMemsetAsync((void *)g.C.p, 0, sizeof(double2) * (size_t)g.zero_elems, s));
  fn(P, ma, mb, grid, s);
  if (te) {
    NEDY_CUDA(cudaEventRecord(tev[1], s));
    std::lock_guard<std::mutex> lk(g_tune_mu);
    te->pend.push_back({tune_c, g.nb, tev[0], tev[1]});
    te->inflight[tune_c]++;
  }
  if (ev[0]) {
    std::lock_guard<std::mutex> lk(g_stats_mu);
    NEDY_CUDA(cudaEventRecord(ev[1], s));
    char cls[96];
    snprintf(cls, sizeof(cls), "M=%d N=%d K=%d %s %s np=%d", g.M, g.N, g.A.kpad,
             P.nA == 2 ? (P.nB == 2 ? "cxc" : "cxr") : "rxc", g.out_pieces ? "pieces" : "fp64", P.np);
    g_stats_ev.push_back({ev[0], ev[1], cls});
  }
}

// ---- check of one kernel instance against an FP64 product on seeded operands
namespace {
__device__ __forceinline__ double check_uniform(unsigned long long x) {
  // splitmix64 finaliser -> uniform in [-1, 1)
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  x ^= x >> 31;
  return (double)(x >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}
__global__ void check_fill_kernel(i64 n, unsigned long long seed, double *out) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
    out[i] = check_uniform(seed * 0x100000001B3ULL + (unsigned long long)i);
}
// ref[b][m][n] += alpha * sum_k op(A[b][m][k]) op(B[b][n][k]); real operands have one double per element
__global__ void check_ref_kernel(int M, int N, int K, int nb, int ac, int bc, int cA, int cB, const double *A,
                                 const double *B, double alpha, double2 *ref) {
  const i64 tot = (i64)nb * M * N;
  for (i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x; idx < tot; idx += (i64)gridDim.x * blockDim.x) {
    const int n = (int)(idx % N);
    const i64 bm = idx / N;
    const int m = (int)(bm % M), b = (int)(bm / M);
    double re = 0.0, im = 0.0;
    for (int k = 0; k < K; k++) {
      const i64 ia = ((i64)b * M + m) * K + k, ib = ((i64)b * N + n) * K + k;
      const double ar = ac ? A[2 * ia] : A[ia], ai = ac ? (cA ? -A[2 * ia + 1] : A[2 * ia + 1]) : 0.0;
      const double br = bc ? B[2 * ib] : B[ib], bi = bc ? (cB ? -B[2 * ib + 1] : B[2 * ib + 1]) : 0.0;
      re += ar * br - ai * bi;
      im += ar * bi + ai * br;
    }
    ref[idx].x += alpha * re;
    ref[idx].y += alpha * im;
  }
}
// got[b][m][n] = sum of the BF16 pieces of the piece output (planes [comp][piece])
__global__ void check_unpieces_kernel(int M, int N, int nb, int kpad, int np, i64 plane, const __nv_bfloat16 *cp,
                                      double2 *got) {
  const i64 tot = (i64)nb * M * N;
  for (i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x; idx < tot; idx += (i64)gridDim.x * blockDim.x) {
    const int n = (int)(idx % N);
    const i64 bm = idx / N;
    const i64 off = bm * kpad + n;
    double v[2] = {0.0, 0.0};
    for (int c = 0; c < 2; c++)
      for (int p = 0; p < np; p++) v[c] += (double)__bfloat162float(cp[(i64)(c * np + p) * plane + off]);
    got[idx] = make_double2(v[0], v[1]);
  }
}
// maxima of |got - ref| and |ref| as ordered bit patterns of non-negative doubles
__global__ void check_err_kernel(i64 n, const double2 *ref, const double2 *got, unsigned long long *mx) {
  unsigned long long d = 0, r = 0;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    const double dd = fmax(fabs(got[i].x - ref[i].x), fabs(got[i].y - ref[i].y));
    const double rr = fmax(fabs(ref[i].x), fabs(ref[i].y));
    d = max(d, (unsigned long long)__double_as_longlong(dd));
    r = max(r, (unsigned long long)__double_as_longlong(rr));
  }
  atomicMax(&mx[0], d);
  atomicMax(&mx[1], r);
}
}  // namespace

double split_gemm_check(const SplitCheck &k, cudaStream_t s) {
  NEDY_REQUIRE(k.M > 0 && k.N > 0 && k.K > 0 && k.nb > 0 && (k.a_cplx || k.b_cplx) && k.np >= 1 && k.np <= 3,
               "split_gemm_check: bad sizes");
  NEDY_REQUIRE((i64)k.nb * k.M * k.N <= (1LL << 24) && (i64)k.nb * (k.M + k.N) * k.K <= (1LL << 26),
               "split_gemm_check: sizes too large for the check");
  std::vector<void *> held;
  auto dalloc = [&](size_t bytes) {
    void *p = nullptr;
    NEDY_CUDA(cudaMalloc(&p, bytes));
    held.push_back(p);
    return p;
  };
  double result = 0.0;
  try {
    const int ca = k.a_cplx ? 2 : 1, cb = k.b_cplx ? 2 : 1;
    const i64 na = (i64)k.nb * k.M * k.K * ca, nbv = (i64)k.nb * k.N * k.K * cb, nc = (i64)k.nb * k.M * k.N;
    double *A = (double *)dalloc(sizeof(double) * na), *B = (double *)dalloc(sizeof(double) * nbv);
    double2 *C = (double2 *)dalloc(sizeof(double2) * nc), *ref = (double2 *)dalloc(sizeof(double2) * nc);
    check_fill_kernel<<<592, 256, 0, s>>>(na, k.seed * 3 + 1, A);
    check_fill_kernel<<<592, 256, 0, s>>>(nbv, k.seed * 3 + 2, B);
    // accumulate 1: C += ...; 2: overwrite (C holds values that must not be read)
    if (k.accumulate)
      check_fill_kernel<<<592, 256, 0, s>>>(2 * nc, k.seed * 3 + 3, (double *)C);
    else
      NEDY_CUDA(cudaMemsetAsync(C, 0, sizeof(double2) * nc, s));
    if (k.accumulate == 2)
      NEDY_CUDA(cudaMemsetAsync(ref, 0, sizeof(double2) * nc, s));
    else
      NEDY_CUDA(cudaMemcpyAsync(ref, C, sizeof(double2) * nc, cudaMemcpyDeviceToDevice, s));
    NEDY_CHECK_LAUNCH();
    check_ref_kernel<<<592, 256, 0, s>>>(k.M, k.N, k.K, k.nb, k.a_cplx, k.b_cplx, k.conjA, k.conjB, A, B, k.alpha,
                                         ref);
    NEDY_CHECK_LAUNCH();
    Pieces ap, bp;
    ap.rows = k.M; ap.kpad = kpad64(k.K); ap.nb = k.nb; ap.ncomp = ca; ap.np = k.np;
    bp.rows = k.N; bp.kpad = ap.kpad; bp.nb = k.nb; bp.ncomp = cb; bp.np = k.np;
    ap.p = (__nv_bfloat16 *)dalloc(ap.elems() * 2);
    bp.p = (__nv_bfloat16 *)dalloc(bp.elems() * 2);
    View va = rowmajor(A, k.K); va.bs1 = (i64)k.M * k.K;
    View vb = rowmajor(B, k.K); vb.bs1 = (i64)k.N * k.K;
    split_pieces(va, k.a_cplx != 0, false, k.K, ap, s);
    split_pieces(vb, k.b_cplx != 0, false, k.K, bp, s);
    SplitGemmArgs g;
    g.M = k.M; g.N = k.N; g.K = k.K; g.nb = k.nb;
    g.A = ap; g.B = bp;
    g.conjA = k.conjA != 0; g.conjB = k.conjB != 0;
    g.alpha = k.alpha;
    g.force_bn = k.bn; g.force_stages = k.stages; g.force_bk = k.bk; g.force_kdiv = k.kdiv;
    g.force_persist = k.persist == 1 || k.persist == 3;
    g.force_pair = k.persist == 2 || k.persist == 3;
    double2 *got = C;
    if (k.out_pieces) {
      Pieces cp;
      cp.rows = k.M; cp.kpad = kpad64(k.N); cp.nb = k.nb; cp.ncomp = 2; cp.np = k.np;
      cp.p = (__nv_bfloat16 *)dalloc(cp.elems() * 2);
      NEDY_CUDA(cudaMemsetAsync(cp.p, 0, cp.elems() * 2, s));
      g.out_pieces = true;
      g.Cp = cp;
      g.C.rs_lo = cp.kpad; g.C.cs_lo = 1; g.C.bs1 = (i64)k.M * cp.kpad;
      split_gemm(g, s);
      check_unpieces_kernel<<<592, 256, 0, s>>>(k.M, k.N, k.nb, cp.kpad, k.np, cp.plane(), cp.p, C);
      NEDY_CHECK_LAUNCH();
    } else {
      g.C = rowmajor(C, k.N); g.C.bs1 = (i64)k.M * k.N;
      g.accumulate = k.accumulate == 1;
      g.overwrite = k.accumulate == 2;
      g.zero_elems = nc;
      split_gemm(g, s);
    }
    unsigned long long *mx = (unsigned long long *)dalloc(2 * sizeof(unsigned long long));
    NEDY_CUDA(cudaMemsetAsync(mx, 0, 2 * sizeof(unsigned long long), s));
    check_err_kernel<<<592, 256, 0, s>>>(nc, ref, got, mx);
    NEDY_CHECK_LAUNCH();
    unsigned long long h[2] = {0, 0};
    NEDY_CUDA(cudaMemcpyAsync(h, mx, sizeof(h), cudaMemcpyDeviceToHost, s));
    NEDY_CUDA(cudaStreamSynchronize(s));
    if (split_gemm_error(s) != 0)  // NEDY_ERR_TIMEOUT at the C ABI, not an absent instance
      throw CudaError("split_gemm_check: a bounded device wait timed out");
    double d, r;
    memcpy(&d, &h[0], 8);
    memcpy(&r, &h[1], 8);
    result = d / (r > 0 ? r : 1.0);
  } catch (...) {
    cudaStreamSynchronize(s);
    for (void *p : held) cudaFree(p);
    throw;
  }
  for (void *p : held) cudaFree(p);
  return result;
}

int split_gemm_error(cudaStream_t s) {
  int *w = err_word(s);
  int h = 0;
  NEDY_CUDA(cudaMemcpyAsync(&h, w, sizeof(int), cudaMemcpyDeviceToHost, s));
  NEDY_CUDA(cudaStreamSynchronize(s));
  if (h != 0) {  // reported once: the next launch on this stream starts clean
    NEDY_CUDA(cudaMemsetAsync(w, 0, sizeof(int), s));
    NEDY_CUDA(cudaStreamSynchronize(s));
  }
  return h;
}

void split_gemm_set_error(cudaStream_t s, int code) {
  int *w = err_word(s);
  NEDY_CUDA(cudaMemcpyAsync(w, &code, sizeof(int), cudaMemcpyHostToDevice, s));
  NEDY_CUDA(cudaStreamSynchronize(s));
}

}  // namespace nedy
