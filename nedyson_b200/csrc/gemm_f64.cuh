// Batched FP64 / complex128 GEMM on the FP64 tensor pipe (DMMA, mma.sync m8n8k4).
//
// Blackwell's tcgen05 tensor core has no FP64 kind, so FP64 contractions run on
// the DMMA path.  One kernel covers every FP64 contraction of the GF2 hot path:
// operands are described by "strided views" whose row, column and batch indices
// may each be split in two levels (idx -> (idx / div) * s_hi + (idx % div) * s_lo).
// That expresses the packed block layouts of the Green's functions directly
// (e.g. a row of G^tv(t, tau) blocks seen as one nao x (ntau+1)*nao matrix), so
// no operand is ever repacked in HBM.
//
// C[b] (M x N, complex) = alpha * opA(A[b]) (M x K) * opB(B[b]) (K x N) + beta * C[b]
// A and B are real (double) or complex (double2); C is complex.
#pragma once
#include "common.cuh"

namespace nedy {

struct View {
  const void *p = nullptr;
  i64 rs_hi = 0, rs_lo = 0;  // row r -> (r / rdiv) * rs_hi + (r % rdiv) * rs_lo   (rdiv == 0: r * rs_lo)
  int rdiv = 0;
  i64 cs_hi = 0, cs_lo = 0;  // col c -> (c / cdiv) * cs_hi + (c % cdiv) * cs_lo
  int cdiv = 0;
  i64 bs1 = 0, bs2 = 0;      // batch (b1, b2) -> b1 * bs1 + b2 * bs2
};

// Plain row-major matrix with leading dimension ld.
inline View rowmajor(const void *p, i64 ld) {
  View v;
  v.p = p;
  v.rs_lo = ld;
  v.cs_lo = 1;
  return v;
}
// Transposed view of a row-major matrix with leading dimension ld (element (r,c) = M[c][r]).
inline View transposed(const void *p, i64 ld) {
  View v;
  v.p = p;
  v.rs_lo = 1;
  v.cs_lo = ld;
  return v;
}

struct GemmArgs {
  int M = 0, N = 0, K = 0, nb1 = 1, nb2 = 1;
  View A, B, C;
  bool a_cplx = true, b_cplx = true;
  bool conjA = false, conjB = false;
  double2 alpha = {1.0, 0.0}, beta = {0.0, 0.0};
  const double *kscale = nullptr;  // optional: A(:, k) *= kscale[b1 * kscale_bs1 + k / kdiv]
  int kdiv = 1;
  i64 kscale_bs1 = 0;
  // grouped mode (all optional, device arrays indexed by b1):
  const i64 *goffA = nullptr, *goffB = nullptr, *goffC = nullptr;  // extra element offsets
  const int *gM = nullptr, *gK = nullptr;                           // per-group M and K (<= M, K)
  const double *bscale = nullptr;                                   // per-group real factor on alpha
  bool atomic = false;  // epilogue C += alpha * acc with atomics (beta must be 0 or 1; C pre-set)
};

// Launch on `stream`.  Throws on bad arguments.
void gemm(const GemmArgs &g, cudaStream_t stream);

} // namespace nedy
