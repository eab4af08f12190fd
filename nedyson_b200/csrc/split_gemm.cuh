// Split-precision GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// An FP64 operand x is held as BF16 pieces x = x0 + x1 + x2 (+ O(2^-24 |x|)),
// each piece the BF16 rounding of what the previous ones left over.  A product
// a*b is then the sum of the piece products a_i b_j with i + j < npieces (6
// products for 3 pieces, 3 for 2), which the tensor cores form exactly and
// accumulate in FP32 in tensor memory.  Complex operands are separate real and
// imaginary piece planes; one output tile holds both parts (two TMEM
// accumulators), so a complex x complex product is 4 real BF16 GEMMs per piece
// product, a real x complex one 2.
//
// Storage of an operand ("piece planes"): BF16, [comp][piece][batch][row][kpad],
// K contiguous and padded with zeros to kpad, a multiple of 64 (one 128-byte
// swizzle atom).  A is M x K (rows = M), B is N x K (rows = N): C = A * B^T.
#pragma once
#include "common.cuh"
#include "gemm_f64.cuh"
#include <cuda_bf16.h>
#include <string>

namespace nedy {

struct Pieces {
  __nv_bfloat16 *p = nullptr;
  int rows = 0, kpad = 0, nb = 1;  // nb = 1 with a batched GEMM: shared by every batch
  int ncomp = 1, np = 3;           // ncomp 2: complex (re plane group, then im)
  int b0 = 0;                      // first stored batch a batched GEMM uses (nb > 1)
  i64 plane() const { return (i64)nb * rows * kpad; }
  i64 elems() const { return plane() * ncomp * np; }
};

inline int kpad64(int k) { return (k + 63) / 64 * 64; }

// FP64 (complex or real) matrix rows x K, read through a View (units: complex or
// real elements), batch b at b * v.bs1  ->  piece planes (allocated by the caller,
// rows/kpad/nb/ncomp/np set).  conj negates the imaginary part.
void split_pieces(const View &v, bool cplx, bool conj, int K, Pieces &out, cudaStream_t s);

struct SplitGemmArgs {
  int M = 0, N = 0, K = 0, nb = 1;  // C[b] (M x N) = alpha * A[b] (M x K) * B[b]^T (+ C[b])
  Pieces A, B;                       // complex when ncomp == 2; at least one is complex
  bool conjA = false, conjB = false;
  double alpha = 1.0;
  // output: FP64 complex through a View (units: complex elements), or BF16 pieces
  bool out_pieces = false;
  View C;                 // FP64 output (C.bs1 = batch stride); element offsets for pieces
  Pieces Cp;              // piece output: planes [comp][piece] of Cp.plane() elements, offsets from C
  bool accumulate = false;  // FP64 output only: C += alpha * A B^T
  // FP64 output only: C = alpha * A B^T replaces the old contents, which are not read.
  // Without a K split every element is stored once; with one, the first zero_elems complex
  // elements from C.p (the whole output range) are cleared on the stream first and the
  // partial sums are added atomically.
  bool overwrite = false;
  i64 zero_elems = 0;
  int ksplit = 0;           // 0: choose; > 1 needs accumulate or overwrite (FP64 atomics)
  int max_kblocks = 0;      // upper bound on 64-wide K blocks accumulated in FP32 per tile (0: none)
  // a given kernel instance instead of the autotuner's (force_bn 0: autotuner); force_bk 0
  // is the per-product kernel, 32 / 64 the one-load kernel with that K block
  int force_bn = 0, force_stages = 0, force_bk = 0, force_kdiv = 1;
  int force_persist = 0;  // with force_bn: the persistent one-load kernel (force_bk 32 / 64, force_bn 128)
  int force_pair = 0;     // with force_bn: the CTA-pair one-load kernel (complex x complex)
};

void split_gemm(const SplitGemmArgs &g, cudaStream_t s);

// One kernel instance (tile width bn, stages, K block bk: 0 per-product kernel, 32 / 64
// one-load kernel; kdiv as in the autotuner) on seeded uniform operands: returns
// max |split - FP64| / max |FP64| over the output (piece outputs summed back).
struct SplitCheck {
  int M = 0, N = 0, K = 0, nb = 1;
  int a_cplx = 1, b_cplx = 1, conjA = 0, conjB = 0, np = 3, out_pieces = 0, accumulate = 0;
  int bn = 128, stages = 2, bk = 0, kdiv = 1, persist = 0;  // persist 1: persistent kernel, 2: CTA pair, 3: both
  double alpha = 1.0;
  unsigned long long seed = 1;
};
double split_gemm_check(const SplitCheck &k, cudaStream_t s);

// Accounting of split kernel launches: returns the algorithmic BF16 tensor-pipe FLOPs and
// the summed device time (ms) since the last call, then turns the accounting on or off.
void split_stats(bool on, double *flops, double *ms);

// Autotuner of the tile shapes (on by default): each problem class (operand kinds, output
// kind, M, N, padded K) tries its candidate shapes on its first launches and keeps the
// fastest.  split_tune_report lists the classes, candidate timings and choices.
void split_autotune(bool on);
std::string split_tune_report();
// problem classes whose candidates are still being timed
int split_tune_pending();

// Error word of the split kernels launched on stream s: non-zero after a bounded wait gave
// up (1 producer, 2 MMA issuer, 3 epilogue, 4 drain); reading a non-zero word clears it.
// While it is set, the CTAs of later launches on s skip their work.
int split_gemm_error(cudaStream_t s);
// Test hook: preset the error word of stream s (CTAs then skip, as after a timeout).
void split_gemm_set_error(cudaStream_t s, int code);

}  // namespace nedy
