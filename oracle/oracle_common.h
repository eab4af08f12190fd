// CPU oracle for the GF2 Kadanoff-Baym hot path: shared types and dense
// linear-algebra helpers.
//
// TEST INFRASTRUCTURE ONLY.  This directory is a plain C++ restatement of the
// reference solver (tblommel/NEdyson) used as the parity checker for the CUDA
// path and as the timed CPU baseline.  Nothing in the product library links,
// loads or calls it.
//
// Storage conventions follow src/greens.h / src/greens.cpp of the reference:
//   les  : upper triangle, block (i,j) with i<=j at index j(j+1)/2+i   (greens.cpp:177-180)
//   ret  : lower triangle, block (i,j) with j<=i at index i(i+1)/2+j   (greens.cpp:182-185)
//   tv   : block (i,m) at index i*(ntau+1)+m                            (greens.cpp:187-190)
//   mat  : block m                                                       (greens.cpp:192-195)
// Every block is an nao x nao row-major complex<double> matrix (utils.h:49-50).
// Indices are 64-bit here (the reference uses int, which overflows at large nt).
#pragma once
#include <complex>
#include <vector>
#include <cstdint>
#include <cstring>
#include <cmath>
#include <cassert>

namespace orc {

using cplx = std::complex<double>;
using i64 = int64_t;

// Plain-C view of one contour Green's function (mirrors green_func, greens.h:17-112).
struct GF {
  int nt, ntau, nao, sig;
  cplx *les, *ret, *tv, *mat;
  i64 es() const { return (i64)nao * nao; }
  cplx *lesptr(i64 i, i64 j) const { assert(i >= 0 && i <= j && j <= nt); return les + ((j * (j + 1)) / 2 + i) * es(); }
  cplx *retptr(i64 i, i64 j) const { assert(j >= 0 && j <= i && i <= nt); return ret + ((i * (i + 1)) / 2 + j) * es(); }
  cplx *tvptr(i64 i, i64 m) const { assert(i >= 0 && i <= nt && m >= 0 && m <= ntau); return tv + (i * (ntau + 1) + m) * es(); }
  cplx *matptr(i64 m) const { assert(m >= 0 && m <= ntau); return mat + m * es(); }
  // greens.h:76-86
  void set_tstp_zero(int tstp) const {
    if (tstp == -1) { std::memset((void*)matptr(0), 0, sizeof(cplx) * (ntau + 1) * es()); return; }
    std::memset((void*)retptr(tstp, 0), 0, sizeof(cplx) * (tstp + 1) * es());
    std::memset((void*)lesptr(0, tstp), 0, sizeof(cplx) * (tstp + 1) * es());
    std::memset((void*)tvptr(tstp, 0), 0, sizeof(cplx) * (ntau + 1) * es());
  }
  // greens.h:68-74 : rho = i*sig*G^<(t,t), or -G^M(beta) for t=-1
  void get_dm(int t, cplx *rho) const {
    if (t == -1) { for (i64 e = 0; e < es(); e++) rho[e] = -matptr(ntau)[e]; return; }
    cplx f(0.0, (double)sig);
    for (i64 e = 0; e < es(); e++) rho[e] = f * lesptr(t, t)[e];
  }
};

// ---------------------------------------------------------------------------
// BLAS shim.  When a CBLAS library has been registered (orc_set_blas), the
// large products go through its dgemm/zgemm; otherwise through plain loops.
// ---------------------------------------------------------------------------
enum Op { N = 0, T = 1, C = 2 };

void set_blas(const char *path, int threads);
bool have_blas();

// C[M x Nn] = alpha * op(A) * op(B) + beta * C   (row-major, complex)
void zgemm(Op oa, Op ob, int M, int Nn, int K, cplx alpha, const cplx *A, int lda,
           const cplx *B, int ldb, cplx beta, cplx *C, int ldc);
// C[M x Nn] (complex) = alpha * R[M x K] (real) * Z[K x Nn] (complex) + beta * C   (row-major)
void rzgemm(int M, int Nn, int K, double alpha, const double *R, int ldr,
            const cplx *Z, int ldz, double beta, cplx *C, int ldc);
// C[M x Nn] (real) = alpha * op(A) * op(B) + beta * C   (row-major, real)
void dgemm(Op oa, Op ob, int M, int Nn, int K, double alpha, const double *A, int lda,
           const double *B, int ldb, double beta, double *C, int ldc);

// Dense helpers on n x n row-major complex matrices.
void lu_solve(int n, int nrhs, cplx *A, cplx *B);           // A X = B, B overwritten by X (A destroyed)
void lu_solve_right(int n, int nrows, const cplx *A, cplx *B); // X A = B, B (nrows x n) overwritten by X
void herm_eig(int n, const cplx *A, double *evals, cplx *evecs); // ascending eigenvalues, evecs columns
double fro_norm(i64 n, const cplx *A);

} // namespace orc
