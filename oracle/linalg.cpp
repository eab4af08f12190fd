// CPU oracle (test infrastructure): BLAS shim and dense helpers.
// See oracle_common.h for the storage conventions.
#include "oracle_common.h"
#include <dlfcn.h>
#include <algorithm>
#include <stdexcept>

namespace orc {

namespace {
enum { RowMajor = 101, NoTrans = 111, Trans = 112, ConjTrans = 113 };
typedef void (*zgemm_t)(int, int, int, int, int, int, const void *, const void *, int,
                        const void *, int, const void *, void *, int);
typedef void (*dgemm_t)(int, int, int, int, int, int, double, const double *, int,
                        const double *, int, double, double *, int);
typedef void (*setthr_t)(int);
zgemm_t g_zgemm = nullptr;
dgemm_t g_dgemm = nullptr;

int cb(Op o) { return o == N ? NoTrans : (o == T ? Trans : ConjTrans); }

inline cplx opget(Op o, const cplx *A, int ld, int r, int c) {
  // element (r,c) of op(A)
  if (o == N) return A[(i64)r * ld + c];
  if (o == T) return A[(i64)c * ld + r];
  return std::conj(A[(i64)c * ld + r]);
}
} // namespace

void set_blas(const char *path, int threads) {
  void *h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) throw std::runtime_error(std::string("oracle: cannot load BLAS ") + path);
  // The scipy-bundled OpenBLAS prefixes its CBLAS symbols with "scipy_".
  const char *zn[] = {"scipy_cblas_zgemm", "cblas_zgemm"};
  const char *dn[] = {"scipy_cblas_dgemm", "cblas_dgemm"};
  const char *tn[] = {"scipy_openblas_set_num_threads", "openblas_set_num_threads"};
  for (auto n : zn) if (!g_zgemm) g_zgemm = (zgemm_t)dlsym(h, n);
  for (auto n : dn) if (!g_dgemm) g_dgemm = (dgemm_t)dlsym(h, n);
  setthr_t st = nullptr;
  for (auto n : tn) if (!st) st = (setthr_t)dlsym(h, n);
  if (st && threads > 0) st(threads);
  if (!g_zgemm || !g_dgemm) throw std::runtime_error("oracle: BLAS symbols missing");
}

bool have_blas() { return g_zgemm != nullptr; }

void zgemm(Op oa, Op ob, int M, int Nn, int K, cplx alpha, const cplx *A, int lda,
           const cplx *B, int ldb, cplx beta, cplx *C, int ldc) {
  if (M <= 0 || Nn <= 0) return;
  if (g_zgemm && K > 0) {
    g_zgemm(RowMajor, cb(oa), cb(ob), M, Nn, K, &alpha, A, lda, B, ldb, &beta, C, ldc);
    return;
  }
  for (int i = 0; i < M; i++)
    for (int j = 0; j < Nn; j++) {
      cplx s = 0;
      for (int k = 0; k < K; k++) s += opget(oa, A, lda, i, k) * opget(ob, B, ldb, k, j);
      cplx &c = C[(i64)i * ldc + j];
      c = (beta == cplx(0) ? cplx(0) : beta * c) + alpha * s;
    }
}

void dgemm(Op oa, Op ob, int M, int Nn, int K, double alpha, const double *A, int lda,
           const double *B, int ldb, double beta, double *C, int ldc) {
  if (M <= 0 || Nn <= 0) return;
  if (g_dgemm && K > 0) {
    g_dgemm(RowMajor, oa == N ? NoTrans : Trans, ob == N ? NoTrans : Trans, M, Nn, K, alpha, A,
            lda, B, ldb, beta, C, ldc);
    return;
  }
  for (int i = 0; i < M; i++)
    for (int j = 0; j < Nn; j++) {
      double s = 0;
      for (int k = 0; k < K; k++) {
        double a = oa == N ? A[(i64)i * lda + k] : A[(i64)k * lda + i];
        double b = ob == N ? B[(i64)k * ldb + j] : B[(i64)j * ldb + k];
        s += a * b;
      }
      double &c = C[(i64)i * ldc + j];
      c = (beta == 0.0 ? 0.0 : beta * c) + alpha * s;
    }
}

void rzgemm(int M, int Nn, int K, double alpha, const double *R, int ldr, const cplx *Z, int ldz,
            double beta, cplx *C, int ldc) {
  // A row-major interleaved complex matrix Z[K x Nn] is a real matrix [K x 2Nn];
  // R * Z is then one real product.
  dgemm(N, N, M, 2 * Nn, K, alpha, R, ldr, reinterpret_cast<const double *>(Z), 2 * ldz, beta,
        reinterpret_cast<double *>(C), 2 * ldc);
}

void lu_solve(int n, int nrhs, cplx *A, cplx *B) {
  // Gaussian elimination with partial pivoting.  A: n x n, B: n x nrhs (row-major).
  std::vector<int> piv(n);
  for (int k = 0; k < n; k++) {
    int p = k;
    double best = std::abs(A[(i64)k * n + k]);
    for (int r = k + 1; r < n; r++) {
      double v = std::abs(A[(i64)r * n + k]);
      if (v > best) { best = v; p = r; }
    }
    if (p != k) {
      for (int c = 0; c < n; c++) std::swap(A[(i64)k * n + c], A[(i64)p * n + c]);
      for (int c = 0; c < nrhs; c++) std::swap(B[(i64)k * nrhs + c], B[(i64)p * nrhs + c]);
    }
    cplx inv = 1.0 / A[(i64)k * n + k];
    for (int r = k + 1; r < n; r++) {
      cplx f = A[(i64)r * n + k] * inv;
      if (f == cplx(0)) continue;
      for (int c = k + 1; c < n; c++) A[(i64)r * n + c] -= f * A[(i64)k * n + c];
      for (int c = 0; c < nrhs; c++) B[(i64)r * nrhs + c] -= f * B[(i64)k * nrhs + c];
    }
  }
  for (int k = n - 1; k >= 0; k--) {
    cplx inv = 1.0 / A[(i64)k * n + k];
    for (int c = 0; c < nrhs; c++) {
      cplx s = B[(i64)k * nrhs + c];
      for (int j = k + 1; j < n; j++) s -= A[(i64)k * n + j] * B[(i64)j * nrhs + c];
      B[(i64)k * nrhs + c] = s * inv;
    }
  }
}

void lu_solve_right(int n, int nrows, const cplx *A, cplx *B) {
  // X A = B  <=>  A^T X^T = B^T
  std::vector<cplx> At((i64)n * n), Bt((i64)n * nrows);
  for (int r = 0; r < n; r++)
    for (int c = 0; c < n; c++) At[(i64)c * n + r] = A[(i64)r * n + c];
  for (int r = 0; r < nrows; r++)
    for (int c = 0; c < n; c++) Bt[(i64)c * nrows + r] = B[(i64)r * n + c];
  lu_solve(n, nrows, At.data(), Bt.data());
  for (int r = 0; r < nrows; r++)
    for (int c = 0; c < n; c++) B[(i64)r * n + c] = Bt[(i64)c * nrows + r];
}

void herm_eig(int n, const cplx *Ain, double *evals, cplx *V) {
  // Cyclic complex Jacobi for a Hermitian matrix.  Columns of V are eigenvectors.
  std::vector<cplx> A(Ain, Ain + (i64)n * n);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) V[(i64)i * n + j] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0, tot = 0;
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        double a = std::norm(A[(i64)i * n + j]);
        tot += a;
        if (i != j) off += a;
      }
    if (off <= 1e-32 * tot || off == 0.0) break;
    for (int p = 0; p < n - 1; p++)
      for (int q = p + 1; q < n; q++) {
        cplx apq = A[(i64)p * n + q];
        double mag = std::abs(apq);
        if (mag < 1e-300) continue;
        double app = A[(i64)p * n + p].real(), aqq = A[(i64)q * n + q].real();
        cplx ph = apq / mag;  // e^{i phi}
        double theta = 0.5 * std::atan2(2.0 * mag, aqq - app);
        double c = std::cos(theta), s = std::sin(theta);
        // Rotation J acting on columns p,q:  col_p' = c col_p - s conj(ph) col_q ; col_q' = s ph col_p + c col_q
        cplx s1 = s * std::conj(ph), s2 = s * ph;
        for (int k = 0; k < n; k++) {  // A <- A J
          cplx akp = A[(i64)k * n + p], akq = A[(i64)k * n + q];
          A[(i64)k * n + p] = c * akp - s1 * akq;
          A[(i64)k * n + q] = s2 * akp + c * akq;
        }
        for (int k = 0; k < n; k++) {  // A <- J^H A
          cplx apk = A[(i64)p * n + k], aqk = A[(i64)q * n + k];
          A[(i64)p * n + k] = c * apk - std::conj(s1) * aqk;
          A[(i64)q * n + k] = std::conj(s2) * apk + c * aqk;
        }
        for (int k = 0; k < n; k++) {  // V <- V J
          cplx vkp = V[(i64)k * n + p], vkq = V[(i64)k * n + q];
          V[(i64)k * n + p] = c * vkp - s1 * vkq;
          V[(i64)k * n + q] = s2 * vkp + c * vkq;
        }
      }
  }
  std::vector<int> idx(n);
  for (int i = 0; i < n; i++) idx[i] = i;
  std::vector<double> ev(n);
  for (int i = 0; i < n; i++) ev[i] = A[(i64)i * n + i].real();
  std::sort(idx.begin(), idx.end(), [&](int a, int b) { return ev[a] < ev[b]; });
  std::vector<cplx> Vs((i64)n * n);
  for (int j = 0; j < n; j++) {
    evals[j] = ev[idx[j]];
    for (int i = 0; i < n; i++) Vs[(i64)i * n + j] = V[(i64)i * n + idx[j]];
  }
  std::copy(Vs.begin(), Vs.end(), V);
}

double fro_norm(i64 n, const cplx *A) {
  double s = 0;
  for (i64 i = 0; i < n; i++) s += std::norm(A[i]);
  return std::sqrt(s);
}

} // namespace orc
