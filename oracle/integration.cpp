// CPU oracle (test infrastructure): Gregory / BDF / polynomial calculus weights.
// Restates src/integration.cpp (builders :8-174) and src/integration.h (accessors
// :23-124) of the reference: every table is built in long double and rounded to
// double, exactly like the reference.
#include "oracle_common.h"
#include "oracle_integ.h"
#include <algorithm>

namespace orc {

namespace {
typedef long double LD;

// Inverse of an n x n long-double matrix by Gauss-Jordan with full pivoting
// (the reference uses Eigen::FullPivLU<long double>, integration.cpp:17-18).
std::vector<LD> inverse_full_pivot(int n, std::vector<LD> M) {
  std::vector<LD> Inv((size_t)n * n, 0.0L);
  for (int i = 0; i < n; i++) Inv[(size_t)i * n + i] = 1.0L;
  std::vector<int> colperm(n);
  for (int i = 0; i < n; i++) colperm[i] = i;
  // Solve M X = I by full-pivot elimination on an augmented system.
  std::vector<LD> A = M;
  std::vector<LD> B = Inv;
  for (int k = 0; k < n; k++) {
    int pr = k, pc = k;
    LD best = -1;
    for (int r = k; r < n; r++)
      for (int c = k; c < n; c++) {
        LD v = fabsl(A[(size_t)r * n + c]);
        if (v > best) { best = v; pr = r; pc = c; }
      }
    if (pr != k) {
      for (int c = 0; c < n; c++) std::swap(A[(size_t)k * n + c], A[(size_t)pr * n + c]);
      for (int c = 0; c < n; c++) std::swap(B[(size_t)k * n + c], B[(size_t)pr * n + c]);
    }
    if (pc != k) {
      for (int r = 0; r < n; r++) std::swap(A[(size_t)r * n + k], A[(size_t)r * n + pc]);
      std::swap(colperm[k], colperm[pc]);
    }
    LD piv = A[(size_t)k * n + k];
    for (int r = 0; r < n; r++) {
      if (r == k) continue;
      LD f = A[(size_t)r * n + k] / piv;
      if (f == 0) continue;
      for (int c = 0; c < n; c++) A[(size_t)r * n + c] -= f * A[(size_t)k * n + c];
      for (int c = 0; c < n; c++) B[(size_t)r * n + c] -= f * B[(size_t)k * n + c];
    }
  }
  // Now diag(A) * Y = B with Y = P^T X (column permutation of unknowns).
  std::vector<LD> X((size_t)n * n);
  for (int k = 0; k < n; k++) {
    LD piv = A[(size_t)k * n + k];
    for (int c = 0; c < n; c++) X[(size_t)colperm[k] * n + c] = B[(size_t)k * n + c] / piv;
  }
  return X;
}

// integration.cpp:8-26
std::vector<LD> poly_interp_ld(int k) {
  int k1 = k + 1;
  std::vector<LD> M((size_t)k1 * k1);
  for (int i = 0; i <= k; i++) {
    M[(size_t)i * k1 + 0] = 1.0L;
    for (int n = 1; n <= k; n++) M[(size_t)i * k1 + n] = M[(size_t)i * k1 + n - 1] * i;
  }
  return inverse_full_pivot(k1, M);
}

// integration.cpp:39-54
std::vector<LD> poly_diff_ld(int k, const std::vector<LD> &P) {
  int k1 = k + 1;
  std::vector<LD> D((size_t)k1 * k1);
  for (int n = 0; n <= k; n++)
    for (int l = 0; l <= k; l++) {
      LD npow = 1.0L, x = 0.0L;
      for (int a = 1; a <= k; a++) {
        if (a > 1) npow *= n;
        x += P[(size_t)a * k1 + l] * a * npow;
      }
      D[(size_t)n * k1 + l] = x;
    }
  return D;
}

int fact(int n) { return n > 1 ? n * fact(n - 1) : 1; }
int pascal(int row, int col) { return fact(row) / (fact(row - col) * fact(col)); }
} // namespace

Integrator::Integrator(int k) : k_(k) {
  int k1 = k + 1;
  std::vector<LD> P = poly_interp_ld(k);
  poly_interp_.resize((size_t)k1 * k1);
  for (size_t i = 0; i < P.size(); i++) poly_interp_[i] = (double)P[i];

  std::vector<LD> D = poly_diff_ld(k, P);
  poly_diff_.resize((size_t)k1 * k1);
  for (size_t i = 0; i < D.size(); i++) poly_diff_[i] = (double)D[i];

  // integration.cpp:66-88
  poly_integ_.resize((size_t)k1 * k1 * k1);
  for (int m = 0; m <= k; m++)
    for (int n = 0; n <= k; n++)
      for (int l = 0; l <= k; l++) {
        LD mpow = m, npow = n, x = 0.0L;
        for (int a = 0; a <= k; a++) {
          x += P[(size_t)a * k1 + l] * (npow - mpow) / (a + 1);
          mpow *= m;
          npow *= n;
        }
        poly_integ_[(size_t)m * k1 * k1 + (size_t)n * k1 + l] = (double)x;
      }

  // integration.cpp:105-116 : bd_weights(i) = -D_{k+1}(0,i)
  {
    std::vector<LD> P2 = poly_interp_ld(k + 1);
    std::vector<LD> D2 = poly_diff_ld(k + 1, P2);
    bd_weights_.resize(k + 2);
    for (int i = 0; i < k + 2; i++) bd_weights_[i] = (double)(-D2[i]);
  }

  // integration.cpp:118-134 : gregory start weights (int_0^n l_l)
  start_.resize((size_t)k1 * k1);
  for (int n = 0; n <= k; n++)
    for (int l = 0; l <= k; l++) {
      LD x = 0.0L, npow = n;
      for (int a = 0; a <= k; a++) {
        x += P[(size_t)a * k1 + l] * npow / (a + 1.0L);
        npow *= n;
      }
      start_[(size_t)n * k1 + l] = (double)x;
    }

  // integration.cpp:145-163 : Omega
  {
    std::vector<LD> A((size_t)k1 * k1, 0.0L), y(k1);
    for (int i = 0; i <= k; i++) {
      y[i] = (LD)(1 - 2 * ((i + 1) % 2)) / (i + 2.0L);
      for (int j = 0; j <= i; j++) A[(size_t)i * k1 + j] = (LD)(1 - 2 * ((i + j) % 2)) / (i - j + 1.0L);
    }
    std::vector<LD> Ainv = inverse_full_pivot(k1, A);
    std::vector<LD> res(k1, 0.0L);
    for (int i = 0; i <= k; i++)
      for (int j = 0; j <= k; j++) res[i] += Ainv[(size_t)i * k1 + j] * y[j];
    Omega_.resize((size_t)k1 * k1);
    for (int n = 0; n <= k; n++) {
      std::vector<LD> I(k + n + 2, 1.0L);
      for (int i = 0; i <= k; i++)
        for (int j = 0; j <= i; j++) {
          LD x = (LD)(1 - 2 * ((i + j) % 2)) * res[i] * (LD)pascal(i, j);
          I[j] += x;
          I[k + n - j + 1] += x;
        }
      for (int i = 0; i <= k; i++) Omega_[(size_t)n * k1 + i] = (double)I[i];
    }
  }

  // integration.cpp:165-173 (double arithmetic on the rounded interpolation table)
  ex_weights_.assign(k1, 0.0);
  for (int l = 0; l <= k; l++)
    for (int j = 0; j <= k; j++) ex_weights_[l] += poly_interp_[(size_t)j * k1 + l] * (1 - 2 * (j % 2));
}

// integration.h:78-91
double Integrator::gregory_weights(int n, int j) const {
  int k = k_;
  if (n <= k && j <= k) return start(n, j);
  if (n <= 2 * k + 1) {
    if (j <= k) return Omega(n - k - 1, j);
    return omega(n - j);
  }
  if (j <= k) return omega(j);
  if (j < n - k) return 1.0;
  return omega(n - j);
}

} // namespace orc
