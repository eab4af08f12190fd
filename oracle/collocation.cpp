// CPU oracle (test infrastructure): Legendre-Gauss-Lobatto collocation on the
// imaginary-time axis, replacing the external cpsitop convolution class.
//
// The node family is pinned by the reference's golden sums: the fixtures of
// tests/set_up_g.h place tau = beta*(x_i+1)/2 on the collocation nodes, and the
// Ctv_tstp / Cles3_tstp / energy goldens of tests/integrals-test.cpp:8-212 are
// reproduced with the LGL nodes (and not with Chebyshev-Lobatto or Gauss nodes).
// Each operation below is the exact integral of the degree-ntau interpolants:
//   mixing : reference call src/dyson_integrals.h:295 (Conv.mixing)
//   lesser : reference call src/dyson_integrals.h:424 (Conv.lesser)
//   energy : reference call src/dyson_integrals.h:63  (Conv.energy)
#include "oracle_integ.h"
#include <algorithm>

namespace orc {

namespace {
typedef long double LD;

void legendre_all(int n, LD x, LD *P) {  // P_0..P_n at x
  P[0] = 1.0L;
  if (n >= 1) P[1] = x;
  for (int k = 2; k <= n; k++) P[k] = ((2 * k - 1) * x * P[k - 1] - (k - 1) * P[k - 2]) / k;
}

void gauss_legendre(int q, std::vector<double> &xs, std::vector<double> &ws) {
  xs.resize(q);
  ws.resize(q);
  std::vector<LD> P(q + 1);
  for (int i = 0; i < q; i++) {
    LD x = -cosl(M_PIl * (i + 0.75L) / (q + 0.5L));
    for (int it = 0; it < 100; it++) {
      legendre_all(q, x, P.data());
      LD dp = q * (x * P[q] - P[q - 1]) / (x * x - 1.0L);
      LD dx = P[q] / dp;
      x -= dx;
      if (fabsl(dx) < 1e-19L) break;
    }
    legendre_all(q, x, P.data());
    LD dp = q * (x * P[q] - P[q - 1]) / (x * x - 1.0L);
    xs[i] = (double)x;
    ws[i] = (double)(2.0L / ((1.0L - x * x) * dp * dp));
  }
}

uint64_t fnv(const void *p, size_t n) {
  const unsigned char *c = (const unsigned char *)p;
  uint64_t h = 1469598103934665603ull;
  for (size_t i = 0; i < n; i++) { h ^= c[i]; h *= 1099511628211ull; }
  return h;
}
} // namespace

Collocation::Collocation(int ntau) : n_(ntau) {
  int n = ntau;
  x_.resize(n + 1);
  w_.resize(n + 1);
  u_.resize(n + 1);
  std::vector<LD> xl(n + 1), P(n + 1);
  xl[0] = -1.0L;
  xl[n] = 1.0L;
  // Interior LGL nodes: roots of P_n'.  Newton on P_n' with P_n'' from the
  // Legendre differential equation.
  for (int i = 1; i < n; i++) {
    LD x = -cosl(M_PIl * i / n);
    for (int it = 0; it < 100; it++) {
      legendre_all(n, x, P.data());
      LD d1 = n * (x * P[n] - P[n - 1]) / (x * x - 1.0L);
      LD d2 = (2.0L * x * d1 - n * (n + 1.0L) * P[n]) / (1.0L - x * x);
      LD dx = d1 / d2;
      x -= dx;
      if (fabsl(dx) < 1e-19L) break;
    }
    xl[i] = x;
  }
  for (int i = 0; i <= n / 2; i++) {  // exact mirror symmetry x_{n-i} = -x_i
    LD a = 0.5L * (xl[i] - xl[n - i]);
    xl[i] = a;
    xl[n - i] = -a;
  }
  if (n % 2 == 0) xl[n / 2] = 0.0L;
  for (int i = 0; i <= n; i++) {
    legendre_all(n, xl[i], P.data());
    LD wi = 2.0L / (n * (n + 1.0L) * P[n] * P[n]);
    x_[i] = (double)xl[i];
    w_[i] = (double)wi;
    // top Legendre coefficient of the interpolant: f_n = sum_i u_i f_i (discrete norm 2/n)
    u_[i] = (double)(wi * P[n] * n / 2.0L);
  }
  ctop_ = (double)(2.0L / (2.0L * n + 1.0L) - 2.0L / n);
  Q_ = n + 1;
}

void Collocation::basis(double xe, double *out) const {
  // Barycentric form; weights lambda_i = 1/prod_{j!=i}(x_i - x_j) in long double.
  static thread_local std::vector<LD> lam;
  static thread_local int lam_n = -1;
  static thread_local const Collocation *lam_owner = nullptr;
  int n = n_;
  if (lam_n != n || lam_owner != this) {
    lam.assign(n + 1, 1.0L);
    for (int i = 0; i <= n; i++) {
      LD p = 1.0L;
      for (int j = 0; j <= n; j++)
        if (j != i) p *= (LD)x_[i] - (LD)x_[j];
      lam[i] = 1.0L / p;
    }
    LD mx = 0;
    for (int i = 0; i <= n; i++) mx = std::max(mx, fabsl(lam[i]));
    for (int i = 0; i <= n; i++) lam[i] /= mx;
    lam_n = n;
    lam_owner = this;
  }
  for (int i = 0; i <= n; i++)
    if ((LD)xe == (LD)x_[i]) {
      for (int j = 0; j <= n; j++) out[j] = (i == j) ? 1.0 : 0.0;
      return;
    }
  LD den = 0;
  std::vector<LD> t(n + 1);
  for (int i = 0; i <= n; i++) {
    t[i] = lam[i] / ((LD)xe - (LD)x_[i]);
    den += t[i];
  }
  for (int i = 0; i <= n; i++) out[i] = (double)(t[i] / den);
}

void Collocation::build_eval() {
  if (!EA_.empty()) return;
  int n = n_, Q = Q_;
  int np = n + 1;
  std::vector<double> gx, gw;
  gauss_legendre(Q, gx, gw);
  // EA_[m] is stored transposed: (n+1) x 2Q, entry (i,q) = W_q l_i(x(s_q)) with the
  // x-space quadrature weight (tau-space weight is applied by the caller's beta/2).
  // EB_[m]: 2Q x (n+1), entry (q,j) = c_q l_j(x'(s_q)).
  EA_.assign((size_t)np * np * 2 * Q, 0.0);
  EB_.assign((size_t)np * 2 * Q * np, 0.0);
  std::vector<double> bas(np);
  for (int m = 0; m <= n; m++) {
    double xm = x_[m];  // split point in x-space
    double *EAm = &EA_[(size_t)m * np * 2 * Q];
    double *EBm = &EB_[(size_t)m * 2 * Q * np];
    for (int part = 0; part < 2; part++) {
      double a = part == 0 ? -1.0 : xm, b = part == 0 ? xm : 1.0;
      double half = 0.5 * (b - a);
      for (int q = 0; q < Q; q++) {
        int qq = part * Q + q;
        double xs = a + half * (gx[q] + 1.0);
        double wq = half * gw[q];
        basis(xs, bas.data());
        for (int i = 0; i <= n; i++) EAm[(size_t)i * 2 * Q + qq] = wq * bas[i];
        // shifted argument: tau - tau_m (+beta on the first part), in x-space
        double xsh = part == 0 ? (xs - xm + 1.0) : (xs - xm - 1.0);
        if (xsh > 1.0) xsh = 1.0;
        if (xsh < -1.0) xsh = -1.0;
        basis(xsh, bas.data());
        for (int j = 0; j <= n; j++) EBm[(size_t)qq * np + j] = bas[j];
      }
    }
  }
}

const std::vector<cplx> &Collocation::kernel(const cplx *B, int nao, double beta, double sig) {
  int n = n_, np = n + 1, Q = Q_;
  i64 es = (i64)nao * nao;
  uint64_t h = fnv(B, sizeof(cplx) * np * es);
  for (auto &e : cache_)
    if (e.hash == h && e.nao == nao && e.beta == beta && e.sig == sig) return e.K;
  build_eval();
  KEntry ent;
  ent.hash = h;
  ent.nao = nao;
  ent.beta = beta;
  ent.sig = sig;
  ent.K.assign((size_t)np * np * es, cplx(0));
#pragma omp parallel
  {
    std::vector<cplx> BB((size_t)2 * Q * es);
#pragma omp for schedule(dynamic)
    for (int m = 0; m <= n; m++) {
      const double *EBm = &EB_[(size_t)m * 2 * Q * np];
      const double *EAm = &EA_[(size_t)m * np * 2 * Q];
      rzgemm(2 * Q, (int)es, np, 1.0, EBm, np, B, (int)es, 0.0, BB.data(), (int)es);
      // antiperiodic sign on the first part (tau < tau_m)
      for (int q = 0; q < Q; q++)
        for (i64 e = 0; e < es; e++) BB[(size_t)q * es + e] *= sig;
      rzgemm(np, (int)es, 2 * Q, 0.5 * beta, EAm, 2 * Q, BB.data(), (int)es, 0.0,
             &ent.K[(size_t)m * np * es], (int)es);
    }
  }
  if (cache_.size() >= 2) cache_.erase(cache_.begin());
  cache_.push_back(std::move(ent));
  return cache_.back().K;
}

void Collocation::mixing(cplx *res, const cplx *A, const cplx *B, int nao, double beta, double sig) {
  int np = n_ + 1;
  i64 es = (i64)nao * nao;
  const std::vector<cplx> &K = kernel(B, nao, beta, sig);
  // A'[a][(i,c)] = A[i][a][c]
  std::vector<cplx> Ap((size_t)np * es);
  for (int i = 0; i < np; i++)
    for (int a = 0; a < nao; a++)
      for (int c = 0; c < nao; c++) Ap[(size_t)a * np * nao + (size_t)i * nao + c] = A[(size_t)i * es + a * nao + c];
  for (int m = 0; m < np; m++)
    zgemm(N, N, nao, nao, np * nao, 1.0, Ap.data(), np * nao, &K[(size_t)m * np * es], nao, 0.0,
          res + (size_t)m * es, nao);
}

void Collocation::lesser(cplx *res, const cplx *A, const cplx *B, int nao, double beta) const {
  int np = n_ + 1;
  i64 es = (i64)nao * nao;
  std::vector<cplx> UA(es, 0.0), UB(es, 0.0), acc(es, 0.0);
  for (int i = 0; i < np; i++) {
    zgemm(N, N, nao, nao, nao, w_[i], A + i * es, nao, B + i * es, nao, 1.0, acc.data(), nao);
    for (i64 e = 0; e < es; e++) {
      UA[e] += u_[i] * A[i * es + e];
      UB[e] += u_[i] * B[i * es + e];
    }
  }
  zgemm(N, N, nao, nao, nao, ctop_, UA.data(), nao, UB.data(), nao, 1.0, acc.data(), nao);
  for (i64 e = 0; e < es; e++) res[e] += 0.5 * beta * acc[e];
}

cplx Collocation::energy(const cplx *A, const cplx *B, int nao, double beta, double sig) const {
  int n = n_, np = n + 1;
  i64 es = (i64)nao * nao;
  cplx s = 0;
  std::vector<cplx> UA(es, 0.0), UB(es, 0.0);
  for (int i = 0; i < np; i++) {
    const cplx *Ai = A + i * es, *Bi = B + (i64)(n - i) * es;
    cplx t = 0;
    for (i64 e = 0; e < es; e++) {
      t += Ai[e] * std::conj(Bi[e]);
      UA[e] += u_[i] * Ai[e];
      UB[e] += u_[i] * std::conj(Bi[e]);
    }
    s += w_[i] * t;
  }
  cplx t = 0;
  for (i64 e = 0; e < es; e++) t += UA[e] * UB[e];
  s += ctop_ * t;
  return -sig * 0.5 * beta * s;
}

} // namespace orc
