// Host-side tables of the engine: calculus weights and the Legendre collocation.
//
// Weights restate Integration::Integrator (reference src/integration.cpp:8-174,
// src/integration.h:78-91): every table is built in long double and rounded.
// Collocation: ntau+1 Legendre-Gauss-Lobatto nodes on [-1,1] (tau = beta(x+1)/2),
// the node set that reproduces the reference's imaginary-time known answers
// (tests/integrals-test.cpp:8-212).  The mixing quadrature splits [0,beta] at
// each node tau_m and integrates the product of interpolants exactly with
// ntau+1 Gauss-Legendre points per piece.
#include "engine.cuh"
#include <cmath>
#include <algorithm>

namespace nedy {

namespace {
typedef long double LD;

// Gauss-Jordan inverse with full pivoting in long double.
std::vector<LD> inv_fp(int n, std::vector<LD> A) {
  std::vector<LD> B((size_t)n * n, 0.0L);
  for (int i = 0; i < n; i++) B[(size_t)i * n + i] = 1.0L;
  std::vector<int> perm(n);
  for (int i = 0; i < n; i++) perm[i] = i;
  for (int k = 0; k < n; k++) {
    int pr = k, pc = k;
    LD best = -1;
    for (int r = k; r < n; r++)
      for (int c = k; c < n; c++)
        if (fabsl(A[(size_t)r * n + c]) > best) { best = fabsl(A[(size_t)r * n + c]); pr = r; pc = c; }
    if (pr != k)
      for (int c = 0; c < n; c++) {
        std::swap(A[(size_t)k * n + c], A[(size_t)pr * n + c]);
        std::swap(B[(size_t)k * n + c], B[(size_t)pr * n + c]);
      }
    if (pc != k) {
      for (int r = 0; r < n; r++) std::swap(A[(size_t)r * n + k], A[(size_t)r * n + pc]);
      std::swap(perm[k], perm[pc]);
    }
    for (int r = 0; r < n; r++) {
      if (r == k) continue;
      LD f = A[(size_t)r * n + k] / A[(size_t)k * n + k];
      if (f == 0) continue;
      for (int c = 0; c < n; c++) {
        A[(size_t)r * n + c] -= f * A[(size_t)k * n + c];
        B[(size_t)r * n + c] -= f * B[(size_t)k * n + c];
      }
    }
  }
  std::vector<LD> X((size_t)n * n);
  for (int k = 0; k < n; k++)
    for (int c = 0; c < n; c++) X[(size_t)perm[k] * n + c] = B[(size_t)k * n + c] / A[(size_t)k * n + k];
  return X;
}

std::vector<LD> interp(int k) {
  int k1 = k + 1;
  std::vector<LD> M((size_t)k1 * k1);
  for (int i = 0; i <= k; i++) {
    M[(size_t)i * k1] = 1.0L;
    for (int n = 1; n <= k; n++) M[(size_t)i * k1 + n] = M[(size_t)i * k1 + n - 1] * i;
  }
  return inv_fp(k1, M);
}

std::vector<LD> diffm(int k, const std::vector<LD> &P) {
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

void legendre_all(int n, LD x, LD *P) {
  P[0] = 1.0L;
  if (n >= 1) P[1] = x;
  for (int k = 2; k <= n; k++) P[k] = ((2 * k - 1) * x * P[k - 1] - (k - 1) * P[k - 2]) / k;
}
} // namespace

Weights make_weights(int k) {
  NEDY_REQUIRE(k >= 1 && k <= 10, "weights: k out of range");
  Weights W;
  W.k = k;
  int k1 = k + 1;
  std::vector<LD> P = interp(k), D = diffm(k, P);
  W.poly_interp.resize((size_t)k1 * k1);
  W.poly_diff.resize((size_t)k1 * k1);
  for (size_t i = 0; i < P.size(); i++) { W.poly_interp[i] = (double)P[i]; W.poly_diff[i] = (double)D[i]; }
  W.poly_integ.resize((size_t)k1 * k1 * k1);
  for (int m = 0; m <= k; m++)
    for (int n = 0; n <= k; n++)
      for (int l = 0; l <= k; l++) {
        LD mp = m, np = n, x = 0;
        for (int a = 0; a <= k; a++) { x += P[(size_t)a * k1 + l] * (np - mp) / (a + 1); mp *= m; np *= n; }
        W.poly_integ[((size_t)m * k1 + n) * k1 + l] = (double)x;
      }
  std::vector<LD> P2 = interp(k + 1), D2 = diffm(k + 1, P2);
  W.bd.resize(k + 2);
  for (int i = 0; i < k + 2; i++) W.bd[i] = (double)(-D2[i]);
  W.start.resize((size_t)k1 * k1);
  for (int n = 0; n <= k; n++)
    for (int l = 0; l <= k; l++) {
      LD x = 0, np = n;
      for (int a = 0; a <= k; a++) { x += P[(size_t)a * k1 + l] * np / (a + 1.0L); np *= n; }
      W.start[(size_t)n * k1 + l] = (double)x;
    }
  {
    std::vector<LD> A((size_t)k1 * k1, 0.0L), y(k1), res(k1, 0.0L);
    for (int i = 0; i <= k; i++) {
      y[i] = (LD)(1 - 2 * ((i + 1) % 2)) / (i + 2.0L);
      for (int j = 0; j <= i; j++) A[(size_t)i * k1 + j] = (LD)(1 - 2 * ((i + j) % 2)) / (i - j + 1.0L);
    }
    std::vector<LD> Ai = inv_fp(k1, A);
    for (int i = 0; i <= k; i++)
      for (int j = 0; j <= k; j++) res[i] += Ai[(size_t)i * k1 + j] * y[j];
    W.Omega.resize((size_t)k1 * k1);
    for (int n = 0; n <= k; n++) {
      std::vector<LD> I(k + n + 2, 1.0L);
      for (int i = 0; i <= k; i++)
        for (int j = 0; j <= i; j++) {
          LD x = (LD)(1 - 2 * ((i + j) % 2)) * res[i] * (LD)(fact(i) / (fact(i - j) * fact(j)));
          I[j] += x;
          I[k + n - j + 1] += x;
        }
      for (int i = 0; i <= k; i++) W.Omega[(size_t)n * k1 + i] = (double)I[i];
    }
  }
  W.ex.assign(k1, 0.0);
  for (int l = 0; l <= k; l++)
    for (int j = 0; j <= k; j++) W.ex[l] += W.poly_interp[(size_t)j * k1 + l] * (1 - 2 * (j % 2));
  return W;
}

double Weights::gregory(int n, int j) const {
  if (n <= k && j <= k) return start[(size_t)n * (k + 1) + j];
  if (n <= 2 * k + 1) {
    if (j <= k) return Omega[(size_t)(n - k - 1) * (k + 1) + j];
    return omega(n - j);
  }
  if (j <= k) return omega(j);
  if (j < n - k) return 1.0;
  return omega(n - j);
}

Colloc make_colloc(int ntau) {
  NEDY_REQUIRE(ntau >= 2, "collocation: ntau must be >= 2");
  Colloc c;
  int n = ntau;
  c.ntau = n;
  c.x.resize(n + 1);
  c.w.resize(n + 1);
  c.u.resize(n + 1);
  std::vector<LD> xl(n + 1), P(n + 1);
  xl[0] = -1.0L;
  xl[n] = 1.0L;
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
  for (int i = 0; i <= n / 2; i++) {
    LD a = 0.5L * (xl[i] - xl[n - i]);
    xl[i] = a;
    xl[n - i] = -a;
  }
  if (n % 2 == 0) xl[n / 2] = 0.0L;
  for (int i = 0; i <= n; i++) {
    legendre_all(n, xl[i], P.data());
    LD wi = 2.0L / (n * (n + 1.0L) * P[n] * P[n]);
    c.x[i] = (double)xl[i];
    c.w[i] = (double)wi;
    c.u[i] = (double)(wi * P[n] * n / 2.0L);
  }
  c.ctop = (double)(2.0L / (2.0L * n + 1.0L) - 2.0L / n);
  c.Q = n + 1;
  return c;
}

void build_mixing_eval(Colloc &c) {
  if (!c.EA.empty()) return;
  int n = c.ntau, np = n + 1, Q = c.Q;
  // Gauss-Legendre points / weights (Q points)
  std::vector<double> gx(Q), gw(Q);
  {
    std::vector<LD> P(Q + 1);
    for (int i = 0; i < Q; i++) {
      LD x = -cosl(M_PIl * (i + 0.75L) / (Q + 0.5L));
      for (int it = 0; it < 100; it++) {
        legendre_all(Q, x, P.data());
        LD dp = Q * (x * P[Q] - P[Q - 1]) / (x * x - 1.0L);
        LD dx = P[Q] / dp;
        x -= dx;
        if (fabsl(dx) < 1e-19L) break;
      }
      legendre_all(Q, x, P.data());
      LD dp = Q * (x * P[Q] - P[Q - 1]) / (x * x - 1.0L);
      gx[i] = (double)x;
      gw[i] = (double)(2.0L / ((1.0L - x * x) * dp * dp));
    }
  }
  // barycentric weights of the LGL nodes
  std::vector<LD> lam(np, 1.0L);
  for (int i = 0; i < np; i++) {
    LD p = 1.0L;
    for (int j = 0; j < np; j++)
      if (j != i) p *= (LD)c.x[i] - (LD)c.x[j];
    lam[i] = 1.0L / p;
  }
  LD mx = 0;
  for (int i = 0; i < np; i++) mx = std::max(mx, fabsl(lam[i]));
  for (int i = 0; i < np; i++) lam[i] /= mx;
  auto basis = [&](double xe, double *out) {
    for (int i = 0; i < np; i++)
      if ((LD)xe == (LD)c.x[i]) {
        for (int j = 0; j < np; j++) out[j] = i == j ? 1.0 : 0.0;
        return;
      }
    LD den = 0;
    std::vector<LD> t(np);
    for (int i = 0; i < np; i++) { t[i] = lam[i] / ((LD)xe - (LD)c.x[i]); den += t[i]; }
    for (int i = 0; i < np; i++) out[i] = (double)(t[i] / den);
  };
  c.EA.assign((size_t)np * np * 2 * Q, 0.0);
  c.EB.assign((size_t)np * 2 * Q * np, 0.0);
  std::vector<double> bas(np);
  for (int m = 0; m <= n; m++) {
    double xm = c.x[m];
    double *EAm = &c.EA[(size_t)m * np * 2 * Q];
    double *EBm = &c.EB[(size_t)m * 2 * Q * np];
    for (int part = 0; part < 2; part++) {
      double a = part == 0 ? -1.0 : xm, b = part == 0 ? xm : 1.0, half = 0.5 * (b - a);
      for (int q = 0; q < Q; q++) {
        int qq = part * Q + q;
        double xs = a + half * (gx[q] + 1.0), wq = half * gw[q];
        basis(xs, bas.data());
        for (int i = 0; i <= n; i++) EAm[(size_t)i * 2 * Q + qq] = wq * bas[i];
        double xsh = part == 0 ? (xs - xm + 1.0) : (xs - xm - 1.0);
        xsh = std::min(1.0, std::max(-1.0, xsh));
        basis(xsh, bas.data());
        for (int j = 0; j <= n; j++) EBm[(size_t)qq * np + j] = bas[j];
      }
    }
  }
}

} // namespace nedy
