// CPU oracle (test infrastructure): the Dyson time step, its history integrals,
// the predictor, the bootstrap and the free Green's function.
//
//   Extrapolate        : reference src/dyson.cpp:47-117
//   CTV1, Ctv_tstp     : reference src/dyson_integrals.h:80-116, :254-324
//   Cles2, Cles3       : reference src/dyson_integrals.h:336-386, :393-461
//   energy_conv        : reference src/dyson_integrals.h:24-70
//   tv_it_conv         : reference src/dyson_integrals.h:7-15
//   dyson_step_*       : reference src/dyson_step.h:7-382
//   dyson_start_*      : reference src/dyson_boot.h:6-230
//   G0_from_h0 (const) : reference src/dyson_free.h:226-297
#include "oracle_integ.h"

namespace orc {

namespace {
typedef std::vector<cplx> Buf;
constexpr Op N_ = Op::N, C_ = Op::C;
inline void madd(int n, cplx f, const cplx *A, cplx *out) {  // out += f*A
  for (int e = 0; e < n * n; e++) out[e] += f * A[e];
}
inline void mm(int n, cplx f, Op oa, const cplx *A, Op ob, const cplx *B, cplx *out) {  // out += f op(A) op(B)
  zgemm(oa, ob, n, n, n, f, A, n, B, n, 1.0, out, n);
}
inline void adj(int n, const cplx *A, cplx *out) {
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) out[j * n + i] = std::conj(A[i * n + j]);
}
inline void tr(int n, const cplx *A, cplx *out) {
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) out[j * n + i] = A[i * n + j];
}
inline double diffnorm(int n, const cplx *A, const cplx *B) {
  double s = 0;
  for (int e = 0; e < n * n; e++) s += std::norm(A[e] - B[e]);
  return std::sqrt(s);
}
// block (r,c) of a (kn x kn) row-major matrix
inline cplx &blk(cplx *M, int kn, int n, int r, int c, int i, int j) {
  return M[(i64)(r * n + i) * kn + (c * n + j)];
}

double fermi(double beta, double omega) {  // dyson_free.h:9-17
  double arg = omega * beta;
  if (std::fabs(arg) > 100.0) return arg > 0.0 ? 0.0 : 1.0;
  return 1.0 / (1.0 + std::exp(arg));
}
double fermi_exp(double beta, double tau, double omega) {  // dyson_free.h:31-39
  if (omega < 0) return std::exp(omega * tau) * fermi(beta, omega);
  return std::exp((tau - beta) * omega) * fermi(beta, -omega);
}
} // namespace

Dyson::Dyson(int nt, int ntau, int nao, int k)
    : I(k), Conv(ntau), nt_(nt), ntau_(ntau), nao_(nao), es_(nao * nao), k_(k) {}

void Dyson::Extrapolate(int n, const GF &G) const {
  int k = k_, N = nao_, es = es_;
  std::vector<double> exw(k + 1, 0.0);
  for (int l = 0; l <= k; l++)
    for (int j = 0; j <= k; j++) exw[l] += I.poly_interp(j, l) * (1 - 2 * (j % 2));
  // right mixing
  std::memset((void *)G.tvptr(n, 0), 0, sizeof(cplx) * es * (ntau_ + 1));
  for (int l = 0; l <= ntau_; l++)
    for (int j = 0; j <= k; j++) madd(N, exw[j], G.tvptr(n - j - 1, l), G.tvptr(n, l));
  // retarded
  std::memset((void *)G.retptr(n, 0), 0, sizeof(cplx) * (n + 1) * es);
  for (int l = 0; l < n - k; l++)
    for (int j = 0; j <= k; j++) madd(N, exw[j], G.retptr(n - j - 1, n - l - j - 1), G.retptr(n, n - l));
  Buf tmp(es);
  for (int l = 0; l <= k; l++) {
    int jcut = (l <= n - k - 1) ? k : (n - l - 1);
    for (int j = 0; j <= jcut; j++) madd(N, exw[j], G.retptr(n - j - 1, l), G.retptr(n, l));
    for (int j = jcut + 1; j <= k; j++) {
      adj(N, G.retptr(l, n - j - 1), tmp.data());
      madd(N, -exw[j], tmp.data(), G.retptr(n, l));
    }
  }
  // lesser
  std::memset((void *)G.lesptr(0, n), 0, sizeof(cplx) * (n + 1) * es);
  adj(N, G.tvptr(n, 0), tmp.data());
  for (int e = 0; e < es; e++) G.lesptr(0, n)[e] = -tmp[e];
  for (int l = 1; l <= k; l++) {
    int jcut = (k > n - l - 1) ? (n - l - 1) : k;
    for (int j = 0; j <= jcut; j++) madd(N, exw[j], G.lesptr(l, n - 1 - j), G.lesptr(l, n));
    for (int j = jcut + 1; j <= k; j++) {
      adj(N, G.lesptr(n - 1 - j, l), tmp.data());
      madd(N, -exw[j], tmp.data(), G.lesptr(l, n));
    }
  }
  for (int l = k + 1; l <= n; l++)
    for (int j = 0; j <= k; j++) madd(N, exw[j], G.lesptr(l - j - 1, n - j - 1), G.lesptr(l, n));
}

void Dyson::CTV1(cplx *ctv, const GF &A, const GF &Acc, const GF &B, int n, double dt) const {
  int N = nao_, es = es_, k = k_;
  int ntop = n > k ? n : k;
  Buf tmp(es);
  for (int j = 0; j <= ntop; j++) {
    if (j > n) {
      adj(N, Acc.retptr(j, n), tmp.data());
      for (int e = 0; e < es; e++) tmp[e] *= -dt * I.gregory_weights(n, j);
    } else {
      const cplx *Ar = A.retptr(n, j);
      for (int e = 0; e < es; e++) tmp[e] = dt * I.gregory_weights(n, j) * Ar[e];
    }
    // ctv[m] += tmp * B.tv(j,m) for all m: one product (N x N)(N x (ntau+1)N) in tv layout
    for (int m = 0; m <= ntau_; m++) mm(N, 1.0, N_, tmp.data(), N_, B.tvptr(j, m), ctv + (i64)m * es);
  }
}

void Dyson::Ctv_tstp(int tstp, const GF &C, const GF &A, const GF &Acc, const GF &B, const GF &Bcc,
                     double beta, double dt) {
  (void)Bcc;
  int es = es_;
  Buf ntt((size_t)(ntau_ + 1) * es);
  Conv.mixing(ntt.data(), A.tvptr(tstp, 0), B.matptr(0), nao_, beta, (double)B.sig);
  CTV1(ntt.data(), A, Acc, B, tstp, dt);
  std::memcpy((void *)C.tvptr(tstp, 0), ntt.data(), sizeof(cplx) * (ntau_ + 1) * es);
}

void Dyson::Cles2_tstp(int j1, int j2, const GF &A, const GF &Acc, const GF &B, const GF &Bcc, int m,
                       double dt, cplx *res) const {
  int N = nao_, es = es_, k = k_;
  int top = m > k ? m : k;
  Buf X((size_t)(top + 1) * es);
  Buf tmp(es);
  for (int j = 0; j <= top; j++) {
    if (m >= j) {
      adj(N, Bcc.retptr(m, j), X.data() + (i64)j * es);
      for (int e = 0; e < es; e++) X[(i64)j * es + e] *= dt * I.gregory_weights(m, j);
    } else {
      const cplx *Br = B.retptr(j, m);
      for (int e = 0; e < es; e++) X[(i64)j * es + e] = -dt * I.gregory_weights(m, j) * Br[e];
    }
  }
#pragma omp parallel for schedule(dynamic)
  for (int n = j1; n <= j2; n++) {
    cplx *r = res + (i64)(n - j1) * es;
    for (int j = 0; j < n; j++) mm(N, -1.0, C_, Acc.lesptr(j, n), N_, X.data() + (i64)j * es, r);
    for (int j = n; j <= top; j++) mm(N, 1.0, N_, A.lesptr(n, j), N_, X.data() + (i64)j * es, r);
  }
}

void Dyson::Cles3_tstp(int j1, int j2, const GF &A, const GF &Acc, const GF &B, const GF &Bcc, int m,
                       double beta, cplx *res) {
  (void)Acc;
  int N = nao_, es = es_;
  Buf ntt((size_t)(ntau_ + 1) * es), tmp(es);
  for (int j = 0; j <= ntau_; j++) {
    adj(N, Bcc.tvptr(m, ntau_ - j), tmp.data());
    for (int e = 0; e < es; e++) ntt[(i64)j * es + e] = (double)B.sig * cplx(0, 1) * tmp[e];
  }
  for (int n = j1; n <= j2; n++) Conv.lesser(res + (i64)(n - j1) * es, A.tvptr(n, 0), ntt.data(), N, beta);
}

double Dyson::energy_conv(int tstp, const GF &Sig, const GF &G, double beta, double dt) {
  int N = nao_, es = es_, k = k_;
  int top = tstp >= k ? tstp : k, sig = G.sig;
  cplx res1 = 0, res2 = 0;
  auto tsum = [&](const cplx *A, const cplx *B) {  // sum_ij A_ij (B^T)_ij
    cplx s = 0;
    for (int i = 0; i < N; i++)
      for (int j = 0; j < N; j++) s += A[i * N + j] * B[j * N + i];
    return s;
  };
  for (int i = 0; i <= tstp; i++) res1 += I.gregory_weights(tstp, i) * tsum(Sig.retptr(tstp, i), G.lesptr(i, tstp));
  for (int i = tstp + 1; i <= top; i++)
    res1 += std::conj(I.gregory_weights(tstp, i) * tsum(Sig.retptr(i, tstp), G.lesptr(tstp, i)));
  for (int i = 0; i <= tstp; i++)
    res1 -= std::conj(I.gregory_weights(tstp, i) * tsum(Sig.lesptr(i, tstp), G.retptr(tstp, i)));
  for (int i = tstp + 1; i <= top; i++)
    res1 -= I.gregory_weights(tstp, i) * tsum(Sig.lesptr(tstp, i), G.retptr(i, tstp));
  res1 *= dt;
  (void)es;
  res2 = Conv.energy(Sig.tvptr(tstp, 0), G.tvptr(tstp, 0), N, beta, (double)G.sig);
  res2 *= cplx(0., -1.);
  return (cplx(0., sig * 0.5) * (res1 + res2)).real();
}

void Dyson::tv_it_conv(int m, int n, const GF &Sig, const GF &G, double beta, cplx *res) {
  tv_it_conv_k(m, n, Sig, Conv.kernel(G.matptr(0), nao_, beta, (double)G.sig), res);
}

void Dyson::tv_it_conv_k(int m, int n, const GF &Sig, const std::vector<cplx> &K, cplx *res) const {
  // res += int_0^beta Sig^tv(n,tau) G^M(tau - tau_m) dtau, through the real part of the
  // mixing kernel of G^M (the reference keeps only .real() of its precomputed
  // tensor, src/greens.cpp:140-142).
  int N = nao_, es = es_, np = ntau_ + 1;
  Buf Kr(es);
  for (int i = 0; i < np; i++) {
    const cplx *Kmi = &K[((size_t)m * np + i) * es];
    for (int e = 0; e < es; e++) Kr[e] = Kmi[e].real();
    mm(N, 1.0, N_, Sig.tvptr(n, i), N_, Kr.data(), res);
  }
}

double Dyson::dyson_step_ret(int tstp, const GF &G, const GF &Sig, const cplx *hmf, double mu, double dt) {
  int N = nao_, es = es_, k = k_, kn = k * N;
  double err = 0;
  const cplx ncplxi(0, -1);
  Buf Q((size_t)(tstp + 1) * es, 0.0), M((size_t)kn * kn, 0.0), tmp(es), tmp2(es);
  // initial condition
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++) G.retptr(tstp, tstp)[i * N + j] = i == j ? ncplxi : 0.0;
  for (int n = 1; n <= k; n++) {
    cplx *Qn = Q.data() + (i64)(n - 1) * es;
    for (int l = 0; l <= k; l++) {
      int bc = (l == 0) ? 0 : l - 1;
      if (l == 0) {
        tr(N, G.retptr(tstp, tstp), tmp.data());
        madd(N, ncplxi / dt * I.poly_diff(n, l), tmp.data(), Qn);
      } else {
        for (int i = 0; i < N; i++) blk(M.data(), kn, N, n - 1, bc, i, i) -= ncplxi / dt * I.poly_diff(n, l);
      }
      if (l == n) {
        const cplx *h = hmf + (i64)(tstp - n) * es;
        for (int i = 0; i < N; i++)
          for (int j = 0; j < N; j++) blk(M.data(), kn, N, n - 1, bc, i, j) += (i == j ? mu : 0.0) - h[j * N + i];
      }
      if (l == 0) {
        std::fill(tmp.begin(), tmp.end(), 0.0);
        mm(N, 1.0, N_, G.retptr(tstp, tstp), N_, Sig.retptr(tstp, tstp - n), tmp.data());
        tr(N, tmp.data(), tmp2.data());
        madd(N, dt * I.gregory_weights(n, l), tmp2.data(), Qn);
      } else {
        double w = dt * I.gregory_weights(n, l);
        if (tstp - l >= tstp - n) {
          const cplx *S = Sig.retptr(tstp - l, tstp - n);
          for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++) blk(M.data(), kn, N, n - 1, bc, i, j) -= w * S[j * N + i];
        } else {
          const cplx *S = Sig.retptr(tstp - n, tstp - l);
          for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++) blk(M.data(), kn, N, n - 1, bc, i, j) += w * std::conj(S[i * N + j]);
        }
      }
    }
  }
  // M X = Q  (X: kN x N)
  Buf X(Q.begin(), Q.begin() + (i64)k * es);
  lu_solve(kn, N, M.data(), X.data());
  for (int l = 0; l < k; l++) {
    tr(N, X.data() + (i64)l * es, tmp.data());
    err += diffnorm(N, G.retptr(tstp, tstp - l - 1), tmp.data());
    std::memcpy((void *)G.retptr(tstp, tstp - l - 1), tmp.data(), sizeof(cplx) * es);
  }
  for (int n = k + 1; n <= tstp; n++) {
    cplx *Qn = Q.data() + (i64)n * es;
    for (int l = 0; l <= k; l++)
      mm(N, I.gregory_weights(n, l), N_, G.retptr(tstp, tstp - l), N_, Sig.retptr(tstp - l, tstp - n), Qn);
  }
  Buf Ms(es);
  for (int n = k + 1; n <= tstp; n++) {
    cplx *Qn = Q.data() + (i64)n * es;
    for (int e = 0; e < es; e++) Qn[e] *= dt;
    for (int l = 1; l <= k + 1; l++) madd(N, I.bd_weights(l) * ncplxi / dt, G.retptr(tstp, tstp - n + l), Qn);
    const cplx *h = hmf + (i64)(tstp - n) * es;
    const cplx *S = Sig.retptr(tstp - n, tstp - n);
    cplx diag = mu - I.bd_weights(0) * ncplxi / dt;
    for (int i = 0; i < N; i++)
      for (int j = 0; j < N; j++)
        Ms[i * N + j] = -h[j * N + i] - dt * I.omega(0) * S[j * N + i] + (i == j ? diag : 0.0);
    // X M = Q  (X = Q M^{-1}), the reference solves M^T-transposed form (dyson_step.h:100-101)
    std::memcpy(tmp.data(), Qn, sizeof(cplx) * es);
    // X = (M^{-1} Q^T)^T
    Buf Mc(Ms), QT(es);
    tr(N, tmp.data(), QT.data());
    lu_solve(N, N, Mc.data(), QT.data());
    tr(N, QT.data(), tmp.data());
    err += diffnorm(N, G.retptr(tstp, tstp - n), tmp.data());
    std::memcpy((void *)G.retptr(tstp, tstp - n), tmp.data(), sizeof(cplx) * es);
    for (int m = n + 1; m <= tstp; m++)
      mm(N, I.gregory_weights(m, n), N_, G.retptr(tstp, tstp - n), N_, Sig.retptr(tstp - n, tstp - m),
         Q.data() + (i64)m * es);
  }
  return err;
}

double Dyson::dyson_step_tv(int tstp, const GF &G, const GF &Sig, const cplx *hmf, double mu, double beta,
                            double dt) {
  int N = nao_, es = es_, k = k_, np = ntau_ + 1;
  double err = 0;
  const cplx cplxi(0, 1);
  Buf old((size_t)np * es);
  std::memcpy(old.data(), G.tvptr(tstp, 0), sizeof(cplx) * np * es);
  std::memset((void *)G.tvptr(tstp, 0), 0, sizeof(cplx) * np * es);
  Ctv_tstp(tstp, G, Sig, Sig, G, G, beta, dt);
  for (int l = 1; l <= k + 1; l++) {
    cplx f = -cplxi / dt * I.bd_weights(l);
    const cplx *src = G.tvptr(tstp - l, 0);
    cplx *dst = G.tvptr(tstp, 0);
    for (i64 e = 0; e < (i64)np * es; e++) dst[e] += f * src[e];
  }
  Buf M(es);
  const cplx *h = hmf + (i64)tstp * es;
  const cplx *S = Sig.retptr(tstp, tstp);
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++)
      M[i * N + j] = (i == j ? cplxi / dt * I.bd_weights(0) + mu : 0.0) - h[i * N + j] - dt * I.omega(0) * S[i * N + j];
  // one factorization, ntau+1 right-hand sides: M X_m = Q_m for all m at once
  Buf Rhs((size_t)N * np * N);  // N x (np*N): column block m = Q_m
  for (int m = 0; m < np; m++)
    for (int i = 0; i < N; i++)
      for (int j = 0; j < N; j++) Rhs[(i64)i * np * N + m * N + j] = G.tvptr(tstp, m)[i * N + j];
  Buf Mc(M);
  lu_solve(N, np * N, Mc.data(), Rhs.data());
  for (int m = 0; m < np; m++) {
    cplx *dst = G.tvptr(tstp, m);
    for (int i = 0; i < N; i++)
      for (int j = 0; j < N; j++) dst[i * N + j] = Rhs[(i64)i * np * N + m * N + j];
    err += diffnorm(N, old.data() + (i64)m * es, dst);
  }
  return err;
}

double Dyson::dyson_step_les(int n, const GF &G, const GF &Sig, const cplx *hmf, double mu, double beta,
                             double dt) {
  int N = nao_, es = es_, k = k_, kn = k * N;
  int num = n >= k ? n : k;
  double err = 0;
  const cplx cplxi(0, 1);
  Buf tmp(es);
  adj(N, G.tvptr(n, 0), tmp.data());
  {
    double s = 0;
    for (int e = 0; e < es; e++) s += std::norm(G.lesptr(0, n)[e] + tmp[e]);
    err += std::sqrt(s);
  }
  for (int e = 0; e < es; e++) G.lesptr(0, n)[e] = -tmp[e];
  Buf Q((size_t)(num + 1) * es, 0.0), M((size_t)kn * kn, 0.0), X((size_t)(num + 1) * es, 0.0);
  Cles3_tstp(0, (n <= k ? k : n), Sig, Sig, G, G, n, beta, Q.data());
  Cles2_tstp(0, num, Sig, Sig, G, G, n, dt, Q.data());
  for (int m = 1; m <= k; m++) {
    cplx *Qm = Q.data() + (i64)m * es;
    for (int l = 0; l <= k; l++) {
      int bc = l - 1;
      if (l == 0) madd(N, -cplxi / dt * I.poly_diff(m, l), G.lesptr(l, n), Qm);
      else for (int i = 0; i < N; i++) blk(M.data(), kn, N, m - 1, bc, i, i) += cplxi / dt * I.poly_diff(m, l);
      if (m == l) {
        const cplx *h = hmf + (i64)l * es;
        for (int i = 0; i < N; i++)
          for (int j = 0; j < N; j++) blk(M.data(), kn, N, m - 1, bc, i, j) += (i == j ? mu : 0.0) - h[i * N + j];
      }
      if (l == 0) mm(N, dt * I.gregory_weights(m, l), N_, Sig.retptr(m, l), N_, G.lesptr(l, n), Qm);
      else {
        double w = dt * I.gregory_weights(m, l);
        if (m >= l) {
          const cplx *S = Sig.retptr(m, l);
          for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++) blk(M.data(), kn, N, m - 1, bc, i, j) -= w * S[i * N + j];
        } else {
          const cplx *S = Sig.retptr(l, m);
          for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++) blk(M.data(), kn, N, m - 1, bc, i, j) += w * std::conj(S[j * N + i]);
        }
      }
    }
  }
  std::memcpy(X.data() + es, Q.data() + es, sizeof(cplx) * kn * N);
  lu_solve(kn, N, M.data(), X.data() + es);
  for (int e = 0; e < es; e++) X[e] = -tmp[e];
  Buf Ms(es);
  for (int m = k + 1; m < n; m++) {
    cplx *Qm = Q.data() + (i64)m * es;
    const cplx *h = hmf + (i64)m * es;
    const cplx *S = Sig.retptr(m, m);
    for (int i = 0; i < N; i++)
      for (int j = 0; j < N; j++)
        Ms[i * N + j] = -h[i * N + j] + (i == j ? cplxi / dt * I.bd_weights(0) + mu : 0.0) - dt * I.omega(0) * S[i * N + j];
    for (int l = 0; l < m; l++)
      mm(N, dt * I.gregory_weights(m, l), N_, Sig.retptr(m, l), N_, X.data() + (i64)l * es, Qm);
    for (int l = 1; l <= k + 1; l++) madd(N, -cplxi / dt * I.bd_weights(l), X.data() + (i64)(m - l) * es, Qm);
    std::memcpy(X.data() + (i64)m * es, Qm, sizeof(cplx) * es);
    lu_solve(N, N, Ms.data(), X.data() + (i64)m * es);
  }
  // diagonal
  cplx *Xn = X.data() + (i64)n * es;
  std::fill(Xn, Xn + es, 0.0);
  for (int jj = 0; jj <= k; jj++) madd(N, I.ex_weights(jj), G.lesptr(n - jj - 1, n - jj - 1), Xn);
  cplx *Qn = Q.data() + (i64)n * es;
  for (int l = 0; l <= n; l++) mm(N, dt * I.gregory_weights(n, l), N_, Sig.retptr(n, l), N_, X.data() + (i64)l * es, Qn);
  {
    const cplx *h = hmf + (i64)n * es;
    Buf hm(es);
    for (int i = 0; i < N; i++)
      for (int j = 0; j < N; j++) hm[i * N + j] = h[i * N + j] - (i == j ? mu : 0.0);
    mm(N, 1.0, N_, hm.data(), N_, Xn, Qn);
  }
  Buf Q0(es);
  adj(N, Qn, tmp.data());
  for (int e = 0; e < es; e++) Q0[e] = -cplxi * (Qn[e] + tmp[e]);
  for (int l = 1; l <= k + 1; l++) madd(N, -1. / dt * I.bd_weights(l), G.lesptr(n - l, n - l), Q0.data());
  for (int e = 0; e < es; e++) Xn[e] = Q0[e] / (1. / dt * I.bd_weights(0));
  for (int l = 0; l <= n; l++) {
    err += diffnorm(N, G.lesptr(l, n), X.data() + (i64)l * es);
    std::memcpy((void *)G.lesptr(l, n), X.data() + (i64)l * es, sizeof(cplx) * es);
  }
  return err;
}

double Dyson::dyson_step(int n, const GF &G, const GF &Sig, const cplx *hmf, double mu, double beta, double dt,
                         double *parts) {
  double e1 = dyson_step_ret(n, G, Sig, hmf, mu, dt);
  double e2 = dyson_step_tv(n, G, Sig, hmf, mu, beta, dt);
  double e3 = dyson_step_les(n, G, Sig, hmf, mu, beta, dt);
  if (parts) { parts[0] = e1; parts[1] = e2; parts[2] = e3; }
  return e1 + e2 + e3;
}

double Dyson::dyson_start(const GF &G, const GF &Sig, const cplx *hmf, double mu, double beta, double dt) {
  int N = nao_, es = es_, k = k_, kn = k * N, nt = ntau_;
  double err = 0;
  const cplx cplxi(0, 1);
  // dyson_start_tv (dyson_boot.h:93-179)
  for (int m = 0; m <= nt; m++) {
    cplx *tv = G.tvptr(0, m);
    const cplx *mat = G.matptr(nt - m);
    double s = 0;
    for (int e = 0; e < es; e++) {
      cplx v = (double)G.sig * cplxi * mat[e];
      s += std::norm(tv[e] - v);
      tv[e] = v;
    }
    err += std::sqrt(s);
  }
  // the mixing kernel of G^M is built once, before the parallel region
  const std::vector<cplx> &KM = Conv.kernel(G.matptr(0), N, beta, (double)G.sig);
  double err_tv = 0;
#pragma omp parallel for reduction(+ : err_tv) schedule(dynamic)
  for (int m = 0; m <= nt; m++) {
    Buf M((size_t)kn * kn, 0.0), Q((size_t)k * es, 0.0);
    for (int n = 1; n <= k; n++) {
      cplx *Qn = Q.data() + (i64)(n - 1) * es;
      tv_it_conv_k(m, n, Sig, KM, Qn);
      for (int l = 0; l <= k; l++) {
        int bc = (l == 0 ? 1 : l) - 1;
        if (l == 0) madd(N, -cplxi * I.poly_diff(n, l) / dt, G.tvptr(0, m), Qn);
        else for (int i = 0; i < N; i++) blk(M.data(), kn, N, n - 1, bc, i, i) += cplxi * I.poly_diff(n, l) / dt;
        if (l == n) {
          const cplx *h = hmf + (i64)l * es;
          for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++) blk(M.data(), kn, N, n - 1, bc, i, j) += (i == j ? mu : 0.0) - h[i * N + j];
        }
        if (l == 0) mm(N, dt * I.gregory_weights(n, l), N_, Sig.retptr(n, l), N_, G.tvptr(l, m), Qn);
        else {
          double w = dt * I.gregory_weights(n, l);
          if (n >= l) {
            const cplx *S = Sig.retptr(n, l);
            for (int i = 0; i < N; i++)
              for (int j = 0; j < N; j++) blk(M.data(), kn, N, n - 1, bc, i, j) -= w * S[i * N + j];
          } else {
            const cplx *S = Sig.retptr(l, n);
            for (int i = 0; i < N; i++)
              for (int j = 0; j < N; j++) blk(M.data(), kn, N, n - 1, bc, i, j) += w * std::conj(S[j * N + i]);
          }
        }
      }
    }
    lu_solve(kn, N, M.data(), Q.data());
    for (int l = 0; l < k; l++) {
      err_tv += diffnorm(N, G.tvptr(l + 1, m), Q.data() + (i64)l * es);
      std::memcpy((void *)G.tvptr(l + 1, m), Q.data() + (i64)l * es, sizeof(cplx) * es);
    }
  }
  err += err_tv;
  // dyson_start_ret (dyson_boot.h:79-88)
  Buf GR(es);
  for (int n = 0; n <= k; n++) {
    if (n == 0) {
      for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) GR[i * N + j] = i == j ? cplx(0, -1) : 0.0;
    } else {
      const cplx *a = G.tvptr(n, nt), *b = G.tvptr(n, 0);
      for (int e = 0; e < es; e++) GR[e] = (double)G.sig * a[e] - b[e];
    }
    for (int l = 0; l <= k - n; l++) {
      err += diffnorm(N, GR.data(), G.retptr(n + l, l));
      std::memcpy((void *)G.retptr(n + l, l), GR.data(), sizeof(cplx) * es);
    }
  }
  // dyson_start_les (dyson_boot.h:181-192)
  Buf tmp(es);
  for (int l = 0; l <= k; l++)
    for (int n = 0; n <= l; n++) {
      adj(N, G.tvptr(l - n, 0), tmp.data());
      double s = 0;
      for (int e = 0; e < es; e++) s += std::norm(G.lesptr(n, l)[e] + tmp[e]);
      err += std::sqrt(s);
      for (int e = 0; e < es; e++) G.lesptr(n, l)[e] = -tmp[e];
    }
  return err;
}

void Dyson::G0_from_h0(const GF &G, double mu, const double *H0, double beta, double h) const {
  int N = nao_, es = es_, k = k_;
  Buf Hmu(es), evec(es);
  std::vector<double> ev(N), evm(N);
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++) Hmu[i * N + j] = (i == j ? mu : 0.0) - H0[i * N + j];
  herm_eig(N, Hmu.data(), ev.data(), evec.data());
  for (int i = 0; i < N; i++) evm[i] = -ev[i];
  // U(dt) = exp(i h Hmu) through the eigen-decomposition
  auto vdv = [&](const std::vector<cplx> &d, cplx *out) {  // evec diag(d) evec^H
    for (int i = 0; i < N; i++)
      for (int j = 0; j < N; j++) {
        cplx s = 0;
        for (int q = 0; q < N; q++) s += evec[i * N + q] * d[q] * std::conj(evec[j * N + q]);
        out[i * N + j] = s;
      }
  };
  std::vector<cplx> d(N);
  for (int q = 0; q < N; q++) d[q] = std::exp(cplx(0, h * ev[q]));
  Buf Udt(es);
  vdv(d, Udt.data());
  std::vector<Buf> Ut(k + 1, Buf(es, 0.0));
  for (int i = 0; i < N; i++) Ut[0][i * N + i] = 1.0;
  for (int n = 1; n <= k; n++) zgemm(N_, N_, N, N, N, 1.0, Ut[n - 1].data(), N, Udt.data(), N, 0.0, Ut[n].data(), N);
  Buf tmp(es);
  for (int m = 0; m <= ntau_; m++) {
    double tau = beta / 2. * (Conv.x()[m] + 1.);
    for (int q = 0; q < N; q++) d[q] = fermi_exp(beta, tau, evm[q]);
    vdv(d, tmp.data());
    for (int n = 0; n <= k; n++) {
      cplx *dst = G.tvptr(n, m);
      std::fill(dst, dst + es, 0.0);
      zgemm(N_, N_, N, N, N, (G.sig == -1 ? cplx(0, 1) : cplx(0, -1)), Ut[n].data(), N, tmp.data(), N, 0.0, dst, N);
    }
  }
  for (int q = 0; q < N; q++) d[q] = fermi(beta, evm[q]);
  Buf value(es);
  vdv(d, value.data());
  Buf t2(es);
  for (int m = 0; m <= k; m++)
    for (int n = 0; n <= m; n++) {
      zgemm(N_, C_, N, N, N, cplx(0, -1), Ut[m].data(), N, Ut[n].data(), N, 0.0, G.retptr(m, n), N);
      zgemm(N_, N_, N, N, N, 1.0, Ut[n].data(), N, value.data(), N, 0.0, t2.data(), N);
      zgemm(N_, C_, N, N, N, cplx(0, 1), t2.data(), N, Ut[m].data(), N, 0.0, G.lesptr(n, m), N);
    }
}

} // namespace orc
