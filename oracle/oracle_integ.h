// CPU oracle (test infrastructure): calculus weights, Legendre collocation and
// the Dyson-step machinery.  See oracle_common.h.
#pragma once
#include "oracle_common.h"
#include <map>
#include <memory>

namespace orc {

// Restatement of Integration::Integrator (reference src/integration.h:23-124).
class Integrator {
 public:
  explicit Integrator(int k);
  int k() const { return k_; }
  double poly_interp(int a, int l) const { return poly_interp_[(size_t)a * (k_ + 1) + l]; }
  double poly_diff(int m, int l) const { return poly_diff_[(size_t)m * (k_ + 1) + l]; }
  double poly_integ(int m, int n, int l) const {
    return poly_integ_[(size_t)m * (k_ + 1) * (k_ + 1) + (size_t)n * (k_ + 1) + l];
  }
  double bd_weights(int l) const { return bd_weights_[l]; }
  double gregory_weights(int n, int j) const;
  double omega(int j) const { return Omega_[(size_t)k_ * (k_ + 1) + j]; }
  double start(int i, int j) const { return start_[(size_t)i * (k_ + 1) + j]; }
  double Omega(int i, int j) const { return Omega_[(size_t)i * (k_ + 1) + j]; }
  double ex_weights(int j) const { return ex_weights_[j]; }
  const std::vector<double> &poly_interp_tab() const { return poly_interp_; }
  const std::vector<double> &poly_diff_tab() const { return poly_diff_; }
  const std::vector<double> &poly_integ_tab() const { return poly_integ_; }
  const std::vector<double> &bd_tab() const { return bd_weights_; }
  const std::vector<double> &start_tab() const { return start_; }
  const std::vector<double> &Omega_tab() const { return Omega_; }
  const std::vector<double> &ex_tab() const { return ex_weights_; }

 private:
  int k_;
  std::vector<double> poly_interp_, poly_diff_, poly_integ_, bd_weights_, start_, Omega_, ex_weights_;
};

// Legendre collocation on the ntau+1 Legendre-Gauss-Lobatto nodes of [-1,1],
// tau = beta*(x+1)/2.  This takes the place of the external cpsitop
// `nonequilibrium::convolution` (reference call sites src/dyson.h:37,
// src/dyson.cpp:40, src/dyson_integrals.h:63,295,424).  Every operation is the
// exact integral of the degree-ntau interpolants of the sampled functions.
class Collocation {
 public:
  explicit Collocation(int ntau);
  int ntau() const { return n_; }
  const std::vector<double> &x() const { return x_; }
  const std::vector<double> &w() const { return w_; }
  const std::vector<double> &u() const { return u_; }
  double top_corr() const { return ctop_; }
  // Lagrange basis l_i(xe), i=0..ntau
  void basis(double xe, double *out) const;
  // res(tau_m) = int_0^beta A(tau) B~(tau - tau_m) dtau, B~ antiperiodic (sign sig)
  void mixing(cplx *res, const cplx *A, const cplx *B, int nao, double beta, double sig);
  // res += int_0^beta A(tau) B(tau) dtau
  void lesser(cplx *res, const cplx *A, const cplx *B, int nao, double beta) const;
  // int_0^beta sum_ij A_ij(tau) (-sig) conj(B_ij(beta - tau)) dtau
  cplx energy(const cplx *A, const cplx *B, int nao, double beta, double sig) const;
  // Mixing kernel K[m][i] (nao x nao) with res_m = sum_i A_i K[m][i]; cached per B.
  const std::vector<cplx> &kernel(const cplx *B, int nao, double beta, double sig);

 private:
  int n_;
  std::vector<double> x_, w_, u_;
  double ctop_;
  std::vector<double> EA_, EB_;  // per m: (2Q x (n+1)) evaluation matrices (weights folded in EA)
  int Q_;
  struct KEntry { uint64_t hash; int nao; double beta, sig; std::vector<cplx> K; };
  std::vector<KEntry> cache_;
  void build_eval();
};

// Restatement of NEdyson::dyson (reference src/dyson.h:17-143) for the two-time
// (non-TTI) GF2 path.
class Dyson {
 public:
  Dyson(int nt, int ntau, int nao, int k);
  const Integrator I;
  Collocation Conv;
  int nt_, ntau_, nao_, es_, k_;

  // src/dyson.cpp:47-117
  void Extrapolate(int n, const GF &G) const;
  // src/dyson_integrals.h
  void CTV1(cplx *ctv, const GF &A, const GF &Acc, const GF &B, int n, double dt) const;
  void Ctv_tstp(int tstp, const GF &C, const GF &A, const GF &Acc, const GF &B, const GF &Bcc,
                double beta, double dt);
  void Cles2_tstp(int j1, int j2, const GF &A, const GF &Acc, const GF &B, const GF &Bcc, int m,
                  double dt, cplx *res) const;
  void Cles3_tstp(int j1, int j2, const GF &A, const GF &Acc, const GF &B, const GF &Bcc, int m,
                  double beta, cplx *res);
  double energy_conv(int tstp, const GF &Sig, const GF &G, double beta, double dt);
  void tv_it_conv(int m, int n, const GF &Sig, const GF &G, double beta, cplx *res);
  void tv_it_conv_k(int m, int n, const GF &Sig, const std::vector<cplx> &K, cplx *res) const;
  // src/dyson_step.h
  double dyson_step_ret(int tstp, const GF &G, const GF &Sig, const cplx *hmf, double mu, double dt);
  double dyson_step_tv(int tstp, const GF &G, const GF &Sig, const cplx *hmf, double mu, double beta,
                       double dt);
  double dyson_step_les(int n, const GF &G, const GF &Sig, const cplx *hmf, double mu, double beta,
                        double dt);
  double dyson_step(int n, const GF &G, const GF &Sig, const cplx *hmf, double mu, double beta,
                    double dt, double *parts);
  // src/dyson_boot.h
  double dyson_start(const GF &G, const GF &Sig, const cplx *hmf, double mu, double beta, double dt);
  // src/dyson_free.h:226-297 (constant Hamiltonian)
  void G0_from_h0(const GF &G, double mu, const double *H0, double beta, double dt) const;
};

} // namespace orc
