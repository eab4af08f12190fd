// CPU oracle (test infrastructure): GF2 self-energy and HF solvers.  See sigma.cpp.
#pragma once
#include "oracle_common.h"

namespace orc {

// molGF2SolverDecomp / molGF2SolverSpinDecomp (reference src/mol2bSolver.h:19-129).
// Vija is (nao,nao,naux) row-major, Viaj = (nao,naux,nao) with Viaj(i,a,j) = Vija(i,j,a).
struct DFSolver {
  DFSolver(int nao, int naux, const double *Vija, const double *Viaj);
  int nao_, naux_;
  std::vector<double> Vija_, Viaj_;
  std::vector<cplx> VijaC_, ViajC_;
  void solve(int tstp, const GF &Sig, const GF &G) const;
  // slices [job_lo, job_hi) of the restricted row (lesser t, retarded t, mixed tau), not zeroed first
  void solve_jobs(int tstp, const GF &Sig, const GF &G, int job_lo, int job_hi) const;
  void solve_loop(int tstp, const GF &Sig, const GF &G) const;
  void solve_spin(int tstp, const GF *Sig, const GF *G) const;       // Sig[2], G[2]
  // slices [job_lo, job_hi) of the unrestricted row, Sigma not zeroed first
  void solve_spin_jobs(int tstp, const GF *Sig, const GF *G, int job_lo, int job_hi) const;
  void solve_spin_loop(int tstp, const GF *Sig, const GF *G) const;
};

// molGF2Solver (reference src/mol2bSolver.h:178-209).  U, Uexch: (nao)^4 row-major.
struct FullSolver {
  FullSolver(int nao, const double *U, const double *Uexch);
  int nao_;
  std::vector<double> U_, Uexch_;
  std::vector<cplx> UC_, UexchC_;
  void solve(int tstp, const GF &Sig, const GF &G) const;
  void solve_loop(int tstp, const GF &Sig, const GF &G) const;
};

void hf_decomp(int nao, int naux, const double *Vija, cplx *hmf_t, const cplx *rho);
void hf_decomp_loop(int nao, int naux, const double *Vija, cplx *hmf_t, const cplx *rho);
void hf_spin_decomp(int nao, int naux, const double *Vija, cplx *hmf_up, cplx *hmf_dn, const cplx *rho2);
void hf_spin_decomp_loop(int nao, int naux, const double *Vija, cplx *hmf_up, cplx *hmf_dn, const cplx *rho2);
void hf_full(int nao, const double *U, cplx *hmf_t, const cplx *rho);
void hf_full_loop(int nao, const double *U, cplx *hmf_t, const cplx *rho);

} // namespace orc
