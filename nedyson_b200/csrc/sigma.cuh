// Hot-path entry points of the engine (device work enqueued on ctx.stream).
#pragma once
#include "engine.cuh"

namespace nedy {

// molGF2SolverDecomp::solve (nspin = 1) / molGF2SolverSpinDecomp::solve (nspin = 2)
void sigma_df(Ctx &c, int T, int nspin, DevGF *const *Sig, const DevGF *const *G);
// Slices per chunk and exchange units per launch of sigma_df for a workspace budget
// (bytes); vsym: real symmetric B^Q (the all-split chain when split); np_pieces: BF16
// pieces per operand; sms: streaming multiprocessors of the device.
void chunk_plan(i64 N, i64 A, i64 budget, bool split, bool vsym, int np_pieces, int sms, int &chunk, int &sub);
// molGF2Solver::solve (full U_ijkl, restricted)
void sigma_full(Ctx &c, int T, DevGF &Sig, const DevGF &G);

// hmf(T) += HF(rho); hmf points at the nao x nao block of time T.
// molHFSolverDecomp::solve_HF (nspin = 1) / molHFSolverSpinDecomp::solve_HF (nspin = 2: rho[2], hmf[2])
void hf_decomp(Ctx &c, int nspin, double2 *const *hmf_T, const double2 *rho);
// molHFSolver::solve_HF (full U)
void hf_full(Ctx &c, double2 *hmf_T, const double2 *rho);
// rho = i*sig*G^<(T,T) (greens.h:68-74), device to device
void get_dm(Ctx &c, const DevGF &G, int T, double2 *rho);

// dyson::Extrapolate (dyson.cpp:47-117)
void extrapolate(Ctx &c, int n, DevGF &G);
// calculus tables (Gregory, BDF, extrapolation weights) on the device
void ensure_tables(Ctx &c);
// dyson::dyson_step (dyson_step.h:329-382); hmf: (nt+1) x nao x nao on the device.
// Returns the sum of the three component errors (ret, tv, les) when err != nullptr.
void dyson_step(Ctx &c, int n, DevGF &G, const DevGF &Sig, const double2 *hmf, double mu, double *err);
// The Dyson steps of both spins of an unrestricted step, side by side: spin 0 on c's stream,
// spin 1 on the stream of c's second context from a helper thread; c's stream continues
// after both.
void dyson_step_spins(Ctx &c, int n, DevGF &G0, const DevGF &S0, const double2 *h0, double mu0, double *e0,
                      DevGF &G1, const DevGF &S1, const double2 *h1, double mu1, double *e1);
// dyson::dyson_start (dyson_boot.h:195-230)
double dyson_start(Ctx &c, DevGF &G, const DevGF &Sig, const double2 *hmf, double mu);
// dyson::energy_conv (dyson_integrals.h:24-70)
double energy_conv(Ctx &c, int T, const DevGF &Sig, const DevGF &G);
// Mixing kernel of G^M (rebuilt when G^M changes)
void ensure_mixing_kernel(Ctx &c, const DevGF &G);
// Kernel of the imaginary-time integral int_0^beta f(tau') B(tau' - tau_m) dtau' = sum_i f_i K[m][i]
// for nodal blocks Bn (np x N x N) extended by B(x) = sig B(x + beta); K: np x np x N x N
void build_tau_kernel(Ctx &c, const double2 *Bn, int N, double sig, double2 *K);
// Cached inverse of the time-local Dyson matrix for times [t0, t1] (after their rows are final)
void update_minv(Ctx &c, const DevGF &Sig, const double2 *hmf, double mu, int t0, int t1);
// X = A^-1 B for nb systems (A n x n at stride sA, B n x nrhs at stride sB, row-major) by
// Gauss-Jordan with partial pivoting; B is overwritten.  A zero pivot is reported by
// check_status, which also waits for the device.
void gj_public(Ctx &c, int n, int nrhs, int nb, double2 *A, i64 sA, double2 *B, i64 sB);
void check_status(Ctx &c);

} // namespace nedy
