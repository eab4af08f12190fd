// CPU oracle (test infrastructure): flat C interface for ctypes.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this.
#include "oracle_integ.h"
#include "oracle_sigma.h"
#include <omp.h>
#include <exception>
#include <cstdio>

using namespace orc;

extern "C" {

typedef struct { int nt, ntau, nao, sig; void *les, *ret, *tv, *mat; } orc_gf;

static inline const GF &G_(const orc_gf *g) { return *reinterpret_cast<const GF *>(g); }
static inline cplx *Z_(void *p) { return reinterpret_cast<cplx *>(p); }
static inline const cplx *Zc_(const void *p) { return reinterpret_cast<const cplx *>(p); }

int orc_set_blas(const char *path, int threads) {
  try { set_blas(path, threads); return 0; } catch (std::exception &e) { fprintf(stderr, "%s\n", e.what()); return 1; }
}
int orc_have_blas() { return have_blas() ? 1 : 0; }
void orc_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
int orc_get_threads() { return omp_get_max_threads(); }

void orc_integrator_tables(int k, double *pi, double *pd, double *pint, double *bd, double *start, double *Om,
                           double *ex) {
  Integrator I(k);
  std::copy(I.poly_interp_tab().begin(), I.poly_interp_tab().end(), pi);
  std::copy(I.poly_diff_tab().begin(), I.poly_diff_tab().end(), pd);
  std::copy(I.poly_integ_tab().begin(), I.poly_integ_tab().end(), pint);
  std::copy(I.bd_tab().begin(), I.bd_tab().end(), bd);
  std::copy(I.start_tab().begin(), I.start_tab().end(), start);
  std::copy(I.Omega_tab().begin(), I.Omega_tab().end(), Om);
  std::copy(I.ex_tab().begin(), I.ex_tab().end(), ex);
}
double orc_gregory_weight(int k, int n, int j) {
  static thread_local Integrator *I = nullptr;
  if (!I || I->k() != k) { delete I; I = new Integrator(k); }
  return I->gregory_weights(n, j);
}
void orc_colloc_nodes(int ntau, double *x, double *w) {
  Collocation c(ntau);
  std::copy(c.x().begin(), c.x().end(), x);
  std::copy(c.w().begin(), c.w().end(), w);
}

void *orc_dyson_new(int nt, int ntau, int nao, int k) { return new Dyson(nt, ntau, nao, k); }
void orc_dyson_free(void *d) { delete static_cast<Dyson *>(d); }
#define DY static_cast<Dyson *>(d)

void orc_mixing(void *d, void *res, const void *A, const void *B, double beta, double sig) {
  DY->Conv.mixing(Z_(res), Zc_(A), Zc_(B), DY->nao_, beta, sig);
}
void orc_mixing_kernel(void *d, void *K, const void *B, double beta, double sig) {
  const std::vector<cplx> &k = DY->Conv.kernel(Zc_(B), DY->nao_, beta, sig);
  std::copy(k.begin(), k.end(), Z_(K));
}
void orc_lesser(void *d, void *res, const void *A, const void *B, double beta) {
  DY->Conv.lesser(Z_(res), Zc_(A), Zc_(B), DY->nao_, beta);
}
void orc_energy(void *d, const void *A, const void *B, double beta, double sig, double *out) {
  cplx e = DY->Conv.energy(Zc_(A), Zc_(B), DY->nao_, beta, sig);
  out[0] = e.real();
  out[1] = e.imag();
}
void orc_extrapolate(void *d, int n, const orc_gf *G) { DY->Extrapolate(n, G_(G)); }
void orc_ctv1(void *d, void *ctv, const orc_gf *A, const orc_gf *Acc, const orc_gf *B, int n, double dt) {
  DY->CTV1(Z_(ctv), G_(A), G_(Acc), G_(B), n, dt);
}
void orc_ctv_tstp(void *d, int tstp, const orc_gf *C, const orc_gf *A, const orc_gf *Acc, const orc_gf *B,
                  const orc_gf *Bcc, double beta, double dt) {
  DY->Ctv_tstp(tstp, G_(C), G_(A), G_(Acc), G_(B), G_(Bcc), beta, dt);
}
void orc_cles2(void *d, const orc_gf *A, const orc_gf *Acc, const orc_gf *B, const orc_gf *Bcc, int m, double dt,
               void *res) {
  int num = m >= DY->k_ ? m : DY->k_;
  DY->Cles2_tstp(0, num, G_(A), G_(Acc), G_(B), G_(Bcc), m, dt, Z_(res));
}
void orc_cles3(void *d, const orc_gf *A, const orc_gf *Acc, const orc_gf *B, const orc_gf *Bcc, int m, double beta,
               void *res) {
  int top = m <= DY->k_ ? DY->k_ : m;
  DY->Cles3_tstp(0, top, G_(A), G_(Acc), G_(B), G_(Bcc), m, beta, Z_(res));
}
double orc_energy_conv(void *d, int tstp, const orc_gf *Sig, const orc_gf *G, double beta, double dt) {
  return DY->energy_conv(tstp, G_(Sig), G_(G), beta, dt);
}
double orc_dyson_step(void *d, int n, const orc_gf *G, const orc_gf *Sig, const void *hmf, double mu, double beta,
                      double dt, double *parts) {
  return DY->dyson_step(n, G_(G), G_(Sig), Zc_(hmf), mu, beta, dt, parts);
}
double orc_dyson_start(void *d, const orc_gf *G, const orc_gf *Sig, const void *hmf, double mu, double beta,
                       double dt) {
  return DY->dyson_start(G_(G), G_(Sig), Zc_(hmf), mu, beta, dt);
}
void orc_g0_from_h0(void *d, const orc_gf *G, double mu, const double *H0, double beta, double dt) {
  DY->G0_from_h0(G_(G), mu, H0, beta, dt);
}
void orc_herm_eig(int n, const void *A, double *ev, void *V) { herm_eig(n, Zc_(A), ev, Z_(V)); }

void *orc_df_new(int nao, int naux, const double *Vija, const double *Viaj) {
  return new DFSolver(nao, naux, Vija, Viaj);
}
void orc_df_free(void *s) { delete static_cast<DFSolver *>(s); }
void orc_df_solve(void *s, int tstp, const orc_gf *Sig, const orc_gf *G) {
  static_cast<DFSolver *>(s)->solve(tstp, G_(Sig), G_(G));
}
void orc_df_solve_loop(void *s, int tstp, const orc_gf *Sig, const orc_gf *G) {
  static_cast<DFSolver *>(s)->solve_loop(tstp, G_(Sig), G_(G));
}
void orc_df_solve_spin(void *s, int tstp, const orc_gf *Sig, const orc_gf *G) {
  static_cast<DFSolver *>(s)->solve_spin(tstp, &G_(Sig), &G_(G));
}
void orc_df_solve_jobs(void *s, int tstp, const orc_gf *Sig, const orc_gf *G, int job_lo, int job_hi) {
  static_cast<DFSolver *>(s)->solve_jobs(tstp, G_(Sig), G_(G), job_lo, job_hi);
}
void orc_df_solve_spin_jobs(void *s, int tstp, const orc_gf *Sig, const orc_gf *G, int job_lo, int job_hi) {
  static_cast<DFSolver *>(s)->solve_spin_jobs(tstp, &G_(Sig), &G_(G), job_lo, job_hi);
}
void orc_df_solve_spin_loop(void *s, int tstp, const orc_gf *Sig, const orc_gf *G) {
  static_cast<DFSolver *>(s)->solve_spin_loop(tstp, &G_(Sig), &G_(G));
}
void *orc_full_new(int nao, const double *U, const double *Uexch) { return new FullSolver(nao, U, Uexch); }
void orc_full_free(void *s) { delete static_cast<FullSolver *>(s); }
void orc_full_solve(void *s, int tstp, const orc_gf *Sig, const orc_gf *G) {
  static_cast<FullSolver *>(s)->solve(tstp, G_(Sig), G_(G));
}
void orc_full_solve_loop(void *s, int tstp, const orc_gf *Sig, const orc_gf *G) {
  static_cast<FullSolver *>(s)->solve_loop(tstp, G_(Sig), G_(G));
}
void orc_hf_decomp(int nao, int naux, const double *Vija, void *hmf_t, const void *rho) {
  hf_decomp(nao, naux, Vija, Z_(hmf_t), Zc_(rho));
}
void orc_hf_decomp_loop(int nao, int naux, const double *Vija, void *hmf_t, const void *rho) {
  hf_decomp_loop(nao, naux, Vija, Z_(hmf_t), Zc_(rho));
}
void orc_hf_spin_decomp(int nao, int naux, const double *Vija, void *hu, void *hd, const void *rho2) {
  hf_spin_decomp(nao, naux, Vija, Z_(hu), Z_(hd), Zc_(rho2));
}
void orc_hf_spin_decomp_loop(int nao, int naux, const double *Vija, void *hu, void *hd, const void *rho2) {
  hf_spin_decomp_loop(nao, naux, Vija, Z_(hu), Z_(hd), Zc_(rho2));
}
void orc_hf_full(int nao, const double *U, void *hmf_t, const void *rho) { hf_full(nao, U, Z_(hmf_t), Zc_(rho)); }
void orc_hf_full_loop(int nao, const double *U, void *hmf_t, const void *rho) {
  hf_full_loop(nao, U, Z_(hmf_t), Zc_(rho));
}

} // extern "C"
