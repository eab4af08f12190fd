// CPU oracle (test infrastructure): second-Born (GF2) self-energies and the
// Hartree-Fock mean field.
//
//   DF restricted      : reference src/mol2bSolver_decomp_impl.h (chain :6-429, loops :431-670)
//   DF unrestricted    : reference src/mol2bSolver_spin_decomp_impl.h (chain :9-466, loops :468-738)
//   full-U restricted  : reference src/mol2bSolver_impl.h (chain :5-182, loops :186-285)
//   HF                 : reference src/molHFSolver.cpp (:13-110 restricted, :173-239 spin)
//
// The "chain" functions follow the reference's contraction order one product at
// a time; the "loop" functions are the reference's brute-force definitions.
// Slices (t' or tau) are independent and run on OpenMP threads.
#include "oracle_sigma.h"
#include <omp.h>
#include <algorithm>

namespace orc {

namespace {
// M[r][c] -> out[c][r] for a rows x cols block
inline void tpose(const cplx *in, int rows, int cols, cplx *out) {
  for (int r = 0; r < rows; r++)
    for (int c = 0; c < cols; c++) out[(i64)c * rows + r] = in[(i64)r * cols + c];
}
// For each of `nb` blocks of (rows x cols), transpose into (cols x rows).
inline void tpose_blocks(const cplx *in, int nb, int rows, int cols, cplx *out) {
  i64 bs = (i64)rows * cols;
  for (int b = 0; b < nb; b++) tpose(in + b * bs, rows, cols, out + b * bs);
}
inline void conjm(const cplx *in, i64 n, cplx *out, double f = 1.0) {
  for (i64 i = 0; i < n; i++) out[i] = f * std::conj(in[i]);
}
} // namespace

DFSolver::DFSolver(int nao, int naux, const double *Vija, const double *Viaj)
    : nao_(nao), naux_(naux), Vija_(Vija, Vija + (size_t)nao * nao * naux),
      Viaj_(Viaj, Viaj + (size_t)nao * nao * naux) {
  VijaC_.assign(Vija_.begin(), Vija_.end());
  ViajC_.assign(Viaj_.begin(), Viaj_.end());
}

struct DFScratch {
  std::vector<cplx> X1, X2, X3, Y1, Y2, P1, P2, Z, g1, g2;
  DFScratch(int n, int a, int ns) {
    size_t nna = (size_t)n * n * a * ns;
    X1.resize(nna); X2.resize(nna); X3.resize(nna); Y1.resize(nna); Y2.resize(nna);
    P1.resize((size_t)a * a); P2.resize((size_t)a * a);
    Z.resize((size_t)n * n * n * n);
    g1.resize((size_t)n * n); g2.resize((size_t)n * n);
  }
};

// ---------------- restricted DF: bubble ----------------
// les/tv share one form: (Gf = G, Gb = "backward" matrix already formed)
// mol2bSolver_decomp_impl.h:6-49 (les) and :51-91 (tv)
static void df_bubble_lesform(const DFSolver &s, const cplx *Gf, const cplx *Gb, cplx *Sig,
                              DFScratch &w, double fac) {
  int n = s.nao_, a = s.naux_, naa = n * a, n2 = n * n;
  rzgemm(naa, n, n, 1.0, s.Viaj_.data(), n, Gf, n, 0.0, w.X1.data(), n);      // X_naq = V_nap G_pq
  tpose_blocks(w.X1.data(), n, a, n, w.Y1.data());                           // Y_nqa
  zgemm(N, T, n, naa, n, 1.0, Gb, n, s.ViajC_.data(), n, 0.0, w.X1.data(), naa);  // X_nqb = Gb V^T
  zgemm(T, N, a, a, n2, 1.0, w.Y1.data(), a, w.X1.data(), a, 0.0, w.P1.data(), a);  // P = Y^T X
  zgemm(N, T, n2, a, a, 1.0, s.VijaC_.data(), a, w.P1.data(), a, 0.0, w.X1.data(), a);  // Z_kja
  tpose_blocks(w.X1.data(), n, n, a, w.X2.data());                           // Z_kaj
  zgemm(N, N, n, n, naa, fac, w.Y1.data(), naa, w.X2.data(), n, 1.0, Sig, n);
}

// mol2bSolver_decomp_impl.h:94-172
static void df_bubble_ret(const DFSolver &s, const cplx *L, const cplx *R, cplx *Sig, DFScratch &w) {
  int n = s.nao_, a = s.naux_, naa = n * a, n2 = n * n;
  zgemm(N, C, naa, n, n, -1.0, s.ViajC_.data(), n, L, n, 0.0, w.X1.data(), n);
  rzgemm(naa, n, n, 1.0, s.Viaj_.data(), n, R, n, 0.0, w.X2.data(), n);
  tpose_blocks(w.X1.data(), n, a, n, w.Y1.data());
  tpose_blocks(w.X2.data(), n, a, n, w.Y2.data());
  conjm(R, n2, w.g1.data());
  zgemm(N, T, n, naa, n, 1.0, w.g1.data(), n, s.ViajC_.data(), n, 0.0, w.X1.data(), naa);
  zgemm(T, T, n, naa, n, 1.0, L, n, s.ViajC_.data(), n, 0.0, w.X2.data(), naa);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) w.g2[i * n + j] = L[j * n + i] - std::conj(R[i * n + j]);
  zgemm(N, T, n, naa, n, 1.0, w.g2.data(), n, s.ViajC_.data(), n, 0.0, w.X3.data(), naa);
  zgemm(T, N, a, a, n2, 1.0, w.Y1.data(), a, w.X3.data(), a, 0.0, w.P1.data(), a);
  zgemm(T, N, a, a, n2, 1.0, w.Y2.data(), a, w.X2.data(), a, 0.0, w.P2.data(), a);
  zgemm(T, N, a, a, n2, 1.0, w.Y1.data(), a, w.X1.data(), a, 1.0, w.P2.data(), a);
  zgemm(N, T, n2, a, a, 1.0, s.VijaC_.data(), a, w.P1.data(), a, 0.0, w.X1.data(), a);
  zgemm(N, T, n2, a, a, 1.0, s.VijaC_.data(), a, w.P2.data(), a, 0.0, w.X2.data(), a);
  for (int k = 0; k < n; k++) {
    tpose(w.X2.data() + (i64)k * naa, n, a, w.X3.data() + (i64)k * naa);
    tpose(w.X1.data() + (i64)k * naa, n, a, w.X2.data() + (i64)k * naa);
  }
  zgemm(N, N, n, n, naa, 2.0, w.Y2.data(), naa, w.X3.data(), n, 1.0, Sig, n);
  zgemm(N, N, n, n, naa, 2.0, w.Y1.data(), naa, w.X3.data(), n, 1.0, Sig, n);
  zgemm(N, N, n, n, naa, 2.0, w.Y2.data(), naa, w.X2.data(), n, 1.0, Sig, n);
}

// ---------------- restricted DF: exchange ----------------
// les/tv form: mol2bSolver_decomp_impl.h:182-233 (les), :236-289 (tv)
static void df_exch_lesform(const DFSolver &s, const cplx *Gf, const cplx *Gb, cplx *Sig, DFScratch &w) {
  int n = s.nao_, a = s.naux_, naa = n * a, n2 = n * n, n3 = n2 * n;
  zgemm(N, T, n, naa, n, 1.0, Gb, n, s.ViajC_.data(), n, 0.0, w.X1.data(), naa);  // X_nkb
  tpose_blocks(w.X1.data(), n, n, a, w.X2.data());                            // X_nbk
  zgemm(N, T, naa, n, n, 1.0, w.X2.data(), n, Gf, n, 0.0, w.X1.data(), n);        // X_nbl = X_nbk G^T_kl
  for (int q = 0; q < n; q++)
    rzgemm(n2, n, a, 1.0, s.Vija_.data(), a, w.X1.data() + (i64)q * naa, n, 0.0, w.Z.data() + (i64)q * n3, n);
  rzgemm(naa, n, n, 1.0, s.Viaj_.data(), n, Gf, n, 0.0, w.Y1.data(), n);       // Y_naq
  tpose_blocks(w.Y1.data(), n, a, n, w.Y2.data());                            // Y_nqa
  zgemm(T, N, n2, a, n2, 1.0, w.Z.data(), n2, w.Y2.data(), a, 0.0, w.X1.data(), a);  // X_jla
  zgemm(N, T, n, n, naa, -1.0, s.VijaC_.data(), naa, w.X1.data(), naa, 1.0, Sig, n);
}

// mol2bSolver_decomp_impl.h:293-402
static void df_exch_ret(const DFSolver &s, const cplx *L, const cplx *R, cplx *Sig, DFScratch &w) {
  int n = s.nao_, a = s.naux_, naa = n * a, n2 = n * n, n3 = n2 * n;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) w.g1[i * n + j] = -std::conj(R[i * n + j]) + L[j * n + i];
  zgemm(N, T, n, naa, n, 1.0, w.g1.data(), n, s.ViajC_.data(), n, 0.0, w.X2.data(), naa);
  tpose_blocks(w.X2.data(), n, n, a, w.Y1.data());      // X^>_nbk
  zgemm(T, T, n, naa, n, 1.0, L, n, s.ViajC_.data(), n, 0.0, w.X2.data(), naa);
  tpose_blocks(w.X2.data(), n, n, a, w.Y2.data());      // X^<_nbk
  conjm(R, n2, w.g1.data());
  zgemm(N, T, n, naa, n, 1.0, w.g1.data(), n, s.ViajC_.data(), n, 0.0, w.X2.data(), naa);
  tpose_blocks(w.X2.data(), n, n, a, w.X3.data());      // X^A_nbk
  conjm(L, n2, w.g2.data());
  zgemm(N, N, naa, n, n, -1.0, w.Y1.data(), n, w.g2.data(), n, 0.0, w.X1.data(), n);   // ~X^<
  zgemm(N, T, naa, n, n, 1.0, w.Y2.data(), n, R, n, 0.0, w.X2.data(), n);              // ~X^R
  zgemm(N, N, naa, n, n, -1.0, w.X3.data(), n, w.g2.data(), n, 1.0, w.X2.data(), n);
  zgemm(N, C, naa, n, n, -1.0, s.ViajC_.data(), n, L, n, 0.0, w.X3.data(), n);
  tpose_blocks(w.X3.data(), n, a, n, w.Y1.data());      // Y^<_nqa
  rzgemm(naa, n, n, 1.0, s.Viaj_.data(), n, R, n, 0.0, w.X3.data(), n);
  tpose_blocks(w.X3.data(), n, a, n, w.Y2.data());      // Y^R_nqa
  for (int q = 0; q < n; q++)
    rzgemm(n2, n, a, 1.0, s.Vija_.data(), a, w.X1.data() + (i64)q * naa, n, 0.0, w.Z.data() + (i64)q * n3, n);
  zgemm(T, N, n2, a, n2, 1.0, w.Z.data(), n2, w.Y2.data(), a, 0.0, w.X3.data(), a);
  for (int q = 0; q < n; q++)
    rzgemm(n2, n, a, 1.0, s.Vija_.data(), a, w.X2.data() + (i64)q * naa, n, 0.0, w.Z.data() + (i64)q * n3, n);
  for (size_t e = 0; e < (size_t)n2 * a; e++) w.Y1[e] += w.Y2[e];
  zgemm(T, N, n2, a, n2, 1.0, w.Z.data(), n2, w.Y1.data(), a, 1.0, w.X3.data(), a);
  zgemm(N, T, n, n, naa, -1.0, s.VijaC_.data(), naa, w.X3.data(), naa, 1.0, Sig, n);
}

// Build the "backward" matrix of a les/tv slice.
static void les_back(int n, const cplx *L, const cplx *R, cplx *out) {  // R^T - conj(L)
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) out[i * n + j] = R[j * n + i] - std::conj(L[i * n + j]);
}
static void tv_back(int n, const cplx *Gvt, int sig, cplx *out) {  // -sig conj(G^tv(ntau-t))
  for (int e = 0; e < n * n; e++) out[e] = -(double)sig * std::conj(Gvt[e]);
}

// mol2bSolver_decomp_impl.h:412-429
void DFSolver::solve(int tstp, const GF &Sig, const GF &G) const {
  Sig.set_tstp_zero(tstp);
  solve_jobs(tstp, Sig, G, 0, 2 * (tstp + 1) + G.ntau + 1);
}

// Slices job_lo .. job_hi-1 of the restricted row, numbered as in solve_spin_jobs.
void DFSolver::solve_jobs(int tstp, const GF &Sig, const GF &G, int job_lo, int job_hi) const {
  int n = nao_, ntau = G.ntau, sig = G.sig;
  int nles = tstp + 1, ntv = ntau + 1;
  job_lo = std::max(0, job_lo);
  job_hi = std::min(2 * nles + ntv, job_hi);
#pragma omp parallel
  {
    DFScratch w(n, naux_, 1);
    std::vector<cplx> gb((size_t)n * n);
#pragma omp for schedule(dynamic)
    for (int job = job_lo; job < job_hi; job++) {
      if (job < nles) {
        int t = job;
        les_back(n, G.lesptr(t, tstp), G.retptr(tstp, t), gb.data());
        df_bubble_lesform(*this, G.lesptr(t, tstp), gb.data(), Sig.lesptr(t, tstp), w, 2.0);
        df_exch_lesform(*this, G.lesptr(t, tstp), gb.data(), Sig.lesptr(t, tstp), w);
      } else if (job < 2 * nles) {
        int t = job - nles;
        df_bubble_ret(*this, G.lesptr(t, tstp), G.retptr(tstp, t), Sig.retptr(tstp, t), w);
        df_exch_ret(*this, G.lesptr(t, tstp), G.retptr(tstp, t), Sig.retptr(tstp, t), w);
      } else {
        int t = job - 2 * nles;
        tv_back(n, G.tvptr(tstp, ntau - t), sig, gb.data());
        df_bubble_lesform(*this, G.tvptr(tstp, t), gb.data(), Sig.tvptr(tstp, t), w, 2.0);
        df_exch_lesform(*this, G.tvptr(tstp, t), gb.data(), Sig.tvptr(tstp, t), w);
      }
    }
  }
}

// mol2bSolver_decomp_impl.h:431-670 (brute force definition)
void DFSolver::solve_loop(int tstp, const GF &Sig, const GF &G) const {
  Sig.set_tstp_zero(tstp);
  int n = nao_, na = naux_, sig = G.sig, ntau = G.ntau;
  auto V = [&](int i, int j, int a) { return Vija_[((size_t)i * n + j) * na + a]; };
  // contraction with slot values X_lk, Y_mn, Z_pq; bubble factor fb, exchange sign
  auto tri = [&](const cplx *X, const cplx *Y, const cplx *Z, cplx *out, double fb) {
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        cplx acc = 0;
        for (int l = 0; l < n; l++)
          for (int nn = 0; nn < n; nn++)
            for (int p = 0; p < n; p++)
              for (int k = 0; k < n; k++)
                for (int q = 0; q < n; q++)
                  for (int m = 0; m < n; m++) {
                    cplx g = X[l * n + k] * Y[m * n + nn] * Z[p * n + q];
                    double vb = 0, ve = 0;
                    for (int a = 0; a < na; a++)
                      for (int b = 0; b < na; b++) {
                        vb += V(i, l, a) * V(nn, p, a) * V(k, j, b) * V(q, m, b);
                        ve += V(i, l, a) * V(nn, p, a) * V(q, j, b) * V(k, m, b);
                      }
                    acc += (fb * vb - ve) * g;
                  }
        out[i * n + j] += acc;
      }
  };
  std::vector<cplx> Y((size_t)n * n), Lh((size_t)n * n), Rh((size_t)n * n), Zd((size_t)n * n);
  for (int t = 0; t <= tstp; t++) {
    const cplx *L = G.lesptr(t, tstp), *R = G.retptr(tstp, t);
    for (int m = 0; m < n; m++)
      for (int nn = 0; nn < n; nn++) {
        Y[m * n + nn] = R[m * n + nn] - std::conj(L[nn * n + m]);  // G^>(T,t)
        Lh[m * n + nn] = std::conj(L[nn * n + m]);                 // L^dagger
        Rh[m * n + nn] = std::conj(R[nn * n + m]);                 // R^dagger
        Zd[m * n + nn] = R[m * n + nn] - Lh[m * n + nn];
      }
    tri(L, Y.data(), L, Sig.lesptr(t, tstp), 2.0);
    // retarded: (R,L,R-L^+) + (L^+,R^+,L^+) - (L^+,L,R)
    std::vector<cplx> tmp((size_t)n * n, 0.0);
    tri(R, L, Zd.data(), Sig.retptr(tstp, t), 2.0);
    tri(Lh.data(), Rh.data(), Lh.data(), Sig.retptr(tstp, t), 2.0);
    tri(Lh.data(), L, R, tmp.data(), 2.0);
    for (int e = 0; e < n * n; e++) Sig.retptr(tstp, t)[e] -= tmp[e];
  }
  for (int t = 0; t <= ntau; t++) {
    const cplx *Gt = G.tvptr(tstp, t), *Gv = G.tvptr(tstp, ntau - t);
    for (int m = 0; m < n; m++)
      for (int nn = 0; nn < n; nn++) Y[m * n + nn] = -(double)sig * std::conj(Gv[nn * n + m]);
    tri(Gt, Y.data(), Gt, Sig.tvptr(tstp, t), 2.0);
  }
}

// ---------------- unrestricted DF ----------------
// bubble les/tv form: mol2bSolver_spin_decomp_impl.h:9-60 (les), :62-110 (tv)
static void sdf_bubble_lesform(const DFSolver &s, const cplx *Gf[2], const cplx *Gb[2], cplx *Sig[2],
                               DFScratch &w) {
  int n = s.nao_, a = s.naux_, naa = n * a, n2 = n * n;
  size_t off = (size_t)n2 * a;
  for (int sp = 0; sp < 2; sp++) {
    rzgemm(naa, n, n, 1.0, s.Viaj_.data(), n, Gf[sp], n, 0.0, w.X1.data() + sp * off, n);
    tpose_blocks(w.X1.data() + sp * off, n, a, n, w.Y1.data() + sp * off);
    zgemm(N, T, n, naa, n, 1.0, Gb[sp], n, s.ViajC_.data(), n, 0.0, w.X1.data() + sp * off, naa);
  }
  zgemm(T, N, a, a, 2 * n2, 1.0, w.Y1.data(), a, w.X1.data(), a, 0.0, w.P1.data(), a);
  zgemm(N, T, n2, a, a, 1.0, s.VijaC_.data(), a, w.P1.data(), a, 0.0, w.X1.data(), a);
  tpose_blocks(w.X1.data(), n, n, a, w.X2.data());
  for (int sp = 0; sp < 2; sp++)
    zgemm(N, N, n, n, naa, 1.0, w.Y1.data() + sp * off, naa, w.X2.data(), n, 1.0, Sig[sp], n);
}

// mol2bSolver_spin_decomp_impl.h:113-199
static void sdf_bubble_ret(const DFSolver &s, const cplx *L[2], const cplx *R[2], cplx *Sig[2], DFScratch &w) {
  int n = s.nao_, a = s.naux_, naa = n * a, n2 = n * n;
  size_t off = (size_t)n2 * a;
  for (int sp = 0; sp < 2; sp++) {
    zgemm(N, C, naa, n, n, -1.0, s.ViajC_.data(), n, L[sp], n, 0.0, w.X1.data() + sp * off, n);
    rzgemm(naa, n, n, 1.0, s.Viaj_.data(), n, R[sp], n, 0.0, w.X2.data() + sp * off, n);
    tpose_blocks(w.X1.data() + sp * off, n, a, n, w.Y1.data() + sp * off);
    tpose_blocks(w.X2.data() + sp * off, n, a, n, w.Y2.data() + sp * off);
  }
  for (int sp = 0; sp < 2; sp++) {
    conjm(R[sp], n2, w.g1.data());
    zgemm(N, T, n, naa, n, 1.0, w.g1.data(), n, s.ViajC_.data(), n, 0.0, w.X1.data() + sp * off, naa);
    zgemm(T, T, n, naa, n, 1.0, L[sp], n, s.ViajC_.data(), n, 0.0, w.X2.data() + sp * off, naa);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) w.g2[i * n + j] = L[sp][j * n + i] - std::conj(R[sp][i * n + j]);
    zgemm(N, T, n, naa, n, 1.0, w.g2.data(), n, s.ViajC_.data(), n, 0.0, w.X3.data() + sp * off, naa);
  }
  zgemm(T, N, a, a, 2 * n2, 1.0, w.Y1.data(), a, w.X3.data(), a, 0.0, w.P1.data(), a);
  zgemm(T, N, a, a, 2 * n2, 1.0, w.Y2.data(), a, w.X2.data(), a, 0.0, w.P2.data(), a);
  zgemm(T, N, a, a, 2 * n2, 1.0, w.Y1.data(), a, w.X1.data(), a, 1.0, w.P2.data(), a);
  zgemm(N, T, n2, a, a, 1.0, s.VijaC_.data(), a, w.P1.data(), a, 0.0, w.X1.data(), a);
  zgemm(N, T, n2, a, a, 1.0, s.VijaC_.data(), a, w.P2.data(), a, 0.0, w.X2.data(), a);
  for (int k = 0; k < n; k++) {
    tpose(w.X1.data() + (i64)k * naa, n, a, w.X1.data() + off + (i64)k * naa);
    tpose(w.X2.data() + (i64)k * naa, n, a, w.X2.data() + off + (i64)k * naa);
  }
  for (int sp = 0; sp < 2; sp++) {
    zgemm(N, N, n, n, naa, 1.0, w.Y2.data() + sp * off, naa, w.X2.data() + off, n, 1.0, Sig[sp], n);
    zgemm(N, N, n, n, naa, 1.0, w.Y1.data() + sp * off, naa, w.X2.data() + off, n, 1.0, Sig[sp], n);
    zgemm(N, N, n, n, naa, 1.0, w.Y2.data() + sp * off, naa, w.X1.data() + off, n, 1.0, Sig[sp], n);
  }
}

// mol2bSolver_spin_decomp_impl.h:436-466
void DFSolver::solve_spin(int tstp, const GF *Sig, const GF *G) const {
  Sig[0].set_tstp_zero(tstp);
  Sig[1].set_tstp_zero(tstp);
  solve_spin_jobs(tstp, Sig, G, 0, 2 * (tstp + 1) + G[0].ntau + 1);
}

// Slices job_lo .. job_hi-1 of the unrestricted row (both spins of one slice per job):
// jobs [0, tstp] lesser slices t, [tstp+1, 2 tstp+1] retarded slices, then the ntau+1
// mixed slices.  Every slice is an independent piece of the reference's row
// (mol2bSolver_spin_decomp_impl.h:436-466), so a row can be computed -- or timed -- in parts.
void DFSolver::solve_spin_jobs(int tstp, const GF *Sig, const GF *G, int job_lo, int job_hi) const {
  int n = nao_, ntau = G[0].ntau, sig = G[0].sig;
  int nles = tstp + 1, ntv = ntau + 1;
  job_lo = std::max(0, job_lo);
  job_hi = std::min(2 * nles + ntv, job_hi);
#pragma omp parallel
  {
    DFScratch w(n, naux_, 2);
    std::vector<cplx> gb0((size_t)n * n), gb1((size_t)n * n);
#pragma omp for schedule(dynamic)
    for (int job = job_lo; job < job_hi; job++) {
      if (job < nles) {
        int t = job;
        const cplx *Gf[2] = {G[0].lesptr(t, tstp), G[1].lesptr(t, tstp)};
        les_back(n, Gf[0], G[0].retptr(tstp, t), gb0.data());
        les_back(n, Gf[1], G[1].retptr(tstp, t), gb1.data());
        const cplx *Gb[2] = {gb0.data(), gb1.data()};
        cplx *S[2] = {Sig[0].lesptr(t, tstp), Sig[1].lesptr(t, tstp)};
        sdf_bubble_lesform(*this, Gf, Gb, S, w);
        for (int s = 0; s < 2; s++) df_exch_lesform(*this, Gf[s], Gb[s], S[s], w);
      } else if (job < 2 * nles) {
        int t = job - nles;
        const cplx *L[2] = {G[0].lesptr(t, tstp), G[1].lesptr(t, tstp)};
        const cplx *R[2] = {G[0].retptr(tstp, t), G[1].retptr(tstp, t)};
        cplx *S[2] = {Sig[0].retptr(tstp, t), Sig[1].retptr(tstp, t)};
        sdf_bubble_ret(*this, L, R, S, w);
        for (int s = 0; s < 2; s++) df_exch_ret(*this, L[s], R[s], S[s], w);
      } else {
        int t = job - 2 * nles;
        const cplx *Gf[2] = {G[0].tvptr(tstp, t), G[1].tvptr(tstp, t)};
        tv_back(n, G[0].tvptr(tstp, ntau - t), sig, gb0.data());
        tv_back(n, G[1].tvptr(tstp, ntau - t), sig, gb1.data());
        const cplx *Gb[2] = {gb0.data(), gb1.data()};
        cplx *S[2] = {Sig[0].tvptr(tstp, t), Sig[1].tvptr(tstp, t)};
        sdf_bubble_lesform(*this, Gf, Gb, S, w);
        for (int s = 0; s < 2; s++) df_exch_lesform(*this, Gf[s], Gb[s], S[s], w);
      }
    }
  }
}

// mol2bSolver_spin_decomp_impl.h:468-738 (brute force definition)
void DFSolver::solve_spin_loop(int tstp, const GF *Sig, const GF *G) const {
  Sig[0].set_tstp_zero(tstp);
  Sig[1].set_tstp_zero(tstp);
  int n = nao_, na = naux_, sig = G[0].sig, ntau = G[0].ntau;
  auto V = [&](int i, int j, int a) { return Vija_[((size_t)i * n + j) * na + a]; };
  // bubble: X from spin s, (Y,Z) from spin sp, summed over sp; exchange: all from spin s
  auto bub = [&](const cplx *X, const cplx *Y, const cplx *Z, cplx *out) {
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        cplx acc = 0;
        for (int l = 0; l < n; l++) for (int nn = 0; nn < n; nn++) for (int p = 0; p < n; p++)
          for (int k = 0; k < n; k++) for (int q = 0; q < n; q++) for (int m = 0; m < n; m++) {
            double vb = 0;
            for (int a = 0; a < na; a++) for (int b = 0; b < na; b++)
              vb += V(i, l, a) * V(nn, p, a) * V(k, j, b) * V(q, m, b);
            acc += vb * X[l * n + k] * Y[m * n + nn] * Z[p * n + q];
          }
        out[i * n + j] += acc;
      }
  };
  auto exc = [&](const cplx *X, const cplx *Y, const cplx *Z, cplx *out) {
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        cplx acc = 0;
        for (int l = 0; l < n; l++) for (int nn = 0; nn < n; nn++) for (int p = 0; p < n; p++)
          for (int k = 0; k < n; k++) for (int q = 0; q < n; q++) for (int m = 0; m < n; m++) {
            double ve = 0;
            for (int a = 0; a < na; a++) for (int b = 0; b < na; b++)
              ve += V(i, l, a) * V(nn, p, a) * V(q, j, b) * V(k, m, b);
            acc += ve * X[l * n + k] * Y[m * n + nn] * Z[p * n + q];
          }
        out[i * n + j] -= acc;
      }
  };
  size_t e2 = (size_t)n * n;
  std::vector<cplx> Yg(2 * e2), Lh(2 * e2), Rh(2 * e2), Zd(2 * e2), Yt(2 * e2), tmp(e2);
  for (int t = 0; t <= tstp; t++) {
    const cplx *L[2] = {G[0].lesptr(t, tstp), G[1].lesptr(t, tstp)};
    const cplx *R[2] = {G[0].retptr(tstp, t), G[1].retptr(tstp, t)};
    for (int s = 0; s < 2; s++)
      for (int m = 0; m < n; m++)
        for (int nn = 0; nn < n; nn++) {
          Yg[s * e2 + m * n + nn] = R[s][m * n + nn] - std::conj(L[s][nn * n + m]);
          Lh[s * e2 + m * n + nn] = std::conj(L[s][nn * n + m]);
          Rh[s * e2 + m * n + nn] = std::conj(R[s][nn * n + m]);
          Zd[s * e2 + m * n + nn] = R[s][m * n + nn] - Lh[s * e2 + m * n + nn];
        }
    for (int s = 0; s < 2; s++) {
      cplx *SL = Sig[s].lesptr(t, tstp), *SR = Sig[s].retptr(tstp, t);
      for (int sp = 0; sp < 2; sp++) {
        bub(L[s], &Yg[sp * e2], L[sp], SL);
        bub(R[s], L[sp], &Zd[sp * e2], SR);
        bub(&Lh[s * e2], &Rh[sp * e2], &Lh[sp * e2], SR);
        std::fill(tmp.begin(), tmp.end(), 0.0);
        bub(&Lh[s * e2], L[sp], R[sp], tmp.data());
        for (size_t e = 0; e < e2; e++) SR[e] -= tmp[e];
      }
      exc(L[s], &Yg[s * e2], L[s], SL);
      exc(R[s], L[s], &Zd[s * e2], SR);
      exc(&Lh[s * e2], &Rh[s * e2], &Lh[s * e2], SR);
      std::fill(tmp.begin(), tmp.end(), 0.0);
      exc(&Lh[s * e2], L[s], R[s], tmp.data());
      for (size_t e = 0; e < e2; e++) SR[e] -= tmp[e];
    }
  }
  for (int t = 0; t <= ntau; t++) {
    const cplx *Gt[2] = {G[0].tvptr(tstp, t), G[1].tvptr(tstp, t)};
    for (int s = 0; s < 2; s++) {
      const cplx *Gv = G[s].tvptr(tstp, ntau - t);
      for (int m = 0; m < n; m++)
        for (int nn = 0; nn < n; nn++) Yt[s * e2 + m * n + nn] = -(double)sig * std::conj(Gv[nn * n + m]);
    }
    for (int s = 0; s < 2; s++) {
      cplx *ST = Sig[s].tvptr(tstp, t);
      for (int sp = 0; sp < 2; sp++) bub(Gt[s], &Yt[sp * e2], Gt[sp], ST);
      exc(Gt[s], &Yt[s * e2], Gt[s], ST);
    }
  }
}

// ---------------- full U ----------------
FullSolver::FullSolver(int nao, const double *U, const double *Uexch)
    : nao_(nao), U_(U, U + (size_t)nao * nao * nao * nao), Uexch_(Uexch, Uexch + (size_t)nao * nao * nao * nao) {
  UC_.assign(U_.begin(), U_.end());
  UexchC_.assign(Uexch_.begin(), Uexch_.end());
}

// mol2bSolver_impl.h:5-182
void FullSolver::solve(int tstp, const GF &Sig, const GF &G) const {
  Sig.set_tstp_zero(tstp);
  int n = nao_, n2 = n * n, n3 = n2 * n, ntau = G.ntau, sig = G.sig;
  int nles = tstp + 1, ntv = ntau + 1;
  // row i of Sigma += Uexch_{j,(qkm)} A_{(qkm)}
  auto contract = [&](const cplx *A1, cplx *Srow) {
    for (int j = 0; j < n; j++) {
      cplx s = 0;
      for (int e = 0; e < n3; e++) s += Uexch_[(size_t)j * n3 + e] * A1[e];
      Srow[j] += s;
    }
  };
#pragma omp parallel
  {
    std::vector<cplx> A1(n3), B1(n3), B2(n3), tmp(n3), g1(n2), g2(n2);
#pragma omp for schedule(dynamic)
    for (int job = 0; job < 2 * nles + ntv; job++) {
      if (job < nles) {  // solve_les :5-38
        int t = job;
        const cplx *L = G.lesptr(t, tstp), *R = G.retptr(tstp, t);
        for (int i = 0; i < n; i++)
          for (int j = 0; j < n; j++) g1[i * n + j] = R[j * n + i] - std::conj(L[i * n + j]);
        for (int i = 0; i < n; i++) {
          zgemm(T, N, n, n2, n, 1.0, L, n, UC_.data() + (i64)i * n3, n2, 0.0, A1.data(), n2);
          zgemm(N, N, n2, n, n, 1.0, A1.data(), n, L, n, 0.0, tmp.data(), n);
          tpose(tmp.data(), n2, n, B1.data());
          zgemm(N, N, n2, n, n, 1.0, B1.data(), n, g1.data(), n, 0.0, A1.data(), n);
          contract(A1.data(), Sig.lesptr(t, tstp) + i * n);
        }
      } else if (job < 2 * nles) {  // solve_ret :78-120
        int t = job - nles;
        const cplx *L = G.lesptr(t, tstp), *R = G.retptr(tstp, t);
        for (int e = 0; e < n2; e++) g1[e] = -std::conj(L[e]);
        for (int i = 0; i < n; i++)
          for (int j = 0; j < n; j++) g2[i * n + j] = R[i * n + j] - std::conj(L[j * n + i]);
        for (int i = 0; i < n; i++) {
          zgemm(N, N, n, n2, n, 1.0, g1.data(), n, UC_.data() + (i64)i * n3, n2, 0.0, A1.data(), n2);
          zgemm(N, C, n2, n, n, -1.0, A1.data(), n, L, n, 0.0, tmp.data(), n);
          tpose(tmp.data(), n2, n, B1.data());
          zgemm(N, N, n2, n, n, 1.0, A1.data(), n, R, n, 0.0, tmp.data(), n);
          tpose(tmp.data(), n2, n, B2.data());
          zgemm(T, N, n, n2, n, 1.0, R, n, UC_.data() + (i64)i * n3, n2, 0.0, A1.data(), n2);
          zgemm(N, N, n2, n, n, 1.0, A1.data(), n, g2.data(), n, 0.0, tmp.data(), n);
          for (int r = 0; r < n2; r++)
            for (int c = 0; c < n; c++) B2[(i64)c * n2 + r] += tmp[(i64)r * n + c];
          std::vector<cplx> Rc(n2);
          conjm(R, n2, Rc.data());
          zgemm(N, T, n2, n, n, 1.0, B2.data(), n, L, n, 0.0, A1.data(), n);
          zgemm(N, N, n2, n, n, 1.0, B1.data(), n, Rc.data(), n, 1.0, A1.data(), n);
          contract(A1.data(), Sig.retptr(tstp, t) + i * n);
        }
      } else {  // solve_tv :41-75
        int t = job - 2 * nles;
        const cplx *gtv = G.tvptr(tstp, t), *gvt = G.tvptr(tstp, ntau - t);
        conjm(gvt, n2, g1.data(), -(double)sig);
        for (int i = 0; i < n; i++) {
          zgemm(T, N, n, n2, n, 1.0, gtv, n, UC_.data() + (i64)i * n3, n2, 0.0, A1.data(), n2);
          zgemm(N, N, n2, n, n, 1.0, A1.data(), n, gtv, n, 0.0, tmp.data(), n);
          tpose(tmp.data(), n2, n, B1.data());
          zgemm(N, N, n2, n, n, 1.0, B1.data(), n, g1.data(), n, 0.0, A1.data(), n);
          contract(A1.data(), Sig.tvptr(tstp, t) + i * n);
        }
      }
    }
  }
}

// mol2bSolver_impl.h:186-285
void FullSolver::solve_loop(int tstp, const GF &Sig, const GF &G) const {
  Sig.set_tstp_zero(tstp);
  int n = nao_, sig = G.sig, ntau = G.ntau;
  auto U = [&](int i, int j, int k, int l) { return U_[(((size_t)i * n + j) * n + k) * n + l]; };
  auto tri = [&](const cplx *X, const cplx *Y, const cplx *Z, cplx *out, double f) {
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        cplx acc = 0;
        for (int l = 0; l < n; l++) for (int nn = 0; nn < n; nn++) for (int p = 0; p < n; p++)
          for (int k = 0; k < n; k++) for (int q = 0; q < n; q++) for (int m = 0; m < n; m++)
            acc += U(i, l, nn, p) * (2 * U(j, k, q, m) - U(j, q, k, m)) * X[l * n + k] * Y[m * n + nn] * Z[p * n + q];
        out[i * n + j] += f * acc;
      }
  };
  size_t e2 = (size_t)n * n;
  std::vector<cplx> Y(e2), Lh(e2), Rh(e2), Zd(e2);
  for (int t = 0; t <= tstp; t++) {
    const cplx *L = G.lesptr(t, tstp), *R = G.retptr(tstp, t);
    for (int m = 0; m < n; m++)
      for (int nn = 0; nn < n; nn++) {
        Y[m * n + nn] = R[m * n + nn] - std::conj(L[nn * n + m]);
        Lh[m * n + nn] = std::conj(L[nn * n + m]);
        Rh[m * n + nn] = std::conj(R[nn * n + m]);
        Zd[m * n + nn] = R[m * n + nn] - Lh[m * n + nn];
      }
    tri(L, Y.data(), L, Sig.lesptr(t, tstp), 1.0);
    tri(R, L, Zd.data(), Sig.retptr(tstp, t), 1.0);
    tri(Lh.data(), Rh.data(), Lh.data(), Sig.retptr(tstp, t), 1.0);
    tri(Lh.data(), L, R, Sig.retptr(tstp, t), -1.0);
  }
  for (int t = 0; t <= ntau; t++) {
    const cplx *Gt = G.tvptr(tstp, t), *Gv = G.tvptr(tstp, ntau - t);
    for (int m = 0; m < n; m++)
      for (int nn = 0; nn < n; nn++) Y[m * n + nn] = -(double)sig * std::conj(Gv[nn * n + m]);
    tri(Gt, Y.data(), Gt, Sig.tvptr(tstp, t), 1.0);
  }
}

// ---------------- Hartree-Fock ----------------
// molHFSolver.cpp:81-110 (restricted DF)
void hf_decomp(int nao, int naux, const double *Vija, cplx *hmf_t, const cplx *rho) {
  int n = nao, a = naux, n2 = n * n;
  std::vector<cplx> Xa(a, 0.0);
  for (int e = 0; e < n2; e++)
    for (int q = 0; q < a; q++) Xa[q] += rho[e] * Vija[(size_t)e * a + q];
  for (int e = 0; e < n2; e++) {
    cplx s = 0;
    for (int q = 0; q < a; q++) s += Xa[q] * Vija[(size_t)e * a + q];
    hmf_t[e] += 2.0 * s;
  }
  // Fock: hmf_ij -= sum_{l,k} rho_kl sum_a V_il^a V_kj^a
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      cplx s = 0;
      for (int l = 0; l < n; l++)
        for (int k = 0; k < n; k++) {
          double v = 0;
          for (int q = 0; q < a; q++) v += Vija[((size_t)i * n + l) * a + q] * Vija[((size_t)k * n + j) * a + q];
          s += rho[k * n + l] * v;
        }
      hmf_t[i * n + j] -= s;
    }
}

// molHFSolver.cpp:58-79 (brute force)
void hf_decomp_loop(int nao, int naux, const double *Vija, cplx *hmf_t, const cplx *rho) {
  int n = nao;
  auto V = [&](int i, int j, int a) { return Vija[((size_t)i * n + j) * naux + a]; };
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      for (int k = 0; k < n; k++)
        for (int l = 0; l < n; l++)
          for (int a = 0; a < naux; a++)
            hmf_t[i * n + j] += rho[k * n + l] * (2 * V(i, j, a) * V(k, l, a) - V(i, l, a) * V(k, j, a));
}

// molHFSolver.cpp:203-239 (unrestricted DF); hmf_s[s] -> hmf row of spin s
void hf_spin_decomp(int nao, int naux, const double *Vija, cplx *hmf_up, cplx *hmf_dn, const cplx *rho2) {
  int n = nao, a = naux, n2 = n * n;
  std::vector<cplx> Xa(a, 0.0);
  for (int e = 0; e < n2; e++)
    for (int q = 0; q < a; q++) Xa[q] += (rho2[e] + rho2[n2 + e]) * Vija[(size_t)e * a + q];
  cplx *h[2] = {hmf_up, hmf_dn};
  for (int e = 0; e < n2; e++) {
    cplx s = 0;
    for (int q = 0; q < a; q++) s += Xa[q] * Vija[(size_t)e * a + q];
    h[0][e] += s;
    h[1][e] += s;
  }
  for (int sp = 0; sp < 2; sp++) {
    const cplx *rho = rho2 + sp * n2;
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        cplx s = 0;
        for (int l = 0; l < n; l++)
          for (int k = 0; k < n; k++) {
            double v = 0;
            for (int q = 0; q < a; q++) v += Vija[((size_t)i * n + l) * a + q] * Vija[((size_t)k * n + j) * a + q];
            s += rho[k * n + l] * v;
          }
        h[sp][i * n + j] -= s;
      }
  }
}

// molHFSolver.cpp:173-201 (brute force)
void hf_spin_decomp_loop(int nao, int naux, const double *Vija, cplx *hmf_up, cplx *hmf_dn, const cplx *rho2) {
  int n = nao, n2 = n * n;
  auto V = [&](int i, int j, int a) { return Vija[((size_t)i * n + j) * naux + a]; };
  cplx *h[2] = {hmf_up, hmf_dn};
  for (int s = 0; s < 2; s++)
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++)
        for (int a = 0; a < naux; a++)
          for (int sp = 0; sp < 2; sp++)
            for (int k = 0; k < n; k++)
              for (int l = 0; l < n; l++) {
                h[s][i * n + j] += V(i, j, a) * V(k, l, a) * rho2[sp * n2 + k * n + l];
                if (s == sp) h[s][i * n + j] -= V(i, l, a) * V(k, j, a) * rho2[s * n2 + k * n + l];
              }
}

// molHFSolver.cpp:35-56 (full U) and :13-33 (brute force)
void hf_full(int nao, const double *U, cplx *hmf_t, const cplx *rho) {
  int n = nao;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      cplx s = 0;
      for (int k = 0; k < n; k++)
        for (int l = 0; l < n; l++) {
          s -= rho[k * n + l] * U[(((size_t)i * n + l) * n + k) * n + j];
          s += 2.0 * U[(((size_t)i * n + j) * n + k) * n + l] * rho[k * n + l];
        }
      hmf_t[i * n + j] += s;
    }
}
void hf_full_loop(int nao, const double *U, cplx *hmf_t, const cplx *rho) {
  int n = nao;
  auto Uf = [&](int i, int j, int k, int l) { return U[(((size_t)i * n + j) * n + k) * n + l]; };
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      for (int k = 0; k < n; k++)
        for (int l = 0; l < n; l++) hmf_t[i * n + j] += rho[k * n + l] * (2 * Uf(i, j, k, l) - Uf(i, l, k, j));
}

} // namespace orc
