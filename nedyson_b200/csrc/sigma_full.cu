// Full-U second-Born self-energy for one time row T.  Replaces molGF2Solver::solve
// (reference src/mol2bSolver_impl.h:123-182; definition :186-285).
//
//   Sigma_ij += c * sum_{q,k,m} Uexch[j][q][k][m] A_i[q][k][m]
//   A_i[q][k][m] = sum_{l,n,p} U[i][l][n][p] X_lk Z_pq Y_mn
// with Uexch[j][q][k][m] = 2 U[j][k][q][m] - U[j][q][k][m] and the slot blocks
// (X, Y, Z) of the lesser / mixed / retarded slices (the same trilinear forms as
// the density-fitted solver).  The full-U form is the reference's small-basis
// path (O(nao^5) per slice): one CTA per (slice, i), intermediates in shared memory.
#include "sigma.cuh"
#include <algorithm>

namespace nedy {
namespace {

__global__ void full_tri_kernel(int N, const double *U, const double *Ux, const double2 *X, i64 sX,
                                const double2 *Y, i64 sY, const double2 *Z, i64 sZ, double2 *S, i64 sS,
                                double coef) {
  extern __shared__ double2 sm[];
  const int s = blockIdx.x, i = blockIdx.y;
  const int N2 = N * N, N3 = N2 * N;
  double2 *T1 = sm, *T2 = sm + N3, *A = sm + 2 * N3;
  const double2 *x = X + s * sX, *y = Y + s * sY, *z = Z + s * sZ;
  const double *Ui = U + (i64)i * N3;
  for (int e = threadIdx.x; e < N3; e += blockDim.x) {  // T1[k][n][p] = sum_l X_lk U[i][l][n][p]
    const int k = e / N2, np = e - k * N2;
    double2 acc = czero();
    for (int l = 0; l < N; l++) acc = cadd(acc, cscale(x[l * N + k], Ui[(i64)l * N2 + np]));
    T1[e] = acc;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < N3; e += blockDim.x) {  // T2[q][k][n] = sum_p T1[k][n][p] Z_pq
    const int q = e / N2, kn = e - q * N2;
    double2 acc = czero();
    for (int p = 0; p < N; p++) acc = cadd(acc, cmul(T1[kn * N + p], z[p * N + q]));
    T2[e] = acc;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < N3; e += blockDim.x) {  // A[q][k][m] = sum_n T2[q][k][n] Y_mn
    const int qk = e / N, m = e - qk * N;
    double2 acc = czero();
    for (int n = 0; n < N; n++) acc = cadd(acc, cmul(T2[qk * N + n], y[m * N + n]));
    A[e] = acc;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < N; j += blockDim.x) {
    double2 acc = czero();
    for (int e = 0; e < N3; e++) acc = cadd(acc, cscale(A[e], Ux[(i64)j * N3 + e]));
    double2 *dst = S + s * sS + (i64)i * N + j;
    *dst = cadd(*dst, cscale(acc, coef));
  }
}

__global__ void full_prep_kernel(int mode, int N, int nsl, const double2 *L0, i64 Ls, const double2 *R0, i64 Rs,
                                 double sgn, double2 *out, i64 ostride) {
  const i64 es = (i64)N * N;
  for (i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x; idx < es * nsl; idx += (i64)gridDim.x * blockDim.x) {
    const int s = (int)(idx / es), e = (int)(idx - (i64)s * es);
    const int i = e / N, j = e - (e / N) * N;
    if (mode == 0) {  // les: R - L^+
      const double2 r = R0[s * Rs + e], lt = L0[s * Ls + (i64)j * N + i];
      out[s * es + e] = make_double2(r.x - lt.x, r.y + lt.y);
    } else if (mode == 1) {  // tv: -sig Gv^+
      const double2 g = L0[s * Ls + (i64)j * N + i];
      out[s * es + e] = make_double2(sgn * g.x, -sgn * g.y);
    } else {  // ret: L^+, R^+, R - L^+
      const double2 lt = L0[s * Ls + (i64)j * N + i], r = R0[s * Rs + e], rt = R0[s * Rs + (i64)j * N + i];
      out[0 * ostride + s * es + e] = make_double2(lt.x, -lt.y);
      out[1 * ostride + s * es + e] = make_double2(rt.x, -rt.y);
      out[2 * ostride + s * es + e] = make_double2(r.x - lt.x, r.y + lt.y);
    }
  }
}
} // namespace

void sigma_full(Ctx &c, int T, DevGF &Sig, const DevGF &G) {
  NEDY_REQUIRE(c.U != nullptr, "sigma_full: U tensor not set");
  const int N = c.u_nao;
  NEDY_REQUIRE(G.nao == N && Sig.nao == N, "sigma_full: nao mismatch");
  NEDY_REQUIRE(N * N * N <= 1024, "sigma_full: the full-U path supports nao <= 10");
  NEDY_REQUIRE(T >= 0 && T <= G.nt && T <= Sig.nt, "sigma_full: tstp out of range");
  c.ws.reset();
  const i64 es = (i64)N * N;
  const int ntau = G.ntau, nles = T + 1, ntv = ntau + 1;
  NEDY_CUDA(cudaMemsetAsync(Sig.retptr(T, 0), 0, sizeof(double2) * nles * es, c.stream));
  NEDY_CUDA(cudaMemsetAsync(Sig.lesptr(0, T), 0, sizeof(double2) * nles * es, c.stream));
  NEDY_CUDA(cudaMemsetAsync(Sig.tvptr(T, 0), 0, sizeof(double2) * ntv * es, c.stream));
  const int smem = 3 * N * N * N * sizeof(double2);
  const int th = std::min(256, std::max(32, N * N * N));
  double2 *H = c.ws.alloc<double2>(nles * es);
  double2 *Hv = c.ws.alloc<double2>(ntv * es);
  double2 *D = c.ws.alloc<double2>(3 * nles * es);
  auto nb = [](i64 n) { return (unsigned)std::min<i64>((n + 255) / 256, 65535); };
  full_prep_kernel<<<nb(es * nles), 256, 0, c.stream>>>(0, N, nles, G.lesptr(0, T), es, G.retptr(T, 0), es, 0, H, 0);
  NEDY_CHECK_LAUNCH();
  full_prep_kernel<<<nb(es * ntv), 256, 0, c.stream>>>(1, N, ntv, G.tvptr(T, ntau), -es, nullptr, 0, -(double)G.sig,
                                                       Hv, 0);
  NEDY_CHECK_LAUNCH();
  full_prep_kernel<<<nb(es * nles), 256, 0, c.stream>>>(2, N, nles, G.lesptr(0, T), es, G.retptr(T, 0), es, 0, D,
                                                        nles * es);
  NEDY_CHECK_LAUNCH();
  const double2 *L = G.lesptr(0, T), *R = G.retptr(T, 0), *Gt = G.tvptr(T, 0);
  const double2 *Lh = D, *Rh = D + nles * es, *Zd = D + 2 * nles * es;
  auto tri = [&](int nsl, const double2 *X, const double2 *Y, const double2 *Z, double2 *S, double cf) {
    full_tri_kernel<<<dim3(nsl, N), th, smem, c.stream>>>(N, c.U, c.Uexch, X, es, Y, es, Z, es, S, es, cf);
    NEDY_CHECK_LAUNCH();
  };
  tri(nles, L, H, L, Sig.lesptr(0, T), 1.0);                // lesser  (L, R - L^+, L)
  tri(ntv, Gt, Hv, Gt, Sig.tvptr(T, 0), 1.0);               // mixed
  tri(nles, R, L, Zd, Sig.retptr(T, 0), 1.0);               // retarded: (R, L, R - L^+)
  tri(nles, Lh, Rh, Lh, Sig.retptr(T, 0), 1.0);             //           + (L^+, R^+, L^+)
  tri(nles, Lh, L, R, Sig.retptr(T, 0), -1.0);              //           - (L^+, L, R)
}

} // namespace nedy
