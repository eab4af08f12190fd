// Equilibrium (Matsubara) GF2 solver on the Legendre-Gauss-Lobatto collocation grid.
//
// The reference takes its equilibrium state from the external gfmol solver
// (src/molNEsim_decomp_impl.h:23-33, :45, :51; L_to_Tau :146-167 maps gfmol's
// coefficients onto the collocation grid).  Here it is computed on the grid directly,
// from the same density-fitted contractions as the time stepping:
//
//   Sigma^M(tau)  GF2 self-energy of G^M: the density-fitted contraction of the mixed row
//                 at t = 0, whose blocks are G^tv(0, tau) = -i G^M(beta - tau), then
//                 Sigma^M(tau) = i Sigma^tv(0, beta - tau);
//   F             h0 + HF(rho), rho = -G^M(beta) (green_func::get_dm(-1), src/greens.h:68-74);
//   Dyson         G = G_ref + G_ref * (dF + Sigma^M) * G, with G_ref the free G^M of a
//                 reference Fock matrix F_ref at the same mu, dF = F - F_ref, and
//                 (A * B)(tau) = int_0^beta A(tau - tau') B(tau') dtau' (the Matsubara
//                 convolution) evaluated exactly on the degree-ntau interpolants through the
//                 same quadrature as the mixing kernel: (A * B)(tau_m) = sum_i K_A[m][i] B_i
//                 with K_A the tau-kernel of B(x) = A(-x), whose nodal values are
//                 sig A(tau_{ntau - m}) (antiperiodic extension, symmetric nodes).
//
// The iteration  G <- G + a (G_ref + K_ref (K_Sigma G + dF G) - G)  runs to max |change| <= tol;
// every operation is a device GEMM or kernel on the context's stream.  mu is held fixed (the
// gap of the reference state pins the particle number at low temperature).
#include "handles.cuh"
#include "sigma.cuh"
#include <algorithm>
#include <string>
#include <vector>

namespace nedy {
namespace {

constexpr int TPB = 256;
inline unsigned nblk(i64 n) { return (unsigned)std::min<i64>((n + TPB - 1) / TPB, 65535LL * 16); }

// out[j] = s * A[ntau - j] for j = 0..ntau (blocks), with a complex factor s
__global__ void mirror_kernel(int N, int np, const double2 *A, double2 s, double2 *out) {
  const i64 es = (i64)N * N, tot = es * np;
  for (i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x; idx < tot; idx += (i64)gridDim.x * blockDim.x) {
    const i64 j = idx / es, e = idx - j * es;
    out[idx] = cmul(s, A[(np - 1 - j) * es + e]);
  }
}

// G += a (Gn - G); *mx = max |Gn - G| (bit pattern of a non-negative double)
__global__ void relax_kernel(i64 n, const double2 *Gn, double a, double2 *G, unsigned long long *mx) {
  double m = 0.0;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    const double2 d = csub(Gn[i], G[i]);
    m = fmax(m, hypot(d.x, d.y));
    G[i] = cadd(G[i], cscale(d, a));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(mx, (unsigned long long)__double_as_longlong(m));
}

__global__ void sub_kernel(i64 n, const double2 *a, const double2 *b, double2 *out) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
    out[i] = csub(a[i], b[i]);
}

// rho = -G^M(beta)
__global__ void rho_kernel(int N, const double2 *mat_last, double2 *rho) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < N * N) rho[e] = make_double2(-mat_last[e].x, -mat_last[e].y);
}

// out (np N x N, blocks [m] of N x N) = K (np N x np N) * B (np N x N) (+ beta out)
void apply_kernel(Ctx &c, int N, int np, const double2 *K, const double2 *B, double2 *out, double beta) {
  const i64 es = (i64)N * N;
  GemmArgs g;
  g.M = np * N; g.N = N; g.K = np * N;
  g.A.p = K; g.A.rdiv = N; g.A.rs_hi = (i64)np * es; g.A.rs_lo = N; g.A.cdiv = N; g.A.cs_hi = es; g.A.cs_lo = 1;
  g.B.p = B; g.B.rdiv = N; g.B.rs_hi = es; g.B.rs_lo = N; g.B.cs_lo = 1;
  g.C.p = out; g.C.rdiv = N; g.C.rs_hi = es; g.C.rs_lo = N; g.C.cs_lo = 1;
  g.beta = make_double2(beta, 0.0);
  gemm(g, c.stream);
}

struct DevBuf {
  void *p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
  template <class T> T *get(size_t n) {
    NEDY_CUDA(cudaMalloc(&p, sizeof(T) * n));
    return (T *)p;
  }
};

}  // namespace
}  // namespace nedy

using namespace nedy;

extern "C" int nedy_matsubara_gf2(nedy_ctx *ctx, int nspin, nedy_gf *const *G, nedy_gf *const *Sigma,
                                  const nedy_buf *const *h0, const nedy_buf *const *F_ref, nedy_buf *const *F_out,
                                  double mixing, int max_iter, double tol, int *iters, double *diff) {
  return run_guarded([&] {
    NEDY_REQUIRE(ctx && G && Sigma && h0 && F_ref && F_out, "null argument");
    NEDY_REQUIRE(nspin == 1 || nspin == 2, "nspin must be 1 or 2");
    NEDY_REQUIRE(mixing > 0.0 && mixing <= 1.0 && max_iter >= 1 && tol >= 0.0, "bad iteration parameters");
    Ctx &c = ctx->c;
    NEDY_CUDA(cudaSetDevice(c.device));
    NEDY_REQUIRE(c.Vija, "nedy_matsubara_gf2: density-fitted tensor not set");
    const int N = c.df_nao, ntau = c.ntau, np = ntau + 1;
    const i64 es = (i64)N * N, row = (i64)np * es;
    for (int s = 0; s < nspin; s++) {
      NEDY_REQUIRE(G[s] && Sigma[s] && h0[s] && F_ref[s] && F_out[s], "null argument");
      NEDY_REQUIRE(G[s]->g.nao == N && G[s]->g.ntau == ntau && Sigma[s]->g.nao == N && Sigma[s]->g.ntau == ntau,
                   "G / Sigma sizes differ from the context and the tensor");
      NEDY_REQUIRE(h0[s]->bytes >= es * 16 && F_ref[s]->bytes >= es * 16 && F_out[s]->bytes >= es * 16,
                   "h0 / F buffers smaller than nao x nao complex");
    }
    const double sig = (double)G[0]->g.sig;
    // device scratch (one-time set-up of a simulation)
    DevBuf bK, bX, bGn, bGref, bT, bdF, bmx;
    double2 *Kref = bK.get<double2>((size_t)2 * nspin * np * row);  // [spin] K_ref, then [spin] K_Sigma
    double2 *Ksig = Kref + (size_t)nspin * np * row;
    double2 *X = bX.get<double2>((size_t)nspin * row);
    double2 *Gn = bGn.get<double2>((size_t)nspin * row);
    double2 *Gref = bGref.get<double2>((size_t)nspin * row);
    // t = 0 rows of G and Sigma for the self-energy: les, ret (1 block each), tv (np), mat (np)
    double2 *T0 = bT.get<double2>((size_t)2 * nspin * (2 * es + 2 * row));
    double2 *dF = bdF.get<double2>((size_t)nspin * (2 * es + es));  // dF, F, rho per spin
    unsigned long long *mx = bmx.get<unsigned long long>(1);
    DevGF g0[2], s0[2];
    for (int s = 0; s < nspin; s++) {
      double2 *base = T0 + (size_t)s * 2 * (2 * es + 2 * row);
      for (int k = 0; k < 2; k++) {
        DevGF &d = k == 0 ? g0[s] : s0[s];
        double2 *b = base + (size_t)k * (2 * es + 2 * row);
        d.nt = 0; d.ntau = ntau; d.nao = N; d.sig = G[s]->g.sig; d.es = es;
        d.les = b; d.ret = b + es; d.tv = b + 2 * es; d.mat = b + 2 * es + row;
      }
      NEDY_CUDA(cudaMemsetAsync(base, 0, sizeof(double2) * 2 * (2 * es + 2 * row), c.stream));
      NEDY_CUDA(cudaMemcpyAsync(Gref + s * row, G[s]->g.mat, sizeof(double2) * row, cudaMemcpyDeviceToDevice,
                                c.stream));
      // K_ref: kernel of B(x) = G_ref(-x), nodal values sig G_ref(tau_{ntau - m})
      mirror_kernel<<<nblk(row), TPB, 0, c.stream>>>(N, np, Gref + s * row, make_double2(sig, 0.0), X + s * row);
      NEDY_CHECK_LAUNCH();
      build_tau_kernel(c, X + s * row, N, sig, Kref + (size_t)s * np * row);
    }
    int it = 0;
    double d = 0.0;
    for (; it < max_iter;) {
      // mean field: F = h0 + HF(rho), rho = -G^M(beta); dF = F - F_ref
      double2 *Fp[2], *rho = dF + (size_t)nspin * 2 * es;
      for (int s = 0; s < nspin; s++) {
        Fp[s] = dF + (size_t)nspin * es + s * es;
        NEDY_CUDA(cudaMemcpyAsync(Fp[s], h0[s]->p, sizeof(double2) * es, cudaMemcpyDeviceToDevice, c.stream));
        rho_kernel<<<cdiv(es, 128), 128, 0, c.stream>>>(N, G[s]->g.mat + (i64)ntau * es, rho + s * es);
        NEDY_CHECK_LAUNCH();
      }
      c.ws.reset();
      hf_decomp(c, nspin, Fp, rho);
      for (int s = 0; s < nspin; s++) {
        sub_kernel<<<nblk(es), TPB, 0, c.stream>>>(es, Fp[s], (const double2 *)F_ref[s]->p, dF + s * es);
        NEDY_CHECK_LAUNCH();
        // G^tv(0, tau_m) = -i G^M(tau_{ntau - m})
        mirror_kernel<<<nblk(row), TPB, 0, c.stream>>>(N, np, G[s]->g.mat, make_double2(0.0, -1.0), g0[s].tv);
        NEDY_CHECK_LAUNCH();
      }
      // Sigma^tv(0, .) by the density-fitted GF2 contraction of the t = 0 row
      DevGF *Sp[2] = {&s0[0], nspin > 1 ? &s0[1] : nullptr};
      const DevGF *Gp[2] = {&g0[0], nspin > 1 ? &g0[1] : nullptr};
      sigma_df(c, 0, nspin, Sp, Gp);
      NEDY_CUDA(cudaMemsetAsync(mx, 0, sizeof(unsigned long long), c.stream));
      for (int s = 0; s < nspin; s++) {
        // Sigma^M(tau_m) = i Sigma^tv(0, tau_{ntau - m}); K_Sigma from B(x) = Sigma^M(-x)
        mirror_kernel<<<nblk(row), TPB, 0, c.stream>>>(N, np, s0[s].tv, make_double2(0.0, 1.0), Sigma[s]->g.mat);
        NEDY_CHECK_LAUNCH();
        mirror_kernel<<<nblk(row), TPB, 0, c.stream>>>(N, np, Sigma[s]->g.mat, make_double2(sig, 0.0), X + s * row);
        NEDY_CHECK_LAUNCH();
        double2 *Ks = Ksig + (size_t)s * np * row;
        build_tau_kernel(c, X + s * row, N, sig, Ks);
        // X = Sigma * G + dF G
        apply_kernel(c, N, np, Ks, G[s]->g.mat, X + s * row, 0.0);
        GemmArgs g;
        g.M = N; g.N = N; g.K = N; g.nb1 = np;
        g.A = rowmajor(dF + s * es, N);
        g.B = rowmajor(G[s]->g.mat, N); g.B.bs1 = es;
        g.C = rowmajor(X + s * row, N); g.C.bs1 = es;
        g.beta = make_double2(1.0, 0.0);
        gemm(g, c.stream);
        // Gn = G_ref + G_ref * X
        NEDY_CUDA(cudaMemcpyAsync(Gn + s * row, Gref + s * row, sizeof(double2) * row, cudaMemcpyDeviceToDevice,
                                  c.stream));
        apply_kernel(c, N, np, Kref + (size_t)s * np * row, X + s * row, Gn + s * row, 1.0);
        relax_kernel<<<nblk(row), TPB, 0, c.stream>>>(row, Gn + s * row, mixing, G[s]->g.mat, mx);
        NEDY_CHECK_LAUNCH();
      }
      unsigned long long h = 0;
      NEDY_CUDA(cudaMemcpyAsync(&h, mx, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
      NEDY_CUDA(cudaStreamSynchronize(c.stream));
      d = __builtin_bit_cast(double, h);
      it++;
      if (!(d == d)) throw ArgError("nedy_matsubara_gf2: the iteration diverged (NaN)");
      if (d <= tol) break;
    }
    // final mean field of the returned G^M, and the self-energy's G^M versions
    {
      double2 *Fp[2], *rho = dF + (size_t)nspin * 2 * es;
      for (int s = 0; s < nspin; s++) {
        Fp[s] = (double2 *)F_out[s]->p;
        NEDY_CUDA(cudaMemcpyAsync(Fp[s], h0[s]->p, sizeof(double2) * es, cudaMemcpyDeviceToDevice, c.stream));
        rho_kernel<<<cdiv(es, 128), 128, 0, c.stream>>>(N, G[s]->g.mat + (i64)ntau * es, rho + s * es);
        NEDY_CHECK_LAUNCH();
      }
      c.ws.reset();
      hf_decomp(c, nspin, Fp, rho);
    }
    NEDY_CUDA(cudaStreamSynchronize(c.stream));
    for (int s = 0; s < nspin; s++) {
      G[s]->g.mat_version++;
      Sigma[s]->g.mat_version++;
    }
    if (iters) *iters = it;
    if (diff) *diff = d;
  });
}
