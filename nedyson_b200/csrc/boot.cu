// Bootstrap of the first k+1 time steps and the correlation energy -- device side.
//   dyson_start (tv, ret, les) : reference src/dyson_boot.h:6-230
//   tv_it_conv                 : reference src/dyson_integrals.h:7-15
//   energy_conv                : reference src/dyson_integrals.h:24-70
#include "sigma.cuh"
#include <cmath>
#include <algorithm>

namespace nedy {

namespace {
constexpr int TPB = 256;
inline unsigned nblk(i64 n) { return (unsigned)std::min<i64>((n + TPB - 1) / TPB, 65535LL * 16); }
#define GRID_STRIDE(i, n) for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < (n); i += (i64)gridDim.x * blockDim.x)

// G^tv(0,m) = sig i G^M(ntau-m)  (dyson_boot.h:102-109)
__global__ void boot_tv0_kernel(int N, DevGF G, double *err) {
  const i64 es = (i64)N * N, tot = es * (G.ntau + 1);
  GRID_STRIDE(idx, tot) {
    const int m = (int)(idx / es), e = (int)(idx - (i64)m * es);
    const double2 g = G.matptr(G.ntau - m)[e];
    const double2 v = make_double2(-G.sig * g.y, G.sig * g.x);
    double2 *dst = G.tvptr(0, m) + e;
    const double2 d = csub(*dst, v);
    add_warp(&err[m], d.x * d.x + d.y * d.y);
    *dst = v;
  }
}

// kN x kN matrix of the start system (shared by every tau point), dyson_boot.h:135-168
__global__ void boot_M_kernel(int N, int k, DevGF S, const double2 *hmf, const double *pdiff, const double *greg,
                              int ld, double mu, double dt, double2 *M) {
  const i64 es = (i64)N * N;
  const int kn = k * N;
  GRID_STRIDE(idx, (i64)kn * kn) {
    const int r = (int)(idx / kn), cc = (int)(idx - (i64)r * kn);
    const int n = r / N + 1, i = r % N, l = cc / N + 1, j = cc % N;
    double2 v = czero();
    if (i == j) v.y += pdiff[n * (k + 1) + l] / dt;
    if (l == n) {
      const double2 h = hmf[(i64)l * es + (i64)i * N + j];
      v.x -= h.x; v.y -= h.y;
      if (i == j) v.x += mu;
    }
    const double w = dt * greg[n * ld + l];
    if (n >= l) {
      const double2 s = S.retptr(n, l)[(i64)i * N + j];
      v.x -= w * s.x; v.y -= w * s.y;
    } else {
      const double2 s = S.retptr(l, n)[(i64)j * N + i];
      v.x += w * s.x; v.y -= w * s.y;
    }
    M[idx] = v;
  }
}

// Q(n,m) += -(i/dt) pd(n,0) G^tv(0,m)    (Q laid out like G^tv rows 1..k)
__global__ void boot_Q_kernel(int N, int k, DevGF G, const double *pdiff, double dt, double2 *Q) {
  const i64 es = (i64)N * N, row = es * (G.ntau + 1);
  GRID_STRIDE(idx, row * k) {
    const int n = (int)(idx / row) + 1;
    const i64 r = idx - (i64)(n - 1) * row;
    const double2 g = G.tvptr(0, 0)[r];
    const double pd = pdiff[n * (k + 1)] / dt;
    Q[idx] = cadd(Q[idx], make_double2(pd * g.y, -pd * g.x));
  }
}

__global__ void diffnorm_blocks_kernel(int N, int nb, const double2 *A, const double2 *B, double *err) {
  const i64 es = (i64)N * N;
  GRID_STRIDE(i, es * nb) {
    const double2 d = csub(A[i], B[i]);
    add_warp(&err[i / es], d.x * d.x + d.y * d.y);
  }
}

// G^R(n+l, l) = GR_n  (TTI copy, dyson_boot.h:79-88)
__global__ void boot_ret_kernel(int N, int k, DevGF G, double *err) {
  const i64 es = (i64)N * N;
  const int npairs = (k + 1) * (k + 2) / 2;
  GRID_STRIDE(idx, es * npairs) {
    int p = (int)(idx / es);
    const int e = (int)(idx - (i64)p * es);
    int n = 0;
    while (p > k - n) { p -= (k - n + 1); n++; }
    const int l = p;
    const int i = e / N, j = e - (e / N) * N;
    double2 v;
    if (n == 0) v = make_double2(0.0, i == j ? -1.0 : 0.0);
    else v = csub(cscale(G.tvptr(n, G.ntau)[e], (double)G.sig), G.tvptr(n, 0)[e]);
    double2 *dst = G.retptr(n + l, l) + e;
    const double2 d = csub(v, *dst);
    add_warp(&err[n * (k + 1) + l], d.x * d.x + d.y * d.y);
    *dst = v;
  }
}

// G^<(n,l) = -G^tv(l-n,0)^+  (dyson_boot.h:181-192)
__global__ void boot_les_kernel(int N, int k, DevGF G, double *err) {
  const i64 es = (i64)N * N;
  const int npairs = (k + 1) * (k + 2) / 2;
  GRID_STRIDE(idx, es * npairs) {
    int p = (int)(idx / es);
    const int e = (int)(idx - (i64)p * es);
    int l = 0;
    while (p > l) { p -= (l + 1); l++; }
    const int n = p;
    const int i = e / N, j = e - (e / N) * N;
    const double2 t = G.tvptr(l - n, 0)[(i64)j * N + i];
    const double2 v = make_double2(-t.x, t.y);
    double2 *dst = G.lesptr(n, l) + e;
    const double2 d = csub(*dst, v);
    add_warp(&err[l * (k + 1) + n], d.x * d.x + d.y * d.y);
    *dst = v;
  }
}

// ---- energy
// res1 terms, one block per history index i = 0..top (dyson_integrals.h:40-57)
__global__ void energy_hist_kernel(int N, int T, int top, DevGF S, DevGF G, const double *gregrow, double *out) {
  const int i = blockIdx.x;
  const i64 es = (i64)N * N;
  __shared__ double red[4][TPB];
  double a1 = 0, a2 = 0, b1 = 0, b2 = 0;
  for (i64 e = threadIdx.x; e < es; e += blockDim.x) {
    const int r = (int)(e / N), c = (int)(e - (e / N) * N);
    double2 x, y;
    if (i <= T) {
      x = cmul(S.retptr(T, i)[e], G.lesptr(i, T)[(i64)c * N + r]);
      y = cmul(S.lesptr(i, T)[e], G.retptr(T, i)[(i64)c * N + r]);
    } else {
      x = cmul(S.retptr(i, T)[e], G.lesptr(T, i)[(i64)c * N + r]);
      y = cmul(S.lesptr(T, i)[e], G.retptr(i, T)[(i64)c * N + r]);
    }
    a1 += x.x; a2 += x.y; b1 += y.x; b2 += y.y;
  }
  red[0][threadIdx.x] = a1; red[1][threadIdx.x] = a2; red[2][threadIdx.x] = b1; red[3][threadIdx.x] = b2;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int q = 0; q < 4; q++) red[q][threadIdx.x] += red[q][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double w = gregrow[i];
    double2 x = make_double2(w * red[0][0], w * red[1][0]);
    double2 y = make_double2(w * red[2][0], w * red[3][0]);
    double2 v;
    if (i <= T) v = csub(x, cconj(y));
    else v = csub(cconj(x), y);
    atomicAdd(&out[0], v.x);
    atomicAdd(&out[1], v.y);
  }
}

// res2: (-sig)(beta/2)[ sum_i w_i sum_ab A_i conj(B_{n-i}) + ctop UA : UB ]
__global__ void energy_tv_kernel(int N, int T, DevGF S, DevGF G, const double *w, const double *u, double ctop,
                                 double *out) {
  const i64 es = (i64)N * N;
  const int np = G.ntau + 1;
  double sr = 0, si = 0;
  GRID_STRIDE(e, es) {
    double2 ua = czero(), ub = czero();
    for (int i = 0; i < np; i++) {
      const double2 a = S.tvptr(T, i)[e];
      const double2 b = cconj(G.tvptr(T, np - 1 - i)[e]);
      const double2 p = cmul(a, b);
      sr += w[i] * p.x; si += w[i] * p.y;
      ua = cadd(ua, cscale(a, u[i]));
      ub = cadd(ub, cscale(b, u[i]));
    }
    const double2 q = cmul(ua, ub);
    sr += ctop * q.x; si += ctop * q.y;
  }
  atomicAdd(&out[2], sr);
  atomicAdd(&out[3], si);
}

double host_sum_sqrt(Ctx &c, const double *d, int n) {
  std::vector<double> h(n);
  NEDY_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream));
  NEDY_CUDA(cudaStreamSynchronize(c.stream));
  double s = 0;
  for (double v : h) s += std::sqrt(v);
  return s;
}
} // namespace

double dyson_start(Ctx &c, DevGF &G, const DevGF &Sig, const double2 *hmf, double mu) {
  NEDY_REQUIRE(G.nt >= c.k && G.nt == c.nt && G.ntau == c.ntau, "dyson_start: G does not match the context");
  NEDY_REQUIRE(G.nao == Sig.nao && G.ntau == Sig.ntau && G.nt == Sig.nt, "dyson_start: G and Sigma differ");
  ensure_tables(c);
  ensure_mixing_kernel(c, G);
  c.ws.reset();
  const int N = G.nao, k = c.k, kn = k * N, np = G.ntau + 1, ld = c.nt + 1;
  const i64 es = (i64)N * N, row = es * np;
  const double dt = c.dt;
  double err_total = 0;
  {
    double *e0 = c.ws.alloc<double>(np);
    NEDY_CUDA(cudaMemsetAsync(e0, 0, sizeof(double) * np, c.stream));
    boot_tv0_kernel<<<nblk(row), TPB, 0, c.stream>>>(N, G, e0);
    NEDY_CHECK_LAUNCH();
    err_total += host_sum_sqrt(c, e0, np);
  }
  // right-hand sides Q(n, m), n = 1..k, laid out like G^tv rows 1..k
  double2 *Q = c.ws.alloc<double2>(row * k);
  {  // tv_it_conv(m, n): sum_i Sig^tv(n,i) Re K[m][i]   (real view of the complex kernel)
    GemmArgs g;
    g.M = N; g.N = np * N; g.K = np * N; g.nb1 = k;
    g.A.p = Sig.tvptr(1, 0); g.A.rs_lo = N; g.A.cdiv = N; g.A.cs_hi = es; g.A.cs_lo = 1; g.A.bs1 = row;
    g.B.p = (const double *)c.mixK;
    g.B.rdiv = N; g.B.rs_hi = 2 * es; g.B.rs_lo = 2 * N; g.B.cdiv = N; g.B.cs_hi = 2 * (i64)np * es; g.B.cs_lo = 2;
    g.b_cplx = false;
    g.C.p = Q; g.C.rs_lo = N; g.C.cdiv = N; g.C.cs_hi = es; g.C.cs_lo = 1; g.C.bs1 = row;
    gemm(g, c.stream);
  }
  for (int n = 1; n <= k; n++) {  // += dt w(n,0) Sig^R(n,0) G^tv(0, .)
    GemmArgs g;
    g.M = N; g.N = np * N; g.K = N;
    g.A = rowmajor(Sig.retptr(n, 0), N);
    g.B.p = G.tvptr(0, 0); g.B.rs_lo = N; g.B.cdiv = N; g.B.cs_hi = es; g.B.cs_lo = 1;
    g.C.p = Q + (i64)(n - 1) * row; g.C.rs_lo = N; g.C.cdiv = N; g.C.cs_hi = es; g.C.cs_lo = 1;
    g.alpha = make_double2(dt * c.W.gregory(n, 0), 0.0);
    g.beta = make_double2(1.0, 0.0);
    gemm(g, c.stream);
  }
  boot_Q_kernel<<<nblk(row * k), TPB, 0, c.stream>>>(N, k, G, c.d_pdiff, dt, Q);
  NEDY_CHECK_LAUNCH();
  // the kN x kN matrix is the same for every tau point: invert it once
  double2 *M = c.ws.alloc<double2>((i64)kn * kn);
  double2 *Mi = c.ws.alloc<double2>((i64)kn * kn);
  boot_M_kernel<<<nblk((i64)kn * kn), TPB, 0, c.stream>>>(N, k, Sig, hmf, c.d_pdiff, c.greg, ld, mu, dt, M);
  NEDY_CHECK_LAUNCH();
  {
    std::vector<double2> I((size_t)kn * kn, make_double2(0.0, 0.0));
    for (int i = 0; i < kn; i++) I[(size_t)i * kn + i] = make_double2(1.0, 0.0);
    NEDY_CUDA(cudaMemcpyAsync(Mi, I.data(), sizeof(double2) * I.size(), cudaMemcpyHostToDevice, c.stream));
    gj_public(c, kn, kn, 1, M, 0, Mi, 0);
  }
  double2 *old = c.ws.alloc<double2>(row * k);
  NEDY_CUDA(cudaMemcpyAsync(old, G.tvptr(1, 0), sizeof(double2) * row * k, cudaMemcpyDeviceToDevice, c.stream));
  {  // G^tv(1..k, m) = Minv * Q(., m):  rows (n-1, i), columns (m, j)
    GemmArgs g;
    g.M = kn; g.N = np * N; g.K = kn;
    g.A = rowmajor(Mi, kn);
    g.B.p = Q; g.B.rdiv = N; g.B.rs_hi = row; g.B.rs_lo = N; g.B.cdiv = N; g.B.cs_hi = es; g.B.cs_lo = 1;
    g.C.p = G.tvptr(1, 0); g.C.rdiv = N; g.C.rs_hi = row; g.C.rs_lo = N; g.C.cdiv = N; g.C.cs_hi = es; g.C.cs_lo = 1;
    gemm(g, c.stream);
  }
  {  // error per (n, m) block, summed as norms
    double *e1 = c.ws.alloc<double>((i64)k * np);
    NEDY_CUDA(cudaMemsetAsync(e1, 0, sizeof(double) * k * np, c.stream));
    diffnorm_blocks_kernel<<<nblk(row * k), TPB, 0, c.stream>>>(N, k * np, old, G.tvptr(1, 0), e1);
    NEDY_CHECK_LAUNCH();
    err_total += host_sum_sqrt(c, e1, k * np);
  }
  {
    const int npairs = (k + 1) * (k + 1);
    double *e2 = c.ws.alloc<double>(npairs);
    NEDY_CUDA(cudaMemsetAsync(e2, 0, sizeof(double) * npairs, c.stream));
    boot_ret_kernel<<<nblk(es * (k + 1) * (k + 2) / 2), TPB, 0, c.stream>>>(N, k, G, e2);
    NEDY_CHECK_LAUNCH();
    err_total += host_sum_sqrt(c, e2, npairs);
    double *e3 = c.ws.alloc<double>(npairs);
    NEDY_CUDA(cudaMemsetAsync(e3, 0, sizeof(double) * npairs, c.stream));
    boot_les_kernel<<<nblk(es * (k + 1) * (k + 2) / 2), TPB, 0, c.stream>>>(N, k, G, e3);
    NEDY_CHECK_LAUNCH();
    err_total += host_sum_sqrt(c, e3, npairs);
  }
  check_status(c);
  return err_total;
}

double energy_conv(Ctx &c, int T, const DevGF &Sig, const DevGF &G) {
  NEDY_REQUIRE(T >= 0 && T <= G.nt && G.nt == Sig.nt && G.nao == Sig.nao, "energy_conv: bad arguments");
  ensure_tables(c);
  c.ws.reset();
  const int N = G.nao, k = c.k, top = T >= k ? T : k;
  double *out = c.ws.alloc<double>(4);
  NEDY_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * 4, c.stream));
  energy_hist_kernel<<<top + 1, TPB, 0, c.stream>>>(N, T, top, Sig, G, c.greg + (i64)T * (c.nt + 1), out);
  NEDY_CHECK_LAUNCH();
  energy_tv_kernel<<<nblk((i64)N * N), TPB, 0, c.stream>>>(N, T, Sig, G, c.d_w, c.d_u, c.col.ctop, out);
  NEDY_CHECK_LAUNCH();
  double h[4];
  NEDY_CUDA(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
  NEDY_CUDA(cudaStreamSynchronize(c.stream));
  const int sig = G.sig;
  // res1 = dt * hist ; res2 = -i * (-sig)(beta/2) S
  const double r1x = c.dt * h[0], r1y = c.dt * h[1];
  const double f = -(double)sig * 0.5 * c.beta;
  const double e2x = f * h[2], e2y = f * h[3];
  const double r2y = -e2x;  // Im(-i * e2)
  // Re( i sig/2 (res1 + res2) ) = -(sig/2) Im(res1 + res2)
  return -(double)sig * 0.5 * (r1y + r2y);
}

} // namespace nedy
