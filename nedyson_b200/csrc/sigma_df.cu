// Density-fitted second-Born (GF2) self-energy for one time row T, restricted and
// spin-unrestricted.  Replaces molGF2SolverDecomp::solve
// (reference src/mol2bSolver_decomp_impl.h:412-429) and
// molGF2SolverSpinDecomp::solve (src/mol2bSolver_spin_decomp_impl.h:436-466).
//
// Every slice (t' <= T for the lesser / retarded rows, every tau point for the
// mixed row) is the same trilinear map of three nao x nao blocks (X, Y, Z):
//   bubble   B(X,Y,Z) = f * sum_ab Tr[V^a Z V^b Y] V^a X V^b      (f = 2 restricted)
//   exchange E(X,Y,Z) = sum_ab V^a X V^b Y V^a Z V^b
//   Sigma    = B - E
// with (reference loops :431-670)
//   lesser   (X,Y,Z) = (L, R - L^+, L)                 L = G^<(t',T), R = G^R(T,t')
//   mixed    (X,Y,Z) = (G^tv(T,tau), -sig G^tv(T,ntau-tau)^+, G^tv(T,tau))
//   retarded T(R, L, R-L^+) + T(L^+, R^+, L^+) - T(L^+, L, R)
// The retarded exchange is evaluated as two "units" exactly like the reference
// (src/mol2bSolver_decomp_impl.h:293-402): M = (-L^+) V (L - R^+) with Z = R, and
// M = R V L + (-L^+) V R^+ with Z = R - L^+.
//
// Each contraction is a batched FP64 GEMM over the slices of a chunk; the N^4
// exchange intermediate S_{(l,n),(q,j)} lives only in a chunk-sized workspace.
#include "engine.cuh"
#include "sigma.cuh"
#include "split_gemm.cuh"
#include "../../include/nedy.h"

namespace nedy {
namespace {

enum PrepMode { PREP_LES = 0, PREP_TV = 1, PREP_RET = 2 };

// Per-slice derived blocks.  out[k][s] for k = 0..nout-1, each N x N.
//  LES: out0 = R - L^+                              (G^>(T,t'))
//  TV : out0 = -sig * Gv^+                          (G^lceil)
//  RET: out0 = L^+, out1 = R^+, out2 = R - L^+, out3 = L - R^+
__global__ void prep_kernel(int mode, int N, int nsl, const double2 *L0, i64 Ls, const double2 *R0, i64 Rs,
                            double sgn, double2 *out, i64 out_stride) {
  const i64 es = (i64)N * N;
  for (i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x; idx < es * nsl; idx += (i64)gridDim.x * blockDim.x) {
    const int s = (int)(idx / es);
    const int e = (int)(idx - (i64)s * es);
    const int i = e / N, j = e - (e / N) * N;
    if (mode == PREP_LES) {
      double2 r = R0[s * Rs + e];
      double2 lt = L0[s * Ls + (i64)j * N + i];
      out[s * es + e] = make_double2(r.x - lt.x, r.y + lt.y);
    } else if (mode == PREP_TV) {
      // L0 points at the mirrored node G^tv(T, ntau - tau0 - s), R0 unused; Ls < 0 walks back.
      double2 g = L0[s * Ls + (i64)j * N + i];
      out[s * es + e] = make_double2(sgn * g.x, -sgn * g.y);
    } else {
      double2 l = L0[s * Ls + e], lt = L0[s * Ls + (i64)j * N + i];
      double2 r = R0[s * Rs + e], rt = R0[s * Rs + (i64)j * N + i];
      (void)l;
      out[0 * out_stride + s * es + e] = make_double2(lt.x, -lt.y);            // L^+
      out[1 * out_stride + s * es + e] = make_double2(rt.x, -rt.y);            // R^+
      out[2 * out_stride + s * es + e] = make_double2(r.x - lt.x, r.y + lt.y); // R - L^+
      out[3 * out_stride + s * es + e] = make_double2(l.x - rt.x, l.y + rt.y); // L - R^+
    }
  }
}

struct Blocks {  // a batch of N x N blocks, block s at p + s * stride (elements)
  const double2 *p;
  i64 stride;
};

View blk(Blocks b, int N) {
  View v = rowmajor(b.p, N);
  v.bs1 = b.stride;
  return v;
}
View blkT(Blocks b, int N) {
  View v = transposed(b.p, N);
  v.bs1 = b.stride;
  return v;
}

struct DF {
  Ctx &c;
  int N, A, nsl;
  i64 es, NA, N2A;
  cudaStream_t s;
  DF(Ctx &cx, int nsl_) : c(cx), N(cx.df_nao), A(cx.df_naux), nsl(nsl_), s(cx.stream) {
    es = (i64)N * N;
    NA = (i64)N * A;
    N2A = es * A;
  }
  // VZ[s] = Viaj (NA x N) * Z_s   -> layout [n][a][q] = (V^a Z)_nq
  void VZ(Blocks Z, double2 *out) {
    GemmArgs g;
    g.M = (int)NA; g.N = N; g.K = N; g.nb1 = nsl;
    g.A = rowmajor(c.Viaj, N); g.a_cplx = false;
    g.B = blk(Z, N);
    g.C = rowmajor(out, N); g.C.bs1 = N2A;
    gemm(g, s);
  }
  // VYt[s] = Y_s^T * Vmbq  -> layout [n][b][q] = (V^b Y)_qn
  void VYt(Blocks Y, double2 *out) {
    GemmArgs g;
    g.M = N; g.N = (int)NA; g.K = N; g.nb1 = nsl;
    g.A = blkT(Y, N);
    g.B = rowmajor(c.Vmbq, NA); g.b_cplx = false;
    g.C = rowmajor(out, NA); g.C.bs1 = N2A;
    gemm(g, s);
  }
  // P[s] (+)= sign * sum_{(n,q)} VZ[s][n][a][q] * VYt[s][n][b][q]
  void P(const double2 *vz, const double2 *vyt, double2 *P, double sign, bool acc) {
    GemmArgs g;
    g.M = A; g.N = A; g.K = (int)es; g.nb1 = nsl;
    g.A.p = vz; g.A.rs_lo = N; g.A.cdiv = N; g.A.cs_hi = NA; g.A.cs_lo = 1; g.A.bs1 = N2A;
    g.B.p = vyt; g.B.rdiv = N; g.B.rs_hi = NA; g.B.rs_lo = 1; g.B.cs_lo = N; g.B.bs1 = N2A;
    g.C = rowmajor(P, A); g.C.bs1 = (i64)A * A;
    g.alpha = make_double2(sign, 0);
    g.beta = make_double2(acc ? 1.0 : 0.0, 0);
    gemm(g, s);
  }
  // W[s] = P[s] * Vaij  -> [a][(k,j)]
  void W(const double2 *P, double2 *W) {
    GemmArgs g;
    g.M = A; g.N = (int)es; g.K = A; g.nb1 = nsl;
    g.A = rowmajor(P, A); g.A.bs1 = (i64)A * A;
    g.B = rowmajor(c.Vaij, es); g.b_cplx = false;
    g.C = rowmajor(W, es); g.C.bs1 = N2A;
    gemm(g, s);
  }
  // Sigma_s += f * VZ(X)[s] (N x NA) * W[s] (NA x N)
  void SigB(const double2 *vzx, const double2 *W, Blocks Sig, double f) {
    GemmArgs g;
    g.M = N; g.N = N; g.K = (int)NA; g.nb1 = nsl;
    g.A = rowmajor(vzx, NA); g.A.bs1 = N2A;
    g.B = rowmajor(W, N); g.B.bs1 = N2A;
    g.C = blk(Sig, N);
    g.alpha = make_double2(f, 0);
    g.beta = make_double2(1.0, 0);
    gemm(g, s);
  }
  // M[s] (+)= alpha * X_s (N x N) * VY[s] (N x (b,n))   -> [l][b][n]
  void Mx(Blocks X, const double2 *vy, double2 *M, double alpha, bool acc) {
    GemmArgs g;
    g.M = N; g.N = (int)NA; g.K = N; g.nb1 = nsl;
    g.A = blk(X, N);
    g.B = rowmajor(vy, NA); g.B.bs1 = N2A;
    g.C = rowmajor(M, NA); g.C.bs1 = N2A;
    g.alpha = make_double2(alpha, 0);
    g.beta = make_double2(acc ? 1.0 : 0.0, 0);
    gemm(g, s);
  }
  // Split-precision layouts of the exchange operands:
  //   MT[s] = X_s * VY[s] stored [l][n][b] (rows (l,n), K = b contiguous)
  void MxT(Blocks X, const double2 *vy, double2 *MT, double alpha, bool acc) {
    GemmArgs g;
    g.M = N; g.N = (int)NA; g.K = N; g.nb1 = nsl;
    g.A = blk(X, N);
    g.B = rowmajor(vy, NA); g.B.bs1 = N2A;
    g.C.p = MT; g.C.rs_lo = NA; g.C.cdiv = N; g.C.cs_hi = 1; g.C.cs_lo = A; g.C.bs1 = N2A;
    g.alpha = make_double2(alpha, 0);
    g.beta = make_double2(acc ? 1.0 : 0.0, 0);
    gemm(g, s);
  }
  //   VZT[s] = (V^a Z_s)_{nq} stored [a][q][n] (rows a, K = (q,n) contiguous)
  void VZT(Blocks Z, double2 *out) {
    GemmArgs g;
    g.M = (int)NA; g.N = N; g.K = N; g.nb1 = nsl;
    g.A = rowmajor(c.Viaj, N); g.a_cplx = false;
    g.B = blk(Z, N);
    g.C.p = out; g.C.rdiv = A; g.C.rs_hi = 1; g.C.rs_lo = es; g.C.cs_lo = N; g.C.bs1 = N2A;
    gemm(g, s);
  }
  // BF16 pieces of Vija as the shared B operand of the split S contraction (rows (q,j), K = b).
  // Real static operands are split once into 3 pieces; piece p of a real array is plane p, so
  // the same planes serve a 2-piece view.
  Pieces vpieces(int np) {
    Pieces v;
    v.rows = (int)es; v.kpad = kpad64(A); v.nb = 1; v.ncomp = 1; v.np = 3;
    if (!c.Vp || c.Vp_np != 3) {
      if (c.Vp) cudaFree(c.Vp);
      c.Vp = nullptr;
      NEDY_CUDA(cudaMalloc(&c.Vp, v.elems() * 2));
      c.Vp_np = 3;
      v.p = (__nv_bfloat16 *)c.Vp;
      split_pieces(rowmajor(c.Vija, A), false, false, A, v, s);
    }
    v.p = (__nv_bfloat16 *)c.Vp;
    v.np = np;
    return v;
  }
  // Bubble contractions in split precision (same results as P() and W()):
  //   P[s] (+)= sign * sum_{(n,q)} VZ[s][n][a][q] VYt[s][n][b][q]   (A x A, K = N^2)
  void Psplit(const double2 *vz, const double2 *vyt, double2 *Pm, double sign, bool acc, void *wsA, void *wsB,
              int np) {
    Pieces a, b;
    a.rows = A; a.kpad = kpad64((int)es); a.nb = nsl; a.ncomp = 2; a.np = np; a.p = (__nv_bfloat16 *)wsA;
    b = a;
    b.p = (__nv_bfloat16 *)wsB;
    View va; va.p = vz; va.rs_lo = N; va.cdiv = N; va.cs_hi = NA; va.cs_lo = 1; va.bs1 = N2A;
    View vb; vb.p = vyt; vb.rs_lo = N; vb.cdiv = N; vb.cs_hi = NA; vb.cs_lo = 1; vb.bs1 = N2A;
    split_pieces(va, true, false, (int)es, a, s);
    split_pieces(vb, true, false, (int)es, b, s);
    SplitGemmArgs g;
    g.M = A; g.N = A; g.K = (int)es; g.nb = nsl;
    g.A = a; g.B = b;
    g.C = rowmajor(Pm, A); g.C.bs1 = (i64)A * A;
    g.alpha = sign;
    g.accumulate = acc;  // else P is replaced
    g.overwrite = !acc;
    g.zero_elems = (i64)nsl * A * A;
    split_gemm(g, s);
  }
  //   W[s] = P[s] (A x A) * Vaij (A x N^2): B operand = pieces of Vija (rows (k,j), K = a)
  void Wsplit(const double2 *Pm, double2 *Wm, void *wsP, int np) {
    Pieces a;
    a.rows = A; a.kpad = kpad64(A); a.nb = nsl; a.ncomp = 2; a.np = np; a.p = (__nv_bfloat16 *)wsP;
    View va = rowmajor(Pm, A); va.bs1 = (i64)A * A;
    split_pieces(va, true, false, A, a, s);
    SplitGemmArgs g;
    g.M = A; g.N = (int)es; g.K = A; g.nb = nsl;
    g.A = a; g.B = vpieces(np);
    g.C = rowmajor(Wm, es); g.C.bs1 = N2A;
    split_gemm(g, s);
  }
  i64 pz_bytes(int np) const { return (i64)2 * np * nsl * A * kpad64((int)es) * 2; }
  i64 pp_bytes(int np) const { return (i64)2 * np * nsl * A * kpad64(A) * 2; }
  // ---- all-split chain of the les-form units (X, Y, Z = X): every operand a BF16-piece
  // array written directly by the producing contraction in the layout its consumer reads.
  Pieces static_pieces(void *&slot, const View &v, int rows, int K, int np) {
    Pieces x;
    x.rows = rows; x.kpad = kpad64(K); x.nb = 1; x.ncomp = 1; x.np = 3;
    if (!slot) {
      NEDY_CUDA(cudaMalloc(&slot, x.elems() * 2));
      x.p = (__nv_bfloat16 *)slot;
      split_pieces(v, false, false, K, x, s);
    }
    x.p = (__nv_bfloat16 *)slot;
    x.np = np;
    return x;
  }
  Pieces vanj(int np) {  // rows (a,n), K = j: V^a_nj = Vija[n][j][a]
    View v; v.p = c.Vija; v.rdiv = N; v.rs_hi = 1; v.rs_lo = NA; v.cs_lo = A;
    return static_pieces(c.Vanj_p, v, (int)NA, N, np);
  }
  Pieces vjkb(int np) {  // rows (j,k), K = b: V^b_kj = Vija[k][j][b] (= Vija rows (j,k) when symmetric)
    if (c.V_sym) return vpieces(np);
    View v; v.p = c.Vija; v.rdiv = N; v.rs_hi = A; v.rs_lo = NA; v.cs_lo = 1;
    return static_pieces(c.Vjkb_p, v, (int)es, A, np);
  }
  Pieces vila(int np) {  // rows i, K = (l,a): Vija[i][l][a]
    return static_pieces(c.Vila_p, rowmajor(c.Vija, NA), N, (int)NA, np);
  }
  Pieces arr(void *p, int rows, int K, int nb, int np) {
    Pieces x;
    x.p = (__nv_bfloat16 *)p; x.rows = rows; x.kpad = kpad64(K); x.nb = nb; x.ncomp = 2; x.np = np;
    return x;
  }
  static i64 arr_bytes(int rows, int K, int nb, int np) { return (i64)2 * np * nb * rows * kpad64(K) * 2; }
  // C (pieces, zero-padded K) = A * B^T
  void to_pieces(const Pieces &a, const Pieces &b, int M, int Nn, int K, Pieces &out, const View &ov, int nb,
                 int out_K) {
    if (out.kpad != out_K)  // the GEMM writes columns [0, out_K) of every row; zero the K padding only
      NEDY_CUDA(cudaMemset2DAsync(out.p + out_K, (size_t)out.kpad * 2, 0, (size_t)(out.kpad - out_K) * 2,
                                  (size_t)(out.elems() / out.kpad), s));
    SplitGemmArgs g;
    g.M = M; g.N = Nn; g.K = K; g.nb = nb;
    g.A = a; g.B = b;
    g.out_pieces = true; g.Cp = out; g.C = ov;
    split_gemm(g, s);
  }
  // C (FP64) += alpha * A * B^T, or, with zero_elems > 0, C = alpha * A * B^T replacing the
  // first zero_elems complex elements from cv.p (the whole output range)
  void to_fp64(const Pieces &a, const Pieces &b, int M, int Nn, int K, const View &cv, int nb, double alpha,
               i64 zero_elems = 0) {
    SplitGemmArgs g;
    g.M = M; g.N = Nn; g.K = K; g.nb = nb;
    g.A = a; g.B = b;
    g.C = cv; g.alpha = alpha;
    g.accumulate = zero_elems == 0;
    g.overwrite = zero_elems > 0;
    g.zero_elems = zero_elems;
    split_gemm(g, s);
  }
  Pieces blk_pieces(Blocks b, bool transpose, void *buf, int np) {
    Pieces x = arr(buf, N, N, nsl, np);
    split_pieces(transpose ? blkT(b, N) : blk(b, N), true, false, N, x, s);
    return x;
  }
  // VZa = [a][(q,n)] pieces of (V^a Z)_nq for P (A operand) and Q (B operand)
  Pieces VZa(const Pieces &zt, void *buf, int np) {
    Pieces o = arr(buf, A, (int)es, nsl, np);
    View v; v.rdiv = N; v.rs_hi = o.kpad; v.rs_lo = 1; v.cs_lo = N; v.bs1 = (i64)A * o.kpad;
    to_pieces(vanj(np), zt, (int)NA, N, N, o, v, nsl, (int)es);
    return o;
  }
  // VYb = [b][(q,n)] pieces of (V^b Y)_qn for P (B operand)
  Pieces VYb(const Pieces &yt, void *buf, int np) {
    Pieces o = arr(buf, A, (int)es, nsl, np);
    View v; v.rdiv = N; v.rs_hi = o.kpad; v.rs_lo = N; v.cs_lo = 1; v.bs1 = (i64)A * o.kpad;
    to_pieces(vanj(np), yt, (int)NA, N, N, o, v, nsl, (int)es);
    return o;
  }
  // VZn = [n][(a,k)] pieces of (V^a X)_nk for the bubble contraction (A operand)
  Pieces VZn(const Pieces &xt, void *buf, int np) {
    Pieces o = arr(buf, N, (int)NA, nsl, np);
    View v; v.rdiv = N; v.rs_hi = N; v.rs_lo = o.kpad; v.cs_lo = 1; v.bs1 = (i64)N * o.kpad;
    to_pieces(vanj(np), xt, (int)NA, N, N, o, v, nsl, (int)NA);
    return o;
  }
  // VYp = [(n,b)][k] pieces of (V^b Y)_kn for the M contraction (B operand)
  Pieces VYp(const Pieces &yt, void *buf, int np) {
    Pieces o = arr(buf, (int)NA, N, nsl, np);
    View v; v.rdiv = N; v.rs_hi = o.kpad; v.rs_lo = 1; v.cs_lo = (i64)A * o.kpad; v.bs1 = NA * o.kpad;
    to_pieces(vanj(np), yt, (int)NA, N, N, o, v, nsl, N);
    return o;
  }
  // Wp = [j][(a,k)] pieces of W[a][k][j] = sum_b P[a][b] V^b_kj (B operand of the bubble)
  Pieces Wp(const Pieces &pp, void *buf, int np) {
    Pieces o = arr(buf, N, (int)NA, nsl, np);
    View v; v.rdiv = N; v.rs_hi = o.kpad; v.rs_lo = 1; v.cs_lo = N; v.bs1 = (i64)N * o.kpad;
    to_pieces(vjkb(np), pp, (int)es, A, A, o, v, nsl, (int)NA);
    return o;
  }
  // exchange of units u0..u0+nu-1: Mp = X VY, S', Q, Sigma -= V Q
  void ExchAllSplit(int u0, int nu, const Pieces &xp, const Pieces &vyp, const Pieces &vza, Blocks Sig, double2 *Q,
                    void *wsS, void *wsM, void *wsQ, int np) {
    const int kpN = kpad64((int)es);
    Pieces xs = xp, vs = vyp, zs = vza;
    xs.b0 = vs.b0 = zs.b0 = u0;
    Pieces Mp;
    Mp.p = (__nv_bfloat16 *)wsM; Mp.rows = (int)es; Mp.kpad = kpad64(A); Mp.nb = nu; Mp.ncomp = 2; Mp.np = np;
    {
      View v; v.rs_lo = (i64)N * Mp.kpad; v.cdiv = A; v.cs_hi = Mp.kpad; v.cs_lo = 1; v.bs1 = es * Mp.kpad;
      to_pieces(xs, vs, N, (int)NA, N, Mp, v, nu, A);
    }
    Pieces Sp;
    Sp.p = (__nv_bfloat16 *)wsS; Sp.rows = (int)es; Sp.kpad = kpN; Sp.nb = nu; Sp.ncomp = 2; Sp.np = np;
    {
      View v; v.rdiv = N; v.rs_hi = N; v.rs_lo = kpN; v.cdiv = N; v.cs_hi = (i64)N * kpN; v.cs_lo = 1; v.bs1 = es * kpN;
      to_pieces(vpieces(np), Mp, (int)es, (int)es, A, Sp, v, nu, (int)es);
    }
    {
      View v; v.p = Q; v.rdiv = N; v.rs_hi = A; v.rs_lo = NA; v.cs_lo = 1; v.bs1 = N2A;
      to_fp64(Sp, zs, (int)es, A, (int)es, v, nu, 1.0, (i64)nu * N2A);
    }
    Pieces Qp;
    Qp.p = (__nv_bfloat16 *)wsQ; Qp.rows = N; Qp.kpad = kpad64((int)NA); Qp.nb = nu; Qp.ncomp = 2; Qp.np = np;
    {
      View v = rowmajor(Q, NA); v.bs1 = N2A;
      split_pieces(v, true, false, (int)NA, Qp, s);
    }
    to_fp64(vila(np), Qp, N, N, (int)NA, blk(Sig, N), nu, -1.0);
  }

  // bytes of the MT / VZT piece planes for nu units
  i64 mz_bytes(int nu, int np) const {
    return std::max<i64>((i64)2 * np * nu * es * kpad64(A), (i64)2 * np * nu * A * kpad64((int)es)) * 2;
  }
  // Exchange of nu units with the two N^4 A contractions in split precision:
  //   S'[u][(l,j)][(q,n)] = sum_b V^b_qj MT[u][(l,n)][b]          (BF16 pieces out)
  //   Q[u][j][l][a]      = sum_{(q,n)} S'[u][(l,j)][(q,n)] VZT[u][a][(q,n)]   (FP64 out)
  //   Sigma_u           -= sum_{l,a} V^a_il Q[u][j][l][a]            (FP64)
  // wsS, wsM, wsZ: scratch for the S', MT and VZT pieces (split_bytes() each, for nu units)
  void ExchSplit(int nu, const double2 *MT, const double2 *vzt, Blocks Sig, double2 *Q, void *wsS, void *wsM,
                 void *wsZ, int np) {
    const int kpA = kpad64(A), kpN = kpad64((int)es);
    Pieces Mp, Zp, Sp;
    Mp.rows = (int)es; Mp.kpad = kpA; Mp.nb = nu; Mp.ncomp = 2; Mp.np = np;
    Zp.rows = A; Zp.kpad = kpN; Zp.nb = nu; Zp.ncomp = 2; Zp.np = np;
    Sp.rows = (int)es; Sp.kpad = kpN; Sp.nb = nu; Sp.ncomp = 2; Sp.np = np;
    Sp.p = (__nv_bfloat16 *)wsS;
    Mp.p = (__nv_bfloat16 *)wsM;
    Zp.p = (__nv_bfloat16 *)wsZ;
    {
      View v = rowmajor(MT, A); v.bs1 = N2A;
      split_pieces(v, true, false, A, Mp, s);
      View w = rowmajor(vzt, es); w.bs1 = N2A;
      split_pieces(w, true, false, (int)es, Zp, s);
    }
    if (kpN != es)  // only the K padding of every S' row must be zero (the GEMM writes the rest)
      NEDY_CUDA(cudaMemset2DAsync(Sp.p + es, (size_t)kpN * 2, 0, (size_t)(kpN - es) * 2,
                                  (size_t)(Sp.elems() / kpN), s));
    {  // computed as S^T (rows (q,j), columns (l,n)) so that each thread stores runs of n
      SplitGemmArgs g;
      g.M = (int)es; g.N = (int)es; g.K = A; g.nb = nu;
      g.A = vpieces(np); g.B = Mp;
      g.out_pieces = true; g.Cp = Sp;
      g.C.rdiv = N; g.C.rs_hi = N; g.C.rs_lo = kpN;
      g.C.cdiv = N; g.C.cs_hi = (i64)N * kpN; g.C.cs_lo = 1;
      g.C.bs1 = es * kpN;
      split_gemm(g, s);
    }
    {  // Q replaced (every element of the nu units stored once; cleared first under a K split)
      SplitGemmArgs g;
      g.M = (int)es; g.N = A; g.K = (int)es; g.nb = nu;
      g.A = Sp; g.B = Zp;
      g.C.p = Q; g.C.rdiv = N; g.C.rs_hi = A; g.C.rs_lo = NA; g.C.cs_lo = 1; g.C.bs1 = N2A;
      g.overwrite = true;
      g.zero_elems = (i64)nu * N2A;
      split_gemm(g, s);
    }
    {
      GemmArgs g;
      g.M = N; g.N = N; g.K = (int)NA; g.nb1 = nu;
      g.A = rowmajor(c.Vija, NA); g.a_cplx = false;
      g.B.p = Q; g.B.rs_lo = 1; g.B.cs_lo = NA; g.B.bs1 = N2A;
      g.C = blk(Sig, N);
      g.alpha = make_double2(-1.0, 0);
      g.beta = make_double2(1.0, 0);
      gemm(g, s);
    }
  }
  // Exchange for units u0..u0+nu-1 of this chunk: Sigma_u -= sum_{l,a} V^a_il Q[l][j][a]
  //   S[u][(l,n)][(q,j)] = sum_b M[u][l][b][n] V^b_qj ;  Q[u][j][l][a] = sum_{(n,q)} S[u][l][(n,q)][j] VZ(Z)[u][n][a][q]
  void Exch(int nu, const double2 *M, const double2 *vzz, Blocks Sig, double2 *S, double2 *Q) {
    {
      GemmArgs g;
      g.M = (int)es; g.N = (int)es; g.K = A; g.nb1 = nu;
      g.A.p = M; g.A.rdiv = N; g.A.rs_hi = NA; g.A.rs_lo = 1; g.A.cs_lo = N; g.A.bs1 = N2A;
      g.B = rowmajor(c.Vaij, es); g.b_cplx = false;
      g.C = rowmajor(S, es); g.C.bs1 = es * es;
      gemm(g, s);
    }
    {
      GemmArgs g;
      g.M = N; g.N = A; g.K = (int)es; g.nb1 = nu; g.nb2 = N;
      g.A.p = S; g.A.rs_lo = 1; g.A.cs_lo = N; g.A.bs1 = es * es; g.A.bs2 = es * N;
      g.B.p = vzz; g.B.rdiv = N; g.B.rs_hi = NA; g.B.rs_lo = 1; g.B.cs_lo = N; g.B.bs1 = N2A; g.B.bs2 = 0;
      g.C.p = Q; g.C.rs_lo = NA; g.C.cs_lo = 1; g.C.bs1 = N2A; g.C.bs2 = A;
      gemm(g, s);
    }
    {
      GemmArgs g;
      g.M = N; g.N = N; g.K = (int)NA; g.nb1 = nu;
      g.A = rowmajor(c.Vija, NA); g.a_cplx = false;
      g.B.p = Q; g.B.rs_lo = 1; g.B.cs_lo = NA; g.B.bs1 = N2A;
      g.C = blk(Sig, N);
      g.alpha = make_double2(-1.0, 0);
      g.beta = make_double2(1.0, 0);
      gemm(g, s);
    }
  }
};

// out_s += in_s^+ for nb consecutive N x N blocks
__global__ void adj_add_kernel(int N, int nb, const double2 *in, double2 *out) {
  const i64 es = (i64)N * N;
  for (i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x; idx < es * nb; idx += (i64)gridDim.x * blockDim.x) {
    const int b = (int)(idx / es), e = (int)(idx - (i64)b * es);
    const int i = e / N, j = e - (e / N) * N;
    const double2 v = in[(i64)b * es + (i64)j * N + i];
    out[idx] = make_double2(out[idx].x + v.x, out[idx].y - v.y);
  }
}

void adj_add(Ctx &c, int N, int nb, const double2 *in, double2 *out) {
  i64 tot = (i64)N * N * nb;
  adj_add_kernel<<<(unsigned)std::min<i64>((tot + 255) / 256, 65535LL * 8), 256, 0, c.stream>>>(N, nb, in, out);
  NEDY_CHECK_LAUNCH();
}

void prep(Ctx &c, int mode, int nsl, const double2 *L0, i64 Ls, const double2 *R0, i64 Rs, double sgn,
          double2 *out, i64 out_stride) {
  int N = c.df_nao;
  i64 tot = (i64)N * N * nsl;
  int th = 256;
  unsigned bl = (unsigned)std::min<i64>((tot + th - 1) / th, 65535LL * 8);
  prep_kernel<<<bl, th, 0, c.stream>>>(mode, N, nsl, L0, Ls, R0, Rs, sgn, out, out_stride);
  NEDY_CHECK_LAUNCH();
}

} // namespace

// Chunk sizes: slices per chunk and exchange units per S buffer, from the workspace budget
// (host arithmetic only; sms = streaming multiprocessors of the device).
void chunk_plan(i64 N, i64 A, i64 budget, bool split, bool vsym, int np_pieces, int sms, int &chunk, int &sub) {
  i64 n2a = N * N * A * 16;  // bytes of one [n][a][q] intermediate
  i64 n4 = N * N * N * N * 16;
  // per slice (retarded, the largest): 5 VZ/VYt + 3 VY + 2 M + Q + 2 P/W + prep
  i64 per = 13 * n2a + 2 * A * A * 16;
  if (split) per += 6 * n2a;  // BF16 pieces of the operands (12 bytes per complex element each)
  sub = (int)std::max<i64>(1, std::min<i64>(16, (budget / 3) / n4));
  chunk = (int)std::max<i64>(1, std::min<i64>(64, (budget - sub * n4) / std::max<i64>(per, 1)));
  if (chunk < sub) sub = chunk;
  if (!split || !vsym) return;
  // all-split chain (les-form units only): the intermediates are BF16 pieces
  const i64 np = np_pieces, pb = 4 * np;  // bytes per complex element
  const i64 es = N * N, kpN = kpad64((int)es), kpA = kpad64((int)A), kpNA = kpad64((int)(N * A));
  const i64 unit = pb * (es * kpN + es * kpA + N * kpNA) + n2a;  // S', MT and Q pieces, Q (FP64)
  per = 6 * pb * A * kpN + n2a + A * A * 16 + 8 * es * 16;
  const int sub_max = (int)std::max<i64>(1, std::min<i64>(48, (budget / 2) / unit));
  // units per exchange launch: the Q contraction has ceil(nao^2 / 128) row tiles per unit;
  // take the largest count whose tiles fill at least 95% of their last wave of CTAs (one
  // per SM), else the best filled one
  const i64 tiles = (es + 127) / 128;
  int pick = 0;
  double best = -1.0;
  int best_u = 1;
  for (int u = sub_max; u >= 1; u--) {
    const double w = (double)(tiles * u) / std::max(1, sms), eff = w / std::ceil(w);
    if (eff >= 0.95) {
      pick = u;
      break;
    }
    if (eff > best) {
      best = eff;
      best_u = u;
    }
  }
  sub = pick ? pick : best_u;
  chunk = (int)std::max<i64>(1, std::min<i64>(64, (budget - sub * unit) / std::max<i64>(per, 1)));
  if (chunk >= sub)
    chunk -= chunk % sub;
  else
    sub = chunk;
}

static void chunking(const Ctx &c, int &chunk, int &sub, bool split) {
  int dev = 0, sms = 148;
  if (split && c.V_sym && cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  chunk_plan(c.df_nao, c.df_naux, c.ws_budget, split, c.V_sym, c.precision == NEDY_PREC_SPLIT_BF16X2 ? 2 : 3, sms,
             chunk, sub);
}

void sigma_df(Ctx &c, int T, int nspin, DevGF *const *Sig, const DevGF *const *G) {
  NEDY_REQUIRE(c.Vija != nullptr, "sigma_df: density-fitted tensor not set");
  NEDY_REQUIRE(nspin == 1 || nspin == 2, "sigma_df: nspin must be 1 or 2");
  const int N = c.df_nao, A = c.df_naux;
  for (int s = 0; s < nspin; s++) {
    NEDY_REQUIRE(G[s]->nao == N && Sig[s]->nao == N, "sigma_df: nao mismatch");
    NEDY_REQUIRE(T >= 0 && T <= G[s]->nt && T <= Sig[s]->nt, "sigma_df: tstp out of range");
    NEDY_REQUIRE(G[s]->ntau == Sig[s]->ntau && G[s]->sig == Sig[s]->sig, "sigma_df: shape mismatch");
  }
  const i64 es = (i64)N * N, N2A = es * A, NA = (i64)N * A;
  const int ntau = G[0]->ntau, sig = G[0]->sig;
  const double fb = nspin == 1 ? 2.0 : 1.0;
  // set_tstp_zero (greens.h:76-86)
  for (int s = 0; s < nspin; s++) {
    NEDY_CUDA(cudaMemsetAsync(Sig[s]->retptr(T, 0), 0, sizeof(double2) * (T + 1) * es, c.stream));
    NEDY_CUDA(cudaMemsetAsync(Sig[s]->lesptr(0, T), 0, sizeof(double2) * (T + 1) * es, c.stream));
    NEDY_CUDA(cudaMemsetAsync(Sig[s]->tvptr(T, 0), 0, sizeof(double2) * (ntau + 1) * es, c.stream));
  }
  const bool split = c.precision != NEDY_PREC_FP64;
  int chunk, sub;
  chunking(c, chunk, sub, split);
  const int np = c.precision == NEDY_PREC_SPLIT_BF16X2 ? 2 : 3;
  if (split) NEDY_REQUIRE(kpad64((int)es) <= 65535 * 64, "split self-energy: nao too large");

  // ---------------- lesser and mixed rows: one bubble unit + one exchange unit per slice.
  // With real symmetric B^Q the retarded row is Sigma^>(T,t') + Sigma^<(t',T)^+ (kind 2), where
  // Sigma^>(T,t') is the same les-form unit with X = Z = G^>(T,t') = R - L^+ and Y = L.
  const int nkinds = c.V_sym ? 3 : 2;
  for (int kind = 0; kind < nkinds; kind++) {
    const int nslices = kind == 1 ? ntau + 1 : T + 1;
    for (int t0 = 0; t0 < nslices; t0 += chunk) {
      const int nsl = std::min(chunk, nslices - t0);
      c.ws.reset();
      DF d(c, nsl);
      double2 *Hb[2], *VZ[2], *VYt[2];
      Blocks X[2], Y[2];
      const bool allsplit = split;  // les-form units: every contraction in split precision
      for (int s = 0; s < nspin; s++) {
        Hb[s] = c.ws.alloc<double2>(nsl * es);
        if (kind == 1) {
          X[s] = {G[s]->tvptr(T, t0), es};
          prep(c, PREP_TV, nsl, G[s]->tvptr(T, ntau - t0), -es, nullptr, 0, -(double)sig, Hb[s], 0);
          Y[s] = {Hb[s], es};
        } else {
          prep(c, PREP_LES, nsl, G[s]->lesptr(t0, T), es, G[s]->retptr(T, t0), es, 0, Hb[s], 0);
          if (kind == 0) {
            X[s] = {G[s]->lesptr(t0, T), es};
            Y[s] = {Hb[s], es};
          } else {
            X[s] = {Hb[s], es};
            Y[s] = {G[s]->lesptr(t0, T), es};
          }
        }
        if (allsplit) continue;
        VZ[s] = c.ws.alloc<double2>(nsl * N2A);
        VYt[s] = c.ws.alloc<double2>(nsl * N2A);
        d.VZ(X[s], VZ[s]);
        d.VYt(Y[s], VYt[s]);
      }
      auto outb = [&](int s) {
        return kind == 0 ? Blocks{Sig[s]->lesptr(t0, T), es}
                         : (kind == 1 ? Blocks{Sig[s]->tvptr(T, t0), es} : Blocks{Sig[s]->retptr(T, t0), es});
      };
      if (allsplit) {
        // each piece array sized for its own rows x padded K
        const i64 bb = DF::arr_bytes(N, N, nsl, np), big = DF::arr_bytes(A, (int)es, nsl, np);
        const i64 nk = DF::arr_bytes(N, (int)NA, nsl, np), vyk = DF::arr_bytes((int)NA, N, nsl, np);
        Pieces xp[2], xtp[2], ytp[2], vza[2];
        for (int s = 0; s < nspin; s++) {
          xp[s] = d.blk_pieces(X[s], false, c.ws.get(bb), np);
          xtp[s] = d.blk_pieces(X[s], true, c.ws.get(bb), np);
          ytp[s] = d.blk_pieces(Y[s], true, c.ws.get(bb), np);
          vza[s] = d.VZa(xtp[s], c.ws.get(big), np);
        }
        // bubble: P = sum_s VZa VYb^T (FP64), W pieces, Sigma_s += f VZn W
        double2 *P = c.ws.alloc<double2>((i64)nsl * A * A);
        void *vyb = c.ws.get(big);
        for (int s = 0; s < nspin; s++) {  // the first spin replaces P, the second adds to it
          Pieces yb = d.VYb(ytp[s], vyb, np);
          View pv = rowmajor(P, A); pv.bs1 = (i64)A * A;
          d.to_fp64(vza[s], yb, A, A, (int)es, pv, nsl, 1.0, s == 0 ? (i64)nsl * A * A : 0);
        }
        Pieces pp = d.arr(c.ws.get(DF::arr_bytes(A, A, nsl, np)), A, A, nsl, np);
        {
          View pv = rowmajor(P, A); pv.bs1 = (i64)A * A;
          split_pieces(pv, true, false, A, pp, c.stream);
        }
        Pieces wp = d.Wp(pp, c.ws.get(nk), np);
        void *vzn = c.ws.get(nk);
        for (int s = 0; s < nspin; s++) {
          Pieces zn = d.VZn(xtp[s], vzn, np);
          d.to_fp64(zn, wp, N, N, (int)NA, blk(outb(s), N), nsl, fb);
        }
        // exchange per spin
        double2 *Q = c.ws.alloc<double2>(nsl * N2A);
        void *S = c.ws.get(DF::arr_bytes((int)es, (int)es, sub, np));
        void *vyp = c.ws.get(vyk);
        void *Mb = c.ws.get(DF::arr_bytes((int)es, A, sub, np));
        void *Qb = c.ws.get(DF::arr_bytes(N, (int)NA, sub, np));
        for (int s = 0; s < nspin; s++) {
          Pieces yp = d.VYp(ytp[s], vyp, np);
          Blocks out = outb(s);
          for (int u0 = 0; u0 < nsl; u0 += sub) {
            const int nu = std::min(sub, nsl - u0);
            d.ExchAllSplit(u0, nu, xp[s], yp, vza[s], {out.p + u0 * es, es}, Q + u0 * N2A, S, Mb, Qb, np);
          }
        }
        continue;
      }
      double2 *P = c.ws.alloc<double2>((i64)nsl * A * A);
      double2 *Wb = c.ws.alloc<double2>(nsl * N2A);
      if (split) {
        void *pa = c.ws.get(d.pz_bytes(np)), *pb = c.ws.get(d.pz_bytes(np)), *pp = c.ws.get(d.pp_bytes(np));
        for (int s = 0; s < nspin; s++) d.Psplit(VZ[s], VYt[s], P, 1.0, s > 0, pa, pb, np);
        d.Wsplit(P, Wb, pp, np);
      } else {
        for (int s = 0; s < nspin; s++) d.P(VZ[s], VYt[s], P, 1.0, s > 0);
        d.W(P, Wb);
      }
      for (int s = 0; s < nspin; s++) d.SigB(VZ[s], Wb, outb(s), fb);
      // exchange (per spin): M = X V Y, Z = X
      double2 *VY = c.ws.alloc<double2>(nsl * N2A);
      double2 *M = c.ws.alloc<double2>(nsl * N2A);
      double2 *Q = c.ws.alloc<double2>(nsl * N2A);
      double2 *S = c.ws.alloc<double2>((i64)sub * es * es);
      double2 *VZt = split ? c.ws.alloc<double2>(nsl * N2A) : nullptr;
      void *Mb = split ? c.ws.get(d.mz_bytes(sub, np)) : nullptr;
      void *Zb = split ? c.ws.get(d.mz_bytes(sub, np)) : nullptr;
      for (int s = 0; s < nspin; s++) {
        d.VZ(Y[s], VY);
        Blocks out = outb(s);
        if (split) {
          d.MxT(X[s], VY, M, 1.0, false);
          d.VZT(X[s], VZt);
          for (int u0 = 0; u0 < nsl; u0 += sub) {
            int nu = std::min(sub, nsl - u0);
            d.ExchSplit(nu, M + u0 * N2A, VZt + u0 * N2A, {out.p + u0 * es, es}, Q + u0 * N2A, S, Mb, Zb, np);
          }
          continue;
        }
        d.Mx(X[s], VY, M, 1.0, false);
        for (int u0 = 0; u0 < nsl; u0 += sub) {
          int nu = std::min(sub, nsl - u0);
          d.Exch(nu, M + u0 * N2A, VZ[s] + u0 * N2A, {out.p + u0 * es, es}, S, Q + u0 * N2A);
        }
      }
    }
  }
  if (c.V_sym) {
    for (int s = 0; s < nspin; s++) adj_add(c, N, T + 1, Sig[s]->lesptr(0, T), Sig[s]->retptr(T, 0));
    if (split && split_gemm_error(c.stream)) throw CudaError("split-precision GEMM: a bounded device wait timed out");
    return;
  }

  // ---------------- retarded row: two bubble units + two exchange units per slice
  for (int t0 = 0; t0 <= T; t0 += chunk) {
    const int nsl = std::min(chunk, T + 1 - t0);
    c.ws.reset();
    DF d(c, nsl);
    double2 *D[2];  // per spin: 4 derived blocks per slice (L^+, R^+, R-L^+, L-R^+)
    Blocks L[2], R[2], Lh[2], Rh[2], Zd[2], Y1[2];
    double2 *vzZd[2], *vzLh[2], *vzR[2], *vytL[2], *vytRh[2];
    for (int s = 0; s < nspin; s++) {
      D[s] = c.ws.alloc<double2>(4 * nsl * es);
      prep(c, PREP_RET, nsl, G[s]->lesptr(t0, T), es, G[s]->retptr(T, t0), es, 0, D[s], nsl * es);
      L[s] = {G[s]->lesptr(t0, T), es};
      R[s] = {G[s]->retptr(T, t0), es};
      Lh[s] = {D[s], es};
      Rh[s] = {D[s] + nsl * es, es};
      Zd[s] = {D[s] + 2 * nsl * es, es};
      Y1[s] = {D[s] + 3 * nsl * es, es};
      vzZd[s] = c.ws.alloc<double2>(nsl * N2A);
      vzLh[s] = c.ws.alloc<double2>(nsl * N2A);
      vzR[s] = c.ws.alloc<double2>(nsl * N2A);
      vytL[s] = c.ws.alloc<double2>(nsl * N2A);
      vytRh[s] = c.ws.alloc<double2>(nsl * N2A);
      d.VZ(Zd[s], vzZd[s]);
      d.VZ(Lh[s], vzLh[s]);
      d.VZ(R[s], vzR[s]);
      d.VYt(L[s], vytL[s]);
      d.VYt(Rh[s], vytRh[s]);
    }
    double2 *PA = c.ws.alloc<double2>((i64)nsl * A * A);
    double2 *PB = c.ws.alloc<double2>((i64)nsl * A * A);
    double2 *WA = c.ws.alloc<double2>(nsl * N2A);
    double2 *WB = c.ws.alloc<double2>(nsl * N2A);
    if (split) {
      void *pa = c.ws.get(d.pz_bytes(np)), *pb = c.ws.get(d.pz_bytes(np)), *pp = c.ws.get(d.pp_bytes(np));
      for (int s = 0; s < nspin; s++) {
        d.Psplit(vzZd[s], vytL[s], PA, 1.0, s > 0, pa, pb, np);
        d.Psplit(vzLh[s], vytRh[s], PB, 1.0, s > 0, pa, pb, np);
        d.Psplit(vzR[s], vytL[s], PB, -1.0, true, pa, pb, np);
      }
      d.Wsplit(PA, WA, pp, np);
      d.Wsplit(PB, WB, pp, np);
    } else {
      for (int s = 0; s < nspin; s++) {
        d.P(vzZd[s], vytL[s], PA, 1.0, s > 0);
        d.P(vzLh[s], vytRh[s], PB, 1.0, s > 0);
        d.P(vzR[s], vytL[s], PB, -1.0, true);
      }
      d.W(PA, WA);
      d.W(PB, WB);
    }
    for (int s = 0; s < nspin; s++) {
      Blocks out = {Sig[s]->retptr(T, t0), es};
      d.SigB(vzR[s], WA, out, fb);
      d.SigB(vzLh[s], WB, out, fb);
    }
    // exchange units per spin
    double2 *VY = c.ws.alloc<double2>(nsl * N2A);
    double2 *M = c.ws.alloc<double2>(nsl * N2A);
    double2 *Q = c.ws.alloc<double2>(nsl * N2A);
    double2 *S = c.ws.alloc<double2>((i64)sub * es * es);
    double2 *VZt = split ? c.ws.alloc<double2>(nsl * N2A) : nullptr;
    void *Mb = split ? c.ws.get(d.mz_bytes(sub, np)) : nullptr;
    void *Zb = split ? c.ws.get(d.mz_bytes(sub, np)) : nullptr;
    for (int s = 0; s < nspin; s++) {
      Blocks out = {Sig[s]->retptr(T, t0), es};
      // unit 1: M = (-L^+) V (L - R^+), Z = R
      d.VZ(Y1[s], VY);
      if (split) {
        d.MxT(Lh[s], VY, M, -1.0, false);
        d.VZT(R[s], VZt);
      } else {
        d.Mx(Lh[s], VY, M, -1.0, false);
      }
      for (int u0 = 0; u0 < nsl; u0 += sub) {
        int nu = std::min(sub, nsl - u0);
        if (split)
          d.ExchSplit(nu, M + u0 * N2A, VZt + u0 * N2A, {out.p + u0 * es, es}, Q + u0 * N2A, S, Mb, Zb, np);
        else
          d.Exch(nu, M + u0 * N2A, vzR[s] + u0 * N2A, {out.p + u0 * es, es}, S, Q + u0 * N2A);
      }
      // unit 2: M = R V L + (-L^+) V R^+, Z = R - L^+
      d.VZ(L[s], VY);
      if (split) {
        d.MxT(R[s], VY, M, 1.0, false);
        d.VZ(Rh[s], VY);
        d.MxT(Lh[s], VY, M, -1.0, true);
        d.VZT(Zd[s], VZt);
      } else {
        d.Mx(R[s], VY, M, 1.0, false);
        d.VZ(Rh[s], VY);
        d.Mx(Lh[s], VY, M, -1.0, true);
      }
      for (int u0 = 0; u0 < nsl; u0 += sub) {
        int nu = std::min(sub, nsl - u0);
        if (split)
          d.ExchSplit(nu, M + u0 * N2A, VZt + u0 * N2A, {out.p + u0 * es, es}, Q + u0 * N2A, S, Mb, Zb, np);
        else
          d.Exch(nu, M + u0 * N2A, vzZd[s] + u0 * N2A, {out.p + u0 * es, es}, S, Q + u0 * N2A);
      }
    }
  }
  if (split && split_gemm_error(c.stream)) throw CudaError("split-precision GEMM: a bounded device wait timed out");
  (void)NA;
}

} // namespace nedy
