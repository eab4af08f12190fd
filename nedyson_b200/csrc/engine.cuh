// Device-side objects of the B200 GF2 engine: Green's functions in the
// reference's packed layout, the workspace arena and the engine context.
#pragma once
#include "common.cuh"
#include "gemm_f64.cuh"
#include <vector>
#include <memory>

namespace nedy {

// Contour Green's function resident in HBM, same packing as the reference
// (greens.cpp:34-195): les column T, ret row T and tv row T are contiguous.
// win > 0 (windowed): the retarded rows and lesser columns live in a ring of win slots of
// nt + 1 blocks (row / column t in slot t mod win), i.e. only the last win time steps of the
// two triangles are on the device.  That is all a time step of G reads (its own row, the
// k + 1 rows of the extrapolation, the history of the learned predictor, the diagonal of the
// lesser step); Sigma keeps its full triangles (win = 0), which the Dyson integrals read.
struct DevGF {
  int nt = 0, ntau = 0, nao = 0, sig = -1;
  int win = 0;
  i64 es = 0;
  double2 *les = nullptr, *ret = nullptr, *tv = nullptr, *mat = nullptr;
  unsigned long long mat_version = 0;  // bumped whenever G^M is written
  i64 ntri() const { return (i64)(nt + 1) * (nt + 2) / 2; }
  // blocks held per triangle on the device
  i64 nstore() const { return win ? (i64)win * (nt + 1) : ntri(); }
  __host__ __device__ double2 *lesptr(i64 i, i64 j) const {
    return les + (win ? (j % win) * (i64)(nt + 1) + i : les_idx(i, j)) * es;
  }
  __host__ __device__ double2 *retptr(i64 i, i64 j) const {
    return ret + (win ? (i % win) * (i64)(nt + 1) + j : ret_idx(i, j)) * es;
  }
  __host__ __device__ double2 *tvptr(i64 i, i64 m) const { return tv + (i * (ntau + 1) + m) * es; }
  __host__ __device__ double2 *matptr(i64 m) const { return mat + m * es; }
};

// Bump allocator for per-call workspace.  A request that does not fit opens a
// further device block (live pointers stay valid); at the next reset() the blocks
// are merged into one of 1.5 x the combined size, so steady-state calls allocate
// nothing and a workspace that grows with the time step is rarely reallocated.
// Blocks are allocated and freed in the order of the context's stream
// (cudaMallocAsync / cudaFreeAsync): no device-wide synchronisation, so a context
// that grows its workspace does not stall the streams of other contexts.
class Arena {
 public:
  ~Arena();
  void set_stream(cudaStream_t s) { stream_ = s; }
  void reset();
  void *get(size_t bytes);
  template <class T> T *alloc(i64 n) { return (T *)get(sizeof(T) * (size_t)n); }
  size_t capacity() const;

 private:
  struct Block { char *p; size_t cap, top; };
  std::vector<Block> blocks_;
  cudaStream_t stream_ = nullptr;
  char *alloc_block(size_t bytes);
};

// Calculus weights (host tables) -- the restatement of Integration::Integrator
// lives in weights.cpp.
struct Weights {
  int k = 0;
  std::vector<double> poly_interp, poly_diff, poly_integ, bd, start, Omega, ex;
  double gregory(int n, int j) const;
  double omega(int j) const { return Omega[(size_t)k * (k + 1) + j]; }
  double pdiff(int m, int l) const { return poly_diff[(size_t)m * (k + 1) + l]; }
  double pinterp(int a, int l) const { return poly_interp[(size_t)a * (k + 1) + l]; }
};
Weights make_weights(int k);

// Legendre-Gauss-Lobatto collocation on [0, beta] (collocation.cpp).
struct Colloc {
  int ntau = 0;
  std::vector<double> x, w, u;  // nodes, weights, top-mode coefficients
  double ctop = 0;
  std::vector<double> EA, EB;  // per node m: evaluation matrices of the mixing quadrature
  int Q = 0;
};
Colloc make_colloc(int ntau);
void build_mixing_eval(Colloc &c);

class Predictor;

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int nt = 0, ntau = 0, nao = 0, k = 5;
  double beta = 1.0, dt = 0.01;
  Arena ws;
  i64 ws_budget = 8LL << 30;  // bytes the self-energy may use for chunk intermediates
  std::vector<std::pair<int *, int>> pending_status;  // device status words of batched solves
  // Gregory weights w(n, j) for n, j <= nt (row-major and transposed), small tables
  double *greg = nullptr, *gregT = nullptr;
  int greg_n = -1;
  double *small = nullptr, *d_pdiff = nullptr, *d_bd = nullptr, *d_ex = nullptr, *d_w = nullptr, *d_u = nullptr;
  Weights W;
  Colloc col;
  // density-fitted interaction, several layouts (real, row-major)
  int df_nao = 0, df_naux = 0;
  bool V_sym = false;  // every B^Q real symmetric: retarded row from Sigma^> and the lesser row
  double *Vija = nullptr;  // [i][j][a]
  double *Viaj = nullptr;  // [i][a][j]
  double *Vaij = nullptr;  // [a][i][j]
  double *Vmbq = nullptr;  // [m][b][q] = V^b_qm
  // self-energy arithmetic: NEDY_PREC_FP64 or a split-precision mode; BF16 pieces of
  // Vija ([piece][(i,j)][a], K padded to 64) for the split exchange, built on first use
  int precision = 0;
  void *Vp = nullptr;
  int Vp_np = 0;
  // further BF16-piece layouts of the interaction for the all-split les-form chain:
  // [(a,n)][j] = V^a_nj, [(j,k)][b] = V^b_kj, [i][(l,a)] = V^a_il
  void *Vanj_p = nullptr, *Vjkb_p = nullptr, *Vila_p = nullptr;
  // full U (N^4 real) and the exchange combination Uexch
  int u_nao = 0;
  double *U = nullptr, *Uexch = nullptr;
  // mixing kernel K[m][i] (nao x nao) of the current G^M, keyed by (G^M pointer, version)
  double2 *mixK = nullptr;
  const double2 *mixK_src = nullptr;
  unsigned long long mixK_ver = ~0ULL;
  int mixK_nao = 0;
  // a second cached kernel (the other spin's G^M in unrestricted runs)
  double2 *mixK_alt = nullptr;
  const double2 *mixK_alt_src = nullptr;
  unsigned long long mixK_alt_ver = ~0ULL;
  int mixK_alt_nao = 0;
  // inverses of the time-local Dyson matrices M(t') = (i bd0/dt + mu) - hmf(t') - dt w0 Sig^R(t',t')
  // residual exit of the whole-step entry: copy of the new row before an iteration, the
  // measured contraction of the corrector (ratio of successive changes, with a safety
  // factor) and the steps since it was last measured
  double2 *rowcopy = nullptr;
  i64 rowcopy_cap = 0;
  unsigned long long *d_maxdiff = nullptr;
  double contraction = 1.0;
  int steps_since_measure = 0;
  // learned predictor used by the residual-exit step (not owned); its corrections of the
  // current row, and how it fared against the polynomial prediction after iteration 1
  Predictor *pred = nullptr;
  bool pred_active = false;
  double2 *pred_corr = nullptr;
  i64 pred_corr_cap = 0;
  long long pred_judged = 0, pred_better = 0;
  unsigned pred_window = 0;  // outcomes of the last judged steps, one bit each (1: learned won)
  double pred_last[2] = {0, 0};
  double2 *Minv = nullptr;
  int Minv_cap = 0, Minv_nao = 0;
  // device time per phase of the whole-step entry points (ms): predictor, mean field, self-energy, Dyson
  bool timing = false;
  double phase_ms[4] = {0, 0, 0, 0};
  // second context (own stream, workspace, inverses, mixing kernel; owned) on which the
  // unrestricted whole steps run the second spin's Dyson step beside the first's
  Ctx *aux = nullptr;
  ~Ctx();
};

} // namespace nedy
