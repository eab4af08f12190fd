// nedy_hf_decomp_noalloc: the restricted density-fitted Hartree-Fock update of
// nedy_hf_decomp with its intermediates in a static device array, so the call
// itself never allocates device memory.  Callers that cannot allocate once their
// simulation runs (their pool allocator already holds the free memory, or a
// cudaMalloc/cudaFree would synchronise a device they keep busy) use this one.
#include "handles.cuh"
#include "sigma.cuh"
#include <mutex>
#include <string>
#include <vector>

using namespace nedy;

namespace {

constexpr long long kScratchBytes = NEDY_NOALLOC_SCRATCH_BYTES;

// Scratch shared by every call on a device; it keeps the last call's contents.
// In host code `hf_scratch` is only the host-side stand-in that names the
// symbol: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char hf_scratch[kScratchBytes];

std::mutex g_scratch_mu;
std::vector<void *> g_scratch_addr;  // per device, filled by the first call there

// Set-up, once per device, with that device current.
void *scratch_for_current_device() {
  int dev = -1;
  NEDY_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if ((int)g_scratch_addr.size() <= dev) g_scratch_addr.resize(dev + 1, nullptr);
  if (!g_scratch_addr[dev]) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, hf_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw CudaError(std::string("nedy_hf_decomp_noalloc: cudaGetSymbolAddress of the static scratch failed: ") +
                      cudaGetErrorString(e));
    }
    g_scratch_addr[dev] = ptr;
  }
  return g_scratch_addr[dev];
}

}  // namespace

extern "C" int nedy_hf_decomp_noalloc(nedy_ctx *ctx, int tstp, nedy_buf *hmf, const nedy_buf *rho) {
  return run_guarded([&] {
    NEDY_REQUIRE(ctx && hmf && rho, "null argument");
    Ctx &c = ctx->c;
    NEDY_REQUIRE(c.Vija, "nedy_hf_decomp_noalloc: density-fitted tensor not set");
    NEDY_CUDA(cudaSetDevice(c.device));
    const int N = c.df_nao, A = c.df_naux;
    const i64 es = (i64)N * N;
    NEDY_REQUIRE(tstp >= 0 && hmf->bytes >= (i64)(tstp + 1) * es * 16, "hmf buffer too small for tstp");
    NEDY_REQUIRE(rho->bytes >= es * 16, "rho buffer too small");
    // scratch: Xa (A complex, padded to 256 bytes), then T1 (N*A x N complex)
    const i64 xa_bytes = (((i64)A * 16 + 255) / 256) * 256;
    const i64 need = xa_bytes + es * A * 16;
    if (need > kScratchBytes)
      throw ArgError("nedy_hf_decomp_noalloc: nao=" + std::to_string(N) + ", naux=" + std::to_string(A) + " needs " +
                     std::to_string(need) + " bytes of scratch, more than the static " +
                     std::to_string(kScratchBytes) + " bytes (use nedy_hf_decomp)");
    char *base = (char *)scratch_for_current_device();
    double2 *Xa = (double2 *)base;
    double2 *T1 = (double2 *)(base + xa_bytes);
    double2 *h = (double2 *)hmf->p + (i64)tstp * es;
    const double2 *r = (const double2 *)rho->p;
    // The array holds the previous call's values.  Nothing below reads them: Xa and T1 are
    // written by GEMMs with beta = 0, which never read C (a K-split launch first stores
    // exact zeros and then accumulates), so no clearing is needed.
    {  // Xa = rho_flat (1 x N^2) * Vija (N^2 x A)
      GemmArgs g;
      g.M = 1; g.N = A; g.K = (int)es;
      g.A = rowmajor(r, es);
      g.B = rowmajor(c.Vija, A); g.b_cplx = false;
      g.C = rowmajor(Xa, A);
      gemm(g, c.stream);
    }
    {  // Hartree: h_flat += 2 Vija (N^2 x A) * Xa
      GemmArgs g;
      g.M = (int)es; g.N = 1; g.K = A;
      g.A = rowmajor(c.Vija, A); g.a_cplx = false;
      g.B = rowmajor(Xa, 1);
      g.C = rowmajor(h, 1);
      g.alpha = make_double2(2.0, 0.0);
      g.beta = make_double2(1.0, 0.0);
      gemm(g, c.stream);
    }
    {  // T1[(i,a)][k] = sum_l Viaj[(i,a)][l] rho[k][l]
      GemmArgs g;
      g.M = N * A; g.N = N; g.K = N;
      g.A = rowmajor(c.Viaj, N); g.a_cplx = false;
      g.B = transposed(r, N);
      g.C = rowmajor(T1, N);
      gemm(g, c.stream);
    }
    {  // exchange: h -= T1 (N x (a,k)) * Vaij ((a,k) x j)
      GemmArgs g;
      g.M = N; g.N = N; g.K = N * A;
      g.A = rowmajor(T1, (i64)N * A);
      g.B = rowmajor(c.Vaij, N); g.b_cplx = false;
      g.C = rowmajor(h, N);
      g.alpha = make_double2(-1.0, 0.0);
      g.beta = make_double2(1.0, 0.0);
      gemm(g, c.stream);
    }
    NEDY_CUDA(cudaStreamSynchronize(c.stream));
  });
}
