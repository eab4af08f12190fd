// Shared device/host helpers of the B200 GF2 engine.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <stdexcept>
#include <atomic>

namespace nedy {

using i64 = long long;

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string &m) : std::runtime_error(m) {}
};
struct ArgError : std::runtime_error {
  explicit ArgError(const std::string &m) : std::runtime_error(m) {}
};

#define NEDY_CUDA(call)                                                                        \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess)                                                                     \
      throw ::nedy::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_) + " @ " +     \
                              __FILE__ + ":" + std::to_string(__LINE__));                      \
  } while (0)

// Every kernel launch of the engine is followed by NEDY_CHECK_LAUNCH, which also
// counts it (nedy_launch_count in the C ABI).
extern std::atomic<unsigned long long> g_launches;
#define NEDY_CHECK_LAUNCH()                                                                    \
  do {                                                                                         \
    ++::nedy::g_launches;                                                                      \
    NEDY_CUDA(cudaGetLastError());                                                             \
  } while (0)

#define NEDY_REQUIRE(cond, msg)                                                                \
  do {                                                                                         \
    if (!(cond)) throw ::nedy::ArgError(std::string(msg));                                     \
  } while (0)

#ifdef __CUDACC__
// Adds v to *dst, one atomic per warp when all 32 lanes are active and target the same address
// (the usual case of the per-block error norms, whose blocks are whole warps), one per lane
// otherwise.  Same-address atomics from every thread serialise in L2.
__device__ __forceinline__ void add_warp(double *dst, double v) {
  const unsigned mask = __activemask();
  if (mask == 0xffffffffu) {
    const unsigned long long a = (unsigned long long)dst;
    if (__all_sync(mask, a == __shfl_sync(mask, a, 0))) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
      if ((threadIdx.x & 31) == 0) atomicAdd(dst, v);
      return;
    }
  }
  atomicAdd(dst, v);
}
#endif

// complex helpers on double2 (x = re, y = im)
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 czero() { return make_double2(0.0, 0.0); }

// packed-triangle indices of the reference storage (greens.cpp:177-185)
__host__ __device__ __forceinline__ i64 les_idx(i64 i, i64 j) { return j * (j + 1) / 2 + i; }  // i <= j
__host__ __device__ __forceinline__ i64 ret_idx(i64 i, i64 j) { return i * (i + 1) / 2 + j; }  // j <= i

inline unsigned cdiv(i64 a, i64 b) { return (unsigned)((a + b - 1) / b); }

// Host -> device copy / memset ordered on the engine's stream and completed before
// returning (a pageable cudaMemcpy on the legacy stream may return before its DMA lands).
inline void h2d_sync(void *dst, const void *src, size_t bytes, cudaStream_t s) {
  NEDY_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
  NEDY_CUDA(cudaStreamSynchronize(s));
}
inline void memset_sync(void *dst, size_t bytes, cudaStream_t s) {
  NEDY_CUDA(cudaMemsetAsync(dst, 0, bytes, s));
  NEDY_CUDA(cudaStreamSynchronize(s));
}

} // namespace nedy
