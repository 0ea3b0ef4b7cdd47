// tp_common.cuh -- shared helpers for the P1-tet transport kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "dissolve_tp.h"

namespace tp {

// thread-local detail text behind TP_ERR_* codes (tp_capi.cu)
void set_error(const char* fmt, ...);

#define TP_CUDA_TRY(expr)                                                     \
  do {                                                                        \
    cudaError_t _e = (expr);                                                  \
    if (_e != cudaSuccess) {                                                  \
      ::tp::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), \
                      __FILE__, __LINE__);                                    \
      return TP_ERR_CUDA;                                                     \
    }                                                                         \
  } while (0)

#define TP_LAUNCH_CHECK()                                                        \
  do {                                                                           \
    cudaError_t _e = cudaGetLastError();                                         \
    if (_e != cudaSuccess) {                                                     \
      ::tp::set_error("kernel launch failed: %s (%s:%d)", cudaGetErrorString(_e), \
                      __FILE__, __LINE__);                                       \
      return TP_ERR_CUDA;                                                        \
    }                                                                            \
  } while (0)

#define TP_REQUIRE(cond, ...)       \
  do {                              \
    if (!(cond)) {                  \
      ::tp::set_error(__VA_ARGS__); \
      return TP_ERR_ARG;            \
    }                               \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline int grid_for(int64_t n, int block, int cap = 1 << 30) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

// number of SMs of the current device (cached per process; one device per process)
int sm_count();

// device flag bits written by validating kernels
enum : int32_t {
  FLAG_INDEX = 1,       // a vertex id outside [0, n_verts)
  FLAG_DEGENERATE = 2,  // det J == 0 or not finite
  FLAG_ROWCAP = 4,      // a row longer than the kernel capacity
  FLAG_BCINDEX = 8,     // a Dirichlet dof outside [0, n_verts)
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// deterministic block sum (fixed tree); every thread gets the total.  `sh` must
// hold blockDim.x/32 doubles; blockDim.x a multiple of 32, at most 1024.
__device__ __forceinline__ double block_sum(double v, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double t = (threadIdx.x < (unsigned)nw) ? sh[threadIdx.x] : 0.0;
  if (w == 0) t = warp_sum(t);
  if (threadIdx.x == 0) sh[0] = t;
  __syncthreads();
  t = sh[0];
  __syncthreads();
  return t;
}

// 32-byte read-only load as two 128-bit loads
// One 256-bit read-only load (sm_100): p must be 32-byte aligned (coords4 and geo rows;
// the entry points that read them check the base pointers).
__device__ __forceinline__ double4 ldg_d4(const double4* p) {
  double4 v;
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
      : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w)
      : "l"(p));
  return v;
}

// asynchronous global -> shared copy of NB bytes (4, 8 or 16; both addresses NB-aligned)
template <int NB>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (NB == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(sa), "l"(gmem), "n"(NB)
                 : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

template <typename T>
struct vec_of;
template <>
struct vec_of<float> {
  using t4 = float4;
};
template <>
struct vec_of<double> {
  using t4 = double4;
};

}  // namespace tp
