/*
 * cuda_cpu_shim.h -- lets a plain CUDA C kernel source compile as host C++ (test
 * infrastructure for oracle/ref_recipe.py).  A kernel becomes an ordinary function;
 * the launch wrapper sets blockIdx/threadIdx and calls it once per thread, in
 * order, so atomicAdd can be a plain read-add-write.
 */
#pragma once
#include <cmath>
#include <cstdint>

struct shim_dim3 {
  unsigned x, y, z;
};
static shim_dim3 blockIdx = {0, 0, 0};
static shim_dim3 threadIdx = {0, 0, 0};
static shim_dim3 blockDim = {1, 1, 1};
static shim_dim3 gridDim = {1, 1, 1};

#define __global__
#define __device__
#define __forceinline__ inline
#define __restrict__ __restrict

static inline double atomicAdd(double* p, double v) {
  double o = *p;
  *p = o + v;
  return o;
}
static inline float atomicAdd(float* p, float v) {
  float o = *p;
  *p = o + v;
  return o;
}
static inline int atomicAdd(int* p, int v) {
  int o = *p;
  *p = o + v;
  return o;
}
