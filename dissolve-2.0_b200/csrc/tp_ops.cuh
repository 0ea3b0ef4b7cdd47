// tp_ops.cuh -- device building blocks shared by the operator and Krylov kernels.
#pragma once
#include "tp_common.cuh"

namespace tp {

// load / store LD interleaved columns of row j
template <typename T, int LD>
__device__ __forceinline__ void ldv(const T* __restrict__ x, int64_t j, T v[LD]) {
  if constexpr (LD == 1) {
    v[0] = x[j];
  } else if constexpr (sizeof(T) * LD == 16) {
    const uint4 u = __ldg(reinterpret_cast<const uint4*>(x + j * LD));
    const T* t = reinterpret_cast<const T*>(&u);
#pragma unroll
    for (int s = 0; s < LD; s++) v[s] = t[s];
  } else if constexpr (sizeof(T) * LD == 8) {
    const uint2 u = __ldg(reinterpret_cast<const uint2*>(x + j * LD));
    const T* t = reinterpret_cast<const T*>(&u);
#pragma unroll
    for (int s = 0; s < LD; s++) v[s] = t[s];
  } else {  // 32 bytes: double x 4
    const uint4* p = reinterpret_cast<const uint4*>(x + j * LD);
    const uint4 a = __ldg(p), b = __ldg(p + 1);
    const T* ta = reinterpret_cast<const T*>(&a);
    const T* tb = reinterpret_cast<const T*>(&b);
    v[0] = ta[0];
    v[1] = ta[1];
    v[2] = tb[0];
    v[3] = tb[1];
  }
}

// plain (coherent) load for vectors written earlier in the same kernel sequence
template <typename T, int LD>
__device__ __forceinline__ void ldv_cg(const T* x, int64_t j, T v[LD]) {
  if constexpr (LD == 1) {
    v[0] = x[j];
  } else if constexpr (sizeof(T) * LD == 16) {
    const uint4 u = *reinterpret_cast<const uint4*>(x + j * LD);
    const T* t = reinterpret_cast<const T*>(&u);
#pragma unroll
    for (int s = 0; s < LD; s++) v[s] = t[s];
  } else if constexpr (sizeof(T) * LD == 8) {
    const uint2 u = *reinterpret_cast<const uint2*>(x + j * LD);
    const T* t = reinterpret_cast<const T*>(&u);
#pragma unroll
    for (int s = 0; s < LD; s++) v[s] = t[s];
  } else {
    const uint4* p = reinterpret_cast<const uint4*>(x + j * LD);
    const uint4 a = p[0], b = p[1];
    const T* ta = reinterpret_cast<const T*>(&a);
    const T* tb = reinterpret_cast<const T*>(&b);
    v[0] = ta[0];
    v[1] = ta[1];
    v[2] = tb[0];
    v[3] = tb[1];
  }
}

template <typename T, int LD>
__device__ __forceinline__ void stv(T* x, int64_t j, const T v[LD]) {
  if constexpr (LD == 1) {
    x[j] = v[0];
  } else if constexpr (sizeof(T) * LD == 16) {
    uint4 u;
    T* t = reinterpret_cast<T*>(&u);
#pragma unroll
    for (int s = 0; s < LD; s++) t[s] = v[s];
    *reinterpret_cast<uint4*>(x + j * LD) = u;
  } else if constexpr (sizeof(T) * LD == 8) {
    uint2 u;
    T* t = reinterpret_cast<T*>(&u);
#pragma unroll
    for (int s = 0; s < LD; s++) t[s] = v[s];
    *reinterpret_cast<uint2*>(x + j * LD) = u;
  } else {
    uint4 a, b;
    T* ta = reinterpret_cast<T*>(&a);
    T* tb = reinterpret_cast<T*>(&b);
    ta[0] = v[0];
    ta[1] = v[1];
    tb[0] = v[2];
    tb[1] = v[3];
    uint4* p = reinterpret_cast<uint4*>(x + j * LD);
    p[0] = a;
    p[1] = b;
  }
}

// Multi-column CSR operator description as the kernels see it.
template <typename T>
struct CsrView {
  const int32_t* indptr;
  const int32_t* indices;
  const T* K;
  const T* M;     // nullable
  const T* diag;  // nullable, (n, ld)
  const uint8_t* bc;
  double dscale[4];
  double cscale[4];
};

// y_row = dscale (K x)_row + cscale (M x)_row + diag_row x_row, computed by the G lanes
// of a row group; the result is valid in every lane of the group.  Rows flagged in bc
// are identity rows.  Every lane of the warp must call this (the group reduction
// shuffles across the full warp): callers clamp out-of-range rows and drop the result.
// `x` goes through the read-only path when RO is true (x not written by this kernel).
template <typename T, int LD, int G, bool RO>
__device__ __forceinline__ void csr_row(const CsrView<T>& A, int64_t row, int gl, const T* x,
                                        T y[LD]) {
  T ak[LD], am[LD];
#pragma unroll
  for (int s = 0; s < LD; s++) ak[s] = am[s] = T(0);
  const bool is_bc = A.bc && A.bc[row];
  const int beg = A.indptr[row];
  const int end = is_bc ? beg : A.indptr[row + 1];
  for (int p = beg + gl; p < end; p += G) {
    const int j = __ldg(A.indices + p);
    const T kv = __ldg(A.K + p);
    T xv[LD];
    if (RO)
      ldv<T, LD>(x, j, xv);
    else
      ldv_cg<T, LD>(x, j, xv);
#pragma unroll
    for (int s = 0; s < LD; s++) ak[s] += kv * xv[s];
    if (A.M) {
      const T mv = __ldg(A.M + p);
#pragma unroll
      for (int s = 0; s < LD; s++) am[s] += mv * xv[s];
    }
  }
  if (G > 1) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
#pragma unroll
      for (int s = 0; s < LD; s++) {
        ak[s] += __shfl_xor_sync(0xffffffffu, ak[s], o, G);
        if (A.M) am[s] += __shfl_xor_sync(0xffffffffu, am[s], o, G);
      }
    }
  }
  T xr[LD], dr[LD];
#pragma unroll
  for (int s = 0; s < LD; s++) xr[s] = dr[s] = T(0);
  if (A.diag || is_bc) {
    if (RO)
      ldv<T, LD>(x, row, xr);
    else
      ldv_cg<T, LD>(x, row, xr);
  }
  if (A.diag && !is_bc) ldv<T, LD>(A.diag, row, dr);
#pragma unroll
  for (int s = 0; s < LD; s++) {
    T v = T(A.dscale[s]) * ak[s];
    if (A.M) v += T(A.cscale[s]) * am[s];
    v += dr[s] * xr[s];
    y[s] = is_bc ? xr[s] : v;
  }
}

}  // namespace tp
