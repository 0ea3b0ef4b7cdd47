// tp_mlp.cu -- per-vertex MLP that predicts the next backward-Euler state (the Krylov
// initial guess), BF16 on the tensor cores with FP32 accumulation.
//
// Network: 16 inputs (10 used) -> 64 -> ReLU -> 64 -> ReLU -> 1, one network shared by
// all species; a row is one (vertex, species) pair.  Features (normalised by per-input
// affine maps fixed at training time):
//   0 phi, 1 |grad phi|, 2 u^n, 3 u^{n-1}, 4 u^n - u^{n-1}, 5 log D_s, 6 k_s, 7 1,
//   8 (D_s K u^n)_v, 9 (D_s K (u^n - u^{n-1}))_v -- the stiffness images give the
//   network the local curvature that decides how fast each part of the change decays
// The output y predicts (u^{n+1} - B) / sigma and the guess is B + sigma y, with the base
// B = u^n or the linear extrapolation 2 u^n - u^{n-1} (the network learns the correction
// to the extrapolation: with zero output the guess is the extrapolation itself).
//
// Inference (k_mlp_predict) runs layers 1 and 2 as tcgen05.mma on 128-row tiles with the
// accumulators in tensor memory.  Training uses mma.sync.m16n8k16 fragments (row.col,
// bf16 x bf16 -> f32): a warp owns 16 rows; layer outputs stay in registers and are
// re-packed from the accumulator layout into the next layer's A layout.  Backward: the
// weight gradients
// are GEMMs over the row dimension (dW2 = dZ2^T H1, dW1 = dZ1^T X) fed from transposed
// tiles staged in shared memory; every CTA writes its partial gradient, and the AdamW
// kernel sums the partials in CTA order (training is deterministic for a given grid).
#include <cuda_bf16.h>

#include <algorithm>

#include <atomic>

#include "tp_common.cuh"

namespace tp {

constexpr int MLP_IN = 16, MLP_H = 64;
// shared-memory row strides (bf16 elements) of the weight and staging tiles: 24 and 72
// put the 8 rows a B-fragment load touches into 8 different bank groups (16 and 64
// would hit the same banks 2 and 8 times)
constexpr int W1S = 24, W2S = 72, GS = 72;
// FP32 master parameter vector layout
constexpr int OFF_W1 = 0;                      // [64][16]
constexpr int OFF_B1 = OFF_W1 + MLP_H * MLP_IN;  // [64]
constexpr int OFF_W2 = OFF_B1 + MLP_H;           // [64][64]
constexpr int OFF_B2 = OFF_W2 + MLP_H * MLP_H;   // [64]
constexpr int OFF_W3 = OFF_B2 + MLP_H;           // [64]
constexpr int OFF_B3 = OFF_W3 + MLP_H;           // [1]
constexpr int MLP_P = OFF_B3 + 1;

constexpr int NFEAT = 10;  // used inputs: 0..6 fields, 7 bias, 8..9 operator images

struct MlpFeat {
  const double* U;      // (V, ld) u^n
  const double* Up;     // (V, ld) u^{n-1}
  const double* phi;    // (V) or NULL
  const double* ngphi;  // (V) or NULL
  const double* opU;    // (V, ld) D_s K u^n or NULL
  const double* opDU;   // (V, ld) D_s K (u^n - u^{n-1}) or NULL
  int S, ld;
  int base;  // the guess the output corrects: 0 u^n, 1 2 u^n - u^{n-1}, 2 none
  float logD[4], k[4];
  float mean[NFEAT], istd[NFEAT];
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16(float c[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// the fields row r = v * S + s reads (r < number of rows)
struct RowFields {
  double u, up, phi, ngphi, opu, opdu;
};

__device__ __forceinline__ RowFields row_fields(const MlpFeat& F, int64_t v, int s) {
  const int64_t i = v * F.ld + s;
  RowFields x;
  x.u = F.U[i];
  x.up = F.Up[i];
  x.phi = F.phi ? F.phi[v] : 0.0;
  x.ngphi = F.ngphi ? F.ngphi[v] : 0.0;
  x.opu = F.opU ? F.opU[i] : 0.0;
  x.opdu = F.opDU ? F.opDU[i] : 0.0;
  return x;
}

// all NFEAT normalised features of a row from its fields, branch-free
__device__ __forceinline__ void fields_features(const MlpFeat& F, const RowFields& r, int s,
                                                float f[NFEAT]) {
  float x[NFEAT];
  x[0] = (float)r.phi;
  x[1] = (float)r.ngphi;
  x[2] = (float)r.u;
  x[3] = (float)r.up;
  x[4] = (float)(r.u - r.up);
  x[5] = F.logD[s];
  x[6] = F.k[s];
  x[7] = 0.0f;
  x[8] = (float)r.opu;
  x[9] = (float)r.opdu;
#pragma unroll
  for (int k = 0; k < NFEAT; k++) f[k] = (k == 7) ? 1.0f : (x[k] - F.mean[k]) * F.istd[k];
}

__device__ __forceinline__ void row_features(const MlpFeat& F, int64_t v, int s,
                                             float f[NFEAT]) {
  fields_features(F, row_fields(F, v, s), s, f);
}

// shared-memory copy of the BF16 weights
struct MlpSmem {
  __nv_bfloat16 W1[MLP_H][W1S];
  __nv_bfloat16 W2[MLP_H][W2S];
  float w3[MLP_H];
  float b1[MLP_H], b2[MLP_H];
  float b3;
};

// W2T (optional, the backward pass): W2 transposed, [in][out]
__device__ void load_weights(MlpSmem& sm, const float* __restrict__ P,
                             __nv_bfloat16 (*W2T)[W2S] = nullptr) {
  for (int i = threadIdx.x; i < MLP_H * MLP_IN; i += blockDim.x)
    sm.W1[i / MLP_IN][i % MLP_IN] = __float2bfloat16_rn(P[OFF_W1 + i]);
  for (int i = threadIdx.x; i < MLP_H * MLP_H; i += blockDim.x) {
    const __nv_bfloat16 w = __float2bfloat16_rn(P[OFF_W2 + i]);
    sm.W2[i / MLP_H][i % MLP_H] = w;
    if (W2T) W2T[i % MLP_H][i / MLP_H] = w;
  }
  for (int i = threadIdx.x; i < MLP_H; i += blockDim.x) {
    sm.w3[i] = __bfloat162float(__float2bfloat16_rn(P[OFF_W3 + i]));
    sm.b1[i] = P[OFF_B1 + i];
    sm.b2[i] = P[OFF_B2 + i];
  }
  if (threadIdx.x == 0) sm.b3 = P[OFF_B3];
  __syncthreads();
}

// B fragment of W^T for W stored [n][k] row-major with row length ldk
__device__ __forceinline__ void bfrag(const __nv_bfloat16* W, int ldk, int n0, int k0, int g,
                                      int t, uint32_t& b0, uint32_t& b1) {
  const __nv_bfloat16* row = W + (n0 + g) * ldk + k0 + 2 * t;
  b0 = *reinterpret_cast<const uint32_t*>(row);
  b1 = *reinterpret_cast<const uint32_t*>(row + 8);
}

// Forward pass of one 16-row tile.  xa: the A fragment of the inputs (K = 16).
// On return z1/z2 hold the pre-activations (8 n-tiles x 4), y the output of rows g, g+8
// (valid in every lane of the quad).
__device__ __forceinline__ void mlp_tile_forward(const MlpSmem& sm, const uint32_t xa[4], int g,
                                                 int t, float z1[8][4], float z2[8][4],
                                                 float& y0, float& y1) {
#pragma unroll
  for (int n = 0; n < 8; n++) {
    const float bl = sm.b1[n * 8 + 2 * t], bh = sm.b1[n * 8 + 2 * t + 1];
    z1[n][0] = bl;
    z1[n][1] = bh;
    z1[n][2] = bl;
    z1[n][3] = bh;
    uint32_t b0, b1;
    bfrag(&sm.W1[0][0], W1S, n * 8, 0, g, t, b0, b1);
    mma_bf16(z1[n], xa[0], xa[1], xa[2], xa[3], b0, b1);
  }
  uint32_t ha[4][4];  // h1 as A fragments, 4 k-steps
#pragma unroll
  for (int kk = 0; kk < 4; kk++) {
    const float* lo = z1[2 * kk];
    const float* hi = z1[2 * kk + 1];
    ha[kk][0] = pack_bf16(fmaxf(lo[0], 0.f), fmaxf(lo[1], 0.f));
    ha[kk][1] = pack_bf16(fmaxf(lo[2], 0.f), fmaxf(lo[3], 0.f));
    ha[kk][2] = pack_bf16(fmaxf(hi[0], 0.f), fmaxf(hi[1], 0.f));
    ha[kk][3] = pack_bf16(fmaxf(hi[2], 0.f), fmaxf(hi[3], 0.f));
  }
#pragma unroll
  for (int n = 0; n < 8; n++) {
    const float bl = sm.b2[n * 8 + 2 * t], bh = sm.b2[n * 8 + 2 * t + 1];
    z2[n][0] = bl;
    z2[n][1] = bh;
    z2[n][2] = bl;
    z2[n][3] = bh;
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
      uint32_t b0, b1;
      bfrag(&sm.W2[0][0], W2S, n * 8, kk * 16, g, t, b0, b1);
      mma_bf16(z2[n], ha[kk][0], ha[kk][1], ha[kk][2], ha[kk][3], b0, b1);
    }
  }
  // layer 3 (64 -> 1) on the CUDA cores: BF16-rounded h2 . w3, reduced over the quad
  float s0 = 0.f, s1 = 0.f;
#pragma unroll
  for (int n = 0; n < 8; n++) {
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const float w = sm.w3[n * 8 + 2 * t + e];
      s0 += __bfloat162float(__float2bfloat16_rn(fmaxf(z2[n][e], 0.f))) * w;
      s1 += __bfloat162float(__float2bfloat16_rn(fmaxf(z2[n][2 + e], 0.f))) * w;
    }
  }
  s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
  s0 += __shfl_xor_sync(0xffffffffu, s0, 2);
  s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
  s1 += __shfl_xor_sync(0xffffffffu, s1, 2);
  y0 = s0 + sm.b3;
  y1 = s1 + sm.b3;
}

// ----------------------------------------------------------------- inference
// 5th-generation tensor cores: 128-row tiles, one row per thread of a 128-thread CTA.
// Layer 1 (128 x 64, K = 16) and layer 2 (128 x 64, K = 64 as four K = 16 steps) are
// tcgen05.mma from shared-memory operands into tensor memory (z1 in columns 0..63, z2 in
// columns 64..127 of a 128-column allocation), issued by one thread and completed through
// an mbarrier (tcgen05.commit); every thread reads its own row back with tcgen05.ld (warp w
// owns TMEM lanes 32w..32w+31).  Operands are K-major without swizzle: 8-row x 16-byte
// core matrices, the two 8-element K halves 128 bytes apart, 8-row groups 256 bytes apart.
// Every mbarrier wait is bounded; a wait that runs out sets the call's status word and
// g_mlp_tc_timeout, ends the CTA's tiles and still releases its tensor memory.
constexpr int TC_M = 128, TC_COLS = 128;
constexpr uint32_t TC_WAIT_LIMIT = 1u << 24;  // default polls of one mbarrier phase (~0.1 s)

__device__ int g_mlp_tc_timeout;

// wait bound and failure-path test switch of the next launches (tp_mlp_set_wait_limit)
struct TcWait {
  uint32_t polls;
  int skip_issue;
  int32_t* status;
};

struct TcSmem {
  __nv_bfloat16 A1[TC_M * 16];     // features of the tile, 4 KB
  __nv_bfloat16 A2[4][TC_M * 16];  // h1 of the tile, one 4 KB block per K step
  __nv_bfloat16 W1[MLP_H * 16];    // 2 KB
  __nv_bfloat16 W2[4][MLP_H * 16]; // 8 KB
  float b1[MLP_H], b2[MLP_H], w3[MLP_H];
  float b3;
  uint64_t bar;
  uint32_t taddr;
};

// element offset of (row, k) in a K-major no-swizzle block of 16 K columns
__device__ __forceinline__ int tc_off(int row, int k) {
  return (row >> 3) * 128 + (k >> 3) * 64 + (row & 7) * 8 + (k & 7);
}

__device__ __forceinline__ uint64_t tc_desc(const void* smem) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(smem);
  uint64_t d = (uint64_t)((a >> 4) & 0x3FFFu);  // start address
  d |= (uint64_t)(128 >> 4) << 16;              // leading byte offset: the K halves
  d |= (uint64_t)(256 >> 4) << 32;              // stride byte offset: 8-row groups
  d |= (uint64_t)1 << 46;                       // descriptor version of sm_100
  return d;                                     // base offset 0, no swizzle
}

// kind::f16 instruction descriptor: F32 accumulate, BF16 A and B (K-major), N = 64, M = 128
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(MLP_H >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a, uint64_t b, int accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(TC_IDESC), "r"(accumulate));
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  const uint32_t ba = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(ba)
               : "memory");
}

// bounded wait for the given phase of the mbarrier; false when the limit ran out
__device__ __forceinline__ bool tc_wait(uint64_t* bar, uint32_t phase, uint32_t polls) {
  const uint32_t ba = (uint32_t)__cvta_generic_to_shared(bar);
  for (uint32_t it = 0; it < polls; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(ba), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tc_timed_out(const TcWait& tw) {
  atomicExch(&g_mlp_tc_timeout, 1);
  if (tw.status) atomicExch(tw.status, 1);
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void proxy_fence() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 64 consecutive FP32 columns of this thread's TMEM lane: four loads in flight, one wait
__device__ __forceinline__ void tc_ld64(uint32_t taddr, float v[64]) {
  uint32_t r[64];
#pragma unroll
  for (int j = 0; j < 4; j++)
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15}, [%16];"
        : "=r"(r[16 * j + 0]), "=r"(r[16 * j + 1]), "=r"(r[16 * j + 2]), "=r"(r[16 * j + 3]),
          "=r"(r[16 * j + 4]), "=r"(r[16 * j + 5]), "=r"(r[16 * j + 6]), "=r"(r[16 * j + 7]),
          "=r"(r[16 * j + 8]), "=r"(r[16 * j + 9]), "=r"(r[16 * j + 10]), "=r"(r[16 * j + 11]),
          "=r"(r[16 * j + 12]), "=r"(r[16 * j + 13]), "=r"(r[16 * j + 14]), "=r"(r[16 * j + 15])
        : "r"(taddr + 16u * (uint32_t)j));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 64; k++) v[k] = __uint_as_float(r[k]);
}

// x_out[v, s] = B[v, s] + sigma * y(v, s)  (or y_out[r] = y when x_out is NULL).
// Every thread gathers all features of its row (no divergent per-feature branches).
__global__ void __launch_bounds__(TC_M) k_mlp_predict(MlpFeat F, int64_t nrows,
                                                      const float* __restrict__ P, float sigma,
                                                      double* __restrict__ x_out,
                                                      float* __restrict__ y_out, TcWait tw) {
  __shared__ __align__(128) TcSmem sm;
  const int tid = threadIdx.x, warp = tid >> 5;
  // weights in the operand layout (BF16), biases and w3 (w3 rounded to BF16 as in training)
  for (int i = tid; i < MLP_H * 16; i += blockDim.x) {
    const int n = i >> 4, k = i & 15;
    sm.W1[tc_off(n, k)] = __float2bfloat16_rn(P[OFF_W1 + i]);
  }
  for (int i = tid; i < MLP_H * MLP_H; i += blockDim.x) {
    const int n = i >> 6, k = i & 63;
    sm.W2[k >> 4][tc_off(n, k & 15)] = __float2bfloat16_rn(P[OFF_W2 + i]);
  }
  for (int i = tid; i < MLP_H; i += blockDim.x) {
    sm.b1[i] = P[OFF_B1 + i];
    sm.b2[i] = P[OFF_B2 + i];
    sm.w3[i] = __bfloat162float(__float2bfloat16_rn(P[OFF_W3 + i]));
  }
  if (tid == 0) sm.b3 = P[OFF_B3];
  if (warp == 0) {
    const uint32_t slot = (uint32_t)__cvta_generic_to_shared(&sm.taddr);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
                 "r"(TC_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    const uint32_t ba = (uint32_t)__cvta_generic_to_shared(&sm.bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(ba), "r"(1));
  }
  proxy_fence();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t taddr = sm.taddr;
  const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
  uint32_t phase = 0;
  const int64_t ntiles = (nrows + TC_M - 1) / TC_M;
  // (vertex, species) of this thread's row of a tile (vertex 0 past the last row)
  auto row_of = [&](int64_t tile, int64_t& v, int& s) {
    const int64_t r = tile * TC_M + tid;
    // 32-bit division while the row index fits
    v = r >= nrows ? 0
                   : (r < (int64_t)UINT32_MAX ? (int64_t)((uint32_t)r / (uint32_t)F.S) : r / F.S);
    s = r >= nrows ? 0 : (int)(r - v * F.S);
  };
  // the fields of the CTA's first tile; every tile's MMAs overlap the next tile's loads
  RowFields cur{};
  if (blockIdx.x < ntiles) {
    int64_t v0;
    int s0;
    row_of(blockIdx.x, v0, s0);
    cur = row_fields(F, v0, s0);
  }
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t r = tile * TC_M + tid;
    const bool in = r < nrows;
    int64_t v;
    int s;
    row_of(tile, v, s);
    {
      float f[NFEAT];
      fields_features(F, cur, s, f);
      uint32_t w[8];
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const float lo = (in && 2 * k < NFEAT) ? f[2 * k] : 0.f;
        const float hi = (in && 2 * k + 1 < NFEAT) ? f[2 * k + 1] : 0.f;
        w[k] = pack_bf16(lo, hi);
      }
      *reinterpret_cast<uint4*>(&sm.A1[tc_off(tid, 0)]) = make_uint4(w[0], w[1], w[2], w[3]);
      *reinterpret_cast<uint4*>(&sm.A1[tc_off(tid, 8)]) = make_uint4(w[4], w[5], w[6], w[7]);
    }
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0 && !tw.skip_issue) {
      tc_mma(taddr, tc_desc(sm.A1), tc_desc(sm.W1), 0);
      tc_commit(&sm.bar);
    }
    RowFields nxt{};
    if (tile + gridDim.x < ntiles) {
      int64_t vn;
      int sn;
      row_of(tile + gridDim.x, vn, sn);
      nxt = row_fields(F, vn, sn);
    }
    bool ok = tc_wait(&sm.bar, phase, tw.polls);
    phase ^= 1u;
    tc_fence_after();
    // h1 = relu(z1 + b1), BF16, into the layer-2 operand
    float z1[64];
    tc_ld64(taddr + lane_base, z1);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const float* z = z1 + 16 * j;
      uint32_t w[8];
#pragma unroll
      for (int k = 0; k < 8; k++)
        w[k] = pack_bf16(fmaxf(z[2 * k] + sm.b1[16 * j + 2 * k], 0.f),
                         fmaxf(z[2 * k + 1] + sm.b1[16 * j + 2 * k + 1], 0.f));
      *reinterpret_cast<uint4*>(&sm.A2[j][tc_off(tid, 0)]) = make_uint4(w[0], w[1], w[2], w[3]);
      *reinterpret_cast<uint4*>(&sm.A2[j][tc_off(tid, 8)]) = make_uint4(w[4], w[5], w[6], w[7]);
    }
    proxy_fence();
    tc_fence_before();
    if (__syncthreads_or(!ok)) {
      if (tid == 0) tc_timed_out(tw);
      break;
    }
    tc_fence_after();
    if (tid == 0 && !tw.skip_issue) {
#pragma unroll
      for (int j = 0; j < 4; j++) tc_mma(taddr + MLP_H, tc_desc(sm.A2[j]), tc_desc(sm.W2[j]), j > 0);
      tc_commit(&sm.bar);
    }
    ok = tc_wait(&sm.bar, phase, tw.polls);
    phase ^= 1u;
    tc_fence_after();
    // layer 3 on the CUDA cores: BF16-rounded h2 . w3 + b3
    float y = 0.f;
    {
      float z2[64];
      tc_ld64(taddr + lane_base + MLP_H, z2);
#pragma unroll
      for (int k = 0; k < 64; k++)
        y += __bfloat162float(__float2bfloat16_rn(fmaxf(z2[k] + sm.b2[k], 0.f))) * sm.w3[k];
    }
    y += sm.b3;
    if (in && ok) {
      if (x_out) {
        const int64_t i = v * F.ld + s;
        const double b = F.base == 1 ? 2.0 * cur.u - cur.up : (F.base == 0 ? cur.u : 0.0);
        x_out[i] = b + (double)sigma * (double)y;
      } else {
        y_out[r] = y;
      }
    }
    // the tile's tensor-memory reads and operand reads are done before the next tile
    tc_fence_before();
    if (__syncthreads_or(!ok)) {
      if (tid == 0) tc_timed_out(tw);
      break;
    }
    cur = nxt;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr),
                 "r"(TC_COLS));
}

// features of every row, materialised (training set), BF16 (nrows, 16): one thread per
// row, one 32-byte store
__global__ void k_mlp_features(MlpFeat F, int64_t nrows, __nv_bfloat16* __restrict__ X) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nrows;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = r / F.S;
    const int s = (int)(r - v * F.S);
    float f[NFEAT];
    row_features(F, v, s, f);
    uint32_t w[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const float lo = (2 * k < NFEAT) ? f[2 * k] : 0.f;
      const float hi = (2 * k + 1 < NFEAT) ? f[2 * k + 1] : 0.f;
      w[k] = pack_bf16(lo, hi);
    }
    uint4* dst = reinterpret_cast<uint4*>(X + r * MLP_IN);
    dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
    dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
  }
}

// training target (u^{n+1} - u^n) / sigma per row
__global__ void k_mlp_target(int64_t nrows, int S, int ld, const double* __restrict__ Un,
                             const double* __restrict__ Uprev,
                             const double* __restrict__ Unext, float inv_sigma,
                             float* __restrict__ T) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nrows;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = r / S;
    const int s = (int)(r - v * S);
    const int64_t i = v * ld + s;
    const double b = Uprev ? 2.0 * Un[i] - Uprev[i] : Un[i];
    T[r] = (float)((Unext[i] - b) * inv_sigma);
  }
}

// ----------------------------------------------------------------- training
struct GradSmem {
  __nv_bfloat16 dz2T[MLP_H][GS];  // [out unit][chunk row]
  __nv_bfloat16 h1T[MLP_H][GS];   // [hidden unit][chunk row]
  __nv_bfloat16 dz1T[MLP_H][GS];
  __nv_bfloat16 xT[MLP_IN][GS];
  __nv_bfloat16 W2T[MLP_H][W2S];  // W2 transposed: B operand of dH1 = dZ2 W2
  float dw3[4][MLP_H];  // per warp
  float db3[4];
  float loss[4];
};

// One CTA = 4 warps = 64-row chunks.  Partial gradients (MLP_P floats) and the loss
// partial (sum of squared errors) per CTA.  wscale = 2 / (rows in the batch).
__global__ void __launch_bounds__(128) k_mlp_grad(const __nv_bfloat16* __restrict__ X,
                                                  const float* __restrict__ T, int64_t row0,
                                                  int64_t nrows, const float* __restrict__ P,
                                                  float wscale, float* __restrict__ part,
                                                  float* __restrict__ loss_part) {
  __shared__ MlpSmem sm;
  extern __shared__ __align__(16) unsigned char grad_dyn[];  // GradSmem (> 48 KB static)
  GradSmem& gs = *reinterpret_cast<GradSmem*>(grad_dyn);
  load_weights(sm, P, gs.W2T);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  for (int i = threadIdx.x; i < 4 * MLP_H; i += blockDim.x) gs.dw3[i / MLP_H][i % MLP_H] = 0.f;
  if (threadIdx.x < 4) {
    gs.db3[threadIdx.x] = 0.f;
    gs.loss[threadIdx.x] = 0.f;
  }
  // dW2 rows [16 warp, 16 warp + 16) x 64 cols; dW1 rows [16 warp, +16) x 16 cols
  float dW2[8][4], dW1[2][4];
#pragma unroll
  for (int n = 0; n < 8; n++) dW2[n][0] = dW2[n][1] = dW2[n][2] = dW2[n][3] = 0.f;
#pragma unroll
  for (int n = 0; n < 2; n++) dW1[n][0] = dW1[n][1] = dW1[n][2] = dW1[n][3] = 0.f;
  float db1 = 0.f, db2 = 0.f;  // thread i < 64: db2[i]; 64 <= i < 128: db1[i - 64]
  __syncthreads();
  const int64_t nchunks = (nrows + 63) / 64;
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int64_t r0 = ch * 64 + warp * 16;  // this warp's 16 rows (relative)
    // inputs of rows r0 + g, r0 + g + 8
    uint32_t xa[4];
    {
      const int64_t ra = r0 + g, rb = r0 + g + 8;
      const uint32_t* Xa = reinterpret_cast<const uint32_t*>(X + (row0 + ra) * MLP_IN);
      const uint32_t* Xb = reinterpret_cast<const uint32_t*>(X + (row0 + rb) * MLP_IN);
      xa[0] = ra < nrows ? Xa[t] : 0u;
      xa[1] = rb < nrows ? Xb[t] : 0u;
      xa[2] = ra < nrows ? Xa[t + 4] : 0u;
      xa[3] = rb < nrows ? Xb[t + 4] : 0u;
    }
    float z1[8][4], z2[8][4], y0, y1;
    mlp_tile_forward(sm, xa, g, t, z1, z2, y0, y1);
    const int64_t ra = r0 + g, rb = r0 + g + 8;
    const float e0 = ra < nrows ? y0 - T[row0 + ra] : 0.f;
    const float e1 = rb < nrows ? y1 - T[row0 + rb] : 0.f;
    const float d0 = wscale * e0, d1 = wscale * e1;  // dL/dy
    {
      // every lane of a quad holds its rows' errors: sum over the 8 quads of the warp
      float ls = e0 * e0 + e1 * e1, bs = d0 + d1;
      ls += __shfl_xor_sync(0xffffffffu, ls, 4);
      ls += __shfl_xor_sync(0xffffffffu, ls, 8);
      ls += __shfl_xor_sync(0xffffffffu, ls, 16);
      bs += __shfl_xor_sync(0xffffffffu, bs, 4);
      bs += __shfl_xor_sync(0xffffffffu, bs, 8);
      bs += __shfl_xor_sync(0xffffffffu, bs, 16);
      if (lane == 0) {
        gs.loss[warp] += ls;
        gs.db3[warp] += bs;
      }
    }
    // layer 3 and dZ2 = dy w3 [z2 > 0]
    float dz2[8][4];
#pragma unroll
    for (int n = 0; n < 8; n++) {
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int j = n * 8 + 2 * t + e;
        const float h0 = __bfloat162float(__float2bfloat16_rn(fmaxf(z2[n][e], 0.f)));
        const float h1v = __bfloat162float(__float2bfloat16_rn(fmaxf(z2[n][2 + e], 0.f)));
        float pw = d0 * h0 + d1 * h1v;  // dw3[j] partial over rows g, g+8
        pw += __shfl_xor_sync(0xffffffffu, pw, 4);
        pw += __shfl_xor_sync(0xffffffffu, pw, 8);
        pw += __shfl_xor_sync(0xffffffffu, pw, 16);
        if (g == 0) gs.dw3[warp][j] += pw;
        dz2[n][e] = z2[n][e] > 0.f ? d0 * sm.w3[j] : 0.f;
        dz2[n][2 + e] = z2[n][2 + e] > 0.f ? d1 * sm.w3[j] : 0.f;
      }
    }
    // dH1 = dZ2 W2 (A = dZ2 as bf16 fragments, B = W2 via its transpose)
    uint32_t da[4][4];
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
      da[kk][0] = pack_bf16(dz2[2 * kk][0], dz2[2 * kk][1]);
      da[kk][1] = pack_bf16(dz2[2 * kk][2], dz2[2 * kk][3]);
      da[kk][2] = pack_bf16(dz2[2 * kk + 1][0], dz2[2 * kk + 1][1]);
      da[kk][3] = pack_bf16(dz2[2 * kk + 1][2], dz2[2 * kk + 1][3]);
    }
    float dz1[8][4];
#pragma unroll
    for (int n = 0; n < 8; n++) {
      dz1[n][0] = dz1[n][1] = dz1[n][2] = dz1[n][3] = 0.f;
#pragma unroll
      for (int kk = 0; kk < 4; kk++) {
        uint32_t b0, b1;
        bfrag(&gs.W2T[0][0], W2S, n * 8, kk * 16, g, t, b0, b1);
        mma_bf16(dz1[n], da[kk][0], da[kk][1], da[kk][2], da[kk][3], b0, b1);
      }
#pragma unroll
      for (int e = 0; e < 4; e++) dz1[n][e] = z1[n][e] > 0.f ? dz1[n][e] : 0.f;
    }
    // stage transposed tiles (columns = this chunk's 64 rows)
    const int ca = warp * 16 + g, cb = warp * 16 + g + 8;
#pragma unroll
    for (int n = 0; n < 8; n++) {
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int j = n * 8 + 2 * t + e;
        gs.dz2T[j][ca] = __float2bfloat16_rn(dz2[n][e]);
        gs.dz2T[j][cb] = __float2bfloat16_rn(dz2[n][2 + e]);
        gs.dz1T[j][ca] = __float2bfloat16_rn(dz1[n][e]);
        gs.dz1T[j][cb] = __float2bfloat16_rn(dz1[n][2 + e]);
        gs.h1T[j][ca] = __float2bfloat16_rn(fmaxf(z1[n][e], 0.f));
        gs.h1T[j][cb] = __float2bfloat16_rn(fmaxf(z1[n][2 + e], 0.f));
      }
    }
    {
      const __nv_bfloat162* xa2 = reinterpret_cast<const __nv_bfloat162*>(xa);
      gs.xT[2 * t][ca] = xa2[0].x;
      gs.xT[2 * t + 1][ca] = xa2[0].y;
      gs.xT[2 * t][cb] = xa2[1].x;
      gs.xT[2 * t + 1][cb] = xa2[1].y;
      gs.xT[2 * t + 8][ca] = xa2[2].x;
      gs.xT[2 * t + 9][ca] = xa2[2].y;
      gs.xT[2 * t + 8][cb] = xa2[3].x;
      gs.xT[2 * t + 9][cb] = xa2[3].y;
    }
    __syncthreads();
    // dW2[i][j] += sum_r dZ2T[i][r] H1T[j][r];  dW1[i][j] += sum_r dZ1T[i][r] XT[j][r]
    const int i0 = warp * 16;
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
      const int k0 = kk * 16;
      uint32_t a[4], a1[4];
      a[0] = *reinterpret_cast<const uint32_t*>(&gs.dz2T[i0 + g][k0 + 2 * t]);
      a[1] = *reinterpret_cast<const uint32_t*>(&gs.dz2T[i0 + g + 8][k0 + 2 * t]);
      a[2] = *reinterpret_cast<const uint32_t*>(&gs.dz2T[i0 + g][k0 + 2 * t + 8]);
      a[3] = *reinterpret_cast<const uint32_t*>(&gs.dz2T[i0 + g + 8][k0 + 2 * t + 8]);
      a1[0] = *reinterpret_cast<const uint32_t*>(&gs.dz1T[i0 + g][k0 + 2 * t]);
      a1[1] = *reinterpret_cast<const uint32_t*>(&gs.dz1T[i0 + g + 8][k0 + 2 * t]);
      a1[2] = *reinterpret_cast<const uint32_t*>(&gs.dz1T[i0 + g][k0 + 2 * t + 8]);
      a1[3] = *reinterpret_cast<const uint32_t*>(&gs.dz1T[i0 + g + 8][k0 + 2 * t + 8]);
#pragma unroll
      for (int n = 0; n < 8; n++) {
        uint32_t b0, b1;
        bfrag(&gs.h1T[0][0], GS, n * 8, k0, g, t, b0, b1);
        mma_bf16(dW2[n], a[0], a[1], a[2], a[3], b0, b1);
      }
#pragma unroll
      for (int n = 0; n < 2; n++) {
        uint32_t b0, b1;
        bfrag(&gs.xT[0][0], GS, n * 8, k0, g, t, b0, b1);
        mma_bf16(dW1[n], a1[0], a1[1], a1[2], a1[3], b0, b1);
      }
    }
    // bias gradients: thread i < 64 owns db2[i], 64 <= i < 128 owns db1[i - 64]
    {
      const int i = threadIdx.x & 63;
      const __nv_bfloat16* rowp = threadIdx.x < 64 ? gs.dz2T[i] : gs.dz1T[i];
      float sacc = 0.f;
      for (int c = 0; c < 64; c++) sacc += __bfloat162float(rowp[c]);
      if (threadIdx.x < 64)
        db2 += sacc;
      else
        db1 += sacc;
    }
    __syncthreads();
  }
  // write this CTA's partial gradient
  float* out = part + (int64_t)blockIdx.x * MLP_P;
  const int i0 = warp * 16;
#pragma unroll
  for (int n = 0; n < 8; n++) {
    const int j = n * 8 + 2 * t;
    out[OFF_W2 + (i0 + g) * MLP_H + j] = dW2[n][0];
    out[OFF_W2 + (i0 + g) * MLP_H + j + 1] = dW2[n][1];
    out[OFF_W2 + (i0 + g + 8) * MLP_H + j] = dW2[n][2];
    out[OFF_W2 + (i0 + g + 8) * MLP_H + j + 1] = dW2[n][3];
  }
#pragma unroll
  for (int n = 0; n < 2; n++) {
    const int j = n * 8 + 2 * t;
    out[OFF_W1 + (i0 + g) * MLP_IN + j] = dW1[n][0];
    out[OFF_W1 + (i0 + g) * MLP_IN + j + 1] = dW1[n][1];
    out[OFF_W1 + (i0 + g + 8) * MLP_IN + j] = dW1[n][2];
    out[OFF_W1 + (i0 + g + 8) * MLP_IN + j + 1] = dW1[n][3];
  }
  if (threadIdx.x < 64)
    out[OFF_B2 + threadIdx.x] = db2;
  else
    out[OFF_B1 + threadIdx.x - 64] = db1;
  __syncthreads();
  if (threadIdx.x < MLP_H)
    out[OFF_W3 + threadIdx.x] = ((gs.dw3[0][threadIdx.x] + gs.dw3[1][threadIdx.x]) +
                                 gs.dw3[2][threadIdx.x]) + gs.dw3[3][threadIdx.x];
  if (threadIdx.x == 0) {
    out[OFF_B3] = ((gs.db3[0] + gs.db3[1]) + gs.db3[2]) + gs.db3[3];
    loss_part[blockIdx.x] = ((gs.loss[0] + gs.loss[1]) + gs.loss[2]) + gs.loss[3];
  }
}

// Sum the CTA partials in CTA order, AdamW on the FP32 master parameters.
__global__ void k_mlp_adamw(const float* __restrict__ part, int nparts,
                            const float* __restrict__ loss_part, float* __restrict__ P,
                            float* __restrict__ m, float* __restrict__ v, float lr, float b1,
                            float b2, float eps, float wd, float bc1, float bc2,
                            float* __restrict__ grad_out, float* __restrict__ loss_out) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < MLP_P; p += gridDim.x * blockDim.x) {
    float gsum = 0.f;
    for (int c = 0; c < nparts; c++) gsum += part[(int64_t)c * MLP_P + p];
    if (grad_out) grad_out[p] = gsum;
    if (lr > 0.f) {
      const float mm = b1 * m[p] + (1.f - b1) * gsum;
      const float vv = b2 * v[p] + (1.f - b2) * gsum * gsum;
      m[p] = mm;
      v[p] = vv;
      const bool decay = !((p >= OFF_B1 && p < OFF_W2) || (p >= OFF_B2 && p < OFF_W3) ||
                           p == OFF_B3);
      P[p] -= lr * ((mm / bc1) / (sqrtf(vv / bc2) + eps) + (decay ? wd * P[p] : 0.f));
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && loss_out) {
    float l = 0.f;
    for (int c = 0; c < nparts; c++) l += loss_part[c];
    *loss_out = l;
  }
}

}  // namespace tp

using namespace tp;

static MlpFeat make_feat(const tp_mlp_inputs* in) {
  MlpFeat F;
  F.U = in->U;
  F.Up = in->U_prev;
  F.phi = in->phi;
  F.ngphi = in->normgradphi;
  F.opU = in->opU;
  F.opDU = in->opDU;
  F.S = in->S;
  F.ld = in->ld;
  F.base = in->base;
  for (int s = 0; s < 4; s++) {
    F.logD[s] = (float)in->logD[s];
    F.k[s] = (float)in->k[s];
  }
  for (int f = 0; f < NFEAT; f++) {
    F.mean[f] = (float)in->mean[f];
    F.istd[f] = (float)in->istd[f];
  }
  return F;
}

static std::atomic<uint32_t> g_tc_polls{TC_WAIT_LIMIT};
static std::atomic<int> g_tc_skip{0};

extern "C" int tp_mlp_param_count(void) { return MLP_P; }

extern "C" int tp_mlp_predict(const tp_mlp_inputs* in, const float* params, float sigma,
                              double* x_out, float* y_out, void* stream) {
  TP_REQUIRE(in && in->U && in->U_prev && params && (x_out || y_out), "null pointer");
  TP_REQUIRE(in->S >= 1 && in->S <= 4 && in->ld >= in->S, "bad S/ld");
  TP_REQUIRE(in->base >= 0 && in->base <= 2, "base must be 0 (u^n), 1 (2 u^n - u^{n-1}) or 2 (none)");
  const int64_t nrows = in->n_verts * in->S;
  if (nrows == 0) return TP_OK;
  const int64_t ntiles = (nrows + TC_M - 1) / TC_M;
  // persistent CTAs, 4 per SM (4 x 128 tensor-memory columns = the SM's 512)
  const int grid = (int)std::min<int64_t>(ntiles, (int64_t)sm_count() * 4);
  cudaStream_t st = as_stream(stream);
  TcWait tw{g_tc_polls.load(), g_tc_skip.load(), in->tc_status};
  if (tw.status) TP_CUDA_TRY(cudaMemsetAsync(tw.status, 0, sizeof(int32_t), st));
  k_mlp_predict<<<grid, TC_M, 0, st>>>(make_feat(in), nrows, params, sigma, x_out, y_out, tw);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_mlp_set_wait_limit(unsigned int polls, int skip_issue) {
  g_tc_polls.store(polls ? polls : TC_WAIT_LIMIT);
  g_tc_skip.store(skip_issue ? 1 : 0);
  return TP_OK;
}

extern "C" int tp_mlp_tensor_status(int* timed_out, void* stream) {
  TP_REQUIRE(timed_out, "null pointer");
  cudaStream_t st = as_stream(stream);
  TP_CUDA_TRY(cudaMemcpyFromSymbolAsync(timed_out, g_mlp_tc_timeout, sizeof(int), 0,
                                        cudaMemcpyDeviceToHost, st));
  TP_CUDA_TRY(cudaStreamSynchronize(st));
  return TP_OK;
}

extern "C" int tp_mlp_features(const tp_mlp_inputs* in, void* X, void* stream) {
  TP_REQUIRE(in && in->U && in->U_prev && X, "null pointer");
  const int64_t nrows = in->n_verts * in->S;
  if (nrows == 0) return TP_OK;
  k_mlp_features<<<grid_for(nrows * MLP_IN, 256, 65535), 256, 0, as_stream(stream)>>>(
      make_feat(in), nrows, static_cast<__nv_bfloat16*>(X));
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_mlp_target(int64_t n_verts, int S, int ld, const double* U_n,
                             const double* U_prev, const double* U_next, double sigma, float* T,
                             void* stream) {
  TP_REQUIRE(U_n && U_next && T && sigma > 0, "bad argument");
  const int64_t nrows = n_verts * S;
  if (nrows == 0) return TP_OK;
  k_mlp_target<<<grid_for(nrows, 256, 65535), 256, 0, as_stream(stream)>>>(
      nrows, S, ld, U_n, U_prev, U_next, (float)(1.0 / sigma), T);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" size_t tp_mlp_grad_workspace_floats(int grid) { return (size_t)grid * (MLP_P + 1); }

extern "C" int tp_mlp_train_step(const void* X, const float* T, int64_t row0, int64_t nrows,
                                 float* params, float* adam_m, float* adam_v, int step,
                                 float lr, float beta1, float beta2, float eps,
                                 float weight_decay, int grid, float* workspace,
                                 float* grad_out, float* loss_out, void* stream) {
  TP_REQUIRE(X && T && params && workspace && grid >= 1, "bad argument");
  TP_REQUIRE(lr <= 0.f || (adam_m && adam_v && step >= 1), "AdamW state required");
  cudaStream_t st = as_stream(stream);
  float* part = workspace;
  float* loss_part = workspace + (size_t)grid * MLP_P;
  const float wscale = nrows > 0 ? 2.0f / (float)nrows : 0.f;
  TP_CUDA_TRY(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)sizeof(GradSmem)));
  k_mlp_grad<<<grid, 128, sizeof(GradSmem), st>>>(static_cast<const __nv_bfloat16*>(X), T, row0,
                                                  nrows, params, wscale, part, loss_part);
  TP_LAUNCH_CHECK();
  const float bc1 = 1.f - powf(beta1, (float)std::max(step, 1));
  const float bc2 = 1.f - powf(beta2, (float)std::max(step, 1));
  k_mlp_adamw<<<(MLP_P + 255) / 256, 256, 0, st>>>(part, grid, loss_part, params, adam_m, adam_v,
                                                   lr, beta1, beta2, eps, weight_decay, bc1,
                                                   bc2, grad_out, loss_out);
  TP_LAUNCH_CHECK();
  return TP_OK;
}
