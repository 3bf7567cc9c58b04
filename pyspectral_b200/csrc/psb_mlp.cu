// Training and stand-alone inference of the subgrid-stress MLP on BF16 tensor
// cores (mma.sync m16n8k16, FP32 accumulation).  See psb_mlp.cuh for the
// parameter layout.  One training step = psb_mlp_train_step: a fused forward /
// loss / backward kernel over the minibatch (each CTA: 128 points, weight
// gradients of its points reduced with tensor-core GEMMs over the point axis,
// then added to the global FP32 gradient), followed by an Adam update that also
// clears the gradient.
#include <cuda_bf16.h>

#include "psb_ctx.cuh"
#include "psb_mlp.cuh"
#include "psb_tc.cuh"

using namespace psb;
using namespace psbh;

namespace {

static_assert(kActGelu == PSB_ACT_GELU && kActRelu == PSB_ACT_RELU, "activation codes");

constexpr int kRows = 128;  // points per CTA (8 warps x 16)

template <int H>
struct TrainSmem {
  MlpSmem<H> m;
  __nv_bfloat16 X[kRows * 16];
  __nv_bfloat16 H1[kRows * H];
  __nv_bfloat16 H2[kRows * H];
  __nv_bfloat16 dY[kRows * 16];
  __nv_bfloat16 dZ2[kRows * H];
  __nv_bfloat16 dZ1[kRows * H];
  float db1[H], db2[H], db3[8];
  float loss;
};

// A fragment of M = S^T where S is stored [k][m] row-major (ld = m stride).
__device__ __forceinline__ void afrag_km(uint32_t* a, const __nv_bfloat16* S, int ld, int m0, int k0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  const int k = k0 + 2 * t;
  a[0] = pack_raw(S[k * ld + m0 + g], S[(k + 1) * ld + m0 + g]);
  a[1] = pack_raw(S[k * ld + m0 + g + 8], S[(k + 1) * ld + m0 + g + 8]);
  a[2] = pack_raw(S[(k + 8) * ld + m0 + g], S[(k + 9) * ld + m0 + g]);
  a[3] = pack_raw(S[(k + 8) * ld + m0 + g + 8], S[(k + 9) * ld + m0 + g + 8]);
}
// B fragment of a matrix stored [k][n] row-major.
__device__ __forceinline__ void bfrag_kn(uint32_t* b, const __nv_bfloat16* W, int ld, int k0, int n0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  const int k = k0 + 2 * t;
  b[0] = pack_raw(W[k * ld + n0 + g], W[(k + 1) * ld + n0 + g]);
  b[1] = pack_raw(W[(k + 8) * ld + n0 + g], W[(k + 9) * ld + n0 + g]);
}

// grad[NPARAMS] += dL/dparams over B points; loss_acc += sum of squared errors / (6B)
template <int ACT, int H>
__global__ void __launch_bounds__(256) mlp_train_kernel(const float* __restrict__ P, const float* __restrict__ nrm,
                                                        const float* __restrict__ X, const float* __restrict__ T,
                                                        const int* __restrict__ idx, int B, float* __restrict__ grad,
                                                        double* __restrict__ loss_acc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  using L = MlpLayout<H>;
  constexpr int NJ = H / 8, NK = H / 16;
  TrainSmem<H>& s = *reinterpret_cast<TrainSmem<H>*>(smem_raw);
  mlp_stage<H>(s.m, P, nrm);
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    s.db1[i] = 0.f;
    s.db2[i] = 0.f;
  }
  if (threadIdx.x < 8) s.db3[threadIdx.x] = 0.f;
  if (threadIdx.x == 0) s.loss = 0.f;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int r0 = blockIdx.x * kRows + warp * 16;  // first batch row of this warp
  auto rowid = [&](int r) -> int { return r0 + r < B ? idx[r0 + r] : -1; };
  const int id_lo = rowid(g), id_hi = rowid(g + 8);
  uint32_t xa[4];
  mlp_xfrag(s.m, xa, [&](int r, int f) {
    const int id = r == g ? id_lo : id_hi;
    return id >= 0 ? X[(long long)id * kMlpIn + f] : s.m.xmean[f];
  });
  float z1[NJ][4], z2[NJ][4], y[4];
  mlp_forward_warp<ACT, H>(s.m, xa, y, z1, z2);
  // dY = 2 (y - t) / (6B), rows without a point contribute nothing
  const float sc = 2.f / (6.f * (float)B);
  float dy[4];
  float lsum = 0.f;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int c = 2 * t + (e & 1);
    const int id = e < 2 ? id_lo : id_hi;
    float d = 0.f;
    if (c < kMlpOut && id >= 0) {
      const float tn = (T[(long long)id * kMlpOut + c] - s.m.ymean[c]) / s.m.ystd[c];
      d = y[e] - tn;
      lsum += d * d;
    }
    dy[e] = sc * d;
  }
  atomicAdd(&s.loss, lsum);
  // stage X, H1, H2 (bf16) and dY for the weight-gradient GEMMs
  {
    const int ra = warp * 16 + g, rb = ra + 8;
    // X: features in the same positions as xa
    const __nv_bfloat162* xv = reinterpret_cast<const __nv_bfloat162*>(xa);
    *reinterpret_cast<__nv_bfloat162*>(&s.X[ra * 16 + 2 * t]) = xv[0];
    *reinterpret_cast<__nv_bfloat162*>(&s.X[rb * 16 + 2 * t]) = xv[1];
    *reinterpret_cast<__nv_bfloat162*>(&s.X[ra * 16 + 2 * t + 8]) = xv[2];
    *reinterpret_cast<__nv_bfloat162*>(&s.X[rb * 16 + 2 * t + 8]) = xv[3];
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      const int col = 8 * j + 2 * t;
      *reinterpret_cast<__nv_bfloat162*>(&s.H1[ra * H + col]) =
          __floats2bfloat162_rn(act_f<ACT>(z1[j][0]), act_f<ACT>(z1[j][1]));
      *reinterpret_cast<__nv_bfloat162*>(&s.H1[rb * H + col]) =
          __floats2bfloat162_rn(act_f<ACT>(z1[j][2]), act_f<ACT>(z1[j][3]));
      *reinterpret_cast<__nv_bfloat162*>(&s.H2[ra * H + col]) =
          __floats2bfloat162_rn(act_f<ACT>(z2[j][0]), act_f<ACT>(z2[j][1]));
      *reinterpret_cast<__nv_bfloat162*>(&s.H2[rb * H + col]) =
          __floats2bfloat162_rn(act_f<ACT>(z2[j][2]), act_f<ACT>(z2[j][3]));
    }
    *reinterpret_cast<__nv_bfloat162*>(&s.dY[ra * 16 + 2 * t]) = __floats2bfloat162_rn(dy[0], dy[1]);
    *reinterpret_cast<__nv_bfloat162*>(&s.dY[rb * 16 + 2 * t]) = __floats2bfloat162_rn(dy[2], dy[3]);
    *reinterpret_cast<__nv_bfloat162*>(&s.dY[ra * 16 + 2 * t + 8]) = __floats2bfloat162_rn(0.f, 0.f);
    *reinterpret_cast<__nv_bfloat162*>(&s.dY[rb * 16 + 2 * t + 8]) = __floats2bfloat162_rn(0.f, 0.f);
    if (t < 3) {
      atomicAdd(&s.db3[2 * t], dy[0] + dy[2]);
      atomicAdd(&s.db3[2 * t + 1], dy[1] + dy[3]);
    }
  }
  // dH2 = dY W3 (k = 8 outputs, padded to 16), dZ2 = dH2 * act'(z2)
  uint32_t da[4];
  da[0] = pack_bf16(dy[0], dy[1]);
  da[1] = pack_bf16(dy[2], dy[3]);
  da[2] = 0u;
  da[3] = 0u;
  float dz2[NJ][4];
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    dz2[j][0] = dz2[j][1] = dz2[j][2] = dz2[j][3] = 0.f;
    uint32_t b[2];
    b[0] = pack_raw(s.m.w3[(2 * t) * H + 8 * j + g], s.m.w3[(2 * t + 1) * H + 8 * j + g]);
    b[1] = 0u;
    mma16816(dz2[j], da, b);
#pragma unroll
    for (int e = 0; e < 4; ++e) dz2[j][e] *= act_d<ACT>(z2[j][e]);
  }
  uint32_t a2[NK][4];
#pragma unroll
  for (int kk = 0; kk < NK; ++kk) {
    a2[kk][0] = pack_bf16(dz2[2 * kk][0], dz2[2 * kk][1]);
    a2[kk][1] = pack_bf16(dz2[2 * kk][2], dz2[2 * kk][3]);
    a2[kk][2] = pack_bf16(dz2[2 * kk + 1][0], dz2[2 * kk + 1][1]);
    a2[kk][3] = pack_bf16(dz2[2 * kk + 1][2], dz2[2 * kk + 1][3]);
  }
  // dH1 = dZ2 W2 (W2 stored [out=k][in=n]), dZ1 = dH1 * act'(z1)
  float dz1[NJ][4];
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    dz1[j][0] = dz1[j][1] = dz1[j][2] = dz1[j][3] = 0.f;
#pragma unroll
    for (int kk = 0; kk < NK; ++kk) {
      uint32_t b[2];
      bfrag_kn(b, s.m.w2, H, 16 * kk, 8 * j, lane);
      mma16816(dz1[j], a2[kk], b);
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) dz1[j][e] *= act_d<ACT>(z1[j][e]);
  }
  {
    const int ra = warp * 16 + g, rb = ra + 8;
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      const int col = 8 * j + 2 * t;
      *reinterpret_cast<__nv_bfloat162*>(&s.dZ2[ra * H + col]) = __floats2bfloat162_rn(dz2[j][0], dz2[j][1]);
      *reinterpret_cast<__nv_bfloat162*>(&s.dZ2[rb * H + col]) = __floats2bfloat162_rn(dz2[j][2], dz2[j][3]);
      *reinterpret_cast<__nv_bfloat162*>(&s.dZ1[ra * H + col]) = __floats2bfloat162_rn(dz1[j][0], dz1[j][1]);
      *reinterpret_cast<__nv_bfloat162*>(&s.dZ1[rb * H + col]) = __floats2bfloat162_rn(dz1[j][2], dz1[j][3]);
      atomicAdd(&s.db2[col], dz2[j][0] + dz2[j][2]);
      atomicAdd(&s.db2[col + 1], dz2[j][1] + dz2[j][3]);
      atomicAdd(&s.db1[col], dz1[j][0] + dz1[j][2]);
      atomicAdd(&s.db1[col + 1], dz1[j][1] + dz1[j][3]);
    }
  }
  __syncthreads();
  // weight gradients, contracting over the 128 points of the CTA
  // dW2[o][i] = sum_r dZ2[r][o] H1[r][i]: (H/16) x (H/8) tiles over the warps
#pragma unroll 1
  for (int tile = warp; tile < NK * NJ; tile += 8) {
    const int m0 = (tile / NJ) * 16, n0 = (tile % NJ) * 8;
    float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int k0 = 0; k0 < kRows; k0 += 16) {
      uint32_t a[4], b[2];
      afrag_km(a, s.dZ2, H, m0, k0, lane);
      bfrag_kn(b, s.H1, H, k0, n0, lane);
      mma16816(c, a, b);
    }
    float* G = grad + L::W2;
    atomicAdd(&G[(m0 + g) * H + n0 + 2 * t], c[0]);
    atomicAdd(&G[(m0 + g) * H + n0 + 2 * t + 1], c[1]);
    atomicAdd(&G[(m0 + g + 8) * H + n0 + 2 * t], c[2]);
    atomicAdd(&G[(m0 + g + 8) * H + n0 + 2 * t + 1], c[3]);
  }
  // dW1[o][f] = sum_r dZ1[r][o] X[r][f]: (H/16) x 2 tiles over the warps
#pragma unroll 1
  for (int tile = warp; tile < 2 * NK; tile += 8) {
    const int m0 = (tile / 2) * 16, n0 = (tile % 2) * 8;
    float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int k0 = 0; k0 < kRows; k0 += 16) {
      uint32_t a[4], b[2];
      afrag_km(a, s.dZ1, H, m0, k0, lane);
      bfrag_kn(b, s.X, 16, k0, n0, lane);
      mma16816(c, a, b);
    }
    float* G = grad + L::W1;
    const int f0 = n0 + 2 * t;
    if (f0 < kMlpIn) {
      atomicAdd(&G[(m0 + g) * kMlpIn + f0], c[0]);
      atomicAdd(&G[(m0 + g + 8) * kMlpIn + f0], c[2]);
    }
    if (f0 + 1 < kMlpIn) {
      atomicAdd(&G[(m0 + g) * kMlpIn + f0 + 1], c[1]);
      atomicAdd(&G[(m0 + g + 8) * kMlpIn + f0 + 1], c[3]);
    }
  }
  // dW3[c][i] = sum_r dY[r][c] H2[r][i]: m = 16 (6 used) x H/8 n-tiles over the warps
#pragma unroll 1
  for (int tile = warp; tile < NJ; tile += 8) {
    const int n0 = tile * 8;
    float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int k0 = 0; k0 < kRows; k0 += 16) {
      uint32_t a[4], b[2];
      afrag_km(a, s.dY, 16, 0, k0, lane);
      bfrag_kn(b, s.H2, H, k0, n0, lane);
      mma16816(c, a, b);
    }
    float* G = grad + L::W3;
    if (g < kMlpOut) {
      atomicAdd(&G[g * H + n0 + 2 * t], c[0]);
      atomicAdd(&G[g * H + n0 + 2 * t + 1], c[1]);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    atomicAdd(&grad[L::B1 + i], s.db1[i]);
    atomicAdd(&grad[L::B2 + i], s.db2[i]);
  }
  if (threadIdx.x < kMlpOut) atomicAdd(&grad[L::B3 + threadIdx.x], s.db3[threadIdx.x]);
  if (threadIdx.x == 0) atomicAdd(loss_acc, (double)s.loss / (6.0 * (double)B));
}

__global__ void adam_kernel(float* __restrict__ P, float* __restrict__ m, float* __restrict__ v,
                            float* __restrict__ grad, int n, float lr, float b1, float b2, float eps, float c1,
                            float c2, float wd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gr = grad[i];
  const float mi = b1 * m[i] + (1.f - b1) * gr;
  const float vi = b2 * v[i] + (1.f - b2) * gr * gr;
  m[i] = mi;
  v[i] = vi;
  P[i] -= lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * P[i]);
  grad[i] = 0.f;
}

template <int ACT, int H>
__global__ void __launch_bounds__(256) mlp_forward_kernel(const float* __restrict__ P, const float* __restrict__ nrm,
                                                          const float* __restrict__ X, int B,
                                                          float* __restrict__ Y) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  MlpFwdSmem<H>& s = *reinterpret_cast<MlpFwdSmem<H>*>(smem_raw);
  mlp_stage_fwd<H>(s, P, nrm);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int nw = blockDim.x >> 5;
  for (int r0 = (blockIdx.x * nw + warp) * 16; r0 < B; r0 += gridDim.x * nw * 16) {
    uint32_t xa[4];
    mlp_xfrag(s, xa, [&](int r, int f) {
      return r0 + r < B ? X[(long long)(r0 + r) * kMlpIn + f] : s.xmean[f];
    });
    float y[4];
    mlp_forward_fast<ACT, H>(s, xa, y);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int c = 2 * t + (e & 1), r = r0 + g + (e < 2 ? 0 : 8);
      if (c < kMlpOut && r < B) Y[(long long)r * kMlpOut + c] = y[e] * s.ystd[c] + s.ymean[c];
    }
  }
}

// ---- inference on the fifth-generation tensor cores (tcgen05) -------------
// Tiles of 128 points: the CTA writes the tile's normalised features as the
// A operand of layer 1 (one 128 x 16 slab), one thread issues the MMA into a
// 128-lane x 64-column FP32 accumulator in tensor memory, the eight warps read
// it back (warp w: lanes 32 (w % 4).., columns 32 (w / 4)..), add the bias,
// apply the activation and write BF16 activations as the next layer's A
// operand (four 128 x 16 slabs); layers 2 and 3 are four K-steps each.  The
// weights are staged once per CTA as K-major slabs (B operands).
struct MlpTcSmem {
  unsigned char w1[64 * 16 * 2];      // 64 x 16 (k 10..15 zero)
  unsigned char w2[4 * 64 * 16 * 2];  // 4 slabs of 64 x 16
  unsigned char w3[4 * 16 * 16 * 2];  // 4 slabs of 16 x 16 (rows 6..15 zero)
  unsigned char h[4 * 128 * 16 * 2];  // activations: 4 slabs of 128 x 16 (slab 0 = layer-1 input)
  float b1[kMlpH], b2[kMlpH], b3[16];
  float xmean[16], xistd[16], ymean[8], ystd[8];
  unsigned long long mbar;
  uint32_t tmem;
};
constexpr uint32_t kTcPolls = 1u << 22;  // bound on the polls of one MMA completion

__device__ __forceinline__ void put_bf16(unsigned char* slab, int r, int k, float v) {
  *reinterpret_cast<__nv_bfloat16*>(slab + tc::slab_off(r, k)) = __float2bfloat16_rn(v);
}

__device__ void mlp_tc_stage(MlpTcSmem& s, const float* __restrict__ P, const float* __restrict__ nrm) {
  for (int i = threadIdx.x; i < 64 * 16; i += blockDim.x) {
    const int n = i >> 4, k = i & 15;
    put_bf16(s.w1, n, k, k < kMlpIn ? P[kOffW1 + n * kMlpIn + k] : 0.f);
  }
  for (int i = threadIdx.x; i < 64 * 64; i += blockDim.x) {
    const int n = i >> 6, k = i & 63;
    put_bf16(s.w2 + (k >> 4) * 2048, n, k & 15, P[kOffW2 + n * kMlpH + k]);
  }
  for (int i = threadIdx.x; i < 16 * 64; i += blockDim.x) {
    const int n = i >> 6, k = i & 63;
    put_bf16(s.w3 + (k >> 4) * 512, n, k & 15, n < kMlpOut ? P[kOffW3 + n * kMlpH + k] : 0.f);
  }
  for (int i = threadIdx.x; i < kMlpH; i += blockDim.x) {
    s.b1[i] = P[kOffB1 + i];
    s.b2[i] = P[kOffB2 + i];
  }
  if (threadIdx.x < 16) {
    s.b3[threadIdx.x] = threadIdx.x < kMlpOut ? P[kOffB3 + threadIdx.x] : 0.f;
    s.xmean[threadIdx.x] = threadIdx.x < kMlpIn ? nrm[threadIdx.x] : 0.f;
    s.xistd[threadIdx.x] = threadIdx.x < kMlpIn ? nrm[kMlpIn + threadIdx.x] : 0.f;
  }
  if (threadIdx.x < 8) {
    s.ymean[threadIdx.x] = threadIdx.x < kMlpOut ? nrm[2 * kMlpIn + threadIdx.x] : 0.f;
    s.ystd[threadIdx.x] = threadIdx.x < kMlpOut ? nrm[2 * kMlpIn + kMlpOut + threadIdx.x] : 0.f;
  }
}

// Accumulator columns 32*half.. of this thread's row (+ bias, activation) as
// BF16 into activation slabs 2*half, 2*half+1.
template <int ACT>
__device__ __forceinline__ void mlp_tc_hidden(MlpTcSmem& s, uint32_t taddr, const float* bias, int row, int half) {
  float v[32];
  tc::ld32(taddr, v);
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    uint32_t w[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int col = 32 * half + 8 * c + 2 * e;
      w[e] = act_pack<ACT>(v[8 * c + 2 * e] + bias[col], v[8 * c + 2 * e + 1] + bias[col + 1]);
    }
    const int chunk = 4 * half + c;  // 8-column chunk of the 64 outputs
    *reinterpret_cast<uint4*>(s.h + (chunk >> 1) * 4096 + tc::slab_off(row, (chunk & 1) * 8)) =
        make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// Thread 0 waits for the MMAs it committed; the CTA agrees on the outcome.
__device__ __forceinline__ bool mlp_tc_wait(uint32_t mbar, uint32_t& phase) {
  const bool ok = tc::mbar_wait(mbar, phase, kTcPolls);
  phase ^= 1;
  return __syncthreads_and(ok) != 0;
}

// The three layers of one 128-point tile whose layer-1 input is in slab 0 of
// s.h; returns false if an MMA did not complete within the poll limit.  On
// return warps 0-3 hold their row's 8 output columns (bias added) in y.
template <int ACT>
__device__ __forceinline__ bool mlp_tc_tile(MlpTcSmem& s, uint32_t& phase, float* y) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = warp & 3, half = warp >> 2, row = 32 * q + lane;
  const uint32_t mbar = tc::smem_u32(&s.mbar), tbase = s.tmem;
  const uint32_t trow = tbase + ((uint32_t)(32 * q) << 16);
  const uint32_t hs = tc::smem_u32(s.h);
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    tc::fence_after();
    tc::mma(tbase, tc::desc(hs), tc::desc(tc::smem_u32(s.w1)), tc::idesc_bf16(128, 64), false);
    tc::commit(mbar);
  }
  if (!mlp_tc_wait(mbar, phase)) return false;
  tc::fence_after();
  mlp_tc_hidden<ACT>(s, trow + 32 * half, s.b1, row, half);
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    tc::fence_after();
#pragma unroll
    for (int k = 0; k < 4; ++k)
      tc::mma(tbase, tc::desc(hs + k * 4096), tc::desc(tc::smem_u32(s.w2) + k * 2048), tc::idesc_bf16(128, 64),
              k > 0);
    tc::commit(mbar);
  }
  if (!mlp_tc_wait(mbar, phase)) return false;
  tc::fence_after();
  mlp_tc_hidden<ACT>(s, trow + 32 * half, s.b2, row, half);
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    tc::fence_after();
#pragma unroll
    for (int k = 0; k < 4; ++k)
      tc::mma(tbase, tc::desc(hs + k * 4096), tc::desc(tc::smem_u32(s.w3) + k * 512), tc::idesc_bf16(128, 16),
              k > 0);
    tc::commit(mbar);
  }
  if (!mlp_tc_wait(mbar, phase)) return false;
  tc::fence_after();
  if (half == 0) {
    tc::ld8(trow, y);
#pragma unroll
    for (int c = 0; c < 8; ++c) y[c] += s.b3[c];
  }
  return true;
}

template <int ACT>
__global__ void __launch_bounds__(256) mlp_forward_tc_kernel(const float* __restrict__ P, const float* __restrict__ nrm,
                                                             const float* __restrict__ X, int B,
                                                             float* __restrict__ Y, int* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  MlpTcSmem& s = *reinterpret_cast<MlpTcSmem*>(smem_raw);
  mlp_tc_stage(s, P, nrm);
  if (threadIdx.x == 0) tc::mbar_init(tc::smem_u32(&s.mbar), 1);
  if (threadIdx.x < 32) tc::alloc(tc::smem_u32(&s.tmem), 64);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  uint32_t phase = 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  bool ok = true;
  for (int t0 = blockIdx.x * 128; t0 < B && ok; t0 += gridDim.x * 128) {
    // features: thread -> row m, K half hk (features 8 hk .. 8 hk + 7)
    {
      const int m = threadIdx.x & 127, hk = threadIdx.x >> 7;
      const int r = t0 + m;
      uint32_t w[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        float f2[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int f = 8 * hk + 2 * e + u;
          f2[u] = (f < kMlpIn && r < B) ? (X[(long long)r * kMlpIn + f] - s.xmean[f]) * s.xistd[f] : 0.f;
        }
        w[e] = pack_bf16(f2[0], f2[1]);
      }
      *reinterpret_cast<uint4*>(s.h + tc::slab_off(m, 8 * hk)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    float y[8];
    ok = mlp_tc_tile<ACT>(s, phase, y);
    if (ok && warp < 4) {
      const int r = t0 + 32 * warp + lane;
      if (r < B)
#pragma unroll
        for (int c = 0; c < kMlpOut; ++c) Y[(long long)r * kMlpOut + c] = y[c] * s.ystd[c] + s.ymean[c];
    }
    tc::fence_before();
    __syncthreads();
  }
  if (!ok) {
    // the MMAs may still be in flight: wait once more (bounded) before freeing
    if (threadIdx.x == 0) {
      tc::mbar_wait(tc::smem_u32(&s.mbar), phase ^ 1, kTcPolls);
      if (err) atomicExch(err, 1);
    }
    __syncthreads();
  }
  tc::fence_after();
  if (threadIdx.x < 32) tc::dealloc(s.tmem, 64);
}

}  // namespace

extern "C" {

int psb_mlp_forward_tc(psb_ctx* c, int act, const float* params, const float* norm, const float* X, int B, float* Y,
                       int* err) {
  if (!c) return PSB_ERR_ARG;
  if (!params || !norm || !X || !Y || B < 0 || (act != kActGelu && act != kActRelu))
    return fail(c, PSB_ERR_ARG, "psb_mlp_forward_tc: bad argument");
  PSB_TRY(cuda_ok(c, cudaSetDevice(c->dev), "cudaSetDevice"));
  if (B == 0) return PSB_OK;
  const size_t smem = sizeof(MlpTcSmem);
  auto go = [&](auto k) {
    set_smem(k, smem);
    const long long grid = persistent_grid(k, smem, ((long long)B + 127) / 128);
    ++c->launches;
    k<<<(unsigned)grid, 256, smem, c->stream>>>(params, norm, X, B, Y, err);
    return launch_ok(c, "mlp forward (tcgen05)");
  };
  return act == kActRelu ? go(mlp_forward_tc_kernel<kActRelu>) : go(mlp_forward_tc_kernel<kActGelu>);
}


// width 0 means 64 (the models trained before the width became a property)
static int mlp_width(int hidden) { return hidden == 0 ? 64 : hidden; }
static bool mlp_width_ok(int hidden) { return mlp_width(hidden) == 32 || mlp_width(hidden) == 64; }

int psb_mlp_sizes(int hidden, int* nparams, int* nnorm) {
  if (!nparams || !nnorm || !mlp_width_ok(hidden)) return PSB_ERR_ARG;
  *nparams = mlp_width(hidden) == 32 ? MlpLayout<32>::NPARAMS : MlpLayout<64>::NPARAMS;
  *nnorm = kMlpNorm;
  return PSB_OK;
}

int psb_mlp_forward(psb_ctx* c, int act, int hidden, const float* params, const float* norm, const float* X, int B,
                    float* Y) {
  if (!c) return PSB_ERR_ARG;
  if (!params || !norm || !X || !Y || B < 0 || (act != kActGelu && act != kActRelu) || !mlp_width_ok(hidden))
    return fail(c, PSB_ERR_ARG, "psb_mlp_forward: bad argument");
  PSB_TRY(cuda_ok(c, cudaSetDevice(c->dev), "cudaSetDevice"));
  if (B == 0) return PSB_OK;
  const int blocks = (int)std::min<long long>(((long long)B + 127) / 128, 148 * 8);
  auto go = [&](auto k, size_t smem) {
    ++c->launches;
    k<<<blocks, 256, smem, c->stream>>>(params, norm, X, B, Y);
    return launch_ok(c, "mlp forward");
  };
  if (mlp_width(hidden) == 32)
    return act == kActRelu ? go(mlp_forward_kernel<kActRelu, 32>, sizeof(MlpFwdSmem<32>))
                           : go(mlp_forward_kernel<kActGelu, 32>, sizeof(MlpFwdSmem<32>));
  return act == kActRelu ? go(mlp_forward_kernel<kActRelu, 64>, sizeof(MlpFwdSmem<64>))
                         : go(mlp_forward_kernel<kActGelu, 64>, sizeof(MlpFwdSmem<64>));
}

int psb_mlp_grad(psb_ctx* c, int act, int hidden, const float* params, const float* norm, const float* X,
                 const float* T, const int* idx, int B, float* grad, double* loss) {
  if (!c) return PSB_ERR_ARG;
  if (!params || !norm || !X || !T || !idx || !grad || !loss || B <= 0 || (act != kActGelu && act != kActRelu) ||
      !mlp_width_ok(hidden))
    return fail(c, PSB_ERR_ARG, "psb_mlp_grad: bad argument");
  PSB_TRY(cuda_ok(c, cudaSetDevice(c->dev), "cudaSetDevice"));
  const unsigned grid = (unsigned)((B + kRows - 1) / kRows);
  auto go = [&](auto k, size_t smem) {
    set_smem(k, smem);
    ++c->launches;
    k<<<grid, 256, smem, c->stream>>>(params, norm, X, T, idx, B, grad, loss);
    return launch_ok(c, "mlp train");
  };
  if (mlp_width(hidden) == 32)
    return act == kActRelu ? go(mlp_train_kernel<kActRelu, 32>, sizeof(TrainSmem<32>))
                           : go(mlp_train_kernel<kActGelu, 32>, sizeof(TrainSmem<32>));
  return act == kActRelu ? go(mlp_train_kernel<kActRelu, 64>, sizeof(TrainSmem<64>))
                         : go(mlp_train_kernel<kActGelu, 64>, sizeof(TrainSmem<64>));
}

int psb_mlp_adam(psb_ctx* c, int hidden, float* params, float* m, float* v, float* grad, int step, float lr,
                 float beta1, float beta2, float eps, float weight_decay) {
  if (!c) return PSB_ERR_ARG;
  if (!params || !m || !v || !grad || step < 1 || !mlp_width_ok(hidden))
    return fail(c, PSB_ERR_ARG, "psb_mlp_adam: bad argument");
  PSB_TRY(cuda_ok(c, cudaSetDevice(c->dev), "cudaSetDevice"));
  const int n = mlp_width(hidden) == 32 ? MlpLayout<32>::NPARAMS : MlpLayout<64>::NPARAMS;
  const float c1 = 1.f - std::pow(beta1, (float)step), c2 = 1.f - std::pow(beta2, (float)step);
  ++c->launches;
  adam_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(params, m, v, grad, n, lr, beta1, beta2, eps, c1, c2,
                                                       weight_decay);
  return launch_ok(c, "adam");
}

}  // extern "C"
