// Pointwise subgrid-stress MLP 10 -> H -> H -> 6 on BF16 tensor cores with
// FP32 accumulation (mma.sync.m16n8k16.bf16, FP32 C/D fragments).  Hidden
// width H (32 or 64) and activation (GELU, kActGelu, or ReLU, kActRelu) are
// properties of the model.
//
// This closure has no counterpart in the reference; it replaces the
// Smagorinsky stress of PySpectral/src/RHSfunctions.py:195-212 by a learned
// map from the 9 resolved velocity-gradient components and the filter width
// to the 6 subgrid-stress components tau_ij = filter(u_i u_j) - u_i u_j.
//
// Parameter block (FP32 master copy, MlpLayout<H>::NPARAMS floats, row-major
// [out][in]):  W1[H][10] b1[H] W2[H][H] b2[H] W3[6][H] b3[6]
// Normalisation block (kMlpNorm floats):
//   xmean[10] xistd[10] ymean[6] ystd[6]
// Features x = (raw - xmean) * xistd; outputs tau = y * ystd + ymean.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace psb {

constexpr int kMlpIn = 10, kMlpOut = 6;
constexpr int kMlpNorm = 32;
constexpr int kActGelu = 0, kActRelu = 1;

// Offsets of the parameter block of a width-H network.
template <int H>
struct MlpLayout {
  static_assert(H == 32 || H == 64, "hidden width 32 or 64");
  static constexpr int W1 = 0, B1 = W1 + H * kMlpIn, W2 = B1 + H, B2 = W2 + H * H, W3 = B2 + H,
                       B3 = W3 + kMlpOut * H, NPARAMS = B3 + kMlpOut;
};
// the width-64 network's layout (the tcgen05 inference kernel's)
constexpr int kMlpH = 64;
constexpr int kOffW1 = MlpLayout<64>::W1, kOffB1 = MlpLayout<64>::B1, kOffW2 = MlpLayout<64>::W2,
              kOffB2 = MlpLayout<64>::B2, kOffW3 = MlpLayout<64>::W3, kOffB3 = MlpLayout<64>::B3,
              kMlpParams = MlpLayout<64>::NPARAMS;

// BF16 operand copies staged in shared memory, padded for the m16n8k16 tiles:
//   w1[H][16] (k padded 10->16), w2[H][H], w3[8][H] (n padded 6->8)
template <int H>
struct MlpSmem {
  __nv_bfloat16 w1[H * 16];
  __nv_bfloat16 w2[H * H];
  __nv_bfloat16 w3[8 * H];
  float b1[H], b2[H], b3[8];
  float xmean[16], xistd[16], ymean[8], ystd[8];
};

template <int H>
__device__ __forceinline__ void mlp_stage(MlpSmem<H>& s, const float* __restrict__ P, const float* __restrict__ nrm) {
  using L = MlpLayout<H>;
  for (int i = threadIdx.x; i < H * 16; i += blockDim.x) {
    const int o = i / 16, k = i % 16;
    s.w1[i] = __float2bfloat16_rn(k < kMlpIn ? P[L::W1 + o * kMlpIn + k] : 0.f);
  }
  for (int i = threadIdx.x; i < H * H; i += blockDim.x) s.w2[i] = __float2bfloat16_rn(P[L::W2 + i]);
  for (int i = threadIdx.x; i < 8 * H; i += blockDim.x) {
    const int o = i / H;
    s.w3[i] = __float2bfloat16_rn(o < kMlpOut ? P[L::W3 + i] : 0.f);
  }
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    s.b1[i] = P[L::B1 + i];
    s.b2[i] = P[L::B2 + i];
  }
  if (threadIdx.x < 16) {
    s.xmean[threadIdx.x] = threadIdx.x < kMlpIn ? nrm[threadIdx.x] : 0.f;
    s.xistd[threadIdx.x] = threadIdx.x < kMlpIn ? nrm[kMlpIn + threadIdx.x] : 0.f;
  }
  if (threadIdx.x < 8) {
    s.b3[threadIdx.x] = threadIdx.x < kMlpOut ? P[L::B3 + threadIdx.x] : 0.f;
    s.ymean[threadIdx.x] = threadIdx.x < kMlpOut ? nrm[2 * kMlpIn + threadIdx.x] : 0.f;
    s.ystd[threadIdx.x] = threadIdx.x < kMlpOut ? nrm[2 * kMlpIn + kMlpOut + threadIdx.x] : 0.f;
  }
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ uint32_t pack_raw(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// D = A(16x16, row) * B(16x8, col) + D, BF16 in, FP32 accumulate.
__device__ __forceinline__ void mma16816(float* d, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// GELU x Phi(x) = x (1 + erf(x / sqrt 2)) / 2 and its derivative, with erf from
// Abramowitz & Stegun, Handbook of Mathematical Functions (1964), formula
// 7.1.26: for z >= 0, erf z = 1 - t (a1 + t (a2 + t (a3 + t (a4 + t a5)))) e^{-z^2},
// t = 1 / (1 + p z), |error| <= 1.5e-7; erf(-z) = -erf z.  Branch-free: with
// q = poly(t) e^{-x^2/2} (z = |x|/sqrt 2), 1 + erf(x/sqrt 2) = 2 - q for x >= 0
// and q for x < 0.
struct GeluAS {
  static constexpr float p = 0.3275911f, a1 = 0.254829592f, a2 = -0.284496736f, a3 = 1.421413741f,
                         a4 = -1.453152027f, a5 = 1.061405429f;
};
// 1 + erf(x / sqrt 2), and the Gaussian factor e^{-x^2/2} it used
__device__ __forceinline__ float one_plus_erf_s2(float x, float* gauss) {
  const float z = fabsf(x) * 0.70710678118654752f;
  const float t = __fdividef(1.f, fmaf(GeluAS::p, z, 1.f));
  const float poly =
      t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, GeluAS::a5, GeluAS::a4), GeluAS::a3), GeluAS::a2), GeluAS::a1);
  const float g = __expf(-0.5f * x * x);
  *gauss = g;
  const float q = poly * g;
  return x >= 0.f ? 2.f - q : q;
}
// Forward GELU with one MUFU operation: erf from Abramowitz & Stegun formula
// 7.1.28, erf z = 1 - (1 + a1 z + ... + a6 z^6)^-16 for z >= 0, |error| <=
// 3e-7 (about 2e-6 once evaluated in FP32 -- far below the BF16 rounding the
// activation gets next).  The exponential-based 7.1.26 form above costs two
// MUFU operations and stays in the derivative, which needs e^{-x^2/2} anyway.
struct GeluAS28 {
  static constexpr float a1 = 0.0705230784f, a2 = 0.0422820123f, a3 = 0.0092705272f, a4 = 0.0001520143f,
                         a5 = 0.0002765672f, a6 = 0.0000430638f;
};
__device__ __forceinline__ float gelu_f(float x) {
  const float z = fabsf(x) * 0.70710678118654752f;
  float p = fmaf(z, GeluAS28::a6, GeluAS28::a5);
  p = fmaf(p, z, GeluAS28::a4);
  p = fmaf(p, z, GeluAS28::a3);
  p = fmaf(p, z, GeluAS28::a2);
  p = fmaf(p, z, GeluAS28::a1);
  p = fmaf(p, z, 1.f);
  p *= p;
  p *= p;
  p *= p;
  p *= p;
  const float d = __fdividef(1.f, p);  // 1 - erf(|x|/sqrt 2)
  return 0.5f * x * (x >= 0.f ? 2.f - d : d);
}

// Two forward GELUs with the packed FP32x2 FMA/multiply of sm_100: the same
// operations in the same order as gelu_f on each half, so the results are
// identical, at half the FMA-pipe instructions.
__device__ __forceinline__ float2 gelu2_f(float2 x) {
  const float2 c = make_float2(0.70710678118654752f, 0.70710678118654752f);
  const float2 z = __fmul2_rn(make_float2(fabsf(x.x), fabsf(x.y)), c);
  float2 p = __ffma2_rn(z, make_float2(GeluAS28::a6, GeluAS28::a6), make_float2(GeluAS28::a5, GeluAS28::a5));
  p = __ffma2_rn(p, z, make_float2(GeluAS28::a4, GeluAS28::a4));
  p = __ffma2_rn(p, z, make_float2(GeluAS28::a3, GeluAS28::a3));
  p = __ffma2_rn(p, z, make_float2(GeluAS28::a2, GeluAS28::a2));
  p = __ffma2_rn(p, z, make_float2(GeluAS28::a1, GeluAS28::a1));
  p = __ffma2_rn(p, z, make_float2(1.f, 1.f));
  p = __fmul2_rn(p, p);
  p = __fmul2_rn(p, p);
  p = __fmul2_rn(p, p);
  p = __fmul2_rn(p, p);
  const float d0 = __fdividef(1.f, p.x), d1 = __fdividef(1.f, p.y);
  return make_float2(0.5f * x.x * (x.x >= 0.f ? 2.f - d0 : d0), 0.5f * x.y * (x.y >= 0.f ? 2.f - d1 : d1));
}
__device__ __forceinline__ uint32_t gelu_pack(float lo, float hi) {
  const float2 g = gelu2_f(make_float2(lo, hi));
  return pack_bf16(g.x, g.y);
}
__device__ __forceinline__ float gelu_d(float x) {
  float g;
  const float e = one_plus_erf_s2(x, &g);
  return 0.5f * e + x * 0.39894228040143268f * g;
}

// ReLU of two FP32 pre-activations, rounded to BF16 and packed (lo in the low
// half): one conversion instruction with the clamp built in.
__device__ __forceinline__ uint32_t relu_pack(float lo, float hi) {
  uint32_t d;
  asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}

// Activation, its derivative and the packed BF16 activation of two values.
template <int ACT>
__device__ __forceinline__ float act_f(float x) {
  if constexpr (ACT == kActRelu)
    return fmaxf(x, 0.f);
  else
    return gelu_f(x);
}
template <int ACT>
__device__ __forceinline__ float act_d(float x) {
  if constexpr (ACT == kActRelu)
    return x > 0.f ? 1.f : 0.f;
  else
    return gelu_d(x);
}
template <int ACT>
__device__ __forceinline__ uint32_t act_pack(float lo, float hi) {
  if constexpr (ACT == kActRelu)
    return relu_pack(lo, hi);
  else
    return gelu_pack(lo, hi);
}

// B fragment of a weight stored [n][k] row-major (ld = k stride) for the tile (k0, n0).
__device__ __forceinline__ void bfrag_nk(uint32_t* b, const __nv_bfloat16* W, int ld, int k0, int n0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  const __nv_bfloat16* r = W + (n0 + g) * ld + k0 + 2 * t;
  b[0] = pack_raw(r[0], r[1]);
  b[1] = pack_raw(r[8], r[9]);
}

// Warp-level forward pass of 16 points.  xa: A fragment of the normalised
// features (16 x 16, k 10..15 zero).  Returns y[4]: C fragment of the 16 x 8
// outputs (normalised; columns 6,7 unused).  If z1/z2 are given, the
// pre-activations are kept (for the backward pass).
template <int ACT, int H>
__device__ __forceinline__ void mlp_forward_warp(const MlpSmem<H>& s, const uint32_t* xa, float* y, float (*z1)[4],
                                                 float (*z2)[4]) {
  constexpr int NJ = H / 8, NK = H / 16;  // n-tiles of 8 and k-steps of 16 over the hidden width
  const int lane = threadIdx.x & 31, t = lane & 3;
  float h[NJ][4];
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    const float b0 = s.b1[8 * j + 2 * t], b1 = s.b1[8 * j + 2 * t + 1];
    h[j][0] = b0;
    h[j][1] = b1;
    h[j][2] = b0;
    h[j][3] = b1;
    uint32_t b[2];
    bfrag_nk(b, s.w1, 16, 0, 8 * j, lane);
    mma16816(h[j], xa, b);
  }
  uint32_t a[NK][4];
#pragma unroll
  for (int j = 0; j < NJ; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (z1) z1[j][e] = h[j][e];
      h[j][e] = act_f<ACT>(h[j][e]);
    }
#pragma unroll
  for (int kk = 0; kk < NK; ++kk) {
    a[kk][0] = pack_bf16(h[2 * kk][0], h[2 * kk][1]);
    a[kk][1] = pack_bf16(h[2 * kk][2], h[2 * kk][3]);
    a[kk][2] = pack_bf16(h[2 * kk + 1][0], h[2 * kk + 1][1]);
    a[kk][3] = pack_bf16(h[2 * kk + 1][2], h[2 * kk + 1][3]);
  }
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    const float b0 = s.b2[8 * j + 2 * t], b1 = s.b2[8 * j + 2 * t + 1];
    h[j][0] = b0;
    h[j][1] = b1;
    h[j][2] = b0;
    h[j][3] = b1;
#pragma unroll
    for (int kk = 0; kk < NK; ++kk) {
      uint32_t b[2];
      bfrag_nk(b, s.w2, H, 16 * kk, 8 * j, lane);
      mma16816(h[j], a[kk], b);
    }
  }
#pragma unroll
  for (int j = 0; j < NJ; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (z2) z2[j][e] = h[j][e];
      h[j][e] = act_f<ACT>(h[j][e]);
    }
#pragma unroll
  for (int kk = 0; kk < NK; ++kk) {
    a[kk][0] = pack_bf16(h[2 * kk][0], h[2 * kk][1]);
    a[kk][1] = pack_bf16(h[2 * kk][2], h[2 * kk][3]);
    a[kk][2] = pack_bf16(h[2 * kk + 1][0], h[2 * kk + 1][1]);
    a[kk][3] = pack_bf16(h[2 * kk + 1][2], h[2 * kk + 1][3]);
  }
  const float c0 = s.b3[2 * t], c1 = s.b3[2 * t + 1];
  y[0] = c0;
  y[1] = c1;
  y[2] = c0;
  y[3] = c1;
#pragma unroll
  for (int kk = 0; kk < NK; ++kk) {
    uint32_t b[2];
    bfrag_nk(b, s.w3, H, 16 * kk, 0, lane);
    mma16816(y, a[kk], b);
  }
}

// Inference copy of the network: B fragments of W1, W2, W3 stored in the order
// the m16n8k16 B operand is consumed (tile-major, then lane), so each lane
// fetches its two registers of a tile with one conflict-free 64-bit load.
//   f1[j][lane]      W1 tile (k 0..15, n 8j..8j+7)
//   f2[kk][j][lane]  W2 tile (k 16kk.., n 8j..)
//   f3[kk][lane]     W3 tile (k 16kk.., n 0..7)
template <int H>
struct MlpFwdSmem {
  uint2 f1[(H / 8) * 32];
  uint2 f2[(H / 16) * (H / 8) * 32];
  uint2 f3[(H / 16) * 32];
  float b1[H], b2[H], b3[8];
  float xmean[16], xistd[16], ymean[8], ystd[8];
};

// One B-fragment register pair of the [n][k] row-major FP32 weight W (k < kin,
// n < nout valid; zero elsewhere) for tile (k0, n0) and lane.
__device__ __forceinline__ uint2 bfrag_from_f32(const float* __restrict__ W, int kin, int nout, int k0, int n0,
                                                int lane) {
  const int g = lane >> 2, t = lane & 3;
  const int n = n0 + g;
  float v[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int k = k0 + 2 * t + (e & 1) + (e >> 1) * 8;
    v[e] = (n < nout && k < kin) ? W[n * kin + k] : 0.f;
  }
  return make_uint2(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]));
}

template <int H>
__device__ __forceinline__ void mlp_stage_fwd(MlpFwdSmem<H>& s, const float* __restrict__ P,
                                              const float* __restrict__ nrm) {
  using L = MlpLayout<H>;
  constexpr int NJ = H / 8, NK = H / 16;
  for (int i = threadIdx.x; i < NJ * 32; i += blockDim.x)
    s.f1[i] = bfrag_from_f32(P + L::W1, kMlpIn, H, 0, 8 * (i >> 5), i & 31);
  for (int i = threadIdx.x; i < NK * NJ * 32; i += blockDim.x) {
    const int tile = i >> 5, kk = tile / NJ, j = tile - kk * NJ;
    s.f2[i] = bfrag_from_f32(P + L::W2, H, H, 16 * kk, 8 * j, i & 31);
  }
  for (int i = threadIdx.x; i < NK * 32; i += blockDim.x)
    s.f3[i] = bfrag_from_f32(P + L::W3, H, kMlpOut, 16 * (i >> 5), 0, i & 31);
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    s.b1[i] = P[L::B1 + i];
    s.b2[i] = P[L::B2 + i];
  }
  if (threadIdx.x < 16) {
    s.xmean[threadIdx.x] = threadIdx.x < kMlpIn ? nrm[threadIdx.x] : 0.f;
    s.xistd[threadIdx.x] = threadIdx.x < kMlpIn ? nrm[kMlpIn + threadIdx.x] : 0.f;
  }
  if (threadIdx.x < 8) {
    s.b3[threadIdx.x] = threadIdx.x < kMlpOut ? P[L::B3 + threadIdx.x] : 0.f;
    s.ymean[threadIdx.x] = threadIdx.x < kMlpOut ? nrm[2 * kMlpIn + threadIdx.x] : 0.f;
    s.ystd[threadIdx.x] = threadIdx.x < kMlpOut ? nrm[2 * kMlpIn + kMlpOut + threadIdx.x] : 0.f;
  }
}

// Forward pass of 16 points from the fragment-ordered weights; same
// arithmetic as mlp_forward_warp (BF16 operands, FP32 accumulation, the
// activation on the FP32 pre-activations, BF16 rounding of the activations).
template <int ACT, int H>
__device__ __forceinline__ void mlp_forward_fast(const MlpFwdSmem<H>& s, const uint32_t* xa, float* y) {
  constexpr int NJ = H / 8, NK = H / 16;
  const int lane = threadIdx.x & 31, t = lane & 3;
  float h[NJ][4];
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    const float b0 = s.b1[8 * j + 2 * t], b1 = s.b1[8 * j + 2 * t + 1];
    h[j][0] = b0;
    h[j][1] = b1;
    h[j][2] = b0;
    h[j][3] = b1;
    const uint2 bb = s.f1[j * 32 + lane];
    const uint32_t b[2] = {bb.x, bb.y};
    mma16816(h[j], xa, b);
  }
  uint32_t a[NK][4];
#pragma unroll
  for (int kk = 0; kk < NK; ++kk) {
    a[kk][0] = act_pack<ACT>(h[2 * kk][0], h[2 * kk][1]);
    a[kk][1] = act_pack<ACT>(h[2 * kk][2], h[2 * kk][3]);
    a[kk][2] = act_pack<ACT>(h[2 * kk + 1][0], h[2 * kk + 1][1]);
    a[kk][3] = act_pack<ACT>(h[2 * kk + 1][2], h[2 * kk + 1][3]);
  }
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    const float b0 = s.b2[8 * j + 2 * t], b1 = s.b2[8 * j + 2 * t + 1];
    h[j][0] = b0;
    h[j][1] = b1;
    h[j][2] = b0;
    h[j][3] = b1;
  }
#pragma unroll
  for (int kk = 0; kk < NK; ++kk)
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      const uint2 bb = s.f2[(kk * NJ + j) * 32 + lane];
      const uint32_t b[2] = {bb.x, bb.y};
      mma16816(h[j], a[kk], b);
    }
#pragma unroll
  for (int kk = 0; kk < NK; ++kk) {
    a[kk][0] = act_pack<ACT>(h[2 * kk][0], h[2 * kk][1]);
    a[kk][1] = act_pack<ACT>(h[2 * kk][2], h[2 * kk][3]);
    a[kk][2] = act_pack<ACT>(h[2 * kk + 1][0], h[2 * kk + 1][1]);
    a[kk][3] = act_pack<ACT>(h[2 * kk + 1][2], h[2 * kk + 1][3]);
  }
  const float c0 = s.b3[2 * t], c1 = s.b3[2 * t + 1];
  y[0] = c0;
  y[1] = c1;
  y[2] = c0;
  y[3] = c1;
#pragma unroll
  for (int kk = 0; kk < NK; ++kk) {
    const uint2 bb = s.f3[kk * 32 + lane];
    const uint32_t b[2] = {bb.x, bb.y};
    mma16816(y, a[kk], b);
  }
}

// A fragment of normalised features for 16 points; feat(r, f) returns the raw
// feature f (< 10) of row r (< 16) of this warp's tile.
template <class S, class F>
__device__ __forceinline__ void mlp_xfrag(const S& s, uint32_t* xa, F feat) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float v[8];
  const int rows[2] = {g, g + 8};
#pragma unroll
  for (int hr = 0; hr < 2; ++hr)
#pragma unroll
    for (int hk = 0; hk < 2; ++hk)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int f = 2 * t + 8 * hk + e;
        v[hr * 4 + hk * 2 + e] = f < kMlpIn ? (feat(rows[hr], f) - s.xmean[f]) * s.xistd[f] : 0.f;
      }
  xa[0] = pack_bf16(v[0], v[1]);  // row g,   k 2t..2t+1
  xa[1] = pack_bf16(v[4], v[5]);  // row g+8, k 2t..2t+1
  xa[2] = pack_bf16(v[2], v[3]);  // row g,   k 2t+8..
  xa[3] = pack_bf16(v[6], v[7]);  // row g+8, k 2t+8..
}

}  // namespace psb
