// wt_closure.cuh — the learned LES closure shared by the stream-collide kernels (wt_lbm.cu) and
// the trainer (wt_closure.cu): per-cell features, the network's arithmetic, and the device-side
// copy of a network.
//
// The network (10 -> 32 -> 32 -> 1) and its numerics:
//   x'  = bf16(fma(x, scale, nshift)),  nshift = -shift * scale (f32)      inputs, padded to 16
//   z1  = x' W1 + b1,  h1 = bf16(gelu(z1))                                 W1 rounded to bf16
//   z2  = h1 W2 + b2,  h2 = gelu(z2) (f32: it feeds only the CUDA-core      f32 accumulation
//                                     output layer)
//   z3  = (sum_even h2_j w3_j + sum_odd h2_j w3_j) + b3,  nu_t = nu_scale * softplus(z3)
//   gelu(x) = x * (1/2 + tanh(u) / 2),  u = x (C0 + C1 x^2),  C0 = sqrt(2/pi), C1 = 0.044715 C0
//             (the tanh form of gelu; tanh.approx.f32)
// The two 32-wide layers run on tcgen05 tensor cores in the bulk kernel, in the row pass that
// serves the face rows and wall cells, and in the trainer.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>
#include <string.h>

#include "../../include/wt.h"
#include "wt_umma.cuh"

namespace wt {

constexpr int CL_IN = WT_CLOSURE_IN;    // 10 features
constexpr int CL_K1 = 16;               // layer-1 K, padded for the K = 16 MMA step
constexpr int CL_H = WT_CLOSURE_HID;    // 32 hidden units
constexpr int CL_NPARAM = CL_IN * CL_H + CL_H + CL_H * CL_H + CL_H + CL_H + 1;  // 1441 trainable values
constexpr float GELU_C0 = 0.7978845608028654f;
constexpr float GELU_C1 = 0.035677408136300125f;
constexpr float GELU_C1x3 = 0.10703222440890037f;

// The small per-network values: biases, the bf16-rounded output weights, the input normalisation
// as fma(x, scale, nshift). The bulk kernel takes them by value (constant bank).
struct ClosureParams {
  float b1[CL_H];
  float b2[CL_H];
  float w3[CL_H];
  float b3, nu_scale;
  float scale[CL_IN];
  float nshift[CL_IN];
};

// Device copy of a network's weight images, the tcgen05 B operands (N x K, K-major, no swizzle):
// w1img[n = hidden j][k = input], w2img[n = out j][k = in i] (forward), w2timg[n = in i][k = out j]
// (the dH1 = dZ2 W2^T product of the backward pass).
struct __align__(128) ClosureDev {
  uint16_t w1img[CL_H * CL_K1];
  uint16_t w2img[CL_H * CL_H];
  uint16_t w2timg[CL_H * CL_H];
};

// bf16 round to nearest even (finite inputs), as a float and as raw bits
__host__ __device__ __forceinline__ uint16_t bf16_bits(float v) {
#if defined(__CUDA_ARCH__)
  return __bfloat16_as_ushort(__float2bfloat16_rn(v));
#else
  uint32_t u;
  memcpy(&u, &v, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
#endif
}
__host__ __device__ __forceinline__ float bf16_val(uint16_t b) {
  const uint32_t u = (uint32_t)b << 16;
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}
__host__ __device__ __forceinline__ float bf16r(float v) { return bf16_val(bf16_bits(v)); }

// two floats -> bf16x2 bits (lo = a), one cvt.rn.bf16x2.f32
__device__ __forceinline__ uint32_t bf16x2_bits(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ float2 bf16x2_vals(uint32_t w) {
  return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xFFFF0000u));
}

__device__ __forceinline__ float tanh_fast(float x) {
  float r;
  asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// gelu, tanh form, as (x + x tanh(u)) / 2 with one fma; explicit roundings so every kernel
// evaluates it identically
__device__ __forceinline__ float cl_gelu(float x) {
  const float u = __fmul_rn(x, __fmaf_rn(GELU_C1, __fmul_rn(x, x), GELU_C0));
  return __fmul_rn(0.5f, __fmaf_rn(x, tanh_fast(u), x));
}
// twice gelu on two lanes with f32x2 instructions: x + x tanh(u), the same per-lane roundings as
// cl_gelu without its exact halving. The inference kernels fold the 1/2 into the next layer's
// weights (the bf16 W2 image and w3 are stored halved), which leaves every product unchanged.
__device__ __forceinline__ float2 cl_gelu2x(float2 x) {
  const float2 u = __fmul2_rn(x, __ffma2_rn(make_float2(GELU_C1, GELU_C1), __fmul2_rn(x, x),
                                            make_float2(GELU_C0, GELU_C0)));
  const float2 t = make_float2(tanh_fast(u.x), tanh_fast(u.y));
  return __ffma2_rn(x, t, x);
}
// gelu and its derivative d = q + (x/2)(1 - t^2)(C0 + 3 C1 x^2), q = 1/2 + t/2
__device__ __forceinline__ float cl_gelu_d(float x, float& d) {
  const float x2 = __fmul_rn(x, x);
  const float t = tanh_fast(__fmul_rn(x, __fmaf_rn(GELU_C1, x2, GELU_C0)));
  const float q = __fmaf_rn(0.5f, t, 0.5f);
  const float du = __fmaf_rn(GELU_C1x3, x2, GELU_C0);
  d = __fmaf_rn(__fmul_rn(__fmul_rn(0.5f, x), __fmaf_rn(-t, t, 1.0f)), du, q);
  return __fmul_rn(0.5f, __fmaf_rn(x, t, x));
}
// softplus(z) = max(z, 0) + log1p(e), e = exp(-|z|) in (0, 1], from the fast exponential; log1p
// from its Taylor series e - e^2/2 + e^3/3 - e^4/4 below e = 1/32 (truncation under 2e-7 of the
// result), else the fast logarithm of 1 + e (absolute error near 4e-7 on a result of at least 0.03)
__device__ __forceinline__ float cl_softplus(float z) {
  const float e = __expf(-fabsf(z));
  const float l = e < 0.03125f
                      ? e * __fmaf_rn(e, __fmaf_rn(e, __fmaf_rn(e, -0.25f, 0.333333343f), -0.5f), 1.0f)
                      : __logf(1.0f + e);
  return fmaxf(z, 0.0f) + l;
}
__device__ __forceinline__ float cl_sigmoid(float z) { return 1.0f / (1.0f + expf(-z)); }

__device__ __forceinline__ float cl_sqrt(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// wall-distance feature from the sdf word of a cell (~bits(d), 0 = unknown)
__device__ __forceinline__ float cl_wall_dist(uint32_t s) {
  return s == 0u ? WT_CLOSURE_WALL_CAP : fminf(__uint_as_float(~s), WT_CLOSURE_WALL_CAP);
}

// the 10 features of a cell from its moments: non-equilibrium stress Pi (lattice units), density,
// velocity, the handle's molecular tau0 and the wall distance. |S| is the strain rate the
// Smagorinsky relation assigns to |Pi| at Cs = WT_CLOSURE_FEATURE_CS:
//   tau_s = (tau0 + sqrt(tau0^2 + 18 sqrt(2) Cs^2 |Pi| / rho)) / 2,  |S| = 3 |Pi| / (sqrt(2) rho tau_s)
// (approximate square roots and quotients: the features are network inputs, not conserved
// quantities)
__device__ __forceinline__ void cl_features(float pxx, float pyy, float pzz, float pxy, float pxz, float pyz,
                                            float rho, float ux, float uy, float uz, float tau0, float wall_d,
                                            float (&x)[CL_IN]) {
  float pn = __fmaf_rn(pxx, pxx, __fmaf_rn(pyy, pyy, __fmul_rn(pzz, pzz)));
  pn = __fmaf_rn(2.0f, __fmaf_rn(pxy, pxy, __fmaf_rn(pxz, pxz, __fmul_rn(pyz, pyz))), pn);
  const float piN = cl_sqrt(pn);
  const float k = (float)(18.0 * 1.4142135623730951) * (WT_CLOSURE_FEATURE_CS * WT_CLOSURE_FEATURE_CS);
  const float ts = 0.5f * (tau0 + cl_sqrt(__fmaf_rn(tau0, tau0, __fdividef(k * piN, rho))));
  x[0] = pxx;
  x[1] = pyy;
  x[2] = pzz;
  x[3] = pxy;
  x[4] = pxz;
  x[5] = pyz;
  x[6] = __fdividef(2.1213203435596424f * piN, rho * ts);
  x[7] = wall_d;
  x[8] = rho;
  x[9] = cl_sqrt(__fmaf_rn(ux, ux, __fmaf_rn(uy, uy, __fmul_rn(uz, uz))));
}

// the by-value part of a network
__host__ __device__ inline ClosureParams closure_params(const wt_closure& c) {
  ClosureParams p;
  for (int j = 0; j < CL_H; j++) {
    p.b1[j] = c.b1[j];
    p.b2[j] = c.b2[j];
    p.w3[j] = 0.5f * bf16r(c.w3[j]);  // halved: the kernels' hidden layers hold twice gelu
  }
  p.b3 = c.b3;
  p.nu_scale = c.nu_scale;
  for (int k = 0; k < CL_IN; k++) {
    p.scale[k] = c.scale[k];
    p.nshift[k] = -(c.shift[k] * c.scale[k]);
  }
  return p;
}

// fills the bf16 images of `c` into `d` (host or device)
__host__ __device__ inline void closure_pack(const wt_closure& c, ClosureDev& d) {
  for (int j = 0; j < CL_H; j++)
    for (int k = 0; k < CL_K1; k++) {
      const float v = k < CL_IN ? c.w1[k][j] : 0.0f;
      d.w1img[umma::kmaj_off(j, k, CL_K1) / 2] = bf16_bits(v);
    }
  for (int i = 0; i < CL_H; i++)
    for (int j = 0; j < CL_H; j++) {
      // bf16(w / 2) = bf16(w) / 2: the forward image is halved like w3
      d.w2img[umma::kmaj_off(j, i, CL_H) / 2] = bf16_bits(0.5f * c.w2[i][j]);
      d.w2timg[umma::kmaj_off(i, j, CL_H) / 2] = bf16_bits(c.w2[i][j]);
    }
}

}  // namespace wt
