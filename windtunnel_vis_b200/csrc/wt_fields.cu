// wt_fields.cu — derived flow fields and the strided field export.
//
//   k_derive ... vorticity and Q-criterion from central differences of the half4 velocity field,
//                Q faded out within two cells of a solid, turbulence intensity from the EMA
//                statistics, binary16 copy of the mean field (src/solver/wgslLbm.ts:527-592)
//   k_export ... every stride-th cell (clamped to the last cell) of velocity, mean and vorticity
//                as three float4 arrays (the export pass of src/solver/SolverGPU.ts:374-425)
//
// One thread per cell along x-rows; the velocity stencil (six neighbours) and the solid flags two
// cells out along each axis are read through L1/L2, all of a cell's loads issued before its
// arithmetic; the kernel streams 8 + 16 + 4 + 4 B in and 24 B out per cell. Compiled without FMA
// contraction: every output is bit-identical to the oracle's f32 restatement.
#include <cuda_fp16.h>

#include <algorithm>

#include "wt_internal.h"

namespace wt {
namespace {

__device__ __forceinline__ float3 vel_at(const uint2* __restrict__ vel, int x, int y, int z, int NX, int NY,
                                         int NZ) {
  x = min(max(x, 0), NX - 1);
  y = min(max(y, 0), NY - 1);
  z = min(max(z, 0), NZ - 1);
  const uint2 v = __ldg(vel + (size_t)x + (size_t)NX * ((size_t)y + (size_t)NY * (size_t)z));
  const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&v.x));
  const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&v.y));
  return make_float3(a.x, a.y, b.x);
}

__device__ __forceinline__ uint2 pack_half4(float a, float b, float c, float d) {
  __half2 h0 = __floats2half2_rn(a, b), h1 = __floats2half2_rn(c, d);
  return make_uint2(*reinterpret_cast<uint32_t*>(&h0), *reinterpret_cast<uint32_t*>(&h1));
}

__device__ __forceinline__ float4 unpack_half4(uint2 v) {
  const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&v.x));
  const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&v.y));
  return make_float4(a.x, a.y, b.x, b.y);
}

// the solid flag of cell (x, y, z), false outside the grid; the load is always issued (from a
// clamped address) so that all of a cell's stencil loads are in flight together
__device__ __forceinline__ bool solid_near(const uint32_t* __restrict__ flags, int x, int y, int z, int NX, int NY,
                                           int NZ) {
  const bool in = x >= 0 && y >= 0 && z >= 0 && x < NX && y < NY && z < NZ;
  const int cx = min(max(x, 0), NX - 1), cy = min(max(y, 0), NY - 1), cz = min(max(z, 0), NZ - 1);
  return in && __ldg(flags + (size_t)cx + (size_t)NX * ((size_t)cy + (size_t)NY * (size_t)cz)) != 0u;
}

template <int DIM>
__global__ void __launch_bounds__(256) k_derive(const __grid_constant__ wt_kparams P, const uint2* __restrict__ vel,
                                                const uint32_t* __restrict__ flags,
                                                const float4* __restrict__ meanA, const float* __restrict__ meanB,
                                                uint2* __restrict__ vort, uint2* __restrict__ stat,
                                                uint2* __restrict__ mean) {
  const int NX = P.nx, NY = P.ny, NZ = P.nz;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z;
  if (x >= NX) return;
  const size_t idx = (size_t)x + (size_t)NX * ((size_t)y + (size_t)NY * (size_t)z);
  // every load of the cell first (the stencil's velocities and flags, the EMA statistics), then the
  // arithmetic: no load waits behind a branch on another
  const bool solid = __ldg(flags + idx) != 0u;
  const float4 m = __ldg(meanA + idx);
  const float mb = __ldg(meanB + idx);
  const float3 xp = vel_at(vel, x + 1, y, z, NX, NY, NZ), xm = vel_at(vel, x - 1, y, z, NX, NY, NZ);
  const float3 yp = vel_at(vel, x, y + 1, z, NX, NY, NZ), ym = vel_at(vel, x, y - 1, z, NX, NY, NZ);
  float3 zp = make_float3(0.f, 0.f, 0.f), zm = zp;
  if (DIM == 3) zp = vel_at(vel, x, y, z + 1, NX, NY, NZ), zm = vel_at(vel, x, y, z - 1, NX, NY, NZ);
  bool hit[2][3];  // a solid d cells away along axis a, either side
#pragma unroll
  for (int d = 1; d <= 2; d++)
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const int ex = a == 0 ? d : 0, ey = a == 1 ? d : 0, ez = a == 2 ? d : 0;
      hit[d - 1][a] = a < DIM && (solid_near(flags, x + ex, y + ey, z + ez, NX, NY, NZ) |
                                  solid_near(flags, x - ex, y - ey, z - ez, NX, NY, NZ));
    }
  float4 vo = make_float4(0.f, 0.f, 0.f, 0.f);
  if (!solid) {
    float J[3][3];  // J[j][i] = d u_i / d x_j
    J[0][0] = 0.5f * (xp.x - xm.x);
    J[0][1] = 0.5f * (xp.y - xm.y);
    J[0][2] = 0.5f * (xp.z - xm.z);
    J[1][0] = 0.5f * (yp.x - ym.x);
    J[1][1] = 0.5f * (yp.y - ym.y);
    J[1][2] = 0.5f * (yp.z - ym.z);
    if (DIM == 3) {
      J[2][0] = 0.5f * (zp.x - zm.x);
      J[2][1] = 0.5f * (zp.y - zm.y);
      J[2][2] = 0.5f * (zp.z - zm.z);
    } else {
      J[2][0] = J[2][1] = J[2][2] = 0.0f;
    }
    const float wx = J[1][2] - J[2][1];
    const float wy = J[2][0] - J[0][2];
    const float wz = J[0][1] - J[1][0];
    float S2 = 0.0f, W2 = 0.0f;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) {
        const float s = 0.5f * (J[j][i] + J[i][j]);
        const float w = 0.5f * (J[j][i] - J[i][j]);
        S2 += s * s;
        W2 += w * w;
      }
    // fade Q out within two cells of a solid (wall shear of the staircase surface)
    float near = 0.0f;
#pragma unroll
    for (int d = 1; d <= 2; d++)
#pragma unroll
      for (int a = 0; a < DIM; a++)
        if (hit[d - 1][a]) near = fmaxf(near, d == 1 ? 1.0f : 0.5f);
    vo = make_float4(wx, wy, wz, 0.5f * (W2 - S2) * (1.0f - near));
  }
  const float k = fmaxf(mb - (m.x * m.x + m.y * m.y + m.z * m.z), 0.0f);
  const float ti = sqrtf(k / 3.0f) / fmaxf(P.u_ref, 1e-6f);
  vort[idx] = pack_half4(vo.x, vo.y, vo.z, vo.w);
  stat[idx] = pack_half4(solid ? 0.0f : ti, solid ? 1.0f : 0.0f, 0.0f, 0.0f);
  mean[idx] = pack_half4(m.x, m.y, m.z, m.w);
}

__global__ void __launch_bounds__(256) k_export(int NX, int NY, int NZ, int stride, int ox, int oy, int oz,
                                                const uint2* __restrict__ vel, const uint2* __restrict__ mean,
                                                const uint2* __restrict__ vort, float4* __restrict__ vel_out,
                                                float4* __restrict__ mean_out, float4* __restrict__ vort_out) {
  const int64_t n = (int64_t)ox * oy * oz;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int gx = (int)(i % ox);
    const int gy = (int)((i / ox) % oy);
    const int gz = (int)(i / ((int64_t)ox * oy));
    const int px = min(gx * stride, NX - 1), py = min(gy * stride, NY - 1), pz = min(gz * stride, NZ - 1);
    const size_t c = (size_t)px + (size_t)NX * ((size_t)py + (size_t)NY * (size_t)pz);
    vel_out[i] = unpack_half4(__ldg(vel + c));
    mean_out[i] = unpack_half4(__ldg(mean + c));
    vort_out[i] = unpack_half4(__ldg(vort + c));
  }
}

__global__ void __launch_bounds__(256) k_widen(const uint2* __restrict__ src, float4* __restrict__ dst, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = unpack_half4(__ldg(src + i));
}

}  // namespace

cudaError_t launch_derive(wt_solver* s) {
  const int NX = s->dims.nx;
  const int bx = NX >= 256 ? 256 : ((NX + 31) / 32) * 32;
  const dim3 grid((NX + bx - 1) / bx, s->dims.ny, s->dims.nz);
  if (s->is3d)
    k_derive<3><<<grid, bx, 0, s->stream>>>(s->kp, s->vel, s->flags, s->meanA, s->meanB, s->dvort, s->dstat,
                                              s->dmean);
  else
    k_derive<2><<<grid, bx, 0, s->stream>>>(s->kp, s->vel, s->flags, s->meanA, s->meanB, s->dvort, s->dstat,
                                              s->dmean);
  s->launches++;
  return cudaGetLastError();
}

cudaError_t launch_export(wt_solver* s, int stride, int ox, int oy, int oz, float4* out) {
  // out: three consecutive arrays of ox * oy * oz float4 (velocity, mean, vorticity)
  const int64_t n = (int64_t)ox * oy * oz;
  const unsigned blocks = (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16);
  k_export<<<blocks, 256, 0, s->stream>>>(s->dims.nx, s->dims.ny, s->dims.nz, stride, ox, oy, oz, s->vel, s->dmean,
                                          s->dvort, out, out + n, out + 2 * n);
  s->launches++;
  return cudaGetLastError();
}

cudaError_t launch_widen_half4(wt_solver* s, const uint2* src, float4* dst, size_t n) {
  const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_widen<<<blocks, 256, 0, s->stream>>>(src, dst, n);
  s->launches++;
  return cudaGetLastError();
}

}  // namespace wt
