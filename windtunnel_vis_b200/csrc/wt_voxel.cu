// wt_voxel.cu — GPU triangle voxelizer for sm_100a: solid flags, wall distances and frontal
// projection from an indexed triangle mesh (the reference's VoxelizerGPU, src/voxelize/
// VoxelizerGPU.ts:48-151, kernels src/voxelize/wgslVoxel.ts:33-322).
//
// Algorithm (same as the reference): signed ray crossings along x, y and z (winding numbers) ->
// per-axis inside votes -> a thin 6-separating surface shell -> 2-of-3 vote with shell-only
// cells kept where no neighbour owns an interior vote -> exact point-triangle distances of cell
// centres within 2.5 cells (min via atomicMax of ~bits) -> wheel tags -> frontal projection.
//
// Work mapping differs from the reference for the B200: one warp per triangle (lanes stride over
// the triangle's cell columns or surface samples) instead of one thread per triangle, warp
// prefix scans along x, coalesced column walks along y and z, and a warp per (y, z) column for
// the projection. Integer atomics make every result independent of execution order.
//
// This translation unit is compiled with -fmad=false: every f32 expression is evaluated
// operation by operation, so the flags are bit-identical to the f32 CPU restatement.
#include <climits>

#include "wt_internal.h"

namespace wt {
namespace {

struct VP {
  float M[16];
  int nx, ny, nz;
  size_t n;
  __device__ __forceinline__ int dim_of(int a) const { return a == 0 ? nx : (a == 1 ? ny : nz); }
  __device__ __forceinline__ size_t cell(uint32_t x, uint32_t y, uint32_t z) const {
    return (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z);
  }
};

__device__ __forceinline__ float3 vtx(const VP& V, const float* __restrict__ pos, const uint32_t* __restrict__ idx,
                                      size_t i) {
  const uint32_t k = idx[i];
  const float x = pos[3 * (size_t)k], y = pos[3 * (size_t)k + 1], z = pos[3 * (size_t)k + 2];
  return make_float3(V.M[0] * x + V.M[4] * y + V.M[8] * z + V.M[12], V.M[1] * x + V.M[5] * y + V.M[9] * z + V.M[13],
                     V.M[2] * x + V.M[6] * y + V.M[10] * z + V.M[14]);
}

__device__ __forceinline__ float comp(float3 p, int a) { return a == 0 ? p.x : (a == 1 ? p.y : p.z); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 mul3(float3 a, float k) { return make_float3(a.x * k, a.y * k, a.z * k); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len3(float3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

constexpr int WARPS = 8;  // warps per block for the per-triangle kernels

// 1. signed crossings (wgslVoxel.ts:33-94)
__global__ void __launch_bounds__(WARPS * 32) k_crossings(const VP V, const float* __restrict__ pos,
                                                          const uint32_t* __restrict__ idx, int64_t ntri,
                                                          int32_t* __restrict__ hits) {
  const int lane = threadIdx.x & 31;
  for (int64_t t = (int64_t)blockIdx.x * WARPS + (threadIdx.x >> 5); t < ntri; t += (int64_t)gridDim.x * WARPS) {
    const float3 p0 = vtx(V, pos, idx, 3 * t), p1 = vtx(V, pos, idx, 3 * t + 1), p2 = vtx(V, pos, idx, 3 * t + 2);
    for (int a = 0; a < 3; a++) {
      const int ua = (a + 1) % 3, va = (a + 2) % 3;
      const float Ax = comp(p0, ua), Ay = comp(p0, va), Bx = comp(p1, ua), By = comp(p1, va), Cx = comp(p2, ua),
                  Cy = comp(p2, va);
      const float area = (Bx - Ax) * (Cy - Ay) - (By - Ay) * (Cx - Ax);
      if (fabsf(area) < 1e-12f) continue;
      const int sgn = area > 0.0f ? -1 : 1;
      const int nu = V.dim_of(ua), nv = V.dim_of(va), na = V.dim_of(a);
      const float lox = fminf(fminf(Ax, Bx), Cx), loy = fminf(fminf(Ay, By), Cy);
      const float hix = fmaxf(fmaxf(Ax, Bx), Cx), hiy = fmaxf(fmaxf(Ay, By), Cy);
      const int u0 = max((int)ceilf(lox - 0.5f), 0), u1 = min((int)floorf(hix - 0.5f), nu - 1);
      const int v0 = max((int)ceilf(loy - 0.5f), 0), v1 = min((int)floorf(hiy - 0.5f), nv - 1);
      if (u1 < u0 || v1 < v0) continue;
      const float ha = comp(p0, a), hb = comp(p1, a), hc = comp(p2, a);
      const float inv = 1.0f / area;
      const int nvv = v1 - v0 + 1;
      const int64_t cols = (int64_t)(u1 - u0 + 1) * nvv;
      for (int64_t k = lane; k < cols; k += 32) {
        const int iu = u0 + (int)(k / nvv), iv = v0 + (int)(k % nvv);
        const float Px = (float)iu + 0.5f + 1.37e-4f, Py = (float)iv + 0.5f + 2.71e-4f;
        const float w0 = ((Bx - Px) * (Cy - Py) - (By - Py) * (Cx - Px)) * inv;
        const float w1 = ((Cx - Px) * (Ay - Py) - (Cy - Py) * (Ax - Px)) * inv;
        const float w2 = 1.0f - w0 - w1;
        if (w0 < 0.0f || w1 < 0.0f || w2 < 0.0f) continue;
        const float h = w0 * ha + w1 * hb + w2 * hc;
        int kk = (int)floorf(h - 0.5f) + 1;
        if (kk >= na) continue;
        kk = max(kk, 0);
        const size_t c = a == 0 ? V.cell(kk, iu, iv) : (a == 1 ? V.cell(iv, kk, iu) : V.cell(iu, iv, kk));
        atomicAdd(&hits[(size_t)a * V.n + c], sgn);
      }
    }
  }
}

// 2a. scan along x: one warp per (y, z) row, warp-wide inclusive prefix sums with a carry
__global__ void __launch_bounds__(256) k_scan_x(const VP V, const int32_t* __restrict__ hits, uint32_t* __restrict__ vote) {
  const int lane = threadIdx.x & 31;
  const int64_t rows = (int64_t)V.ny * V.nz;
  for (int64_t r = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5); r < rows; r += (int64_t)gridDim.x * 8) {
    const size_t base = (size_t)r * V.nx;
    int32_t carry = 0;
    for (int x0 = 0; x0 < V.nx; x0 += 32) {
      const int x = x0 + lane;
      int32_t v = x < V.nx ? hits[base + x] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
      }
      const int32_t s = carry + v;
      if (x < V.nx && s != 0) vote[base + x] |= 1u;
      carry += __shfl_sync(0xffffffffu, v, 31);
    }
  }
}

// 2b. scan along y (axis 1) or z (axis 2): one thread per column, consecutive threads on
// consecutive x so each step of the walk is a coalesced row access
__global__ void __launch_bounds__(256) k_scan_yz(const VP V, int axis, const int32_t* __restrict__ hits,
                                                 uint32_t* __restrict__ vote) {
  const int64_t other = axis == 1 ? V.nz : V.ny;
  const int64_t cols = (int64_t)V.nx * other;
  const size_t stride = axis == 1 ? (size_t)V.nx : (size_t)V.nx * V.ny;
  const int na = axis == 1 ? V.ny : V.nz;
  const uint32_t bit = 1u << axis;
  const int32_t* h = hits + (size_t)axis * V.n;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(c % V.nx);
    const int o = (int)(c / V.nx);
    size_t id = axis == 1 ? V.cell(x, 0, o) : V.cell(x, o, 0);
    int32_t s = 0;
    for (int k = 0; k < na; k++, id += stride) {
      s += h[id];
      if (s != 0) vote[id] |= bit;
    }
  }
}

// 3. surface shell (wgslVoxel.ts:126-170)
__global__ void __launch_bounds__(WARPS * 32) k_surface(const VP V, const float* __restrict__ pos,
                                                        const uint32_t* __restrict__ idx, int64_t ntri,
                                                        uint32_t* __restrict__ vote) {
  const int lane = threadIdx.x & 31;
  for (int64_t t = (int64_t)blockIdx.x * WARPS + (threadIdx.x >> 5); t < ntri; t += (int64_t)gridDim.x * WARPS) {
    const float3 p0 = vtx(V, pos, idx, 3 * t);
    const float3 e1 = sub3(vtx(V, pos, idx, 3 * t + 1), p0);
    const float3 e2 = sub3(vtx(V, pos, idx, 3 * t + 2), p0);
    const float m = fmaxf(fmaxf(len3(e1), len3(e2)), len3(sub3(e2, e1)));
    const uint32_t steps = (uint32_t)fminf(fmaxf(ceilf(m / 0.4f), 1.0f), 384.0f);
    const float fs = (float)steps;
    const float3 cr = cross3(e1, e2);
    const float cl = len3(cr);
    if (cl < 1e-12f) continue;
    const float3 nrm = make_float3(cr.x / cl, cr.y / cl, cr.z / cl);
    const float tol = 0.5f * fmaxf(fmaxf(fabsf(nrm.x), fabsf(nrm.y)), fabsf(nrm.z));
    const bool is2D = V.nz == 1;
    for (uint32_t i = 0; i <= steps; i++) {
      for (uint32_t j = lane; j <= steps - i; j += 32) {
        const float3 p = add3(add3(p0, mul3(e1, (float)i / fs)), mul3(e2, (float)j / fs));
        if (p.x < 0.0f || p.y < 0.0f || p.z < 0.0f || p.x >= (float)V.nx || p.y >= (float)V.ny || p.z >= (float)V.nz) continue;
        const float3 c = make_float3(floorf(p.x), floorf(p.y), floorf(p.z));
        float3 ctr = make_float3(c.x + 0.5f, c.y + 0.5f, c.z + 0.5f);
        float tt = tol;
        if (is2D) {
          const float n2 = sqrtf(nrm.x * nrm.x + nrm.y * nrm.y);
          if (n2 < 1e-4f) continue;
          ctr.z = p.z;
          tt = 0.5f * fmaxf(fabsf(nrm.x), fabsf(nrm.y)) / n2 * n2;
          if (fabsf(p.z - 0.5f) > 0.5f) continue;
        }
        if (fabsf(dot3(sub3(ctr, p0), nrm)) > tt) continue;
        atomicOr(&vote[V.cell((uint32_t)c.x, (uint32_t)c.y, (uint32_t)c.z)], 8u);
      }
    }
  }
}

__device__ __forceinline__ bool votes(uint32_t v) { return __popc(v & 7u) >= 2; }

// 4. vote -> flags (wgslVoxel.ts:172-199)
__global__ void __launch_bounds__(256) k_finalize(const VP V, const uint32_t* __restrict__ vote, uint32_t* __restrict__ flags) {
  for (size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x; id < V.n; id += (size_t)gridDim.x * blockDim.x) {
    const uint32_t v = vote[id];
    bool solid = votes(v);
    if (!solid && (v & 8u)) {
      const uint32_t x = id % V.nx, y = (id / V.nx) % V.ny, z = id / ((size_t)V.nx * V.ny);
      const size_t sxy = (size_t)V.nx * V.ny;
      bool near = false;
      if (x > 0) near = near || votes(vote[id - 1]);
      if (x + 1 < (uint32_t)V.nx) near = near || votes(vote[id + 1]);
      if (y > 0) near = near || votes(vote[id - V.nx]);
      if (y + 1 < (uint32_t)V.ny) near = near || votes(vote[id + V.nx]);
      if (z > 0) near = near || votes(vote[id - sxy]);
      if (z + 1 < (uint32_t)V.nz) near = near || votes(vote[id + sxy]);
      solid = !near;
    }
    flags[id] = solid ? 1u : 0u;
  }
}

// closest point on triangle abc to p (Ericson, Real-Time Collision Detection 5.1.5)
__device__ __forceinline__ float3 closest_pt(float3 p, float3 a, float3 b, float3 c) {
  const float3 ab = sub3(b, a), ac = sub3(c, a), ap = sub3(p, a);
  const float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  if (d1 <= 0.0f && d2 <= 0.0f) return a;
  const float3 bp = sub3(p, b);
  const float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
  if (d3 >= 0.0f && d4 <= d3) return b;
  const float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) return add3(a, mul3(ab, d1 / (d1 - d3)));
  const float3 cp = sub3(p, c);
  const float d5 = dot3(ab, cp), d6 = dot3(ac, cp);
  if (d6 >= 0.0f && d5 <= d6) return c;
  const float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) return add3(a, mul3(ac, d2 / (d2 - d6)));
  const float va = d3 * d6 - d5 * d4;
  if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f)
    return add3(b, mul3(sub3(c, b), (d4 - d3) / ((d4 - d3) + (d5 - d6))));
  const float den = 1.0f / (va + vb + vc);
  return add3(add3(a, mul3(ab, vb * den)), mul3(ac, vc * den));
}

// 5. wall distances of cell centres within 2.5 cells (wgslVoxel.ts:205-265). The reference's set:
// each surface sample p of a triangle (a (steps+1) x (steps+2) / 2 barycentric grid) scans the
// 5 x 5 x 5 cells around floor(p), and every scanned cell whose centre lies within 2.5 of the
// triangle gets that exact distance (min over triangles via atomicMax of ~bits). The distance
// does not depend on which sample reached the cell, so the result is the union of the boxes,
// each cell evaluated once:
//   - one warp per triangle; the floor cells of its samples are marked in a bitmap of 32-bit rows
//     (x in bits, one row per (y, z)) over their bounding box widened by 2, which is then dilated
//     by +-2 along x (shifts), y and z (row ORs), and every set cell is evaluated once;
//   - triangles whose widened box exceeds 32 cells along x or 256 rows, and 2-D grids, scan every
//     sample's box as the reference does (atomicMax makes repeated cells harmless).
constexpr int SDF_ROWS = 256;  // bitmap rows per warp

__device__ __forceinline__ void tri_sample(uint32_t s, uint32_t steps, float3 a, float3 e1, float3 e2, float fs,
                                           float3& p) {
  // decode the sample index into (i, j), j <= steps - i, rows of length steps + 1 - i
  uint32_t i = 0, rem = s;
  while (rem >= steps + 1 - i) {
    rem -= steps + 1 - i;
    i++;
  }
  p = add3(add3(a, mul3(e1, (float)i / fs)), mul3(e2, (float)rem / fs));
}

__device__ __forceinline__ void sdf_cell(const VP& V, int qx, int qy, int qz, float3 a, float3 b, float3 c,
                                         uint32_t* __restrict__ sdf) {
  if (qx < 0 || qy < 0 || qz < 0 || qx >= V.nx || qy >= V.ny || qz >= V.nz) return;
  const float3 ctr = make_float3((float)qx + 0.5f, (float)qy + 0.5f, (float)qz + 0.5f);
  const float d = len3(sub3(ctr, closest_pt(ctr, a, b, c)));
  if (d > 2.5f) return;
  atomicMax(&sdf[V.cell(qx, qy, qz)], ~__float_as_uint(d));
}

__global__ void __launch_bounds__(WARPS * 32) k_sdf(const VP V, const float* __restrict__ pos,
                                                    const uint32_t* __restrict__ idx, int64_t ntri,
                                                    uint32_t* __restrict__ sdf) {
  __shared__ uint32_t bm[WARPS][2][SDF_ROWS];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t* rows = bm[w][0];
  uint32_t* tmp = bm[w][1];
  for (int64_t t = (int64_t)blockIdx.x * WARPS + w; t < ntri; t += (int64_t)gridDim.x * WARPS) {
    const float3 a = vtx(V, pos, idx, 3 * t), b = vtx(V, pos, idx, 3 * t + 1), c = vtx(V, pos, idx, 3 * t + 2);
    const float3 e1 = sub3(b, a), e2 = sub3(c, a);
    if (len3(cross3(e1, e2)) < 1e-12f) continue;
    const float m = fmaxf(fmaxf(len3(e1), len3(e2)), len3(sub3(e2, e1)));
    const uint32_t steps = (uint32_t)fminf(fmaxf(ceilf(m / 0.7f), 1.0f), 256.0f);
    const float fs = (float)steps;
    const bool is2D = V.nz == 1;
    const uint32_t total = (steps + 1) * (steps + 2) / 2;
    // bounding box of the samples' floor cells
    int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
    for (uint32_t s = lane; s < total; s += 32) {
      float3 p;
      tri_sample(s, steps, a, e1, e2, fs, p);
      const int f[3] = {(int)floorf(p.x), (int)floorf(p.y), (int)floorf(p.z)};
#pragma unroll
      for (int k = 0; k < 3; k++) {
        lo[k] = min(lo[k], f[k]);
        hi[k] = max(hi[k], f[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
      lo[k] = __reduce_min_sync(0xffffffffu, lo[k]);
      hi[k] = __reduce_max_sync(0xffffffffu, hi[k]);
    }
    const int ox = lo[0] - 2, oy = lo[1] - 2, oz = lo[2] - 2;
    const int lx = hi[0] - lo[0] + 5, ly = hi[1] - lo[1] + 5, lz = hi[2] - lo[2] + 5;
    if (is2D || lx > 32 || ly * lz > SDF_ROWS) {
      // the reference's scan: every sample's 5 x 5 x 5 (2-D: 5 x 5) box
      for (uint32_t s = lane; s < total; s += 32) {
        float3 p;
        tri_sample(s, steps, a, e1, e2, fs, p);
        if (is2D && fabsf(p.z - 0.5f) > 2.5f) continue;
        const int bx = (int)floorf(p.x), by = (int)floorf(p.y), bz = (int)floorf(p.z);
        for (int dz = -2; dz <= 2; dz++) {
          if (is2D && dz != 0) continue;
          for (int dy = -2; dy <= 2; dy++)
            for (int dx = -2; dx <= 2; dx++) sdf_cell(V, bx + dx, by + dy, is2D ? 0 : bz + dz, a, b, c, sdf);
        }
      }
      continue;
    }
    const int nrow = ly * lz;
    for (int r = lane; r < nrow; r += 32) rows[r] = 0u;
    __syncwarp();
    for (uint32_t s = lane; s < total; s += 32) {
      float3 p;
      tri_sample(s, steps, a, e1, e2, fs, p);
      const int fx = (int)floorf(p.x) - ox, fy = (int)floorf(p.y) - oy, fz = (int)floorf(p.z) - oz;
      atomicOr(&rows[fy + ly * fz], 1u << fx);
    }
    __syncwarp();
    // dilate by +-2: x within each row, then y, then z (through the second buffer)
    const uint32_t xmask = lx == 32 ? 0xffffffffu : ((1u << lx) - 1u);
    for (int r = lane; r < nrow; r += 32) {
      const uint32_t v = rows[r];
      tmp[r] = (v | (v << 1) | (v << 2) | (v >> 1) | (v >> 2)) & xmask;
    }
    __syncwarp();
    for (int r = lane; r < nrow; r += 32) {
      const int y = r % ly, z = r / ly;
      uint32_t v = 0u;
      for (int d = -2; d <= 2; d++)
        if (y + d >= 0 && y + d < ly) v |= tmp[(y + d) + ly * z];
      rows[r] = v;
    }
    __syncwarp();
    for (int r = lane; r < nrow; r += 32) {
      const int y = r % ly, z = r / ly;
      uint32_t v = 0u;
      for (int d = -2; d <= 2; d++)
        if (z + d >= 0 && z + d < lz) v |= rows[y + ly * (z + d)];
      tmp[r] = v;
    }
    __syncwarp();
    // every cell of the union once
    for (int r = lane; r < nrow; r += 32) {
      uint32_t v = tmp[r];
      const int qy = oy + r % ly, qz = oz + r / ly;
      while (v) {
        const int bit = __ffs(v) - 1;
        v &= v - 1u;
        sdf_cell(V, ox + bit, qy, qz, a, b, c, sdf);
      }
    }
    __syncwarp();
  }
}

// 6. wheel tags (wgslVoxel.ts:268-290)
__global__ void __launch_bounds__(256) k_wheel_tag(const VP V, const Wheels W, uint32_t* __restrict__ flags) {
  for (size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x; id < V.n; id += (size_t)gridDim.x * blockDim.x) {
    if (flags[id] == 0u) continue;
    const float3 p = make_float3((float)(id % V.nx) + 0.5f, (float)((id / V.nx) % V.ny) + 0.5f,
                                 (float)(id / ((size_t)V.nx * V.ny)) + 0.5f);
    for (uint32_t k = 0; k < W.count; k++) {
      const float4 a = W.w[2 * k], b = W.w[2 * k + 1];
      const float3 d = sub3(p, make_float3(a.x, a.y, a.z));
      const float3 ax = make_float3(b.x, b.y, b.z);
      const float al = dot3(d, ax);
      const float rad = len3(sub3(d, mul3(ax, al)));
      if (fabsf(al) <= b.w + 0.6f && rad <= 1.0f / a.w + 0.75f) {
        flags[id] = 1u | ((k + 1u) << 8u);
        break;
      }
    }
  }
}

// 7. frontal projection + bounding box (wgslVoxel.ts:295-322): one warp per (y, z) column
__global__ void __launch_bounds__(256) k_project(const VP V, const uint32_t* __restrict__ flags, uint32_t* __restrict__ info) {
  const int lane = threadIdx.x & 31;
  const int64_t cols = (int64_t)V.ny * V.nz;
  for (int64_t col = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5); col < cols; col += (int64_t)gridDim.x * 8) {
    const uint32_t y = (uint32_t)(col % V.ny), z = (uint32_t)(col / V.ny);
    const size_t base = V.cell(0, y, z);
    uint32_t cnt = 0, xmin = 0xffffffffu, xmax = 0;
    for (int x0 = 0; x0 < V.nx; x0 += 32) {
      const int x = x0 + lane;
      const bool s = x < V.nx && flags[base + x] != 0u;
      const uint32_t bal = __ballot_sync(0xffffffffu, s);
      if (bal) {
        cnt += __popc(bal);
        if (xmin == 0xffffffffu) xmin = x0 + __ffs(bal) - 1;
        xmax = x0 + 31 - __clz(bal);
      }
    }
    if (lane == 0 && cnt > 0) {
      atomicMin(&info[2], xmin);
      atomicMax(&info[5], xmax);
      atomicAdd(&info[0], 1u);
      atomicAdd(&info[1], cnt);
      atomicMin(&info[3], y);
      atomicMax(&info[6], y);
      atomicMin(&info[4], z);
      atomicMax(&info[7], z);
    }
  }
}

unsigned blocks_for(int64_t items, int per_block) {
  int64_t b = (items + per_block - 1) / per_block;
  if (b > 148 * 64) b = 148 * 64;
  return (unsigned)(b < 1 ? 1 : b);
}

}  // namespace

cudaError_t launch_voxelize(wt_solver* s, const VoxelJob& job) {
  VP V;
  for (int k = 0; k < 16; k++) V.M[k] = job.M[k];
  V.nx = s->dims.nx;
  V.ny = s->dims.ny;
  V.nz = s->dims.nz;
  V.n = s->n;
  cudaStream_t st = s->stream;
  cudaError_t e;
  if ((e = cudaMemsetAsync(job.hits, 0, 3 * V.n * 4, st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(job.vote, 0, V.n * 4, st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(s->sdf, 0, V.n * 4, st)) != cudaSuccess) return e;
  k_crossings<<<blocks_for(job.ntri, WARPS), WARPS * 32, 0, st>>>(V, job.pos, job.idx, job.ntri, job.hits);
  k_scan_x<<<blocks_for((int64_t)V.ny * V.nz, 8), 256, 0, st>>>(V, job.hits, job.vote);
  k_scan_yz<<<blocks_for((int64_t)V.nx * V.nz, 256), 256, 0, st>>>(V, 1, job.hits, job.vote);
  k_scan_yz<<<blocks_for((int64_t)V.nx * V.ny, 256), 256, 0, st>>>(V, 2, job.hits, job.vote);
  k_surface<<<blocks_for(job.ntri, WARPS), WARPS * 32, 0, st>>>(V, job.pos, job.idx, job.ntri, job.vote);
  k_finalize<<<blocks_for((int64_t)V.n, 256), 256, 0, st>>>(V, job.vote, s->flags);
  k_sdf<<<blocks_for(job.ntri, WARPS), WARPS * 32, 0, st>>>(V, job.pos, job.idx, job.ntri, s->sdf);
  s->launches += 7;
  if (s->wheels.count > 0) {
    k_wheel_tag<<<blocks_for((int64_t)V.n, 256), 256, 0, st>>>(V, s->wheels, s->flags);
    s->launches++;
  }
  k_project<<<blocks_for((int64_t)V.ny * V.nz, 8), 256, 0, st>>>(V, s->flags, job.info);
  s->launches++;
  return cudaGetLastError();
}

}  // namespace wt
