// wt_lbm.cu — lattice Boltzmann kernels for sm_100a: cell classification, initialisation,
// fused pull-stream + collide (D2Q9 / D3Q19; f32, shifted-f16 and f64 storage), and the macro
// pass (velocity field, EMA statistics, momentum-exchange force, reductions).
//
// Physics follows the reference's generated WGSL (paths relative to the reference project):
//   stream + collide ... src/solver/wgslLbm.ts:134-293     init ... wgslLbm.ts:296-341
//   macro / force ...... src/solver/wgslLbm.ts:347-489     reduce . wgslLbm.ts:491-521
//
// Layout: populations SoA, f[i * N + cell], cell = x + nx * (y + ny * z). One thread per cell;
// a block covers a run of consecutive x in one (y, z) row, so the 19 loads and 19 stores of a
// warp are contiguous 64-byte (f16) / 128-byte (f32) segments. Cells whose pull stencil stays
// inside the domain and touches no solid (the bulk of the tunnel) take a branch-free pull; the
// reference's full boundary logic runs only for cells next to walls, the floor, the roof and
// the z sides.
#include <cuda_fp16.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>

#include "wt_internal.h"
#include "wt_closure.cuh"

namespace wt {

// ---------------------------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ R sdf_at(const uint32_t* __restrict__ sdf, size_t id) {
  uint32_t s = __ldg(sdf + id);
  if (s == 0u) return (R)-1;
  return (R)__uint_as_float(~s);
}

// linkQ (wgslLbm.ts:37-43)
template <class R>
__device__ __forceinline__ R link_q(const wt_kparams& P, const uint32_t* __restrict__ sdf, size_t fluid, size_t solid) {
  if (P.interp == 0u) return (R)0.5;
  R a = sdf_at<R>(sdf, fluid);
  R b = sdf_at<R>(sdf, solid);
  if (a < (R)0 || b < (R)0 || a + b < (R)1e-6f) return (R)0.5;
  R q = a / (a + b);
  return q < (R)0.01f ? (R)0.01f : (q > (R)0.99f ? (R)0.99f : q);
}

// wheelVel (wgslLbm.ts:21-28): u_w = U_g * (1/R) * axis x (p - c)
template <class R>
__device__ __forceinline__ void wheel_vel(const wt_kparams& P, const Wheels& W, uint32_t k, R px, R py, R pz, R& ux,
                                          R& uy, R& uz) {
  const float4 a = W.w[2 * k];
  const float4 b = W.w[2 * k + 1];
  R dx = px - (R)a.x, dy = py - (R)a.y, dz = pz - (R)a.z;
  R s = (R)P.u_ground * (R)a.w;
  ux = s * ((R)b.y * dz - (R)b.z * dy);
  uy = s * ((R)b.z * dx - (R)b.x * dz);
  uz = s * ((R)b.x * dy - (R)b.y * dx);
}

__device__ __forceinline__ size_t cell_id(int x, int y, int z, int NX, int NY) {
  return (size_t)x + (size_t)NX * ((size_t)y + (size_t)NY * (size_t)z);
}

// ---------------------------------------------------------------------------------------------
// classify: per-cell class byte (solid / fluid next to a solid pull source)
// ---------------------------------------------------------------------------------------------
template <class L>
__global__ void __launch_bounds__(256) k_classify(const wt_kparams P, const uint32_t* __restrict__ flags,
                                                  uint8_t* __restrict__ cls) {
  const int NX = P.nx, NY = P.ny, NZ = P.nz;
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y, iz = blockIdx.z;
  if (ix >= NX) return;
  const size_t idx = cell_id(ix, iy, iz, NX, NY);
  if (flags[idx] != 0u) {
    cls[idx] = CLS_SOLID;
    return;
  }
  uint8_t c = 0;
  if (iy == 0) {
    // tyre contact patch: a non-wheel solid within |dx|, |dz| <= contactH, dy in {0, 1}
    const int r = (int)P.contact_h;
    for (int dz = -r; dz <= r; dz++)
      for (int dx = -r; dx <= r; dx++)
        for (int dy = 0; dy <= 1 && dy < NY; dy++) {
          const int qx = ix + dx, qz = iz + dz;
          if (qx >= 0 && qx < NX && qz >= 0 && qz < NZ) {
            const uint32_t fq = flags[cell_id(qx, dy, qz, NX, NY)];
            if (fq != 0u && (fq >> 8u) == 0u) c |= CLS_BELT_STILL;
          }
        }
  }
  static_for<L::Q>([&](auto I) {
    constexpr int i = I;
    if constexpr (i > 0) {
      constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
      int sx = ix - cx, sy = iy - cy, sz = L::DIM == 3 ? iz - cz : 0;
      if (cx < 0) sx = min(sx, NX - 1);
      const bool inlet = cx > 0 && sx < 0;
      const bool yOut = sy < 0 || sy >= NY;
      const bool zOut = L::DIM == 3 && (sz < 0 || sz >= NZ);
      if (!inlet && !yOut && !zOut) {
        const int sxc = min(max(sx, 0), NX - 1);
        if (flags[cell_id(sxc, sy, sz, NX, NY)] != 0u) c |= CLS_NEAR_SOLID;
      }
    }
  });
  cls[idx] = c;
}

// ---------------------------------------------------------------------------------------------
// init (wgslLbm.ts:296-341) + rest-state-with-noise extension
// ---------------------------------------------------------------------------------------------
template <class L, class S>
__global__ void __launch_bounds__(256) k_init(const wt_kparams P, typename S::T* __restrict__ fa,
                                              typename S::T* __restrict__ fb, const uint32_t* __restrict__ flags,
                                              int mode, uint32_t seed, float amp) {
  typedef typename S::R R;
  const size_t N = P.n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < N; idx += (size_t)gridDim.x * blockDim.x) {
    const bool solid = flags[idx] != 0u;
    float un[3] = {0.f, 0.f, 0.f};
    if (mode == WT_INIT_FREESTREAM) {
      un[0] = solid ? 0.0f : P.uin;
    } else if (!solid) {
      for (int a = 0; a < L::DIM; a++) un[a] = noise_component(seed, idx, a, amp);
    }
    static_for<L::Q>([&](auto I) {
      constexpr int i = I;
      constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
      typename S::T v;
      if constexpr (S::PREC == WT_PREC_F16) {
        // shifted storage: f - w written directly (wgslLbm.ts:297-303)
        float r;
        if (mode == WT_INIT_FREESTREAM) {
          const float ua = un[0];
          r = (float)Wc<L, i>::v * ((float)(3 * cx) * ua + (float)(4.5 * cx * cx) * ua * ua - 1.5f * ua * ua);
        } else {
          float cu = (float)cx * un[0] + (float)cy * un[1] + (float)cz * un[2];
          float usq = un[0] * un[0] + un[1] * un[1] + un[2] * un[2];
          r = (float)Wc<L, i>::v * (3.0f * cu + 4.5f * cu * cu - 1.5f * usq);
        }
        v = __float2half_rn(r);
      } else {
        R r;
        if (mode == WT_INIT_FREESTREAM) {
          const R U = (R)un[0];
          r = (R)Wc<L, i>::v * ((R)1 + (R)(3 * cx) * U + (R)(4.5 * cx * cx) * U * U - (R)1.5 * U * U);
        } else {
          const R cu = (R)cx * (R)un[0] + (R)cy * (R)un[1] + (R)cz * (R)un[2];
          const R usq = (R)un[0] * (R)un[0] + (R)un[1] * (R)un[1] + (R)un[2] * (R)un[2];
          r = (R)Wc<L, i>::v * ((R)1 + (R)3 * cu + (R)4.5 * cu * cu - (R)1.5 * usq);
        }
        v = (typename S::T)r;
      }
      fa[(size_t)i * N + idx] = v;
      fb[(size_t)i * N + idx] = v;
    });
  }
}

// ---------------------------------------------------------------------------------------------
// fused pull-stream + collide
// ---------------------------------------------------------------------------------------------

// Collision on full populations, in the reference's formulation: regularized BGK (or BGK on wall
// cells / collision = bgk) with the Smagorinsky relaxation time and the outlet / inlet sponges
// (wgslLbm.ts:177-240). fo receives the post-collision populations.
//
// With nu_in >= 0 (the learned closure's eddy viscosity of the cell) it replaces the Smagorinsky
// term: tau = tau0' + 3 nu_in (tau0' = tau0 with the outlet sponge and the wall floor). With xout
// (f32 D3Q19 only) the closure's 10 features of the cell go to xout and nothing is collided.
template <class L, class R>
__device__ __forceinline__ void collide_full(const wt_kparams& P, const R (&f)[L::Q], int ix, bool wall, bool gwall,
                                             R (&fo)[L::Q], float nu_in = -1.0f, float* xout = nullptr,
                                             float wall_d = 0.0f) {
  constexpr int Q = L::Q;
  constexpr bool D3 = L::DIM == 3;
  const R U = (R)P.uin;
  R rho = f[0];
  R jx = 0, jy = 0, jz = 0, sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
    if constexpr (i > 0) rho += f[i];
    if constexpr (cx != 0) jx += (R)cx * f[i];
    if constexpr (cy != 0) jy += (R)cy * f[i];
    if constexpr (cz != 0) jz += (R)cz * f[i];
    if constexpr (cx != 0) sxx += f[i];
    if constexpr (cy != 0) syy += f[i];
    if constexpr (cz != 0) szz += f[i];
    if constexpr (cx * cy != 0) sxy += (R)(cx * cy) * f[i];
    if constexpr (cx * cz != 0) sxz += (R)(cx * cz) * f[i];
    if constexpr (cy * cz != 0) syz += (R)(cy * cz) * f[i];
  });
  const R irho = (R)1 / rho;
  const R ux = jx * irho, uy = jy * irho, uz = D3 ? jz * irho : (R)0;
  const R usq = ux * ux + uy * uy + uz * uz;
  const R third = (R)(1.0 / 3.0);
  const R pxx = sxx - rho * (ux * ux + third);
  const R pyy = syy - rho * (uy * uy + third);
  const R pxy = sxy - rho * ux * uy;
  R pzz = 0, pxz = 0, pyz = 0;
  if constexpr (D3) {
    pzz = szz - rho * (uz * uz + third);
    pxz = sxz - rho * ux * uz;
    pyz = syz - rho * uy * uz;
  }
  if constexpr (std::is_same<R, float>::value && D3) {
    if (xout != nullptr) {
      cl_features(pxx, pyy, pzz, pxy, pxz, pyz, rho, ux, uy, uz, P.tau0, wall_d,
                  *reinterpret_cast<float(*)[CL_IN]>(xout));
      return;
    }
  }
  R pn = pxx * pxx + (R)2 * pxy * pxy + pyy * pyy;
  if constexpr (D3) pn = pxx * pxx + (R)2 * pxy * pxy + (R)2 * pxz * pxz + pyy * pyy + (R)2 * pyz * pyz + pzz * pzz;
  const R piN = sqrt(pn);
  const R fx = (R)ix;
  const R den = (R)P.nx - (R)P.sponge_start;
  R sp = (fx - (R)P.sponge_start) / (den > (R)1 ? den : (R)1);
  sp = sp < (R)0 ? (R)0 : (sp > (R)1 ? (R)1 : sp);
  R t0 = (R)P.tau0 + (R)3 * (R)P.sponge_nu * sp * sp;
  if (gwall) t0 = t0 > (R)P.tau_wall ? t0 : (R)P.tau_wall;
  const R tau = nu_in >= 0.0f
                    ? t0 + (R)3 * (R)nu_in
                    : (R)0.5 * (t0 + sqrt(t0 * t0 + (R)(18.0 * 1.4142135623730951) * (R)P.csmag2 * piN * irho));
  const R omega = (R)1 - (R)1 / tau;
  const R k1 = omega * (R)4.5;
  const bool useBGK = wall || P.collision == 1u;
  const R sInDen = (R)P.sponge_in > (R)1 ? (R)P.sponge_in : (R)1;
  R si = (R)1 - fx / sInDen;
  si = si < (R)0 ? (R)0 : (si > (R)1 ? (R)1 : si);
  const R sIn = (R)P.sponge_in > (R)0 ? (R)0.08 * si * si : (R)0;
  const R trP = (pxx + pyy + pzz) * third;
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
    const R w = (R)Wc<L, i>::v;
    const R cu = (R)cx * ux + (R)cy * uy + (R)cz * uz;
    // the reference's evaluation order (wgslLbm.ts:221-236): feq from 1 + 3 cu + 4.5 cu^2 - 1.5 u^2,
    // and Q_i : Pi summed over the stress components in the order xx, xy, xz, yy, yz, zz with the
    // zero terms left out
    const R feq = w * rho * ((R)1 + (R)3 * cu + (R)4.5 * cu * cu - (R)1.5 * usq);
    R qp = (R)0;
    bool qf = true;
    auto addq = [&](int coef, R p) {
      if (coef == 0) return;
      const R t = (R)coef * p;
      qp = qf ? t : qp + t;
      qf = false;
    };
    addq(cx * cx, pxx);
    addq(2 * cx * cy, pxy);
    if constexpr (D3) addq(2 * cx * cz, pxz);
    addq(cy * cy, pyy);
    if constexpr (D3) {
      addq(2 * cy * cz, pyz);
      addq(cz * cz, pzz);
    }
    const R qpi = qp - trP;
    R v = feq + (useBGK ? omega * (f[i] - feq) : w * k1 * qpi);
    if (sIn > (R)0) {
      const R eq = w * ((R)1 + (R)(3 * cx) * U + (R)(4.5 * cx * cx) * U * U - (R)1.5 * U * U);
      v = v * ((R)1 - sIn) + eq * sIn;
    }
    fo[i] = v;
  });
}

// Reference-exact update of one fluid cell with every boundary rule of the pull (inlet
// equilibrium, zero-gradient outlet, free-slip / no-slip / moving-belt floor with tyre contact
// patches, specular or periodic sides, Bouzidi walls, rotating wheels with their mass fix;
// wgslLbm.ts:138-175, 276-291), for cells in groups that touch a solid.
//
// Organised as gather-then-apply. The cell's own 19 populations are loaded first; then, for groups
// of six links, every value a link can need (its source population, the source flags and wall
// distance, the Bouzidi partner population and flags at x + c_i) is fetched through a clamped,
// always-valid address without being inspected, and only after the whole group is in flight are
// the raw values converted and the reference's rules applied. A group therefore costs one memory
// round trip instead of a chain of dependent loads per link. `cl` is the cell's class byte: its
// near-solid bit enables the solid checks, its belt-still bit holds the moving belt still (the
// tyre contact patch test of wgslLbm.ts:276-287, evaluated once by k_classify). Kept out of line
// so that it does not inflate the register budget of the kernels that call it. With PULL the
// pulled (pre-collision) populations are returned instead of the collided ones.
template <class L, class S, bool PULL = false>
__device__ __noinline__ void cell_general(const wt_kparams& P, const typename S::T* __restrict__ fin,
                                          const uint32_t* __restrict__ flags, const uint32_t* __restrict__ sdf,
                                          const Wheels& W, int ix, int iy, int iz, uint32_t cl, typename S::R* out) {
  typedef typename S::R R;
  typedef typename S::T T;
  constexpr int Q = L::Q;
  constexpr bool D3 = L::DIM == 3;
  constexpr int CH = 6;  // links per gather group
  constexpr int NCH = (Q - 1 + CH - 1) / CH;
  enum : int { K_INLET = 0, K_GROUND = 1, K_MIRROR = 2, K_INTERIOR = 3 };
  const int NX = P.nx, NY = P.ny, NZ = P.nz;
  const size_t N = P.n;
  const size_t idx = cell_id(ix, iy, iz, NX, NY);
  const bool near = (cl & CLS_NEAR_SOLID) != 0;
  const R U = (R)P.uin;
  // the cell's own populations: bounce partners f_opp(x) and the q > 1/2 Bouzidi term f_i(x)
  T own_raw[Q];
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    own_raw[i] = __ldg(fin + (size_t)i * N + idx);
  });
  const uint32_t sdf_self_raw = __ldg(sdf + idx);
  R own[Q];
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    own[i] = S::cvt(own_raw[i], (R)Wc<L, i>::v);
  });
  R f[Q];
  f[0] = own[0];
  bool wall = false, gwall = false;
  R mvSum = 0, mvW = 0;
  uint32_t wm = 0;
  const R belt = (P.ground == 2u && !(cl & CLS_BELT_STILL)) ? (R)1 : (R)0;
  const R sdf_self = (P.interp != 0u && sdf_self_raw != 0u) ? (R)__uint_as_float(~sdf_self_raw) : (R)-1;
  static_for<NCH>([&](auto C) {
    constexpr int c0 = 1 + CH * decltype(C)::value;
    int kind[CH], sxcv[CH], syv[CH], szv[CH];
    bool inA[CH];
    T rsrc[CH], rah[CH];
    uint32_t rfs[CH], rfa[CH], rsd[CH];
    // ---- gather: addresses from coordinates only, every load issued before any is inspected ----
    static_for<CH>([&](auto J) {
      constexpr int j = J;
      constexpr int i = c0 + j;
      if constexpr (i < Q) {
        constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
        constexpr int io = opp<L>(i);
        int sx = ix - cx;
        const int sy = iy - cy, sz = D3 ? iz - cz : 0;
        if constexpr (cx < 0) sx = min(sx, NX - 1);
        const bool yOut = cy > 0 ? sy < 0 : (cy < 0 ? sy >= NY : false);
        const bool zOut = D3 ? (cz > 0 ? sz < 0 : (cz < 0 ? sz >= NZ : false)) : false;
        const int sxc = min(max(sx, 0), NX - 1);
        const int syc = min(max(sy, 0), NY - 1), szc = D3 ? min(max(sz, 0), NZ - 1) : 0;
        sxcv[j] = sxc;
        syv[j] = sy;
        szv[j] = sz;
        int k;
        size_t a = idx;
        if (cx > 0 && sx < 0) {
          k = K_INLET;
        } else if (cy > 0 && yOut && P.ground != 0u) {
          k = K_GROUND;
        } else if (D3 && yOut && zOut) {
          k = K_MIRROR;
          a = (size_t)mirYZ<L>(i) * N + cell_id(sxc, iy, iz, NX, NY);
        } else if (yOut) {
          k = K_MIRROR;
          a = (size_t)mirY<L>(i) * N + cell_id(sxc, iy, szc, NX, NY);
        } else if (D3 && zOut) {
          k = K_MIRROR;
          a = P.side_mode == 1u ? (size_t)i * N + cell_id(sxc, sy, (sz + NZ) % NZ, NX, NY)
                                : (size_t)mirZ<L>(i) * N + cell_id(sxc, sy, iz, NX, NY);
        } else {
          k = K_INTERIOR;
          a = (size_t)i * N + cell_id(sxc, sy, sz, NX, NY);
        }
        kind[j] = k;
        const size_t sc = cell_id(sxc, syc, szc, NX, NY);
        const int ax = ix + cx, ay = iy + cy, az = D3 ? iz + cz : 0;
        inA[j] = ax >= 0 && ay >= 0 && az >= 0 && ax < NX && ay < NY && az < NZ;
        const size_t ac = inA[j] ? cell_id(ax, ay, az, NX, NY) : idx;
        rsrc[j] = __ldg(fin + a);
        rfs[j] = __ldg(flags + sc);
        rsd[j] = __ldg(sdf + sc);
        rfa[j] = __ldg(flags + ac);
        rah[j] = __ldg(fin + (size_t)io * N + ac);
      }
    });
    // ---- apply the reference's rules ----
    static_for<CH>([&](auto J) {
      constexpr int j = J;
      constexpr int i = c0 + j;
      if constexpr (i < Q) {
        constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
        constexpr int io = opp<L>(i);
        const R w = (R)Wc<L, i>::v;
        R v;
        const uint32_t fs = (near && kind[j] == K_INTERIOR) ? rfs[j] : 0u;
        if (kind[j] == K_INLET) {
          const R cu = (R)1 * U;
          v = w * (R)P.rho_in * ((R)1 + (R)3 * cu + (R)4.5 * cu * cu - (R)1.5 * U * U);
        } else if (kind[j] == K_GROUND) {
          wall = true;
          gwall = true;
          v = own[io];
          if constexpr (cx != 0) v = v + belt * ((R)(6.0 * Wc<L, i>::v * cx) * (R)P.u_ground);
        } else if (fs == 0u) {
          // mirror / periodic image or an interior fluid source; every such plane has weight w_i
          v = S::cvt(rsrc[j], w);
        } else {
          // interpolated bounce-back (Bouzidi) on a solid source
          wall = true;
          const R fb = own[io];
          R q = (R)0.5;
          if (P.interp != 0u) {
            const R a = sdf_self, b = rsd[j] != 0u ? (R)__uint_as_float(~rsd[j]) : (R)-1;
            if (!(a < (R)0 || b < (R)0 || a + b < (R)1e-6f)) {
              q = a / (a + b);
              q = q < (R)0.01f ? (R)0.01f : (q > (R)0.99f ? (R)0.99f : q);
            }
          }
          v = fb;
          if (q < (R)0.5) {
            if (inA[j] && rfa[j] == 0u) v = (R)2 * q * fb + ((R)1 - (R)2 * q) * S::cvt(rah[j], (R)Wc<L, io>::v);
            else q = (R)0.5;
          } else if (q > (R)0.5) {
            v = ((R)0.5 / q) * fb + ((R)1 - (R)0.5 / q) * own[i];
          }
          if ((fs >> 8u) != 0u) {
            R ux, uy, uz;
            wheel_vel<R>(P, W, (fs >> 8u) - 1u, (R)0.5 * (R)(ix + sxcv[j]) + (R)0.5,
                         (R)0.5 * (R)(iy + syv[j]) + (R)0.5, (R)0.5 * (R)(iz + szv[j]) + (R)0.5, ux, uy, uz);
            const R dot = (R)cx * ux + (R)cy * uy + (R)cz * uz;
            const R mv = (R)(6.0 * Wc<L, i>::v) * dot * (q > (R)0.5 ? (R)0.5 / q : (R)1);
            v += mv;
            mvSum += mv;
            mvW += w;
            wm |= 1u << i;
          }
        }
        f[i] = v;
      }
    });
  });
  // wheel links: remove the net mass of the moving-wall terms (wgslLbm.ts:289-291)
  if (mvW > (R)0) {
    const R corr = mvSum / mvW;
    static_for<Q>([&](auto I) {
      constexpr int i = I;
      if constexpr (i > 0)
        if (wm & (1u << i)) f[i] -= (R)Wc<L, i>::v * corr;
    });
  }
  if constexpr (PULL) {
    static_for<Q>([&](auto I) {
      constexpr int i = I;
      out[i] = f[i];
    });
  } else {
    R fo[Q];
    collide_full<L, R>(P, f, ix, wall, gwall, fo);
    static_for<Q>([&](auto I) {
      constexpr int i = I;
      out[i] = fo[i];
    });
  }
}

// One cell per thread; any storage. Used for f64 and for odd nx.
template <class L, class S>
__global__ void __launch_bounds__(256) k_stream_collide(const __grid_constant__ wt_kparams P,
                                                        const typename S::T* __restrict__ fin,
                                                        typename S::T* __restrict__ fout,
                                                        const uint8_t* __restrict__ cls,
                                                        const uint32_t* __restrict__ flags,
                                                        const uint32_t* __restrict__ sdf,
                                                        const __grid_constant__ Wheels W) {
  typedef typename S::R R;
  constexpr int Q = L::Q;
  constexpr bool D3 = L::DIM == 3;
  const int NX = P.nx, NY = P.ny, NZ = P.nz;
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y, iz = blockIdx.z;
  if (ix >= NX) return;
  const size_t N = P.n;
  const size_t idx = cell_id(ix, iy, iz, NX, NY);
  const uint8_t cl = __ldg(cls + idx);
  if (cl & CLS_SOLID) {
    static_for<Q>([&](auto I) {
      constexpr int i = I;
      fout[(size_t)i * N + idx] = S::solid((R)Wc<L, i>::v);
    });
    return;
  }
  R fo[Q];
  const bool fast = (cl & CLS_BOUNDARY) == 0 && iy > 0 && iy < NY - 1 && (!D3 || (iz > 0 && iz < NZ - 1));
  if (fast) {
    // bulk: every pull source is an in-domain fluid cell, except the inlet / outlet columns
    const R U = (R)P.uin;
    R f[Q];
    static_for<Q>([&](auto I) {
      constexpr int i = I;
      constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
      const R w = (R)Wc<L, i>::v;
      int sx = ix - cx;
      if constexpr (cx < 0) sx = min(sx, NX - 1);
      const size_t src = cell_id(max(sx, 0), iy - cy, D3 ? iz - cz : 0, NX, NY);
      R v = S::ld(fin, (size_t)i * N + src, w);
      if constexpr (cx > 0) {
        if (sx < 0) {
          const R cu = (R)1 * U;
          v = w * (R)P.rho_in * ((R)1 + (R)3 * cu + (R)4.5 * cu * cu - (R)1.5 * U * U);
        }
      }
      f[i] = v;
    });
    collide_full<L, R>(P, f, ix, false, false, fo);
  } else {
    cell_general<L, S>(P, fin, flags, sdf, W, ix, iy, iz, cl, fo);
  }
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    S::st(fout, (size_t)i * N + idx, fo[i], (R)Wc<L, i>::v);
  });
}

// ---- vectorised bulk kernel: V consecutive cells per thread ---------------------------------
//
// Works on shifted populations h = f - w throughout (the FP16 storage format): with
// drho = sum h, j = sum c h and S = sum c c h, the reference's regularized collision becomes
//   out_i - w_i = w_i (drho - 1.5 j.u + 4.5 (c_i.j)(c_i.u) + 3 c_i.j + k1 (Q_i : Pi_neq))
//   Pi_neq = S - j u^T - I drho / 3,   k1 = 4.5 (1 - 1/tau)
// which is the same algebra as wgslLbm.ts:177-240 without the +w / -w round trip. Moments are
// built from opposite-direction pair sums h_i + h_opp and differences h_i - h_opp.
template <class S, int V> struct VecIO;
template <> struct VecIO<StF16, 2> {
  __device__ __forceinline__ static void ld(const __half* __restrict__ p, uint32_t o, float (&h)[2], float /*w*/) {
    const uint32_t u = __ldg(reinterpret_cast<const unsigned int*>(p + o));
    const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&u));
    h[0] = f.x;
    h[1] = f.y;
  }
  __device__ __forceinline__ static void st(__half* __restrict__ p, uint32_t o, const float (&h)[2], float /*w*/) {
    const __half2 v = __floats2half2_rn(h[0], h[1]);
    *reinterpret_cast<__half2*>(p + o) = v;
  }
};
template <> struct VecIO<StF16, 4> {
  __device__ __forceinline__ static void ld(const __half* __restrict__ p, uint32_t o, float (&h)[4], float /*w*/) {
    const uint2 u = __ldg(reinterpret_cast<const uint2*>(p + o));
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
    h[0] = a.x;
    h[1] = a.y;
    h[2] = b.x;
    h[3] = b.y;
  }
  __device__ __forceinline__ static void st(__half* __restrict__ p, uint32_t o, const float (&h)[4], float /*w*/) {
    const __half2 a = __floats2half2_rn(h[0], h[1]);
    const __half2 b = __floats2half2_rn(h[2], h[3]);
    uint2 u;
    u.x = *reinterpret_cast<const uint32_t*>(&a);
    u.y = *reinterpret_cast<const uint32_t*>(&b);
    *reinterpret_cast<uint2*>(p + o) = u;
  }
};
template <> struct VecIO<StF32, 2> {
  __device__ __forceinline__ static void ld(const float* __restrict__ p, uint32_t o, float (&h)[2], float w) {
    const float2 f = __ldg(reinterpret_cast<const float2*>(p + o));
    h[0] = f.x - w;
    h[1] = f.y - w;
  }
  __device__ __forceinline__ static void st(float* __restrict__ p, uint32_t o, const float (&h)[2], float w) {
    *reinterpret_cast<float2*>(p + o) = make_float2(h[0] + w, h[1] + w);
  }
};
template <> struct VecIO<StF32, 4> {
  __device__ __forceinline__ static void ld(const float* __restrict__ p, uint32_t o, float (&h)[4], float w) {
    const float4 f = __ldg(reinterpret_cast<const float4*>(p + o));
    h[0] = f.x - w;
    h[1] = f.y - w;
    h[2] = f.z - w;
    h[3] = f.w - w;
  }
  __device__ __forceinline__ static void st(float* __restrict__ p, uint32_t o, const float (&h)[4], float w) {
    *reinterpret_cast<float4*>(p + o) = make_float4(h[0] + w, h[1] + w, h[2] + w, h[3] + w);
  }
};
__device__ __forceinline__ float ld_shift(const __half* __restrict__ p, uint32_t o, float /*w*/) {
  return __half2float(__ldg(p + o));
}
__device__ __forceinline__ float ld_shift(const float* __restrict__ p, uint32_t o, float w) { return __ldg(p + o) - w; }

// Regularized / BGK collision of one bulk cell on shifted populations (see the block comment).
template <class L>
__device__ __forceinline__ void collide_shifted(const wt_kparams& P, const float (&h)[L::Q], int ix, float (&o)[L::Q]) {
  constexpr int Q = L::Q;
  constexpr bool D3 = L::DIM == 3;
  float drho = h[0];
  float jx = 0.f, jy = 0.f, jz = 0.f, sxx = 0.f, syy = 0.f, szz = 0.f, sxy = 0.f, sxz = 0.f, syz = 0.f;
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    constexpr int io = opp<L>(i);
    if constexpr (i > 0 && i < io) {
      constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
      const float s = h[i] + h[io];
      const float d = h[i] - h[io];
      drho += s;
      if constexpr (cx > 0) jx += d;
      if constexpr (cx < 0) jx -= d;
      if constexpr (cy > 0) jy += d;
      if constexpr (cy < 0) jy -= d;
      if constexpr (cz > 0) jz += d;
      if constexpr (cz < 0) jz -= d;
      if constexpr (cx != 0) sxx += s;
      if constexpr (cy != 0) syy += s;
      if constexpr (cz != 0) szz += s;
      if constexpr (cx * cy > 0) sxy += s;
      if constexpr (cx * cy < 0) sxy -= s;
      if constexpr (cx * cz > 0) sxz += s;
      if constexpr (cx * cz < 0) sxz -= s;
      if constexpr (cy * cz > 0) syz += s;
      if constexpr (cy * cz < 0) syz -= s;
    }
  });
  const float rho = 1.0f + drho;
  const float irho = __frcp_rn(rho);
  const float ux = jx * irho, uy = jy * irho, uz = D3 ? jz * irho : 0.0f;
  const float d3 = drho * (1.0f / 3.0f);
  const float pxx = sxx - jx * ux - d3;
  const float pyy = syy - jy * uy - d3;
  const float pxy = sxy - jx * uy;
  float pzz = 0.f, pxz = 0.f, pyz = 0.f;
  if constexpr (D3) {
    pzz = szz - jz * uz - d3;
    pxz = sxz - jx * uz;
    pyz = syz - jy * uz;
  }
  float pn = pxx * pxx + 2.0f * pxy * pxy + pyy * pyy;
  if constexpr (D3) pn += 2.0f * pxz * pxz + pzz * pzz + 2.0f * pyz * pyz;
  const float fx = (float)ix;
  const float den = (float)P.nx - P.sponge_start;
  const float sp = fminf(fmaxf((fx - P.sponge_start) / (den > 1.0f ? den : 1.0f), 0.0f), 1.0f);
  const float t0 = P.tau0 + 3.0f * P.sponge_nu * sp * sp;
  const float tau = 0.5f * (t0 + sqrtf(t0 * t0 + (float)(18.0 * 1.4142135623730951) * P.csmag2 * sqrtf(pn) * irho));
  const float omega = 1.0f - __frcp_rn(tau);
  const float k1 = 4.5f * omega;
  const float trP = (pxx + pyy + pzz) * (1.0f / 3.0f);
  const float ju = jx * ux + jy * uy + jz * uz;
  const float base = drho - 1.5f * ju;
  const bool bgk = P.collision == 1u;
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    constexpr int io = opp<L>(i);
    if constexpr (i == 0 || i < io) {
      constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
      constexpr float w = (float)Wc<L, i>::v;
      const float cj = (float)cx * jx + (float)cy * jy + (float)cz * jz;
      const float cu = (float)cx * ux + (float)cy * uy + (float)cz * uz;
      const float qp = (float)(cx * cx) * pxx + (float)(cy * cy) * pyy + (float)(cz * cz) * pzz +
                       (float)(2 * cx * cy) * pxy + (float)(2 * cx * cz) * pxz + (float)(2 * cy * cz) * pyz - trP;
      const float e = base + 4.5f * cj * cu;  // even part of (feq - w) / w
      const float od = 3.0f * cj;             // odd part
      if (!bgk) {
        const float t = e + k1 * qp;
        o[i] = w * (t + od);
        if constexpr (i > 0) o[io] = w * (t - od);
      } else {
        const float a = 1.0f - omega;
        o[i] = a * (w * (e + od)) + omega * h[i];
        if constexpr (i > 0) o[io] = a * (w * (e - od)) + omega * h[io];
      }
    }
  });
  // inlet absorbing layer: blend towards the free-stream equilibrium (wgslLbm.ts:224-237)
  if (P.sponge_in > 0.0f) {
    const float si = fminf(fmaxf(1.0f - fx / fmaxf(P.sponge_in, 1.0f), 0.0f), 1.0f);
    const float sIn = 0.08f * si * si;
    if (sIn > 0.0f) {
      const float U = P.uin;
      static_for<Q>([&](auto I) {
        constexpr int i = I;
        constexpr int cx = L::c[i][0];
        constexpr float w = (float)Wc<L, i>::v;
        const float eqw = w * ((float)(3 * cx) * U + (float)(4.5 * cx * cx) * U * U - 1.5f * U * U);
        o[i] = o[i] * (1.0f - sIn) + eqw * sIn;
      });
    }
  }
}

// ---- packed two-cell collision (sm_100 f32x2 arithmetic) ------------------------------------
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.0f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// relaxation time of one bulk cell: molecular tau0 + outlet sponge, Smagorinsky closure
__device__ __forceinline__ void relax_cell(const wt_kparams& P, float fx, float pn, float irho, float& omega,
                                           float t_floor) {
  float t0 = P.tau0;
  if (fx > P.sponge_start) {
    const float den = (float)P.nx - P.sponge_start;
    const float sp = fminf(__fdividef(fx - P.sponge_start, den > 1.0f ? den : 1.0f), 1.0f);
    t0 += 3.0f * P.sponge_nu * sp * sp;
  }
  t0 = fmaxf(t0, t_floor);
  float tau = t0;
  if (P.csmag2 > 0.0f) {
    const float k = (float)(18.0 * 1.4142135623730951) * P.csmag2;
    tau = 0.5f * (t0 + sqrt_approx(t0 * t0 + k * sqrt_approx(pn) * irho));
  }
  omega = 1.0f - __fdividef(1.0f, tau);
}

// tau0 of one cell with the outlet sponge and a floor (the part of relax_cell before the closure)
__device__ __forceinline__ float tau0_eff(const wt_kparams& P, float fx, float t_floor) {
  float t0 = P.tau0;
  if (fx > P.sponge_start) {
    const float den = (float)P.nx - P.sponge_start;
    const float sp = fminf(__fdividef(fx - P.sponge_start, den > 1.0f ? den : 1.0f), 1.0f);
    t0 += 3.0f * P.sponge_nu * sp * sp;
  }
  return fmaxf(t0, t_floor);
}

// Regularized / BGK collision of two bulk cells at once on shifted populations (lanes .x, .y),
// same algebra as collide_shifted. `ofn(rho, irho, ux, uy, uz, pxx, pyy, pzz, pxy, pxz, pyz)`
// returns the two cells' omega = 1 - 1 / tau (the closure). SP: whether the cells lie in the inlet
// absorbing layer: SP_ON / SP_OFF when the caller has branched on it once per cell pair (no test
// per direction), SP_TEST to test it here (for callers whose ofn holds block-wide barriers, which
// every thread must reach through the same call).
enum : int { SP_OFF = 0, SP_ON = 1, SP_TEST = 2 };
template <class L, bool BGK, int SP = SP_TEST, class Emit, class OmegaFn>
__device__ __forceinline__ void collide_shifted2x(const wt_kparams& P, const float2 (&h)[L::Q], int x, Emit&& emit,
                                                  OmegaFn&& ofn) {
  constexpr int Q = L::Q;
  constexpr bool D3 = L::DIM == 3;
  float2 drho = h[0];
  float2 jx = f2(0.f), jy = f2(0.f), jz = f2(0.f), sxx = f2(0.f), syy = f2(0.f), szz = f2(0.f), sxy = f2(0.f),
         sxz = f2(0.f), syz = f2(0.f);
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    constexpr int io = opp<L>(i);
    if constexpr (i > 0 && i < io) {
      constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
      const float2 s = add2(h[i], h[io]);
      const float2 d = sub2(h[i], h[io]);
      drho = add2(drho, s);
      if constexpr (cx > 0) jx = add2(jx, d);
      if constexpr (cx < 0) jx = sub2(jx, d);
      if constexpr (cy > 0) jy = add2(jy, d);
      if constexpr (cy < 0) jy = sub2(jy, d);
      if constexpr (cz > 0) jz = add2(jz, d);
      if constexpr (cz < 0) jz = sub2(jz, d);
      if constexpr (cx != 0) sxx = add2(sxx, s);
      if constexpr (cy != 0) syy = add2(syy, s);
      if constexpr (cz != 0) szz = add2(szz, s);
      if constexpr (cx * cy > 0) sxy = add2(sxy, s);
      if constexpr (cx * cy < 0) sxy = sub2(sxy, s);
      if constexpr (cx * cz > 0) sxz = add2(sxz, s);
      if constexpr (cx * cz < 0) sxz = sub2(sxz, s);
      if constexpr (cy * cz > 0) syz = add2(syz, s);
      if constexpr (cy * cz < 0) syz = sub2(syz, s);
    }
  });
  const float2 rho = add2(f2(1.0f), drho);
  const float2 irho = make_float2(__fdividef(1.0f, rho.x), __fdividef(1.0f, rho.y));
  const float2 ux = mul2(jx, irho), uy = mul2(jy, irho), uz = D3 ? mul2(jz, irho) : f2(0.f);
  const float2 nux = mul2(ux, f2(-1.f)), nuy = mul2(uy, f2(-1.f)), nuz = mul2(uz, f2(-1.f));
  const float2 d3 = mul2(drho, f2(1.0f / 3.0f));
  const float2 pxx = fma2(jx, nux, sub2(sxx, d3));
  const float2 pyy = fma2(jy, nuy, sub2(syy, d3));
  const float2 pxy = fma2(jx, nuy, sxy);
  float2 pzz = f2(0.f), pxz = f2(0.f), pyz = f2(0.f);
  if constexpr (D3) {
    pzz = fma2(jz, nuz, sub2(szz, d3));
    pxz = fma2(jx, nuz, sxz);
    pyz = fma2(jy, nuz, syz);
  }
  const float2 omega = ofn(rho, irho, ux, uy, uz, pxx, pyy, pzz, pxy, pxz, pyz);
  const float2 k1 = mul2(f2(4.5f), omega);
  const float2 trP = mul2(add2(add2(pxx, pyy), pzz), f2(1.0f / 3.0f));
  // Q_i : Pi - trP for axis directions (Daa) and for two-component directions (Eab +- 2 Pab)
  const float2 Dxx = sub2(pxx, trP), Dyy = sub2(pyy, trP), Dzz = sub2(pzz, trP);
  const float2 Exy = add2(Dxx, pyy), Exz = add2(Dxx, pzz), Eyz = add2(Dyy, pzz);
  const float2 ju = fma2(jx, ux, fma2(jy, uy, mul2(jz, uz)));
  const float2 base = fma2(f2(-1.5f), ju, drho);
  const float2 a = sub2(f2(1.0f), omega);
  // inlet absorbing layer: blend towards the free-stream equilibrium (wgslLbm.ts:224-237)
  float2 keep = f2(1.0f), sIn = f2(0.0f);
  const bool sponge_in = SP == SP_TEST ? P.sponge_in > 0.0f && (float)x < P.sponge_in : SP == SP_ON;
  if (sponge_in) {
    const float inv = __fdividef(1.0f, fmaxf(P.sponge_in, 1.0f));
    const float s0 = fminf(fmaxf(1.0f - (float)x * inv, 0.0f), 1.0f);
    const float s1 = fminf(fmaxf(1.0f - (float)(x + 1) * inv, 0.0f), 1.0f);
    sIn = make_float2(0.08f * s0 * s0, 0.08f * s1 * s1);
    keep = sub2(f2(1.0f), sIn);
  }
  auto out = [&](auto I, float2 v) {
    if (sponge_in) {
      constexpr int i = decltype(I)::value;
      constexpr int cx = L::c[i][0];
      constexpr float w = (float)Wc<L, i>::v;
      const float U = P.uin;
      const float eqw = w * ((float)(3 * cx) * U + (float)(4.5 * cx * cx) * U * U - 1.5f * U * U);
      v = fma2(v, keep, mul2(f2(eqw), sIn));
    }
    emit(I, v);
  };
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    constexpr int io = opp<L>(i);
    if constexpr (i == 0 || i < io) {
      constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
      constexpr int nc = (cx != 0) + (cy != 0) + (cz != 0);
      constexpr float w = (float)Wc<L, i>::v;
      float2 cj = f2(0.f), cu = f2(0.f), qp;
      if constexpr (nc == 0) {
        qp = mul2(trP, f2(-1.f));
      } else if constexpr (nc == 1) {
        cj = cx > 0 ? jx : (cx < 0 ? mul2(jx, f2(-1.f)) : cy > 0 ? jy : (cy < 0 ? mul2(jy, f2(-1.f)) : cz > 0 ? jz : mul2(jz, f2(-1.f))));
        cu = cx > 0 ? ux : (cx < 0 ? nux : cy > 0 ? uy : (cy < 0 ? nuy : cz > 0 ? uz : nuz));
        qp = cx != 0 ? Dxx : (cy != 0 ? Dyy : Dzz);
      } else {
        // two non-zero components (a, b) with signs (sa, sb)
        constexpr int ax = cx != 0 ? 0 : 1;
        constexpr int bx = cz != 0 ? 2 : 1;
        constexpr int sa = ax == 0 ? cx : cy;
        constexpr int sb = bx == 2 ? cz : cy;
        const float2 ja = ax == 0 ? jx : jy, jb = bx == 2 ? jz : jy;
        const float2 ua = ax == 0 ? ux : uy, ub = bx == 2 ? uz : uy;
        cj = sa > 0 ? (sb > 0 ? add2(ja, jb) : sub2(ja, jb)) : (sb > 0 ? sub2(jb, ja) : mul2(add2(ja, jb), f2(-1.f)));
        cu = sa > 0 ? (sb > 0 ? add2(ua, ub) : sub2(ua, ub)) : (sb > 0 ? sub2(ub, ua) : mul2(add2(ua, ub), f2(-1.f)));
        const float2 E = ax == 0 ? (bx == 1 ? Exy : Exz) : Eyz;
        const float2 Pab = ax == 0 ? (bx == 1 ? pxy : pxz) : pyz;
        qp = fma2(f2((float)(2 * sa * sb)), Pab, E);
      }
      const float2 e = fma2(mul2(f2(4.5f), cj), cu, base);  // even part of (feq - w) / w
      if constexpr (!BGK) {
        const float2 wt = mul2(f2(w), fma2(k1, qp, e));
        out(std::integral_constant<int, i>{}, fma2(f2(3.0f * w), cj, wt));
        if constexpr (i > 0) out(std::integral_constant<int, io>{}, fma2(f2(-3.0f * w), cj, wt));
      } else {
        const float2 we = mul2(f2(w), e);
        out(std::integral_constant<int, i>{}, fma2(a, fma2(f2(3.0f * w), cj, we), mul2(omega, h[i])));
        if constexpr (i > 0)
          out(std::integral_constant<int, io>{}, fma2(a, fma2(f2(-3.0f * w), cj, we), mul2(omega, h[io])));
      }
    }
  });
}

// collide_shifted2x with the reference's closure: molecular tau0, outlet sponge, wall floor and
// the Smagorinsky eddy viscosity
template <class L, bool BGK, class Emit>
__device__ __forceinline__ void collide_shifted2(const wt_kparams& P, const float2 (&h)[L::Q], int x, Emit&& emit,
                                                 float t_floor = 0.0f) {
  auto ofn = [&](float2 /*rho*/, float2 irho, float2, float2, float2, float2 pxx, float2 pyy, float2 pzz,
                 float2 pxy, float2 pxz, float2 pyz) {
    float2 omega;
    if (P.csmag2 > 0.0f || P.sponge_start < (float)P.nx || t_floor > P.tau0) {
      float2 pn = fma2(pxx, pxx, fma2(pyy, pyy, mul2(f2(2.f), mul2(pxy, pxy))));
      if constexpr (L::DIM == 3) pn = fma2(pzz, pzz, fma2(f2(2.f), fma2(pxz, pxz, mul2(pyz, pyz)), pn));
      relax_cell(P, (float)x, pn.x, irho.x, omega.x, t_floor);
      relax_cell(P, (float)(x + 1), pn.y, irho.y, omega.y, t_floor);
    } else {
      omega = f2(1.0f - __fdividef(1.0f, P.tau0));
    }
    return omega;
  };
  if (P.sponge_in > 0.0f && (float)x < P.sponge_in) collide_shifted2x<L, BGK, SP_ON>(P, h, x, emit, ofn);
  else collide_shifted2x<L, BGK, SP_OFF>(P, h, x, emit, ofn);
}

// the learned closure with the two cells' eddy viscosities given (face rows)
template <class L, bool BGK, class Emit>
__device__ __forceinline__ void collide_shifted2_nu(const wt_kparams& P, const float2 (&h)[L::Q], int x, Emit&& emit,
                                                    float t_floor, float2 nu) {
  auto ofn = [&](float2, float2, float2, float2, float2, float2, float2, float2, float2, float2, float2) {
    const float ta = tau0_eff(P, (float)x, t_floor) + 3.0f * nu.x;
    const float tb = tau0_eff(P, (float)(x + 1), t_floor) + 3.0f * nu.y;
    return make_float2(1.0f - __fdividef(1.0f, ta), 1.0f - __fdividef(1.0f, tb));
  };
  if (P.sponge_in > 0.0f && (float)x < P.sponge_in) collide_shifted2x<L, BGK, SP_ON>(P, h, x, emit, ofn);
  else collide_shifted2x<L, BGK, SP_OFF>(P, h, x, emit, ofn);
}

// the closure features of two cells (the moments of the pulled populations) into rows
// xrow, xrow + 1 of x (10 floats each)
template <class L>
__device__ __forceinline__ void features2(const wt_kparams& P, const float2 (&h)[L::Q], float2 wd,
                                          float* __restrict__ x, size_t row) {
  collide_shifted2x<L, true, SP_OFF>(P, h, 0, [&](auto, float2) {},
                             [&](float2 rho, float2, float2 ux, float2 uy, float2 uz, float2 pxx, float2 pyy,
                                 float2 pzz, float2 pxy, float2 pxz, float2 pyz) {
                               float xa[CL_IN], xb[CL_IN];
                               cl_features(pxx.x, pyy.x, pzz.x, pxy.x, pxz.x, pyz.x, rho.x, ux.x, uy.x, uz.x,
                                           P.tau0, wd.x, xa);
                               cl_features(pxx.y, pyy.y, pzz.y, pxy.y, pxz.y, pyz.y, rho.y, ux.y, uy.y, uz.y,
                                           P.tau0, wd.y, xb);
#pragma unroll
                               for (int k = 0; k < CL_IN; k++) {
                                 x[row * CL_IN + k] = xa[k];
                                 x[(row + 1) * CL_IN + k] = xb[k];
                               }
                               return f2(0.0f);
                             });
}

// two-cell loads / stores of shifted populations: elements (o, o + 1), o even. Loads are split
// into a raw fetch and a later conversion so that a thread can put all of its loads in flight
// before it converts any of them.
// ---- per-cell arithmetic of the sampling pass, shared by k_macro and the fused sampling step ----
// The sampling pass (wgslLbm.ts:347-489) can run on its own (k_macro, re-reading every stored
// population) or inside the last step of a stepAndSample chunk, on the values that step stores.
// Both give the same bits: a cell's density and momentum are summed from its populations exactly
// as stored, in the order the step kernels emit them (direction 0, then each direction followed by
// its opposite), and the rest uses correctly rounded operations only.
template <class L> struct EmitOrder {
  int d[L::Q];
  constexpr EmitOrder() : d() {
    int k = 0;
    for (int i = 0; i < L::Q; i++) {
      const int io = opp<L>(i);
      if (i == 0) {
        d[k++] = 0;
      } else if (i < io) {
        d[k++] = i;
        d[k++] = io;
      }
    }
  }
};
template <class L> constexpr int emit_dir(int k) { return EmitOrder<L>().d[k]; }

template <class R> __device__ __forceinline__ R add_rn(R a, R b);
template <> __device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
template <> __device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
template <class R> __device__ __forceinline__ R mul_rn(R a, R b);
template <> __device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
template <> __device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
template <class R> __device__ __forceinline__ R div_rn(R a, R b);
template <> __device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
template <> __device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }

// velocity from the summed density and momentum, and |u|^2 (no contraction)
template <class R>
__device__ __forceinline__ void cell_velocity(R rho, R jx, R jy, R jz, R& ux, R& uy, R& uz, R& uu) {
  const R ir = div_rn((R)1, rho);
  ux = mul_rn(jx, ir);
  uy = mul_rn(jy, ir);
  uz = mul_rn(jz, ir);
  uu = add_rn(add_rn(mul_rn(ux, ux), mul_rn(uy, uy)), mul_rn(uz, uz));
}

// Accumulators of one thread. k_macro sums the densities in FP64 (MacroSums). The fused sampling
// step (SampleSums) sums a thread's densities in FP64, then each warp's sum goes into 2^-30 fixed
// point: an f32 density in [1/128, 16) is an integer multiple of 2^-30, so every partial sum is
// exact and the totals do not depend on the order of the atomics; they equal the FP64 sums of the
// same densities, which are exact too for densities in [0.5, 2) on grids below 2^28 cells. A
// density outside [1/128, 16) (an unstable run) is counted in `nbig` and makes the fused sums NaN.
struct MacroSums {
  double rho_ref = 0.0, mass = 0.0;
  float maxuu = 0.0f;
  uint32_t nref = 0, nan = 0, nfluid = 0, nbig = 0;
  template <class R> __device__ __forceinline__ void density(R rho, bool ref) {
    if (ref) {
      rho_ref += (double)rho;
      nref++;
    }
    mass += (double)rho;
    nfluid++;
  }
};
struct SampleSums {
  double rho_ref = 0.0, mass = 0.0;
  float maxuu = 0.0f;
  uint32_t nref = 0, nan = 0, nfluid = 0, nbig = 0;
  __device__ __forceinline__ void density(float rho, bool ref) {
    nfluid++;
    if (ref) nref++;
    if (!(rho >= 0.0078125f && rho < 16.0f)) {
      nbig++;
      return;
    }
    mass += (double)rho;
    if (ref) rho_ref += (double)rho;
  }
};
constexpr double SMP_FIXED = 1073741824.0;  // 2^30

// Everything the sampling pass does with one fluid cell after its moments: the instability test,
// the velocity texel (half4, returned), the EMA statistics and the accumulators. `m` / `mb` are the
// cell's EMA state when `loaded`, else they are read here if needed (ema_alpha != 0, or a
// non-finite value with ema_alpha == 0, where 0 x NaN must still poison the means).
template <class R, class Sums>
__device__ __forceinline__ uint2 fluid_sample(const wt_kparams& P, size_t idx, int ix, R rho, R ux, R uy, R uz, R uu,
                                              float4* __restrict__ meanA, float* __restrict__ meanB, float4 m,
                                              float mb, bool loaded, Sums& acc) {
  const float a = P.ema_alpha;
  const bool bad = !(uu < (R)1.0e6) || !(rho > (R)0);
  const float o0 = (float)ux, o1 = (float)uy, o2 = (float)uz, o3 = (float)rho;
  acc.maxuu = fmaxf(acc.maxuu, bad ? 1.0e6f : (float)uu);
  acc.nan += bad ? 1u : 0u;
  acc.density(rho, (uint32_t)ix == P.ref_x);
  const bool finite = isfinite(o0) && isfinite(o1) && isfinite(o2) && isfinite(o3) && isfinite((float)uu);
  if (a != 0.0f || !finite) {
    if (!loaded) {
      m = meanA[idx];
      mb = meanB[idx];
    }
    m.x = m.x * (1.0f - a) + o0 * a;
    m.y = m.y * (1.0f - a) + o1 * a;
    m.z = m.z * (1.0f - a) + o2 * a;
    m.w = m.w * (1.0f - a) + o3 * a;
    meanA[idx] = m;
    meanB[idx] = mb * (1.0f - a) + (float)uu * a;
  }
  __half2 h01 = __floats2half2_rn(o0, o1);
  __half2 h23 = __floats2half2_rn(o2, o3);
  return make_uint2(*reinterpret_cast<uint32_t*>(&h01), *reinterpret_cast<uint32_t*>(&h23));
}

// The sampling pass fused into a step: where the step's last kernels put the per-cell results.
// `sets` holds SMP_SETS sets of accumulators, one 128-byte line each (SS_* slots), zeroed before
// the step; warps add into set (warp index % SMP_SETS), so the atomics spread over 64 lines.
constexpr int SMP_SETS = 64;
constexpr int SMP_SET_U64 = 16;
enum { SS_MAX = 0, SS_NAN, SS_NREF, SS_NFLUID, SS_NBIG, SS_RHOREF, SS_MASS, SS_COUNT };
constexpr int SS_DONE = SMP_SET_U64 - 1;  // set 0: blocks of k_sample_post that have finished
static_assert(SMP_SETS * SMP_SET_U64 * sizeof(unsigned long long) == SMP_SETS_BYTES, "accumulator sets");
struct SampleOut {
  uint2* vel;
  float4* meanA;
  float* meanB;
  unsigned long long* sets;
};

// warp-wide: adds the lanes' accumulators into one set (every lane of the warp calls it)
__device__ __forceinline__ void smp_flush(const SampleSums& acc, unsigned long long* __restrict__ sets,
                                          uint32_t warp_id) {
  const unsigned full = 0xffffffffu;
  const uint32_t nfluid = __reduce_add_sync(full, acc.nfluid);
  if (nfluid == 0u) return;  // uniform across the warp
  const uint32_t mx = __reduce_max_sync(full, __float_as_uint(acc.maxuu));  // values >= 0
  const uint32_t nan = __reduce_add_sync(full, acc.nan);
  const uint32_t nref = __reduce_add_sync(full, acc.nref);
  const uint32_t nbig = __reduce_add_sync(full, acc.nbig);
  double rr = acc.rho_ref, ms = acc.mass;  // exact warp sums (see SampleSums)
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    rr += __shfl_xor_sync(full, rr, o);
    ms += __shfl_xor_sync(full, ms, o);
  }
  const uint32_t lane = threadIdx.x & 31u;
  unsigned long long* set = sets + (size_t)(warp_id % SMP_SETS) * SMP_SET_U64;
  if (lane == SS_MAX) {
    atomicMax(set + SS_MAX, (unsigned long long)mx);
  } else if (lane < SS_COUNT) {
    const unsigned long long v =
        lane == SS_NAN ? nan : lane == SS_NREF ? nref : lane == SS_NFLUID ? nfluid : lane == SS_NBIG ? nbig
        : lane == SS_RHOREF ? (unsigned long long)__double2ll_rn(rr * SMP_FIXED)
                            : (unsigned long long)__double2ll_rn(ms * SMP_FIXED);
    atomicAdd(set + lane, v);
  }
}

__device__ __forceinline__ uint32_t global_warp_id() {
  const uint32_t b = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  const uint32_t t = (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
  return b * ((blockDim.x * blockDim.y * blockDim.z + 31u) / 32u) + t / 32u;
}

// Sampling state of two cells (f32x2 lanes) while a pair kernel emits them: their density and
// momentum summed from the stored values in emission order (lane-wise IEEE adds, as the scalar
// sums of k_macro).
struct PairMoments {
  float2 rho, jx, jy, jz;
  // called with the directions in emission order, which starts with direction 0
  template <class L, int I>
  __device__ __forceinline__ void add(float2 f) {
    constexpr int cx = L::c[I][0], cy = L::c[I][1], cz = L::c[I][2];
    if constexpr (I == 0) {
      rho = f;
      jx = jy = jz = make_float2(0.0f, 0.0f);
    } else {
      rho = __fadd2_rn(rho, f);
    }
    if constexpr (cx > 0) jx = __fadd2_rn(jx, f);
    if constexpr (cx < 0) jx = __fadd2_rn(jx, make_float2(-f.x, -f.y));
    if constexpr (cy > 0) jy = __fadd2_rn(jy, f);
    if constexpr (cy < 0) jy = __fadd2_rn(jy, make_float2(-f.x, -f.y));
    if constexpr (cz > 0) jz = __fadd2_rn(jz, f);
    if constexpr (cz < 0) jz = __fadd2_rn(jz, make_float2(-f.x, -f.y));
  }
};

// The two cells of a pair kernel (x0, x0 + 1; x0 even) once their outputs were emitted into `pm`:
// velocity texels (one 16-byte store), EMA statistics, accumulators.
template <class L>
__device__ __forceinline__ void pair_sample(const wt_kparams& P, uint32_t idx0, int x0, const PairMoments& pm,
                                            const SampleOut& O, SampleSums& acc) {
  float ux, uy, uz, uu;
  cell_velocity<float>(pm.rho.x, pm.jx.x, pm.jy.x, pm.jz.x, ux, uy, uz, uu);
  const uint2 ta = fluid_sample<float>(P, idx0, x0, pm.rho.x, ux, uy, uz, uu, O.meanA, O.meanB,
                                       make_float4(0.f, 0.f, 0.f, 0.f), 0.0f, false, acc);
  cell_velocity<float>(pm.rho.y, pm.jx.y, pm.jy.y, pm.jz.y, ux, uy, uz, uu);
  const uint2 tb = fluid_sample<float>(P, idx0 + 1u, x0 + 1, pm.rho.y, ux, uy, uz, uu, O.meanA, O.meanB,
                                       make_float4(0.f, 0.f, 0.f, 0.f), 0.0f, false, acc);
  *reinterpret_cast<uint4*>(O.vel + idx0) = make_uint4(ta.x, ta.y, tb.x, tb.y);
}

// Population loads. The step kernels read their input buffer through the read-only cache (ld.nc):
// nothing writes it while they run. COH selects loads cached in L2 only (ld.cg) instead, for the
// persistent kernel, whose blocks read in one step what other SMs wrote in the step before.
template <bool COH, class T>
__device__ __forceinline__ T ldp(const T* p) {
  if constexpr (COH) return __ldcg(p);
  else return __ldg(p);
}

// Per-direction population plane bases of a step, computed on the host and passed by value, so a
// thread reaches direction i's source or destination with one multiply-add from the constant
// bank: in[i] = fin + i N - c_iy nx - c_iz nx ny (the plane of direction i shifted back by c_i
// along y and z; a bulk cell's index lands inside the buffer), out[i] = fout + i N.
template <class T> struct DirPtrs {
  const T* in[19];
  T* out[19];
};
template <class S> struct PairIO;
template <> struct PairIO<StF16> {
  typedef uint32_t pair_t;
  typedef unsigned short one_t;
  template <bool COH = false>
  __device__ __forceinline__ static pair_t ld(const __half* __restrict__ p, uint32_t o) {
    return ldp<COH>(reinterpret_cast<const unsigned int*>(p + o));
  }
  template <bool COH = false>
  __device__ __forceinline__ static one_t ld1(const __half* __restrict__ p, uint32_t o) {
    return ldp<COH>(reinterpret_cast<const unsigned short*>(p + o));
  }
  // elements (o .. o + 3), o a multiple of 4: one 8-byte load
  template <bool COH = false>
  __device__ __forceinline__ static void ld4(const __half* __restrict__ p, uint32_t o, pair_t& a, pair_t& b) {
    const uint2 q = ldp<COH>(reinterpret_cast<const uint2*>(p + o));
    a = q.x;
    b = q.y;
  }
  __device__ __forceinline__ static float2 cvt(pair_t u, float /*w*/) {
    return __half22float2(*reinterpret_cast<const __half2*>(&u));
  }
  __device__ __forceinline__ static float cvt1(one_t u, float /*w*/) {
    return __half2float(*reinterpret_cast<const __half*>(&u));
  }
  __device__ __forceinline__ static void st(__half* __restrict__ p, uint32_t o, float2 v, float /*w*/) {
    *reinterpret_cast<__half2*>(p + o) = __float22half2_rn(v);
  }
  // st as one predicated store (no branch around it): nothing is written unless c
  __device__ __forceinline__ static void st_if(__half* __restrict__ p, uint32_t o, float2 v, float, bool c) {
    const __half2 h = __float22half2_rn(v);
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t@q st.global.b32 [%0], %1;\n\t}" ::"l"(p + o),
                 "r"(*reinterpret_cast<const uint32_t*>(&h)), "r"((uint32_t)c)
                 : "memory");
  }
  // the populations st stores for v, as a later pass reads them back (f = stored + w)
  __device__ __forceinline__ static float2 readback(float2 v, float w) {
    const __half2 h = __float22half2_rn(v);
    return make_float2(h2f_add(__low2half(h), w), h2f_add(__high2half(h), w));
  }
};
template <> struct PairIO<StF32> {
  typedef float2 pair_t;
  typedef float one_t;
  template <bool COH = false>
  __device__ __forceinline__ static pair_t ld(const float* __restrict__ p, uint32_t o) {
    return ldp<COH>(reinterpret_cast<const float2*>(p + o));
  }
  template <bool COH = false>
  __device__ __forceinline__ static one_t ld1(const float* __restrict__ p, uint32_t o) { return ldp<COH>(p + o); }
  // elements (o .. o + 3), o a multiple of 4: one 16-byte load
  template <bool COH = false>
  __device__ __forceinline__ static void ld4(const float* __restrict__ p, uint32_t o, pair_t& a, pair_t& b) {
    const float4 q = ldp<COH>(reinterpret_cast<const float4*>(p + o));
    a = make_float2(q.x, q.y);
    b = make_float2(q.z, q.w);
  }
  __device__ __forceinline__ static float2 cvt(pair_t f, float w) { return make_float2(f.x - w, f.y - w); }
  __device__ __forceinline__ static float cvt1(one_t f, float w) { return f - w; }
  __device__ __forceinline__ static void st(float* __restrict__ p, uint32_t o, float2 v, float w) {
    *reinterpret_cast<float2*>(p + o) = make_float2(__fadd_rn(v.x, w), __fadd_rn(v.y, w));
  }
  __device__ __forceinline__ static void st_if(float* __restrict__ p, uint32_t o, float2 v, float w, bool c) {
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %3, 0;\n\t@q st.global.v2.f32 [%0], {%1, %2};\n\t}" ::"l"(p + o),
                 "f"(__fadd_rn(v.x, w)), "f"(__fadd_rn(v.y, w)), "r"((uint32_t)c)
                 : "memory");
  }
  __device__ __forceinline__ static float2 readback(float2 v, float w) {
    return make_float2(__fadd_rn(v.x, w), __fadd_rn(v.y, w));
  }
};

// MINB: CTAs of 256 threads the register allocation must leave room for (0 = no constraint)
template <int MINB> struct Bounds { static constexpr int v = MINB; };

// The V cells x0 .. x0 + V - 1 of row (iy, iz) (bulk rows only); shared by the single-tunnel
// kernel and the batch kernel.
// With SMP the cells also run the per-cell part of the sampling pass on what they store.
template <class L, class S, int V, bool BGK, bool SMP = false, bool COH = false, bool TAB = false>
__device__ __forceinline__ void bulk_cells(const wt_kparams& P, const typename S::T* __restrict__ fin,
                                           typename S::T* __restrict__ fout, const uint8_t* __restrict__ cls,
                                           int gs, int x0, int iy, int iz, const SampleOut* O = nullptr,
                                           SampleSums* acc = nullptr, const DirPtrs<typename S::T>* D = nullptr) {
  typedef PairIO<S> IO;
  constexpr int Q = L::Q;
  constexpr bool D3 = L::DIM == 3;
  constexpr int G = V / 2;  // groups of two cells collided together in f32x2 lanes
  const int NX = P.nx, NY = P.ny, NZ = P.nz;
  if (x0 >= NX || iy >= NY) return;
  // rows on the domain faces belong to k_face_v, groups holding solid / near-solid cells to
  // k_boundary_tab (fluid cells) or to nobody (solid cells keep the rest state)
  if (iy == 0 || iy == NY - 1 || (D3 && (iz == 0 || iz == NZ - 1))) return;
  const uint32_t N = P.n;
  const uint32_t sy = (uint32_t)NX, sz = (uint32_t)NX * (uint32_t)NY;
  const uint32_t idx0 = (uint32_t)x0 + sy * (uint32_t)iy + sz * (uint32_t)iz;
  uint32_t cv;
  if (gs == 4) cv = __ldg(reinterpret_cast<const unsigned int*>(cls + (idx0 & ~3u)));
  else cv = __ldg(reinterpret_cast<const unsigned short*>(cls + idx0));
  // groups holding solid / near-solid cells are not written here; their loads are still
  // issued (every address is inside the domain for an interior row) so that the class byte does
  // not add a memory round trip in front of the population loads, and only the stores are skipped
  const bool clean = (cv & 0x03030303u) == 0u;
  // phase 1: every load of the V cells in flight (bulk cells: y - cy, z - cz inside the domain)
  typename IO::pair_t rp[G][Q];
  typename IO::one_t r1[Q];
  const bool last = x0 + V >= NX;
  // TAB: direction i's source is D->in[i] + idx0 (one multiply-add from the constant bank);
  // otherwise one 64-bit base per thread, and each direction adds an offset that is the same for
  // every thread (plane i, shifted back by c_i along y and z)
  const typename S::T* fb = fin + idx0;
  typename S::T* ob = fout + idx0;
  const uint32_t idxm = x0 > 0 ? idx0 - 1u : idx0, idxp = idx0 + (uint32_t)(last ? V - 1 : V);
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    [[maybe_unused]] constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
    const typename S::T* ps;
    if constexpr (TAB) {
      ps = D->in[i] + idx0;
    } else {
      const ptrdiff_t off = (ptrdiff_t)i * N - (ptrdiff_t)cy * sy - (ptrdiff_t)cz * sz;
      ps = fb + off;
    }
    if constexpr (G == 2) {
      IO::template ld4<COH>(ps, 0u, rp[0][i], rp[1][i]);  // 8- or 16-byte aligned when nx % 4 == 0
    } else {
#pragma unroll
      for (int g = 0; g < G; g++) rp[g][i] = IO::template ld<COH>(ps, 2 * g);
    }
    if constexpr (TAB) {
      if constexpr (cx > 0) r1[i] = IO::template ld1<COH>(D->in[i] + idxm, 0u);
      if constexpr (cx < 0) r1[i] = IO::template ld1<COH>(D->in[i] + idxp, 0u);
    } else {
      if constexpr (cx > 0) r1[i] = IO::template ld1<COH>(x0 > 0 ? ps - 1 : ps, 0u);     // x - 1
      if constexpr (cx < 0) r1[i] = IO::template ld1<COH>(ps + (last ? V - 1 : V), 0u);  // x + 1, outlet clamp
    }
  });
  // phase 2, one pair of cells at a time (the other pairs stay packed in their raw registers):
  // convert and shift into the pulled populations, collide, store
#pragma unroll
  for (int g = 0; g < G; g++) {
    float2 h[Q];
    static_for<Q>([&](auto I) {
      constexpr int i = I;
      constexpr int cx = L::c[i][0];
      constexpr float w = (float)Wc<L, i>::v;
      const float2 cur = IO::cvt(rp[g][i], w);
      if constexpr (cx == 0) {
        h[i] = cur;
      } else if constexpr (cx > 0) {
        h[i] = make_float2(g == 0 ? IO::cvt1(r1[i], w) : IO::cvt(rp[g > 0 ? g - 1 : 0][i], w).y, cur.x);
      } else {
        h[i] = make_float2(cur.y, g == G - 1 ? IO::cvt1(r1[i], w) : IO::cvt(rp[g < G - 1 ? g + 1 : g][i], w).x);
      }
    });
    if (g == 0 && x0 == 0) {
      // inlet column: populations entering from x < 0 are the free-stream equilibrium
      const float U = P.uin;
      static_for<Q>([&](auto I) {
        constexpr int i = I;
        constexpr int cx = L::c[i][0];
        if constexpr (cx > 0) {
          constexpr float w = (float)Wc<L, i>::v;
          h[i].x = w * P.rho_in * (1.0f + 3.0f * U + 4.5f * U * U - 1.5f * U * U) - w;
        }
      });
    }
    PairMoments pm;
    collide_shifted2<L, BGK>(P, h, x0 + 2 * g, [&](auto I, float2 v) {
      constexpr int i = decltype(I)::value;
      if constexpr (TAB) IO::st_if(D->out[i] + idx0, 2 * g, v, (float)Wc<L, i>::v, clean);
      else IO::st_if(ob + (ptrdiff_t)i * N, 2 * g, v, (float)Wc<L, i>::v, clean);
      if constexpr (SMP) pm.template add<L, i>(IO::readback(v, (float)Wc<L, i>::v));
    });
    if constexpr (SMP) {
      if (clean) pair_sample<L>(P, idx0 + 2u * (uint32_t)g, x0 + 2 * g, pm, *O, *acc);
    }
  }
}

// zrev != 0 sweeps the z-planes in descending order (block z index nz - 1 - blockIdx.z). Steps
// alternate the direction, so each step starts on the planes the previous step wrote last, which
// are still in L2 (the two population buffers are larger than L2; a fixed order would always
// start on the planes evicted first). Every cell's result is the same in either order.
// SMP: the last step of a stepAndSample chunk, which also runs the sampling pass's per-cell work
// on its bulk cells (accumulators flushed per warp into O.sets).
template <class L, class S, int V, int MINB, bool BGK, bool SMP = false>
__global__ void __launch_bounds__(256, MINB > 0 ? MINB : 1) k_stream_collide_v(const __grid_constant__ wt_kparams P,
                                                          const typename S::T* __restrict__ fin,
                                                          typename S::T* __restrict__ fout,
                                                          const uint8_t* __restrict__ cls, int gs, int zrev,
                                                          const __grid_constant__ SampleOut O,
                                                          const __grid_constant__ DirPtrs<typename S::T> D) {
  SampleSums acc;
  bulk_cells<L, S, V, BGK, SMP, false, true>(P, fin, fout, cls, gs, (blockIdx.x * blockDim.x + threadIdx.x) * V,
                                blockIdx.y * blockDim.y + threadIdx.y,
                                zrev ? (int)(gridDim.z - 1u - blockIdx.z) : (int)blockIdx.z, &O, &acc, &D);
  if constexpr (SMP) smp_flush(acc, O.sets, global_warp_id());
}

// ---- row pipeline: interior rows streamed through shared memory by bulk copies ---------------
//
// In k_stream_collide_v every thread's loads sit in front of its own collision, so memory latency
// is hidden only by other warps. Here the loads of a block's next rows are in flight while its
// current row collides: a producer warp streams whole interior rows into a ring of RP_STAGES
// shared-memory stages with 1-D bulk copies (cp.async.bulk, completion counted in bytes on the
// stage's mbarrier), and four consumer warps collide two cells per thread from shared memory and
// store to global memory directly. For direction i the source row (y - c_iy, z - c_iz) of plane i
// is one contiguous copy of nx populations; whole rows need no x halo, since x - 1 at the inlet is
// replaced by the inlet equilibrium and x + 1 at the outlet is clamped, as in the vectorised
// kernel. Block b takes `rows` consecutive interior rows (row r: y = 1 + r % (ny - 2),
// z = 1 + r / (ny - 2)). Rows of plane i start 16-byte aligned when nx % 8 == 0 (f16) or
// nx % 4 == 0 (f32); the ring must fit the default 48 KB of shared memory. Every wait is bounded: a
// timeout sets bit 8 of the error word and the block stores nothing more. Consumers release a stage
// after reading it; the producer reuses it only after all four consumer warps have.
// Teardown: no block may exit while a bulk copy it issued can still write its shared memory. A
// consumer warp whose wait on a stage gives up raises a shared abort flag before it releases the
// stage, so the producer, which reads the flag after each wait on a released stage, never issues a
// copy into a stage whose previous copy may still be landing. Every copy but the last one issued
// into each stage was therefore waited for by the consumers; before exiting, the producer waits
// (bounded) for those last ones.
constexpr int RP_CONSUMERS = 128;              // four consumer warps, two cells per thread
constexpr int RP_THREADS = RP_CONSUMERS + 32;  // and one producer warp
constexpr int RP_STAGES = 3;
constexpr int RP_MINB = 6;                     // blocks per SM the registers are capped for
constexpr uint32_t RP_WAIT_LIMIT = 1u << 22;  // polls per wait (the consumers' limit is a parameter)

__device__ __forceinline__ void rp_copy_row(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}
__device__ __forceinline__ void rp_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(mbar),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void rp_arrive(uint32_t mbar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(mbar) : "memory");
}

template <class S, bool BGK>
__global__ void __launch_bounds__(RP_THREADS, RP_MINB) k_stream_collide_rows(const __grid_constant__ wt_kparams P,
                                                                          const typename S::T* __restrict__ fin,
                                                                          typename S::T* __restrict__ fout,
                                                                          const uint8_t* __restrict__ cls, int gs,
                                                                          uint32_t nrows, uint32_t rows,
                                                                          uint32_t cwait, int* __restrict__ err) {
  typedef D3Q19 L;
  typedef PairIO<S> IO;
  typedef typename S::T T;
  constexpr int Q = L::Q;
  extern __shared__ __align__(128) uint8_t rp_smem[];
  const int NX = P.nx, NY = P.ny;
  const uint32_t N = P.n;
  const uint32_t sy = (uint32_t)NX, sz = (uint32_t)NX * (uint32_t)NY;
  const uint32_t stage_elems = (uint32_t)Q * (uint32_t)NX;
  T* const ring = reinterpret_cast<T*>(rp_smem);
  uint64_t* const full = reinterpret_cast<uint64_t*>(rp_smem + (size_t)RP_STAGES * stage_elems * sizeof(T));
  uint64_t* const empty = full + RP_STAGES;
  volatile uint32_t* const abort_flag = reinterpret_cast<volatile uint32_t*>(empty + RP_STAGES);
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
  const uint32_t row0 = blockIdx.x * rows;
  const uint32_t nblk = min(rows, nrows - row0);
  const uint32_t iny = (uint32_t)(NY - 2);
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < RP_STAGES; k++) {
      umma::mbar_init(full + k, 1);
      umma::mbar_init(empty + k, RP_CONSUMERS / 32);
    }
    *abort_flag = 0u;
  }
  __syncthreads();
  bool ok = true;
  if (warp == RP_CONSUMERS / 32) {
    // producer: lane 0 announces the stage's bytes, lanes 0 .. 18 copy one direction's row each
    ptrdiff_t off = 0;  // plane i, shifted back by c_i along y and z
    static_for<Q>([&](auto I) {
      constexpr int i = I;
      constexpr int cy = L::c[i][1], cz = L::c[i][2];
      if (lane == (uint32_t)i) off = (ptrdiff_t)i * N - (ptrdiff_t)cy * sy - (ptrdiff_t)cz * sz;
    });
    uint32_t issued = 0;
    for (uint32_t j = 0; j < nblk && ok; j++) {
      const uint32_t st = j % RP_STAGES;
      if (j >= RP_STAGES) {
        ok = umma::mbar_wait(empty + st, ((j / RP_STAGES) - 1u) & 1u, RP_WAIT_LIMIT);
        // a consumer that gave up on this stage's previous copy raised the flag before releasing it
        if (ok && *abort_flag != 0u) break;
      }
      if (!ok) break;
      const uint32_t r = row0 + j;
      const uint32_t iy = 1u + r % iny, iz = 1u + r / iny;
      const uint32_t fb = umma::smem_u32(full + st);
      if (lane == 0) rp_expect_tx(fb, stage_elems * (uint32_t)sizeof(T));
      __syncwarp();
      if (lane < (uint32_t)Q)
        rp_copy_row(umma::smem_u32(ring + (size_t)st * stage_elems + (size_t)lane * NX),
                    fin + ((ptrdiff_t)(sy * iy + sz * iz) + off), (uint32_t)NX * (uint32_t)sizeof(T), fb);
      issued = j + 1;
    }
    // drain: the last copy issued into each stage has landed before the block may exit
    const uint32_t first = issued > (uint32_t)RP_STAGES ? issued - (uint32_t)RP_STAGES : 0u;
    for (uint32_t j = first; j < issued; j++)
      ok = umma::mbar_wait(full + j % RP_STAGES, (j / RP_STAGES) & 1u, RP_WAIT_LIMIT) && ok;
  } else {
    for (uint32_t j = 0; j < nblk; j++) {
      const uint32_t st = j % RP_STAGES;
      const uint32_t r = row0 + j;
      const uint32_t iy = 1u + r % iny, iz = 1u + r / iny;
      const uint32_t rowbase = sy * iy + sz * iz;
      int x0 = 2 * (int)tid;
      auto cls_of = [&](int x) -> uint32_t {
        const uint32_t idx = rowbase + (uint32_t)x;
        return gs == 4 ? __ldg(reinterpret_cast<const unsigned int*>(cls + (idx & ~3u)))
                       : (uint32_t)__ldg(reinterpret_cast<const unsigned short*>(cls + idx));
      };
      uint32_t cv = x0 < NX ? cls_of(x0) : 0u;  // in flight during the wait
      const bool landed = umma::mbar_wait(full + st, (j / RP_STAGES) & 1u, cwait);
      if (!landed && lane == 0) *abort_flag = 1u;  // before this warp releases the stage below
      ok = landed && ok;
      const T* const sp0 = ring + (size_t)st * stage_elems;
      for (; x0 < NX; x0 += 2 * RP_CONSUMERS) {
        if (x0 != 2 * (int)tid) cv = cls_of(x0);
        const bool clean = (cv & 0x03030303u) == 0u && ok;
        const bool last = x0 + 2 >= NX;
        float2 h[Q];
        static_for<Q>([&](auto I) {
          constexpr int i = I;
          constexpr int cx = L::c[i][0];
          constexpr float w = (float)Wc<L, i>::v;
          const T* sp = sp0 + i * NX;
          const float2 cur = IO::cvt(*reinterpret_cast<const typename IO::pair_t*>(sp + x0), w);
          if constexpr (cx == 0) {
            h[i] = cur;
          } else if constexpr (cx > 0) {
            h[i] = make_float2(IO::cvt1(*reinterpret_cast<const typename IO::one_t*>(sp + (x0 > 0 ? x0 - 1 : x0)), w),
                               cur.x);
          } else {
            h[i] = make_float2(cur.y,
                               IO::cvt1(*reinterpret_cast<const typename IO::one_t*>(sp + (last ? x0 + 1 : x0 + 2)), w));
          }
        });
        if (x0 == 0) {
          // inlet column: populations entering from x < 0 are the free-stream equilibrium
          const float U = P.uin;
          static_for<Q>([&](auto I) {
            constexpr int i = I;
            constexpr int cx = L::c[i][0];
            if constexpr (cx > 0) {
              constexpr float w = (float)Wc<L, i>::v;
              h[i].x = w * P.rho_in * (1.0f + 3.0f * U + 4.5f * U * U - 1.5f * U * U) - w;
            }
          });
        }
        T* const ob = fout + rowbase + (uint32_t)x0;
        collide_shifted2<L, BGK>(P, h, x0, [&](auto I, float2 v) {
          constexpr int i = decltype(I)::value;
          if (clean) IO::st(ob + (ptrdiff_t)i * N, 0u, v, (float)Wc<L, i>::v);
        });
      }
      // this warp has read the stage: release it to the producer
      __syncwarp();
      if (lane == 0) rp_arrive(umma::smem_u32(empty + st));
    }
  }
  if (!ok) atomicOr(err, 8);
}

// dynamic shared memory of the row pipeline (stages and barriers), 0 where it does not apply
template <class S>
static size_t rows_smem_bytes(const wt_solver* s) {
  const int nx = s->dims.nx;
  const int align = 16 / (int)sizeof(typename S::T);
  if (!s->is3d || nx % align != 0 || nx < 8 || s->dims.ny < 3 || s->dims.nz < 3) return 0;
  // the ring, full and empty barriers per stage, the abort flag (padded to 8 bytes)
  const size_t b = (size_t)RP_STAGES * 19 * (size_t)nx * sizeof(typename S::T) + 2 * RP_STAGES * sizeof(uint64_t) + 8;
  return b <= 48 * 1024 ? b : 0;
}

// The bulk rows of every tunnel of a batch (D3Q19, two cells per thread): block b belongs to the
// tunnel m with tile0[m] <= b < tile0[m + 1], and covers tile b - tile0[m] of its grid.
// The block's tunnel parameters are copied to shared memory once, so the body reads them with
// uniform shared loads instead of indexed constant-bank loads.
template <class S, int MINB, bool BGK>
__global__ void __launch_bounds__(256, MINB > 0 ? MINB : 1) k_batch_bulk(const __grid_constant__ BatchTable T) {
  __shared__ uint32_t member;
  __shared__ wt_kparams sp;
  const uint32_t tid = threadIdx.x + blockDim.x * threadIdx.y;
  if (tid == 0) {
    uint32_t lo = 0, hi = T.count;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (T.tile0[mid] <= blockIdx.x) lo = mid;
      else hi = mid;
    }
    member = lo;
  }
  __syncthreads();
  const uint32_t m = member;
  static_assert(sizeof(wt_kparams) % 4 == 0 && sizeof(wt_kparams) / 4 <= 32, "parameter block copy");
  if (tid < sizeof(wt_kparams) / 4)
    reinterpret_cast<uint32_t*>(&sp)[tid] = reinterpret_cast<const uint32_t*>(&T.t[m].P)[tid];
  __syncthreads();
  const BatchTunnel& t = T.t[m];
  const uint32_t tile = blockIdx.x - T.tile0[m];
  const uint32_t bx = tile % t.tiles_x, by = (tile / t.tiles_x) % t.tiles_y, bz = tile / (t.tiles_x * t.tiles_y);
  bulk_cells<D3Q19, S, 2, BGK>(sp, (const typename S::T*)t.fin, (typename S::T*)t.fout, t.cls, t.gs,
                               (int)(bx * blockDim.x + threadIdx.x) * 2, (int)(by * blockDim.y + threadIdx.y),
                               (int)bz);
}

// Rows on the domain faces (y = 0 or ny - 1, and z = 0 or nz - 1 in 3-D), vectorised like the
// bulk. The boundary rule of a direction is the same along a whole row, so each direction's source
// is a (population plane, row, x shift) triple chosen once per row (wgslLbm.ts:138-175): the
// specular images mirrorY / mirrorZ / mirrorYZ or the periodic image for pulls from beyond the
// roof and sides, bounce-back of the cell's own opposite population plus the belt term on a
// no-slip or moving floor, and the inlet equilibrium / zero-gradient outlet as in the bulk. Floor
// rows with bounce-back collide with BGK and the tauWall floor, like the reference's wall cells.
// Groups holding a solid or a fluid cell next to a solid are left to k_boundary_tab.
// MODE 0: Smagorinsky. With the learned closure, MODE 1 writes the features of every face cell
// (row r * nx + x of `xb`) and stores nothing; MODE 2 collides with the eddy viscosities nub[row].
enum : int { FM_SMAG = 0, FM_FEATURES = 1, FM_NU = 2 };

template <class L, class S, int MODE, bool SMP = false, bool COH = false>
__device__ __forceinline__ void face_rows(const wt_kparams& P, const typename S::T* __restrict__ fin,
                                          typename S::T* __restrict__ fout, const uint8_t* __restrict__ cls, int gs,
                                          const uint32_t* __restrict__ sdf, float* __restrict__ xb,
                                          const float* __restrict__ nub, const SampleOut* O, SampleSums* acc,
                                          int x0, int r) {
  typedef PairIO<S> IO;
  constexpr int Q = L::Q;
  constexpr bool D3 = L::DIM == 3;
  const int NX = P.nx, NY = P.ny, NZ = P.nz;
  int iy, iz;
  if constexpr (!D3) {
    if (r >= 2) return;
    iy = r == 0 ? 0 : NY - 1;
    iz = 0;
  } else {
    if (r >= 2 * NY + 2 * (NZ - 2)) return;
    if (r < NY) {
      iy = r;
      iz = 0;
    } else if (r < 2 * NY) {
      iy = r - NY;
      iz = NZ - 1;
    } else {
      const int k = r - 2 * NY;
      iz = 1 + (k >> 1);
      iy = (k & 1) ? NY - 1 : 0;
    }
  }
  if (x0 >= NX) return;
  const uint32_t N = P.n;
  const uint32_t sy = (uint32_t)NX, sz = (uint32_t)NX * (uint32_t)NY;
  const uint32_t idx0 = (uint32_t)x0 + sy * (uint32_t)iy + sz * (uint32_t)iz;
  uint32_t cv, c0, c1;
  if (gs == 4) {
    cv = __ldg(reinterpret_cast<const unsigned int*>(cls + (idx0 & ~3u)));
    const int sh = 8 * (int)(idx0 & 3u);
    c0 = (cv >> sh) & 0xffu;
    c1 = (cv >> (sh + 8)) & 0xffu;
  } else {
    cv = __ldg(reinterpret_cast<const unsigned short*>(cls + idx0));
    c0 = cv & 0xffu;
    c1 = (cv >> 8) & 0xffu;
  }
  // groups holding solid / near-solid cells belong to k_boundary_tab: their loads are still issued
  // (every source address is valid) so the class byte adds no round trip; only the stores are skipped
  const bool clean = (cv & 0x03030303u) == 0u;
  const bool gwall = iy == 0 && P.ground != 0u;
  const float2 belt = (gwall && P.ground == 2u)
                          ? make_float2((c0 & CLS_BELT_STILL) ? 0.0f : 1.0f, (c1 & CLS_BELT_STILL) ? 0.0f : 1.0f)
                          : f2(0.0f);
  const bool last = x0 + 2 >= NX;
  typename IO::pair_t rp[Q];
  typename IO::one_t r1[Q];
  bool bnc[Q];
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
    const int syy = iy - cy, szz = D3 ? iz - cz : 0;
    const bool yOut = syy < 0 || syy >= NY;
    const bool zOut = D3 && (szz < 0 || szz >= NZ);
    int k = i, ry = syy, rz = szz;
    bool bounce = false;
    if (cy > 0 && yOut && P.ground != 0u) {
      bounce = true;
      k = opp<L>(i);
      ry = iy;
      rz = iz;
    } else if (D3 && yOut && zOut) {
      k = mirYZ<L>(i);
      ry = iy;
      rz = iz;
    } else if (yOut) {
      k = mirY<L>(i);
      ry = iy;
      rz = D3 ? min(max(szz, 0), NZ - 1) : 0;
    } else if (D3 && zOut) {
      if (P.side_mode == 1u) {
        rz = (szz + NZ) % NZ;
      } else {
        k = mirZ<L>(i);
        rz = iz;
      }
    }
    bnc[i] = bounce;
    const uint32_t src = (uint32_t)k * N + sy * (uint32_t)ry + sz * (uint32_t)rz + (uint32_t)x0;
    rp[i] = IO::template ld<COH>(fin, src);
    if constexpr (cx > 0) r1[i] = IO::template ld1<COH>(fin, (x0 > 0 && !bounce) ? src - 1u : src);
    if constexpr (cx < 0) r1[i] = IO::template ld1<COH>(fin, (last || bounce) ? src + 1u : src + 2u);
  });
  float2 h[Q];
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    constexpr int cx = L::c[i][0];
    constexpr float w = (float)Wc<L, i>::v;  // mirror and opposite planes share w_i
    const float2 cur = IO::cvt(rp[i], w);
    if constexpr (cx == 0) {
      h[i] = cur;
    } else {
      if (bnc[i]) {
        h[i] = fma2(belt, f2((float)(6.0 * Wc<L, i>::v * cx) * P.u_ground), cur);
      } else if constexpr (cx > 0) {
        h[i] = make_float2(IO::cvt1(r1[i], w), cur.x);
      } else {
        h[i] = make_float2(cur.y, IO::cvt1(r1[i], w));
      }
    }
  });
  if (x0 == 0) {
    const float U = P.uin;
    static_for<Q>([&](auto I) {
      constexpr int i = I;
      constexpr int cx = L::c[i][0];
      if constexpr (cx > 0) {
        constexpr float w = (float)Wc<L, i>::v;
        h[i].x = w * P.rho_in * (1.0f + 3.0f * U + 4.5f * U * U - 1.5f * U * U) - w;
      }
    });
  }
  PairMoments pm;
  auto emit = [&](auto I, float2 v) {
    constexpr int i = decltype(I)::value;
    if (clean) IO::st(fout, i * N + idx0, v, (float)Wc<L, i>::v);
    if constexpr (SMP) pm.template add<L, i>(IO::readback(v, (float)Wc<L, i>::v));
  };
  const size_t slot = (size_t)r * (size_t)NX + (size_t)x0;
  if constexpr (MODE == FM_FEATURES) {
    const uint2 sw = __ldg(reinterpret_cast<const uint2*>(sdf + idx0));
    features2<L>(P, h, make_float2(cl_wall_dist(sw.x), cl_wall_dist(sw.y)), xb, slot);
  } else if constexpr (MODE == FM_NU) {
    const float2 nu = make_float2(__ldg(nub + slot), __ldg(nub + slot + 1));
    if (gwall) collide_shifted2_nu<L, true>(P, h, x0, emit, P.tau_wall, nu);
    else if (P.collision == 1u) collide_shifted2_nu<L, true>(P, h, x0, emit, 0.0f, nu);
    else collide_shifted2_nu<L, false>(P, h, x0, emit, 0.0f, nu);
  } else {
    if (gwall) collide_shifted2<L, true>(P, h, x0, emit, P.tau_wall);
    else if (P.collision == 1u) collide_shifted2<L, true>(P, h, x0, emit);
    else collide_shifted2<L, false>(P, h, x0, emit);
    if constexpr (SMP) {
      if (clean) pair_sample<L>(P, idx0, x0, pm, *O, *acc);
    }
  }
}

template <class L, class S, bool SMP = false>
__global__ void __launch_bounds__(256) k_face_v(const __grid_constant__ wt_kparams P,
                                                const typename S::T* __restrict__ fin,
                                                typename S::T* __restrict__ fout,
                                                const uint8_t* __restrict__ cls, int gs,
                                                const __grid_constant__ SampleOut O) {
  SampleSums acc;
  face_rows<L, S, FM_SMAG, SMP>(P, fin, fout, cls, gs, nullptr, nullptr, nullptr, &O, &acc,
                                (blockIdx.x * blockDim.x + threadIdx.x) * 2, blockIdx.y * blockDim.y + threadIdx.y);
  if constexpr (SMP) smp_flush(acc, O.sets, global_warp_id());
}

// face rows with the learned closure: MODE FM_FEATURES (inputs of the network) or FM_NU (collision
// with the network's eddy viscosities)
template <class L, class S, int MODE>
__global__ void __launch_bounds__(256) k_face_lc(const __grid_constant__ wt_kparams P,
                                                 const typename S::T* __restrict__ fin,
                                                 typename S::T* __restrict__ fout,
                                                 const uint8_t* __restrict__ cls, int gs,
                                                 const uint32_t* __restrict__ sdf, float* __restrict__ xb,
                                                 const float* __restrict__ nub) {
  face_rows<L, S, MODE>(P, fin, fout, cls, gs, sdf, xb, nub, nullptr, nullptr,
                        (blockIdx.x * blockDim.x + threadIdx.x) * 2, blockIdx.y * blockDim.y + threadIdx.y);
}

// ---- bulk kernel with the learned closure: the network on tcgen05 tensor cores -----------------
//
// Same pull as the vectorised kernel with two cells per thread (x0, x0 + 1), 128 threads per
// block. Between the moments and the relaxation the block evaluates the network for its 256 cells:
// every thread writes the bf16 inputs of its two cells as row `tid` of two 128 x 16 A tiles in
// shared memory (tile 0: cells x0, tile 1: cells x0 + 1), one thread issues the layer-1 MMAs
// (M = 128, N = 32, K = 16; tile t accumulates in tensor-memory columns 32 t .. 32 t + 31), every
// thread reads its row back (tensor-memory lane = tid), adds the bias, applies gelu and writes row
// `tid` of two 128 x 32 hidden tiles, and the layer-2 MMAs (two K = 16 steps per tile) reuse the
// same columns. The 32 -> 1 output layer and softplus run on CUDA cores. Rows of threads outside
// the interior rows carry the rest state and are not stored. Waits on the MMA barrier are bounded;
// a timeout sets bit 4 of the error word and the block stores nothing.
constexpr int LC_THREADS = 128;
constexpr uint32_t LC_TMEM_COLS = 64;
constexpr int LC_SMEM_A = 0;       // 2 tiles x 128 x 16 bf16
constexpr int LC_SMEM_H = 8192;    // 2 tiles x 128 x 32 bf16
constexpr int LC_SMEM_W1 = 24576;  // W1 image, 32 x 16 bf16 (followed by the W2 image: one 3 KB copy)
constexpr int LC_SMEM_W2 = 25600;  // W2 image, 32 x 32 bf16
constexpr int LC_SMEM_BAR = 27648; // mbarrier (8 B), the tensor-memory address (4 B), pad, drain barrier (8 B)
// dynamic shared memory per block: more than 228 KB / 8, so at most 7 blocks share an SM and their
// 7 x 64 tensor-memory columns fit in the SM's 512 (an allocation never has to wait)
constexpr int LC_SMEM_BYTES = 29 * 1024;
constexpr uint32_t LC_WAIT_LIMIT = 1u << 22;
constexpr int LC_SMEM_DRAIN = LC_SMEM_BAR + 16;
static_assert(LC_SMEM_DRAIN + 8 <= LC_SMEM_BYTES, "shared-memory layout");
static_assert(offsetof(ClosureDev, w2img) == offsetof(ClosureDev, w1img) + 1024, "weight images are contiguous");

// row r of a 128 x 16 A tile: the normalised, bf16-rounded features (10) and zero padding
__device__ __forceinline__ void lc_write_inputs(uint8_t* tile, uint32_t r, const float (&x)[CL_IN],
                                                const ClosureParams& CP) {
  uint32_t w[5];
#pragma unroll
  for (int k = 0; k < 5; k++)
    w[k] = bf16x2_bits(__fmaf_rn(x[2 * k], CP.scale[2 * k], CP.nshift[2 * k]),
                       __fmaf_rn(x[2 * k + 1], CP.scale[2 * k + 1], CP.nshift[2 * k + 1]));
  *reinterpret_cast<uint4*>(tile + umma::kmaj_off(r, 0, CL_K1)) = make_uint4(w[0], w[1], w[2], w[3]);
  *reinterpret_cast<uint4*>(tile + umma::kmaj_off(r, 8, CL_K1)) = make_uint4(w[4], 0u, 0u, 0u);
}

// The network for two 128-row tiles, called by all LC_THREADS threads of the block with the
// weight images at LC_SMEM_W1 / LC_SMEM_W2, the barrier at LC_SMEM_BAR (phases 0 and 1 are used)
// and 64 tensor-memory columns at tmem. Thread tid's features xa / xb are row tid of tiles 0 / 1;
// the result holds their eddy viscosities nu_scale softplus(z3). A wait that times out clears ok.
__device__ __forceinline__ float2 lc_network2(uint8_t* smem, uint32_t tmem, uint64_t* mbar, uint32_t tid,
                                              const float (&xa)[CL_IN], const float (&xb)[CL_IN],
                                              const ClosureParams& CP, bool& ok) {
  uint8_t* const sA = smem + LC_SMEM_A;
  uint8_t* const sH = smem + LC_SMEM_H;
  const uint32_t warp = tid >> 5;
  lc_write_inputs(sA, tid, xa, CP);
  lc_write_inputs(sA + 4096, tid, xb, CP);
  constexpr uint32_t ID = umma::idesc_bf16<128, CL_H>();
  umma::fence_async_smem();
  umma::fence_before_sync();  // tensor-memory reads of a previous call come before these MMAs
  __syncthreads();
  if (tid == 0) {
    umma::fence_after_sync();
    const uint64_t bw1 = umma::sdesc(umma::smem_u32(smem + LC_SMEM_W1), 128, 256);
    umma::mma_bf16(tmem, umma::sdesc(umma::smem_u32(sA), 128, 256), bw1, ID, false);
    umma::mma_bf16(tmem + 32, umma::sdesc(umma::smem_u32(sA + 4096), 128, 256), bw1, ID, false);
    umma::commit(mbar);
  }
  ok = umma::mbar_wait(mbar, 0, LC_WAIT_LIMIT) && ok;
  umma::fence_after_sync();
  // hidden layer 1: bias, gelu (two units per f32x2 lane pair), bf16x2 -> row tid of the hidden tiles
#pragma unroll
  for (int t = 0; t < 2; t++) {
    float v[4][8];
#pragma unroll
    for (int c = 0; c < 4; c++) umma::tmem_ld8(umma::tmem_lane_addr(tmem, warp, 32 * t + 8 * c), v[c]);
    umma::tmem_wait_ld();
#pragma unroll
    for (int c = 0; c < 4; c++) {
      uint32_t pk[4];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int j = 8 * c + 2 * e;
        const float2 g = cl_gelu2x(__fadd2_rn(make_float2(v[c][2 * e], v[c][2 * e + 1]),
                                             make_float2(CP.b1[j], CP.b1[j + 1])));
        pk[e] = bf16x2_bits(g.x, g.y);
      }
      *reinterpret_cast<uint4*>(sH + 8192 * t + umma::kmaj_off(tid, 8 * c, CL_H)) =
          make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
  }
  umma::fence_before_sync();
  umma::fence_async_smem();
  __syncthreads();
  if (tid == 0) {
    umma::fence_after_sync();
    const uint32_t w2 = umma::smem_u32(smem + LC_SMEM_W2);
#pragma unroll
    for (int t = 0; t < 2; t++) {
      const uint32_t a = umma::smem_u32(sH + 8192 * t);
      umma::mma_bf16(tmem + 32 * t, umma::sdesc(a, 128, 512), umma::sdesc(w2, 128, 512), ID, false);
      umma::mma_bf16(tmem + 32 * t, umma::sdesc(a + 256, 128, 512), umma::sdesc(w2 + 256, 128, 512), ID, true);
    }
    umma::commit(mbar);
  }
  ok = umma::mbar_wait(mbar, 1, LC_WAIT_LIMIT) && ok;
  umma::fence_after_sync();
  // hidden layer 2 (f32) and the output layer: even units in lane .x, odd units in lane .y
  float z3[2];
#pragma unroll
  for (int t = 0; t < 2; t++) {
    float v[4][8];
#pragma unroll
    for (int c = 0; c < 4; c++) umma::tmem_ld8(umma::tmem_lane_addr(tmem, warp, 32 * t + 8 * c), v[c]);
    umma::tmem_wait_ld();
    float2 z = f2(0.0f);
#pragma unroll
    for (int c = 0; c < 4; c++)
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int j = 8 * c + 2 * e;
        const float2 g = cl_gelu2x(__fadd2_rn(make_float2(v[c][2 * e], v[c][2 * e + 1]),
                                             make_float2(CP.b2[j], CP.b2[j + 1])));
        z = __ffma2_rn(g, make_float2(CP.w3[j], CP.w3[j + 1]), z);
      }
    z3[t] = __fmul_rn(CP.nu_scale, cl_softplus(__fadd_rn(__fadd_rn(z.x, z.y), CP.b3)));
  }
  return make_float2(z3[0], z3[1]);
}

// The eddy viscosities of `rows` feature rows (xb: [rows][10], the face rows' and wall cells'
// features) into nub[rows], on the tensor cores with the bulk kernel's arithmetic: 256 rows per
// block, row b * 256 + tid in tile 0 and b * 256 + 128 + tid in tile 1. A timed-out wait sets
// bit 4 of the error word and the block stores nothing.
__global__ void __launch_bounds__(LC_THREADS) k_closure_rows(const float* __restrict__ xb, uint32_t rows,
                                                              float* __restrict__ nub,
                                                              const ClosureDev* __restrict__ cw,
                                                              const __grid_constant__ ClosureParams CP,
                                                              int* __restrict__ err) {
  extern __shared__ __align__(128) uint8_t lc_smem[];
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  uint64_t* const mbar = reinterpret_cast<uint64_t*>(lc_smem + LC_SMEM_BAR);
  uint32_t* const tslot = reinterpret_cast<uint32_t*>(lc_smem + LC_SMEM_BAR + 8);
  {
    const uint4* src = reinterpret_cast<const uint4*>(cw->w1img);
    uint4* dst = reinterpret_cast<uint4*>(lc_smem + LC_SMEM_W1);
    for (uint32_t k = tid; k < 192u; k += LC_THREADS) dst[k] = __ldg(src + k);
  }
  uint64_t* const dbar = reinterpret_cast<uint64_t*>(lc_smem + LC_SMEM_DRAIN);
  if (tid == 0) {
    umma::mbar_init(mbar, 1);
    umma::mbar_init(dbar, 1);
  }
  if (warp == 0) umma::tmem_alloc(tslot, LC_TMEM_COLS);
  const uint32_t r0 = blockIdx.x * (2u * LC_THREADS) + tid, r1 = r0 + LC_THREADS;
  float xa[CL_IN], xc[CL_IN];
#pragma unroll
  for (int k = 0; k < CL_IN; k++) {
    xa[k] = r0 < rows ? __ldg(xb + (size_t)r0 * CL_IN + k) : 0.0f;
    xc[k] = r1 < rows ? __ldg(xb + (size_t)r1 * CL_IN + k) : 0.0f;
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  bool ok = true;
  const float2 nu = lc_network2(lc_smem, tmem, mbar, tid, xa, xc, CP, ok);
  if (ok) {
    if (r0 < rows) nub[r0] = nu.x;
    if (r1 < rows) nub[r1] = nu.y;
  }
  // after a timed-out wait, the MMAs finish before their tensor memory is released
  const bool drained = umma::drain_before_free(dbar, !ok, LC_WAIT_LIMIT);
  __syncthreads();
  if (warp == 0) umma::tmem_free(tmem, LC_TMEM_COLS);
  if (!ok || !drained) atomicOr(err, 4);
}

// Tiles of tpr cell pairs x 128 / tpr rows; block b takes tiles b, b + grid, ... (LC_TILES_PER_BLOCK
// of them) and keeps its weight images, barrier and tensor memory for all of them. 29 KB of shared
// memory per block: at most 7 blocks share an SM, and their 7 x 64 tensor-memory columns fit in
// its 512. After each tile the block agrees on `ok`; a timed-out wait ends the loop for the whole
// block.
constexpr int LC_TILES_PER_BLOCK = 4;
constexpr int LC_BLOCKS_PER_SM = 7;  // the shared-memory limit; registers are capped to match
template <class S, bool BGK>
__global__ void __launch_bounds__(LC_THREADS, LC_BLOCKS_PER_SM) k_stream_collide_lc(const __grid_constant__ wt_kparams P,
                                                                   const typename S::T* __restrict__ fin,
                                                                   typename S::T* __restrict__ fout,
                                                                   const uint8_t* __restrict__ cls, int gs,
                                                                   const uint32_t* __restrict__ sdf,
                                                                   const ClosureDev* __restrict__ cw,
                                                                   const __grid_constant__ ClosureParams CP,
                                                                   int tpr, uint32_t ntiles,
                                                                   int* __restrict__ err) {
  typedef D3Q19 L;
  typedef PairIO<S> IO;
  constexpr int Q = L::Q;
  extern __shared__ __align__(128) uint8_t lc_smem[];
  const int NX = P.nx, NY = P.ny, NZ = P.nz;
  const uint32_t tid = threadIdx.x;
  const uint32_t warp = tid >> 5;
  const int rpb = LC_THREADS / tpr;
  const int tx = (int)tid % tpr, ty = (int)tid / tpr;
  const int tiles_x = (NX / 2 + tpr - 1) / tpr, tiles_y = (NY + rpb - 1) / rpb;
  const uint32_t N = P.n;
  const uint32_t sy = (uint32_t)NX, sz = (uint32_t)NX * (uint32_t)NY;
  uint64_t* const mbar = reinterpret_cast<uint64_t*>(lc_smem + LC_SMEM_BAR);
  uint32_t* const tslot = reinterpret_cast<uint32_t*>(lc_smem + LC_SMEM_BAR + 8);
  uint64_t* const dbar = reinterpret_cast<uint64_t*>(lc_smem + LC_SMEM_DRAIN);
  {
    const uint4* src = reinterpret_cast<const uint4*>(cw->w1img);
    uint4* dst = reinterpret_cast<uint4*>(lc_smem + LC_SMEM_W1);
    for (uint32_t k = tid; k < 192u; k += LC_THREADS) dst[k] = __ldg(src + k);
  }
  if (tid == 0) {
    umma::mbar_init(mbar, 1);
    umma::mbar_init(dbar, 1);
  }
  if (warp == 0) umma::tmem_alloc(tslot, LC_TMEM_COLS);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  bool ok = true;
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int bx = (int)(tile % (uint32_t)tiles_x);
    const int by = (int)((tile / (uint32_t)tiles_x) % (uint32_t)tiles_y);
    const int iz = (int)(tile / ((uint32_t)tiles_x * (uint32_t)tiles_y));
    const int x0 = (bx * tpr + tx) * 2;
    const int iy = by * rpb + ty;
    const bool inside = x0 < NX && iy > 0 && iy < NY - 1 && iz > 0 && iz < NZ - 1;
    const uint32_t idx0 = inside ? (uint32_t)x0 + sy * (uint32_t)iy + sz * (uint32_t)iz : 0u;
    // the loads of the two cells in flight (as k_stream_collide_v)
    uint32_t cv = 0x01010101u;
    typename IO::pair_t rp[Q];
    typename IO::one_t r1[Q];
    uint2 sw = make_uint2(0u, 0u);
    if (inside) {
      if (gs == 4) cv = __ldg(reinterpret_cast<const unsigned int*>(cls + (idx0 & ~3u)));
      else cv = __ldg(reinterpret_cast<const unsigned short*>(cls + idx0));
      const bool last = x0 + 2 >= NX;
      const typename S::T* fb = fin + idx0;
      static_for<Q>([&](auto I) {
        constexpr int i = I;
        constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
        const typename S::T* ps = fb + ((ptrdiff_t)i * N - (ptrdiff_t)cy * sy - (ptrdiff_t)cz * sz);
        rp[i] = IO::ld(ps, 0u);
        if constexpr (cx > 0) r1[i] = IO::ld1(x0 > 0 ? ps - 1 : ps, 0u);
        if constexpr (cx < 0) r1[i] = IO::ld1(ps + (last ? 1 : 2), 0u);
      });
      sw = __ldg(reinterpret_cast<const uint2*>(sdf + idx0));
    } else {
      static_for<Q>([&](auto I) {
        constexpr int i = I;
        rp[i] = typename IO::pair_t{};
        r1[i] = typename IO::one_t{};
      });
    }
    // pulled populations (rest state outside), the network, collision, stores
    float2 h[Q];
    static_for<Q>([&](auto I) {
      constexpr int i = I;
      constexpr int cx = L::c[i][0];
      constexpr float w = (float)Wc<L, i>::v;
      const float2 cur = IO::cvt(rp[i], w);
      float2 v;
      if constexpr (cx == 0) v = cur;
      else if constexpr (cx > 0) v = make_float2(IO::cvt1(r1[i], w), cur.x);
      else v = make_float2(cur.y, IO::cvt1(r1[i], w));
      h[i] = inside ? v : f2(0.0f);
    });
    if (inside && x0 == 0) {
      const float U = P.uin;
      static_for<Q>([&](auto I) {
        constexpr int i = I;
        constexpr int cx = L::c[i][0];
        if constexpr (cx > 0) {
          constexpr float w = (float)Wc<L, i>::v;
          h[i].x = w * P.rho_in * (1.0f + 3.0f * U + 4.5f * U * U - 1.5f * U * U) - w;
        }
      });
    }
    const float2 wd = make_float2(cl_wall_dist(sw.x), cl_wall_dist(sw.y));
    const bool store = inside && (cv & 0x03030303u) == 0u;
    typename S::T* ob = fout + idx0;
    collide_shifted2x<L, BGK, SP_TEST>(
        P, h, x0,
        [&](auto I, float2 v) {
          constexpr int i = decltype(I)::value;
          if (store && ok) IO::st(ob + (ptrdiff_t)i * N, 0u, v, (float)Wc<L, i>::v);
        },
        [&](float2 rho, float2, float2 ux, float2 uy, float2 uz, float2 pxx, float2 pyy, float2 pzz, float2 pxy,
            float2 pxz, float2 pyz) {
          {
            float xa[CL_IN], xb[CL_IN];
            cl_features(pxx.x, pyy.x, pzz.x, pxy.x, pxz.x, pyz.x, rho.x, ux.x, uy.x, uz.x, P.tau0, wd.x, xa);
            cl_features(pxx.y, pyy.y, pzz.y, pxy.y, pxz.y, pyz.y, rho.y, ux.y, uy.y, uz.y, P.tau0, wd.y, xb);
            const float2 nu = lc_network2(lc_smem, tmem, mbar, tid, xa, xb, CP, ok);
            const float ta = tau0_eff(P, (float)x0, 0.0f) + 3.0f * nu.x;
            const float tb = tau0_eff(P, (float)(x0 + 1), 0.0f) + 3.0f * nu.y;
            return make_float2(1.0f - __fdividef(1.0f, ta), 1.0f - __fdividef(1.0f, tb));
          }
        });
    if (!__syncthreads_and(ok)) {
      ok = false;
      break;
    }
  }
  // release the tensor memory once every thread's reads have completed and, after a timed-out
  // wait, once the MMAs issued before it have completed
  const bool drained = umma::drain_before_free(dbar, !ok, LC_WAIT_LIMIT);
  __syncthreads();
  if (warp == 0) umma::tmem_free(tmem, LC_TMEM_COLS);
  if (!ok || !drained) atomicOr(err, 4);
}

// ---------------------------------------------------------------------------------------------
// cells next to walls: per-link recipes built at classification, applied every step
// ---------------------------------------------------------------------------------------------
// Every incoming population of a fluid cell next to a wall is an affine combination of at most
// two stored populations, v = alpha * F[a1] + beta * F[a2] + gamma: an interior, mirrored or
// periodic pull has alpha = 1; floor bounce-back adds the belt term in gamma; a Bouzidi link mixes
// f_opp(x) with f_opp(x + c_i) (q < 1/2) or f_i(x) (q > 1/2) and carries the wheel's moving-wall
// term and its mass fix in gamma; an inlet link is gamma alone. Geometry, parameters and wheels
// are fixed between classifications, so k_boundary_build evaluates the reference's rules
// (wgslLbm.ts:138-175, 276-291; the same rules as cell_general) once per cell and link, and
// k_boundary_tab applies them every step with one record load and two gathers per link, no
// dependent flag or distance loads. The FP16 shift is folded into gamma: every population a link
// of direction i reads has the weight w_i (direction i, its opposite, or a mirror image of i).
//
// Records are stored link-major, record (link i, cell k) at i * cap + k (cap = capacity in
// cells), so the record loads of a warp of consecutive cells are contiguous.
enum : uint32_t { BC_WALL = 1u, BC_GWALL = 2u };

// one thread per listed fluid cell; writes its cell word {cell, BC_* bits} and its Q link records
template <class L, class S>
__global__ void __launch_bounds__(128) k_boundary_build(const __grid_constant__ wt_kparams P,
                                                        const uint32_t* __restrict__ flags,
                                                        const uint32_t* __restrict__ sdf,
                                                        const uint8_t* __restrict__ cls,
                                                        const __grid_constant__ Wheels W,
                                                        const uint32_t* __restrict__ list, uint32_t count,
                                                        uint32_t cap, uint2* __restrict__ bcell,
                                                        uint4* __restrict__ rec, float* __restrict__ gam) {
  constexpr int Q = L::Q;
  constexpr bool D3 = L::DIM == 3;
  constexpr bool SHIFT = S::PREC == WT_PREC_F16;
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const uint32_t c = list[k];
  const int NX = P.nx, NY = P.ny, NZ = P.nz;
  const uint32_t N = P.n;  // q * n < 2^32 on the vectorised path
  const int ix = (int)(c % (uint32_t)NX);
  const int iy = (int)((c / (uint32_t)NX) % (uint32_t)NY);
  const int iz = (int)(c / ((uint32_t)NX * (uint32_t)NY));
  auto cid = [&](int x, int y, int z) -> uint32_t { return (uint32_t)x + (uint32_t)NX * ((uint32_t)y + (uint32_t)NY * (uint32_t)z); };
  const uint8_t cl = cls[c];
  const bool near = (cl & CLS_NEAR_SOLID) != 0;
  const float U = P.uin;
  const float belt = (P.ground == 2u && !(cl & CLS_BELT_STILL)) ? 1.0f : 0.0f;
  const uint32_t sdf_raw = sdf[c];
  const float sdf_self = (P.interp != 0u && sdf_raw != 0u) ? __uint_as_float(~sdf_raw) : -1.0f;
  const size_t rb = k;  // record of link i: rb + i * cap
  float ga[Q];
  uint32_t bits = 0, wm = 0;
  float mvSum = 0.f, mvW = 0.f;
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
    constexpr int io = opp<L>(i);
    const float w = (float)Wc<L, i>::v;
    uint32_t A = (uint32_t)i * N + c, B = 0xffffffffu;
    float alpha = 1.f, beta = 0.f, gamma = 0.f;
    if constexpr (i > 0) {
      int sx = ix - cx;
      const int sy = iy - cy, sz = D3 ? iz - cz : 0;
      if constexpr (cx < 0) sx = min(sx, NX - 1);
      const bool yOut = cy > 0 ? sy < 0 : (cy < 0 ? sy >= NY : false);
      const bool zOut = D3 ? (cz > 0 ? sz < 0 : (cz < 0 ? sz >= NZ : false)) : false;
      const int sxc = min(max(sx, 0), NX - 1);
      const int szc = D3 ? min(max(sz, 0), NZ - 1) : 0;
      if (cx > 0 && sx < 0) {
        // inlet: equilibrium at (rho_in, U)
        const float cu = 1.0f * U;
        alpha = 0.f;
        gamma = w * P.rho_in * (1.0f + 3.0f * cu + 4.5f * cu * cu - 1.5f * U * U);
      } else if (cy > 0 && yOut && P.ground != 0u) {
        // no-slip / moving floor: bounce-back plus the belt term
        bits |= BC_WALL | BC_GWALL;
        A = (uint32_t)io * N + c;
        if constexpr (cx != 0) gamma = belt * ((float)(6.0 * Wc<L, i>::v * cx) * P.u_ground);
      } else if (D3 && yOut && zOut) {
        A = (uint32_t)mirYZ<L>(i) * N + cid(sxc, iy, iz);
      } else if (yOut) {
        A = (uint32_t)mirY<L>(i) * N + cid(sxc, iy, szc);
      } else if (D3 && zOut) {
        A = P.side_mode == 1u ? (uint32_t)i * N + cid(sxc, sy, (sz + NZ) % NZ)
                              : (uint32_t)mirZ<L>(i) * N + cid(sxc, sy, iz);
      } else {
        const uint32_t sc = cid(sxc, sy, sz);
        const uint32_t fs = near ? flags[sc] : 0u;
        if (fs == 0u) {
          A = (uint32_t)i * N + sc;
        } else {
          // interpolated bounce-back (Bouzidi) on a solid source
          bits |= BC_WALL;
          A = (uint32_t)io * N + c;
          float q = 0.5f;
          if (P.interp != 0u) {
            const uint32_t rs = sdf[sc];
            const float a = sdf_self, b = rs != 0u ? __uint_as_float(~rs) : -1.0f;
            if (!(a < 0.f || b < 0.f || a + b < 1e-6f)) {
              q = a / (a + b);
              q = q < 0.01f ? 0.01f : (q > 0.99f ? 0.99f : q);
            }
          }
          if (q < 0.5f) {
            const int ax = ix + cx, ay = iy + cy, az = D3 ? iz + cz : 0;
            const bool inA = ax >= 0 && ay >= 0 && az >= 0 && ax < NX && ay < NY && az < NZ;
            if (inA && flags[cid(ax, ay, az)] == 0u) {
              alpha = 2.0f * q;
              beta = 1.0f - 2.0f * q;
              B = (uint32_t)io * N + cid(ax, ay, az);
            } else {
              q = 0.5f;
            }
          } else if (q > 0.5f) {
            alpha = 0.5f / q;
            beta = 1.0f - 0.5f / q;
            B = (uint32_t)i * N + c;
          }
          if ((fs >> 8u) != 0u) {
            float ux, uy, uz;
            wheel_vel<float>(P, W, (fs >> 8u) - 1u, 0.5f * (float)(ix + sxc) + 0.5f, 0.5f * (float)(iy + sy) + 0.5f,
                             0.5f * (float)(iz + sz) + 0.5f, ux, uy, uz);
            const float dot = (float)cx * ux + (float)cy * uy + (float)cz * uz;
            const float mv = (float)(6.0 * Wc<L, i>::v) * dot * (q > 0.5f ? 0.5f / q : 1.0f);
            gamma += mv;
            mvSum += mv;
            mvW += w;
            wm |= 1u << i;
          }
        }
      }
    }
    if (B == 0xffffffffu) B = A;
    ga[i] = gamma;
    rec[rb + (size_t)i * cap] = make_uint4(A, B, __float_as_uint(alpha), __float_as_uint(SHIFT ? alpha + beta : beta));
  });
  // wheel links: remove the net mass of the moving-wall terms (wgslLbm.ts:289-291)
  const float corr = mvW > 0.f ? mvSum / mvW : 0.f;
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    float g = ga[i];
    if (wm & (1u << i)) g -= (float)Wc<L, i>::v * corr;
    if constexpr (SHIFT) {
      // stored h = f - w_i for both sources: alpha (h1 + w) + beta (h2 + w) + g
      const uint4 r = rec[rb + (size_t)i * cap];
      const float alpha = __uint_as_float(r.z), ab = __uint_as_float(r.w);
      const float beta = ab - alpha;
      rec[rb + (size_t)i * cap] = make_uint4(r.x, r.y, r.z, __float_as_uint(beta));
      g += ab * (float)Wc<L, i>::v;
    }
    gam[rb + (size_t)i * cap] = g;
  });
  bcell[k] = make_uint2(c, bits);
}

// Applies the link records, one thread per listed cell: every record load of the cell in flight
// at once (coalesced across the warp), then every gather, then the collision and the stores.
// MODE as for the face rows: FM_SMAG, FM_FEATURES (the listed cell's features into row k of xb,
// nothing stored) or FM_NU (collision with the eddy viscosity nub[k]).
template <class L, class S, int MODE = FM_SMAG, bool SMP = false, bool COH = false>
__device__ __forceinline__ void boundary_cell(const wt_kparams& P, const typename S::T* __restrict__ fin,
                                              typename S::T* __restrict__ fout, const uint2* __restrict__ bcell,
                                              const uint4* __restrict__ rec, const float* __restrict__ gam,
                                              uint32_t k, uint32_t cap, const uint32_t* __restrict__ sdf,
                                              float* __restrict__ xb, const float* __restrict__ nub,
                                              const SampleOut* O, SampleSums* acc) {
  constexpr int Q = L::Q;
  const uint2 hc = bcell[k];
  uint4 r[Q];
  float g[Q];
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    r[i] = __ldg(rec + (size_t)i * cap + k);
    g[i] = __ldg(gam + (size_t)i * cap + k);
  });
  typename S::T x1[Q], x2[Q];
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    x1[i] = ldp<COH>(fin + r[i].x);
    x2[i] = ldp<COH>(fin + r[i].y);
  });
  float f[Q], fo[Q];
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    f[i] = fmaf(__uint_as_float(r[i].z), S::cvt(x1[i], 0.0f), fmaf(__uint_as_float(r[i].w), S::cvt(x2[i], 0.0f), g[i]));
  });
  const int ix = (int)(hc.x % P.nx);
  if constexpr (MODE == FM_FEATURES) {
    float x[CL_IN];
    collide_full<L, float>(P, f, ix, false, false, fo, -1.0f, x, cl_wall_dist(__ldg(sdf + hc.x)));
#pragma unroll
    for (int q = 0; q < CL_IN; q++) xb[(size_t)k * CL_IN + q] = x[q];
    return;
  } else if constexpr (MODE == FM_NU) {
    collide_full<L, float>(P, f, ix, (hc.y & BC_WALL) != 0u, (hc.y & BC_GWALL) != 0u, fo, __ldg(nub + k));
  } else {
    collide_full<L, float>(P, f, ix, (hc.y & BC_WALL) != 0u, (hc.y & BC_GWALL) != 0u, fo);
  }
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    S::st(fout, (size_t)i * P.n + hc.x, fo[i], (float)Wc<L, i>::v);
  });
  if constexpr (SMP) {
    // the sampling pass on the stored values, summed in the pair kernels' emission order
    float rho = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
    static_for<Q>([&](auto K) {
      constexpr int i = emit_dir<L>(K);
      constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
      float f;
      if constexpr (S::PREC == WT_PREC_F16) {
        constexpr float w = (float)Wc<L, i>::v;
        f = h2f_add(__float2half_rn(__fsub_rn(fo[i], w)), w);
      } else {
        f = fo[i];
      }
      if constexpr (K == 0) rho = f;
      else rho = __fadd_rn(rho, f);
      if constexpr (cx > 0) jx = __fadd_rn(jx, f);
      if constexpr (cx < 0) jx = __fadd_rn(jx, -f);
      if constexpr (cy > 0) jy = __fadd_rn(jy, f);
      if constexpr (cy < 0) jy = __fadd_rn(jy, -f);
      if constexpr (cz > 0) jz = __fadd_rn(jz, f);
      if constexpr (cz < 0) jz = __fadd_rn(jz, -f);
    });
    float ux, uy, uz, uu;
    cell_velocity<float>(rho, jx, jy, jz, ux, uy, uz, uu);
    O->vel[hc.x] = fluid_sample<float>(P, hc.x, ix, rho, ux, uy, uz, uu, O->meanA, O->meanB,
                                       make_float4(0.f, 0.f, 0.f, 0.f), 0.0f, false, *acc);
  }
}

template <class L, class S, int MODE = FM_SMAG, bool SMP = false>
__global__ void __launch_bounds__(64) k_boundary_tab(const __grid_constant__ wt_kparams P,
                                                     const typename S::T* __restrict__ fin,
                                                     typename S::T* __restrict__ fout,
                                                     const uint2* __restrict__ bcell, const uint4* __restrict__ rec,
                                                     const float* __restrict__ gam, uint32_t count, uint32_t cap,
                                                     const uint32_t* __restrict__ sdf, float* __restrict__ xb,
                                                     const float* __restrict__ nub,
                                                     const __grid_constant__ SampleOut O) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  SampleSums acc;
  if (k < count) boundary_cell<L, S, MODE, SMP>(P, fin, fout, bcell, rec, gam, k, cap, sdf, xb, nub, &O, &acc);
  if constexpr (SMP) smp_flush(acc, O.sets, global_warp_id());
}

// ---- persistent steps: many lattice updates of one or more tunnels in one launch ---------------
// On small grids a step's kernels finish faster than they can be launched (the D2Q9 channel of
// 65,536 cells: about 5.5 us per step in captured graphs, most of it launch and dependency
// latency). Here one cooperative launch runs `steps` updates of every tunnel in its table. A step's
// work items are, in this order, the wall-cell chunks of every tunnel, then their face-row tiles,
// then their bulk tiles (the slow items first, so that the step ends on short ones); blocks take
// the next item from a per-step atomic counter, and a grid-wide barrier separates the steps. Each
// cell goes through the same device code as in the per-step kernels (bulk_cells, face_rows,
// boundary_cell), so the results are bit-identical to stepping alone; its population loads are
// cached in L2 only (ld.cg), since the input of one step is what other SMs wrote in the step
// before. In D3Q19 the face and wall items run out of line, so that their register demand does not
// set the bulk tiles' occupancy.
// The barrier's waits are bounded: a block that gives up sets bit 16 of the error word and
// returns, and every other block then gives up too.
constexpr int PS_THREADS = 256;
constexpr int PS_MIN_BLOCKS = 4;  // resident blocks per SM the register budget is set for
constexpr int PS_MAX_TUNNELS = 48;
constexpr uint32_t PS_BARRIER_POLLS = 1u << 22;

struct PersistTunnel {
  wt_kparams P;
  void* f[2];             // step k reads f[(p0 + k) & 1] and writes the other
  const uint8_t* cls;
  const uint2* bcell;     // link records of the wall cells (k_boundary_tab's tables)
  const uint4* brec;
  const float* bgam;
  uint32_t nbnd, btab_cap;
  int32_t gs, p0;
  uint32_t tbx, tby;      // bulk tile: tbx cell pairs along x by tby rows (tbx * tby = PS_THREADS)
  uint32_t ttx, tty;      // bulk tiles per z-plane along x and y
  uint32_t wi0, fi0, bi0; // first wall chunk, face tile and bulk tile of this tunnel in the step's items
  uint32_t pad;
};
struct PersistTable {
  uint32_t count;         // tunnels
  uint32_t fseg, bseg;    // first face item and first bulk item of a step (the wall items come first)
  uint32_t items;         // work items per step
  PersistTunnel t[PS_MAX_TUNNELS];
};

// grid-wide barrier over bar[0] (arrivals) and bar[1] (generation), both zero before the launch;
// false if this block gave up waiting
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned nblocks) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = bar + 1;
    const unsigned g = *gen;  // read before arriving: the generation cannot move until this block has
    __threadfence();
    int done = 1;
    if (atomicAdd(bar, 1u) == nblocks - 1u) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      uint32_t it = 0;
      while (*gen == g) {
        if (++it > PS_BARRIER_POLLS) {
          done = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    ok = done;
  }
  __syncthreads();
  return ok != 0;
}

// last tunnel m of the table with first(t[m]) <= item (first is nondecreasing in m; tunnels with no
// items of the segment share their successor's start and are passed over)
template <class F>
__device__ __forceinline__ uint32_t ps_find(const PersistTable& T, uint32_t item, F first) {
  uint32_t lo = 0, hi = T.count;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (first(T.t[mid]) <= item) lo = mid;
    else hi = mid;
  }
  return lo;
}

// wall cells c of one chunk (one per thread)
template <class L, class S, bool COH>
__device__ __forceinline__ void ps_wall_cells(const PersistTunnel& t, const typename S::T* fin, typename S::T* fout,
                                              uint32_t c) {
  if (c < t.nbnd)
    boundary_cell<L, S, FM_SMAG, false, COH>(t.P, fin, fout, t.bcell, t.brec, t.bgam, c, t.btab_cap, nullptr,
                                              nullptr, nullptr, nullptr, nullptr);
}

// face-row cell pair g (row g / (nx / 2), pair g % (nx / 2))
template <class L, class S, bool COH>
__device__ __forceinline__ void ps_face_cells(const PersistTunnel& t, const typename S::T* fin, typename S::T* fout,
                                              uint32_t g) {
  const uint32_t half = t.P.nx / 2u;
  face_rows<L, S, FM_SMAG, false, COH>(t.P, fin, fout, t.cls, t.gs, nullptr, nullptr, nullptr, nullptr, nullptr,
                                        (int)(g % half) * 2, (int)(g / half));
}

// the same, out of line: in D3Q19 their register demand is above the bulk tiles' budget
template <class L, class S, bool COH>
__device__ __noinline__ void ps_wall(const PersistTunnel& t, const typename S::T* fin, typename S::T* fout, uint32_t c) {
  ps_wall_cells<L, S, COH>(t, fin, fout, c);
}
template <class L, class S, bool COH>
__device__ __noinline__ void ps_face(const PersistTunnel& t, const typename S::T* fin, typename S::T* fout, uint32_t g) {
  ps_face_cells<L, S, COH>(t, fin, fout, g);
}

// COH: the population loads bypass the read-only cache (a launch of several steps reads what its
// own blocks wrote in the step before); one step per launch (k0 = the step's index in its graph,
// which alternates the item counters) keeps the read-only path of the per-step kernels.
template <class L, class S, bool BGK, bool COH>
__global__ void __launch_bounds__(PS_THREADS, PS_MIN_BLOCKS)
    k_steps_persistent(const __grid_constant__ PersistTable T, int steps, int k0, unsigned* __restrict__ bar,
                       int* __restrict__ err) {
  typedef typename S::T ST;
  // A block's first item of a step is its block index; thread 0 takes each further item from the
  // step's counter (item = grid size + counter) while the block works on the current one, and
  // passes it on through shared memory, double-buffered so that one barrier per item suffices.
  __shared__ uint32_t s_item[2];
  const uint32_t tid = threadIdx.x;
  uint32_t sl = 0;
  // one step per launch: a launch with programmatic stream serialisation may start before the
  // previous step has finished; wait for it (and its memory) before touching any buffer or counter
  if constexpr (!COH) asm volatile("griddepcontrol.wait;" ::: "memory");
  for (int k = 0; k < steps; k++) {
    // COH (several steps per launch): two counters alternate, the next step's cleared by block 0
    // (it was last used by the step before this one, which every block has left). One step per
    // launch: one counter, cleared by the last block to finish (below).
    unsigned* const ctr = COH ? bar + 2 + ((k0 + k) & 1) : bar + 2;
    if (COH && blockIdx.x == 0 && tid == 0) atomicExch(bar + 2 + ((k0 + k + 1) & 1), 0u);
    for (uint32_t item = blockIdx.x; item < T.items; sl ^= 1u) {
      uint32_t nxt = 0;
      if (tid == 0) nxt = atomicAdd(ctr, 1u);  // consumed after this item's cells
      uint32_t m;
      if (item < T.fseg) m = ps_find(T, item, [](const PersistTunnel& q) { return q.wi0; });
      else if (item < T.bseg) m = ps_find(T, item, [](const PersistTunnel& q) { return q.fi0; });
      else m = ps_find(T, item, [](const PersistTunnel& q) { return q.bi0; });
      const PersistTunnel& t = T.t[m];
      const int par = (t.p0 + k) & 1;
      const ST* fin = (const ST*)t.f[par];
      ST* fout = (ST*)t.f[par ^ 1];
      if (item >= T.bseg) {
        const uint32_t j = item - t.bi0;
        const uint32_t bx = j % t.ttx, by = (j / t.ttx) % t.tty;
        uint32_t bz = j / (t.ttx * t.tty);
        if (par == 1) bz = (uint32_t)t.P.nz - 1u - bz;  // writing buffer 0: z downwards, as the step kernels
        bulk_cells<L, S, 2, BGK, false, COH>(t.P, fin, fout, t.cls, t.gs, (int)(bx * t.tbx + tid % t.tbx) * 2,
                                             (int)(by * t.tby + tid / t.tbx), (int)bz);
      } else if (item >= T.fseg) {
        if constexpr (L::DIM == 3) ps_face<L, S, COH>(t, fin, fout, (item - t.fi0) * PS_THREADS + tid);
        else ps_face_cells<L, S, COH>(t, fin, fout, (item - t.fi0) * PS_THREADS + tid);
      } else {
        if constexpr (L::DIM == 3) ps_wall<L, S, COH>(t, fin, fout, (item - t.wi0) * PS_THREADS + tid);
        else ps_wall_cells<L, S, COH>(t, fin, fout, (item - t.wi0) * PS_THREADS + tid);
      }
      if (tid == 0) s_item[sl] = gridDim.x + nxt;
      __syncthreads();
      item = s_item[sl];
    }
    if (k + 1 < steps && !grid_barrier(bar, gridDim.x)) {
      if (tid == 0) atomicOr(err, 16);
      return;
    }
  }
  if constexpr (!COH) {
    // the next step's blocks may be scheduled now (they wait for this grid to complete)
    asm volatile("griddepcontrol.launch_dependents;");
    // every block has taken its last item once it gets here: the last one clears the counter and
    // the arrival count for the next launch
    __syncthreads();
    if (tid == 0 && atomicAdd(bar + 3, 1u) == gridDim.x - 1u) {
      atomicExch(bar + 2, 0u);
      atomicExch(bar + 3, 0u);
    }
  }
}

// Rest state written into the solid cells of one population buffer.
template <class L, class S>
__global__ void __launch_bounds__(256) k_fill_solid(const __grid_constant__ wt_kparams P,
                                                    const uint8_t* __restrict__ cls, typename S::T* __restrict__ f) {
  const size_t N = P.n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < N; idx += (size_t)gridDim.x * blockDim.x) {
    if (cls[idx] & CLS_SOLID) {
      static_for<L::Q>([&](auto I) {
        constexpr int i = I;
        f[(size_t)i * N + idx] = S::solid((typename S::R)Wc<L, i>::v);
      });
    }
  }
}

// Builds the boundary list (which = 0: every fluid cell of a group holding a solid or near-solid
// cell; solid cells keep the rest state and need no per-step work) or the solid list (which = 1:
// every solid cell, for the fused sampling pass): pass 0 counts, pass 1 writes (warp-aggregated
// slots, in x order inside each warp).
template <class L>
__global__ void __launch_bounds__(256) k_boundary_list(const __grid_constant__ wt_kparams P,
                                                       const uint8_t* __restrict__ cls, int gs,
                                                       uint32_t* __restrict__ counter, uint32_t* __restrict__ list,
                                                       int pass, int which) {
  const uint32_t NX = P.nx;
  const uint32_t N = P.n;
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t base = (blockIdx.x * blockDim.x + (threadIdx.x & ~31u)); base < N; base += gridDim.x * blockDim.x) {
    const uint32_t c = base + lane;
    bool sel = false;
    if (c < N && which == 1) {
      sel = (cls[c] & CLS_SOLID) != 0;
    } else if (c < N) {
      const uint32_t g0 = c - (c % NX) % (uint32_t)gs;
      bool dirty = false;
      for (int k = 0; k < gs; k++) dirty = dirty || (cls[g0 + k] & CLS_BOUNDARY) != 0;
      sel = dirty && (cls[c] & CLS_SOLID) == 0;
    }
    const uint32_t ball = __ballot_sync(0xffffffffu, sel);
    if (ball == 0u) continue;
    uint32_t slot = 0;
    if (lane == 0) slot = atomicAdd(counter, __popc(ball));
    slot = __shfl_sync(0xffffffffu, slot, 0);
    if (pass == 1 && sel) list[slot + __popc(ball & ((1u << lane) - 1u))] = c;
  }
}

// ---------------------------------------------------------------------------------------------
// macro pass: velocity field, EMA statistics, momentum-exchange force, partial reductions
// ---------------------------------------------------------------------------------------------
constexpr int MACRO_THREADS = 256;
// per-block partial slots: the reference's 8 ([sum F (3), max |u|^2, sum rho on x = refX, n_ref,
// nan count, solid count]) and the mass-conservation pair [sum rho over fluid cells (FP64), fluid count]
static_assert(MACRO_SLOTS == 10, "partial slot layout");

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Momentum exchange of one fluid cell (wgslLbm.ts:370-392, 446-453): for every link into a solid,
// the value streaming would build there (Bouzidi with its q branches, the wheel's moving-wall term)
// plus the outgoing population, minus the mass fix of the wheel links. f[] are the cell's stored
// populations (shift undone); Bouzidi partners at x - c_i are read from `fin`.
// GATHER issues the loads in two rounds (every neighbour's flags; then, for the solid links, the
// wall distances and the partner's flags and population) instead of one chain per link: for a
// kernel whose few threads all take this path (k_sample_post). Without it the loads sit at each
// link and hold no registers, for k_macro, where most cells skip the path and occupancy hides the
// latency. Both give the same bits.
template <class L, class S, bool GATHER>
__device__ __forceinline__ void cell_force(const wt_kparams& P, const typename S::T* __restrict__ fin,
                                           const uint32_t* __restrict__ flags, const uint32_t* __restrict__ sdf,
                                           const Wheels& W, size_t idx, int ix, int iy, int iz,
                                           const typename S::R (&f)[L::Q], typename S::R& Fx, typename S::R& Fy,
                                           typename S::R& Fz) {
  typedef typename S::R R;
  constexpr int Q = L::Q;
  const int NX = P.nx, NY = P.ny, NZ = P.nz;
  const size_t N = P.n;
  auto safe = [&](int x, int y, int z) -> int64_t {
    if (x < 0 || y < 0 || z < 0 || x >= NX || y >= NY || z >= NZ) return -1;
    return (int64_t)cell_id(x, y, z, NX, NY);
  };
  const bool interp = P.interp != 0u;
  const uint32_t sd_self = interp ? __ldg(sdf + idx) : 0u;
  // link i's words: the solid neighbour's flags, its wall distance, the partner's (x - c_i) flags
  // (1 outside the domain) and population
  auto link_words = [&](auto I, uint32_t& fli, uint32_t& sdi, uint32_t& flbi, R& fbi) {
    constexpr int i = decltype(I)::value;
    constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
    const int64_t sn = safe(ix + cx, iy + cy, iz + cz);
    fli = sn >= 0 ? __ldg(flags + sn) : 0u;
    sdi = 0u;
    flbi = 1u;
    fbi = (R)0;
    if (fli != 0u) {
      if (interp) sdi = __ldg(sdf + sn);
      const int64_t bk = safe(ix - cx, iy - cy, iz - cz);
      if (bk >= 0) {
        flbi = __ldg(flags + bk);
        fbi = S::ld(fin, (size_t)i * N + (size_t)bk, (R)Wc<L, i>::v);
      }
    }
  };
  uint32_t gfl[GATHER ? Q : 1], gsd[GATHER ? Q : 1], gflb[GATHER ? Q : 1];
  R gfb[GATHER ? Q : 1];
  if constexpr (GATHER) {
    // first wave of loads: every neighbour's flags
    gfl[0] = 0u;
    static_for<Q>([&](auto I) {
      constexpr int i = I;
      if constexpr (i > 0) {
        constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
        const int64_t sn = safe(ix + cx, iy + cy, iz + cz);
        gfl[i] = sn >= 0 ? __ldg(flags + sn) : 0u;
      }
    });
    // second wave: the solid links' distances and partners
    static_for<Q>([&](auto I) {
      constexpr int i = I;
      gsd[i] = 0u;
      gflb[i] = 1u;
      gfb[i] = (R)0;
      if constexpr (i > 0) {
        if (gfl[i] != 0u) {
          constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
          if (interp) gsd[i] = __ldg(sdf + safe(ix + cx, iy + cy, iz + cz));
          const int64_t bk = safe(ix - cx, iy - cy, iz - cz);
          if (bk >= 0) {
            gflb[i] = __ldg(flags + bk);
            gfb[i] = S::ld(fin, (size_t)i * N + (size_t)bk, (R)Wc<L, i>::v);
          }
        }
      }
    });
  }
  R mvSum = 0, mvW = 0, Cwx = 0, Cwy = 0, Cwz = 0;
  Fx = 0;
  Fy = 0;
  Fz = 0;
  static_for<Q>([&](auto I) {
    constexpr int i = I;
    if constexpr (i > 0) {
      constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
      constexpr R w = (R)Wc<L, i>::v;
      uint32_t fli, sdi, flbi;
      R fbi;
      if constexpr (GATHER) {
        fli = gfl[i];
        sdi = gsd[i];
        flbi = gflb[i];
        fbi = gfb[i];
      } else {
        link_words(I, fli, sdi, flbi, fbi);
      }
      if (fli != 0u) {
        // linkQ (wgslLbm.ts:37-43)
        R q = (R)0.5;
        if (interp) {
          const R a = sd_self == 0u ? (R)-1 : (R)__uint_as_float(~sd_self);
          const R b = sdi == 0u ? (R)-1 : (R)__uint_as_float(~sdi);
          if (!(a < (R)0 || b < (R)0 || a + b < (R)1e-6f)) {
            q = a / (a + b);
            q = q < (R)0.01f ? (R)0.01f : (q > (R)0.99f ? (R)0.99f : q);
          }
        }
        R fr = f[i];
        if (q < (R)0.5) {
          if (flbi == 0u) fr = (R)2 * q * f[i] + ((R)1 - (R)2 * q) * fbi;
          else q = (R)0.5;
        } else if (q > (R)0.5) {
          constexpr int oi = opp<L>(i);
          fr = ((R)0.5 / q) * f[i] + ((R)1 - (R)0.5 / q) * f[oi];
        }
        const uint32_t tg = fli >> 8u;
        if (tg != 0u) {
          R wx, wy, wz;
          wheel_vel<R>(P, W, tg - 1u, (R)ix + (R)(0.5 + cx / 2.0), (R)iy + (R)(0.5 + cy / 2.0),
                       (R)iz + (R)(0.5 + cz / 2.0), wx, wy, wz);
          const R dot = (R)cx * wx + (R)cy * wy + (R)cz * wz;
          const R mv = -(R)(6.0 * Wc<L, i>::v) * (q > (R)0.5 ? (R)0.5 / q : (R)1) * dot;
          fr += mv;
          mvSum += mv;
          mvW += w;
          Cwx += (R)cx * w;
          Cwy += (R)cy * w;
          Cwz += (R)cz * w;
        }
        const R t = f[i] + fr - (R)(2.0 * Wc<L, i>::v);
        Fx += (R)cx * t;
        Fy += (R)cy * t;
        Fz += (R)cz * t;
      }
    }
  });
  if (mvW > (R)0) {
    const R k = mvSum / mvW;
    Fx -= Cwx * k;
    Fy -= Cwy * k;
    Fz -= Cwz * k;
  }
}

// A solid cell of the sampling pass: density extrapolated from its fluid face neighbours
// (wgslLbm.ts:460-466), zero velocity, EMA towards that state (meanB cleared). Returns the texel.
// GATHER (for k_sample_post) loads every neighbour's flags, then every population it needs, in two
// rounds; without it (k_macro) the loads sit at each neighbour. Both give the same bits.
template <class L, class S, bool GATHER>
__device__ __forceinline__ uint2 solid_sample(const wt_kparams& P, const typename S::T* __restrict__ fin,
                                              const uint32_t* __restrict__ flags, size_t idx, int ix, int iy, int iz,
                                              float4* __restrict__ meanA, float* __restrict__ meanB, float4 m) {
  typedef typename S::R R;
  constexpr int NB = L::DIM == 3 ? 6 : 4;
  const int NX = P.nx, NY = P.ny, NZ = P.nz;
  const size_t N = P.n;
  const float a = P.ema_alpha;
  const int nb[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  int64_t sn[NB];
  bool fluid[NB];
#pragma unroll
  for (int k = 0; k < NB; k++) {
    const int x = ix + nb[k][0], y = iy + nb[k][1], z = iz + nb[k][2];
    const bool in = !(x < 0 || y < 0 || z < 0 || x >= NX || y >= NY || z >= NZ);
    sn[k] = in ? (int64_t)cell_id(x, y, z, NX, NY) : -1;
    if constexpr (GATHER) fluid[k] = in && __ldg(flags + sn[k]) == 0u;
  }
  R rs = 0, rn = 0;
#pragma unroll
  for (int k = 0; k < NB; k++) {
    R r = 0;
    if constexpr (GATHER) {
      // the fluid neighbours' populations, as predicated loads that are all in flight together
      // (a solid cell inside the body has no fluid neighbour and reads nothing)
      R v[L::Q];
      static_for<L::Q>([&](auto I) {
        constexpr int j = I;
        v[j] = fluid[k] ? S::ld(fin, (size_t)j * N + (size_t)sn[k], (R)Wc<L, j>::v) : (R)0;
      });
      static_for<L::Q>([&](auto I) {
        constexpr int j = I;
        r += v[j];
      });
    } else {
      fluid[k] = sn[k] >= 0 && flags[sn[k]] == 0u;
      if (fluid[k]) {
        static_for<L::Q>([&](auto I) {
          constexpr int j = I;
          r += S::ld(fin, (size_t)j * N + (size_t)sn[k], (R)Wc<L, j>::v);
        });
      }
    }
    if (fluid[k]) {
      rs += r;
      rn += (R)1;
    }
  }
  const float o3 = rn > (R)0 ? (float)(rs / rn) : 1.0f;
  m.x = m.x * (1.0f - a) + 0.0f * a;
  m.y = m.y * (1.0f - a) + 0.0f * a;
  m.z = m.z * (1.0f - a) + 0.0f * a;
  m.w = m.w * (1.0f - a) + o3 * a;
  meanA[idx] = m;
  meanB[idx] = 0.0f;
  __half2 h01 = __floats2half2_rn(0.0f, 0.0f);
  __half2 h23 = __floats2half2_rn(0.0f, o3);
  return make_uint2(*reinterpret_cast<uint32_t*>(&h01), *reinterpret_cast<uint32_t*>(&h23));
}

// Grid-stride over cells (one per thread when the grid has a block per 256 cells). `cls` (may be NULL)
// is the class byte: a fluid cell without CLS_NEAR_SOLID has no in-domain solid neighbour, so its
// 18 link checks are skipped; with NULL every fluid cell checks its links.
template <class L, class S>
__global__ void __launch_bounds__(MACRO_THREADS, 3) k_macro(const wt_kparams P, const typename S::T* __restrict__ fin,
                                                         const uint32_t* __restrict__ flags,
                                                         const uint32_t* __restrict__ sdf,
                                                         const uint8_t* __restrict__ cls, const Wheels W,
                                                         uint2* __restrict__ vel, float4* __restrict__ meanA,
                                                         float* __restrict__ meanB, double* __restrict__ partials) {
  typedef typename S::R R;
  constexpr int Q = L::Q;
  const int NX = P.nx, NY = P.ny;
  const size_t N = P.n;
  const float a = P.ema_alpha;
  double accF[3] = {0, 0, 0};
  MacroSums acc;
  uint32_t accSolid = 0;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < N; idx += (size_t)gridDim.x * blockDim.x) {
    const uint32_t c32 = (uint32_t)idx;  // n < 2^32
    const int ix = (int)(c32 % (uint32_t)NX);
    // y and z only on the paths that visit neighbours (cells next to walls, solid cells)
    auto cell_yz = [&](int& y, int& z) {
      const uint32_t t = c32 / (uint32_t)NX;
      y = (int)(t % (uint32_t)NY);
      z = (int)(t / (uint32_t)NY);
    };
    // every load of the cell is issued before the first branch: one memory round trip per cell.
    // With the class byte, the cell's own solid test reads it (1 B) instead of the flags (4 B).
    const uint8_t cl = cls != nullptr ? cls[idx] : (uint8_t)0;
    const bool solid = cls != nullptr ? (cl & CLS_SOLID) != 0 : flags[idx] != 0u;
    const bool links = cls == nullptr || (cl & CLS_NEAR_SOLID) != 0;
    // EMA: with a = 0, m (1 - a) + v a leaves a fluid cell's means unchanged unless v or |u|^2 is
    // not finite (0 x NaN = NaN); they are then read and written only in that case
    float4 m = make_float4(0.f, 0.f, 0.f, 0.f);
    float mb = 0.0f;
    const bool loaded = a != 0.0f || solid;
    if (loaded) {
      m = meanA[idx];
      mb = meanB[idx];
    }
    R f[Q];
    static_for<Q>([&](auto I) {
      constexpr int i = I;
      f[i] = S::ld(fin, (size_t)i * N + idx, (R)Wc<L, i>::v);
    });
    uint2 texel;
    if (!solid) {
      // density and momentum in the step kernels' emission order (the fused sampling pass's sums)
      R rho = 0, jx = 0, jy = 0, jz = 0;
      static_for<Q>([&](auto K) {
        constexpr int i = emit_dir<L>(K);
        constexpr int cx = L::c[i][0], cy = L::c[i][1], cz = L::c[i][2];
        if constexpr (K == 0) rho = f[i];
        else rho = add_rn(rho, f[i]);
        if constexpr (cx > 0) jx = add_rn(jx, f[i]);
        if constexpr (cx < 0) jx = add_rn(jx, -f[i]);
        if constexpr (cy > 0) jy = add_rn(jy, f[i]);
        if constexpr (cy < 0) jy = add_rn(jy, -f[i]);
        if constexpr (cz > 0) jz = add_rn(jz, f[i]);
        if constexpr (cz < 0) jz = add_rn(jz, -f[i]);
      });
      R ux, uy, uz, uu;
      cell_velocity<R>(rho, jx, jy, jz, ux, uy, uz, uu);
      if (links) {
        int iy, iz;
        cell_yz(iy, iz);
        R Fx, Fy, Fz;
        cell_force<L, S, false>(P, fin, flags, sdf, W, idx, ix, iy, iz, f, Fx, Fy, Fz);
        accF[0] += (double)Fx;
        accF[1] += (double)Fy;
        accF[2] += (double)Fz;
      }
      texel = fluid_sample<R>(P, idx, ix, rho, ux, uy, uz, uu, meanA, meanB, m, mb, loaded, acc);
    } else {
      int iy, iz;
      cell_yz(iy, iz);
      texel = solid_sample<L, S, false>(P, fin, flags, idx, ix, iy, iz, meanA, meanB, m);
      accSolid++;
    }
    vel[idx] = texel;
  }
  // block reduction. Counts by warp votes / integer reductions; the FP64 sums are shuffled only in
  // warps that hold a non-zero value (most warps have no wall link and no reference-plane cell).
  __shared__ double sh[MACRO_THREADS / 32][MACRO_SLOTS];
  const unsigned full = 0xffffffffu;
  if (__any_sync(full, accF[0] != 0.0 || accF[1] != 0.0 || accF[2] != 0.0)) {
    accF[0] = warp_sum(accF[0]);
    accF[1] = warp_sum(accF[1]);
    accF[2] = warp_sum(accF[2]);
  }
  double accRho = acc.rho_ref;
  if (__any_sync(full, acc.nref != 0u)) accRho = warp_sum(accRho);
  const double accMass = warp_sum(acc.mass);
  const float mx = warp_max(acc.maxuu);
  const uint32_t nref = __reduce_add_sync(full, acc.nref);
  const uint32_t nnan = __reduce_add_sync(full, acc.nan);
  const uint32_t nsolid = __reduce_add_sync(full, accSolid);
  const uint32_t nfluid = __reduce_add_sync(full, acc.nfluid);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    sh[wid][0] = accF[0];
    sh[wid][1] = accF[1];
    sh[wid][2] = accF[2];
    sh[wid][3] = (double)mx;
    sh[wid][4] = accRho;
    sh[wid][5] = (double)nref;
    sh[wid][6] = (double)nnan;
    sh[wid][7] = (double)nsolid;
    sh[wid][8] = accMass;
    sh[wid][9] = (double)nfluid;
  }
  __syncthreads();
  if (wid == 0) {
    constexpr int NW = MACRO_THREADS / 32;
#pragma unroll
    for (int k = 0; k < MACRO_SLOTS; k++) {
      double x = lane < NW ? sh[lane][k] : 0.0;
      if (k == 3) {
        float m = warp_max((float)x);
        x = (double)m;
      } else {
        x = warp_sum(x);
      }
      if (lane == 0) partials[(size_t)blockIdx.x * MACRO_SLOTS + k] = x;
    }
  }
}

// The part of the fused sampling pass that needs the whole step done (runs right after the
// sampling step): the momentum-exchange force of the listed fluid cells (the boundary list holds
// every fluid cell next to a solid) and every solid cell (density extrapolated from its fluid face
// neighbours, velocity texel, EMA statistics, count). Each block writes [sum Fx, Fy, Fz (FP64),
// solid count] to partials[4 b ..]; the block that finishes last (a counter in set 0, no waiting)
// reduces the accumulator sets and the partials, in a fixed order, into the MACRO_SLOTS result.
// Densities come back from fixed point; any density outside its range makes both density sums NaN.
constexpr int POST_SLOTS = 4;
template <class L, class S>
__global__ void __launch_bounds__(MACRO_THREADS) k_sample_post(const __grid_constant__ wt_kparams P,
                                                              const typename S::T* __restrict__ fin,
                                                              const uint32_t* __restrict__ flags,
                                                              const uint32_t* __restrict__ sdf,
                                                              const uint8_t* __restrict__ cls,
                                                              const __grid_constant__ Wheels W,
                                                              const uint32_t* __restrict__ bnd, uint32_t nbnd,
                                                              const uint32_t* __restrict__ solids, uint32_t nsolid,
                                                              uint2* __restrict__ vel, float4* __restrict__ meanA,
                                                              float* __restrict__ meanB, double* __restrict__ partials,
                                                              unsigned long long* __restrict__ sets,
                                                              double* __restrict__ result) {
  typedef typename S::R R;
  constexpr int Q = L::Q;
  constexpr int NW = MACRO_THREADS / 32;
  const int NX = P.nx, NY = P.ny;
  const size_t N = P.n;
  double accF[3] = {0, 0, 0};
  uint32_t accSolid = 0;
  const uint32_t items = nbnd + nsolid;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < items; k += gridDim.x * blockDim.x) {
    const bool is_solid = k >= nbnd;
    const uint32_t c = is_solid ? solids[k - nbnd] : bnd[k];
    const int ix = (int)(c % (uint32_t)NX);
    const uint32_t t = c / (uint32_t)NX;
    const int iy = (int)(t % (uint32_t)NY), iz = (int)(t / (uint32_t)NY);
    if (is_solid) {
      vel[c] = solid_sample<L, S, true>(P, fin, flags, c, ix, iy, iz, meanA, meanB, meanA[c]);
      accSolid++;
    } else if (cls[c] & CLS_NEAR_SOLID) {
      R f[Q];
      static_for<Q>([&](auto I) {
        constexpr int i = I;
        f[i] = S::ld(fin, (size_t)i * N + c, (R)Wc<L, i>::v);
      });
      R Fx, Fy, Fz;
      cell_force<L, S, true>(P, fin, flags, sdf, W, c, ix, iy, iz, f, Fx, Fy, Fz);
      accF[0] += (double)Fx;
      accF[1] += (double)Fy;
      accF[2] += (double)Fz;
    }
  }
  __shared__ double sh[NW][POST_SLOTS];
  __shared__ bool last;
  const unsigned full = 0xffffffffu;
  accF[0] = warp_sum(accF[0]);
  accF[1] = warp_sum(accF[1]);
  accF[2] = warp_sum(accF[2]);
  const uint32_t nsol = __reduce_add_sync(full, accSolid);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    sh[wid][0] = accF[0];
    sh[wid][1] = accF[1];
    sh[wid][2] = accF[2];
    sh[wid][3] = (double)nsol;
  }
  __syncthreads();
  if (threadIdx.x < POST_SLOTS) {
    double x = 0.0;
    for (int w = 0; w < NW; w++) x += sh[w][threadIdx.x];
    partials[(size_t)blockIdx.x * POST_SLOTS + threadIdx.x] = x;
  }
  // the last block to get here reduces everything (its partials are visible after the fence)
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(sets + SS_DONE, 1ull) == (unsigned long long)(gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  // accumulator sets: warp w < SS_COUNT takes slot w of the 64 sets (two per lane)
  __shared__ unsigned long long shS[SS_COUNT];
  if (wid < SS_COUNT) {
    unsigned long long v0 = sets[(size_t)lane * SMP_SET_U64 + wid];
    unsigned long long v1 = sets[(size_t)(lane + 32) * SMP_SET_U64 + wid];
    unsigned long long v = wid == SS_MAX ? (v0 > v1 ? v0 : v1) : v0 + v1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long u = __shfl_xor_sync(full, v, o);
      v = wid == SS_MAX ? (u > v ? u : v) : v + u;
    }
    if (lane == 0) shS[wid] = v;
  }
  // the blocks' partials in a fixed order
  double v[POST_SLOTS] = {0, 0, 0, 0};
  for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < POST_SLOTS; k++) v[k] += partials[(size_t)b * POST_SLOTS + k];
#pragma unroll
  for (int k = 0; k < POST_SLOTS; k++) v[k] = warp_sum(v[k]);
  __syncthreads();  // sh is reused
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < POST_SLOTS; k++) sh[wid][k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    double F[POST_SLOTS] = {0, 0, 0, 0};
    for (int w = 0; w < NW; w++)
      for (int k = 0; k < POST_SLOTS; k++) F[k] += sh[w][k];
    const bool big = shS[SS_NBIG] != 0ull;
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    result[0] = F[0];
    result[1] = F[1];
    result[2] = F[2];
    result[3] = (double)__uint_as_float((uint32_t)shS[SS_MAX]);
    result[4] = big ? nan : (double)(long long)shS[SS_RHOREF] / SMP_FIXED;
    result[5] = (double)shS[SS_NREF];
    result[6] = (double)shS[SS_NAN];
    result[7] = F[3];
    result[8] = big ? nan : (double)(long long)shS[SS_MASS] / SMP_FIXED;
    result[9] = (double)shS[SS_NFLUID];
  }
}

// final reduction of the per-block partials (one block of REDUCE_THREADS; fixed order, so the
// result is deterministic for a given number of partials)
constexpr int REDUCE_THREADS = 1024;

__global__ void __launch_bounds__(REDUCE_THREADS) k_reduce_partials(const double* __restrict__ partials,
                                                                   int nblocks, double* __restrict__ result,
                                                                   int nres) {
  __shared__ double sh[REDUCE_THREADS / 32][MACRO_SLOTS];
  double v[MACRO_SLOTS] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 4
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    const double2* p2 = reinterpret_cast<const double2*>(partials + (size_t)b * MACRO_SLOTS);
    const double2 a0 = p2[0], a1 = p2[1], a2 = p2[2], a3 = p2[3], a4 = p2[4];
    v[0] += a0.x;
    v[1] += a0.y;
    v[2] += a1.x;
    v[3] = fmax(v[3], a1.y);
    v[4] += a2.x;
    v[5] += a2.y;
    v[6] += a3.x;
    v[7] += a3.y;
    v[8] += a4.x;
    v[9] += a4.y;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < MACRO_SLOTS; k++) {
    if (k == 3) v[k] = (double)warp_max((float)v[k]);
    else v[k] = warp_sum(v[k]);
  }
  if (lane == 0)
    for (int k = 0; k < MACRO_SLOTS; k++) sh[wid][k] = v[k];
  __syncthreads();
  if (threadIdx.x < nres && threadIdx.x < MACRO_SLOTS) {
    const int k = threadIdx.x;
    double x = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) x = k == 3 ? fmax(x, sh[w][k]) : x + sh[w][k];
    result[k] = x;
  }
}

// ---------------------------------------------------------------------------------------------
// learned closure: box filter of a fine run onto the coarse grid (training data)
// ---------------------------------------------------------------------------------------------
// One thread per coarse cell (cx, cy, cz) over the fine cells (2 cx + a, 2 cy + b, 2 cz + c). Each
// fine cell's pulled, pre-collision populations (every boundary rule, cell_general) give rho, j and
// the non-equilibrium stress Pi; the fine run's own Smagorinsky stress is
//   sigma = -2 nu_sgs S = 3 nu_sgs Pi / (rho tau_s),  tau_s = (t0 + sqrt(t0^2 + 18 sqrt(2) Cs^2 |Pi| / rho)) / 2,
//   nu_sgs = (tau_s - t0) / 3 (t0 = the fine tau0),
// and the filtered quantities are
//   rho~ = <rho>,  u~ = <j> / <rho>,  T = <rho u u> / <rho> - u~ u~ + <sigma>
// (< > = mean over the 8 fine cells; stresses are invariant between the two lattices under the
// same lattice velocity). out (11 floats per coarse cell, structure of arrays [k * nc + cell]):
// rho~, u~ (3), T (xx, yy, zz, xy, xz, yz), valid (1 if all 8 fine cells are fluid, else 0).
template <class S>
__global__ void __launch_bounds__(128) k_closure_filter(const __grid_constant__ wt_kparams P,
                                                        const typename S::T* __restrict__ fin,
                                                        const uint32_t* __restrict__ flags,
                                                        const uint32_t* __restrict__ sdf,
                                                        const uint8_t* __restrict__ cls,
                                                        const __grid_constant__ Wheels W, int cnx, int cny, int cnz,
                                                        float* __restrict__ out) {
  typedef D3Q19 L;
  typedef typename S::R R;
  constexpr int Q = L::Q;
  const int cx = blockIdx.x * blockDim.x + threadIdx.x, cy = blockIdx.y, cz = blockIdx.z;
  if (cx >= cnx) return;
  const size_t nc = (size_t)cnx * cny * cnz;
  const size_t cidx = (size_t)cx + (size_t)cnx * ((size_t)cy + (size_t)cny * (size_t)cz);
  double srho = 0, sj[3] = {0, 0, 0}, suu[6] = {0, 0, 0, 0, 0, 0}, ssg[6] = {0, 0, 0, 0, 0, 0};
  bool valid = true;
  const double t0 = P.tau0;
  const double k = 18.0 * 1.4142135623730951 * (double)P.csmag2;
  for (int c = 0; c < 8 && valid; c++) {
    const int ix = 2 * cx + (c & 1), iy = 2 * cy + ((c >> 1) & 1), iz = 2 * cz + (c >> 2);
    const size_t idx = cell_id(ix, iy, iz, P.nx, P.ny);
    const uint8_t cl = cls[idx];
    if (cl & CLS_SOLID) {
      valid = false;
      break;
    }
    R f[Q];
    cell_general<L, S, true>(P, fin, flags, sdf, W, ix, iy, iz, cl, f);
    double rho = 0, j[3] = {0, 0, 0}, m[6] = {0, 0, 0, 0, 0, 0};
    static_for<Q>([&](auto I) {
      constexpr int i = I;
      constexpr int ex = L::c[i][0], ey = L::c[i][1], ez = L::c[i][2];
      const double v = (double)f[i];
      rho += v;
      j[0] += ex * v;
      j[1] += ey * v;
      j[2] += ez * v;
      m[0] += ex * ex * v;
      m[1] += ey * ey * v;
      m[2] += ez * ez * v;
      m[3] += ex * ey * v;
      m[4] += ex * ez * v;
      m[5] += ey * ez * v;
    });
    const double u[3] = {j[0] / rho, j[1] / rho, j[2] / rho};
    const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
    double pi[6], pn = 0;
    for (int q = 0; q < 6; q++) {
      pi[q] = m[q] - rho * (u[pa[q]] * u[pb[q]] + (q < 3 ? 1.0 / 3.0 : 0.0));
      pn += (q < 3 ? 1.0 : 2.0) * pi[q] * pi[q];
    }
    const double ts = 0.5 * (t0 + sqrt(t0 * t0 + k * sqrt(pn) / rho));
    const double nus = (ts - t0) / 3.0;
    srho += rho;
    for (int a = 0; a < 3; a++) sj[a] += j[a];
    for (int q = 0; q < 6; q++) {
      suu[q] += j[pa[q]] * j[pb[q]] / rho;
      ssg[q] += 3.0 * nus * pi[q] / (rho * ts);
    }
  }
  if (!valid) {
    for (int q = 0; q < 11; q++) out[(size_t)q * nc + cidx] = 0.0f;
    return;
  }
  const double u[3] = {sj[0] / srho, sj[1] / srho, sj[2] / srho};
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  out[cidx] = (float)(srho / 8.0);
  for (int a = 0; a < 3; a++) out[(size_t)(1 + a) * nc + cidx] = (float)u[a];
  for (int q = 0; q < 6; q++)
    out[(size_t)(4 + q) * nc + cidx] = (float)(suu[q] / srho - u[pa[q]] * u[pb[q]] + ssg[q] / 8.0);
  out[(size_t)10 * nc + cidx] = 1.0f;
}

// ---------------------------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------------------------
#define WT_DISPATCH(FN, ...)                                                                  \
  do {                                                                                        \
    if (s->is3d) {                                                                            \
      if (s->prec == WT_PREC_F16) return FN<D3Q19, StF16>(__VA_ARGS__);                      \
      if (s->prec == WT_PREC_F64) return FN<D3Q19, StF64>(__VA_ARGS__);                      \
      return FN<D3Q19, StF32>(__VA_ARGS__);                                                  \
    }                                                                                         \
    if (s->prec == WT_PREC_F16) return FN<D2Q9, StF16>(__VA_ARGS__);                         \
    if (s->prec == WT_PREC_F64) return FN<D2Q9, StF64>(__VA_ARGS__);                         \
    return FN<D2Q9, StF32>(__VA_ARGS__);                                                     \
  } while (0)

static bool offsets32(const wt_solver* s) { return (uint64_t)s->q * (uint64_t)s->n < (1ull << 32); }

static unsigned grid_cells(const wt_solver* s) { return (unsigned)std::min<size_t>((s->n + 255) / 256, 148 * 16); }

int lbm_block_x(const wt_solver* s) {
  if (s->block_x > 0) return s->block_x;
  const int nx = s->dims.nx;
  const int nb = (nx + 255) / 256;
  int bx = (nx + nb - 1) / nb;
  bx = (bx + 31) / 32 * 32;
  return bx < 32 ? 32 : bx;
}

static dim3 row_grid(const wt_solver* s, int bx) {
  return dim3((unsigned)((s->dims.nx + bx - 1) / bx), (unsigned)s->dims.ny, (unsigned)s->dims.nz);
}

template <class L>
static cudaError_t classify_t(wt_solver* s) {
  const int bx = lbm_block_x(s);
  k_classify<L><<<row_grid(s, bx), bx, 0, s->stream>>>(s->kp, s->flags, s->cls);
  s->launches++;
  return cudaGetLastError();
}

// Counts, then writes, the cells k_boundary_list selects (which: 0 boundary list, 1 solid list)
// into *list (grown to the count; *cap its capacity), *count the number of cells.
template <class L>
static cudaError_t cell_list_t(wt_solver* s, int which, uint32_t** list, size_t* cap, uint32_t* count) {
  cudaError_t e;
  const unsigned blocks = (unsigned)std::min<size_t>((s->n + 255) / 256, 148 * 16);
  if ((e = cudaMemsetAsync(s->bnd_count, 0, 4, s->stream)) != cudaSuccess) return e;
  k_boundary_list<L><<<blocks, 256, 0, s->stream>>>(s->kp, s->cls, s->gs, s->bnd_count, nullptr, 0, which);
  s->launches++;
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(s->bnd_count_host, s->bnd_count, 4, cudaMemcpyDeviceToHost, s->stream)) != cudaSuccess)
    return e;
  if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) return e;
  const uint32_t n = *s->bnd_count_host;
  if ((size_t)n > *cap) {
    if (*list) cudaFree(*list);
    *list = nullptr;
    *cap = 0;
    if ((e = cudaMalloc((void**)list, (size_t)n * 4)) != cudaSuccess) return e;
    *cap = n;
  }
  *count = n;
  if (n == 0) return cudaSuccess;
  if ((e = cudaMemsetAsync(s->bnd_count, 0, 4, s->stream)) != cudaSuccess) return e;
  k_boundary_list<L><<<blocks, 256, 0, s->stream>>>(s->kp, s->cls, s->gs, s->bnd_count, *list, 1, which);
  s->launches++;
  return cudaGetLastError();
}

template <class L>
static cudaError_t boundary_list_t(wt_solver* s) {
  cudaError_t e = cell_list_t<L>(s, 0, &s->bnd, &s->bnd_cap, &s->nbnd);
  if (e != cudaSuccess) return e;
  // the solid cells, for the fused sampling pass
  return cell_list_t<L>(s, 1, &s->solids, &s->solid_cap, &s->nsolid);
}

// Link records of the listed cells (vectorised f16 / f32 path only; see k_boundary_build).
template <class L, class S>
static cudaError_t boundary_table_t(wt_solver* s) {
  if constexpr (S::PREC == WT_PREC_F64) {
    return cudaSuccess;
  } else {
    if (s->nbnd == 0 || !offsets32(s)) return cudaSuccess;
    const size_t cap = ((size_t)s->nbnd + 63) / 64 * 64;
    cudaError_t e;
    if (cap > s->btab_cap) {
      cudaFree(s->bcell);
      cudaFree(s->brec);
      cudaFree(s->bgam);
      s->bcell = nullptr;
      s->brec = nullptr;
      s->bgam = nullptr;
      s->btab_cap = 0;
      if ((e = cudaMalloc((void**)&s->bcell, cap * sizeof(uint2))) != cudaSuccess) return e;
      if ((e = cudaMalloc((void**)&s->brec, cap * L::Q * sizeof(uint4))) != cudaSuccess) return e;
      if ((e = cudaMalloc((void**)&s->bgam, cap * L::Q * sizeof(float))) != cudaSuccess) return e;
      s->btab_cap = cap;
    }
    k_boundary_build<L, S><<<(s->nbnd + 127) / 128, 128, 0, s->stream>>>(
        s->kp, s->flags, s->sdf, s->cls, s->wheels, s->bnd, s->nbnd, (uint32_t)s->btab_cap, s->bcell, s->brec,
        s->bgam);
    s->launches++;
    return cudaGetLastError();
  }
}

template <class L, class S>
static cudaError_t classify_all_t(wt_solver* s) {
  cudaError_t e = classify_t<L>(s);
  if (e != cudaSuccess) return e;
  // solid cells are written with the rest state when each buffer is next a step's output
  s->solid_ok[0] = s->solid_ok[1] = false;
  if (s->gs == 1) {
    s->nbnd = 0;
    return cudaSuccess;
  }
  if ((e = boundary_list_t<L>(s)) != cudaSuccess) return e;
  return boundary_table_t<L, S>(s);
}

size_t rows_pipeline_smem(const wt_solver* s) {
  if (s->prec == WT_PREC_F16) return rows_smem_bytes<StF16>(s);
  if (s->prec == WT_PREC_F32) return rows_smem_bytes<StF32>(s);
  return 0;
}

cudaError_t launch_boundary_table(wt_solver* s) {
  if (s->gs == 1) return cudaSuccess;
  WT_DISPATCH(boundary_table_t, s);
}

cudaError_t launch_classify(wt_solver* s) {
  // group size of the bulk kernel's clean / boundary decision along x
  s->gs = s->dims.nx % 4 == 0 ? 4 : (s->dims.nx % 2 == 0 ? 2 : 1);
  WT_DISPATCH(classify_all_t, s);
}

template <class L, class S>
static cudaError_t init_t(wt_solver* s) {
  const int threads = 256;
  size_t blocks = (s->n + threads - 1) / threads;
  if (blocks > 148 * 32) blocks = 148 * 32;
  const int mode = s->params.init_mode == WT_INIT_REST_NOISE ? WT_INIT_REST_NOISE : WT_INIT_FREESTREAM;
  k_init<L, S><<<(unsigned)blocks, threads, 0, s->stream>>>(s->kp, (typename S::T*)s->f[0], (typename S::T*)s->f[1],
                                                            s->flags, mode, s->params.init_seed,
                                                            (float)s->params.init_noise);
  s->launches++;
  return cudaGetLastError();
}

// face cells of the learned closure's row buffer: every cell of the 2 ny + 2 (nz - 2) face rows
static size_t closure_face_cells(const wt_solver* s) {
  return (size_t)(2 * s->dims.ny + 2 * (s->dims.nz - 2)) * (size_t)s->dims.nx;
}

cudaError_t closure_rows_reserve(wt_solver* s, bool* grown) {
  *grown = false;
  if (!s->is3d) return cudaSuccess;
  const size_t rows = closure_face_cells(s) + s->btab_cap;
  if (rows <= s->lc_rows_cap && s->lc_rows) return cudaSuccess;
  cudaError_t e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return e;
  cudaFree(s->lc_rows);
  s->lc_rows = nullptr;
  s->lc_rows_cap = 0;
  if ((e = cudaMalloc((void**)&s->lc_rows, rows * (CL_IN + 1) * sizeof(float))) != cudaSuccess) return e;
  s->lc_rows_cap = rows;
  *grown = true;
  return cudaSuccess;
}

// the vectorised kernel indexes populations with 32-bit element offsets

// One step, fin -> fout. With smp (the fused sampling step, see sample_step_ok) the face, wall-cell
// and bulk kernels also run the sampling pass's per-cell work on what they store.
template <class L, class S>
static cudaError_t queue_step_t(wt_solver* const* ms, int count, int flip, unsigned* bar, int* err, cudaStream_t st);

template <class L, class S>
static cudaError_t sc_t(wt_solver* s, const void* fin, void* fout, const SampleOut* smp) {
  constexpr bool vec_ok = S::PREC == WT_PREC_F16 || S::PREC == WT_PREC_F32;
  const SampleOut none{};
  if (s->sc_kernel == WT_LAUNCH_QUEUE && smp == nullptr && persistent_ok(s)) {
    // the whole step (wall chunks, face tiles, bulk tiles) in one launch of the work queue
    const int par = fin == s->f[0] ? 0 : 1;
    wt_solver* one[1] = {s};
    s->launches++;
    return queue_step_t<L, S>(one, 1, s->parity ^ par, s->ps_bar, s->err_dev, s->stream);
  }
  if constexpr (vec_ok) {
    const int V = s->sc_param;
    const bool faces_ok = s->dims.ny >= 2 && (L::DIM == 2 || s->dims.nz >= 2);
    // the learned closure runs on this path only (bulk kernel k_stream_collide_lc)
    const ClosureDev* cw = L::DIM == 3 ? s->closure_dev : nullptr;
    if (cw != nullptr && !(s->dims.nx % 2 == 0 && s->gs >= 2 && faces_ok && offsets32(s)))
      return cudaErrorNotSupported;
    if (cw != nullptr || ((V == 2 || V == 4) && s->dims.nx % V == 0 && s->gs >= V && faces_ok && offsets32(s))) {
      const int runs = s->dims.nx / V;
      int bx = s->sc_bx, by = s->sc_by;
      if (bx <= 0 || by <= 0) {
        // default block: one row of up to 128 threads (the tuner's usual choice on large tunnels)
        bx = runs >= 128 ? 128 : ((runs + 31) / 32) * 32;
        by = 1;
      }
      const dim3 block(bx, by);
      const dim3 grid((runs + bx - 1) / bx, (s->dims.ny + by - 1) / by, s->dims.nz);
      cudaError_t e = cudaSuccess;
      // no kernel of this path writes solid cells: the output buffer gets the rest state once
      const int out = fout == s->f[0] ? 0 : 1;
      if (!s->solid_ok[out]) {
        k_fill_solid<L, S><<<grid_cells(s), 256, 0, s->stream>>>(s->kp, s->cls, (typename S::T*)fout);
        s->launches++;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        s->solid_ok[out] = true;
      }
      // face rows and the per-cell boundary list on the auxiliary stream, overlapping the bulk
      cudaStream_t bs = s->aux ? s->aux : s->stream;
      if (s->aux) {
        if ((e = cudaEventRecord(s->ev_fork, s->stream)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s->aux, s->ev_fork, 0)) != cudaSuccess) return e;
      }
      {
        const int fr = L::DIM == 3 ? 2 * s->dims.ny + 2 * (s->dims.nz - 2) : 2;
        const int runs2 = s->dims.nx / 2;
        const int fbx = runs2 >= 128 ? 128 : ((runs2 + 31) / 32) * 32;
        const int fby = 256 / fbx;
        const dim3 fgrid((runs2 + fbx - 1) / fbx, (fr + fby - 1) / fby, 1);
        if constexpr (L::DIM == 3) {
          if (cw != nullptr) {
            // learned closure: features of the face rows and wall cells, one tensor-core pass for
            // their eddy viscosities, then their collisions
            const size_t fc = closure_face_cells(s);
            const size_t rows = fc + (size_t)s->nbnd;
            if (s->lc_rows == nullptr || rows > s->lc_rows_cap) return cudaErrorInvalidValue;
            float* xb = s->lc_rows;
            float* nub = s->lc_rows + s->lc_rows_cap * CL_IN;
            k_face_lc<L, S, FM_FEATURES><<<fgrid, dim3(fbx, fby), 0, bs>>>(
                s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->cls, s->gs, s->sdf, xb, nub);
            s->launches++;
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
            if (s->nbnd > 0) {
              k_boundary_tab<L, S, FM_FEATURES><<<(s->nbnd + 63) / 64, 64, 0, bs>>>(
                  s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->bcell, s->brec, s->bgam, s->nbnd,
                  (uint32_t)s->btab_cap, s->sdf, xb + fc * CL_IN, nub + fc, none);
              s->launches++;
              if ((e = cudaGetLastError()) != cudaSuccess) return e;
            }
            k_closure_rows<<<(unsigned)((rows + 2 * LC_THREADS - 1) / (2 * LC_THREADS)), LC_THREADS, LC_SMEM_BYTES,
                             bs>>>(xb, (uint32_t)rows, nub, cw, s->closure_p, s->err_dev);
            s->launches++;
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
            k_face_lc<L, S, FM_NU><<<fgrid, dim3(fbx, fby), 0, bs>>>(
                s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->cls, s->gs, s->sdf, xb, nub);
          } else if (smp) {
            k_face_v<L, S, true><<<fgrid, dim3(fbx, fby), 0, bs>>>(s->kp, (const typename S::T*)fin,
                                                                   (typename S::T*)fout, s->cls, s->gs, *smp);
          } else {
            k_face_v<L, S><<<fgrid, dim3(fbx, fby), 0, bs>>>(s->kp, (const typename S::T*)fin,
                                                             (typename S::T*)fout, s->cls, s->gs, none);
          }
        } else if (smp) {
          k_face_v<L, S, true><<<fgrid, dim3(fbx, fby), 0, bs>>>(s->kp, (const typename S::T*)fin,
                                                                 (typename S::T*)fout, s->cls, s->gs, *smp);
        } else {
          k_face_v<L, S><<<fgrid, dim3(fbx, fby), 0, bs>>>(s->kp, (const typename S::T*)fin, (typename S::T*)fout,
                                                           s->cls, s->gs, none);
        }
        s->launches++;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
      }
      if (s->nbnd > 0) {
        if (cw != nullptr) {
          if constexpr (L::DIM == 3) {
            const size_t fc = closure_face_cells(s);
            k_boundary_tab<L, S, FM_NU><<<(s->nbnd + 63) / 64, 64, 0, bs>>>(
                s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->bcell, s->brec, s->bgam, s->nbnd,
                (uint32_t)s->btab_cap, s->sdf, nullptr, s->lc_rows + s->lc_rows_cap * CL_IN + fc, none);
          }
        } else if (smp) {
          k_boundary_tab<L, S, FM_SMAG, true><<<(s->nbnd + 63) / 64, 64, 0, bs>>>(
              s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->bcell, s->brec, s->bgam, s->nbnd,
              (uint32_t)s->btab_cap, s->sdf, nullptr, nullptr, *smp);
        } else {
          k_boundary_tab<L, S><<<(s->nbnd + 63) / 64, 64, 0, bs>>>(
              s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->bcell, s->brec, s->bgam, s->nbnd,
              (uint32_t)s->btab_cap, s->sdf, nullptr, nullptr, none);
        }
        s->launches++;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
      }
      // the bulk kernel on the main stream, concurrently with the auxiliary work; steps writing
      // buffer 1 sweep z upwards, steps writing buffer 0 downwards
      const int zrev = fout == s->f[0] ? 1 : 0;
      // the vectorised kernel's per-direction plane bases for this step (pointer arithmetic on
      // integers: a base may lie before the buffer; the cells that use it index into it)
      DirPtrs<typename S::T> dp;
      {
        const int64_t N = (int64_t)s->kp.n, sy = s->dims.nx, sz = (int64_t)s->dims.nx * s->dims.ny;
        for (int i = 0; i < L::Q; i++) {
          const int64_t off = (int64_t)i * N - (int64_t)L::c[i][1] * sy - (int64_t)(L::DIM == 3 ? L::c[i][2] : 0) * sz;
          dp.in[i] = (const typename S::T*)((uintptr_t)fin + (uintptr_t)(off * (int64_t)sizeof(typename S::T)));
          dp.out[i] = (typename S::T*)fout + (size_t)i * (size_t)N;
        }
        for (int i = L::Q; i < 19; i++) dp.in[i] = nullptr, dp.out[i] = nullptr;
      }
#define WT_LAUNCH_V(VV, MB)                                                                                     \
  do {                                                                                                             \
    if (s->kp.collision == 1u)                                                                                     \
      k_stream_collide_v<L, S, VV, MB, true><<<grid, block, 0, s->stream>>>(                                       \
          s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->cls, s->gs, zrev, none, dp);                  \
    else                                                                                                           \
      k_stream_collide_v<L, S, VV, MB, false><<<grid, block, 0, s->stream>>>(                                      \
          s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->cls, s->gs, zrev, none, dp);                  \
  } while (0)
      const int mb = s->sc_kernel;
      if constexpr (L::DIM == 3) {
        if (cw != nullptr) {
          // learned closure: 128-thread blocks, one tile of tpr cell pairs x 128 / tpr rows each
          const int runs2 = s->dims.nx / 2;
          const int tpr = runs2 > 64 ? 128 : (runs2 > 32 ? 64 : 32);
          const int rpb = LC_THREADS / tpr;
          const int64_t ntiles = (int64_t)((runs2 + tpr - 1) / tpr) * ((s->dims.ny + rpb - 1) / rpb) * s->dims.nz;
          auto kern = s->kp.collision == 1u ? k_stream_collide_lc<S, true> : k_stream_collide_lc<S, false>;
          const int64_t grid_lc = (ntiles + LC_TILES_PER_BLOCK - 1) / LC_TILES_PER_BLOCK;
          kern<<<(unsigned)grid_lc, LC_THREADS, LC_SMEM_BYTES, s->stream>>>(
              s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->cls, s->gs, s->sdf, cw, s->closure_p,
              tpr, (uint32_t)ntiles, s->err_dev);
          s->launches++;
          if ((e = cudaGetLastError()) != cudaSuccess) return e;
          if (s->aux) {
            if ((e = cudaEventRecord(s->ev_join, s->aux)) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(s->stream, s->ev_join, 0)) != cudaSuccess) return e;
          }
          return cudaSuccess;
        }
      }
      if constexpr (L::DIM == 3) {
        const size_t rp_smem = rows_smem_bytes<S>(s);
        if (mb == WT_LAUNCH_ROW_PIPELINE && V == 2 && rp_smem > 0 && !smp) {
          // row pipeline: `by` interior rows per block (default 4)
          const uint32_t nrows = (uint32_t)(s->dims.ny - 2) * (uint32_t)(s->dims.nz - 2);
          const uint32_t rows = s->sc_by > 0 ? (uint32_t)s->sc_by : 4u;
          auto kern = s->kp.collision == 1u ? k_stream_collide_rows<S, true> : k_stream_collide_rows<S, false>;
          kern<<<(nrows + rows - 1) / rows, RP_THREADS, rp_smem, s->stream>>>(
              s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->cls, s->gs, nrows, rows, s->rp_wait_limit,
              s->err_dev);
          s->launches++;
          if ((e = cudaGetLastError()) != cudaSuccess) return e;
          if (s->aux) {
            if ((e = cudaEventRecord(s->ev_join, s->aux)) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(s->stream, s->ev_join, 0)) != cudaSuccess) return e;
          }
          return cudaSuccess;
        }
      }
      if (smp) {
        // the sampling step: the regularized collision keeps the bulk kernel's occupancy hint of 4
        // (64 registers, no spills with the sampling state); BGK and four cells per thread run
        // without a register cap (they would spill under it)
        const bool bgk = s->kp.collision == 1u;
        if (V == 2) {
          if (bgk) k_stream_collide_v<L, S, 2, 0, true, true><<<grid, block, 0, s->stream>>>(
                       s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->cls, s->gs, zrev, *smp, dp);
          else k_stream_collide_v<L, S, 2, 4, false, true><<<grid, block, 0, s->stream>>>(
                   s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->cls, s->gs, zrev, *smp, dp);
        } else {
          if (bgk) k_stream_collide_v<L, S, 4, 0, true, true><<<grid, block, 0, s->stream>>>(
                       s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->cls, s->gs, zrev, *smp, dp);
          else k_stream_collide_v<L, S, 4, 0, false, true><<<grid, block, 0, s->stream>>>(
                   s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->cls, s->gs, zrev, *smp, dp);
        }
      } else if (V == 2) {
        if (mb == 2) WT_LAUNCH_V(2, 2);
        else if (mb == 3) WT_LAUNCH_V(2, 3);
        else if (mb == 4) WT_LAUNCH_V(2, 4);
        else WT_LAUNCH_V(2, 0);
      } else {
        if (mb == 2) WT_LAUNCH_V(4, 2);
        else if (mb == 3) WT_LAUNCH_V(4, 3);
        else WT_LAUNCH_V(4, 0);
      }
#undef WT_LAUNCH_V
      s->launches++;
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      if (s->aux) {
        if ((e = cudaEventRecord(s->ev_join, s->aux)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s->stream, s->ev_join, 0)) != cudaSuccess) return e;
      }
      return cudaSuccess;
    }
  }
  if (smp) return cudaErrorNotSupported;  // sample_step_ok excludes the scalar kernel
  const int bx = lbm_block_x(s);
  k_stream_collide<L, S><<<row_grid(s, bx), bx, 0, s->stream>>>(
      s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->cls, s->flags, s->sdf, s->wheels);
  s->launches++;
  s->solid_ok[fout == s->f[0] ? 0 : 1] = true;  // this kernel writes the solid cells itself
  return cudaGetLastError();
}

template <class L, class S>
static cudaError_t macro_t(wt_solver* s) {
  k_macro<L, S><<<s->partial_blocks, MACRO_THREADS, 0, s->stream>>>(
      s->kp, (const typename S::T*)s->f[s->parity], s->flags, s->sdf, s->cls, s->wheels, s->vel, s->meanA, s->meanB,
      s->partials);
  s->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_reduce_partials<<<1, REDUCE_THREADS, 0, s->stream>>>(s->partials, s->partial_blocks, s->result_dev, MACRO_SLOTS);
  s->launches++;
  return cudaGetLastError();
}


cudaError_t launch_init(wt_solver* s) { WT_DISPATCH(init_t, s); }

bool sample_step_ok(const wt_solver* s) {
  if (!(s->prec == WT_PREC_F16 || s->prec == WT_PREC_F32) || s->closure_dev != nullptr || s->cls_dirty) return false;
  const int V = s->sc_param;
  const bool faces_ok = s->dims.ny >= 2 && (!s->is3d || s->dims.nz >= 2);
  if (!((V == 2 || V == 4) && s->dims.nx % V == 0 && s->gs >= V && faces_ok && offsets32(s))) return false;
  // the row pipeline has no sampling form (its steps stay unfused)
  return !(s->is3d && s->sc_kernel == WT_LAUNCH_ROW_PIPELINE && V == 2 && rows_pipeline_smem(s) > 0);
}

template <class L, class S>
static cudaError_t sample_step_t(wt_solver* s, const void* fin, void* fout) {
  if constexpr (S::PREC == WT_PREC_F64) {
    return cudaErrorNotSupported;
  } else {
    cudaError_t e;
    if ((e = cudaMemsetAsync(s->smp_sets, 0, SMP_SETS * SMP_SET_U64 * sizeof(unsigned long long), s->stream)) !=
        cudaSuccess)
      return e;
    const SampleOut O{s->vel, s->meanA, s->meanB, s->smp_sets};
    if ((e = sc_t<L, S>(s, fin, fout, &O)) != cudaSuccess) return e;
    // after the whole step: the wall force of the listed cells and the solid cells, on what it stored
    const uint32_t items = s->nbnd + s->nsolid;
    const int blocks = (int)std::max<size_t>(1, std::min<size_t>(((size_t)items + MACRO_THREADS - 1) / MACRO_THREADS,
                                                                  (size_t)s->partial_blocks));
    k_sample_post<L, S><<<blocks, MACRO_THREADS, 0, s->stream>>>(
        s->kp, (const typename S::T*)fout, s->flags, s->sdf, s->cls, s->wheels, s->bnd, s->nbnd, s->solids,
        s->nsolid, s->vel, s->meanA, s->meanB, s->partials, s->smp_sets, s->result_dev);
    s->launches++;
    return cudaGetLastError();
  }
}

cudaError_t launch_sample_step(wt_solver* s, const void* fin, void* fout) { WT_DISPATCH(sample_step_t, s, fin, fout); }
cudaError_t launch_stream_collide(wt_solver* s, const void* fin, void* fout) {
  const SampleOut* none = nullptr;
  WT_DISPATCH(sc_t, s, fin, fout, none);
}
cudaError_t launch_macro(wt_solver* s) { WT_DISPATCH(macro_t, s); }

bool persistent_ok(const wt_solver* s) {
  if (!(s->prec == WT_PREC_F16 || s->prec == WT_PREC_F32) || s->closure_dev != nullptr || s->cls_dirty) return false;
  const bool faces_ok = s->dims.ny >= 2 && (!s->is3d || s->dims.nz >= 2);
  return s->dims.nx % 2 == 0 && s->gs >= 2 && faces_ok && offsets32(s) && s->solid_ok[0] && s->solid_ok[1] &&
         (s->nbnd == 0 || s->btab_cap >= s->nbnd);
}

// The step items of `count` tunnels (wall chunks, then face tiles, then bulk tiles of every
// tunnel); tunnel k starts at parity ms[k]->parity ^ flip.
static cudaError_t persistent_table(wt_solver* const* ms, int count, int flip, PersistTable& tab) {
  if (count < 1 || count > PS_MAX_TUNNELS) return cudaErrorInvalidValue;
  std::memset(&tab, 0, sizeof tab);
  uint32_t nwall[PS_MAX_TUNNELS], nface[PS_MAX_TUNNELS], nbulk[PS_MAX_TUNNELS];
  for (int k = 0; k < count; k++) {
    const wt_solver* s = ms[k];
    PersistTunnel& t = tab.t[k];
    t.P = s->kp;
    t.f[0] = s->f[0];
    t.f[1] = s->f[1];
    t.cls = s->cls;
    t.bcell = s->bcell;
    t.brec = s->brec;
    t.bgam = s->bgam;
    t.nbnd = s->nbnd;
    t.btab_cap = (uint32_t)s->btab_cap;
    t.gs = s->gs;
    t.p0 = s->parity ^ flip;
    const uint32_t half = (uint32_t)s->dims.nx / 2u;
    t.tbx = half >= 256 ? 256u : (half >= 128 ? 128u : (half >= 64 ? 64u : 32u));
    t.tby = (uint32_t)PS_THREADS / t.tbx;
    t.ttx = (half + t.tbx - 1) / t.tbx;
    t.tty = ((uint32_t)s->dims.ny + t.tby - 1) / t.tby;
    nbulk[k] = t.ttx * t.tty * (uint32_t)s->dims.nz;
    const uint32_t fr = s->is3d ? 2u * (uint32_t)s->dims.ny + 2u * (uint32_t)(s->dims.nz - 2) : 2u;
    nface[k] = (fr * half + PS_THREADS - 1) / PS_THREADS;
    nwall[k] = (s->nbnd + PS_THREADS - 1) / PS_THREADS;
  }
  uint32_t items = 0;
  for (int k = 0; k < count; k++) tab.t[k].wi0 = items, items += nwall[k];
  tab.fseg = items;
  for (int k = 0; k < count; k++) tab.t[k].fi0 = items, items += nface[k];
  tab.bseg = items;
  for (int k = 0; k < count; k++) tab.t[k].bi0 = items, items += nbulk[k];
  tab.count = (uint32_t)count;
  tab.items = items;
  return cudaSuccess;
}

// resident blocks of `kern` on the device of ms[0], at most `items`
template <class K>
static cudaError_t persistent_grid(K kern, wt_solver* const* ms, uint32_t items, unsigned* grid) {
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, PS_THREADS, 0);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  *grid = (unsigned)std::min<size_t>(items, (size_t)per_sm * (size_t)ms[0]->num_sms);
  return cudaSuccess;
}

template <class L, class S>
static cudaError_t persistent_t(wt_solver* const* ms, int count, int steps, unsigned* bar, int* err,
                                cudaStream_t st) {
  if constexpr (S::PREC == WT_PREC_F64) {
    return cudaErrorNotSupported;
  } else {
    if (steps < 1) return cudaErrorInvalidValue;
    PersistTable tab;
    cudaError_t e = persistent_table(ms, count, 0, tab);
    if (e != cudaSuccess) return e;
    auto kern = ms[0]->kp.collision == 1u ? k_steps_persistent<L, S, true, true> : k_steps_persistent<L, S, false, true>;
    unsigned grid = 0;
    if ((e = persistent_grid(kern, ms, tab.items, &grid)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(bar, 0, PS_BAR_WORDS * sizeof(unsigned), st)) != cudaSuccess) return e;
    int k0 = 0;
    void* args[] = {(void*)&tab, (void*)&steps, (void*)&k0, (void*)&bar, (void*)&err};
    return cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(PS_THREADS), args, 0, st);
  }
}

cudaError_t launch_persistent(wt_solver* const* ms, int count, int steps, unsigned* bar, int* err, cudaStream_t st) {
  const wt_solver* s = ms[0];
  for (int k = 1; k < count; k++)
    if (ms[k]->is3d != s->is3d || ms[k]->prec != s->prec || ms[k]->kp.collision != s->kp.collision)
      return cudaErrorInvalidValue;
  WT_DISPATCH(persistent_t, ms, count, steps, bar, err, st);
}

template <class L, class S>
static cudaError_t queue_step_t(wt_solver* const* ms, int count, int flip, unsigned* bar, int* err, cudaStream_t st) {
  if constexpr (S::PREC == WT_PREC_F64) {
    return cudaErrorNotSupported;
  } else {
    PersistTable tab;
    cudaError_t e = persistent_table(ms, count, flip, tab);
    if (e != cudaSuccess) return e;
    auto kern =
        ms[0]->kp.collision == 1u ? k_steps_persistent<L, S, true, false> : k_steps_persistent<L, S, false, false>;
    unsigned grid = 0;
    if ((e = persistent_grid(kern, ms, tab.items, &grid)) != cudaSuccess) return e;
    // Programmatic stream serialisation for steps of at most two item waves (launch-bound steps,
    // such as small 2-D channels): the launch may overlap the end of the previous kernel on the
    // stream (the kernel waits for it before its first access). Large steps launch plainly: blocks
    // scheduled early would only hold slots the previous step's last items need.
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(PS_THREADS);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = tab.items <= 2u * grid ? 1 : 0;
    int one = 1, zero = 0;
    return cudaLaunchKernelEx(&cfg, kern, tab, one, zero, bar, err);
  }
}

cudaError_t launch_queue_step(wt_solver* const* ms, int count, int k0, unsigned* bar, int* err, cudaStream_t st) {
  const wt_solver* s = ms[0];
  for (int k = 1; k < count; k++)
    if (ms[k]->is3d != s->is3d || ms[k]->prec != s->prec || ms[k]->kp.collision != s->kp.collision)
      return cudaErrorInvalidValue;
  WT_DISPATCH(queue_step_t, ms, count, k0 & 1, bar, err, st);
}

bool batch_fusable(const wt_solver* s) {
  return s->is3d && (s->prec == WT_PREC_F16 || s->prec == WT_PREC_F32) && s->closure_dev == nullptr &&
         s->dims.nx % 2 == 0 && s->gs >= 2 && s->dims.ny >= 2 && s->dims.nz >= 2 && offsets32(s) &&
         s->solid_ok[0] && s->solid_ok[1];
}

template <class L, class S>
static cudaError_t aux_t(wt_solver* s, const void* fin, void* fout, cudaStream_t origin) {
  if constexpr (L::DIM == 3 && (S::PREC == WT_PREC_F16 || S::PREC == WT_PREC_F32)) {
    cudaError_t e;
    if ((e = cudaEventRecord(s->ev_fork, origin)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(s->aux, s->ev_fork, 0)) != cudaSuccess) return e;
    const int fr = 2 * s->dims.ny + 2 * (s->dims.nz - 2);
    const int runs2 = s->dims.nx / 2;
    const int fbx = runs2 >= 128 ? 128 : ((runs2 + 31) / 32) * 32;
    const int fby = 256 / fbx;
    const dim3 fgrid((runs2 + fbx - 1) / fbx, (fr + fby - 1) / fby, 1);
    k_face_v<L, S><<<fgrid, dim3(fbx, fby), 0, s->aux>>>(s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->cls,
                                                         s->gs, SampleOut{});
    s->launches++;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (s->nbnd > 0) {
      k_boundary_tab<L, S><<<(s->nbnd + 63) / 64, 64, 0, s->aux>>>(
          s->kp, (const typename S::T*)fin, (typename S::T*)fout, s->bcell, s->brec, s->bgam, s->nbnd,
          (uint32_t)s->btab_cap, s->sdf, nullptr, nullptr, SampleOut{});
      s->launches++;
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaEventRecord(s->ev_join, s->aux);
  } else {
    return cudaErrorNotSupported;
  }
}

cudaError_t launch_aux_kernels(wt_solver* s, const void* fin, void* fout, cudaStream_t origin) {
  WT_DISPATCH(aux_t, s, fin, fout, origin);
}

cudaError_t launch_batch_bulk(int prec, bool bgk, const BatchTable& tab, uint32_t tiles, cudaStream_t st) {
  const dim3 block(BATCH_BX, BATCH_BY);
  if (prec == WT_PREC_F16) {
    if (bgk) k_batch_bulk<StF16, 0, true><<<tiles, block, 0, st>>>(tab);
    else k_batch_bulk<StF16, 4, false><<<tiles, block, 0, st>>>(tab);
  } else {
    if (bgk) k_batch_bulk<StF32, 0, true><<<tiles, block, 0, st>>>(tab);
    else k_batch_bulk<StF32, 4, false><<<tiles, block, 0, st>>>(tab);
  }
  return cudaGetLastError();
}

cudaError_t launch_closure_filter(wt_solver* fine, int cnx, int cny, int cnz, float* out, cudaStream_t st) {
  const wt_solver* s = fine;
  if (!s->is3d) return cudaErrorNotSupported;
  const int bx = cnx >= 128 ? 128 : ((cnx + 31) / 32) * 32;
  const dim3 grid((unsigned)((cnx + bx - 1) / bx), (unsigned)cny, (unsigned)cnz);
#define WT_FILTER(SS)                                                                                         \
  k_closure_filter<SS><<<grid, bx, 0, st>>>(s->kp, (const typename SS::T*)s->f[s->parity], s->flags, s->sdf, \
                                            s->cls, s->wheels, cnx, cny, cnz, out)
  if (s->prec == WT_PREC_F16) WT_FILTER(StF16);
  else if (s->prec == WT_PREC_F64) WT_FILTER(StF64);
  else WT_FILTER(StF32);
#undef WT_FILTER
  fine->launches++;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// sampling pass on caller-owned buffers, with its reduction scratch in a fixed device array
// ---------------------------------------------------------------------------------------------
// Some hosts may not allocate device memory at all (their memory belongs to another allocator,
// and cudaMalloc / cudaFree would synchronise the device behind its back). For them the macro
// pass's per-block partial sums live in this file-scope array instead of a handle's buffer: one
// MACRO_SLOTS-double record per block of MACRO_THREADS cells, enough for WT_SAMPLE_NOALLOC_MAX_CELLS
// cells (1.25 MiB). k_macro writes all slots of every block it runs before k_reduce_partials reads them, so what
// an earlier call left in the array is never read and nothing is cleared. The array is shared by
// every call on a device: calls that overlap on the GPU race on it.
constexpr int NOALLOC_MAX_BLOCKS = WT_SAMPLE_NOALLOC_MAX_CELLS / MACRO_THREADS;
static_assert(NOALLOC_MAX_BLOCKS * MACRO_THREADS == WT_SAMPLE_NOALLOC_MAX_CELLS, "whole blocks");
static __device__ __align__(256) double g_sample_scratch[NOALLOC_MAX_BLOCKS * MACRO_SLOTS];

namespace {

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_scratch_mu;
double* g_scratch_ptr[NOALLOC_MAX_DEVICES] = {};

// Device address of g_sample_scratch on `dev`, which must be the current device. Looked up on the
// first call for that device (this may load the module's device code) and cached.
// A cached address is checked against the current context first: after cudaDeviceReset (a new
// primary context, the module loaded again) the old address no longer names device memory of
// `dev`, and the symbol is looked up again.
cudaError_t scratch_address(int dev, double** out) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (g_scratch_ptr[dev]) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, g_scratch_ptr[dev]) != cudaSuccess || a.type != cudaMemoryTypeDevice ||
        a.device != dev) {
      cudaGetLastError();
      g_scratch_ptr[dev] = nullptr;
    }
  }
  if (!g_scratch_ptr[dev]) {
    double* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_sample_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = ptr;
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

template <class L, class S>
cudaError_t sample_noalloc_t(const wt_kparams& kp, const void* fin, const uint32_t* flags, const uint32_t* sdf,
                             const Wheels& W, uint2* vel, float4* meanA, float* meanB, double* scratch, int nblocks,
                             double* result, cudaStream_t st) {
  k_macro<L, S><<<nblocks, MACRO_THREADS, 0, st>>>(kp, (const typename S::T*)fin, flags, sdf, nullptr, W, vel, meanA,
                                                    meanB, scratch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_reduce_partials<<<1, REDUCE_THREADS, 0, st>>>(scratch, nblocks, result, 8);
  return cudaGetLastError();
}

// a caller's buffer must be device (or managed) memory of `dev`, aligned to `align` bytes
const char* buffer_problem(const void* p, size_t align, int dev) {
  if (!p) return "is NULL";
  if ((uintptr_t)p % align != 0) return "is misaligned for its element type";
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return "is not a CUDA pointer";
  }
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) return "is not device memory";
  if (a.device != dev) return "is on another device than the current one";
  return nullptr;
}

}  // namespace
}  // namespace wt

extern "C" int wt_sample_noalloc(const wt_dims* dims, const wt_params* p, const wt_wheel* wheels, int32_t nwheels,
                                 const void* populations, const uint32_t* flags, const uint32_t* sdf_encoded,
                                 void* vel_half4, float* mean4, float* meanb, double* result8, void* stream) {
  using namespace wt;
  auto invalid = [](const std::string& m) { return fail_unbound(WT_E_INVALID, "wt_sample_noalloc: " + m); };
  if (!dims || !p) return invalid("dims and params are required");
  if (dims->nx < 1 || dims->ny < 1 || dims->nz < 1) return invalid("dims must be >= 1");
  const uint64_t n = (uint64_t)dims->nx * (uint64_t)dims->ny * (uint64_t)dims->nz;
  if (n > (uint64_t)WT_SAMPLE_NOALLOC_MAX_CELLS)
    return invalid(std::to_string(n) + " cells exceed the limit of " + std::to_string(WT_SAMPLE_NOALLOC_MAX_CELLS) +
                   " cells set by the fixed reduction scratch (1.25 MiB); use a handle (wt_create) for larger grids");
  if (p->precision < WT_PREC_F32 || p->precision > WT_PREC_F64) return invalid("bad precision");
  if (nwheels < 0 || nwheels > 16 || (nwheels > 0 && !wheels)) return invalid("need 0..16 wheels and a wheel array");
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
    cudaGetLastError();
    return fail_unbound(WT_E_NO_DEVICE, "wt_sample_noalloc: no CUDA device");
  }
  if (dev >= NOALLOC_MAX_DEVICES) return invalid("device ordinal above 63");
  const size_t elem = p->precision == WT_PREC_F16 ? 2 : (p->precision == WT_PREC_F64 ? 8 : 4);
  const struct {
    const void* ptr;
    size_t align;
    const char* name;
  } bufs[] = {{populations, elem, "populations"}, {flags, 4, "flags"},  {sdf_encoded, 4, "sdf_encoded"},
              {vel_half4, 8, "vel_half4"},      {mean4, 16, "mean4"}, {meanb, 4, "meanb"},
              {result8, 8, "result8"}};
  for (const auto& b : bufs)
    if (const char* why = buffer_problem(b.ptr, b.align, dev)) return invalid(std::string(b.name) + " " + why);

  double* scratch = nullptr;
  cudaError_t e = scratch_address(dev, &scratch);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail_unbound(WT_E_CUDA, std::string("wt_sample_noalloc: cudaGetSymbolAddress(scratch): ") +
                                       cudaGetErrorString(e));
  }
  wt_kparams kp;
  wt_pack_params(dims, p, &kp);
  Wheels W{};
  W.count = (uint32_t)nwheels;
  for (int k = 0; k < nwheels; k++) {
    const double r = wheels[k].r > 1e-3 ? wheels[k].r : 1e-3;
    W.w[2 * k] = make_float4((float)wheels[k].c[0], (float)wheels[k].c[1], (float)wheels[k].c[2], (float)(1.0 / r));
    W.w[2 * k + 1] =
        make_float4((float)wheels[k].axis[0], (float)wheels[k].axis[1], (float)wheels[k].axis[2], (float)wheels[k].hw);
  }
  const int nblocks = (int)((n + MACRO_THREADS - 1) / MACRO_THREADS);
  const cudaStream_t st = (cudaStream_t)stream;
  auto* vel = (uint2*)vel_half4;
  auto* mA = (float4*)mean4;
  if (dims->nz > 1) {
    if (p->precision == WT_PREC_F16)
      e = sample_noalloc_t<D3Q19, StF16>(kp, populations, flags, sdf_encoded, W, vel, mA, meanb, scratch, nblocks,
                                         result8, st);
    else if (p->precision == WT_PREC_F64)
      e = sample_noalloc_t<D3Q19, StF64>(kp, populations, flags, sdf_encoded, W, vel, mA, meanb, scratch, nblocks,
                                         result8, st);
    else
      e = sample_noalloc_t<D3Q19, StF32>(kp, populations, flags, sdf_encoded, W, vel, mA, meanb, scratch, nblocks,
                                         result8, st);
  } else {
    if (p->precision == WT_PREC_F16)
      e = sample_noalloc_t<D2Q9, StF16>(kp, populations, flags, sdf_encoded, W, vel, mA, meanb, scratch, nblocks,
                                        result8, st);
    else if (p->precision == WT_PREC_F64)
      e = sample_noalloc_t<D2Q9, StF64>(kp, populations, flags, sdf_encoded, W, vel, mA, meanb, scratch, nblocks,
                                        result8, st);
    else
      e = sample_noalloc_t<D2Q9, StF32>(kp, populations, flags, sdf_encoded, W, vel, mA, meanb, scratch, nblocks,
                                        result8, st);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail_unbound(WT_E_CUDA, std::string("wt_sample_noalloc: launch: ") + cudaGetErrorString(e));
  }
  return WT_OK;
}
