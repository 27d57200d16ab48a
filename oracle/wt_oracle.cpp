/*
 * wt_oracle.cpp — CPU restatement of the reference's hot-path arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the parity checker for the CUDA path: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it. The product path
 * (windtunnel_vis_b200, libwt.so) never links, loads or calls it.
 *
 * Parity status: the reference (TypeScript generating WGSL, run through WebGPU) cannot execute
 * on these machines, and it ships no golden vectors. This restatement is pinned to the
 * reference's own lattice tables (tests/golden/lattice.json, extracted from
 * src/solver/lattice.ts) and to the pass bands of the reference's validation cases
 * (src/analysis/validation.ts:61-136, src/test/harness.ts:20-39). Bit-level agreement with the
 * reference's shaders themselves is unpinned.
 *
 * What is restated (paths relative to the reference project):
 *   lattice tables ............ src/solver/lattice.ts:20-60
 *   parameter packing ......... src/solver/SolverGPU.ts:160-187
 *   wheel / sdf packing ....... src/solver/SolverGPU.ts:312-335
 *   stream + collide .......... src/solver/wgslLbm.ts:58-293 (f32, packed f16, and an f64 variant)
 *   init ...................... src/solver/wgslLbm.ts:296-341
 *   macro / force / reduce .... src/solver/wgslLbm.ts:347-521, SolverGPU.ts:272-308
 *   GPU voxelizer (f32) ....... src/voxelize/wgslVoxel.ts:33-322, VoxelizerGPU.ts:48-151
 *   CPU voxelizer (f64) ....... src/voxelize/voxelizeCPU.ts:11-199
 *   particle tracers .......... src/render/tracers.ts:3-106, render/wgslRender.ts:22-37
 *   derived fields, export .... src/solver/wgslLbm.ts:527-592, SolverGPU.ts:374-425
 *   streamlines, probes ....... src/render/tracers.ts:109-125, 152-200
 *   learned closure ........... no counterpart in the reference: the network of include/wt.h
 *                               (wt_closure), its features, loss gradient and the collision with
 *                               tau = tau0' + 3 nu_t in place of the Smagorinsky closure
 *                               (wgslLbm.ts:206-214)
 *
 * Arithmetic follows the WGSL expression order, evaluated left to right in IEEE single precision
 * without contraction (build with -ffp-contract=off). Float literals of the generated WGSL
 * (`fl()`, lattice.ts:70-73) equal the f32 rounding of the exact rationals for every constant
 * used here, so they are written as (float) casts.
 */
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../include/wt.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

/* ------------------------------------------------------------------------------------------ */
/* lattice tables (lattice.ts:20-60)                                                            */
/* ------------------------------------------------------------------------------------------ */
struct Lat {
  int q, dim;
  int c[19][3];
  double w[19];
  int opp[19], my[19], mz[19], myz[19];
};

static Lat build_lat(int q, int dim, const int (*c)[3], const double* w) {
  Lat L;
  L.q = q;
  L.dim = dim;
  for (int i = 0; i < q; i++) {
    for (int a = 0; a < 3; a++) L.c[i][a] = c[i][a];
    L.w[i] = w[i];
  }
  auto find = [&](int x, int y, int z) {
    for (int k = 0; k < q; k++)
      if (L.c[k][0] == x && L.c[k][1] == y && L.c[k][2] == z) return k;
    std::abort();
  };
  for (int i = 0; i < q; i++) {
    const int* v = L.c[i];
    L.opp[i] = find(-v[0], -v[1], -v[2]);
    L.my[i] = find(v[0], -v[1], v[2]);
    L.mz[i] = find(v[0], v[1], -v[2]);
    L.myz[i] = find(v[0], -v[1], -v[2]);
  }
  return L;
}

static const int C9[9][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {-1, 0, 0}, {0, -1, 0},
                             {1, 1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, -1, 0}};
static const double W9[9] = {4.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9,
                             1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};
static const int C19[19][3] = {{0, 0, 0},   {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0},
                               {0, 0, 1},   {0, 0, -1}, {1, 1, 0},  {-1, -1, 0}, {1, 0, 1},
                               {-1, 0, -1}, {0, 1, 1},  {0, -1, -1}, {1, -1, 0}, {-1, 1, 0},
                               {1, 0, -1},  {-1, 0, 1}, {0, 1, -1}, {0, -1, 1}};
static double W19[19];

static const Lat& lattice(int dim) {
  static Lat L9 = build_lat(9, 2, C9, W9);
  static Lat L19 = [] {
    W19[0] = 1.0 / 3;
    for (int i = 1; i < 7; i++) W19[i] = 1.0 / 18;
    for (int i = 7; i < 19; i++) W19[i] = 1.0 / 36;
    return build_lat(19, 3, C19, W19);
  }();
  return dim == 3 ? L19 : L9;
}

/* ------------------------------------------------------------------------------------------ */
/* population storage                                                                           */
/* ------------------------------------------------------------------------------------------ */
template <int PREC> struct RT { typedef float T; };
template <> struct RT<WT_PREC_F64> { typedef double T; };

template <int PREC> struct Pops {
  typedef typename RT<PREC>::T R;
  const void* in;
  void* out;
  size_t N;
  const Lat* L;
  R ld(int k, size_t c) const {
    if (PREC == WT_PREC_F32) return (R)((const float*)in)[(size_t)k * N + c];
    if (PREC == WT_PREC_F64) return (R)((const double*)in)[(size_t)k * N + c];
    /* packed FP16: unpack + WREST[k] (wgslLbm.ts:68-73) */
    _Float16 h = ((const _Float16*)in)[(size_t)k * N + c];
    return (R)((float)h + (float)L->w[k]);
  }
  void st(int k, size_t c, R v) const {
    if (PREC == WT_PREC_F32) ((float*)out)[(size_t)k * N + c] = (float)v;
    else if (PREC == WT_PREC_F64) ((double*)out)[(size_t)k * N + c] = (double)v;
    else ((_Float16*)out)[(size_t)k * N + c] = (_Float16)((float)v - (float)L->w[k]);
  }
};

template <class R> static R wconst(double w) { return (R)w; }

/* ------------------------------------------------------------------------------------------ */
/* shared context                                                                               */
/* ------------------------------------------------------------------------------------------ */
struct Ctx {
  wt_kparams P;
  const Lat* L;
  int NX, NY, NZ;
  size_t N;
  bool is3D;
  const uint32_t* flags;
  const uint32_t* sdf;
  uint32_t nwheels;
  float wh[32][4]; /* w[2k] = (centre, 1/R), w[2k+1] = (axis, half-width) */
  const wt_closure* closure; /* learned closure (f32 / f16 storage), nullptr = Smagorinsky */
  size_t cellId(int x, int y, int z) const { return (size_t)x + (size_t)NX * ((size_t)y + (size_t)NY * (size_t)z); }
};

/* sdfAt / linkQ (wgslLbm.ts:31-44) */
template <class R> static R sdfAt(const Ctx& X, size_t id) {
  uint32_t s = X.sdf[id];
  if (s == 0u) return (R)-1.0;
  uint32_t b = ~s;
  float d;
  std::memcpy(&d, &b, 4);
  return (R)d;
}
template <class R> static R linkQ(const Ctx& X, size_t fluid, size_t solid) {
  if (X.P.interp == 0u) return (R)0.5;
  R a = sdfAt<R>(X, fluid);
  R b = sdfAt<R>(X, solid);
  if (a < (R)0 || b < (R)0 || a + b < (R)1e-6f) return (R)0.5;
  R q = a / (a + b);
  if (q < (R)0.01f) q = (R)0.01f;
  if (q > (R)0.99f) q = (R)0.99f;
  return q;
}

/* wheelVel (wgslLbm.ts:21-28) */
template <class R> static void wheelVel(const Ctx& X, uint32_t k, R px, R py, R pz, R out[3]) {
  const float* a = X.wh[2 * k];
  const float* b = X.wh[2 * k + 1];
  R dx = px - (R)a[0], dy = py - (R)a[1], dz = pz - (R)a[2];
  R s = (R)X.P.u_ground * (R)a[3];
  R cx = (R)b[1] * dz - (R)b[2] * dy;
  R cy = (R)b[2] * dx - (R)b[0] * dz;
  R cz = (R)b[0] * dy - (R)b[1] * dx;
  out[0] = s * cx;
  out[1] = s * cy;
  out[2] = s * cz;
}

/* Left-to-right signed sum of the populations with coefficient k(i) in {-1, 0, 1}, as the
 * generated `sumExpr` (wgslLbm.ts:245-253) spells it. */
template <class R, class Coef> static R signed_sum(const Lat& L, const R* f, Coef coef) {
  bool first = true;
  R acc = 0;
  for (int i = 0; i < L.q; i++) {
    int k = coef(i);
    if (k == 0) continue;
    if (first) {
      acc = k > 0 ? f[i] : -f[i];
      first = false;
    } else {
      acc = k > 0 ? acc + f[i] : acc - f[i];
    }
  }
  return acc;
}

/* ------------------------------------------------------------------------------------------ */
/* fused pull-stream + collide for one cell (wgslLbm.ts:134-293)                                */
/* ------------------------------------------------------------------------------------------ */
/* ---- learned closure: features and network (the arithmetic of include/wt.h's wt_closure) ---- */
static float cl_bf16r(float v) {
  uint32_t u;
  std::memcpy(&u, &v, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  u &= 0xFFFF0000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

static void cl_features(float pxx, float pyy, float pzz, float pxy, float pxz, float pyz, float rho, float ux,
                        float uy, float uz, float tau0, float wall_d, float* x) {
  float pn = std::fma(pxx, pxx, std::fma(pyy, pyy, pzz * pzz));
  pn = std::fma(2.0f, std::fma(pxy, pxy, std::fma(pxz, pxz, pyz * pyz)), pn);
  const float piN = std::sqrt(pn);
  const float k = (float)(18.0 * 1.4142135623730951) * (WT_CLOSURE_FEATURE_CS * WT_CLOSURE_FEATURE_CS);
  const float ts = 0.5f * (tau0 + std::sqrt(std::fma(tau0, tau0, (k * piN) / rho)));
  x[0] = pxx;
  x[1] = pyy;
  x[2] = pzz;
  x[3] = pxy;
  x[4] = pxz;
  x[5] = pyz;
  x[6] = (2.1213203435596424f * piN) / (rho * ts);
  x[7] = wall_d;
  x[8] = rho;
  x[9] = std::sqrt(std::fma(ux, ux, std::fma(uy, uy, uz * uz)));
}

static float cl_wall_dist(uint32_t s) {
  if (s == 0u) return WT_CLOSURE_WALL_CAP;
  const uint32_t b = ~s;
  float d;
  std::memcpy(&d, &b, 4);
  return d < WT_CLOSURE_WALL_CAP ? d : WT_CLOSURE_WALL_CAP;
}

/* gelu(x) = (x + x tanh(u)) / 2, u = x (C0 + C1 x^2), C0 = sqrt(2/pi), C1 = 0.044715 C0; x + x tanh(u)
 * is one fma, halved exactly */
static const float GELU_C0 = 0.7978845608028654f, GELU_C1 = 0.035677408136300125f,
                   GELU_C1x3 = 0.10703222440890037f;

static float cl_gelu(float x) {
  const float t = std::tanh(x * std::fma(GELU_C1, x * x, GELU_C0));
  return 0.5f * std::fma(x, t, x);
}

static float cl_gelu_d(float x, float& d) {
  const float x2 = x * x;
  const float t = std::tanh(x * std::fma(GELU_C1, x2, GELU_C0));
  const float q = std::fma(0.5f, t, 0.5f);
  const float du = std::fma(GELU_C1x3, x2, GELU_C0);
  d = std::fma((0.5f * x) * std::fma(-t, t, 1.0f), du, q);
  return 0.5f * std::fma(x, t, x);
}

static float cl_softplus(float z) { return z > 20.0f ? z : std::log1p(std::exp(z)); }

/* network input k: bf16(fma(x, scale, nshift)), nshift = -(shift * scale) */
static float cl_input(const wt_closure& C, const float* x, int k) {
  return cl_bf16r(std::fma(x[k], C.scale[k], -(C.shift[k] * C.scale[k])));
}

/* forward pass of one sample; the optional outputs keep the intermediate values for the gradient */
static float cl_forward(const wt_closure& C, const float* xin, float* xn = nullptr, float* z1 = nullptr,
                        float* h1 = nullptr, float* z2 = nullptr, float* h2 = nullptr, float* z3o = nullptr) {
  float x[WT_CLOSURE_IN], a1[WT_CLOSURE_HID], b1[WT_CLOSURE_HID], a2[WT_CLOSURE_HID], b2[WT_CLOSURE_HID];
  for (int k = 0; k < WT_CLOSURE_IN; k++) x[k] = cl_input(C, xin, k);
  for (int j = 0; j < WT_CLOSURE_HID; j++) {
    float a = 0.0f;
    for (int k = 0; k < WT_CLOSURE_IN; k++) a = std::fma(x[k], cl_bf16r(C.w1[k][j]), a);
    a1[j] = a + C.b1[j];
    b1[j] = cl_bf16r(cl_gelu(a1[j]));
  }
  float ze = 0.0f, zo = 0.0f; /* even and odd hidden units summed separately */
  for (int j = 0; j < WT_CLOSURE_HID; j++) {
    float a = 0.0f;
    for (int i = 0; i < WT_CLOSURE_HID; i++) a = std::fma(b1[i], cl_bf16r(C.w2[i][j]), a);
    a2[j] = a + C.b2[j];
    b2[j] = cl_gelu(a2[j]); /* h2 stays f32 */
    if (j & 1) zo = std::fma(b2[j], cl_bf16r(C.w3[j]), zo);
    else ze = std::fma(b2[j], cl_bf16r(C.w3[j]), ze);
  }
  const float z3 = (ze + zo) + C.b3;
  if (xn) std::memcpy(xn, x, sizeof x);
  if (z1) std::memcpy(z1, a1, sizeof a1);
  if (h1) std::memcpy(h1, b1, sizeof b1);
  if (z2) std::memcpy(z2, a2, sizeof a2);
  if (h2) std::memcpy(h2, b2, sizeof b2);
  if (z3o) *z3o = z3;
  return C.nu_scale * cl_softplus(z3);
}

template <int PREC> static void sc_cell(const Ctx& X, const Pops<PREC>& F, size_t idx) {
  typedef typename RT<PREC>::T R;
  const Lat& L = *X.L;
  const wt_kparams& P = X.P;
  const int NX = X.NX, NY = X.NY, NZ = X.NZ;
  const int ix = (int)(idx % P.nx);
  const int iy = (int)((idx / P.nx) % P.ny);
  const int iz = (int)(idx / ((size_t)P.nx * P.ny));
  const R U = (R)P.uin;
  bool wall = false, gwall = false;
  R mvSum = 0, mvW = 0;
  uint32_t wm = 0;
  R belt = P.ground == 2u ? (R)1 : (R)0;
  if (belt > 0 && iy == 0) {
    const int r = (int)P.contact_h;
    for (int dz = -r; dz <= r; dz++)
      for (int dx = -r; dx <= r; dx++)
        for (int dy = 0; dy <= 1; dy++) {
          int qx = ix + dx, qz = iz + dz;
          if (qx >= 0 && qx < NX && qz >= 0 && qz < NZ) {
            uint32_t fq = X.flags[X.cellId(qx, dy, qz)];
            if (fq != 0u && (fq >> 8u) == 0u) belt = 0;
          }
        }
  }
  if (X.flags[idx] != 0u) {
    for (int i = 0; i < L.q; i++) F.st(i, idx, wconst<R>(L.w[i]));
    return;
  }
  R f[19];
  f[0] = F.ld(0, idx);
  for (int i = 1; i < L.q; i++) {
    const int cx = L.c[i][0], cy = L.c[i][1], cz = L.c[i][2];
    const R w = wconst<R>(L.w[i]);
    int sx = ix - cx, sy = iy - cy, sz = X.is3D ? iz - cz : 0;
    if (cx < 0) sx = sx < NX - 1 ? sx : NX - 1;
    const bool yOut = cy > 0 ? sy < 0 : (cy < 0 ? sy >= NY : false);
    const bool zOut = X.is3D ? (cz > 0 ? sz < 0 : (cz < 0 ? sz >= NZ : false)) : false;
    if (cx > 0 && sx < 0) {
      /* inlet equilibrium (cu = 1.0 * U) */
      R cu = (R)1 * U;
      f[i] = w * (R)P.rho_in * ((R)1 + (R)3 * cu + (R)4.5 * cu * cu - (R)1.5 * U * U);
    } else if (cy > 0 && yOut && P.ground != 0u) {
      wall = true;
      gwall = true;
      R v = F.ld(L.opp[i], idx);
      if (cx != 0) v = v + belt * (wconst<R>(6 * L.w[i] * cx) * (R)P.u_ground);
      f[i] = v;
    } else {
      const int sxc = sx < 0 ? 0 : (sx > NX - 1 ? NX - 1 : sx);
      if (X.is3D && yOut && zOut) {
        f[i] = F.ld(L.myz[i], X.cellId(sxc, iy, iz));
      } else if (yOut) {
        int zz = X.is3D ? (sz < 0 ? 0 : (sz > NZ - 1 ? NZ - 1 : sz)) : 0;
        f[i] = F.ld(L.my[i], X.cellId(sxc, iy, zz));
      } else if (X.is3D && zOut) {
        if (P.side_mode == 1u) f[i] = F.ld(i, X.cellId(sxc, sy, (sz + NZ) % NZ));
        else f[i] = F.ld(L.mz[i], X.cellId(sxc, sy, iz));
      } else {
        const size_t sc = X.cellId(sxc, sy, sz);
        const uint32_t fs = X.flags[sc];
        if (fs != 0u) {
          wall = true;
          const R fb = F.ld(L.opp[i], idx);
          R q = linkQ<R>(X, idx, sc);
          R v = fb;
          if (q < (R)0.5) {
            const int ax = ix + cx, ay = iy + cy, az = X.is3D ? iz + cz : 0;
            if (ax >= 0 && ay >= 0 && az >= 0 && ax < NX && ay < NY && az < NZ && X.flags[X.cellId(ax, ay, az)] == 0u) {
              v = (R)2 * q * fb + ((R)1 - (R)2 * q) * F.ld(L.opp[i], X.cellId(ax, ay, az));
            } else {
              q = (R)0.5;
            }
          } else if (q > (R)0.5) {
            v = ((R)0.5 / q) * fb + ((R)1 - (R)0.5 / q) * F.ld(i, idx);
          }
          f[i] = v;
          if ((fs >> 8u) != 0u) {
            R uw[3];
            wheelVel<R>(X, (fs >> 8u) - 1u, (R)0.5 * (R)(ix + sxc) + (R)0.5, (R)0.5 * (R)(iy + sy) + (R)0.5,
                        (R)0.5 * (R)(iz + sz) + (R)0.5, uw);
            R dot = (R)cx * uw[0] + (R)cy * uw[1] + (R)cz * uw[2];
            R mv = wconst<R>(6 * L.w[i]) * dot * (q > (R)0.5 ? (R)0.5 / q : (R)1);
            f[i] += mv;
            mvSum += mv;
            mvW += w;
            wm |= 1u << i;
          }
        } else {
          f[i] = F.ld(i, sc);
        }
      }
    }
  }
  if (mvW > 0) {
    R corr = mvSum / mvW;
    for (int i = 1; i < L.q; i++)
      if (wm & (1u << i)) f[i] -= wconst<R>(L.w[i]) * corr;
  }

  /* collision (wgslLbm.ts:177-240) */
  const int dim = L.dim;
  R rho = signed_sum<R>(L, f, [](int) { return 1; });
  R irho = (R)1 / rho;
  R u[3] = {0, 0, 0};
  for (int a = 0; a < dim; a++) u[a] = signed_sum<R>(L, f, [&](int i) { return L.c[i][a]; }) * irho;
  R usq = 0;
  for (int a = 0; a < dim; a++) usq = a == 0 ? u[0] * u[0] : usq + u[a] * u[a];
  int pa[6], pb[6], np = 0;
  for (int a = 0; a < dim; a++)
    for (int b = a; b < dim; b++) {
      pa[np] = a;
      pb[np] = b;
      np++;
    }
  R pi[6];
  for (int k = 0; k < np; k++) {
    int a = pa[k], b = pb[k];
    R s = signed_sum<R>(L, f, [&](int i) { return L.c[i][a] * L.c[i][b]; });
    R eq = a == b ? rho * (u[a] * u[b] + (R)(1.0 / 3.0)) : rho * u[a] * u[b];
    pi[k] = s - eq;
  }
  R pn = 0;
  for (int k = 0; k < np; k++) {
    R t = pa[k] == pb[k] ? pi[k] * pi[k] : (R)2 * pi[k] * pi[k];
    pn = k == 0 ? t : pn + t;
  }
  R piN = std::sqrt(pn);
  R fx = (R)ix;
  R den = (R)NX - (R)P.sponge_start;
  R sp = (fx - (R)P.sponge_start) / (den > (R)1 ? den : (R)1);
  sp = sp < 0 ? 0 : (sp > 1 ? 1 : sp);
  R t0 = (R)P.tau0 + (R)3 * (R)P.sponge_nu * sp * sp;
  if (gwall) t0 = t0 > (R)P.tau_wall ? t0 : (R)P.tau_wall;
  R tau = (R)0.5 * (t0 + std::sqrt(t0 * t0 + (R)(18.0 * std::sqrt(2.0)) * (R)P.csmag2 * piN * irho));
  if (X.closure != nullptr && dim == 3 && PREC != WT_PREC_F64) {
    /* pi[] is ordered xx, xy, xz, yy, yz, zz */
    float x[WT_CLOSURE_IN];
    cl_features((float)pi[0], (float)pi[3], (float)pi[5], (float)pi[1], (float)pi[2], (float)pi[4], (float)rho,
                (float)u[0], (float)u[1], (float)u[2], P.tau0, cl_wall_dist(X.sdf[idx]), x);
    tau = t0 + (R)3 * (R)cl_forward(*X.closure, x);
  }
  R k1 = ((R)1 - (R)1 / tau) * (R)4.5;
  bool useBGK = wall || P.collision == 1u;
  R sIn_den = (R)P.sponge_in > (R)1 ? (R)P.sponge_in : (R)1;
  R si = (R)1 - fx / sIn_den;
  si = si < 0 ? 0 : (si > 1 ? 1 : si);
  R sIn = (R)P.sponge_in > (R)0 ? (R)0.08 * si * si : (R)0;
  R trace = 0;
  bool tf = true;
  for (int k = 0; k < np; k++)
    if (pa[k] == pb[k]) {
      trace = tf ? pi[k] : trace + pi[k];
      tf = false;
    }
  R trP = trace * (R)(1.0 / 3.0);
  for (int i = 0; i < L.q; i++) {
    const int* cv = L.c[i];
    const R w = wconst<R>(L.w[i]);
    R cu = 0;
    bool first = true;
    for (int a = 0; a < dim; a++) {
      if (cv[a] == 0) continue;
      if (first) {
        cu = cv[a] == 1 ? u[a] : -u[a];
        first = false;
      } else {
        cu = cv[a] == 1 ? cu + u[a] : cu - u[a];
      }
    }
    R feq = w * rho * ((R)1 + (R)3 * cu + (R)4.5 * cu * cu - (R)1.5 * usq);
    R qp = 0;
    bool qf = true;
    for (int k = 0; k < np; k++) {
      int coef = cv[pa[k]] * cv[pb[k]] * (pa[k] == pb[k] ? 1 : 2);
      if (coef == 0) continue;
      R t = (R)coef * pi[k];
      qp = qf ? t : qp + t;
      qf = false;
    }
    R qpi = qp - trP; /* "0.0 - trP" when no component is set */
    R fr = w * k1 * qpi;
    R fo = feq + (useBGK ? ((R)1 - (R)1 / tau) * (f[i] - feq) : fr);
    if (sIn > 0) {
      const int cx2 = cv[0];
      R eq = w * ((R)1 + (R)(3 * cx2) * U + (R)(4.5 * cx2 * cx2) * U * U - (R)1.5 * U * U);
      fo = fo * ((R)1 - sIn) + eq * sIn;
    }
    F.st(i, idx, fo);
  }
}

/* init (wgslLbm.ts:296-341), plus the rest-state-with-noise extension */
static uint32_t pcg(uint32_t v) {
  uint32_t s = v * 747796405u + 2891336453u;
  uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  return (w >> 22u) ^ w;
}

/* Seeded noise in [-amp, amp] for component a of cell `cell` (rest-state initialisation). */
static float noise_component(uint32_t seed, uint64_t cell, int a, float amp) {
  uint32_t h = pcg((uint32_t)(cell * 3u + (uint64_t)a) ^ pcg(seed ^ (uint32_t)(cell >> 32)));
  float r = (float)(h >> 8) * (1.0f / 16777216.0f); /* [0, 1) */
  return amp * (2.0f * r - 1.0f);
}

template <int PREC> static void init_cell(const Ctx& X, const Pops<PREC>& F, size_t idx, int mode, uint32_t seed, float amp) {
  typedef typename RT<PREC>::T R;
  const Lat& L = *X.L;
  const bool solid = X.flags[idx] != 0u;
  if (mode == WT_INIT_FREESTREAM) {
    if (PREC == WT_PREC_F16) {
      /* packed init stores f - w directly (wgslLbm.ts:297-303) */
      float ua = solid ? 0.0f : X.P.uin;
      for (int i = 0; i < L.q; i++) {
        const int cx = L.c[i][0];
        float v = (float)L.w[i] * ((float)(3 * cx) * ua + (float)(4.5 * cx * cx) * ua * ua - 1.5f * ua * ua);
        ((_Float16*)F.out)[(size_t)i * F.N + idx] = (_Float16)v;
      }
      return;
    }
    R U = solid ? (R)0 : (R)X.P.uin;
    for (int i = 0; i < L.q; i++) {
      const int cx = L.c[i][0];
      R v = wconst<R>(L.w[i]) * ((R)1 + (R)(3 * cx) * U + (R)(4.5 * cx * cx) * U * U - (R)1.5 * U * U);
      F.st(i, idx, v);
    }
    return;
  }
  /* rest state with seeded velocity noise: f = feq(rho = 1, u = noise); solids u = 0 */
  float un[3] = {0, 0, 0};
  if (!solid)
    for (int a = 0; a < L.dim; a++) un[a] = noise_component(seed, idx, a, amp);
  for (int i = 0; i < L.q; i++) {
    if (PREC == WT_PREC_F16) {
      float cu = (float)L.c[i][0] * un[0] + (float)L.c[i][1] * un[1] + (float)L.c[i][2] * un[2];
      float usq = un[0] * un[0] + un[1] * un[1] + un[2] * un[2];
      float v = (float)L.w[i] * (3.0f * cu + 4.5f * cu * cu - 1.5f * usq);
      ((_Float16*)F.out)[(size_t)i * F.N + idx] = (_Float16)v;
    } else {
      R cu = (R)L.c[i][0] * (R)un[0] + (R)L.c[i][1] * (R)un[1] + (R)L.c[i][2] * (R)un[2];
      R usq = (R)un[0] * (R)un[0] + (R)un[1] * (R)un[1] + (R)un[2] * (R)un[2];
      R v = wconst<R>(L.w[i]) * ((R)1 + (R)3 * cu + (R)4.5 * cu * cu - (R)1.5 * usq);
      F.st(i, idx, v);
    }
  }
}

/* ------------------------------------------------------------------------------------------ */
/* macro: ρ, u, EMA, momentum exchange, partial reductions (wgslLbm.ts:353-489)                 */
/* ------------------------------------------------------------------------------------------ */
struct MacroAcc {
  double F[3];
  float maxuu;
  double rho_ref, n_ref, nan, solid;
  double mass, fluid; /* global mass-conservation check (extension): FP64 sum of fluid densities */
};

template <int PREC> static void macro_cell(const Ctx& X, const Pops<PREC>& Fp, size_t idx, float* vel4,
                                          float* meanA, float* meanB, MacroAcc& acc) {
  typedef typename RT<PREC>::T R;
  const Lat& L = *X.L;
  const wt_kparams& P = X.P;
  const int NX = X.NX, NY = X.NY, NZ = X.NZ;
  const int ix = (int)(idx % P.nx);
  const int iy = (int)((idx / P.nx) % P.ny);
  const int iz = (int)(idx / ((size_t)P.nx * P.ny));
  auto safe = [&](int x, int y, int z) -> int64_t {
    if (x < 0 || y < 0 || z < 0 || x >= NX || y >= NY || z >= NZ) return -1;
    return (int64_t)X.cellId(x, y, z);
  };
  float out[4] = {0, 0, 0, 1};
  float A[4] = {0, 0, 0, 0};
  double Fd[3] = {0, 0, 0};
  float B[4] = {0, 0, 0, 0};
  const float a = P.ema_alpha;
  if (X.flags[idx] == 0u) {
    R f[19];
    for (int i = 0; i < L.q; i++) f[i] = Fp.ld(i, idx);
    R rho = signed_sum<R>(L, f, [](int) { return 1; });
    R u[3] = {0, 0, 0};
    for (int d = 0; d < L.dim; d++) u[d] = signed_sum<R>(L, f, [&](int i) { return L.c[i][d]; }) / rho;
    R Fv[3] = {0, 0, 0};
    R mvSum = 0, mvW = 0, Cw[3] = {0, 0, 0};
    for (int i = 1; i < L.q; i++) {
      const int cx = L.c[i][0], cy = L.c[i][1], cz = L.c[i][2];
      int64_t s = safe(ix + cx, iy + cy, iz + cz);
      if (s < 0 || X.flags[s] == 0u) continue;
      R q = linkQ<R>(X, idx, (size_t)s);
      R fr = f[i];
      if (q < (R)0.5) {
        int64_t bk = safe(ix - cx, iy - cy, iz - cz);
        if (bk >= 0 && X.flags[bk] == 0u) fr = (R)2 * q * f[i] + ((R)1 - (R)2 * q) * Fp.ld(i, (size_t)bk);
        else q = (R)0.5;
      } else if (q > (R)0.5) {
        fr = ((R)0.5 / q) * f[i] + ((R)1 - (R)0.5 / q) * f[L.opp[i]];
      }
      uint32_t tg = X.flags[s] >> 8u;
      if (tg != 0u) {
        R uw[3];
        wheelVel<R>(X, tg - 1u, (R)ix + (R)(0.5 + cx / 2.0), (R)iy + (R)(0.5 + cy / 2.0), (R)iz + (R)(0.5 + cz / 2.0), uw);
        R dot = (R)cx * uw[0] + (R)cy * uw[1] + (R)cz * uw[2];
        R mv = -wconst<R>(6 * L.w[i]) * (q > (R)0.5 ? (R)0.5 / q : (R)1) * dot;
        fr += mv;
        mvSum += mv;
        mvW += wconst<R>(L.w[i]);
        Cw[0] += (R)cx * wconst<R>(L.w[i]);
        Cw[1] += (R)cy * wconst<R>(L.w[i]);
        Cw[2] += (R)cz * wconst<R>(L.w[i]);
      }
      R t = f[i] + fr - wconst<R>(2 * L.w[i]);
      Fv[0] += (R)cx * t;
      Fv[1] += (R)cy * t;
      Fv[2] += (R)cz * t;
    }
    if (mvW > 0) {
      R k = mvSum / mvW;
      for (int d = 0; d < 3; d++) Fv[d] -= Cw[d] * k;
    }
    R uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    bool bad = !(uu < (R)1.0e6) || !(rho > 0);
    for (int d = 0; d < 3; d++) {
      Fd[d] = (double)Fv[d];
      out[d] = (float)u[d];
    }
    out[3] = (float)rho;
    A[3] = bad ? 1.0e6f : (float)uu;
    if ((uint32_t)ix == P.ref_x) {
      B[0] = (float)rho;
      B[1] = 1;
    }
    B[2] = bad ? 1.0f : 0.0f;
    /* EMA (wgslLbm.ts:456-459): mix(m, out, a) = m * (1 - a) + out * a */
    for (int d = 0; d < 4; d++) meanA[4 * idx + d] = meanA[4 * idx + d] * (1.0f - a) + out[d] * a;
    meanB[idx] = meanB[idx] * (1.0f - a) + (float)uu * a;
    acc.rho_ref += (uint32_t)ix == P.ref_x ? (double)rho : 0.0;
    acc.mass += (double)rho;
    acc.fluid += 1.0;
  } else {
    /* density extrapolated into the solid from fluid face neighbours */
    static const int nb[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    const int nn = L.dim == 3 ? 6 : 4;
    R rs = 0, rn = 0;
    for (int k = 0; k < nn; k++) {
      int64_t s = safe(ix + nb[k][0], iy + nb[k][1], iz + nb[k][2]);
      if (s >= 0 && X.flags[s] == 0u) {
        R r = 0;
        for (int j = 0; j < L.q; j++) r += Fp.ld(j, (size_t)s);
        rs += r;
        rn += 1;
      }
    }
    if (rn > 0) out[3] = (float)(rs / rn);
    for (int d = 0; d < 4; d++) meanA[4 * idx + d] = meanA[4 * idx + d] * (1.0f - a) + out[d] * a;
    meanB[idx] = 0;
    B[3] = 1;
  }
  for (int d = 0; d < 4; d++) vel4[4 * idx + d] = (float)(_Float16)out[d];
  for (int d = 0; d < 3; d++) acc.F[d] += Fd[d];
  if (A[3] > acc.maxuu) acc.maxuu = A[3];
  acc.n_ref += B[1];
  acc.nan += B[2];
  acc.solid += B[3];
}

static int make_ctx(Ctx& X, const wt_dims* d, const wt_kparams* kp, const uint32_t* flags, const uint32_t* sdf,
                    const float* wheels8, int nwheels) {
  if (!d || !kp || d->nx < 1 || d->ny < 1 || d->nz < 1) return WT_E_INVALID;
  std::memset(&X, 0, sizeof X);
  X.P = *kp;
  X.is3D = d->nz > 1;
  X.L = &lattice(X.is3D ? 3 : 2);
  X.NX = d->nx;
  X.NY = d->ny;
  X.NZ = d->nz;
  X.N = (size_t)d->nx * d->ny * d->nz;
  X.flags = flags;
  X.sdf = sdf;
  X.nwheels = nwheels < 0 ? 0 : (nwheels > 16 ? 16 : nwheels);
  if (wheels8)
    for (uint32_t k = 0; k < X.nwheels; k++)
      for (int j = 0; j < 8; j++) X.wh[2 * k + j / 4][j % 4] = wheels8[8 * k + j];
  return WT_OK;
}

/* ------------------------------------------------------------------------------------------ */
/* voxelizer, f32 GPU semantics (wgslVoxel.ts)                                                  */
/* ------------------------------------------------------------------------------------------ */
struct V3 {
  float x, y, z;
};
static inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
static inline V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 mul(V3 a, float k) { return v3(a.x * k, a.y * k, a.z * k); }
static inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float len(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
static inline V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline float comp(V3 p, int a) { return a == 0 ? p.x : (a == 1 ? p.y : p.z); }

struct Vox {
  float M[16];
  int nx, ny, nz;
  size_t n;
  const float* pos;
  const uint32_t* idx;
  int dimOf(int a) const { return a == 0 ? nx : (a == 1 ? ny : nz); }
  size_t cellOf(uint32_t x, uint32_t y, uint32_t z) const { return (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z); }
  V3 vtx(size_t i) const {
    uint32_t k = idx[i];
    float x = pos[3 * (size_t)k], y = pos[3 * (size_t)k + 1], z = pos[3 * (size_t)k + 2];
    return v3(M[0] * x + M[4] * y + M[8] * z + M[12], M[1] * x + M[5] * y + M[9] * z + M[13],
              M[2] * x + M[6] * y + M[10] * z + M[14]);
  }
};

static inline int f2i(float v) {
  /* WGSL i32(f32) saturates */
  if (!(v == v)) return 0;
  if (v >= 2147483520.0f) return 2147483647;
  if (v <= -2147483648.0f) return (-2147483647 - 1);
  return (int)v;
}

static void vox_crossings(const Vox& V, size_t t, int32_t* hits) {
  V3 p0 = V.vtx(3 * t), p1 = V.vtx(3 * t + 1), p2 = V.vtx(3 * t + 2);
  for (int a = 0; a < 3; a++) {
    int ua = (a + 1) % 3, va = (a + 2) % 3;
    float Ax = comp(p0, ua), Ay = comp(p0, va), Bx = comp(p1, ua), By = comp(p1, va), Cx = comp(p2, ua), Cy = comp(p2, va);
    float area = (Bx - Ax) * (Cy - Ay) - (By - Ay) * (Cx - Ax);
    if (std::fabs(area) < 1e-12f) continue;
    int sgn = area > 0.0f ? -1 : 1;
    int nu = V.dimOf(ua), nv = V.dimOf(va), na = V.dimOf(a);
    float lox = std::fmin(std::fmin(Ax, Bx), Cx), loy = std::fmin(std::fmin(Ay, By), Cy);
    float hix = std::fmax(std::fmax(Ax, Bx), Cx), hiy = std::fmax(std::fmax(Ay, By), Cy);
    int u0 = std::max(f2i(std::ceil(lox - 0.5f)), 0);
    int u1 = std::min(f2i(std::floor(hix - 0.5f)), nu - 1);
    int v0 = std::max(f2i(std::ceil(loy - 0.5f)), 0);
    int v1 = std::min(f2i(std::floor(hiy - 0.5f)), nv - 1);
    float ha = comp(p0, a), hb = comp(p1, a), hc = comp(p2, a);
    float inv = 1.0f / area;
    for (int iu = u0; iu <= u1; iu++)
      for (int iv = v0; iv <= v1; iv++) {
        float Px = (float)iu + 0.5f + 1.37e-4f, Py = (float)iv + 0.5f + 2.71e-4f;
        float w0 = ((Bx - Px) * (Cy - Py) - (By - Py) * (Cx - Px)) * inv;
        float w1 = ((Cx - Px) * (Ay - Py) - (Cy - Py) * (Ax - Px)) * inv;
        float w2 = 1.0f - w0 - w1;
        if (w0 < 0.0f || w1 < 0.0f || w2 < 0.0f) continue;
        float h = w0 * ha + w1 * hb + w2 * hc;
        int k = f2i(std::floor(h - 0.5f)) + 1;
        if (k >= na) continue;
        k = std::max(k, 0);
        size_t c = a == 0 ? V.cellOf(k, iu, iv) : (a == 1 ? V.cellOf(iv, k, iu) : V.cellOf(iu, iv, k));
        __atomic_fetch_add(&hits[(size_t)a * V.n + c], sgn, __ATOMIC_RELAXED);
      }
  }
}

static void vox_surface(const Vox& V, size_t t, uint32_t* vote) {
  V3 p0 = V.vtx(3 * t);
  V3 e1 = sub(V.vtx(3 * t + 1), p0);
  V3 e2 = sub(V.vtx(3 * t + 2), p0);
  float m = std::fmax(std::fmax(len(e1), len(e2)), len(sub(e2, e1)));
  float sc = std::ceil(m / 0.4f);
  sc = std::fmin(std::fmax(sc, 1.0f), 384.0f);
  uint32_t steps = (uint32_t)sc;
  float fs = (float)steps;
  V3 cr = cross(e1, e2);
  float cl = len(cr);
  if (cl < 1e-12f) return;
  V3 nrm = v3(cr.x / cl, cr.y / cl, cr.z / cl);
  float tol = 0.5f * std::fmax(std::fmax(std::fabs(nrm.x), std::fabs(nrm.y)), std::fabs(nrm.z));
  bool is2D = V.nz == 1;
  for (uint32_t i = 0; i <= steps; i++)
    for (uint32_t j = 0; j <= steps - i; j++) {
      V3 p = add(add(p0, mul(e1, (float)i / fs)), mul(e2, (float)j / fs));
      if (p.x < 0.0f || p.y < 0.0f || p.z < 0.0f || p.x >= (float)V.nx || p.y >= (float)V.ny || p.z >= (float)V.nz) continue;
      V3 c = v3(std::floor(p.x), std::floor(p.y), std::floor(p.z));
      V3 ctr = v3(c.x + 0.5f, c.y + 0.5f, c.z + 0.5f);
      float tt = tol;
      if (is2D) {
        float n2 = std::sqrt(nrm.x * nrm.x + nrm.y * nrm.y);
        if (n2 < 1e-4f) continue;
        ctr.z = p.z;
        tt = 0.5f * std::fmax(std::fabs(nrm.x), std::fabs(nrm.y)) / n2 * n2;
        if (std::fabs(p.z - 0.5f) > 0.5f) continue;
      }
      if (std::fabs(dot(sub(ctr, p0), nrm)) > tt) continue;
      __atomic_fetch_or(&vote[V.cellOf((uint32_t)c.x, (uint32_t)c.y, (uint32_t)c.z)], 8u, __ATOMIC_RELAXED);
    }
}

/* closest point on triangle (Ericson, Real-Time Collision Detection 5.1.5; wgslVoxel.ts:210-226) */
template <class T, class VT> static VT closest_pt(VT p, VT a, VT b, VT c, VT (*mk)(T, T, T)) {
  auto sb = [&](VT u, VT v) { return mk(u.x - v.x, u.y - v.y, u.z - v.z); };
  auto dt = [&](VT u, VT v) { return u.x * v.x + u.y * v.y + u.z * v.z; };
  auto ad = [&](VT u, VT v, T k) { return mk(u.x + v.x * k, u.y + v.y * k, u.z + v.z * k); };
  VT ab = sb(b, a), ac = sb(c, a), ap = sb(p, a);
  T d1 = dt(ab, ap), d2 = dt(ac, ap);
  if (d1 <= 0 && d2 <= 0) return a;
  VT bp = sb(p, b);
  T d3 = dt(ab, bp), d4 = dt(ac, bp);
  if (d3 >= 0 && d4 <= d3) return b;
  T vc = d1 * d4 - d3 * d2;
  if (vc <= 0 && d1 >= 0 && d3 <= 0) return ad(a, ab, d1 / (d1 - d3));
  VT cp = sb(p, c);
  T d5 = dt(ab, cp), d6 = dt(ac, cp);
  if (d6 >= 0 && d5 <= d6) return c;
  T vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) return ad(a, ac, d2 / (d2 - d6));
  T va = d3 * d6 - d5 * d4;
  if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) return ad(b, sb(c, b), (d4 - d3) / ((d4 - d3) + (d5 - d6)));
  T den = (T)1 / (va + vb + vc);
  return ad(ad(a, ab, vb * den), ac, vc * den);
}

static inline void atomic_max_u32(uint32_t* p, uint32_t v) {
  uint32_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
  while (cur < v && !__atomic_compare_exchange_n(p, &cur, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
  }
}

static void vox_sdf(const Vox& V, size_t t, uint32_t* sdf) {
  V3 a = V.vtx(3 * t), b = V.vtx(3 * t + 1), c = V.vtx(3 * t + 2);
  V3 e1 = sub(b, a), e2 = sub(c, a);
  if (len(cross(e1, e2)) < 1e-12f) return;
  float m = std::fmax(std::fmax(len(e1), len(e2)), len(sub(e2, e1)));
  float sc = std::ceil(m / 0.7f);
  sc = std::fmin(std::fmax(sc, 1.0f), 256.0f);
  uint32_t steps = (uint32_t)sc;
  float fs = (float)steps;
  bool is2D = V.nz == 1;
  const int R = 2;
  for (uint32_t i = 0; i <= steps; i++)
    for (uint32_t j = 0; j <= steps - i; j++) {
      V3 p = add(add(a, mul(e1, (float)i / fs)), mul(e2, (float)j / fs));
      if (is2D && std::fabs(p.z - 0.5f) > 2.5f) continue;
      int bx = f2i(std::floor(p.x)), by = f2i(std::floor(p.y)), bz = f2i(std::floor(p.z));
      for (int dz = -R; dz <= R; dz++) {
        if (is2D && dz != 0) continue;
        for (int dy = -R; dy <= R; dy++)
          for (int dx = -R; dx <= R; dx++) {
            int qx = bx + dx, qy = by + dy, qz = bz + dz;
            if (is2D) qz = 0;
            if (qx < 0 || qy < 0 || qz < 0 || qx >= V.nx || qy >= V.ny || qz >= V.nz) continue;
            V3 ctr = v3((float)qx + 0.5f, (float)qy + 0.5f, (float)qz + 0.5f);
            V3 cp = closest_pt<float, V3>(ctr, a, b, c, v3);
            float d = len(sub(ctr, cp));
            if (d > 2.5f) continue;
            uint32_t bits;
            std::memcpy(&bits, &d, 4);
            atomic_max_u32(&sdf[V.cellOf(qx, qy, qz)], ~bits);
          }
      }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* voxelizer, f64 CPU port (voxelizeCPU.ts:32-199)                                              */
/* ------------------------------------------------------------------------------------------ */
struct D3 {
  double x, y, z;
};
static inline D3 d3(double x, double y, double z) { return D3{x, y, z}; }

/* ------------------------------------------------------------------------------------------ */
/* tracers (tracers.ts:3-106)                                                                   */
/* ------------------------------------------------------------------------------------------ */
struct Tr {
  wt_tracer_params P;
  float dims[4];
  const uint16_t* vel; /* half4 per cell */
  const uint32_t* flags;
  uint32_t rng;
  float rnd() {
    rng = pcg(rng);
    return (float)rng / 4294967295.0f;
  }
  static float h2f(uint16_t h) {
    _Float16 v;
    std::memcpy(&v, &h, 2);
    return (float)v;
  }
  bool solidAt(V3 p) const {
    int nx = (int)dims[0], ny = (int)dims[1], nz = (int)dims[2];
    int cx = f2i(std::floor(p.x)), cy = f2i(std::floor(p.y)), cz = f2i(std::floor(p.z));
    if (dims[3] > 0.5f) cz = 0;
    if (cx < 0 || cy < 0 || cz < 0 || cx >= nx || cy >= ny || cz >= nz) return false;
    return flags[(size_t)cx + (size_t)nx * ((size_t)cy + (size_t)ny * cz)] != 0u;
  }
  /* textureSampleLevel with a linear clamp-to-edge sampler on rgba16float (texel centres) */
  V3 sVel(V3 p) const {
    int n[3] = {(int)dims[0], (int)dims[1], (int)dims[2]};
    float t[3] = {p.x / dims[0], p.y / dims[1], p.z / dims[2]};
    if (dims[3] > 0.5f) t[2] = 0.5f;
    int i0[3], i1[3];
    float fr[3];
    for (int a = 0; a < 3; a++) {
      float u = t[a] * (float)n[a] - 0.5f;
      float fl = std::floor(u);
      fr[a] = u - fl;
      int k = f2i(fl);
      i0[a] = k < 0 ? 0 : (k > n[a] - 1 ? n[a] - 1 : k);
      i1[a] = k + 1 < 0 ? 0 : (k + 1 > n[a] - 1 ? n[a] - 1 : k + 1);
    }
    float out[3];
    for (int ch = 0; ch < 3; ch++) {
      auto at = [&](int x, int y, int z) { return h2f(vel[4 * ((size_t)x + (size_t)n[0] * ((size_t)y + (size_t)n[1] * z)) + ch]); };
      float c00 = at(i0[0], i0[1], i0[2]) * (1.0f - fr[0]) + at(i1[0], i0[1], i0[2]) * fr[0];
      float c10 = at(i0[0], i1[1], i0[2]) * (1.0f - fr[0]) + at(i1[0], i1[1], i0[2]) * fr[0];
      float c01 = at(i0[0], i0[1], i1[2]) * (1.0f - fr[0]) + at(i1[0], i0[1], i1[2]) * fr[0];
      float c11 = at(i0[0], i1[1], i1[2]) * (1.0f - fr[0]) + at(i1[0], i1[1], i1[2]) * fr[0];
      float c0 = c00 * (1.0f - fr[1]) + c10 * fr[1];
      float c1 = c01 * (1.0f - fr[1]) + c11 * fr[1];
      out[ch] = c0 * (1.0f - fr[2]) + c1 * fr[2];
    }
    return v3(out[0], out[1], out[2]);
  }
  /* the same sampling of all four channels of any half4 field */
  void sF4(const uint16_t* f, V3 p, float out[4]) const {
    int n[3] = {(int)dims[0], (int)dims[1], (int)dims[2]};
    float t[3] = {p.x / dims[0], p.y / dims[1], p.z / dims[2]};
    if (dims[3] > 0.5f) t[2] = 0.5f;
    int i0[3], i1[3];
    float fr[3];
    for (int a = 0; a < 3; a++) {
      float u = t[a] * (float)n[a] - 0.5f;
      float fl = std::floor(u);
      fr[a] = u - fl;
      int k = f2i(fl);
      i0[a] = k < 0 ? 0 : (k > n[a] - 1 ? n[a] - 1 : k);
      i1[a] = k + 1 < 0 ? 0 : (k + 1 > n[a] - 1 ? n[a] - 1 : k + 1);
    }
    for (int ch = 0; ch < 4; ch++) {
      auto at = [&](int x, int y, int z) { return h2f(f[4 * ((size_t)x + (size_t)n[0] * ((size_t)y + (size_t)n[1] * z)) + ch]); };
      float c00 = at(i0[0], i0[1], i0[2]) * (1.0f - fr[0]) + at(i1[0], i0[1], i0[2]) * fr[0];
      float c10 = at(i0[0], i1[1], i0[2]) * (1.0f - fr[0]) + at(i1[0], i1[1], i0[2]) * fr[0];
      float c01 = at(i0[0], i0[1], i1[2]) * (1.0f - fr[0]) + at(i1[0], i0[1], i1[2]) * fr[0];
      float c11 = at(i0[0], i1[1], i1[2]) * (1.0f - fr[0]) + at(i1[0], i1[1], i1[2]) * fr[0];
      float c0 = c00 * (1.0f - fr[1]) + c10 * fr[1];
      float c1 = c01 * (1.0f - fr[1]) + c11 * fr[1];
      out[ch] = c0 * (1.0f - fr[2]) + c1 * fr[2];
    }
  }
  V3 vel3(V3 p) const {
    V3 v = sVel(p);
    if (dims[3] > 0.5f) v.z = 0.0f;
    return v;
  }
  V3 spawn() {
    bool is2D = dims[3] > 0.5f;
    if (P.emitter == 0u) {
      float x = 1.0f + rnd() * 2.0f;
      float y = 0.5f + rnd() * (dims[1] - 1.0f);
      float z3 = 0.5f + rnd() * (dims[2] - 1.0f); /* select() evaluates both operands */
      return v3(x, y, is2D ? 0.5f : z3);
    }
    uint32_t lines = P.lines > 1u ? P.lines : 1u;
    uint32_t tot = P.nozzles * lines;
    float r = rnd() * (float)tot;
    uint32_t k = r >= 4294967040.0f ? 0xffffffffu : (r <= 0.0f || !(r == r) ? 0u : (uint32_t)r);
    k = k < tot - 1u ? k : tot - 1u;
    float t = ((float)(k % P.nozzles) + 0.5f) / (float)P.nozzles;
    float l = (float)(k / P.nozzles) - 0.5f * (float)(lines - 1u);
    V3 A = v3(P.rake_a[0], P.rake_a[1], P.rake_a[2]), Bv = v3(P.rake_b[0], P.rake_b[1], P.rake_b[2]);
    V3 D = v3(P.rake_d[0], P.rake_d[1], P.rake_d[2]);
    V3 p = add(add(mul(A, 1.0f - t), mul(Bv, t)), mul(D, l));
    float jx = rnd() - 0.5f;
    float jy = rnd() - 0.5f;
    float jz = rnd() - 0.5f;
    p = add(p, mul(v3(jx, jy, jz), 0.35f));
    if (is2D) p.z = 0.5f;
    return p;
  }
  V3 fillPos() {
    bool is2D = dims[3] > 0.5f;
    for (int k = 0; k < 8; k++) {
      float x = 1.0f + rnd() * (dims[0] - 2.0f);
      float y = 0.5f + rnd() * (dims[1] - 1.0f);
      float z3 = 0.5f + rnd() * (dims[2] - 1.0f);
      V3 p = v3(x, y, is2D ? 0.5f : z3);
      if (!solidAt(p)) return p;
    }
    return spawn();
  }
  bool outside(V3 p) const {
    if (dims[3] > 0.5f) return p.x < 0.0f || p.y < 0.0f || p.x >= dims[0] - 1.0f || p.y >= dims[1];
    return p.x < 0.0f || p.y < 0.0f || p.z < 0.0f || p.x >= dims[0] - 1.0f || p.y >= dims[1] || p.z >= dims[2];
  }
};

}  // namespace

/* ============================================================================================ */
/* exported C API of the oracle                                                                 */
/* ============================================================================================ */
extern "C" {

int or_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

/* lattice tables: c (q*3 ints), w (q doubles), opp/mirrors (q ints each) */
int or_lattice(int dim, int* c, double* w, int* opp, int* my, int* mz, int* myz) {
  const Lat& L = lattice(dim == 3 ? 3 : 2);
  for (int i = 0; i < L.q; i++) {
    for (int a = 0; a < 3; a++) c[3 * i + a] = L.c[i][a];
    w[i] = L.w[i];
    opp[i] = L.opp[i];
    my[i] = L.my[i];
    mz[i] = L.mz[i];
    myz[i] = L.myz[i];
  }
  return L.q;
}

/* SolverGPU.writeParams (SolverGPU.ts:160-187) */
int or_pack_params(const wt_dims* d, const wt_params* p, wt_kparams* k) {
  if (!d || !p || !k) return WT_E_INVALID;
  std::memset(k, 0, sizeof *k);
  uint32_t nx = d->nx, ny = d->ny, nz = d->nz;
  k->nx = nx;
  k->ny = ny;
  k->nz = nz;
  k->n = nx * ny * nz;
  k->tau0 = (float)(3 * p->nu + 0.5);
  k->csmag2 = (float)(p->cs * p->cs);
  k->uin = (float)p->u;
  k->rho_in = 1.0f;
  k->ground = p->ground == WT_GROUND_FREESLIP ? 0 : (p->ground == WT_GROUND_NOSLIP ? 1 : 2);
  k->sponge_start = (float)(p->sponge_start * nx);
  k->sponge_nu = (float)p->sponge_nu;
  k->u_ground = p->ground == WT_GROUND_MOVING ? (float)p->u : 0.0f;
  k->ema_alpha = (float)p->ema_alpha;
  k->u_ref = (float)(p->u > 1e-4 ? p->u : 1e-4);
  k->ref_x = nx - 1 < 4 ? nx - 1 : 4;
  k->side_mode = p->sides == WT_SIDES_PERIODIC ? 1 : 0;
  k->collision = p->collision == WT_COLL_BGK ? 1 : 0;
  k->tau_wall = (float)p->tau_wall;
  k->sponge_in = (float)(p->sponge_in * nx);
  k->contact_h = 2.0f;
  k->interp = p->interp ? 1 : 0;
  return WT_OK;
}

/* setWheels packing (SolverGPU.ts:325-335): 8 floats per wheel (c, 1/max(r,1e-3), axis, hw) */
int or_pack_wheels(const wt_wheel* w, int count, float* out8) {
  int n = count < 16 ? count : 16;
  for (int k = 0; k < n; k++) {
    out8[8 * k + 0] = (float)w[k].c[0];
    out8[8 * k + 1] = (float)w[k].c[1];
    out8[8 * k + 2] = (float)w[k].c[2];
    out8[8 * k + 3] = (float)(1.0 / (w[k].r > 1e-3 ? w[k].r : 1e-3));
    out8[8 * k + 4] = (float)w[k].axis[0];
    out8[8 * k + 5] = (float)w[k].axis[1];
    out8[8 * k + 6] = (float)w[k].axis[2];
    out8[8 * k + 7] = (float)w[k].hw;
  }
  return n;
}

/* uploadSdf encoding (SolverGPU.ts:312-322): ~bits(d) for d >= 0, 0 = unknown */
void or_encode_sdf(const float* d, int64_t n, uint32_t* out) {
  for (int64_t i = 0; i < n; i++) {
    float v = d[i];
    if (!(v >= 0.0f)) {
      out[i] = 0;
      continue;
    }
    uint32_t b;
    std::memcpy(&b, &v, 4);
    out[i] = ~b;
  }
}

int or_init(const wt_dims* d, const wt_kparams* kp, int prec, const uint32_t* flags, void* fout, int mode,
            uint32_t seed, float amp) {
  Ctx X;
  int rc = make_ctx(X, d, kp, flags, nullptr, nullptr, 0);
  if (rc) return rc;
  const int64_t N = (int64_t)X.N;
#define OR_INIT(PR)                                          \
  {                                                          \
    Pops<PR> F{nullptr, fout, X.N, X.L};                     \
    _Pragma("omp parallel for schedule(static)") for (int64_t c = 0; c < N; c++) \
        init_cell<PR>(X, F, (size_t)c, mode, seed, amp);     \
  }
  if (prec == WT_PREC_F32) OR_INIT(WT_PREC_F32)
  else if (prec == WT_PREC_F16) OR_INIT(WT_PREC_F16)
  else if (prec == WT_PREC_F64) OR_INIT(WT_PREC_F64)
  else return WT_E_INVALID;
#undef OR_INIT
  return WT_OK;
}

/* `steps` fused stream-collide steps, ping-ponging a <-> b; the result is left in a when steps
 * is even and in b when it is odd. sdf is the encoded u32 buffer; wheels8 as or_pack_wheels. */
int or_stream_collide(const wt_dims* d, const wt_kparams* kp, int prec, void* a, void* b, const uint32_t* flags,
                      const uint32_t* sdf, const float* wheels8, int nwheels, int steps) {
  Ctx X;
  int rc = make_ctx(X, d, kp, flags, sdf, wheels8, nwheels);
  if (rc) return rc;
  const int64_t N = (int64_t)X.N;
  void* src = a;
  void* dst = b;
  for (int s = 0; s < steps; s++) {
#define OR_SC(PR)                                                                     \
  {                                                                                   \
    Pops<PR> F{src, dst, X.N, X.L};                                                   \
    _Pragma("omp parallel for schedule(static)") for (int64_t c = 0; c < N; c++) sc_cell<PR>(X, F, (size_t)c); \
  }
    if (prec == WT_PREC_F32) OR_SC(WT_PREC_F32)
    else if (prec == WT_PREC_F16) OR_SC(WT_PREC_F16)
    else if (prec == WT_PREC_F64) OR_SC(WT_PREC_F64)
    else return WT_E_INVALID;
#undef OR_SC
    void* t = src;
    src = dst;
    dst = t;
  }
  return WT_OK;
}

/* or_stream_collide with the learned closure in place of Smagorinsky (f32 / f16 storage, D3Q19) */
int or_stream_collide_lc(const wt_dims* d, const wt_kparams* kp, int prec, void* a, void* b, const uint32_t* flags,
                         const uint32_t* sdf, const float* wheels8, int nwheels, int steps, const wt_closure* c) {
  if (!c || prec == WT_PREC_F64 || !d || d->nz < 2 || !sdf) return WT_E_INVALID;
  Ctx X;
  int rc = make_ctx(X, d, kp, flags, sdf, wheels8, nwheels);
  if (rc) return rc;
  X.closure = c;
  const int64_t N = (int64_t)X.N;
  void* src = a;
  void* dst = b;
  for (int s = 0; s < steps; s++) {
    if (prec == WT_PREC_F32) {
      Pops<WT_PREC_F32> F{src, dst, X.N, X.L};
#pragma omp parallel for schedule(static)
      for (int64_t cc = 0; cc < N; cc++) sc_cell<WT_PREC_F32>(X, F, (size_t)cc);
    } else {
      Pops<WT_PREC_F16> F{src, dst, X.N, X.L};
#pragma omp parallel for schedule(static)
      for (int64_t cc = 0; cc < N; cc++) sc_cell<WT_PREC_F16>(X, F, (size_t)cc);
    }
    void* t = src;
    src = dst;
    dst = t;
  }
  return WT_OK;
}

/* the 10 closure features of n cells from their moments: m (n x 10) = pi xx, yy, zz, xy, xz, yz,
 * rho, ux, uy, uz; wall (n) = wall distance */
void or_closure_features(const float* m, const float* wall, int64_t n, float tau0, float* out) {
  for (int64_t r = 0; r < n; r++) {
    const float* q = m + r * 10;
    cl_features(q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8], q[9], tau0, wall[r], out + r * WT_CLOSURE_IN);
  }
}

/* nu_t of n feature rows */
void or_closure_forward(const wt_closure* c, const float* x, int64_t n, float* nu) {
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < n; r++) nu[r] = cl_forward(*c, x + r * WT_CLOSURE_IN);
}

/* loss L = mean(((nu - y) / nu_scale)^2) and dL / d(w1, b1, w2, b2, w3, b3) (1441 values, in the
 * wt_closure field order), with the rounding points of the training kernel: dz2 = bf16(dz3 w3
 * gelu'(z2)), dz1 = bf16((dz2 W2^T) gelu'(z1)) */
void or_closure_grad(const wt_closure* c, const float* x, const float* y, int64_t n, double* grad, double* loss) {
  const int H = WT_CLOSURE_HID, I = WT_CLOSURE_IN;
  const int NP = I * H + H + H * H + H + H + 1;
  std::vector<double> g((size_t)NP, 0.0);
  double ls = 0.0;
  for (int64_t r = 0; r < n; r++) {
    float xn[WT_CLOSURE_IN], z1[WT_CLOSURE_HID], h1[WT_CLOSURE_HID], z2[WT_CLOSURE_HID], h2[WT_CLOSURE_HID], z3;
    const float nu = cl_forward(*c, x + r * I, xn, z1, h1, z2, h2, &z3);
    const float d = (nu - y[r]) / c->nu_scale;
    ls += (double)(d * d);
    const float dz3 = 2.0f * d * (1.0f / (1.0f + std::exp(-z3)));
    float dz2[WT_CLOSURE_HID], dz1[WT_CLOSURE_HID];
    for (int j = 0; j < H; j++) {
      float gd;
      cl_gelu_d(z2[j], gd);
      dz2[j] = cl_bf16r(dz3 * cl_bf16r(c->w3[j]) * gd);
    }
    for (int i = 0; i < H; i++) {
      float a = 0.0f;
      for (int j = 0; j < H; j++) a = std::fma(dz2[j], cl_bf16r(c->w2[i][j]), a);
      float gd;
      cl_gelu_d(z1[i], gd);
      dz1[i] = cl_bf16r(a * gd);
    }
    double* gw1 = g.data();
    double* gb1 = gw1 + I * H;
    double* gw2 = gb1 + H;
    double* gb2 = gw2 + H * H;
    double* gw3 = gb2 + H;
    double* gb3 = gw3 + H;
    for (int k = 0; k < I; k++)
      for (int j = 0; j < H; j++) gw1[k * H + j] += (double)xn[k] * dz1[j];
    for (int j = 0; j < H; j++) gb1[j] += dz1[j];
    for (int i = 0; i < H; i++)
      for (int j = 0; j < H; j++) gw2[i * H + j] += (double)h1[i] * dz2[j];
    for (int j = 0; j < H; j++) {
      gb2[j] += dz2[j];
      gw3[j] += (double)dz3 * h2[j];
    }
    gb3[0] += dz3;
  }
  for (int p = 0; p < NP; p++) grad[p] = n > 0 ? g[(size_t)p] / (double)n : 0.0;
  if (loss) *loss = n > 0 ? ls / (double)n : 0.0;
}

/* macro pass on the current populations: vel4 (f32 view of the half4 velTex), EMA buffers
 * updated in place, result[10] = [ΣFx, ΣFy, ΣFz, max|u|², Σρ_ref, n_ref, nan, solid] (the
 * reference's reduction) followed by [Σρ over fluid cells in FP64, fluid cell count]. */
int or_macro(const wt_dims* d, const wt_kparams* kp, int prec, const void* fin, const uint32_t* flags,
             const uint32_t* sdf, const float* wheels8, int nwheels, float* vel4, float* meanA, float* meanB,
             double* result) {
  Ctx X;
  int rc = make_ctx(X, d, kp, flags, sdf, wheels8, nwheels);
  if (rc) return rc;
  MacroAcc acc;
  std::memset(&acc, 0, sizeof acc);
  for (size_t c = 0; c < X.N; c++) {
    if (prec == WT_PREC_F32) macro_cell<WT_PREC_F32>(X, Pops<WT_PREC_F32>{fin, nullptr, X.N, X.L}, c, vel4, meanA, meanB, acc);
    else if (prec == WT_PREC_F16) macro_cell<WT_PREC_F16>(X, Pops<WT_PREC_F16>{fin, nullptr, X.N, X.L}, c, vel4, meanA, meanB, acc);
    else macro_cell<WT_PREC_F64>(X, Pops<WT_PREC_F64>{fin, nullptr, X.N, X.L}, c, vel4, meanA, meanB, acc);
  }
  result[0] = acc.F[0];
  result[1] = acc.F[1];
  result[2] = acc.F[2];
  result[3] = acc.maxuu;
  result[4] = acc.rho_ref;
  result[5] = acc.n_ref;
  result[6] = acc.nan;
  result[7] = acc.solid;
  result[8] = acc.mass;
  result[9] = acc.fluid;
  return WT_OK;
}

/* GPU voxelizer semantics in f32 (VoxelizerGPU.voxelize, wgslVoxel.ts). flags/sdf are outputs
 * (u32 flags incl. wheel tags, encoded u32 sdf); info[8] as the project pass; wheels8 as
 * or_pack_wheels. hits (3n i32) and vote (n u32) are caller scratch. */
int or_voxelize_f32(const wt_dims* d, const float* pos, const uint32_t* idx, int64_t ntri, const float* M,
                    const float* wheels8, int nwheels, uint32_t* flags, uint32_t* sdf, int32_t* hits, uint32_t* vote,
                    uint32_t* info) {
  Vox V;
  std::memcpy(V.M, M, sizeof V.M);
  V.nx = d->nx;
  V.ny = d->ny;
  V.nz = d->nz;
  V.n = (size_t)d->nx * d->ny * d->nz;
  V.pos = pos;
  V.idx = idx;
  const int64_t n = (int64_t)V.n;
  std::memset(hits, 0, 3 * V.n * sizeof(int32_t));
  std::memset(vote, 0, V.n * sizeof(uint32_t));
  std::memset(sdf, 0, V.n * sizeof(uint32_t));
  info[0] = 0;
  info[1] = 0;
  info[2] = info[3] = info[4] = 0xffffffffu;
  info[5] = info[6] = info[7] = 0;
  if (ntri == 0) {
    std::memset(flags, 0, V.n * sizeof(uint32_t));
    info[2] = info[3] = info[4] = 0;
    return WT_OK;
  }
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t t = 0; t < ntri; t++) vox_crossings(V, (size_t)t, hits);
  const int dims[3] = {V.nx, V.ny, V.nz};
  for (int a = 0; a < 3; a++) {
    int ua = (a + 1) % 3, va = (a + 2) % 3;
    int nu = dims[ua], nv = dims[va], na = dims[a];
#pragma omp parallel for schedule(static)
    for (int64_t col = 0; col < (int64_t)nu * nv; col++) {
      int iu = (int)(col % nu), iv = (int)(col / nu);
      int32_t s = 0;
      for (int k = 0; k < na; k++) {
        size_t c = a == 0 ? V.cellOf(k, iu, iv) : (a == 1 ? V.cellOf(iv, k, iu) : V.cellOf(iu, iv, k));
        s += hits[(size_t)a * V.n + c];
        if (s != 0) __atomic_fetch_or(&vote[c], 1u << a, __ATOMIC_RELAXED);
      }
    }
  }
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t t = 0; t < ntri; t++) vox_surface(V, (size_t)t, vote);
  auto votes = [&](uint32_t v) { return __builtin_popcount(v & 7u) >= 2; };
#pragma omp parallel for schedule(static)
  for (int64_t id = 0; id < n; id++) {
    uint32_t v = vote[id];
    bool solid = votes(v);
    if (!solid && (v & 8u)) {
      uint32_t x = id % V.nx, y = (id / V.nx) % V.ny, z = id / ((int64_t)V.nx * V.ny);
      bool near = false;
      if (x > 0) near = near || votes(vote[id - 1]);
      if (x + 1 < (uint32_t)V.nx) near = near || votes(vote[id + 1]);
      if (y > 0) near = near || votes(vote[id - V.nx]);
      if (y + 1 < (uint32_t)V.ny) near = near || votes(vote[id + V.nx]);
      if (z > 0) near = near || votes(vote[id - (int64_t)V.nx * V.ny]);
      if (z + 1 < (uint32_t)V.nz) near = near || votes(vote[id + (int64_t)V.nx * V.ny]);
      solid = !near;
    }
    flags[id] = solid ? 1u : 0u;
  }
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t t = 0; t < ntri; t++) vox_sdf(V, (size_t)t, sdf);
  int nw = nwheels < 16 ? nwheels : 16;
  if (nw > 0) {
#pragma omp parallel for schedule(static)
    for (int64_t id = 0; id < n; id++) {
      if (flags[id] == 0u) continue;
      V3 p = v3((float)(id % V.nx) + 0.5f, (float)((id / V.nx) % V.ny) + 0.5f, (float)(id / ((int64_t)V.nx * V.ny)) + 0.5f);
      for (int k = 0; k < nw; k++) {
        const float* a = wheels8 + 8 * k;
        const float* b = a + 4;
        V3 dd = sub(p, v3(a[0], a[1], a[2]));
        V3 ax = v3(b[0], b[1], b[2]);
        float al = dot(dd, ax);
        float rad = len(sub(dd, mul(ax, al)));
        if (std::fabs(al) <= b[3] + 0.6f && rad <= 1.0f / a[3] + 0.75f) {
          flags[id] = 1u | ((uint32_t)(k + 1) << 8u);
          break;
        }
      }
    }
  }
  for (int z = 0; z < V.nz; z++)
    for (int y = 0; y < V.ny; y++) {
      bool hit = false;
      uint32_t cnt = 0;
      for (int x = 0; x < V.nx; x++) {
        if (flags[V.cellOf(x, y, z)] != 0u) {
          if (!hit) info[2] = std::min(info[2], (uint32_t)x);
          info[5] = std::max(info[5], (uint32_t)x);
          hit = true;
          cnt++;
        }
      }
      if (hit) {
        info[0]++;
        info[1] += cnt;
        info[3] = std::min(info[3], (uint32_t)y);
        info[6] = std::max(info[6], (uint32_t)y);
        info[4] = std::min(info[4], (uint32_t)z);
        info[7] = std::max(info[7], (uint32_t)z);
      }
    }
  return WT_OK;
}

/* voxelizeCPU (voxelizeCPU.ts:184-199) in f64: flags u8 (1 solid), sdf f32 (-1 unknown),
 * info[8] = frontal, solidCells, min[3], max[3] (max exclusive). */
int or_voxelize_f64(const wt_dims* d, const float* pos, int64_t nverts, const uint32_t* idx, int64_t ntri,
                    const double* M, uint8_t* flags, float* sdf, int32_t* info) {
  const int nx = d->nx, ny = d->ny, nz = d->nz;
  const size_t n = (size_t)nx * ny * nz;
  std::memset(flags, 0, n);
  for (size_t i = 0; i < n; i++) sdf[i] = -1.0f;
  for (int k = 0; k < 8; k++) info[k] = 0;
  if (ntri == 0) return WT_OK;
  const int dims[3] = {nx, ny, nz};
  auto cell = [&](int x, int y, int z) { return (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z); };
  std::vector<float> T(3 * (size_t)nverts);
  for (int64_t i = 0; i < nverts; i++) {
    double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    T[3 * i] = (float)(M[0] * x + M[4] * y + M[8] * z + M[12]);
    T[3 * i + 1] = (float)(M[1] * x + M[5] * y + M[9] * z + M[13]);
    T[3 * i + 2] = (float)(M[2] * x + M[6] * y + M[10] * z + M[14]);
  }
  std::vector<int16_t> hits(3 * n, 0);
  std::vector<uint8_t> vote(n, 0);
  std::vector<double> sd(n, -1.0);
  for (int64_t t = 0; t < ntri; t++) {
    double p0[3], p1[3], p2[3];
    for (int k = 0; k < 3; k++) {
      p0[k] = T[3 * (size_t)idx[3 * t] + k];
      p1[k] = T[3 * (size_t)idx[3 * t + 1] + k];
      p2[k] = T[3 * (size_t)idx[3 * t + 2] + k];
    }
    if (nz == 1 && (std::fmin(std::fmin(p0[2], p1[2]), p2[2]) > 1 || std::fmax(std::fmax(p0[2], p1[2]), p2[2]) < 0)) continue;
    for (int a = 0; a < 3; a++) {
      int ua = (a + 1) % 3, va = (a + 2) % 3;
      double Ax = p0[ua], Ay = p0[va], Bx = p1[ua], By = p1[va], Cx = p2[ua], Cy = p2[va];
      double area = (Bx - Ax) * (Cy - Ay) - (By - Ay) * (Cx - Ax);
      if (std::fabs(area) < 1e-12) continue;
      int sgn = area > 0 ? -1 : 1;
      int u0 = std::max((int)std::ceil(std::fmin(std::fmin(Ax, Bx), Cx) - 0.5), 0);
      int u1 = std::min((int)std::floor(std::fmax(std::fmax(Ax, Bx), Cx) - 0.5), dims[ua] - 1);
      int v0 = std::max((int)std::ceil(std::fmin(std::fmin(Ay, By), Cy) - 0.5), 0);
      int v1 = std::min((int)std::floor(std::fmax(std::fmax(Ay, By), Cy) - 0.5), dims[va] - 1);
      double inv = 1 / area;
      for (int iu = u0; iu <= u1; iu++)
        for (int iv = v0; iv <= v1; iv++) {
          double px = iu + 0.5 + 1.37e-4, py = iv + 0.5 + 2.71e-4;
          double w0 = ((Bx - px) * (Cy - py) - (By - py) * (Cx - px)) * inv;
          double w1 = ((Cx - px) * (Ay - py) - (Cy - py) * (Ax - px)) * inv;
          double w2 = 1 - w0 - w1;
          if (w0 < 0 || w1 < 0 || w2 < 0) continue;
          double h = w0 * p0[a] + w1 * p1[a] + w2 * p2[a];
          int k = (int)std::floor(h - 0.5) + 1;
          if (k >= dims[a]) continue;
          k = std::max(k, 0);
          size_t c = a == 0 ? cell(k, iu, iv) : (a == 1 ? cell(iv, k, iu) : cell(iu, iv, k));
          hits[(size_t)a * n + c] = (int16_t)(hits[(size_t)a * n + c] + sgn);
        }
    }
    {
      D3 a = d3(p0[0], p0[1], p0[2]), b = d3(p1[0], p1[1], p1[2]), c = d3(p2[0], p2[1], p2[2]);
      double m0 = std::fmax(std::fmax(std::hypot(std::hypot(b.x - a.x, b.y - a.y), b.z - a.z),
                                      std::hypot(std::hypot(c.x - a.x, c.y - a.y), c.z - a.z)),
                            std::hypot(std::hypot(c.x - b.x, c.y - b.y), c.z - b.z));
      int st = (int)std::fmin(std::fmax(std::ceil(m0 / 0.7), 1), 256);
      const int R = 2;
      for (int i = 0; i <= st; i++)
        for (int j = 0; j <= st - i; j++) {
          double u = (double)i / st, v = (double)j / st;
          double px = a.x + (b.x - a.x) * u + (c.x - a.x) * v;
          double py = a.y + (b.y - a.y) * u + (c.y - a.y) * v;
          double pz = a.z + (b.z - a.z) * u + (c.z - a.z) * v;
          if (nz == 1 && std::fabs(pz - 0.5) > 2.5) continue;
          int bx = (int)std::floor(px), by = (int)std::floor(py), bz = (int)std::floor(pz);
          for (int dz = nz == 1 ? 0 : -R; dz <= (nz == 1 ? 0 : R); dz++) {
            int qz = nz == 1 ? 0 : bz + dz;
            if (qz < 0 || qz >= nz) continue;
            for (int dy = -R; dy <= R; dy++) {
              int qy = by + dy;
              if (qy < 0 || qy >= ny) continue;
              for (int dx = -R; dx <= R; dx++) {
                int qx = bx + dx;
                if (qx < 0 || qx >= nx) continue;
                D3 ctr = d3(qx + 0.5, qy + 0.5, qz + 0.5);
                D3 cp = closest_pt<double, D3>(ctr, a, b, c, d3);
                double dd = std::hypot(std::hypot(ctr.x - cp.x, ctr.y - cp.y), ctr.z - cp.z);
                if (dd > 2.5) continue;
                size_t id = cell(qx, qy, qz);
                if (sd[id] < 0 || dd < sd[id]) sd[id] = dd;
              }
            }
          }
        }
    }
    double e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    double e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    double cl = std::hypot(std::hypot(cr[0], cr[1]), cr[2]);
    if (cl < 1e-12) continue;
    double nrm[3] = {cr[0] / cl, cr[1] / cl, cr[2] / cl};
    double m = std::fmax(std::fmax(std::hypot(std::hypot(e1[0], e1[1]), e1[2]), std::hypot(std::hypot(e2[0], e2[1]), e2[2])),
                         std::hypot(std::hypot(e2[0] - e1[0], e2[1] - e1[1]), e2[2] - e1[2]));
    int steps = (int)std::fmin(std::fmax(std::ceil(m / 0.4), 1), 384);
    double tol = 0.5 * std::fmax(std::fmax(std::fabs(nrm[0]), std::fabs(nrm[1])), std::fabs(nrm[2]));
    if (nz == 1) {
      if (std::hypot(nrm[0], nrm[1]) < 1e-4) continue;
      tol = 0.5 * std::fmax(std::fabs(nrm[0]), std::fabs(nrm[1]));
    }
    for (int i = 0; i <= steps; i++)
      for (int j = 0; j <= steps - i; j++) {
        double a = (double)i / steps, b = (double)j / steps;
        double x = p0[0] + e1[0] * a + e2[0] * b, y = p0[1] + e1[1] * a + e2[1] * b, z = p0[2] + e1[2] * a + e2[2] * b;
        if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) continue;
        int cx = (int)std::floor(x), cy = (int)std::floor(y), cz = (int)std::floor(z);
        double ctr[3] = {cx + 0.5, cy + 0.5, nz == 1 ? z : cz + 0.5};
        double dd = (ctr[0] - p0[0]) * nrm[0] + (ctr[1] - p0[1]) * nrm[1] + (ctr[2] - p0[2]) * nrm[2];
        if (std::fabs(dd) > tol) continue;
        vote[cell(cx, cy, cz)] |= 8;
      }
  }
  for (int a = 0; a < 3; a++) {
    int ua = (a + 1) % 3, va = (a + 2) % 3;
    for (int iv = 0; iv < dims[va]; iv++)
      for (int iu = 0; iu < dims[ua]; iu++) {
        int s = 0;
        for (int k = 0; k < dims[a]; k++) {
          size_t c = a == 0 ? cell(k, iu, iv) : (a == 1 ? cell(iv, k, iu) : cell(iu, iv, k));
          s += hits[(size_t)a * n + c];
          if (s != 0) vote[c] |= (uint8_t)(1 << a);
        }
      }
  }
  auto votes = [](int v) { return ((v & 1) + ((v >> 1) & 1) + ((v >> 2) & 1)) >= 2; };
  int solidCells = 0;
  int mn[3] = {2147483647, 2147483647, 2147483647}, mx[3] = {-1, -1, -1};
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++) {
        size_t c = cell(x, y, z);
        int v = vote[c];
        bool solid = votes(v);
        if (!solid && (v & 8)) {
          bool near = (x > 0 && votes(vote[c - 1])) || (x + 1 < nx && votes(vote[c + 1])) ||
                      (y > 0 && votes(vote[c - nx])) || (y + 1 < ny && votes(vote[c + nx])) ||
                      (z > 0 && votes(vote[c - (size_t)nx * ny])) || (z + 1 < nz && votes(vote[c + (size_t)nx * ny]));
          solid = !near;
        }
        if (solid) {
          flags[c] = 1;
          solidCells++;
          mn[0] = std::min(mn[0], x);
          mn[1] = std::min(mn[1], y);
          mn[2] = std::min(mn[2], z);
          mx[0] = std::max(mx[0], x);
          mx[1] = std::max(mx[1], y);
          mx[2] = std::max(mx[2], z);
        }
      }
  int frontal = 0;
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++)
        if (flags[cell(x, y, z)]) {
          frontal++;
          break;
        }
  for (size_t i = 0; i < n; i++) sdf[i] = (float)sd[i];
  info[0] = frontal;
  info[1] = solidCells;
  bool ok = solidCells > 0;
  for (int k = 0; k < 3; k++) {
    info[2 + k] = ok ? mn[k] : 0;
    info[5 + k] = ok ? mx[k] + 1 : 0;
  }
  return WT_OK;
}

/* one dispatch of PARTICLES_WGSL. vel is half4 bits per cell, state count*4, hist count*trail*4 */
int or_tracers(const wt_dims* d, const wt_tracer_params* p, const uint16_t* vel, const uint32_t* flags, float* state,
               float* hist) {
  Tr T0;
  std::memset(&T0, 0, sizeof T0);
  T0.P = *p;
  T0.dims[0] = (float)d->nx;
  T0.dims[1] = (float)d->ny;
  T0.dims[2] = (float)d->nz;
  T0.dims[3] = d->nz == 1 ? 1.0f : 0.0f;
  T0.vel = vel;
  T0.flags = flags;
  const uint32_t count = p->count;
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)count; ii++) {
    uint32_t i = (uint32_t)ii;
    Tr T = T0;
    T.rng = pcg(i ^ pcg(p->seed));
    float s[4] = {state[4 * ii], state[4 * ii + 1], state[4 * ii + 2], state[4 * ii + 3]};
    if (p->fill != 0u) {
      V3 q;
      if (p->emitter == 0u) {
        q = T.fillPos();
        s[3] = (float)p->trail;
      } else {
        q = T.spawn();
        s[3] = -std::floor(T.rnd() * p->max_age);
      }
      s[0] = q.x;
      s[1] = q.y;
      s[2] = q.z;
      for (int k = 0; k < 4; k++) state[4 * ii + k] = s[k];
      for (uint32_t k = 0; k < p->trail; k++) {
        float* h = hist + 4 * ((size_t)k * count + i);
        h[0] = s[0];
        h[1] = s[1];
        h[2] = s[2];
        h[3] = 0.0f;
      }
      continue;
    }
    if (p->advance == 0u) continue;
    if (s[3] < 0.0f) {
      s[3] += 1.0f;
      if (s[3] >= 0.0f) {
        V3 q = T.spawn();
        s[0] = q.x;
        s[1] = q.y;
        s[2] = q.z;
        s[3] = 0.0f;
      }
    } else {
      V3 pp = v3(s[0], s[1], s[2]);
      V3 v0 = T.vel3(pp);
      float disp = len(v0) * p->steps;
      float ns = std::ceil(disp / 0.6f);
      ns = std::fmin(std::fmax(ns, 1.0f), 24.0f);
      uint32_t nsub = (uint32_t)ns;
      float h = p->steps / (float)nsub;
      for (uint32_t k = 0; k < nsub; k++) {
        V3 a = T.vel3(pp);
        V3 b = T.vel3(add(pp, mul(a, 0.5f * h)));
        pp = add(pp, mul(b, h));
      }
      s[0] = pp.x;
      s[1] = pp.y;
      s[2] = pp.z;
      s[3] = s[3] + 1.0f;
      if (T.outside(pp) || T.solidAt(pp) || s[3] > p->max_age * 4.0f) {
        V3 q = T.spawn();
        s[0] = q.x;
        s[1] = q.y;
        s[2] = q.z;
        s[3] = 0.0f;
      }
    }
    for (int k = 0; k < 4; k++) state[4 * ii + k] = s[k];
    float* h = hist + 4 * ((size_t)p->head * count + i);
    h[0] = s[0];
    h[1] = s[1];
    h[2] = s[2];
    h[3] = 0.0f;
  }
  return WT_OK;
}

uint32_t or_pcg(uint32_t v) { return pcg(v); }

/* Streamlines (src/render/tracers.ts:152-200): pts seeds x points float4, seed-major. */
int or_streamlines(const wt_dims* d, const wt_streamline_params* S, float u_lat, const uint16_t* vel,
                   const uint16_t* mean, const uint32_t* flags, float* pts) {
  Tr T;
  std::memset(&T, 0, sizeof T);
  T.dims[0] = (float)d->nx;
  T.dims[1] = (float)d->ny;
  T.dims[2] = (float)d->nz;
  T.dims[3] = d->nz == 1 ? 1.0f : 0.0f;
  T.vel = vel;
  T.flags = flags;
  const bool is2D = T.dims[3] > 0.5f;
  auto velf = [&](V3 p) {
    float v4[4];
    T.sF4(S->use_mean ? mean : vel, p, v4);
    V3 v = v3(v4[0], v4[1], v4[2]);
    if (is2D) v.z = 0.0f;
    return v;
  };
  auto outside = [&](V3 p) {
    if (is2D) return p.x < 0.0f || p.y < 0.0f || p.x >= T.dims[0] || p.y >= T.dims[1];
    return p.x < 0.0f || p.y < 0.0f || p.z < 0.0f || p.x >= T.dims[0] || p.y >= T.dims[1] || p.z >= T.dims[2];
  };
  const uint32_t per = S->per_line > 1u ? S->per_line : 1u;
  for (uint32_t s = 0; s < S->seeds; s++) {
    const float l = (float)(s / per) - 0.5f * (float)(S->seeds / per - 1u);
    const float t = ((float)(s % per) + 0.5f) / (float)per;
    V3 A = v3(S->rake_a[0], S->rake_a[1], S->rake_a[2]), B = v3(S->rake_b[0], S->rake_b[1], S->rake_b[2]);
    V3 D = v3(S->rake_d[0], S->rake_d[1], S->rake_d[2]);
    V3 p = add(add(mul(A, 1.0f - t), mul(B, t)), mul(D, l));
    if (is2D) p.z = 0.5f;
    bool alive = true;
    const float U = u_lat > 1e-5f ? u_lat : 1e-5f;
    for (uint32_t k = 0; k < S->points; k++) {
      const V3 v = velf(p);
      const float sp = len(v);
      if (alive && (outside(p) || T.solidAt(p) || sp < U * 1e-3f)) alive = false;
      float* o = pts + 4 * ((size_t)s * S->points + k);
      o[0] = p.x;
      o[1] = p.y;
      o[2] = p.z;
      o[3] = alive ? sp : -1.0f;
      if (!alive) continue;
      const V3 a = v3(v.x / sp, v.y / sp, v.z / sp);
      const V3 vm = velf(add(p, mul(a, 0.5f * S->h)));
      const float lm = len(vm);
      if (lm < 1e-9f) {
        alive = false;
        continue;
      }
      p = add(p, mul(v3(vm.x / lm, vm.y / lm, vm.z / lm), S->h));
    }
  }
  return WT_OK;
}

/* Probes (src/render/tracers.ts:109-125): out 2 float4 per probe (instantaneous, mean). */
int or_probes(const wt_dims* d, const float* pos4, int count, const uint16_t* vel, const uint16_t* mean, float* out) {
  Tr T;
  std::memset(&T, 0, sizeof T);
  T.dims[0] = (float)d->nx;
  T.dims[1] = (float)d->ny;
  T.dims[2] = (float)d->nz;
  T.dims[3] = d->nz == 1 ? 1.0f : 0.0f;
  for (int i = 0; i < count; i++) {
    V3 p = v3(pos4[4 * i], pos4[4 * i + 1], pos4[4 * i + 2]);
    float v[4], m[4];
    T.sF4(vel, p, v);
    T.sF4(mean, p, m);
    if (T.dims[3] > 0.5f) {
      v[2] = 0.0f;
      m[2] = 0.0f;
    }
    for (int k = 0; k < 4; k++) {
      out[8 * i + k] = v[k];
      out[8 * i + 4 + k] = m[k];
    }
  }
  return WT_OK;
}

/* Derived fields (src/solver/wgslLbm.ts:527-592): inputs are the half4 velocity texture (raw
 * binary16 bits), the flags, the EMA statistics and uRef; outputs vort / stat / mean as raw
 * binary16 x 4 per cell (the reference's rgba16float textures). */
int or_derive(const wt_dims* d, float u_ref, const uint16_t* vel_h, const uint32_t* flags, const float* meanA,
              const float* meanB, uint16_t* vort_h, uint16_t* stat_h, uint16_t* mean_h) {
  const int NX = d->nx, NY = d->ny, NZ = d->nz;
  const int dim = NZ > 1 ? 3 : 2;
  const size_t N = (size_t)NX * NY * NZ;
  auto cell = [&](int x, int y, int z) { return (size_t)x + (size_t)NX * ((size_t)y + (size_t)NY * (size_t)z); };
  auto vel = [&](int x, int y, int z, float out[3]) {
    x = x < 0 ? 0 : (x > NX - 1 ? NX - 1 : x);
    y = y < 0 ? 0 : (y > NY - 1 ? NY - 1 : y);
    z = z < 0 ? 0 : (z > NZ - 1 ? NZ - 1 : z);
    const uint16_t* v = vel_h + 4 * cell(x, y, z);
    for (int k = 0; k < 3; k++) {
      _Float16 h;
      std::memcpy(&h, v + k, 2);
      out[k] = (float)h;
    }
  };
  auto solidAt = [&](int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= NX || y >= NY || z >= NZ) return false;
    return flags[cell(x, y, z)] != 0u;
  };
  auto put = [&](uint16_t* o, const float v[4]) {
    for (int k = 0; k < 4; k++) {
      _Float16 h = (_Float16)v[k];
      std::memcpy(o + k, &h, 2);
    }
  };
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)N; ii++) {
    const size_t idx = (size_t)ii;
    const int x = (int)(idx % NX), y = (int)((idx / NX) % NY), z = (int)(idx / ((size_t)NX * NY));
    const bool solid = flags[idx] != 0u;
    float vort[4] = {0.f, 0.f, 0.f, 0.f};
    if (!solid) {
      float xp[3], xm[3], yp[3], ym[3], zp[3] = {0, 0, 0}, zm[3] = {0, 0, 0};
      vel(x + 1, y, z, xp);
      vel(x - 1, y, z, xm);
      vel(x, y + 1, z, yp);
      vel(x, y - 1, z, ym);
      float J[3][3];  // J[j][i] = d u_i / d x_j; columns dx, dy, dz of mat3x3(dx, dy, dz)
      for (int i = 0; i < 3; i++) {
        J[0][i] = 0.5f * (xp[i] - xm[i]);
        J[1][i] = 0.5f * (yp[i] - ym[i]);
      }
      if (dim == 3) {
        vel(x, y, z + 1, zp);
        vel(x, y, z - 1, zm);
        for (int i = 0; i < 3; i++) J[2][i] = 0.5f * (zp[i] - zm[i]);
      } else {
        for (int i = 0; i < 3; i++) J[2][i] = 0.0f;
      }
      const float wx = J[1][2] - J[2][1];
      const float wy = J[2][0] - J[0][2];
      const float wz = J[0][1] - J[1][0];
      float S2 = 0.0f, W2 = 0.0f;
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          const float sv = 0.5f * (J[j][i] + J[i][j]);
          const float wv = 0.5f * (J[j][i] - J[i][j]);
          S2 += sv * sv;
          W2 += wv * wv;
        }
      float near = 0.0f;
      for (int dd = 1; dd <= 2; dd++)
        for (int a = 0; a < dim; a++) {
          const int ex = a == 0 ? dd : 0, ey = a == 1 ? dd : 0, ez = a == 2 ? dd : 0;
          if (solidAt(x + ex, y + ey, z + ez) || solidAt(x - ex, y - ey, z - ez)) {
            const float v = dd == 1 ? 1.0f : 0.5f;
            near = near > v ? near : v;
          }
        }
      vort[0] = wx;
      vort[1] = wy;
      vort[2] = wz;
      vort[3] = 0.5f * (W2 - S2) * (1.0f - near);
    }
    const float* m = meanA + 4 * idx;
    const float dotm = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
    float k = meanB[idx] - dotm;
    k = k > 0.0f ? k : 0.0f;
    const float ur = u_ref > 1e-6f ? u_ref : 1e-6f;
    const float ti = std::sqrt(k / 3.0f) / ur;
    const float st[4] = {solid ? 0.0f : ti, solid ? 1.0f : 0.0f, 0.0f, 0.0f};
    put(vort_h + 4 * idx, vort);
    put(stat_h + 4 * idx, st);
    put(mean_h + 4 * idx, m);
  }
  return WT_OK;
}

/* Strided export (src/solver/SolverGPU.ts:374-425): the raw half4 fields at every stride-th cell,
 * clamped to the last cell, x fastest. */
int or_export(const wt_dims* d, int stride, const uint16_t* vel_h, const uint16_t* mean_h, const uint16_t* vort_h,
              float* vel4, float* mean4, float* vort4) {
  const int NX = d->nx, NY = d->ny, NZ = d->nz;
  const int ox = (NX + stride - 1) / stride, oy = (NY + stride - 1) / stride, oz = (NZ + stride - 1) / stride;
  const int64_t n = (int64_t)ox * oy * oz;
  for (int64_t i = 0; i < n; i++) {
    const int gx = (int)(i % ox), gy = (int)((i / ox) % oy), gz = (int)(i / ((int64_t)ox * oy));
    const int px = gx * stride < NX - 1 ? gx * stride : NX - 1;
    const int py = gy * stride < NY - 1 ? gy * stride : NY - 1;
    const int pz = gz * stride < NZ - 1 ? gz * stride : NZ - 1;
    const size_t c = (size_t)px + (size_t)NX * ((size_t)py + (size_t)NY * (size_t)pz);
    const uint16_t* src[3] = {vel_h, mean_h, vort_h};
    float* dst[3] = {vel4, mean4, vort4};
    for (int f = 0; f < 3; f++)
      for (int k = 0; k < 4; k++) {
        _Float16 h;
        std::memcpy(&h, src[f] + 4 * c + k, 2);
        dst[f][4 * i + k] = (float)h;
      }
  }
  return WT_OK;
}

}  // extern "C"
