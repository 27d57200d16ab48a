// wt_closure.cu — trainer of the learned LES closure: the sample pool, the training-data kernels
// (targets from the box-filtered fine run, selection), the BF16 training and inference kernel
// (tcgen05 MMAs for the two forward layers, the input gradient of layer 2 and the weight gradients
// of both layers, f32 accumulation), the gradient reduction and Adam. No counterpart in the reference, whose only closure is Smagorinsky (wgslLbm.ts:206-214).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "wt_closure.cuh"
#include "wt_internal.h"

using namespace wt;

struct wt_trainer {
  int device = 0;
  cudaStream_t stream = nullptr;
  int64_t cap = 0, count = 0;
  float* xs = nullptr;  // pool: features [cap][10]
  float* ys = nullptr;  // pool: targets [cap]
  float* P = nullptr;   // master parameters (CL_NPARAM), the wt_closure fields w1 .. b3 in order
  float* m = nullptr;   // Adam moments
  float* v = nullptr;
  int64_t adam_t = 0;
  float shift[CL_IN] = {}, scale[CL_IN] = {}, nu_scale = 1.0f;
  bool have_model = false;
  float* partials = nullptr;  // per-block gradient partials [blocks][CL_NPARAM + 1]
  int64_t partial_blocks = 0;
  double* grad = nullptr;      // reduced gradient sums (CL_NPARAM) and loss sum (+1)
  float* scratch = nullptr;    // training-data scratch
  size_t scratch_floats = 0;
  float* io = nullptr;         // staging for host rows
  size_t io_floats = 0;
  int radius = 1;              // projection sums over (2 radius + 1)^3 coarse cells
  std::string err;
};

namespace {

constexpr int TR_THREADS = 128;
constexpr int TR_NOUT = CL_NPARAM + 1;  // gradient entries + loss
// tensor-memory columns: z1 (0-31), z2 (32-63), dH1 (64-95); training adds dW2 (96-127) and dW1 (128-159)
constexpr uint32_t TR_TMEM_COLS_INFER = 128;
constexpr uint32_t TR_TMEM_COLS_TRAIN = 256;
constexpr uint32_t TR_WAIT_LIMIT = 1u << 22;
// shared-memory layout of k_train (bytes)
constexpr int TS_A = 0;          // inputs x', 128 x 16 bf16, K-major (A of layer 1)
constexpr int TS_H1 = 4096;      // h1, 128 x 32 bf16, K-major (A of layer 2)
constexpr int TS_DZ2 = 12288;    // dz2, 128 x 32 bf16, K-major (A of the dH1 product)
constexpr int TS_H2 = 20480;     // h2, [128][32] f32
constexpr int TS_W1 = 36864;     // W1 image (N = 32 hidden, K = 16 inputs)
constexpr int TS_W2 = 37888;     // W2 image (N = out, K = in)
constexpr int TS_W2T = 39936;    // W2 transposed image (N = in, K = out)
constexpr int TS_DZ3 = 41984;    // dz3 [128] f32
constexpr int TS_LOSS = 42496;   // per-row loss [128] f32
constexpr int TS_BAR = 43008;    // mbarrier, the tensor-memory address, pad, drain barrier
constexpr int TS_DRAIN = TS_BAR + 16;
// inference: 45 KB of dynamic shared memory, so at most 4 blocks share an SM and their
// 4 x 128 tensor-memory columns fit in its 512
constexpr int TS_BYTES_INFER = 45 * 1024;
// Training adds the operands of the weight-gradient products, summed over the block's 128 samples
// (the K dimension):
//   dW2 and db2 = [h1^T ; 1] dz2: A = h1^T in rows 0-31, ones in row 32, zeros below (128 x 128
//                 bf16, K-major); B = dz2^T (32 x 128)
//   dW1 and db1 = [x'^T ; 1] dz1: A = x'^T in rows 0-9, ones in row 16, zeros elsewhere; B = dz1^T
// M = 128 (tensor-memory lane = row), N = 32, eight K = 16 steps each. 125 KB: one block per SM,
// with 256 tensor-memory columns.
constexpr int TS_GA2 = 46080;
constexpr int TS_GA1 = TS_GA2 + 32768;
constexpr int TS_GB2 = TS_GA1 + 32768;
constexpr int TS_GB1 = TS_GB2 + 8192;
constexpr int TS_BYTES_TRAIN = TS_GB1 + 8192;
constexpr int TR_ONE_K1 = 16;    // the ones row of the dW1 operand (its sums over the samples are db1)
static_assert(TS_DRAIN + 8 <= TS_BYTES_INFER && TS_BYTES_INFER <= TS_GA2 && 5 * (TS_BYTES_INFER + 1024) > 228 * 1024,
              "inference layout");
static_assert(TS_BYTES_TRAIN <= 227 * 1024 && 2 * (TS_BYTES_TRAIN + 1024) > 228 * 1024, "training layout");

// parameter offsets in the master vector
constexpr int PO_W1 = 0, PO_B1 = 320, PO_W2 = 352, PO_B2 = 1376, PO_W3 = 1408, PO_B3 = 1440;
static_assert(PO_B3 + 1 == CL_NPARAM, "parameter count");

struct TrainArgs {
  const float* xs;
  const float* ys;
  int64_t count;      // pool size (random mode)
  int64_t offset;     // first row (range mode)
  int64_t rows;       // rows of this launch
  uint64_t seed;      // random mode when nonzero
  uint64_t draw;      // index of this minibatch
  const float* P;
  float scale[CL_IN], nshift[CL_IN], nu_scale;  // x' = bf16(fma(x, scale, nshift))
  float* nu_out;      // inference
  float* partials;    // training: [block][TR_NOUT]
};

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ float sm_bf16(const uint8_t* base, uint32_t off) {
  return bf16_val(*reinterpret_cast<const uint16_t*>(base + off));
}

// One block = 128 samples (one per thread, tensor-memory lane = thread). Forward: the two 32-wide
// layers on tcgen05 (x' W1 into columns 0-31, h1 W2 into 32-63), the output layer on CUDA cores.
// TRAIN adds the backward pass: dz3 = 2 (nu - y) sigmoid(z3) / nu_scale per sample,
// dz2 = bf16(dz3 w3 gelu'(z2)), dH1 = dz2 W2^T on tcgen05 (columns 64-95), dz1 = bf16(dH1 gelu'(z1)),
// then the block's weight and bias gradients of layers 1 and 2 as two more tcgen05 products over
// its 128 samples ([h1^T ; 1] dz2 into columns 96-127, [x'^T ; 1] dz1 into 128-159) and those of
// the output layer on CUDA cores (f32, rows in order), into partials[block].
template <bool TRAIN>
__global__ void __launch_bounds__(TR_THREADS) k_train(const __grid_constant__ TrainArgs A, int* __restrict__ err) {
  extern __shared__ __align__(128) uint8_t sm[];
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  const int64_t row = (int64_t)blockIdx.x * TR_THREADS + tid;
  const bool valid = row < A.rows;
  int64_t si = 0;
  if (valid) {
    if (A.seed != 0) si = (int64_t)(mix64(A.seed ^ mix64(A.draw * 0x100000001B3ull + (uint64_t)row)) % (uint64_t)A.count);
    else si = A.offset + row;
  }
  float x[CL_IN], y = 0.0f;
#pragma unroll
  for (int k = 0; k < CL_IN; k++) x[k] = valid ? __ldg(A.xs + si * CL_IN + k) : 0.0f;
  if (TRAIN && valid) y = __ldg(A.ys + si);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + TS_BAR);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + TS_BAR + 8);
  uint64_t* dbar = reinterpret_cast<uint64_t*>(sm + TS_DRAIN);
  // weight images from the f32 master weights
  for (uint32_t e = tid; e < (uint32_t)(CL_H * CL_K1); e += TR_THREADS) {
    const uint32_t n = e / CL_K1, k = e % CL_K1;
    const float w = k < (uint32_t)CL_IN ? A.P[PO_W1 + k * CL_H + n] : 0.0f;
    *reinterpret_cast<uint16_t*>(sm + TS_W1 + umma::kmaj_off(n, k, CL_K1)) = bf16_bits(w);
  }
  for (uint32_t e = tid; e < (uint32_t)(CL_H * CL_H); e += TR_THREADS) {
    const uint32_t i = e / CL_H, j = e % CL_H;
    const uint16_t b = bf16_bits(A.P[PO_W2 + i * CL_H + j]);
    *reinterpret_cast<uint16_t*>(sm + TS_W2 + umma::kmaj_off(j, i, CL_H)) = b;
    *reinterpret_cast<uint16_t*>(sm + TS_W2T + umma::kmaj_off(i, j, CL_H)) = b;
  }
  if (tid == 0) {
    umma::mbar_init(mbar, 1);
    umma::mbar_init(dbar, 1);
  }
  constexpr uint32_t TMEM_COLS = TRAIN ? TR_TMEM_COLS_TRAIN : TR_TMEM_COLS_INFER;
  if (warp == 0) umma::tmem_alloc(tslot, TMEM_COLS);
  if constexpr (TRAIN) {
    // the weight-gradient A operands are zero outside their data and ones rows
    uint4* z = reinterpret_cast<uint4*>(sm + TS_GA2);
    for (uint32_t e = tid; e < 2u * 32768u / 16u; e += TR_THREADS) z[e] = make_uint4(0u, 0u, 0u, 0u);
  }
  // x' row (zeros for padding rows)
  {
    uint32_t w[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int k0 = 2 * k, k1 = 2 * k + 1;
      const uint32_t lo = (valid && k0 < CL_IN) ? bf16_bits(__fmaf_rn(x[k0], A.scale[k0], A.nshift[k0])) : 0u;
      const uint32_t hi = (valid && k1 < CL_IN) ? bf16_bits(__fmaf_rn(x[k1], A.scale[k1], A.nshift[k1])) : 0u;
      w[k] = lo | (hi << 16);
    }
    *reinterpret_cast<uint4*>(sm + TS_A + umma::kmaj_off(tid, 0, CL_K1)) = make_uint4(w[0], w[1], w[2], w[3]);
    *reinterpret_cast<uint4*>(sm + TS_A + umma::kmaj_off(tid, 8, CL_K1)) = make_uint4(w[4], w[5], w[6], w[7]);
    if constexpr (TRAIN) {
      // column tid of [x'^T ; 1] and the ones of [h1^T ; 1] (after the zero fill above)
      __syncthreads();
#pragma unroll
      for (int k = 0; k < CL_IN; k++)
        *reinterpret_cast<uint16_t*>(sm + TS_GA1 + umma::kmaj_off(k, tid, TR_THREADS)) =
            (uint16_t)(w[k >> 1] >> (16 * (k & 1)));
      *reinterpret_cast<uint16_t*>(sm + TS_GA1 + umma::kmaj_off(TR_ONE_K1, tid, TR_THREADS)) = 0x3F80u;
      *reinterpret_cast<uint16_t*>(sm + TS_GA2 + umma::kmaj_off(CL_H, tid, TR_THREADS)) = 0x3F80u;
    }
  }
  umma::fence_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  constexpr uint32_t ID = umma::idesc_bf16<128, CL_H>();
  bool ok = true;
  uint32_t phase = 0;
  auto issue_wait = [&]() {
    ok = umma::mbar_wait(mbar, phase, TR_WAIT_LIMIT) && ok;
    phase ^= 1u;
    umma::fence_after_sync();
  };
  // layer 1
  if (tid == 0) {
    umma::mma_bf16(tmem, umma::sdesc(umma::smem_u32(sm + TS_A), 128, 256), umma::sdesc(umma::smem_u32(sm + TS_W1), 128, 256),
                   ID, false);
    umma::commit(mbar);
  }
  issue_wait();
#pragma unroll
  for (int c = 0; c < 4; c++) {
    float v[8];
    umma::tmem_ld8(umma::tmem_lane_addr(tmem, warp, 8 * c), v);
    umma::tmem_wait_ld();
    uint32_t pk[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int j = 8 * c + 2 * e;
      const uint32_t lo = bf16_bits(cl_gelu(__fadd_rn(v[2 * e], A.P[PO_B1 + j])));
      const uint32_t hi = bf16_bits(cl_gelu(__fadd_rn(v[2 * e + 1], A.P[PO_B1 + j + 1])));
      pk[e] = lo | (hi << 16);
    }
    *reinterpret_cast<uint4*>(sm + TS_H1 + umma::kmaj_off(tid, 8 * c, CL_H)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    if constexpr (TRAIN) {
#pragma unroll
      for (int e = 0; e < 8; e++)
        *reinterpret_cast<uint16_t*>(sm + TS_GA2 + umma::kmaj_off(8 * c + e, tid, TR_THREADS)) =
            (uint16_t)(pk[e >> 1] >> (16 * (e & 1)));
    }
  }
  umma::fence_before_sync();
  umma::fence_async_smem();
  __syncthreads();
  // layer 2
  if (tid == 0) {
    umma::fence_after_sync();
    const uint32_t a = umma::smem_u32(sm + TS_H1), b = umma::smem_u32(sm + TS_W2);
    umma::mma_bf16(tmem + 32, umma::sdesc(a, 128, 512), umma::sdesc(b, 128, 512), ID, false);
    umma::mma_bf16(tmem + 32, umma::sdesc(a + 256, 128, 512), umma::sdesc(b + 256, 128, 512), ID, true);
    umma::commit(mbar);
  }
  issue_wait();
  float z2[CL_H];
#pragma unroll
  for (int c = 0; c < 4; c++) {
    float v[8];
    umma::tmem_ld8(umma::tmem_lane_addr(tmem, warp, 32 + 8 * c), v);
    umma::tmem_wait_ld();
#pragma unroll
    for (int e = 0; e < 8; e++) z2[8 * c + e] = __fadd_rn(v[e], A.P[PO_B2 + 8 * c + e]);
  }
  float ze = 0.0f, zo = 0.0f;
  float h2[CL_H];
#pragma unroll
  for (int j = 0; j < CL_H; j++) {
    h2[j] = cl_gelu(z2[j]);
    if (j & 1) zo = __fmaf_rn(h2[j], bf16r(A.P[PO_W3 + j]), zo);
    else ze = __fmaf_rn(h2[j], bf16r(A.P[PO_W3 + j]), ze);
  }
  const float z3 = __fadd_rn(__fadd_rn(ze, zo), A.P[PO_B3]);
  const float nu = __fmul_rn(A.nu_scale, cl_softplus(z3));
  if constexpr (!TRAIN) {
    if (valid) A.nu_out[row] = ok ? nu : __int_as_float(0x7fc00000);
  } else {
    const float d = valid ? (nu - y) / A.nu_scale : 0.0f;
    const float dz3 = valid ? 2.0f * d * cl_sigmoid(z3) : 0.0f;
    reinterpret_cast<float*>(sm + TS_DZ3)[tid] = dz3;
    reinterpret_cast<float*>(sm + TS_LOSS)[tid] = d * d;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      uint32_t pk[4];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int j = 8 * c + 2 * e;
        float g0, g1;
        cl_gelu_d(z2[j], g0);
        cl_gelu_d(z2[j + 1], g1);
        const uint32_t lo = bf16_bits(dz3 * bf16r(A.P[PO_W3 + j]) * g0);
        const uint32_t hi = bf16_bits(dz3 * bf16r(A.P[PO_W3 + j + 1]) * g1);
        pk[e] = lo | (hi << 16);
      }
      *reinterpret_cast<uint4*>(sm + TS_DZ2 + umma::kmaj_off(tid, 8 * c, CL_H)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
#pragma unroll
      for (int e = 0; e < 8; e++)
        *reinterpret_cast<uint16_t*>(sm + TS_GB2 + umma::kmaj_off(8 * c + e, tid, TR_THREADS)) =
            (uint16_t)(pk[e >> 1] >> (16 * (e & 1)));
      float4* hrow = reinterpret_cast<float4*>(sm + TS_H2 + (tid * CL_H + 8 * c) * 4);
      hrow[0] = make_float4(h2[8 * c], h2[8 * c + 1], h2[8 * c + 2], h2[8 * c + 3]);
      hrow[1] = make_float4(h2[8 * c + 4], h2[8 * c + 5], h2[8 * c + 6], h2[8 * c + 7]);
    }
    umma::fence_before_sync();
    umma::fence_async_smem();
    __syncthreads();
    // dH1 = dz2 W2^T
    if (tid == 0) {
      umma::fence_after_sync();
      const uint32_t a = umma::smem_u32(sm + TS_DZ2), b = umma::smem_u32(sm + TS_W2T);
      umma::mma_bf16(tmem + 64, umma::sdesc(a, 128, 512), umma::sdesc(b, 128, 512), ID, false);
      umma::mma_bf16(tmem + 64, umma::sdesc(a + 256, 128, 512), umma::sdesc(b + 256, 128, 512), ID, true);
      umma::commit(mbar);
    }
    issue_wait();
#pragma unroll
    for (int c = 0; c < 4; c++) {
      float dh[8], z1[8];
      umma::tmem_ld8(umma::tmem_lane_addr(tmem, warp, 64 + 8 * c), dh);
      umma::tmem_ld8(umma::tmem_lane_addr(tmem, warp, 8 * c), z1);
      umma::tmem_wait_ld();
      uint32_t pk[4];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int j = 8 * c + 2 * e;
        float g0, g1;
        cl_gelu_d(__fadd_rn(z1[2 * e], A.P[PO_B1 + j]), g0);
        cl_gelu_d(__fadd_rn(z1[2 * e + 1], A.P[PO_B1 + j + 1]), g1);
        const uint32_t lo = valid ? bf16_bits(dh[2 * e] * g0) : 0u;
        const uint32_t hi = valid ? bf16_bits(dh[2 * e + 1] * g1) : 0u;
        pk[e] = lo | (hi << 16);
      }
#pragma unroll
      for (int e = 0; e < 8; e++)
        *reinterpret_cast<uint16_t*>(sm + TS_GB1 + umma::kmaj_off(8 * c + e, tid, TR_THREADS)) =
            (uint16_t)(pk[e >> 1] >> (16 * (e & 1)));
    }
    // the weight and bias gradients of layers 1 and 2 on the tensor cores: sums over the block's
    // 128 samples, eight K = 16 steps per product
    umma::fence_before_sync();
    umma::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
      const uint32_t a2 = umma::smem_u32(sm + TS_GA2), b2 = umma::smem_u32(sm + TS_GB2);
      const uint32_t a1 = umma::smem_u32(sm + TS_GA1), b1 = umma::smem_u32(sm + TS_GB1);
#pragma unroll
      for (int k = 0; k < TR_THREADS / 16; k++) {
        umma::mma_bf16(tmem + 96, umma::sdesc(a2 + 256 * k, 128, 2048), umma::sdesc(b2 + 256 * k, 128, 2048), ID, k > 0);
        umma::mma_bf16(tmem + 128, umma::sdesc(a1 + 256 * k, 128, 2048), umma::sdesc(b1 + 256 * k, 128, 2048), ID,
                       k > 0);
      }
      umma::commit(mbar);
    }
    issue_wait();
    float* out = A.partials + (size_t)blockIdx.x * TR_NOUT;
    // rows 0-31 and 32 of the dW2 product, rows 0-9 and 16 of the dW1 product (lanes of warps 0-1)
    if (warp < 2) {
      float v2[32], v1[32];
      umma::tmem_ld32(umma::tmem_lane_addr(tmem, warp, 96), v2);
      umma::tmem_ld32(umma::tmem_lane_addr(tmem, warp, 128), v1);
      umma::tmem_wait_ld();
      if (tid <= (uint32_t)CL_H) {
        float* o = tid < (uint32_t)CL_H ? out + PO_W2 + tid * CL_H : out + PO_B2;
#pragma unroll
        for (int j = 0; j < CL_H; j++) o[j] = v2[j];
      }
      if (tid < (uint32_t)CL_IN || tid == (uint32_t)TR_ONE_K1) {
        float* o = tid < (uint32_t)CL_IN ? out + PO_W1 + tid * CL_H : out + PO_B1;
#pragma unroll
        for (int j = 0; j < CL_H; j++) o[j] = v1[j];
      }
    }
    // the output layer's weights and bias and the loss: block sums on CUDA cores (rows in order, f32)
    const float* dz = reinterpret_cast<const float*>(sm + TS_DZ3);
    for (int p = PO_W3 + (int)tid; p < TR_NOUT; p += TR_THREADS) {
      float acc = 0.0f;
      if (p < PO_B3) {
        const int j = p - PO_W3;
        const float* h2s = reinterpret_cast<const float*>(sm + TS_H2);
        for (int r = 0; r < TR_THREADS; r++) acc = __fmaf_rn(dz[r], h2s[r * CL_H + j], acc);
      } else if (p == PO_B3) {
        for (int r = 0; r < TR_THREADS; r++) acc = __fadd_rn(acc, dz[r]);
      } else {
        const float* ls = reinterpret_cast<const float*>(sm + TS_LOSS);
        for (int r = 0; r < TR_THREADS; r++) acc = __fadd_rn(acc, ls[r]);
      }
      out[p] = acc;
    }
  }
  // after a timed-out wait, the MMAs finish before their tensor memory is released
  const bool drained = umma::drain_before_free(dbar, !ok, TR_WAIT_LIMIT);
  __syncthreads();
  if (warp == 0) umma::tmem_free(tmem, TMEM_COLS);
  if (!ok || !drained) atomicOr(err, 4);
}

// sums of the block partials in f64, blocks in order
__global__ void k_grad_reduce(const float* __restrict__ partials, int64_t blocks, double* __restrict__ grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= TR_NOUT) return;
  double acc = 0.0;
  for (int64_t b = 0; b < blocks; b++) acc += (double)partials[b * TR_NOUT + p];
  grad[p] = acc;
}

// Adam on the mean gradient (sum / rows); loss[step] = mean minibatch loss
__global__ void k_adam(float* __restrict__ P, float* __restrict__ m, float* __restrict__ v,
                       const double* __restrict__ grad, double inv_rows, float lr, float b1, float b2, float eps,
                       float c1, float c2, float* __restrict__ loss_out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0 && loss_out) *loss_out = (float)(grad[CL_NPARAM] * inv_rows);
  if (p >= CL_NPARAM) return;
  const float g = (float)(grad[p] * inv_rows);
  const float mm = b1 * m[p] + (1.0f - b1) * g;
  const float vv = b2 * v[p] + (1.0f - b2) * g * g;
  m[p] = mm;
  v[p] = vv;
  P[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
}

// ---- training data --------------------------------------------------------------------------
// From the filtered fields (k_closure_filter): per coarse cell, the filtered strain rate S~ from
// central differences of u~ (cells whose six neighbours are all valid, off the domain faces), the
// projection numerator num = -dev(T) : S~ and denominator den = 2 S~ : S~. tgt (8 floats SoA):
// num, den, S~ (xx, yy, zz, xy, xz, yz); den < 0 marks a cell without a stencil.
__global__ void k_closure_strain(const float* __restrict__ F, int nx, int ny, int nz, float* __restrict__ tgt) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
  if (x >= nx) return;
  const size_t n = (size_t)nx * ny * nz;
  const size_t c = (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * (size_t)z);
  bool ok = x > 0 && y > 0 && z > 0 && x < nx - 1 && y < ny - 1 && z < nz - 1 && F[10 * n + c] != 0.0f;
  const size_t sx = 1, sy = (size_t)nx, sz = (size_t)nx * ny;
  if (ok)
    ok = F[10 * n + c + sx] != 0.0f && F[10 * n + c - sx] != 0.0f && F[10 * n + c + sy] != 0.0f &&
         F[10 * n + c - sy] != 0.0f && F[10 * n + c + sz] != 0.0f && F[10 * n + c - sz] != 0.0f;
  if (!ok) {
    tgt[c] = 0.0f;
    tgt[n + c] = -1.0f;
    for (int q = 2; q < 8; q++) tgt[(size_t)q * n + c] = 0.0f;
    return;
  }
  double g[3][3];  // g[a][b] = d u_a / d x_b
  const size_t st[3] = {sx, sy, sz};
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++)
      g[a][b] = 0.5 * ((double)F[(size_t)(1 + a) * n + c + st[b]] - (double)F[(size_t)(1 + a) * n + c - st[b]]);
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  double S[6], T[6];
  for (int q = 0; q < 6; q++) {
    S[q] = 0.5 * (g[pa[q]][pb[q]] + g[pb[q]][pa[q]]);
    T[q] = (double)F[(size_t)(4 + q) * n + c];
  }
  const double tr = (T[0] + T[1] + T[2]) / 3.0;
  double num = 0, den = 0;
  for (int q = 0; q < 6; q++) {
    const double w = q < 3 ? 1.0 : 2.0;
    num -= w * (T[q] - (q < 3 ? tr : 0.0)) * S[q];
    den += 2.0 * w * S[q] * S[q];
  }
  tgt[c] = (float)num;
  tgt[n + c] = (float)den;
  for (int q = 0; q < 6; q++) tgt[(size_t)(2 + q) * n + c] = (float)S[q];
}

struct SelectArgs {
  const float* F;    // filtered fields (11 SoA)
  const float* tgt;  // strain / projection (8 SoA)
  const uint32_t* cflags;
  const uint32_t* csdf;
  int nx, ny, nz;
  float tau0;       // coarse molecular tau0
  float x_lo, x_hi; // kept x range (outside the sponges)
  uint32_t keep;    // keep threshold on a 32-bit hash
  uint64_t seed;
  int radius;       // projection box half-width
};

// the sample of coarse cell c: nu* from the (2 radius + 1)^3 sums of num and den over stencil cells;
// features of the stress the coarse handle sees at that viscosity, Pi = -(2/3) rho~ (tau0 + 3 nu*) S~
__device__ bool closure_sample(const SelectArgs& A, int x, int y, int z, float (&xf)[CL_IN], float& yt) {
  const int R = A.radius;
  if (x < R + 1 || y < R + 1 || z < R + 1 || x > A.nx - R - 2 || y > A.ny - R - 2 || z > A.nz - R - 2) return false;
  if ((float)x < A.x_lo || (float)x >= A.x_hi) return false;
  const size_t n = (size_t)A.nx * A.ny * A.nz;
  const size_t c = (size_t)x + (size_t)A.nx * ((size_t)y + (size_t)A.ny * (size_t)z);
  if (A.cflags[c] != 0u || A.tgt[n + c] < 0.0f) return false;
  const uint32_t h = (uint32_t)(mix64(A.seed ^ (uint64_t)c) >> 32);
  if (h >= A.keep) return false;
  double sn = 0, sd = 0;
  for (int dz = -R; dz <= R; dz++)
    for (int dy = -R; dy <= R; dy++)
      for (int dx = -R; dx <= R; dx++) {
        const size_t q = c + (size_t)((ptrdiff_t)dx + (ptrdiff_t)A.nx * ((ptrdiff_t)dy + (ptrdiff_t)A.ny * dz));
        const float d = A.tgt[n + q];
        if (d >= 0.0f) {
          sn += A.tgt[q];
          sd += d;
        }
      }
  const double nu = sd > 1e-30 ? fmax(sn / sd, 0.0) : 0.0;
  const float rho = A.F[c];
  const float ux = A.F[n + c], uy = A.F[2 * n + c], uz = A.F[3 * n + c];
  const float k = (float)(-(2.0 / 3.0) * (double)rho * ((double)A.tau0 + 3.0 * nu));
  float S[6];
  for (int q = 0; q < 6; q++) S[q] = A.tgt[(size_t)(2 + q) * n + c];
  cl_features(k * S[0], k * S[1], k * S[2], k * S[3], k * S[4], k * S[5], rho, ux, uy, uz, A.tau0,
              cl_wall_dist(A.csdf[c]), xf);
  yt = (float)nu;
  return true;
}

// pass 0: kept cells per block of 256 cells; pass 1: write them in cell order at base[block] + rank
template <int PASS>
__global__ void __launch_bounds__(256) k_closure_select(const __grid_constant__ SelectArgs A, uint32_t* __restrict__ counts,
                                                        const int64_t* __restrict__ base, float* __restrict__ xs,
                                                        float* __restrict__ ys, int64_t cap) {
  __shared__ uint32_t wsum[8];
  const size_t n = (size_t)A.nx * A.ny * A.nz;
  const size_t c = (size_t)blockIdx.x * 256 + threadIdx.x;
  float xf[CL_IN];
  float yt = 0.0f;
  bool keep = false;
  if (c < n) {
    const int x = (int)(c % A.nx), y = (int)((c / A.nx) % A.ny), z = (int)(c / ((size_t)A.nx * A.ny));
    keep = closure_sample(A, x, y, z, xf, yt);
  }
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t bal = __ballot_sync(0xffffffffu, keep);
  if (lane == 0) wsum[w] = __popc(bal);
  __syncthreads();
  if (PASS == 0) {
    if (threadIdx.x == 0) {
      uint32_t t = 0;
      for (int k = 0; k < 8; k++) t += wsum[k];
      counts[blockIdx.x] = t;
    }
    return;
  }
  if (!keep) return;
  uint32_t before = __popc(bal & ((1u << lane) - 1u));
  for (uint32_t k = 0; k < w; k++) before += wsum[k];
  const int64_t slot = base[blockIdx.x] + before;
  if (slot >= cap) return;
  for (int k = 0; k < CL_IN; k++) xs[slot * CL_IN + k] = xf[k];
  ys[slot] = yt;
}

// per-block sums and sums of squares of the 10 features and the target, f64
__global__ void __launch_bounds__(256) k_pool_stats(const float* __restrict__ xs, const float* __restrict__ ys,
                                                    int64_t count, double* __restrict__ out) {
  __shared__ double red[256];
  double s[2 * (CL_IN + 1)];
  for (int q = 0; q < 2 * (CL_IN + 1); q++) s[q] = 0.0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < count; r += (int64_t)gridDim.x * blockDim.x) {
    for (int k = 0; k <= CL_IN; k++) {
      const double v = k < CL_IN ? (double)xs[r * CL_IN + k] : (double)ys[r];
      s[2 * k] += v;
      s[2 * k + 1] += v * v;
    }
  }
  for (int q = 0; q < 2 * (CL_IN + 1); q++) {
    red[threadIdx.x] = s[q];
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
      if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[(size_t)blockIdx.x * 2 * (CL_IN + 1) + q] = red[0];
    __syncthreads();
  }
}

int tfail(wt_trainer* t, int code, const std::string& msg) {
  t->err = msg;
  return code;
}

#define TR_CUDA(t, expr, what)                                                            \
  do {                                                                                    \
    cudaError_t e_ = (expr);                                                              \
    if (e_ != cudaSuccess) return tfail((t), WT_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); \
  } while (0)

struct TrDevice {
  int prev = 0;
  explicit TrDevice(int d) {
    cudaGetDevice(&prev);
    cudaSetDevice(d);
  }
  ~TrDevice() { cudaSetDevice(prev); }
};

int ensure_buf(wt_trainer* t, float** p, size_t* have, size_t want, const char* what) {
  if (*have >= want) return WT_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  if (cudaMalloc((void**)p, want * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    return tfail(t, WT_E_OOM, std::string("trainer: cannot allocate ") + what);
  }
  *have = want;
  return WT_OK;
}

int ensure_partials(wt_trainer* t, int64_t blocks) {
  if (blocks <= t->partial_blocks) return WT_OK;
  if (t->partials) cudaFree(t->partials);
  t->partials = nullptr;
  t->partial_blocks = 0;
  if (cudaMalloc((void**)&t->partials, (size_t)blocks * TR_NOUT * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    return tfail(t, WT_E_OOM, "trainer: cannot allocate gradient partials");
  }
  t->partial_blocks = blocks;
  return WT_OK;
}

// k_train's dynamic shared memory exceeds the 48 KB default: opt in (on the current device)
cudaError_t train_smem_optin() {
  cudaError_t r = cudaFuncSetAttribute(k_train<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, TS_BYTES_TRAIN);
  if (r == cudaSuccess)
    r = cudaFuncSetAttribute(k_train<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, TS_BYTES_INFER);
  return r;
}

TrainArgs make_args(const wt_trainer* t) {
  TrainArgs A;
  std::memset(&A, 0, sizeof A);
  A.xs = t->xs;
  A.ys = t->ys;
  A.count = t->count;
  A.P = t->P;
  for (int k = 0; k < CL_IN; k++) {
    A.scale[k] = t->scale[k];
    A.nshift[k] = -(t->shift[k] * t->scale[k]);
  }
  A.nu_scale = t->nu_scale;
  return A;
}

}  // namespace

extern "C" {

int wt_trainer_create(int32_t device, int64_t capacity, wt_trainer** out) {
  if (!out || capacity < 0) return WT_E_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail_unbound(WT_E_NO_DEVICE, "wt_trainer_create: no CUDA device");
  }
  if (device < 0 || device >= ndev) return fail_unbound(WT_E_INVALID, "wt_trainer_create: bad device ordinal");
  wt_trainer* t = new (std::nothrow) wt_trainer();
  if (!t) return WT_E_OOM;
  t->device = device;
  t->cap = capacity;
  TrDevice g(device);
  bool okk = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking) == cudaSuccess;
  okk = okk && train_smem_optin() == cudaSuccess;
  okk = okk && cudaMalloc((void**)&t->P, CL_NPARAM * sizeof(float)) == cudaSuccess;
  okk = okk && cudaMalloc((void**)&t->m, CL_NPARAM * sizeof(float)) == cudaSuccess;
  okk = okk && cudaMalloc((void**)&t->v, CL_NPARAM * sizeof(float)) == cudaSuccess;
  okk = okk && cudaMalloc((void**)&t->grad, TR_NOUT * sizeof(double)) == cudaSuccess;
  if (okk && capacity > 0) {
    okk = cudaMalloc((void**)&t->xs, (size_t)capacity * CL_IN * sizeof(float)) == cudaSuccess &&
          cudaMalloc((void**)&t->ys, (size_t)capacity * sizeof(float)) == cudaSuccess;
  }
  if (!okk) {
    cudaGetLastError();
    wt_trainer_destroy(t);
    return fail_unbound(WT_E_OOM, "wt_trainer_create: device allocation failed");
  }
  cudaMemset(t->P, 0, CL_NPARAM * sizeof(float));
  cudaMemset(t->m, 0, CL_NPARAM * sizeof(float));
  cudaMemset(t->v, 0, CL_NPARAM * sizeof(float));
  for (int k = 0; k < CL_IN; k++) t->scale[k] = 1.0f;
  *out = t;
  return WT_OK;
}

void wt_trainer_destroy(wt_trainer* t) {
  if (!t) return;
  TrDevice g(t->device);
  if (t->stream) cudaStreamSynchronize(t->stream);
  void* bufs[] = {t->xs, t->ys, t->P, t->m, t->v, t->partials, t->grad, t->scratch, t->io};
  for (void* b : bufs)
    if (b) cudaFree(b);
  if (t->stream) cudaStreamDestroy(t->stream);
  delete t;
}

const char* wt_trainer_last_error(const wt_trainer* t) { return t ? t->err.c_str() : ""; }
int64_t wt_trainer_count(const wt_trainer* t) { return t ? t->count : 0; }

int wt_trainer_clear(wt_trainer* t) {
  if (!t) return WT_E_INVALID;
  t->count = 0;
  return WT_OK;
}

int wt_trainer_set_projection_radius(wt_trainer* t, int32_t radius) {
  if (!t || radius < 1 || radius > 3) return WT_E_INVALID;
  t->radius = radius;
  return WT_OK;
}

int wt_trainer_put_samples(wt_trainer* t, const float* x, const float* y, int64_t n) {
  if (!t || n < 0 || (n > 0 && (!x || !y))) return WT_E_INVALID;
  if (t->count + n > t->cap) return tfail(t, WT_E_INVALID, "wt_trainer_put_samples: pool capacity exceeded");
  if (n == 0) return WT_OK;
  TrDevice g(t->device);
  TR_CUDA(t, cudaMemcpyAsync(t->xs + t->count * CL_IN, x, (size_t)n * CL_IN * sizeof(float), cudaMemcpyHostToDevice,
                             t->stream), "put samples");
  TR_CUDA(t, cudaMemcpyAsync(t->ys + t->count, y, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, t->stream),
          "put samples");
  TR_CUDA(t, cudaStreamSynchronize(t->stream), "put samples");
  t->count += n;
  return WT_OK;
}

int wt_trainer_read_samples(wt_trainer* t, int64_t offset, int64_t n, float* x, float* y) {
  if (!t || offset < 0 || n < 0 || offset + n > t->count) return WT_E_INVALID;
  if (n == 0) return WT_OK;
  TrDevice g(t->device);
  if (x)
    TR_CUDA(t, cudaMemcpyAsync(x, t->xs + offset * CL_IN, (size_t)n * CL_IN * sizeof(float), cudaMemcpyDeviceToHost,
                               t->stream), "read samples");
  if (y)
    TR_CUDA(t, cudaMemcpyAsync(y, t->ys + offset, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, t->stream),
            "read samples");
  TR_CUDA(t, cudaStreamSynchronize(t->stream), "read samples");
  return WT_OK;
}

int wt_trainer_add_samples(wt_trainer* t, wt_solver* fine, wt_solver* coarse, double keep, uint64_t seed,
                           int64_t* added) {
  if (added) *added = 0;
  if (!t || !fine || !coarse || !(keep >= 0.0) || keep > 1.0) return WT_E_INVALID;
  if (!fine->is3d || !coarse->is3d)
    return tfail(t, WT_E_UNSUPPORTED, "wt_trainer_add_samples: both handles must be D3Q19");
  if (fine->dims.nx != 2 * coarse->dims.nx || fine->dims.ny != 2 * coarse->dims.ny ||
      fine->dims.nz != 2 * coarse->dims.nz)
    return tfail(t, WT_E_INVALID, "wt_trainer_add_samples: fine dims must be twice the coarse dims");
  if (fine->device != t->device || coarse->device != t->device)
    return tfail(t, WT_E_INVALID, "wt_trainer_add_samples: handles and trainer must share a device");
  if (fine->pending_init || fine->cls_dirty)
    return tfail(t, WT_E_STATE, "wt_trainer_add_samples: step the fine handle at least once after its geometry");
  TrDevice g(t->device);
  TR_CUDA(t, cudaStreamSynchronize(fine->stream), "add samples: fine stream");
  TR_CUDA(t, cudaStreamSynchronize(coarse->stream), "add samples: coarse stream");
  const int nx = coarse->dims.nx, ny = coarse->dims.ny, nz = coarse->dims.nz;
  const size_t n = (size_t)nx * ny * nz;
  int rc = ensure_buf(t, &t->scratch, &t->scratch_floats, 19 * n, "training-data scratch");
  if (rc) return rc;
  float* F = t->scratch;
  float* T = t->scratch + 11 * n;
  TR_CUDA(t, launch_closure_filter(fine, nx, ny, nz, F, t->stream), "closure filter");
  {
    const int bx = nx >= 128 ? 128 : ((nx + 31) / 32) * 32;
    k_closure_strain<<<dim3((nx + bx - 1) / bx, ny, nz), bx, 0, t->stream>>>(F, nx, ny, nz, T);
    TR_CUDA(t, cudaGetLastError(), "closure strain");
  }
  SelectArgs A;
  A.F = F;
  A.tgt = T;
  A.cflags = coarse->flags;
  A.csdf = coarse->sdf;
  A.nx = nx;
  A.ny = ny;
  A.nz = nz;
  A.tau0 = coarse->kp.tau0;
  A.x_lo = coarse->kp.sponge_in;
  A.x_hi = std::min((float)nx, coarse->kp.sponge_start);
  A.keep = keep >= 1.0 ? 0xFFFFFFFFu : (uint32_t)(keep * 4294967296.0);
  A.seed = seed;
  A.radius = t->radius;
  const int64_t blocks = (int64_t)((n + 255) / 256);
  uint32_t* counts = nullptr;
  int64_t* base = nullptr;
  TR_CUDA(t, cudaMalloc((void**)&counts, (size_t)blocks * 4), "select counts");
  if (cudaMalloc((void**)&base, (size_t)blocks * 8) != cudaSuccess) {
    cudaFree(counts);
    return tfail(t, WT_E_OOM, "select offsets");
  }
  std::vector<uint32_t> hc((size_t)blocks);
  std::vector<int64_t> hb((size_t)blocks);
  k_closure_select<0><<<(unsigned)blocks, 256, 0, t->stream>>>(A, counts, nullptr, nullptr, nullptr, 0);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(hc.data(), counts, (size_t)blocks * 4, cudaMemcpyDeviceToHost, t->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
  int64_t total = 0;
  if (e == cudaSuccess) {
    for (int64_t b = 0; b < blocks; b++) {
      hb[(size_t)b] = t->count + total;
      total += hc[(size_t)b];
    }
    e = cudaMemcpyAsync(base, hb.data(), (size_t)blocks * 8, cudaMemcpyHostToDevice, t->stream);
  }
  if (e == cudaSuccess) {
    k_closure_select<1><<<(unsigned)blocks, 256, 0, t->stream>>>(A, counts, base, t->xs, t->ys, t->cap);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
  cudaFree(counts);
  cudaFree(base);
  if (e != cudaSuccess) return tfail(t, WT_E_CUDA, std::string("add samples: ") + cudaGetErrorString(e));
  const int64_t kept = std::min<int64_t>(total, t->cap - t->count);
  t->count += kept;
  if (added) *added = kept;
  return WT_OK;
}

int wt_trainer_stats(wt_trainer* t, double* mean11, double* std11) {
  if (!t || !mean11 || !std11) return WT_E_INVALID;
  if (t->count == 0) return tfail(t, WT_E_STATE, "wt_trainer_stats: empty pool");
  TrDevice g(t->device);
  const int blocks = (int)std::min<int64_t>((t->count + 255) / 256, 148 * 4);
  const size_t nv = (size_t)blocks * 2 * (CL_IN + 1);
  double* d = nullptr;
  TR_CUDA(t, cudaMalloc((void**)&d, nv * sizeof(double)), "stats");
  std::vector<double> h(nv);
  k_pool_stats<<<blocks, 256, 0, t->stream>>>(t->xs, t->ys, t->count, d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d, nv * sizeof(double), cudaMemcpyDeviceToHost, t->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
  cudaFree(d);
  if (e != cudaSuccess) return tfail(t, WT_E_CUDA, std::string("stats: ") + cudaGetErrorString(e));
  for (int k = 0; k <= CL_IN; k++) {
    double s = 0, s2 = 0;
    for (int b = 0; b < blocks; b++) {
      s += h[(size_t)b * 2 * (CL_IN + 1) + 2 * k];
      s2 += h[(size_t)b * 2 * (CL_IN + 1) + 2 * k + 1];
    }
    const double mean = s / (double)t->count;
    mean11[k] = mean;
    std11[k] = std::sqrt(std::max(0.0, s2 / (double)t->count - mean * mean));
  }
  return WT_OK;
}

int wt_trainer_set_model(wt_trainer* t, const wt_closure* m) {
  if (!t || !m) return WT_E_INVALID;
  const float* v = reinterpret_cast<const float*>(m);
  for (size_t k = 0; k < sizeof(wt_closure) / sizeof(float); k++)
    if (!std::isfinite(v[k])) return tfail(t, WT_E_INVALID, "wt_trainer_set_model: non-finite value");
  if (!(m->nu_scale > 0.0f)) return tfail(t, WT_E_INVALID, "wt_trainer_set_model: nu_scale must be > 0");
  TrDevice g(t->device);
  static_assert(offsetof(wt_closure, b3) - offsetof(wt_closure, w1) == (CL_NPARAM - 1) * sizeof(float),
                "the trainable fields w1 .. b3 are contiguous");
  TR_CUDA(t, cudaMemcpyAsync(t->P, reinterpret_cast<const char*>(m) + offsetof(wt_closure, w1),
                             CL_NPARAM * sizeof(float), cudaMemcpyHostToDevice, t->stream), "set model");
  TR_CUDA(t, cudaMemsetAsync(t->m, 0, CL_NPARAM * sizeof(float), t->stream), "set model");
  TR_CUDA(t, cudaMemsetAsync(t->v, 0, CL_NPARAM * sizeof(float), t->stream), "set model");
  TR_CUDA(t, cudaStreamSynchronize(t->stream), "set model");
  for (int k = 0; k < CL_IN; k++) {
    t->shift[k] = m->shift[k];
    t->scale[k] = m->scale[k];
  }
  t->nu_scale = m->nu_scale;
  t->adam_t = 0;
  t->have_model = true;
  return WT_OK;
}

int wt_trainer_get_model(const wt_trainer* t, wt_closure* out) {
  if (!t || !out) return WT_E_INVALID;
  wt_trainer* tt = const_cast<wt_trainer*>(t);
  if (!t->have_model) return tfail(tt, WT_E_STATE, "wt_trainer_get_model: no model set");
  TrDevice g(t->device);
  std::memset(out, 0, sizeof *out);
  TR_CUDA(tt, cudaMemcpyAsync(reinterpret_cast<char*>(out) + offsetof(wt_closure, w1), t->P, CL_NPARAM * sizeof(float),
                              cudaMemcpyDeviceToHost, t->stream), "get model");
  TR_CUDA(tt, cudaStreamSynchronize(t->stream), "get model");
  for (int k = 0; k < CL_IN; k++) {
    out->shift[k] = t->shift[k];
    out->scale[k] = t->scale[k];
  }
  out->nu_scale = t->nu_scale;
  return WT_OK;
}

int wt_trainer_fit(wt_trainer* t, const wt_train_params* p, float* loss) {
  if (!t || !p || p->steps < 0 || p->batch <= 0) return WT_E_INVALID;
  if (!t->have_model) return tfail(t, WT_E_STATE, "wt_trainer_fit: no model set");
  if (t->count == 0) return tfail(t, WT_E_STATE, "wt_trainer_fit: empty pool");
  if (p->seed == 0) return tfail(t, WT_E_INVALID, "wt_trainer_fit: seed must be nonzero");
  if (p->steps == 0) return WT_OK;
  TrDevice g(t->device);
  const int64_t blocks = ((int64_t)p->batch + TR_THREADS - 1) / TR_THREADS;
  int rc = ensure_partials(t, blocks);
  if (rc) return rc;
  float* dloss = nullptr;
  int* derr = nullptr;
  TR_CUDA(t, cudaMalloc((void**)&dloss, (size_t)p->steps * sizeof(float)), "fit");
  if (cudaMalloc((void**)&derr, sizeof(int)) != cudaSuccess) {
    cudaFree(dloss);
    return tfail(t, WT_E_OOM, "fit");
  }
  cudaMemsetAsync(derr, 0, sizeof(int), t->stream);
  TrainArgs A = make_args(t);
  A.rows = p->batch;
  A.seed = p->seed;
  A.partials = t->partials;
  cudaError_t e = cudaSuccess;
  for (int s = 0; s < p->steps && e == cudaSuccess; s++) {
    A.draw = (uint64_t)s;
    k_train<true><<<(unsigned)blocks, TR_THREADS, TS_BYTES_TRAIN, t->stream>>>(A, derr);
    k_grad_reduce<<<(TR_NOUT + 127) / 128, 128, 0, t->stream>>>(t->partials, blocks, t->grad);
    t->adam_t++;
    const float c1 = (float)(1.0 - std::pow((double)p->beta1, (double)t->adam_t));
    const float c2 = (float)(1.0 - std::pow((double)p->beta2, (double)t->adam_t));
    k_adam<<<(CL_NPARAM + 127) / 128, 128, 0, t->stream>>>(t->P, t->m, t->v, t->grad, 1.0 / (double)p->batch, p->lr,
                                                           p->beta1, p->beta2, p->eps, c1, c2, dloss + s);
    e = cudaGetLastError();
  }
  int herr = 0;
  if (e == cudaSuccess && loss)
    e = cudaMemcpyAsync(loss, dloss, (size_t)p->steps * sizeof(float), cudaMemcpyDeviceToHost, t->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, t->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
  cudaFree(dloss);
  cudaFree(derr);
  if (e != cudaSuccess) return tfail(t, WT_E_CUDA, std::string("fit: ") + cudaGetErrorString(e));
  if (herr) return tfail(t, WT_E_CUDA, "fit: a tensor-core wait timed out");
  return WT_OK;
}

int wt_trainer_grad(wt_trainer* t, int64_t offset, int64_t n, wt_closure* grad, double* loss) {
  if (!t || offset < 0 || n <= 0 || offset + n > t->count) return WT_E_INVALID;
  if (!t->have_model) return tfail(t, WT_E_STATE, "wt_trainer_grad: no model set");
  TrDevice g(t->device);
  const int64_t blocks = (n + TR_THREADS - 1) / TR_THREADS;
  int rc = ensure_partials(t, blocks);
  if (rc) return rc;
  int* derr = nullptr;
  TR_CUDA(t, cudaMalloc((void**)&derr, sizeof(int)), "grad");
  cudaMemsetAsync(derr, 0, sizeof(int), t->stream);
  TrainArgs A = make_args(t);
  A.offset = offset;
  A.rows = n;
  A.partials = t->partials;
  std::vector<double> h(TR_NOUT);
  int herr = 0;
  k_train<true><<<(unsigned)blocks, TR_THREADS, TS_BYTES_TRAIN, t->stream>>>(A, derr);
  k_grad_reduce<<<(TR_NOUT + 127) / 128, 128, 0, t->stream>>>(t->partials, blocks, t->grad);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), t->grad, TR_NOUT * sizeof(double), cudaMemcpyDeviceToHost, t->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, t->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
  cudaFree(derr);
  if (e != cudaSuccess) return tfail(t, WT_E_CUDA, std::string("grad: ") + cudaGetErrorString(e));
  if (herr) return tfail(t, WT_E_CUDA, "grad: a tensor-core wait timed out");
  if (grad) {
    std::memset(grad, 0, sizeof *grad);
    float* gp = reinterpret_cast<float*>(reinterpret_cast<char*>(grad) + offsetof(wt_closure, w1));
    for (int p = 0; p < CL_NPARAM; p++) gp[p] = (float)(h[(size_t)p] / (double)n);
  }
  if (loss) *loss = h[CL_NPARAM] / (double)n;
  return WT_OK;
}

int wt_trainer_infer(wt_trainer* t, const float* x, int64_t n, float* nu) {
  if (!t || n < 0 || (n > 0 && (!x || !nu))) return WT_E_INVALID;
  if (!t->have_model) return tfail(t, WT_E_STATE, "wt_trainer_infer: no model set");
  if (n == 0) return WT_OK;
  TrDevice g(t->device);
  int rc = ensure_buf(t, &t->io, &t->io_floats, (size_t)n * (CL_IN + 1), "inference staging");
  if (rc) return rc;
  int* derr = nullptr;
  TR_CUDA(t, cudaMalloc((void**)&derr, sizeof(int)), "infer");
  cudaMemsetAsync(derr, 0, sizeof(int), t->stream);
  TrainArgs A = make_args(t);
  A.xs = t->io;
  A.ys = nullptr;
  A.offset = 0;
  A.rows = n;
  A.nu_out = t->io + (size_t)n * CL_IN;
  int herr = 0;
  cudaError_t e = cudaMemcpyAsync(t->io, x, (size_t)n * CL_IN * sizeof(float), cudaMemcpyHostToDevice, t->stream);
  if (e == cudaSuccess) {
    k_train<false><<<(unsigned)((n + TR_THREADS - 1) / TR_THREADS), TR_THREADS, TS_BYTES_INFER, t->stream>>>(A, derr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(nu, A.nu_out, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, t->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, t->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
  cudaFree(derr);
  if (e != cudaSuccess) return tfail(t, WT_E_CUDA, std::string("infer: ") + cudaGetErrorString(e));
  if (herr) return tfail(t, WT_E_CUDA, "infer: a tensor-core wait timed out");
  return WT_OK;
}

}  // extern "C"
