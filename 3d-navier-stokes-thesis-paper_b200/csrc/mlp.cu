// mlp.cu -- the learned subgrid-stress closure network (LES mode): BF16
// tensor-core forward (inference), forward + backward with per-batch gradient
// accumulation, and the Adam update, behind the cfg_mlp_* C ABI.  The
// operand layouts, descriptors and TMEM plan are described in mlp.cuh.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "chanflow.h"
#include "mlp.cuh"
#include "mlp_les.h"

using namespace cfd::mlp;

namespace {

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// layer geometry: rows of the weight image (output features, padded), input
// columns (padded) and the real sizes
struct LayerDim {
  int img, rows, kin, nreal, kreal, woff, boff;
};
__device__ __host__ constexpr LayerDim layer(int l) {
  return l == 0 ? LayerDim{IMG_W0, H, KIN, H, IN, OFF_W0, OFF_B0}
       : l == 1 ? LayerDim{IMG_W1, H, H, H, H, OFF_W1, OFF_B1}
       : l == 2 ? LayerDim{IMG_W2, H, H, H, H, OFF_W2, OFF_B2}
                : LayerDim{IMG_W3, NOUT, H, OUT, H, OFF_W3, OFF_B3};
}
// bias of layer l in the padded device bias vector: b0 b1 b2 (64 each), b3 (16)
__device__ __host__ constexpr int bias_base(int l) { return l * H; }
constexpr int NBIAS = 3 * H + NOUT;

// ------------------------------------------------------------- MMA issue
// forward product of layer l: D[128 x rows] = A[128 x kin] * W^T, K-major both
__device__ __forceinline__ void issue_forward(uint32_t d, uint32_t sA, uint32_t sW, int l) {
  const LayerDim L = layer(l);
  const uint32_t idesc = idesc_bf16(TILE, L.rows, 0, 0);
  for (int s = 0; s < L.kin / 16; ++s) {
    const uint64_t a = sdesc(sA + s * 2 * TILE * 16, TILE * 16, 128);
    const uint64_t b = sdesc(sW + (uint32_t)L.img * 16 + s * 2 * L.rows * 16, L.rows * 16, 128);
    mma_bf16(d, a, b, idesc, s > 0);
  }
}
// input gradient of layer l: D[128 x kin] = dZ[128 x rows] * W; dZ K-major,
// W read MN-major (N = kin columns, K = rows)
__device__ __forceinline__ void issue_dx(uint32_t d, uint32_t sDZ, uint32_t sW, int l) {
  const LayerDim L = layer(l);
  const uint32_t idesc = idesc_bf16(TILE, L.kin, 0, 1);
  for (int s = 0; s < L.rows / 16; ++s) {
    const uint64_t a = sdesc(sDZ + s * 2 * TILE * 16, TILE * 16, 128);
    const uint64_t b = sdesc(sW + (uint32_t)L.img * 16 + s * 256, 128, L.rows * 16);
    mma_bf16(d, a, b, idesc, s > 0);
  }
}
// weight gradient of layer l: D[128 (rows used) x kin] = dZ^T * X over the
// tile's 128 points; dZ and X both read MN-major
__device__ __forceinline__ void issue_dw(uint32_t d, uint32_t sDZ, uint32_t sX, int l) {
  const LayerDim L = layer(l);
  const uint32_t idesc = idesc_bf16(TILE, L.kin, 1, 1);
  for (int s = 0; s < TILE / 16; ++s) {
    const uint64_t a = sdesc(sDZ + s * 256, 128, TILE * 16);
    const uint64_t b = sdesc(sX + s * 256, 128, TILE * 16);
    mma_bf16(d, a, b, idesc, s > 0);
  }
}

// ------------------------------------------------------------- tile helpers
// this thread's point of the tile into X0 (10 features, BF16, padded to 16)
__device__ __forceinline__ void load_x0(uint4* sm, const float* __restrict__ x, long long row, bool valid, int p) {
  float v[KIN];
#pragma unroll
  for (int i = 0; i < KIN; ++i) v[i] = 0.f;
  if (valid) {
#pragma unroll
    for (int i = 0; i < IN; ++i) v[i] = __ldg(x + row * IN + i);
  }
  sm[Smem::X0 + unit_of(p, 0, TILE)] = pack8(v);
  sm[Smem::X0 + unit_of(p, 8, TILE)] = pack8(v + 8);
}

// GELU(Z + b) of 64 TMEM columns into activation tile dst (BF16)
__device__ __forceinline__ void gelu_to_tile(uint32_t taddr, const float* sb, uint4* dst, int p) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    float z[32];
    tmem_ld32(taddr + 32 * h, z);
#pragma unroll
    for (int i = 0; i < 32; i += 2) {
      const float2 g = gelu2(add2(make_float2(z[i], z[i + 1]), make_float2(sb[32 * h + i], sb[32 * h + i + 1])));
      z[i] = g.x;
      z[i + 1] = g.y;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) dst[unit_of(p, 32 * h + 8 * q, TILE)] = pack8(z + 8 * q);
  }
}

// the warp's sum over its 32 points of v (a fixed shuffle tree), stored to
// *dst by lane 0
__device__ __forceinline__ void warp_sum_to(float v, float* dst) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) *dst = v;
}

__device__ __forceinline__ void sync_for_mma() {
  fence_async_smem();
  fence_before_sync();
  __syncthreads();
}

// ------------------------------------------------------------- kernels
// the outputs of a point: stored as y[row][6]
struct PlainOut {
  float* y;
  __device__ __forceinline__ void operator()(long long row, bool valid, const float* v) const {
    if (valid) {
#pragma unroll
      for (int c = 0; c < OUT; ++c) y[row * OUT + c] = v[c];
    }
  }
};

// Inference: MLP(x[n][10]) of every point handed to out (PlainOut, or the
// LES blend), persistent over tiles of 128 points.  out is called by every
// lane (valid false past n).
template <class Out>
__global__ void __launch_bounds__(128) k_mlp_fwd(const uint4* __restrict__ img, const float* __restrict__ bias,
                                                 const float* __restrict__ x, Out out, long long n,
                                                 int* __restrict__ err) {
  extern __shared__ __align__(128) uint4 sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tslot;
  __shared__ float sb[NBIAS];
  const int p = threadIdx.x, warp = p >> 5;
  for (int i = p; i < IMG_UNITS; i += 128) sm[Smem::W + i] = img[i];
  for (int i = p; i < NBIAS; i += 128) sb[i] = bias[i];
  if (warp == 0) tmem_alloc(&tslot, TM_FWD_COLS);
  if (p == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tm = tslot, tlane = tm + ((uint32_t)(32 * warp) << 16);
  const uint32_t sbase = smem_u32(sm);
  const uint32_t sW = sbase + Smem::W * 16, sX = sbase + Smem::FWD_ACT * 16;
  uint32_t phase = 0;
  bool ok = true;
  const long long ntiles = (n + TILE - 1) / TILE;
  for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const long long row = tile * TILE + p;
    load_x0(sm, x, row, row < n, p);
    for (int l = 0; l < 4 && ok; ++l) {
      sync_for_mma();
      if (p == 0) {
        fence_after_sync();
        issue_forward(tm, sX, sW, l);
        mma_commit(&bar);
      }
      ok = __syncthreads_and(mbar_wait(&bar, phase));   // uniform across the block
      phase ^= 1;
      fence_after_sync();
      if (!ok) break;
      if (l < 3) {
        gelu_to_tile(tlane, sb + bias_base(l), sm + Smem::FWD_ACT, p);
      } else {
        float z[16];
        tmem_ld16(tlane, z);
#pragma unroll
        for (int c = 0; c < OUT; ++c) z[c] += sb[bias_base(3) + c];
        out(row, row < n, z);
      }
    }
    fence_before_sync();
    __syncthreads();
  }
  if (!ok && p == 0) atomicExch(err, 1);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0) tmem_dealloc(tm, TM_FWD_COLS);
}

// Training: one tile of the batch per CTA.  Forward with the pre-activations
// kept in TMEM, mean-square loss against t over the 6 outputs, backward, and
// the tile's weight and bias gradients (FP32, flat parameter layout) and its
// loss (at NPARAM) stored to its own slice part[blockIdx.x][PART_STRIDE]:
// every weight gradient by the one thread that holds it, every bias gradient
// and the loss as the sum of the four warps' sums in warp order, so that the
// slice does not depend on the order in which warps or tiles finish.
__global__ void __launch_bounds__(128, 1) k_mlp_train(const uint4* __restrict__ img, const float* __restrict__ bias,
                                                      const float* __restrict__ x, const float* __restrict__ t,
                                                      const int* __restrict__ idx, int batch,
                                                      float* __restrict__ part, int* __restrict__ err) {
  extern __shared__ __align__(128) uint4 sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tslot;
  __shared__ float sb[NBIAS];
  __shared__ float sg[4][H + 1];   // per-warp sums: bias gradients, the loss at H
  const int p = threadIdx.x, warp = p >> 5, lane = p & 31;
  for (int i = p; i < IMG_UNITS; i += 128) sm[Smem::W + i] = img[i];
  for (int i = p; i < NBIAS; i += 128) sb[i] = bias[i];
  for (int i = p; i < TILE * 128 / 8; i += 128) sm[Smem::DZ + i] = make_uint4(0, 0, 0, 0);
  if (warp == 0) tmem_alloc(&tslot, TM_TRAIN_COLS);
  if (p == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  float* const grad = part + (size_t)blockIdx.x * PART_STRIDE;
  const int r = blockIdx.x * TILE + p;
  const bool valid = r < batch;
  const long long row = valid ? (long long)idx[r] : 0;
  load_x0(sm, x, row, valid, p);
  sync_for_mma();
  fence_after_sync();
  const uint32_t tm = tslot, tlane = tm + ((uint32_t)(32 * warp) << 16);
  const uint32_t sbase = smem_u32(sm);
  const uint32_t sW = sbase + Smem::W * 16, sDZ = sbase + Smem::DZ * 16;
  const uint32_t sX[4] = {sbase + Smem::X0 * 16, sbase + Smem::X1 * 16, sbase + Smem::X2 * 16,
                          sbase + Smem::X3 * 16};
  const int xu[4] = {Smem::X0, Smem::X1, Smem::X2, Smem::X3};
  const uint32_t tz[4] = {TM_Z0, TM_Z1, TM_Z2, TM_Z3};
  uint32_t phase = 0;
  bool ok = true;
  // forward
  for (int l = 0; l < 4 && ok; ++l) {
    if (p == 0) {
      fence_after_sync();
      issue_forward(tm + tz[l], sX[l], sW, l);
      mma_commit(&bar);
    }
    ok = __syncthreads_and(mbar_wait(&bar, phase));   // uniform across the block
    phase ^= 1;
    fence_after_sync();
    if (ok && l < 3) {
      gelu_to_tile(tlane + tz[l], sb + bias_base(l), sm + xu[l + 1], p);
      sync_for_mma();
    }
  }
  // output layer: loss and dL/dZ3
  if (ok) {
    float z[16], dz[16];
    tmem_ld16(tlane + TM_Z3, z);
    float lsum = 0.f;
    const float sc = 2.0f / (6.0f * (float)batch);
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      dz[c] = 0.f;
      if (c < OUT && valid) {
        const float d = z[c] + sb[bias_base(3) + c] - __ldg(t + row * OUT + c);
        lsum += d * d;
        dz[c] = sc * d;
      }
    }
    sm[Smem::DZ + unit_of(p, 0, TILE)] = pack8(dz);
    sm[Smem::DZ + unit_of(p, 8, TILE)] = pack8(dz + 8);
#pragma unroll
    for (int c = 0; c < OUT; ++c) warp_sum_to(dz[c], &sg[warp][c]);
    warp_sum_to(lsum / (6.0f * (float)batch), &sg[warp][H]);
    sync_for_mma();
    if (p < OUT) grad[OFF_B3 + p] = sg[0][p] + sg[1][p] + sg[2][p] + sg[3][p];
    if (p == TILE - 1) grad[NPARAM] = sg[0][H] + sg[1][H] + sg[2][H] + sg[3][H];
  }
  // backward through layers 3, 2, 1 (weight and input gradients), then the
  // weight gradient of layer 0
  for (int l = 3; l >= 0 && ok; --l) {
    const LayerDim L = layer(l);
    if (p == 0) {
      fence_after_sync();
      issue_dw(tm + TM_DW, sDZ, sX[l], l);
      if (l > 0) issue_dx(tm + TM_DX, sDZ, sW, l);
      mma_commit(&bar);
    }
    ok = __syncthreads_and(mbar_wait(&bar, phase));   // uniform across the block
    phase ^= 1;
    fence_after_sync();
    if (!ok) break;
    // weight gradient rows n (TMEM lane n) of the real outputs
    if (32 * warp < L.nreal) {
      const int n = 32 * warp + lane;
      if (L.kin == 16) {
        float v[16];
        tmem_ld16(tlane + TM_DW, v);
        if (n < L.nreal)
          for (int k = 0; k < L.kreal; ++k) grad[L.woff + n * L.kreal + k] = v[k];
      } else {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float v[32];
          tmem_ld32(tlane + TM_DW + 32 * h, v);
          if (n < L.nreal)
#pragma unroll
            for (int k = 0; k < 32; ++k) grad[L.woff + n * L.kreal + 32 * h + k] = v[k];
        }
      }
    }
    if (l > 0) {
      // dZ_{l-1} = (dZ_l W_l) * GELU'(Z_{l-1} + b_{l-1}), 64 columns
      const int lp = l - 1;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        float dx[32], z[32];
        tmem_ld32(tlane + TM_DX + 32 * h, dx);
        tmem_ld32(tlane + tz[lp] + 32 * h, z);
#pragma unroll
        for (int i = 0; i < 32; ++i) dx[i] = valid ? dx[i] * gelu_d(z[i] + sb[bias_base(lp) + 32 * h + i]) : 0.f;
#pragma unroll
        for (int q = 0; q < 4; ++q) sm[Smem::DZ + unit_of(p, 32 * h + 8 * q, TILE)] = pack8(dx + 8 * q);
#pragma unroll
        for (int i = 0; i < 32; ++i) warp_sum_to(dx[i], &sg[warp][32 * h + i]);
      }
    }
    sync_for_mma();
    // the bias gradient of layer l - 1 (sg is next written after the next
    // product's barrier)
    if (l > 0 && p < H) grad[layer(l - 1).boff + p] = sg[0][p] + sg[1][p] + sg[2][p] + sg[3][p];
  }
  if (!ok && p == 0) atomicExch(err, 1);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0) tmem_dealloc(tm, TM_TRAIN_COLS);
}

// the batch's tile slices summed in tile order into the gradient and the loss
// accumulators (the same sums, bit for bit, on every run)
__global__ void k_mlp_reduce(const float* __restrict__ part, int ntiles, float* __restrict__ G,
                             float* __restrict__ loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > NPARAM) return;
  float s = 0.f;
  for (int b = 0; b < ntiles; ++b) s += part[(size_t)b * PART_STRIDE + i];
  if (i < NPARAM) G[i] += s;
  else *loss += s;
}

// weight images and padded biases from the FP32 parameter vector
__device__ __forceinline__ void pack_param(int i, float v, __nv_bfloat16* img, float* bias) {
  for (int l = 0; l < 4; ++l) {
    const LayerDim L = layer(l);
    if (i >= L.woff && i < L.woff + L.nreal * L.kreal) {
      const int n = (i - L.woff) / L.kreal, k = (i - L.woff) % L.kreal;
      img[((size_t)L.img + unit_of(n, k, L.rows)) * 8 + (k & 7)] = __float2bfloat16_rn(v);
      return;
    }
    if (i >= L.boff && i < L.boff + L.nreal) {
      bias[bias_base(l) + i - L.boff] = v;
      return;
    }
  }
}

__global__ void k_mlp_pack(const float* __restrict__ P, __nv_bfloat16* img, float* bias) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NPARAM; i += gridDim.x * blockDim.x) pack_param(i, P[i], img, bias);
}

// Adam (Kingma & Ba 2015) with bias correction; the gradient is zeroed and
// the BF16 images rewritten
__global__ void k_mlp_adam(float* P, float* G, float* M, float* V, float lr, float b1, float b2, float eps,
                           float c1, float c2, __nv_bfloat16* img, float* bias, float* loss) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NPARAM; i += gridDim.x * blockDim.x) {
    const float g = G[i];
    const float m = b1 * M[i] + (1.f - b1) * g, v = b2 * V[i] + (1.f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    const float p = P[i] - lr * (m / c1) / (sqrtf(v / c2) + eps);
    P[i] = p;
    G[i] = 0.f;
    pack_param(i, p, img, bias);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *loss = 0.f;
}

}  // namespace

struct cfg_mlp {
  int dev = 0;
  float* P = nullptr;   // [NPARAM] FP32 master parameters
  float* G = nullptr;   // [NPARAM] accumulated gradient
  float* M = nullptr;   // Adam moments
  float* V = nullptr;
  float* loss = nullptr;
  int* err = nullptr;
  uint4* img = nullptr;   // [IMG_UNITS] BF16 weight images
  float* bias = nullptr;  // [NBIAS]
  float* part = nullptr;  // [part_tiles][PART_STRIDE] per-tile gradients of a batch
  int part_tiles = 0;
  long long step = 0;
  int nsm = 148;
};

namespace {
constexpr size_t SMEM_FWD = (size_t)Smem::END_FWD * 16;
constexpr size_t SMEM_TRAIN = 120 * 1024;   // >= END_TRAIN*16; one CTA per SM (512 TMEM columns)
constexpr int PART_TILES0 = 512;             // per-tile gradient slices held from creation (batch 65536)
static_assert((size_t)Smem::END_TRAIN * 16 <= SMEM_TRAIN, "training tile plan exceeds its shared memory");
}

extern "C" {

int cfg_mlp_nparams(void) { return NPARAM; }

int cfg_mlp_create(int device, cfg_mlp** out) {
  if (!out) return CFG_E_ARG;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return CFG_E_CUDA;
  int cc = 0;
  cudaDeviceGetAttribute(&cc, cudaDevAttrComputeCapabilityMajor, device);
  if (cc != 10) return CFG_E_ARG;   // tcgen05 needs sm_100
  cfg_mlp* m = new cfg_mlp;
  m->dev = device;
  cudaDeviceGetAttribute(&m->nsm, cudaDevAttrMultiProcessorCount, device);
  bool ok = cudaMalloc(&m->P, 4 * NPARAM * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&m->loss, sizeof(float) + sizeof(int)) == cudaSuccess &&
            cudaMalloc(&m->img, IMG_UNITS * sizeof(uint4)) == cudaSuccess &&
            cudaMalloc(&m->bias, NBIAS * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&m->part, (size_t)PART_TILES0 * PART_STRIDE * sizeof(float)) == cudaSuccess;
  if (ok) m->part_tiles = PART_TILES0;
  if (!ok) {
    cfg_mlp_destroy(m);
    return CFG_E_NOMEM;
  }
  m->G = m->P + NPARAM;
  m->M = m->G + NPARAM;
  m->V = m->M + NPARAM;
  m->err = reinterpret_cast<int*>(m->loss + 1);
  cudaMemset(m->P, 0, 4 * NPARAM * sizeof(float));
  cudaMemset(m->loss, 0, sizeof(float) + sizeof(int));
  cudaMemset(m->img, 0, IMG_UNITS * sizeof(uint4));   // the padding stays zero
  cudaMemset(m->bias, 0, NBIAS * sizeof(float));
  if (cudaFuncSetAttribute(k_mlp_fwd<PlainOut>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_FWD) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_mlp_fwd<cfd::LesBlend<float>>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)SMEM_FWD) != cudaSuccess ||
      cudaFuncSetAttribute(k_mlp_fwd<cfd::LesBlend<double>>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)SMEM_FWD) != cudaSuccess ||
      cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_TRAIN) != cudaSuccess ||
      // the whole of the SM's on-chip memory as shared memory: six forward
      // CTAs per SM
      cudaFuncSetAttribute(k_mlp_fwd<PlainOut>, cudaFuncAttributePreferredSharedMemoryCarveout,
                           (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess ||
      cudaFuncSetAttribute(k_mlp_fwd<cfd::LesBlend<float>>, cudaFuncAttributePreferredSharedMemoryCarveout,
                           (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess ||
      cudaFuncSetAttribute(k_mlp_fwd<cfd::LesBlend<double>>, cudaFuncAttributePreferredSharedMemoryCarveout,
                           (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess ||
      cudaDeviceSynchronize() != cudaSuccess) {
    cfg_mlp_destroy(m);
    return CFG_E_CUDA;
  }
  *out = m;
  return CFG_OK;
}

void cfg_mlp_destroy(cfg_mlp* m) {
  if (!m) return;
  cudaSetDevice(m->dev);
  cudaFree(m->P);
  cudaFree(m->loss);
  cudaFree(m->img);
  cudaFree(m->bias);
  cudaFree(m->part);
  delete m;
}

int cfg_mlp_set_params(cfg_mlp* m, const float* params) {
  if (!m || !params) return CFG_E_ARG;
  cudaSetDevice(m->dev);
  if (cudaMemcpy(m->P, params, NPARAM * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) return CFG_E_CUDA;
  cudaMemset(m->G, 0, 3 * NPARAM * sizeof(float));   // gradient and Adam moments restart
  m->step = 0;
  k_mlp_pack<<<(NPARAM + 255) / 256, 256>>>(m->P, reinterpret_cast<__nv_bfloat16*>(m->img), m->bias);
  return cudaDeviceSynchronize() == cudaSuccess ? CFG_OK : CFG_E_CUDA;
}

int cfg_mlp_get_params(cfg_mlp* m, float* params) {
  if (!m || !params) return CFG_E_ARG;
  cudaSetDevice(m->dev);
  return cudaMemcpy(params, m->P, NPARAM * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess ? CFG_OK
                                                                                                  : CFG_E_CUDA;
}

int cfg_mlp_forward(cfg_mlp* m, const float* x, float* y, long long n, void* stream) {
  if (!m || n < 0 || (n > 0 && (!x || !y))) return CFG_E_ARG;
  if (n == 0) return CFG_OK;
  cudaSetDevice(m->dev);
  const long long ntiles = (n + TILE - 1) / TILE;
  // persistent: six CTAs per SM, as many as the shared memory holds (TMEM
  // would hold eight); a grid past what is resident leaves a second,
  // partial wave (measured 2.5x slower)
  const int grid = (int)(ntiles < 6LL * m->nsm ? ntiles : 6LL * m->nsm);
  k_mlp_fwd<PlainOut><<<grid, 128, SMEM_FWD, (cudaStream_t)stream>>>(m->img, m->bias, x, PlainOut{y}, n, m->err);
  return cudaGetLastError() == cudaSuccess ? CFG_OK : CFG_E_CUDA;
}

int cfg_mlp_accumulate_grad(cfg_mlp* m, const float* x, const float* t, const int* idx, int batch, void* stream) {
  if (!m || !x || !t || !idx || batch <= 0) return CFG_E_ARG;
  cudaSetDevice(m->dev);
  const int ntiles = (batch + TILE - 1) / TILE;
  if (ntiles > m->part_tiles) {
    // a larger batch than any before: the slices grow (cudaFree waits for
    // the kernels still reading the old ones)
    cudaFree(m->part);
    m->part = nullptr;
    m->part_tiles = 0;
    if (cudaMalloc(&m->part, (size_t)ntiles * PART_STRIDE * sizeof(float)) != cudaSuccess) return CFG_E_NOMEM;
    m->part_tiles = ntiles;
  }
  k_mlp_train<<<ntiles, 128, SMEM_TRAIN, (cudaStream_t)stream>>>(m->img, m->bias, x, t, idx, batch, m->part, m->err);
  k_mlp_reduce<<<(NPARAM + 1 + 255) / 256, 256, 0, (cudaStream_t)stream>>>(m->part, ntiles, m->G, m->loss);
  return cudaGetLastError() == cudaSuccess ? CFG_OK : CFG_E_CUDA;
}

int cfg_mlp_get_grads(cfg_mlp* m, float* grads, float* loss) {
  if (!m) return CFG_E_ARG;
  cudaSetDevice(m->dev);
  if (cudaDeviceSynchronize() != cudaSuccess) return CFG_E_CUDA;
  if (grads && cudaMemcpy(grads, m->G, NPARAM * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
    return CFG_E_CUDA;
  if (loss && cudaMemcpy(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) return CFG_E_CUDA;
  return CFG_OK;
}

int cfg_mlp_zero_grads(cfg_mlp* m, void* stream) {
  if (!m) return CFG_E_ARG;
  cudaSetDevice(m->dev);
  cudaMemsetAsync(m->G, 0, NPARAM * sizeof(float), (cudaStream_t)stream);
  cudaMemsetAsync(m->loss, 0, sizeof(float), (cudaStream_t)stream);
  return cudaGetLastError() == cudaSuccess ? CFG_OK : CFG_E_CUDA;
}

int cfg_mlp_adam_step(cfg_mlp* m, float lr, float beta1, float beta2, float eps, void* stream) {
  if (!m || !(lr >= 0.f)) return CFG_E_ARG;
  cudaSetDevice(m->dev);
  m->step += 1;
  const float c1 = 1.f - powf(beta1, (float)m->step), c2 = 1.f - powf(beta2, (float)m->step);
  k_mlp_adam<<<(NPARAM + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
      m->P, m->G, m->M, m->V, lr, beta1, beta2, eps, c1, c2, reinterpret_cast<__nv_bfloat16*>(m->img), m->bias,
      m->loss);
  return cudaGetLastError() == cudaSuccess ? CFG_OK : CFG_E_CUDA;
}

int cfg_mlp_status(cfg_mlp* m) {
  if (!m) return CFG_E_ARG;
  cudaSetDevice(m->dev);
  int e = 0;
  if (cudaMemcpy(&e, m->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return CFG_E_CUDA;
  return e ? CFG_E_STATE : CFG_OK;
}

}  // extern "C"

namespace cfd {
template <typename T>
int mlp_forward_blend(cfg_mlp* m, long long n, const LesBlend<T>& b, void* stream) {
  if (!m || n < 0 || (n > 0 && (!b.F || !b.S || !b.len || !b.nfall))) return CFG_E_ARG;
  if (n == 0) return CFG_OK;
  cudaSetDevice(m->dev);
  const long long ntiles = (n + TILE - 1) / TILE;
  const int grid = (int)(ntiles < 6LL * m->nsm ? ntiles : 6LL * m->nsm);
  k_mlp_fwd<LesBlend<T>><<<grid, 128, SMEM_FWD, (cudaStream_t)stream>>>(m->img, m->bias, b.F, b, n, m->err);
  return cudaGetLastError() == cudaSuccess ? CFG_OK : CFG_E_CUDA;
}
template int mlp_forward_blend<float>(cfg_mlp*, long long, const LesBlend<float>&, void*);
template int mlp_forward_blend<double>(cfg_mlp*, long long, const LesBlend<double>&, void*);
}  // namespace cfd
