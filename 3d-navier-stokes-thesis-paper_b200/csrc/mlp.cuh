// mlp.cuh -- the learned subgrid-stress closure's network on the 5th-generation
// tensor cores (sm_100a tcgen05): a 10 -> 64 -> 64 -> 64 -> 6 perceptron with
// GELU (tanh form) on the three hidden layers, BF16 weights and activations, FP32
// accumulation in tensor memory (TMEM).
//
// One CTA of 128 threads (4 warps) handles a tile of 128 points: thread t owns
// point t of the tile and TMEM lane t.  Every product is one tcgen05.mma
// (kind::f16, M = 128, K = 16 per instruction) issued by thread 0, with both
// operands in shared memory and the accumulator in TMEM; its completion is
// signalled by tcgen05.commit on an mbarrier, after which the warps read their
// 32 TMEM lanes with tcgen05.ld.
//
// Shared-memory operand layout (no swizzle).  A matrix of R rows x K columns
// (BF16) is stored as 16-byte units of 8 consecutive columns of one row:
//   unit(r, c) = (c * R/8 + r/8) * 8 + r%8,  c = col/8, element col%8 in it.
// Read with a K-major descriptor (rows = M or N, columns = K) the 8-row groups
// are 128 B apart (SBO) and the column groups R*16 B apart (LBO).  The same
// buffer read with an MN-major descriptor (columns = M or N, rows = K) has
// SBO = R*16 B (column groups) and LBO = 128 B (row groups).  So activations
// (points x features) serve as the A operand of the forward product and as the
// B operand of the weight gradient, and the gradient tiles as the A operand of
// both backward products, without transposed copies.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cfd {
namespace mlp {

constexpr int IN = 10, H = 64, OUT = 6;
constexpr int KIN = 16;    // input features padded to one MMA K step
constexpr int NOUT = 16;   // output rows padded to the smallest M=128 N
constexpr int TILE = 128;  // points per CTA tile (MMA M)
// flat FP32 parameter vector: W0[H][IN] b0[H] W1[H][H] b1[H] W2[H][H] b2[H] W3[OUT][H] b3[OUT]
constexpr int OFF_W0 = 0, OFF_B0 = OFF_W0 + H * IN, OFF_W1 = OFF_B0 + H, OFF_B1 = OFF_W1 + H * H,
              OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H, OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + OUT * H,
              NPARAM = OFF_B3 + OUT;
// one training tile's gradient slice: the NPARAM gradients and the loss,
// padded to 16 bytes
constexpr int PART_STRIDE = (NPARAM + 1 + 3) / 4 * 4;
// BF16 operand images of the weights (units of 16 B, the layout above with
// rows = output features): W0 64x16, W1 64x64, W2 64x64, W3 16x64
constexpr int IMG_W0 = 0, IMG_W1 = IMG_W0 + H * KIN / 8, IMG_W2 = IMG_W1 + H * H / 8,
              IMG_W3 = IMG_W2 + H * H / 8, IMG_UNITS = IMG_W3 + NOUT * H / 8;

__host__ __device__ constexpr int unit_of(int r, int col, int R) { return ((col >> 3) * (R >> 3) + (r >> 3)) * 8 + (r & 7); }

// ---------------------------------------------------------------- PTX wrappers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, no swizzle, sm_100 version field
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor, kind::f16: BF16 A and B, FP32 D, dense
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, int accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// bounded wait for the mbarrier phase `parity` to complete: false after the
// iteration limit (the caller records an error and leaves)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (int it = 0; it < (1 << 22); ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 consecutive FP32 columns of this warp's 32 TMEM lanes: thread i of the
// warp receives lane (32*warp + i); taddr carries the lane base in bits 16..31
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ---------------------------------------------------------------- activation
// GELU in its tanh form (Hendrycks & Gimpel 2016):
//   g(z) = z (1 + t) / 2,  t = tanh(c (z + a z^3)),  c = sqrt(2/pi), a = 0.044715,
//   g'(z) = (1 + t) / 2 + z (1 - t^2) c (1 + 3 a z^2) / 2,
// with the hardware tanh approximation (tanh.approx.f32, relative error below
// 2^-10, under the BF16 rounding the activations get next)
__device__ __forceinline__ float tanh_hw(float u) {
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
  return t;
}
constexpr float kGeluC = 0.7978845608028654f, kGeluA = 0.044715f, kGeluCA = kGeluC * kGeluA;
// the tanh argument c (z + a z^3) = z (c + c a z^2)
__device__ __forceinline__ float gelu_arg(float z) { return z * fmaf(z * z, kGeluCA, kGeluC); }
__device__ __forceinline__ float gelu(float z) {
  const float h = 0.5f * z;
  return fmaf(h, tanh_hw(gelu_arg(z)), h);
}
__device__ __forceinline__ float gelu_d(float z) {
  const float z2 = z * z;
  const float t = tanh_hw(gelu_arg(z));
  return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * kGeluC * fmaf(3.0f * kGeluA, z2, 1.0f);
}

// two lanes per instruction (add/mul/fma.rn.f32x2, sm_100): the same IEEE
// results as the scalar operations
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
  float2 r;
  asm("{.reg .b64 pa, pb, pr;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "add.rn.f32x2 pr, pa, pb;\n\tmov.b64 {%0, %1}, pr;}"
      : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
  float2 r;
  asm("{.reg .b64 pa, pb, pr;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "mul.rn.f32x2 pr, pa, pb;\n\tmov.b64 {%0, %1}, pr;}"
      : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  float2 r;
  asm("{.reg .b64 pa, pb, pc, pr;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "mov.b64 pc, {%6, %7};\n\tfma.rn.f32x2 pr, pa, pb, pc;\n\tmov.b64 {%0, %1}, pr;}"
      : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return r;
}
// gelu of two values, the arithmetic of gelu() two lanes at a time
__device__ __forceinline__ float2 gelu2(float2 z) {
  const float2 w = fma2(mul2(z, z), make_float2(kGeluCA, kGeluCA), make_float2(kGeluC, kGeluC));
  const float2 u = mul2(z, w);
  const float2 h = mul2(z, make_float2(0.5f, 0.5f));
  return fma2(h, make_float2(tanh_hw(u.x), tanh_hw(u.y)), h);
}

// 8 BF16 values as one 16-byte unit
__device__ __forceinline__ uint4 pack8(const float* v) {
  uint4 u;
  __nv_bfloat162 h;
  h = __floats2bfloat162_rn(v[0], v[1]); u.x = *reinterpret_cast<uint32_t*>(&h);
  h = __floats2bfloat162_rn(v[2], v[3]); u.y = *reinterpret_cast<uint32_t*>(&h);
  h = __floats2bfloat162_rn(v[4], v[5]); u.z = *reinterpret_cast<uint32_t*>(&h);
  h = __floats2bfloat162_rn(v[6], v[7]); u.w = *reinterpret_cast<uint32_t*>(&h);
  return u;
}

// shared-memory plan of a tile kernel (offsets in 16-byte units)
struct Smem {
  static constexpr int W = 0;                               // weight images, IMG_UNITS
  static constexpr int X0 = W + IMG_UNITS;                  // 128 x 16
  static constexpr int X1 = X0 + TILE * KIN / 8;            // 128 x 64
  static constexpr int X2 = X1 + TILE * H / 8;
  static constexpr int X3 = X2 + TILE * H / 8;
  static constexpr int DZ = X3 + TILE * H / 8;              // 128 x 128 gradient tile (upper half zero)
  // inference: the input tile and the activation tile share one buffer at
  // X0 (a layer's product has completed before its epilogue overwrites its
  // input), so that six CTAs fit on an SM
  static constexpr int FWD_ACT = X0;
  static constexpr int END_FWD = FWD_ACT + TILE * H / 8;
  static constexpr int END_TRAIN = DZ + TILE * 128 / 8;
};

// TMEM columns of the training kernel (pre-activations kept for the backward
// pass, then the two backward accumulators)
constexpr uint32_t TM_Z0 = 0, TM_Z1 = 64, TM_Z2 = 128, TM_Z3 = 192, TM_DX = 256, TM_DW = 320, TM_TRAIN_COLS = 512;
constexpr uint32_t TM_FWD_COLS = 64;

}  // namespace mlp
}  // namespace cfd
