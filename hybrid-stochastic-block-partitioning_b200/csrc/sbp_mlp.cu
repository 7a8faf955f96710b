// Tensor-core kernels of the learned proposal's network (64 -> 128 -> 128 -> 16).
//
// Every GEMM is one tcgen05.mma chain D[128 x N] (+)= A[128 x K] * B[N x K]^T with A and B
// BF16 in shared memory, K-major, in the canonical no-swizzle layout (8 x 8 core matrices
// of 128 contiguous bytes; core matrices adjacent in K 128 bytes apart, 8-row groups K*16
// bytes apart), the FP32 accumulator D in tensor memory (TMEM lane = row).  One thread
// issues the MMAs and commits them to an mbarrier; the CTA waits on the mbarrier with an
// iteration limit and reads D back with tcgen05.ld (thread t of the 128 owns row t).
//
// Training keeps every GEMM K-major by having the epilogues also write the transposed
// tiles (features x vertices) that the weight-gradient GEMMs read as operands.
#include <cuda_bf16.h>

#include "sbp_mlp.cuh"

namespace sbpb {
namespace {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (row, k) of a [rows][K] BF16 tile in the canonical K-major layout.
__host__ __device__ __forceinline__ uint32_t kmaj(int row, int k, int K) {
  return (uint32_t)((row >> 3) * (K * 16) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor: start address, LBO = 128 B (K direction), SBO = K*16 B
// (8-row groups), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, int K) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) |
         ((uint64_t)(((uint32_t)K * 16u >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: D FP32, A and B BF16, both K-major, shape M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// D[128 x N] (+)= A[128 x K] * B[N x K]^T, K a multiple of 16 (one MMA per 16 of K).
__device__ __forceinline__ void gemm(uint32_t d_tmem, uint32_t a, uint32_t b, int N, int K, bool acc_first) {
  const uint32_t id = idesc_bf16(128, N);
  for (int s = 0; s < K / 16; ++s)
    umma(d_tmem, umma_desc(a + 256u * s, K), umma_desc(b + 256u * s, K), id, (s > 0 || acc_first) ? 1u : 0u);
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(1u) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the phase with the given parity; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (uint32_t it = 0; it < (1u << 22); ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\tselp.b32 %0, 1, 0, P;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void async_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
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

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 p = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&p);
}

__device__ __forceinline__ float bf16_at(const unsigned char* tile, uint32_t off) {
  return __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(tile + off));
}

__device__ __forceinline__ void put_bf16(unsigned char* tile, uint32_t off, float x) {
  *reinterpret_cast<__nv_bfloat16*>(tile + off) = __float2bfloat16_rn(x);
}

// Weight tile [rows][K] from a row-major BF16 matrix into the canonical layout (16-byte chunks).
__device__ __forceinline__ void load_kmajor(unsigned char* dst, const __nv_bfloat16* src, int rows, int K) {
  const int chunks = rows * (K / 8);
  for (int c = threadIdx.x; c < chunks; c += blockDim.x) {
    const int r = c / (K / 8), kc = (c % (K / 8)) * 8;
    *reinterpret_cast<uint4*>(dst + kmaj(r, kc, K)) = *reinterpret_cast<const uint4*>(src + (size_t)r * K + kc);
  }
}

// Transposed weight tile: dst[N = cols][K = rows] from a row-major [rows][cols] matrix.
__device__ __forceinline__ void load_transposed(unsigned char* dst, const __nv_bfloat16* src, int rows, int cols) {
  for (int i = threadIdx.x; i < rows * cols; i += blockDim.x) {
    const int r = i / cols, c = i % cols;
    *reinterpret_cast<__nv_bfloat16*>(dst + kmaj(c, r, rows)) = src[i];
  }
}

// ReLU(D + bias) of this thread's row -> BF16 row `row` of H (K = 128) and, when HT is given,
// column `row` of HT (rows = hidden units, K = 128 vertices).
__device__ __forceinline__ void epilogue_relu(uint32_t taddr, const float* bias, unsigned char* H, unsigned char* HT,
                                              int row) {
  for (int c0 = 0; c0 < kMlpHid; c0 += 16) {
    float v[16];
    tmem_ld16(taddr + c0, v);
    uint32_t p[8];
#pragma unroll
    for (int j = 0; j < 8; ++j)
      p[j] = pack_bf16(fmaxf(v[2 * j] + bias[c0 + 2 * j], 0.f), fmaxf(v[2 * j + 1] + bias[c0 + 2 * j + 1], 0.f));
    *reinterpret_cast<uint4*>(H + kmaj(row, c0, kMlpHid)) = make_uint4(p[0], p[1], p[2], p[3]);
    *reinterpret_cast<uint4*>(H + kmaj(row, c0 + 8, kMlpHid)) = make_uint4(p[4], p[5], p[6], p[7]);
    if (HT) {
      const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(p);
#pragma unroll
      for (int j = 0; j < 16; ++j)
        *reinterpret_cast<__nv_bfloat16*>(HT + kmaj(c0 + j, row, kMlpTile)) = e[j];
    }
  }
}

// ------------------------------------------------------------------------------------------
// Inference: persistent CTAs of 128 threads over 128-row tiles.
// Shared memory: X 16K | W1 16K | W2 32K | W3 4K | H1 32K | H2 32K | biases | mbarrier | TMEM slot
// TMEM columns: D1 [0,128) D2 [128,256) D3 [256,272) (512 allocated; one CTA per SM).
// ------------------------------------------------------------------------------------------
constexpr int kFwdX = 0, kFwdW1 = 16384, kFwdW2 = 32768, kFwdW3 = 65536, kFwdH1 = 69632, kFwdH2 = 102400,
              kFwdBias = 135168, kFwdBar = kFwdBias + 272 * 4, kFwdSlot = kFwdBar + 8, kFwdSmem = kFwdSlot + 8;

__global__ void __launch_bounds__(128, 1)
    k_mlp_forward(const __nv_bfloat16* __restrict__ X, long long n, MlpWeights w, float* __restrict__ logits,
                  int* status) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int tid = threadIdx.x, warp = tid >> 5;
  float* sb = reinterpret_cast<float*>(sm + kFwdBias);
  const uint32_t bar = smem_u32(sm + kFwdBar);
  load_kmajor(sm + kFwdW1, w.W1, kMlpHid, kMlpIn);
  load_kmajor(sm + kFwdW2, w.W2, kMlpHid, kMlpHid);
  load_kmajor(sm + kFwdW3, w.W3, kMlpOut, kMlpHid);
  for (int i = tid; i < 272; i += blockDim.x) sb[i] = i < 128 ? w.b1[i] : i < 256 ? w.b2[i - 128] : w.b3[i - 256];
  if (tid == 0) mbar_init(bar);
  if (warp == 0) tmem_alloc(smem_u32(sm + kFwdSlot), 512);
  tc_before();
  __syncthreads();
  tc_after();
  const uint32_t tm = *reinterpret_cast<volatile uint32_t*>(sm + kFwdSlot);
  const uint32_t lane_off = (uint32_t)(warp * 32) << 16;
  uint32_t phase = 0;
  int ok = 1;
  const long long tiles = (n + kMlpTile - 1) / kMlpTile;
  for (long long tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    const long long row0 = tile * kMlpTile;
    for (int c = tid; c < kMlpTile * 8; c += blockDim.x) {
      const int r = c >> 3, kc = (c & 7) * 8;
      const long long gr = row0 + r;
      const uint4 val = gr < n ? *reinterpret_cast<const uint4*>(X + gr * kMlpIn + kc) : make_uint4(0, 0, 0, 0);
      *reinterpret_cast<uint4*>(sm + kFwdX + kmaj(r, kc, kMlpIn)) = val;
    }
    async_fence();
    tc_before();
    __syncthreads();
    if (tid == 0) {
      tc_after();
      gemm(tm + 0, smem_u32(sm + kFwdX), smem_u32(sm + kFwdW1), kMlpHid, kMlpIn, false);
      umma_commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase));
    phase ^= 1;
    if (!ok) break;
    tc_after();
    epilogue_relu(tm + lane_off + 0, sb, sm + kFwdH1, nullptr, tid);
    async_fence();
    tc_before();
    __syncthreads();
    if (tid == 0) {
      tc_after();
      gemm(tm + 128, smem_u32(sm + kFwdH1), smem_u32(sm + kFwdW2), kMlpHid, kMlpHid, false);
      umma_commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase));
    phase ^= 1;
    if (!ok) break;
    tc_after();
    epilogue_relu(tm + lane_off + 128, sb + 128, sm + kFwdH2, nullptr, tid);
    async_fence();
    tc_before();
    __syncthreads();
    if (tid == 0) {
      tc_after();
      gemm(tm + 256, smem_u32(sm + kFwdH2), smem_u32(sm + kFwdW3), kMlpOut, kMlpHid, false);
      umma_commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase));
    phase ^= 1;
    if (!ok) break;
    tc_after();
    float v[16];
    tmem_ld16(tm + lane_off + 256, v);
    const long long gr = row0 + tid;
    if (gr < n) {
      float4* o = reinterpret_cast<float4*>(logits + gr * kMlpOut);
#pragma unroll
      for (int q = 0; q < 4; ++q)
        o[q] = make_float4(v[4 * q] + sb[256 + 4 * q], v[4 * q + 1] + sb[257 + 4 * q], v[4 * q + 2] + sb[258 + 4 * q],
                           v[4 * q + 3] + sb[259 + 4 * q]);
    }
    tc_before();
    __syncthreads();
  }
  if (!ok) {
    if (tid == 0) atomicOr(status, kErrTensorWait);
    mbar_wait(bar, phase ^ 1);   // the phase that gave up: let an MMA still in flight finish
  }
  tc_before();
  __syncthreads();
  if (warp == 0) {
    tc_after();
    tmem_dealloc(tm, 512);
  }
}

// ------------------------------------------------------------------------------------------
// Training: one 128-row tile per CTA, forward and backward, weight gradients accumulated
// atomically in global FP32.  Shared memory (bytes):
//   X 0 (later dZ3 at 0 and dZ3T at 4096) | XT 16384 | W1 32768 | W2 49152 (later W2T)
//   W3 81920 | W3T 86016 | H1 90112 (later dZ2) | H1T 122880 (later dZ1T) | H2 155648
//   H2T 188416 (later dZ2T) | biases 221184 | bias-gradient sums 222272 | loss 223360 |
//   mbarrier 223392 | TMEM slot 223400
// TMEM columns: D1/dH2 [0,128) D2/dH1 [128,256) D3 [256,272) dW3^T [288,304) dW2 [320,448)
// dW1 [448,512).
// ------------------------------------------------------------------------------------------
constexpr int kTrX = 0, kTrZ3 = 0, kTrZ3T = 4096, kTrXT = 16384, kTrW1 = 32768, kTrW2 = 49152, kTrW3 = 81920,
              kTrW3T = 86016, kTrH1 = 90112, kTrH1T = 122880, kTrH2 = 155648, kTrH2T = 188416, kTrBias = 221184,
              kTrGb = kTrBias + 272 * 4, kTrLoss = kTrGb + 272 * 4, kTrBar = kTrLoss + 32, kTrSlot = kTrBar + 8,
              kTrSmem = kTrSlot + 8;

__device__ __forceinline__ float warp_sum_f(float x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

__global__ void __launch_bounds__(128, 1)
    k_mlp_train_tile(const __nv_bfloat16* __restrict__ X, const int* __restrict__ target,
                     const int* __restrict__ nvalid, long long n, float inv_count, MlpWeights w,
                     float* __restrict__ grads, double* loss_sum, int* status) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  float* sb = reinterpret_cast<float*>(sm + kTrBias);
  float* gb = reinterpret_cast<float*>(sm + kTrGb);
  float* sloss = reinterpret_cast<float*>(sm + kTrLoss);
  const uint32_t bar = smem_u32(sm + kTrBar);
  const long long row0 = (long long)blockIdx.x * kMlpTile;
  const long long grow = row0 + tid;

  load_kmajor(sm + kTrW1, w.W1, kMlpHid, kMlpIn);
  load_kmajor(sm + kTrW2, w.W2, kMlpHid, kMlpHid);
  load_kmajor(sm + kTrW3, w.W3, kMlpOut, kMlpHid);
  load_transposed(sm + kTrW3T, w.W3, kMlpOut, kMlpHid);   // [128 in][16 out]
  for (int i = tid; i < 272; i += blockDim.x) {
    sb[i] = i < 128 ? w.b1[i] : i < 256 ? w.b2[i - 128] : w.b3[i - 256];
    gb[i] = 0.f;
  }
  if (tid < 4) sloss[tid] = 0.f;
  for (int c = tid; c < kMlpTile * 8; c += blockDim.x) {
    const int r = c >> 3, kc = (c & 7) * 8;
    const long long gr = row0 + r;
    const uint4 val = gr < n ? *reinterpret_cast<const uint4*>(X + gr * kMlpIn + kc) : make_uint4(0, 0, 0, 0);
    *reinterpret_cast<uint4*>(sm + kTrX + kmaj(r, kc, kMlpIn)) = val;
    const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(&val);
#pragma unroll
    for (int j = 0; j < 8; ++j) *reinterpret_cast<__nv_bfloat16*>(sm + kTrXT + kmaj(kc + j, r, kMlpTile)) = e[j];
  }
  if (tid == 0) mbar_init(bar);
  if (warp == 0) tmem_alloc(smem_u32(sm + kTrSlot), 512);
  async_fence();
  tc_before();
  __syncthreads();
  tc_after();
  const uint32_t tm = *reinterpret_cast<volatile uint32_t*>(sm + kTrSlot);
  const uint32_t lane_off = (uint32_t)(warp * 32) << 16;
  uint32_t phase = 0;
  int ok = 1;

  do {
    // ---- forward ----
    if (tid == 0) {
      tc_after();
      gemm(tm + 0, smem_u32(sm + kTrX), smem_u32(sm + kTrW1), kMlpHid, kMlpIn, false);
      umma_commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase));
    phase ^= 1;
    if (!ok) break;
    tc_after();
    epilogue_relu(tm + lane_off + 0, sb, sm + kTrH1, sm + kTrH1T, tid);
    async_fence();
    tc_before();
    __syncthreads();
    if (tid == 0) {
      tc_after();
      gemm(tm + 128, smem_u32(sm + kTrH1), smem_u32(sm + kTrW2), kMlpHid, kMlpHid, false);
      umma_commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase));
    phase ^= 1;
    if (!ok) break;
    tc_after();
    epilogue_relu(tm + lane_off + 128, sb + 128, sm + kTrH2, sm + kTrH2T, tid);
    __syncthreads();   // every read of W2 by the finished MMA is behind us; W2 becomes W2^T
    load_transposed(sm + kTrW2, w.W2, kMlpHid, kMlpHid);
    async_fence();
    tc_before();
    __syncthreads();
    if (tid == 0) {
      tc_after();
      gemm(tm + 256, smem_u32(sm + kTrH2), smem_u32(sm + kTrW3), kMlpOut, kMlpHid, false);
      umma_commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase));
    phase ^= 1;
    if (!ok) break;
    tc_after();

    // ---- softmax cross-entropy on this thread's row ----
    {
      float v[16];
      tmem_ld16(tm + lane_off + 256, v);
      const int t = grow < n ? target[grow] : -1;
      const int nv = grow < n ? nvalid[grow] : 0;
      float mx = -3.0e38f;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        v[j] += sb[256 + j];
        const bool valid = (j < kMlpSlots && j < nv) || j == kMlpEscape;
        if (valid) mx = fmaxf(mx, v[j]);
      }
      float e[16], S = 0.f;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const bool valid = (j < kMlpSlots && j < nv) || j == kMlpEscape;
        e[j] = valid ? __expf(v[j] - mx) : 0.f;
        S += e[j];
      }
      const bool row_on = t >= 0;
      float loss = 0.f;
      if (row_on) loss = -(v[t] - mx - __logf(S));
      float dz[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) dz[j] = row_on ? (e[j] / S - (j == t ? 1.f : 0.f)) * inv_count : 0.f;
      uint32_t p[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) p[j] = pack_bf16(dz[2 * j], dz[2 * j + 1]);
      *reinterpret_cast<uint4*>(sm + kTrZ3 + kmaj(tid, 0, kMlpOut)) = make_uint4(p[0], p[1], p[2], p[3]);
      *reinterpret_cast<uint4*>(sm + kTrZ3 + kmaj(tid, 8, kMlpOut)) = make_uint4(p[4], p[5], p[6], p[7]);
      const __nv_bfloat16* eb = reinterpret_cast<const __nv_bfloat16*>(p);
#pragma unroll
      for (int j = 0; j < 16; ++j) *reinterpret_cast<__nv_bfloat16*>(sm + kTrZ3T + kmaj(j, tid, kMlpTile)) = eb[j];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const float s = warp_sum_f(dz[j]);
        if (lane == 0) atomicAdd(&gb[256 + j], s);
      }
      loss = warp_sum_f(loss);
      if (lane == 0) sloss[warp] = loss;
    }
    async_fence();
    tc_before();
    __syncthreads();

    // ---- backward, layer 3: dW3^T = H2^T dZ3 ; dH2 = dZ3 W3 ----
    if (tid == 0) {
      tc_after();
      gemm(tm + 288, smem_u32(sm + kTrH2T), smem_u32(sm + kTrZ3T), kMlpOut, kMlpTile, false);
      gemm(tm + 0, smem_u32(sm + kTrZ3), smem_u32(sm + kTrW3T), kMlpHid, kMlpOut, false);
      umma_commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase));
    phase ^= 1;
    if (!ok) break;
    tc_after();
    {
      float v[16];
      tmem_ld16(tm + lane_off + 288, v);   // row tid of dW3^T = column tid of dW3
#pragma unroll
      for (int j = 0; j < 16; ++j) atomicAdd(grads + kOffW3 + j * kMlpHid + tid, v[j]);
      for (int c0 = 0; c0 < kMlpHid; c0 += 16) {
        tmem_ld16(tm + lane_off + 0 + c0, v);
        float dz[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) dz[j] = bf16_at(sm + kTrH2, kmaj(tid, c0 + j, kMlpHid)) > 0.f ? v[j] : 0.f;
        uint32_t p[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) p[j] = pack_bf16(dz[2 * j], dz[2 * j + 1]);
        *reinterpret_cast<uint4*>(sm + kTrH1 + kmaj(tid, c0, kMlpHid)) = make_uint4(p[0], p[1], p[2], p[3]);
        *reinterpret_cast<uint4*>(sm + kTrH1 + kmaj(tid, c0 + 8, kMlpHid)) = make_uint4(p[4], p[5], p[6], p[7]);
        const __nv_bfloat16* eb = reinterpret_cast<const __nv_bfloat16*>(p);
#pragma unroll
        for (int j = 0; j < 16; ++j)
          *reinterpret_cast<__nv_bfloat16*>(sm + kTrH2T + kmaj(c0 + j, tid, kMlpTile)) = eb[j];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const float s = warp_sum_f(dz[j]);
          if (lane == 0) atomicAdd(&gb[128 + c0 + j], s);
        }
      }
    }
    async_fence();
    tc_before();
    __syncthreads();

    // ---- backward, layer 2: dW2 = dZ2^T H1 ; dH1 = dZ2 W2 ----
    if (tid == 0) {
      tc_after();
      gemm(tm + 320, smem_u32(sm + kTrH2T), smem_u32(sm + kTrH1T), kMlpHid, kMlpTile, false);
      gemm(tm + 128, smem_u32(sm + kTrH1), smem_u32(sm + kTrW2), kMlpHid, kMlpHid, false);
      umma_commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase));
    phase ^= 1;
    if (!ok) break;
    tc_after();
    {
      float v[16];
      for (int c0 = 0; c0 < kMlpHid; c0 += 16) {
        tmem_ld16(tm + lane_off + 320 + c0, v);   // row tid of dW2
#pragma unroll
        for (int j = 0; j < 16; ++j) atomicAdd(grads + kOffW2 + tid * kMlpHid + c0 + j, v[j]);
      }
      for (int c0 = 0; c0 < kMlpHid; c0 += 16) {
        tmem_ld16(tm + lane_off + 128 + c0, v);
        float dz[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const uint32_t off = kmaj(c0 + j, tid, kMlpTile);
          dz[j] = bf16_at(sm + kTrH1T, off) > 0.f ? v[j] : 0.f;
          put_bf16(sm + kTrH1T, off, dz[j]);   // H1^T column tid becomes dZ1^T column tid
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const float s = warp_sum_f(dz[j]);
          if (lane == 0) atomicAdd(&gb[c0 + j], s);
        }
      }
    }
    async_fence();
    tc_before();
    __syncthreads();

    // ---- backward, layer 1: dW1 = dZ1^T X ----
    if (tid == 0) {
      tc_after();
      gemm(tm + 448, smem_u32(sm + kTrH1T), smem_u32(sm + kTrXT), kMlpIn, kMlpTile, false);
      umma_commit(bar);
    }
    ok = __syncthreads_and(mbar_wait(bar, phase));
    phase ^= 1;
    if (!ok) break;
    tc_after();
    {
      float v[16];
      for (int c0 = 0; c0 < kMlpIn; c0 += 16) {
        tmem_ld16(tm + lane_off + 448 + c0, v);
#pragma unroll
        for (int j = 0; j < 16; ++j) atomicAdd(grads + kOffW1 + tid * kMlpIn + c0 + j, v[j]);
      }
    }
    __syncthreads();
    for (int i = tid; i < 272; i += blockDim.x) {
      const int off = i < 128 ? kOffB1 + i : i < 256 ? kOffB2 + (i - 128) : kOffB3 + (i - 256);
      atomicAdd(grads + off, gb[i]);
    }
    if (tid == 0) atomicAdd(loss_sum, (double)(sloss[0] + sloss[1] + sloss[2] + sloss[3]));
  } while (false);

  if (!ok) {
    if (tid == 0) atomicOr(status, kErrTensorWait);
    mbar_wait(bar, phase ^ 1);   // the phase that gave up: let an MMA still in flight finish
  }
  tc_before();
  __syncthreads();
  if (warp == 0) {
    tc_after();
    tmem_dealloc(tm, 512);
  }
}

__global__ void k_mlp_publish(const float* __restrict__ params, __nv_bfloat16* W1, __nv_bfloat16* W2,
                              __nv_bfloat16* W3, float* bias) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpParams; i += gridDim.x * blockDim.x) {
    const float x = params[i];
    if (i < kOffB1) W1[i - kOffW1] = __float2bfloat16_rn(x);
    else if (i < kOffW2) bias[i - kOffB1] = x;
    else if (i < kOffB2) W2[i - kOffW2] = __float2bfloat16_rn(x);
    else if (i < kOffW3) bias[128 + i - kOffB2] = x;
    else if (i < kOffB3) W3[i - kOffW3] = __float2bfloat16_rn(x);
    else bias[256 + i - kOffB3] = x;
  }
}

__global__ void k_mlp_adam(float* params, float* m, float* v, const float* __restrict__ g, float lr, float beta1,
                           float beta2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpParams; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = beta1 * m[i] + (1.f - beta1) * gi;
    const float vi = beta2 * v[i] + (1.f - beta2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    params[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

__global__ void k_float_to_bf16(const float* __restrict__ in, __nv_bfloat16* out, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn(in[i]);
}

}  // namespace

void mlp_forward(const __nv_bfloat16* features, long long n, MlpWeights w, float* logits, int* status, int sms,
                 cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdSmem);
    attr = true;
  }
  if (n <= 0) return;
  const long long tiles = (n + kMlpTile - 1) / kMlpTile;
  const int grid = (int)(tiles < sms ? tiles : sms);
  k_mlp_forward<<<grid, 128, kFwdSmem, s>>>(features, n, w, logits, status);
}

void mlp_gradients(const __nv_bfloat16* features, const int* target, const int* nvalid, long long n, float inv_count,
                   MlpWeights w, float* grads, double* loss_sum, int* status, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_mlp_train_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrSmem);
    attr = true;
  }
  if (n <= 0) return;
  const long long tiles = (n + kMlpTile - 1) / kMlpTile;
  k_mlp_train_tile<<<(unsigned)tiles, 128, kTrSmem, s>>>(features, target, nvalid, n, inv_count, w, grads, loss_sum,
                                                         status);
}

void mlp_adam(float* params, float* m, float* v, const float* grads, int step, float lr, float beta1, float beta2,
              float eps, __nv_bfloat16* W1, __nv_bfloat16* W2, __nv_bfloat16* W3, float* bias, cudaStream_t s) {
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, s>>>(params, m, v, grads, lr, beta1, beta2, eps, c1, c2);
  k_mlp_publish<<<(kMlpParams + 255) / 256, 256, 0, s>>>(params, W1, W2, W3, bias);
}

void mlp_publish(const float* params, __nv_bfloat16* W1, __nv_bfloat16* W2, __nv_bfloat16* W3, float* bias,
                 cudaStream_t s) {
  k_mlp_publish<<<(kMlpParams + 255) / 256, 256, 0, s>>>(params, W1, W2, W3, bias);
}

void float_to_bf16(const float* in, __nv_bfloat16* out, long long n, cudaStream_t s) {
  if (n <= 0) return;
  long long g = (n + 255) / 256;
  if (g > 4096) g = 4096;
  k_float_to_bf16<<<(unsigned)g, 256, 0, s>>>(in, out, n);
}

}  // namespace sbpb
