// swdk_mlp.cu -- the learned bracket proposal: a 4x256 GELU MLP trained and
// run with hand-written kernels.  Its GEMMs run on the sm_100a tensor cores
// (tcgen05.mma, BF16 operands from shared memory, FP32 accumulators in
// tensor memory); bias/GELU epilogues, the Gaussian negative log-likelihood
// and Adam are plain CUDA kernels.  The network has no counterpart in the
// reference; it only proposes brackets that the FP64 secular function must
// confirm, so it changes the number of secular evaluations, never a root.
//
// Architecture (per wave type): x[320] (258 used: 64 nodes x (vs, vp, rho,
// thickness), log T, mode; zero padded) -> 256 -> 256 -> 256 -> 256 -> out[64]
// (2 used: mu, log sigma of the normalised phase velocity; the output layer
// is stored 64 wide so every GEMM runs on full 128x64 tiles).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "swdk.h"

namespace {

constexpr int MLP_IN = 320, MLP_H = 256, MLP_OUT = 64, MLP_LAYERS = 5;
constexpr int TM = 128, TN = 64, TK = 64;  // CTA tile (M x N), K stage

// ---------------------------------------------------------------------------
// tcgen05 helpers (PTX ISA 8.7, sm_100a)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// K-major, 128-byte swizzled operand tile: rows of 64 bf16 (128 B), 8-row
// groups 1024 B apart (SBO), version 1, layout SWIZZLE_128B (2)
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;            // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;  // stride byte offset
  d |= (uint64_t)1 << 46;            // descriptor version (sm100)
  d |= (uint64_t)2 << 61;            // SWIZZLE_128B
  return d;
}

// kind::f16 instruction descriptor: D=F32, A=B=BF16, both K-major
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// bounded wait on an mbarrier phase; returns false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (int it = 0; it < (1 << 24); ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// ---------------------------------------------------------------------------
// C[M x N] = A[M x K] * B[N x K]^T  (A, B bf16 row-major, K % 64 == 0,
// M % 128 == 0, N % 64 == 0), FP32 accumulate in TMEM, then
//   out_f32 (optional) = C + bias (pre-activation)
//   out_bf16 (optional) = act(C + bias) with act = GELU or identity
// lda/ldb/ldc are row strides in elements.  *err is set when a wait times
// out (the kernel then skips its epilogue and releases its TMEM).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float gelu(float x) {
  return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f));
}

__global__ void __launch_bounds__(128) k_gemm_tn(int M, int N, int K, const __nv_bfloat16* __restrict__ A, int lda,
                                                 const __nv_bfloat16* __restrict__ B, int ldb,
                                                 const float* __restrict__ bias, int act, float* __restrict__ outf,
                                                 __nv_bfloat16* __restrict__ outb, int ldc, int* __restrict__ err) {
  __shared__ __align__(1024) uint8_t sA[TM * TK * 2];
  __shared__ __align__(1024) uint8_t sB[TN * TK * 2];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(TN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base;
  constexpr uint32_t idesc = idesc_bf16(TM, TN);
  bool ok = true;
  uint32_t phase = 0;
  for (int k0 = 0; k0 < K; k0 += TK) {
    // global -> shared, 16-byte chunks, 128B swizzle: chunk j of row r goes
    // to r*128 + ((j ^ (r & 7)) << 4)
    for (int c = tid; c < TM * 8; c += 128) {
      const int r = c >> 3, j = c & 7;
      const uint4 v = *reinterpret_cast<const uint4*>(A + (size_t)(m0 + r) * lda + k0 + j * 8);
      *reinterpret_cast<uint4*>(sA + r * 128 + ((j ^ (r & 7)) << 4)) = v;
    }
    for (int c = tid; c < TN * 8; c += 128) {
      const int r = c >> 3, j = c & 7;
      const uint4 v = *reinterpret_cast<const uint4*>(B + (size_t)(n0 + r) * ldb + k0 + j * 8);
      *reinterpret_cast<uint4*>(sB + r * 128 + ((j ^ (r & 7)) << 4)) = v;
    }
    asm volatile("fence.proxy.async.shared::cta;");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint64_t da = sw128_desc(smem_u32(sA)), db = sw128_desc(smem_u32(sB));
#pragma unroll
      for (int kk = 0; kk < TK / 16; ++kk) {
        const uint64_t a = da + (uint64_t)(kk * 2), b = db + (uint64_t)(kk * 2);  // +32 B per K=16 step
        const uint32_t acc = (k0 > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(&bar)));
    }
    // every thread waits for the MMAs to finish reading shared memory
    if (!mbar_wait(&bar, phase)) ok = false;
    phase ^= 1u;
    __syncthreads();
    if (!__syncthreads_and(ok)) break;
  }
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (__syncthreads_and(ok)) {
    // TMEM lane = row: warp w owns rows 32w..32w+31; 64 fp32 columns
    const int row = m0 + warp * 32 + lane;
    uint32_t v[64];
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]), "=r"(v[36]), "=r"(v[37]), "=r"(v[38]), "=r"(v[39]),
          "=r"(v[40]), "=r"(v[41]), "=r"(v[42]), "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]),
          "=r"(v[48]), "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]), "=r"(v[54]), "=r"(v[55]),
          "=r"(v[56]), "=r"(v[57]), "=r"(v[58]), "=r"(v[59]), "=r"(v[60]), "=r"(v[61]), "=r"(v[62]), "=r"(v[63])
        : "r"(taddr + 32u));
    asm volatile("tcgen05.wait::ld.sync.aligned;");
    if (row < M) {
#pragma unroll 8
      for (int j = 0; j < 64; ++j) {
        const int col = n0 + j;
        float x = __uint_as_float(v[j]) + (bias ? bias[col] : 0.0f);
        if (outf) outf[(size_t)row * ldc + col] = x;
        if (outb) outb[(size_t)row * ldc + col] = __float2bfloat16_rn(act ? gelu(x) : x);
      }
    }
  } else if (tid == 0) {
    atomicExch(err, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TN));
}

// ---------------------------------------------------------------------------
// Fused inference for the engine: one persistent CTA per SM pushes 128-row
// tiles through all five layers.  The tile's activations stay in shared
// memory in the SW128 K-major image the MMA descriptors read (input: 5
// K-blocks of 64 columns, hidden: 4); weight K-blocks (N x 64, pre-swizzled
// in global memory by k_swizzle_weights) stream through a 3-deep ring of
// 32 KB buffers with cp.async.bulk (no multicast) and mbarrier transaction
// counts.  Thread 0 issues copies and tcgen05.mma (M=128, N=256/64, K=16) into
// a 256-column TMEM accumulator; 8 warps run the bias+GELU epilogue (warp w
// reads TMEM lanes 32(w%4).., columns 128(w/4)..) and write the next layer's
// activations back into shared memory; the output layer's epilogue turns
// (mu, log sigma) into the bracket proposal (c = 3.5 + mu, half-width =
// kappa sigma clamped to [2e-5 c, 0.2]).  Every wait is bounded; a timeout
// sets *err, drains the copies in flight and releases TMEM.
// ---------------------------------------------------------------------------
constexpr int PX_ROWS = 128;
constexpr int PX_KB_IN = MLP_IN / 64, PX_KB_H = MLP_H / 64;     // 5, 4
constexpr int PX_TILE_BYTES = PX_ROWS * MLP_IN * 2;              // 80 KB input tile image
constexpr int PX_WBUF = MLP_H * 64 * 2;                          // 32 KB weight block
constexpr int PX_NBUF = 3;
constexpr int PX_BLOCKS = PX_KB_IN + 3 * PX_KB_H + PX_KB_H;      // 21 weight blocks per tile
constexpr int PX_SMEM = PX_TILE_BYTES + PX_NBUF * PX_WBUF + 1024; // + barriers, 1 KB alignment slack

__device__ __forceinline__ int px_layer_of(int idx, int& kb) {
  if (idx < PX_KB_IN) { kb = idx; return 0; }
  idx -= PX_KB_IN;
  kb = idx % PX_KB_H;
  return 1 + idx / PX_KB_H;
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ void mbar_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}

__global__ void __launch_bounds__(256, 1) k_mlp_propose(int ntiles, int nrows, const uint8_t* __restrict__ xtiles,
                                                        const uint8_t* __restrict__ wsw, const float* __restrict__ w,
                                                        const size_t* __restrict__ boffs, double kappa,
                                                        float2* __restrict__ prop, int* __restrict__ err) {
  extern __shared__ uint8_t px_raw[];
  uint8_t* base = (uint8_t*)(((uintptr_t)px_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* act = base;                          // 80 KB activation image
  uint8_t* wbuf = base + PX_TILE_BYTES;         // 3 x 32 KB weight ring
  uint64_t* bars = (uint64_t*)(wbuf + PX_NBUF * PX_WBUF);
  // bars[0..2] full, [3..5] empty, [6] accumulator ready, [7] input tile
  __shared__ uint32_t tmem_base;
  __shared__ int s_fail;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(256));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int i = 0; i < 8; ++i) mbar_init(&bars[i], 1);
    asm volatile("fence.mbarrier_init.release.cluster;");
    s_fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base;
  const uint32_t act_s = smem_u32(act), wbuf_s = smem_u32(wbuf);
  const uint32_t bar_full = smem_u32(&bars[0]), bar_empty = smem_u32(&bars[3]);
  const uint32_t bar_acc = smem_u32(&bars[6]), bar_in = smem_u32(&bars[7]);
  // weight block idx -> global image offset and bytes
  auto wblock = [&](int idx, size_t& off, uint32_t& bytes) {
    int kb;
    const int l = px_layer_of(idx, kb);
    const int n = (l == MLP_LAYERS - 1) ? MLP_OUT : MLP_H;
    size_t o = 0;
    for (int q = 0; q < l; ++q) o += (size_t)MLP_H * ((q == 0) ? MLP_IN : MLP_H) * 2;
    off = o + (size_t)kb * n * 128;
    bytes = (uint32_t)(n * 128);
  };
  const int my_tiles = (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  const long long total = (long long)my_tiles * PX_BLOCKS;
  long long issued = 0, consumed = 0;  // weight blocks copied / handed to the MMA (thread 0)
  uint32_t acc_phase = 0, in_phase = 0;
  bool ok = true, in_pending = false;
  if (tid == 0) {
    for (; issued < total && issued < PX_NBUF; ++issued) {
      size_t off; uint32_t bytes;
      wblock((int)(issued % PX_BLOCKS), off, bytes);
      const int b = (int)(issued % PX_NBUF);
      mbar_expect(bar_full + 8 * b, bytes);
      bulk_g2s(wbuf_s + b * PX_WBUF, wsw + off, bytes, bar_full + 8 * b);
    }
  }
  for (int it = 0; it < my_tiles; ++it) {
    const int tile = (int)blockIdx.x + it * (int)gridDim.x;
    if (tid == 0) {
      mbar_expect(bar_in, PX_TILE_BYTES);
      bulk_g2s(act_s, xtiles + (size_t)tile * PX_TILE_BYTES, PX_TILE_BYTES, bar_in);
      in_pending = true;
    }
    if (!mbar_wait(&bars[7], in_phase)) ok = false;
    else in_pending = false;
    if (!__syncthreads_and(ok)) { ok = false; break; }
    in_phase ^= 1u;
    for (int l = 0; l < MLP_LAYERS; ++l) {
      const int nkb = (l == 0) ? PX_KB_IN : PX_KB_H;
      const int n = (l == MLP_LAYERS - 1) ? MLP_OUT : MLP_H;
      if (tid == 0 && ok) {
        const uint32_t idesc = (n == MLP_H) ? idesc_bf16(128, 256) : idesc_bf16(128, 64);
        for (int kb = 0; kb < nkb && ok; ++kb) {
          const long long g = consumed;
          const int b = (int)(g % PX_NBUF);
          if (!mbar_wait(&bars[b], (uint32_t)((g / PX_NBUF) & 1))) { ok = false; break; }
          asm volatile("tcgen05.fence::after_thread_sync;");
          const uint64_t da = sw128_desc(act_s + kb * (PX_ROWS * 128)), db = sw128_desc(wbuf_s + b * PX_WBUF);
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            const uint32_t accf = (kb > 0 || kk > 0) ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                ::"r"(tmem), "l"(da + (uint64_t)(kk * 2)), "l"(db + (uint64_t)(kk * 2)), "r"(idesc), "r"(accf));
          }
          mma_commit(bar_empty + 8 * b);
          ++consumed;
          // refill the buffer the previous block used, once its MMAs are done
          if (g >= 1 && issued < total) {
            const long long gp = g - 1;
            const int bp = (int)(gp % PX_NBUF);
            if (!mbar_wait(&bars[3 + bp], (uint32_t)((gp / PX_NBUF) & 1))) { ok = false; break; }
            size_t off; uint32_t bytes;
            wblock((int)(issued % PX_BLOCKS), off, bytes);
            mbar_expect(bar_full + 8 * bp, bytes);
            bulk_g2s(wbuf_s + bp * PX_WBUF, wsw + off, bytes, bar_full + 8 * bp);
            ++issued;
          }
        }
        mma_commit(bar_acc);
      }
      if (tid == 0 && !ok) s_fail = 1;
      __syncthreads();
      if (s_fail) { ok = false; break; }
      if (!mbar_wait(&bars[6], acc_phase)) ok = false;
      acc_phase ^= 1u;
      asm volatile("tcgen05.fence::after_thread_sync;");
      if (!__syncthreads_and(ok)) { ok = false; break; }
      const int q = warp & 3, h = warp >> 2;
      const int r = q * 32 + lane;  // tile row = TMEM lane
      const float* bias = w + boffs[l];
      if (l < MLP_LAYERS - 1) {
        for (int cb = 0; cb < 4; ++cb) {  // 32-column chunks of this warp's half
          const int c0 = h * 128 + cb * 32;
          uint32_t v[32];
          tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, v);
          asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
          for (int j8 = 0; j8 < 4; ++j8) {  // 8 columns = one 16-byte chunk
            uint32_t pk[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const int c = c0 + j8 * 8 + 2 * e;
              const float x0 = gelu(__uint_as_float(v[j8 * 8 + 2 * e]) + bias[c]);
              const float x1 = gelu(__uint_as_float(v[j8 * 8 + 2 * e + 1]) + bias[c + 1]);
              const __nv_bfloat162 b2 = __floats2bfloat162_rn(x0, x1);
              pk[e] = *reinterpret_cast<const uint32_t*>(&b2);
            }
            const int c = c0 + j8 * 8;
            const int kb = c >> 6, j = (c & 63) >> 3;
            uint8_t* dst = act + kb * (PX_ROWS * 128) + r * 128 + ((j ^ (r & 7)) << 4);
            *reinterpret_cast<uint4*>(dst) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
          }
        }
        asm volatile("fence.proxy.async.shared::cta;");
      } else if (h == 0) {
        uint32_t v2[2];
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0,%1}, [%2];"
                     : "=r"(v2[0]), "=r"(v2[1])
                     : "r"(tmem + ((uint32_t)(q * 32) << 16)));
        asm volatile("tcgen05.wait::ld.sync.aligned;");
        const long long row = (long long)tile * PX_ROWS + r;
        if (row < nrows) {
          const float mu = __uint_as_float(v2[0]) + bias[0];
          const float ls = __uint_as_float(v2[1]) + bias[1];
          const double c = 3.5 + (double)mu;
          double hw = kappa * exp(fmin(fmax((double)ls, -12.0), 2.0));
          hw = fmin(fmax(hw, 2.0e-5 * c), 0.2);
          prop[row] = (mu == mu && ls == ls) ? make_float2((float)c, (float)hw) : make_float2(0.0f, 0.0f);
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncthreads();
    }
    if (!ok) break;
  }
  // drain: copies still in flight and the last MMAs, then release TMEM
  if (tid == 0) {
    if (in_pending) mbar_wait(&bars[7], in_phase);
    for (long long g = consumed; g < issued; ++g) mbar_wait(&bars[g % PX_NBUF], (uint32_t)((g / PX_NBUF) & 1));
    if (consumed > 0) {
      const long long g = consumed - 1;
      mbar_wait(&bars[3 + g % PX_NBUF], (uint32_t)((g / PX_NBUF) & 1));
    }
    if (!ok) atomicExch(err, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256));
}

// bf16 weights (flat block, layer l: nout x kin row-major) -> the SW128
// K-major image k_mlp_propose streams: layer by layer, K-block by K-block,
// row n of a block at n*128 bytes, 16-byte chunk j at (j ^ (n & 7)) * 16
__global__ void k_swizzle_weights(const __nv_bfloat16* __restrict__ wb, const size_t* __restrict__ woffs,
                                  uint8_t* __restrict__ wsw) {
  const int l = blockIdx.y;
  const int kin = (l == 0) ? MLP_IN : MLP_H, n = (l == MLP_LAYERS - 1) ? MLP_OUT : MLP_H;
  size_t o = 0;
  for (int q = 0; q < l; ++q) o += (size_t)MLP_H * ((q == 0) ? MLP_IN : MLP_H) * 2;
  const int nchunk = n * kin / 8;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nchunk; c += gridDim.x * blockDim.x) {
    const int row = c / (kin / 8), k8 = c % (kin / 8);
    const int kb = k8 >> 3, j = k8 & 7;
    const uint4 v = *reinterpret_cast<const uint4*>(wb + woffs[l] + (size_t)row * kin + k8 * 8);
    *reinterpret_cast<uint4*>(wsw + o + (size_t)kb * n * 128 + row * 128 + ((j ^ (row & 7)) << 4)) = v;
  }
}

// ---------------------------------------------------------------------------
// elementwise kernels of the MLP
// ---------------------------------------------------------------------------
__global__ void k_to_bf16(int n, const float* __restrict__ x, __nv_bfloat16* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16_rn(x[i]);
}

// y[c*rows + r] = x[r*cols + c]  (bf16 transpose of a row-major rows x cols)
__global__ void k_transpose_bf16(int rows, int cols, const __nv_bfloat16* __restrict__ x, int ldx,
                                 __nv_bfloat16* __restrict__ y, int ldy) {
  __shared__ __nv_bfloat16 t[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    t[i][threadIdx.x] = (r < rows && c < cols) ? x[(size_t)r * ldx + c] : __float2bfloat16_rn(0.0f);
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (c < cols && r < rows) y[(size_t)c * ldy + r] = t[threadIdx.x][i];
  }
}

// Gaussian NLL of (mu, log sigma) against y on rows < M (rows of the padded
// batch beyond M get zero gradient); dOut is the bf16 gradient w.r.t. the
// 16-wide output (columns 0,1), loss accumulates the batch mean.
__global__ void k_nll(int M, int Mpad, const float* __restrict__ out, const float* __restrict__ y,
                      __nv_bfloat16* __restrict__ dout, float* __restrict__ loss) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= Mpad) return;
  float g0 = 0.0f, g1 = 0.0f, l = 0.0f;
  if (r < M) {
    const float mu = out[(size_t)r * MLP_OUT], ls = fminf(fmaxf(out[(size_t)r * MLP_OUT + 1], -12.0f), 4.0f);
    const float inv = expf(-ls), e = (y[r] - mu) * inv;
    l = 0.5f * e * e + ls;
    g0 = -e * inv / (float)M;
    g1 = (1.0f - e * e) / (float)M;
  }
  for (int j = 0; j < MLP_OUT; ++j)
    dout[(size_t)r * MLP_OUT + j] = __float2bfloat16_rn(j == 0 ? g0 : j == 1 ? g1 : 0.0f);
  if (r < M) atomicAdd(loss, l / (float)M);
}

// dZ = dH * GELU'(Z)   (bf16 dH in, bf16 dZ out)
__global__ void k_gelu_back(int n, const float* __restrict__ z, const __nv_bfloat16* __restrict__ dh,
                            __nv_bfloat16* __restrict__ dz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x = z[i];
  const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  dz[i] = __float2bfloat16_rn(__bfloat162float(dh[i]) * (cdf + x * pdf));
}

// db[c] = sum_r dz[r, c]
__global__ void k_colsum(int rows, int cols, const __nv_bfloat16* __restrict__ dz, float* __restrict__ db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.0f;
  for (int r = 0; r < rows; ++r) s += __bfloat162float(dz[(size_t)r * cols + c]);
  db[c] = s;
}

// Adam with bias correction on FP32 masters; refreshes the bf16 copies
__global__ void k_adam(int n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                       const unsigned char* __restrict__ mask, __nv_bfloat16* __restrict__ wb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (mask && !mask[i]) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi, vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16_rn(wi);
}

}  // namespace

// ---------------------------------------------------------------------------
// host-side MLP
// ---------------------------------------------------------------------------
struct swdk_mlp {
  int device = 0;
  int kin[MLP_LAYERS], nout[MLP_LAYERS];
  size_t woff[MLP_LAYERS], boff[MLP_LAYERS], nparam = 0;
  // FP32 masters, Adam moments, gradients (one flat block each)
  float *w = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;
  unsigned char* mask = nullptr;  // 1 where a weight is a real (unpadded) parameter
  __nv_bfloat16* wb = nullptr;    // bf16 copy of the flat block (weights usable as GEMM B operand)
  __nv_bfloat16* wt = nullptr;    // bf16 transposed weights (for dX)
  int step = 0;
  // activations for a batch of up to cap rows
  int cap = 0;
  __nv_bfloat16 *xin = nullptr, *h[MLP_LAYERS] = {}, *dz[MLP_LAYERS] = {}, *xt = nullptr, *dzt = nullptr,
                *dh = nullptr;
  float *z[MLP_LAYERS] = {}, *out = nullptr, *y = nullptr, *loss = nullptr, *gscr = nullptr;
  // fused inference: swizzled weight image, layer offsets on the device
  uint8_t* wsw = nullptr;
  size_t* d_offs = nullptr;  // woff[5], boff[5]
  bool wsw_dirty = true;
  int nsm = 0;
  int* err = nullptr;
  cudaStream_t stream = nullptr;
  std::string msg;
};

namespace {

int mlp_fail(swdk_mlp* p, const char* what, cudaError_t e) {
  if (p) p->msg = std::string(what) + ": " + cudaGetErrorString(e);
  return SWDK_E_CUDA;
}
#define MCK(call)                                              \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return mlp_fail(p, #call, e_);      \
  } while (0)

int gemm(swdk_mlp* p, int M, int N, int K, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb,
         const float* bias, int act, float* outf, __nv_bfloat16* outb, int ldc, cudaStream_t st) {
  dim3 grid(M / TM, N / TN);
  k_gemm_tn<<<grid, 128, 0, st>>>(M, N, K, A, lda, B, ldb, bias, act, outf, outb, ldc, p->err);
  MCK(cudaGetLastError());
  return SWDK_OK;
}

int ensure_batch(swdk_mlp* p, int rows) {
  if (rows <= p->cap) return SWDK_OK;
  auto fr = [](void* q) { if (q) cudaFree(q); };
  fr(p->xin); fr(p->xt); fr(p->dzt); fr(p->dh); fr(p->out); fr(p->y);
  for (int l = 0; l < MLP_LAYERS; ++l) { fr(p->h[l]); fr(p->dz[l]); fr(p->z[l]); }
  const size_t R = (size_t)rows;
  MCK(cudaMalloc(&p->xin, R * MLP_IN * sizeof(__nv_bfloat16)));
  MCK(cudaMalloc(&p->xt, R * MLP_IN * sizeof(__nv_bfloat16)));
  MCK(cudaMalloc(&p->dzt, R * MLP_H * sizeof(__nv_bfloat16)));
  MCK(cudaMalloc(&p->dh, R * MLP_IN * sizeof(__nv_bfloat16)));
  MCK(cudaMalloc(&p->out, R * MLP_OUT * sizeof(float)));
  MCK(cudaMalloc(&p->y, R * sizeof(float)));
  for (int l = 0; l < MLP_LAYERS; ++l) {
    MCK(cudaMalloc(&p->h[l], R * p->nout[l] * sizeof(__nv_bfloat16)));
    MCK(cudaMalloc(&p->dz[l], R * p->nout[l] * sizeof(__nv_bfloat16)));
    MCK(cudaMalloc(&p->z[l], R * p->nout[l] * sizeof(float)));
  }
  p->cap = rows;
  return SWDK_OK;
}

// forward pass on p->xin (rows Mpad); the last pre-activation z[4]
// (Mpad x 64) holds (mu, log sigma) in columns 0, 1
int forward(swdk_mlp* p, int Mpad, cudaStream_t st) {
  const __nv_bfloat16* x = p->xin;
  for (int l = 0; l < MLP_LAYERS; ++l) {
    const bool last = (l == MLP_LAYERS - 1);
    const int r = gemm(p, Mpad, p->nout[l], p->kin[l], x, p->kin[l], p->wb + p->woff[l], p->kin[l],
                       p->w + p->boff[l], last ? 0 : 1, p->z[l], last ? nullptr : p->h[l], p->nout[l], st);
    if (r) return r;
    x = p->h[l];
  }
  return SWDK_OK;
}

}  // namespace

extern "C" {

int swdk_mlp_create(swdk_mlp** out, int device, uint64_t seed) {
  if (!out) return SWDK_E_ARG;
  *out = nullptr;
  swdk_mlp* p = new swdk_mlp();
  p->device = device;
  MCK(cudaSetDevice(device));
  MCK(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  const int kin[MLP_LAYERS] = {MLP_IN, MLP_H, MLP_H, MLP_H, MLP_H};
  const int nout[MLP_LAYERS] = {MLP_H, MLP_H, MLP_H, MLP_H, MLP_OUT};
  size_t off = 0;
  for (int l = 0; l < MLP_LAYERS; ++l) {
    p->kin[l] = kin[l];
    p->nout[l] = nout[l];
    p->woff[l] = off;
    off += (size_t)nout[l] * kin[l];
    p->boff[l] = off;
    off += nout[l];
  }
  p->nparam = off;
  std::vector<float> hw(off, 0.0f);
  std::vector<unsigned char> hm(off, 0);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < MLP_LAYERS; ++l) {
    const int used_in = (l == 0) ? 258 : kin[l];
    const int used_out = (l == MLP_LAYERS - 1) ? 2 : nout[l];
    std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (float)used_in));
    for (int o = 0; o < used_out; ++o)
      for (int i = 0; i < used_in; ++i) {
        const size_t k = p->woff[l] + (size_t)o * kin[l] + i;
        hw[k] = (l == MLP_LAYERS - 1) ? 0.1f * nd(rng) : nd(rng);
        hm[k] = 1;
      }
    for (int o = 0; o < used_out; ++o) hm[p->boff[l] + o] = 1;
  }
  MCK(cudaMalloc(&p->w, off * sizeof(float)));
  MCK(cudaMalloc(&p->m, off * sizeof(float)));
  MCK(cudaMalloc(&p->v, off * sizeof(float)));
  MCK(cudaMalloc(&p->g, off * sizeof(float)));
  MCK(cudaMalloc(&p->mask, off));
  MCK(cudaMalloc(&p->wb, off * sizeof(__nv_bfloat16)));
  MCK(cudaMalloc(&p->wt, off * sizeof(__nv_bfloat16)));
  MCK(cudaMalloc(&p->loss, sizeof(float)));
  MCK(cudaMalloc(&p->gscr, (size_t)TM * MLP_IN * sizeof(float)));
  MCK(cudaMalloc(&p->err, sizeof(int)));
  MCK(cudaMemcpy(p->w, hw.data(), off * sizeof(float), cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(p->mask, hm.data(), off, cudaMemcpyHostToDevice));
  MCK(cudaMemset(p->m, 0, off * sizeof(float)));
  MCK(cudaMemset(p->v, 0, off * sizeof(float)));
  MCK(cudaMemset(p->g, 0, off * sizeof(float)));
  MCK(cudaMemset(p->err, 0, sizeof(int)));
  k_to_bf16<<<(int)((off + 255) / 256), 256, 0, p->stream>>>((int)off, p->w, p->wb);
  p->wsw_dirty = true;
  MCK(cudaGetLastError());
  MCK(cudaStreamSynchronize(p->stream));
  *out = p;
  return SWDK_OK;
}

void swdk_mlp_destroy(swdk_mlp* p) {
  if (!p) return;
  cudaSetDevice(p->device);
  if (p->stream) cudaStreamSynchronize(p->stream);
  void* bufs[] = {p->w, p->m, p->v, p->g, p->mask, p->wb, p->wt, p->loss, p->gscr, p->err, p->xin, p->xt, p->dzt,
                  p->dh, p->out, p->y, p->wsw, p->d_offs};
  for (void* b : bufs)
    if (b) cudaFree(b);
  for (int l = 0; l < MLP_LAYERS; ++l) {
    if (p->h[l]) cudaFree(p->h[l]);
    if (p->dz[l]) cudaFree(p->dz[l]);
    if (p->z[l]) cudaFree(p->z[l]);
  }
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
}

int64_t swdk_mlp_num_params(const swdk_mlp* p) { return p ? (int64_t)p->nparam : 0; }

int swdk_mlp_get_params(swdk_mlp* p, float* host, int64_t n) {
  if (!p || !host || n != (int64_t)p->nparam) return SWDK_E_ARG;
  MCK(cudaSetDevice(p->device));
  MCK(cudaMemcpy(host, p->w, p->nparam * sizeof(float), cudaMemcpyDeviceToHost));
  return SWDK_OK;
}

int swdk_mlp_set_params(swdk_mlp* p, const float* host, int64_t n) {
  if (!p || !host || n != (int64_t)p->nparam) return SWDK_E_ARG;
  MCK(cudaSetDevice(p->device));
  MCK(cudaMemcpy(p->w, host, p->nparam * sizeof(float), cudaMemcpyHostToDevice));
  k_to_bf16<<<(int)((p->nparam + 255) / 256), 256, 0, p->stream>>>((int)p->nparam, p->w, p->wb);
  p->wsw_dirty = true;
  MCK(cudaGetLastError());
  MCK(cudaStreamSynchronize(p->stream));
  return SWDK_OK;
}

// y = A * B^T on device bf16 operands (exposed for the GEMM unit test)
int swdk_gemm_bf16_tn(int M, int N, int K, const void* d_a, const void* d_b, float* d_c, int* d_err, void* stream) {
  if (M <= 0 || N <= 0 || K <= 0 || M % TM || N % TN || K % TK || !d_a || !d_b || !d_c || !d_err) return SWDK_E_ARG;
  dim3 grid(M / TM, N / TN);
  k_gemm_tn<<<grid, 128, 0, (cudaStream_t)stream>>>(M, N, K, (const __nv_bfloat16*)d_a, K, (const __nv_bfloat16*)d_b,
                                                     K, nullptr, 0, d_c, nullptr, N, d_err);
  return cudaGetLastError() == cudaSuccess ? SWDK_OK : SWDK_E_CUDA;
}

// fused inference on tile-image features -> bracket proposals
int swdk_mlp_propose(swdk_mlp* p, const void* d_xtiles, int nrows, double kappa, void* d_prop, void* stream) {
  if (!p || !d_xtiles || !d_prop || nrows <= 0 || !(kappa > 0.0)) return SWDK_E_ARG;
  MCK(cudaSetDevice(p->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : p->stream;
  // every call that writes the weights (create, set_params, load, train_step)
  // has finished its work on the network's stream before returning
  if (!p->wsw) {
    size_t bytes = 0;
    for (int l = 0; l < MLP_LAYERS; ++l) bytes += (size_t)p->nout[l] * p->kin[l] * 2;
    MCK(cudaMalloc(&p->wsw, bytes));
    MCK(cudaMalloc(&p->d_offs, 2 * MLP_LAYERS * sizeof(size_t)));
    size_t h[2 * MLP_LAYERS];
    for (int l = 0; l < MLP_LAYERS; ++l) { h[l] = p->woff[l]; h[MLP_LAYERS + l] = p->boff[l]; }
    MCK(cudaMemcpy(p->d_offs, h, sizeof(h), cudaMemcpyHostToDevice));
    MCK(cudaFuncSetAttribute(k_mlp_propose, cudaFuncAttributeMaxDynamicSharedMemorySize, PX_SMEM));
    MCK(cudaDeviceGetAttribute(&p->nsm, cudaDevAttrMultiProcessorCount, p->device));
    p->wsw_dirty = true;
  }
  if (p->wsw_dirty) {
    k_swizzle_weights<<<dim3(64, MLP_LAYERS), 256, 0, st>>>(p->wb, p->d_offs, p->wsw);
    MCK(cudaGetLastError());
    p->wsw_dirty = false;
  }
  const int ntiles = (nrows + PX_ROWS - 1) / PX_ROWS;
  const int grid = std::min(p->nsm > 0 ? p->nsm : 148, ntiles);
  k_mlp_propose<<<grid, 256, PX_SMEM, st>>>(ntiles, nrows, (const uint8_t*)d_xtiles, p->wsw, p->w,
                                            p->d_offs + MLP_LAYERS, kappa, (float2*)d_prop, p->err);
  MCK(cudaGetLastError());
  return SWDK_OK;
}

int swdk_mlp_error_flag(swdk_mlp* p, int* flag) {
  if (!p || !flag) return SWDK_E_ARG;
  MCK(cudaMemcpy(flag, p->err, sizeof(int), cudaMemcpyDeviceToHost));
  return SWDK_OK;
}

// forward on device features x (M x 320 bf16) -> out (M x 2 fp32: mu, log sigma)
int swdk_mlp_forward(swdk_mlp* p, const void* d_x, int M, float* d_out, void* stream) {
  if (!p || !d_x || !d_out || M <= 0) return SWDK_E_ARG;
  MCK(cudaSetDevice(p->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : p->stream;
  const int Mpad = (M + TM - 1) / TM * TM;
  int r = ensure_batch(p, Mpad);
  if (r) return r;
  MCK(cudaMemsetAsync(p->xin + (size_t)M * MLP_IN, 0, (size_t)(Mpad - M) * MLP_IN * sizeof(__nv_bfloat16), st));
  MCK(cudaMemcpyAsync(p->xin, d_x, (size_t)M * MLP_IN * sizeof(__nv_bfloat16), cudaMemcpyDeviceToDevice, st));
  r = forward(p, Mpad, st);
  if (r) return r;
  MCK(cudaMemcpy2DAsync(d_out, 2 * sizeof(float), p->z[MLP_LAYERS - 1], MLP_OUT * sizeof(float), 2 * sizeof(float),
                        M, cudaMemcpyDeviceToDevice, st));
  int herr = 0;
  MCK(cudaMemcpyAsync(&herr, p->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  if (herr) { p->msg = "tensor-core wait timed out"; return SWDK_E_CUDA; }
  return SWDK_OK;
}

// forward + Gaussian NLL + backward on (x, y); gradients land in p->g.
// With lr > 0 an Adam step follows.  *loss_out (host) gets the batch loss.
int swdk_mlp_train_step(swdk_mlp* p, const void* d_x, const float* d_y, int M, float lr, float* loss_out,
                        void* stream) {
  if (!p || !d_x || !d_y || M <= 0) return SWDK_E_ARG;
  MCK(cudaSetDevice(p->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : p->stream;
  const int Mpad = (M + TM - 1) / TM * TM;
  int r = ensure_batch(p, Mpad);
  if (r) return r;
  MCK(cudaMemsetAsync(p->xin + (size_t)M * MLP_IN, 0, (size_t)(Mpad - M) * MLP_IN * sizeof(__nv_bfloat16), st));
  MCK(cudaMemcpyAsync(p->xin, d_x, (size_t)M * MLP_IN * sizeof(__nv_bfloat16), cudaMemcpyDeviceToDevice, st));
  MCK(cudaMemcpyAsync(p->y, d_y, (size_t)M * sizeof(float), cudaMemcpyDeviceToDevice, st));
  MCK(cudaMemsetAsync(p->loss, 0, sizeof(float), st));
  r = forward(p, Mpad, st);
  if (r) return r;
  // output gradient (layer 4 pre-activation = output, no activation)
  k_nll<<<(Mpad + 255) / 256, 256, 0, st>>>(M, Mpad, p->z[MLP_LAYERS - 1], p->y, p->dz[MLP_LAYERS - 1], p->loss);
  MCK(cudaGetLastError());
  // weight transposes for dX (bf16): wt block of layer l is (kin x nout)
  for (int l = 1; l < MLP_LAYERS; ++l) {
    dim3 g((p->kin[l] + 31) / 32, (p->nout[l] + 31) / 32);
    k_transpose_bf16<<<g, dim3(32, 8), 0, st>>>(p->nout[l], p->kin[l], p->wb + p->woff[l], p->kin[l],
                                                 p->wt + p->woff[l], p->nout[l]);
  }
  MCK(cudaGetLastError());
  for (int l = MLP_LAYERS - 1; l >= 0; --l) {
    const int nl = p->nout[l], kl = p->kin[l];
    const __nv_bfloat16* xl = (l == 0) ? p->xin : p->h[l - 1];
    if (l < MLP_LAYERS - 1) {  // dZ = dH * GELU'(Z)
      const int n = Mpad * nl;
      k_gelu_back<<<(n + 255) / 256, 256, 0, st>>>(n, p->z[l], p->dh, p->dz[l]);
    }
    // dW[nl x kl] = dZ^T[nl x M] X[M x kl]: A = dZ^T (nl rows, padded to 128), B = X^T (kl x M)
    const int Mw = (nl + TM - 1) / TM * TM;
    if (Mw > nl) MCK(cudaMemsetAsync(p->dzt + (size_t)nl * Mpad, 0, (size_t)(Mw - nl) * Mpad * 2, st));
    {
      dim3 g1((nl + 31) / 32, (Mpad + 31) / 32);
      k_transpose_bf16<<<g1, dim3(32, 8), 0, st>>>(Mpad, nl, p->dz[l], nl, p->dzt, Mpad);
      dim3 g2((kl + 31) / 32, (Mpad + 31) / 32);
      k_transpose_bf16<<<g2, dim3(32, 8), 0, st>>>(Mpad, kl, xl, kl, p->xt, Mpad);
    }
    float* gw = p->g + p->woff[l];
    r = gemm(p, Mw, kl, Mpad, p->dzt, Mpad, p->xt, Mpad, nullptr, 0, Mw == nl ? gw : p->gscr, nullptr, kl, st);
    if (r) return r;
    if (Mw != nl) MCK(cudaMemcpyAsync(gw, p->gscr, (size_t)nl * kl * sizeof(float), cudaMemcpyDeviceToDevice, st));
    k_colsum<<<(nl + 127) / 128, 128, 0, st>>>(Mpad, nl, p->dz[l], p->g + p->boff[l]);
    if (l > 0) {  // dX[M x kl] = dZ[M x nl] W[nl x kl]: A = dZ, B = W^T (kl x nl)
      r = gemm(p, Mpad, kl, nl, p->dz[l], nl, p->wt + p->woff[l], nl, nullptr, 0, nullptr, p->dh, kl, st);
      if (r) return r;
    }
  }
  MCK(cudaGetLastError());
  if (lr > 0.0f) {
    p->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)p->step), c2 = 1.0f - powf(b2, (float)p->step);
    k_adam<<<(int)((p->nparam + 255) / 256), 256, 0, st>>>((int)p->nparam, p->w, p->g, p->m, p->v, lr, b1, b2, 1e-8f,
                                                           c1, c2, p->mask, p->wb);
  p->wsw_dirty = true;
    MCK(cudaGetLastError());
  }
  if (loss_out) {
    MCK(cudaMemcpyAsync(loss_out, p->loss, sizeof(float), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
  }
  int herr = 0;
  MCK(cudaMemcpyAsync(&herr, p->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  if (herr) { p->msg = "tensor-core wait timed out"; return SWDK_E_CUDA; }
  return SWDK_OK;
}

// gradients of the last train step (host copy, nparam floats)
int swdk_mlp_get_grads(swdk_mlp* p, float* host, int64_t n) {
  if (!p || !host || n != (int64_t)p->nparam) return SWDK_E_ARG;
  MCK(cudaSetDevice(p->device));
  MCK(cudaMemcpy(host, p->g, p->nparam * sizeof(float), cudaMemcpyDeviceToHost));
  return SWDK_OK;
}

// checkpoint: magic, version, nparam, step, FP32 weights, Adam m, v, checksum
int swdk_mlp_save(swdk_mlp* p, const char* path) {
  if (!p || !path) return SWDK_E_ARG;
  MCK(cudaSetDevice(p->device));
  std::vector<float> buf(3 * p->nparam);
  MCK(cudaMemcpy(buf.data(), p->w, p->nparam * 4, cudaMemcpyDeviceToHost));
  MCK(cudaMemcpy(buf.data() + p->nparam, p->m, p->nparam * 4, cudaMemcpyDeviceToHost));
  MCK(cudaMemcpy(buf.data() + 2 * p->nparam, p->v, p->nparam * 4, cudaMemcpyDeviceToHost));
  uint64_t sum = 1469598103934665603ull;
  const unsigned char* b = (const unsigned char*)buf.data();
  for (size_t i = 0; i < buf.size() * 4; ++i) sum = (sum ^ b[i]) * 1099511628211ull;
  FILE* f = fopen(path, "wb");
  if (!f) return SWDK_E_ARG;
  const uint32_t magic = 0x4D4C5053u, version = 1;
  const uint64_t np = p->nparam;
  const int32_t step = p->step;
  bool ok = fwrite(&magic, 4, 1, f) == 1 && fwrite(&version, 4, 1, f) == 1 && fwrite(&np, 8, 1, f) == 1 &&
            fwrite(&step, 4, 1, f) == 1 && fwrite(buf.data(), 4, buf.size(), f) == buf.size() &&
            fwrite(&sum, 8, 1, f) == 1;
  fclose(f);
  return ok ? SWDK_OK : SWDK_E_ARG;
}

int swdk_mlp_load(swdk_mlp* p, const char* path) {
  if (!p || !path) return SWDK_E_ARG;
  MCK(cudaSetDevice(p->device));
  FILE* f = fopen(path, "rb");
  if (!f) return SWDK_E_ARG;
  uint32_t magic = 0, version = 0;
  uint64_t np = 0, sum = 0;
  int32_t step = 0;
  std::vector<float> buf(3 * p->nparam);
  bool ok = fread(&magic, 4, 1, f) == 1 && fread(&version, 4, 1, f) == 1 && fread(&np, 8, 1, f) == 1 &&
            magic == 0x4D4C5053u && version == 1 && np == p->nparam && fread(&step, 4, 1, f) == 1 &&
            fread(buf.data(), 4, buf.size(), f) == buf.size() && fread(&sum, 8, 1, f) == 1;
  fclose(f);
  if (!ok) { p->msg = "bad checkpoint"; return SWDK_E_ARG; }
  uint64_t s2 = 1469598103934665603ull;
  const unsigned char* b = (const unsigned char*)buf.data();
  for (size_t i = 0; i < buf.size() * 4; ++i) s2 = (s2 ^ b[i]) * 1099511628211ull;
  if (s2 != sum) { p->msg = "checkpoint checksum mismatch"; return SWDK_E_ARG; }
  MCK(cudaMemcpy(p->w, buf.data(), p->nparam * 4, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(p->m, buf.data() + p->nparam, p->nparam * 4, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(p->v, buf.data() + 2 * p->nparam, p->nparam * 4, cudaMemcpyHostToDevice));
  p->step = step;
  k_to_bf16<<<(int)((p->nparam + 255) / 256), 256, 0, p->stream>>>((int)p->nparam, p->w, p->wb);
  p->wsw_dirty = true;
  MCK(cudaGetLastError());
  MCK(cudaStreamSynchronize(p->stream));
  return SWDK_OK;
}

const char* swdk_mlp_last_error(const swdk_mlp* p) { return p ? p->msg.c_str() : "null"; }

}  // extern "C"
