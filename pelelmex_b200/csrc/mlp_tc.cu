// mlp_tc.cu -- BF16 tensor-core (tcgen05) GEMM with fused epilogues for the
// chemistry surrogate MLP (inference and training), plus the elementwise
// kernels of its training step.
//
//   C[M, N] = epi(A[M, K] . B[N, K]^T + bias[N])
//
// A and B are BF16, row-major with K contiguous ("K-major" for both UMMA
// operands).  One CTA of 128 threads owns a 128-row tile of C at a time
// (persistent over tiles).  Operand tiles are staged by the CTA's threads into
// shared memory in the UMMA canonical no-swizzle K-major layout: 8-row x
// 16-byte core matrices, core matrices of one 8-row group contiguous along K
// (LBO = 128 B), row groups SBO = KC / 8 * 128 B apart.  One thread issues
// tcgen05.mma (kind::f16, M = 128, N = the N tile, K = 16 per instruction)
// accumulating in tensor memory (FP32, 128 lanes x N columns);
// tcgen05.commit signals an mbarrier when the MMAs are done; each warp then
// reads its 32 lanes (rows) of the accumulator with tcgen05.ld and applies
// the epilogue.  When K and N fit (K <= 256, N <= 256) B is staged once per
// CTA and stays resident across row tiles (the weights of one layer);
// otherwise B is re-staged per K chunk.
//
// Every wait on the mbarrier is bounded; on timeout the kernel raises a flag
// in err (read by the host) and stops issuing work.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/b200chem.h"

namespace b200 {
namespace mlp {

constexpr int kTileM = 128;
constexpr int kThreads = 128;

enum Epilogue : int {
  kEpiF32 = 0,        // C fp32 = acc + bias
  kEpiBf16 = 1,       // C bf16 = acc + bias
  kEpiGeluBf16 = 2,   // C bf16 = gelu(acc + bias); aux fp32 = acc + bias (pre-activation, may be null)
  kEpiDGeluBf16 = 3,  // C bf16 = acc * gelu'(aux[pre-activation])  (backward through GELU)
};

struct GemmArgs {
  const __nv_bfloat16* A;
  const __nv_bfloat16* B;
  long long lda, ldb;  // row strides (elements)
  int M, N, K;         // M % 128 == 0, N % 16 == 0, K % 16 == 0
  void* C;
  long long ldc;
  const float* bias;   // [N] or null
  float* aux;          // epilogue side input/output [M][ldc]
  int epi;
  int n_valid;         // columns of C actually written (<= N)
  int* err;            // raised on an mbarrier timeout
  int vec_ok;          // C (and aux) rows 16-byte aligned: vector epilogue
  int stages;          // A stages of the warp-specialised kernel (<= kMaxStages)
  int arep;            // A holds arep * K columns: arep BF16 terms of one K-wide operand
                       // (hi, then lo), all multiplied by the same B and summed
  int split_out;       // BF16 outputs as two terms: hi at column c, lo = bf16(v - hi) at c + N
};

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory matrix descriptor, no swizzle, K-major.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for this architecture
  // base offset 0, legacy LBO mode, layout type 0 = no swizzle
  return d;
}

// Instruction descriptor: BF16 x BF16 -> F32, both operands K-major, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4)                          // D format F32
         | (1u << 7)                        // A format BF16
         | (1u << 10)                       // B format BF16
         | ((uint32_t)(N >> 3) << 17)       // N / 8
         | ((uint32_t)(M >> 4) << 24);      // M / 16
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// Bounded wait: returns false after ~2^22 polls (seconds) without completion.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase) {
  for (int i = 0; i < (1 << 22); ++i) {
    if (mbar_try_wait(bar, phase)) return true;
    if (i > 64) __nanosleep(64);
  }
  return false;
}

__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
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

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 32 consecutive FP32 accumulator columns of this thread's lane (row).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Two 32-column accumulator loads in flight, one wait: tcgen05.ld is
// asynchronous until tcgen05.wait::ld, whose "+r" operands keep every use of
// the loaded registers after it.
__device__ __forceinline__ void tmem_ld32_async(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld(uint32_t (&r)[32]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                 "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                 "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
               :
               : "memory");
}
// an empty asm that claims to rewrite r: orders the uses of a second buffer
// after the wait that covered it
__device__ __forceinline__ void tmem_claim(uint32_t (&r)[32]) {
  asm volatile(""
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                 "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                 "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
               :
               : "memory");
}

// ------------------------------------------------------------ staging
// rows x kc block of a K-contiguous bf16 matrix into the canonical layout:
// element (r, k) at (r / 8) * (kc / 8) * 128 + (k / 8) * 128 + (r % 8) * 16
// + (k % 8) * 2 bytes.  Rows >= rows_valid are zero.  16-byte copies.
// The copies are asynchronous (cp.async, 16 bytes each, rows >= rows_valid
// zero-filled through a source size of 0), so every thread has all of its
// copies in flight at once; stage_wait() completes them.
__device__ __forceinline__ void stage_tile(unsigned char* dst, const __nv_bfloat16* src, long long ld, int rows,
                                           int rows_valid, int k0, int kc) {
  const int chunks_per_row = kc / 8;
  const int total = rows * chunks_per_row;
  for (int c = threadIdx.x; c < total; c += blockDim.x) {
    const int r = c / chunks_per_row, kb = c % chunks_per_row;
    const bool valid = r < rows_valid;
    const __nv_bfloat16* g = src + (valid ? (long long)r * ld + k0 + kb * 8 : 0);
    const int off = (r >> 3) * chunks_per_row * 128 + kb * 128 + (r & 7) * 16;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst + off)), "l"(g),
                 "r"(valid ? 16 : 0)
                 : "memory");
  }
}

__device__ __forceinline__ void stage_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// hardware tanh approximation (MUFU); ample for BF16 activations
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ float gelu(float x) {
  // tanh form of GELU (Hendrycks & Gimpel 2016)
  const float k0 = 0.7978845608028654f, k1 = 0.044715f;
  return 0.5f * x * (1.0f + tanh_fast(k0 * (x + k1 * x * x * x)));
}

__device__ __forceinline__ float gelu_grad(float x) {
  const float k0 = 0.7978845608028654f, k1 = 0.044715f;
  const float u = k0 * (x + k1 * x * x * x);
  const float t = tanh_fast(u);
  const float du = k0 * (1.0f + 3.0f * k1 * x * x);
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * du;
}

// Epilogue of one 32-column accumulator chunk of row `row`, columns col0 ..
// col0 + 31 of C: bias, then the fused activation, then the stores.
// bias: g.bias itself or a shared-memory copy of it (null: no bias).
__device__ __forceinline__ void epilogue_chunk(const GemmArgs& g, int row, int col0, float (&v)[32],
                                               const float* bias) {
  if (bias) {
#pragma unroll
    for (int i = 0; i < 32; ++i)
      if (col0 + i < g.n_valid) v[i] += bias[col0 + i];
  }
  // full 32-column chunk with 16-byte aligned rows: vector loads / stores
  const bool full = (col0 + 32 <= g.n_valid) && g.vec_ok;
  if (g.epi == kEpiF32) {
    float* C = reinterpret_cast<float*>(g.C) + (long long)row * g.ldc + col0;
    if (full) {
#pragma unroll
      for (int q = 0; q < 8; ++q)
        reinterpret_cast<float4*>(C)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    } else if (g.vec_ok) {
      // ragged end: 16-byte stores for whole groups of four, then scalars
      const int cnt = g.n_valid - col0;
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (4 * q + 4 <= cnt)
          reinterpret_cast<float4*>(C)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
#pragma unroll
      for (int i = 0; i < 32; ++i)
        if (i >= (cnt & ~3) && i < cnt) C[i] = v[i];
    } else {
#pragma unroll
      for (int i = 0; i < 32; ++i)
        if (col0 + i < g.n_valid) C[i] = v[i];
    }
  } else {
    __nv_bfloat16* C = reinterpret_cast<__nv_bfloat16*>(g.C) + (long long)row * g.ldc + col0;
    if (g.epi == kEpiGeluBf16) {
      // pre-activations: row stride ldc, or N when C is written in two terms
      float* P = g.aux ? g.aux + (long long)row * (g.split_out ? (long long)g.N : g.ldc) + col0 : nullptr;
      if (P && full) {
#pragma unroll
        for (int q = 0; q < 8; ++q)
          reinterpret_cast<float4*>(P)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
      } else if (P) {
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (col0 + i < g.n_valid) P[i] = v[i];
      }
#pragma unroll
      for (int i = 0; i < 32; ++i) v[i] = gelu(v[i]);
    } else if (g.epi == kEpiDGeluBf16) {
      const float* P = g.aux + (long long)row * g.ldc + col0;
      if (full) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const float4 p = reinterpret_cast<const float4*>(P)[q];
          v[4 * q] *= gelu_grad(p.x);
          v[4 * q + 1] *= gelu_grad(p.y);
          v[4 * q + 2] *= gelu_grad(p.z);
          v[4 * q + 3] *= gelu_grad(p.w);
        }
      } else {
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (col0 + i < g.n_valid) v[i] *= gelu_grad(P[i]);
      }
    }
    if (full) {
      uint32_t w[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
        w[q] = *reinterpret_cast<const uint32_t*>(&b2);
        if (g.split_out) {
          // keep the rounding residual for the low term
          const float2 hf = __bfloat1622float2(b2);
          v[2 * q] -= hf.x;
          v[2 * q + 1] -= hf.y;
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
        reinterpret_cast<uint4*>(C)[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
      if (g.split_out) {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
          w[q] = *reinterpret_cast<const uint32_t*>(&b2);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
          reinterpret_cast<uint4*>(C + g.N)[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
      }
    } else {
#pragma unroll
      for (int i = 0; i < 32; ++i)
        if (col0 + i < g.n_valid) {
          const __nv_bfloat16 hi = __float2bfloat16_rn(v[i]);
          C[i] = hi;
          if (g.split_out) C[g.N + i] = __float2bfloat16_rn(v[i] - __bfloat162float(hi));
        }
    }
  }
}

// ------------------------------------------------------------ GEMM kernel
__global__ void __launch_bounds__(kThreads, 1) gemm_bf16_tc(GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base_s;
  __shared__ int abort_s;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool resident = (g.K <= 256 && g.N <= 256);
  const int NT = g.N <= 256 ? g.N : 256;          // N tile
  const int KC = resident ? g.K : 64;             // K chunk
  unsigned char* As = smem;                        // [128 x KC]
  unsigned char* Bs = smem + kTileM * KC * 2;      // [NT x KC]
  const uint32_t ncols = NT <= 32 ? 32 : (NT <= 64 ? 64 : (NT <= 128 ? 128 : 256));
  if (warp == 0) tmem_alloc(&tmem_base_s, ncols);
  if (tid == 0) {
    mbar_init(&bar, 1);
    abort_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_s;
  const uint32_t idesc = umma_idesc_bf16(kTileM, NT);
  const int mtiles = g.M / kTileM, ntiles = (g.N + NT - 1) / NT;
  uint32_t phase = 0;
  bool b_loaded = false;
  for (int t = blockIdx.x; t < mtiles * ntiles; t += gridDim.x) {
    const int mt = t / ntiles, nt = t % ntiles;
    const int n0 = nt * NT;
    for (int k0 = 0; k0 < g.K; k0 += KC) {
      stage_tile(As, g.A + (long long)mt * kTileM * g.lda, g.lda, kTileM, kTileM, k0, KC);
      if (!resident || !b_loaded) stage_tile(Bs, g.B + (long long)n0 * g.ldb, g.ldb, NT, NT, k0, KC);
      b_loaded = true;
      stage_wait();
      fence_async_smem();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        const uint32_t a0 = smem_u32(As), b0 = smem_u32(Bs);
        const uint32_t sbo = (uint32_t)(KC / 8) * 128u;
        for (int ks = 0; ks < KC / 16; ++ks) {
          const uint64_t ad = umma_desc(a0 + ks * 256u, 128u, sbo);
          const uint64_t bd = umma_desc(b0 + ks * 256u, 128u, sbo);
          umma_bf16(tmem, ad, bd, idesc, (k0 > 0 || ks > 0) ? 1u : 0u);
        }
        umma_commit(&bar);
      }
      // the staged operands are reused only after the MMAs that read them are done
      const bool ok = mbar_wait_bounded(&bar, phase);
      phase ^= 1u;
      if (!ok) abort_s = 1;
      __syncthreads();
      if (abort_s) break;
    }
    if (abort_s) break;
    tc_fence_after();
    // epilogue: warp w owns accumulator lanes (rows) 32w .. 32w + 31
    const int row = mt * kTileM + warp * 32 + lane;
    for (int c0 = 0; c0 < NT; c0 += 32) {
      float v[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      epilogue_chunk(g, row, n0 + c0, v, g.bias);
    }
    // all warps have read the accumulator before the next tile overwrites it
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  if (abort_s && tid == 0 && g.err) atomicExch(g.err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

// ------------------------------------------------ warp-specialised GEMM
// For B resident in shared memory (K <= 256, N <= 256): the weights of one
// layer times 128-row tiles of activations, pipelined across tiles.
//
//   warp 0 (one lane)  TMA producer: B once, then every A tile in K chunks
//                      into a ring of g.stages shared-memory stages
//   warp 1 (one lane)  MMA issuer: tcgen05.mma of each chunk into one of two
//                      TMEM accumulators (tile i uses accumulator i % 2)
//   warps 2..9         epilogue: tcgen05.ld of accumulator i % 2 while the
//                      MMAs of tile i + 1 run into the other one (two warps
//                      per TMEM lane quarter, alternate 32-column chunks)
//
// Operands arrive by 2-D TMA boxes of 8 columns (16 bytes) x all rows of the
// tile: one box is one 16-byte K group of every row, rows 16 bytes apart,
// i.e. a column of UMMA core matrices.  A stage holds KC / 8 such groups
// `rows * 16` bytes apart (the descriptor's leading byte offset; 8-row groups
// are 128 bytes apart, its stride byte offset).  Barriers: full / empty per
// stage, acc_full / acc_empty per accumulator; every wait is bounded and a
// timeout stops all roles.
#ifndef B200_EPI_PER_QUARTER
#define B200_EPI_PER_QUARTER 2
#endif
constexpr int kEpiPerQuarter = B200_EPI_PER_QUARTER;     // epilogue warps per TMEM lane quarter
constexpr int kEpiWarps = 4 * kEpiPerQuarter;
constexpr int kWsThreads = 64 + 32 * kEpiWarps;
constexpr int kMaxStages = 8;
constexpr int kWsMinSmem = 120 * 1024;  // one CTA per SM, so its TMEM columns are free

struct WsBars {
  uint64_t full[kMaxStages], empty[kMaxStages], acc_full[2], acc_empty[2], b_full, done;
  uint32_t tmem;
  int abort;
};

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// 2-D TMA load of box (x, y) of `map` into shared memory, completing on bar.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Bounded wait that also gives up once another role has aborted (abort may
// be null: wait out the bound regardless).
__device__ __forceinline__ bool ws_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  for (int i = 0; i < (1 << 22); ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (abort && (i & 255) == 255 && *abort) return false;
    if (i > 64) __nanosleep(64);
  }
  if (abort) *abort = 1;
  return false;
}

__global__ void __launch_bounds__(kWsThreads, 1)
    gemm_bf16_ws(GemmArgs g, const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ WsBars sb;
  __shared__ float bias_s[256];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int NT = g.N;                       // one N tile (N <= 256)
  const int NT32 = (NT + 31) & ~31;         // accumulator 1 starts at column NT32
  const int KC = g.K <= 64 ? g.K : 64;      // K chunk of one stage
  const int nchunk = g.K * g.arep / KC;     // A chunks per tile (all terms)
  const int bchunks = g.K / KC;             // B chunks (one term)
  unsigned char* Bs = smem;                                    // [K/8][NT][16 B]
  unsigned char* As = smem + ((NT * g.K * 2 + 1023) & ~1023);  // S x [KC/8][128][16 B]
  const int stage_bytes = kTileM * KC * 2;
  const uint32_t ncols = 2 * NT32 <= 32 ? 32 : (2 * NT32 <= 64 ? 64 : (2 * NT32 <= 128 ? 128 : (2 * NT32 <= 256 ? 256 : 512)));
  if (warp == 1) tmem_alloc(&sb.tmem, ncols);
  const int S = g.stages;
  if (tid == 0) {
    for (int i = 0; i < S; ++i) {
      mbar_init(&sb.full[i], 1);
      mbar_init(&sb.empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&sb.acc_full[i], 1);
      mbar_init(&sb.acc_empty[i], kEpiWarps);
    }
    mbar_init(&sb.b_full, 1);
    mbar_init(&sb.done, 1);
    sb.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  volatile int* abort = &sb.abort;
  const uint32_t tmem = sb.tmem;
  const int mtiles = g.M / kTileM;
  int issued = 0;  // producer: A chunks issued
  if (warp == 0) {
    if (lane == 0) {
      // B once: K/8 boxes of {8 columns, NT rows}
      mbar_expect_tx(&sb.b_full, (uint32_t)(NT * g.K * 2));
      for (int kg = 0; kg < g.K / 8; ++kg) tma_load_2d(Bs + kg * NT * 16, &tmB, kg * 8, 0, &sb.b_full);
      for (int t = blockIdx.x; t < mtiles && !*abort; t += gridDim.x) {
        for (int c = 0; c < nchunk; ++c) {
          const int s = issued % S;
          const uint32_t use = (uint32_t)(issued / S);
          if (!ws_wait(&sb.empty[s], (use & 1u) ^ 1u, abort)) break;
          mbar_expect_tx(&sb.full[s], (uint32_t)stage_bytes);
          unsigned char* dst = As + s * stage_bytes;
          for (int kg = 0; kg < KC / 8; ++kg)
            tma_load_2d(dst + kg * kTileM * 16, &tmA, c * KC + kg * 8, t * kTileM, &sb.full[s]);
          ++issued;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = umma_idesc_bf16(kTileM, NT);
      bool ok = ws_wait(&sb.b_full, 0u, abort);
      tc_fence_after();
      const uint32_t b0 = smem_u32(Bs);
      const uint32_t b_lbo = (uint32_t)NT * 16u;       // between 16-byte K groups of B
      const uint32_t a_lbo = (uint32_t)kTileM * 16u;   // ... of an A stage
      int q = 0, i = 0;
      for (int t = blockIdx.x; ok && t < mtiles; t += gridDim.x, ++i) {
        const int acc = i & 1;
        const uint32_t ause = (uint32_t)(i >> 1);
        if (!ws_wait(&sb.acc_empty[acc], (ause & 1u) ^ 1u, abort)) break;
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(acc * NT32);
        for (int c = 0; c < nchunk; ++c, ++q) {
          const int s = q % S;
          const uint32_t use = (uint32_t)(q / S);
          if (!ws_wait(&sb.full[s], use & 1u, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = smem_u32(As + s * stage_bytes);
          for (int ks = 0; ks < KC / 16; ++ks) {
            const uint64_t ad = umma_desc(a0 + (uint32_t)(2 * ks) * a_lbo, a_lbo, 128u);
            const uint64_t bd = umma_desc(b0 + (uint32_t)((c % bchunks) * (KC / 8) + 2 * ks) * b_lbo, b_lbo, 128u);
            umma_bf16(d, ad, bd, idesc, (c > 0 || ks > 0) ? 1u : 0u);
          }
          umma_commit(&sb.empty[s]);  // the stage is free once these MMAs have read it
        }
        if (ok) umma_commit(&sb.acc_full[acc]);
      }
      // every MMA this thread issued has completed before TMEM is released
      umma_commit(&sb.done);
      ws_wait(&sb.done, 0u, nullptr);
    }
  } else {
    // epilogue warps: warp w reads TMEM lanes 32 * (w % 4) .. + 31, the
    // 32-column chunks c0 = 32 * part, 32 * (part + kEpiPerQuarter), ...
    const int quarter = warp & 3;
    const int part = (warp - 2) >> 2;
    for (int c = tid - 64; c < NT; c += 32 * kEpiWarps) bias_s[c] = g.bias ? g.bias[c] : 0.f;
    asm volatile("bar.sync 1, %0;" ::"r"(32 * kEpiWarps) : "memory");  // epilogue warps only
    const float* bias = g.bias ? bias_s : nullptr;
    int i = 0;
    for (int t = blockIdx.x; t < mtiles; t += gridDim.x, ++i) {
      const int acc = i & 1;
      const uint32_t ause = (uint32_t)(i >> 1);
      int ok = 1;
      if (lane == 0) ok = ws_wait(&sb.acc_full[acc], ause & 1u, abort) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      tc_fence_after();
      const int row = t * kTileM + quarter * 32 + lane;
      const uint32_t tq = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * NT32);
      constexpr int step = 32 * kEpiPerQuarter;
      for (int c0 = 32 * part; c0 < NT; c0 += 2 * step) {
        // two chunks per wait: c0 and c0 + step
        const bool two = c0 + step < NT;
        uint32_t ra[32], rb[32];
        tmem_ld32_async(tq + (uint32_t)c0, ra);
        if (two) tmem_ld32_async(tq + (uint32_t)(c0 + step), rb);
        tmem_wait_ld(ra);
        tmem_claim(rb);
        float v[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(ra[k]);
        epilogue_chunk(g, row, c0, v, bias);
        if (two) {
#pragma unroll
          for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(rb[k]);
          epilogue_chunk(g, row, c0 + step, v, bias);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&sb.acc_empty[acc]);
    }
  }
  // copies still in flight after an abort land before the CTA exits
  if (warp == 0 && lane == 0) {
    ws_wait(&sb.b_full, 0u, nullptr);
    for (int j = issued - 1; j >= 0 && j >= issued - S; --j)
      ws_wait(&sb.full[j % S], (uint32_t)((j / S) & 1), nullptr);
  }
  tc_fence_before();
  __syncthreads();
  if (*abort && tid == 0 && g.err) atomicExch(g.err, 1);
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, ncols);
  }
}

// Fused Adam step of one parameter tensor [rows][cols] (FP32 master copy),
// Kingma & Ba 2015: m = b1 m + (1 - b1) g, v = b2 v + (1 - b2) g^2,
// p -= lr (m / c1) / (sqrt(v / c2) + eps) with the bias corrections c1, c2;
// then the BF16 copies the GEMMs read: wb (same layout) and wbt (transposed,
// [cols][rows]), each optional.
__global__ void adam_step(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, long long n, int cols, float lr, float b1, float b2, float eps,
                          float c1, float c2, __nv_bfloat16* __restrict__ wb, __nv_bfloat16* __restrict__ wbt,
                          int rows) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    const __nv_bfloat16 b = __float2bfloat16_rn(pi);
    if (wb) wb[i] = b;
    if (wbt) {
      const long long r = i / cols, c = i % cols;
      wbt[c * rows + r] = b;
    }
  }
}

// Self-test of the bounded waits: one thread waits on an mbarrier that
// nothing arrives at, with the same polling loop as the GEMM roles but a
// caller-given bound, then raises the error flag and returns -- the path a
// GEMM takes when a copy or an MMA never completes.
__global__ void bounded_wait_selftest(int* err, int polls) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    bool done = false;
    for (int i = 0; i < polls && !done; ++i) {
      done = mbar_try_wait(&bar, 0u);
      if (!done && i > 64) __nanosleep(64);
    }
    if (!done) atomicExch(err, 1);
  }
}

}  // namespace mlp
}  // namespace b200

// ------------------------------------------------------------------ C ABI
using namespace b200::mlp;

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// Tensor map of a row-major BF16 operand [rows][cols] (row stride ld
// elements) read in boxes of 8 columns x box_rows rows.
int make_operand_map(CUtensorMap* map, const void* base, int cols, int rows, long long ld, int box_rows) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return -1;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {8, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -1;
}

}  // namespace

extern "C" int b200chem_mlp_gemm_bf16(const void* A, long long lda, const void* B, long long ldb, int M, int N, int K,
                                      void* C, long long ldc, const float* bias, float* aux, int epi, int n_valid,
                                      int* err, void* stream) {
  if (!A || !B || !C || M <= 0 || N <= 0 || K <= 0) return -1;
  if (M % kTileM || N % 16 || K % 16 || (N > 256 && N % 256)) return -1;
  const int arep = (epi & B200CHEM_GEMM_SPLIT_A) ? 2 : 1;
  const int split_out = (epi & B200CHEM_GEMM_SPLIT_OUT) ? 1 : 0;
  epi &= 0xF;
  if (epi < kEpiF32 || epi > kEpiDGeluBf16) return -1;
  if (split_out && epi != kEpiBf16 && epi != kEpiGeluBf16) return -1;
  if (split_out && (N > 256 || ldc < 2LL * N)) return -1;
  if (lda < (long long)arep * K) return -1;
  if (epi == kEpiDGeluBf16 && !aux) return -1;
  if (lda % 8 || ldb % 8) return -1;  // 16-byte staging loads
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15) return -1;
  GemmArgs g;
  g.A = static_cast<const __nv_bfloat16*>(A);
  g.B = static_cast<const __nv_bfloat16*>(B);
  g.lda = lda;
  g.ldb = ldb;
  g.M = M;
  g.N = N;
  g.K = K;
  g.C = C;
  g.ldc = ldc;
  g.bias = bias;
  g.aux = aux;
  g.epi = epi;
  g.n_valid = n_valid > 0 ? n_valid : N;
  g.err = err;
  g.arep = arep;
  g.split_out = split_out;
  {
    const size_t esz = (epi == kEpiF32) ? 4 : 2;
    const bool cal = (reinterpret_cast<uintptr_t>(C) & 15) == 0 && ((ldc * (long long)esz) & 15) == 0;
    const long long ldaux = split_out ? N : ldc;
    const bool aal = !aux || ((reinterpret_cast<uintptr_t>(aux) & 15) == 0 && ((ldaux * 4) & 15) == 0);
    g.vec_ok = (cal && aal) ? 1 : 0;
  }
  const bool resident = (K <= 256 && N <= 256);
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (resident && (K <= 64 || K % 64 == 0)) {
    // warp-specialised pipeline: TMA producer, MMA issuer, epilogue warps
    CUtensorMap ta, tb;
    if (make_operand_map(&ta, A, arep * K, M, lda, kTileM) || make_operand_map(&tb, B, K, N, ldb, N)) return -2;
    const int KC = K <= 64 ? K : 64;
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const int b_bytes = (N * K * 2 + 1023) & ~1023, stage_bytes = kTileM * KC * 2;
    // as many A stages as fit beside B (2 KB left for the static barriers and bias)
    int stages = (optin - 2048 - b_bytes) / stage_bytes;
    if (stages > kMaxStages) stages = kMaxStages;
    if (stages < 2) return -2;
    g.stages = stages;
    int smem = b_bytes + stages * stage_bytes;
    if (smem < kWsMinSmem) smem = kWsMinSmem;
    if (cudaFuncSetAttribute(gemm_bf16_ws, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
      return -2;
    const int tiles = M / kTileM;
    const int grid = tiles < sms ? tiles : sms;
    gemm_bf16_ws<<<grid, kWsThreads, smem, st>>>(g, ta, tb);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
  }
  if (arep != 1) return -1;  // two-term A operands need the warp-specialised kernel
  const int NT = N <= 256 ? N : 256;
  const int KC = resident ? K : 64;
  const int smem = kTileM * KC * 2 + NT * KC * 2;
  cudaError_t e = cudaFuncSetAttribute(gemm_bf16_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return -2;
  const int tiles = (M / kTileM) * ((N + NT - 1) / NT);
  const int grid = tiles < sms ? tiles : sms;
  gemm_bf16_tc<<<grid, kThreads, smem, st>>>(g);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

extern "C" int b200chem_mlp_adam(float* p, const float* g, float* m, float* v, int rows, int cols, float lr,
                                 float beta1, float beta2, float eps, int step, void* wb, void* wbt, void* stream) {
  if (!p || !g || !m || !v || rows <= 0 || cols <= 0 || step < 1 || !(lr >= 0.0f)) return -1;
  const long long n = (long long)rows * cols;
  const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
  const long long blocks = (n + 255) / 256;
  adam_step<<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      p, g, m, v, n, cols, lr, beta1, beta2, eps, c1, c2, static_cast<__nv_bfloat16*>(wb),
      static_cast<__nv_bfloat16*>(wbt), rows);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

extern "C" int b200chem_selftest_bounded_wait(int* err, int polls, void* stream) {
  if (!err || polls < 1 || polls > (1 << 22)) return -1;
  bounded_wait_selftest<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(err, polls);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}
