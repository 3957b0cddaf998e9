// bgt_mlp.cu -- survival classifier for pruning dynamic-aperture scans:
// feature extraction from tracked particles, a 64-256-256-256-1 MLP whose
// hidden layers are tcgen05 tensor-core GEMMs (BF16 operands, FP32
// accumulators in tensor memory), the output layer / loss / Adam on CUDA
// cores.  C ABI in include/bgt_mlp.h.  No counterpart in the reference.
//
// GEMM kernel (gemm_kernel<NT, EPI>): one CTA of 128 threads computes a
// 128 x NT tile (NT = 256 or 64) of A[M][K] . B[N][K]^T, both operands
// K-major (row-major with K contiguous).  K advances in blocks of 64 bf16
// (128 bytes per row): each block of A (128 rows) and B (NT rows) is copied
// into shared memory with 16-byte cp.async in the canonical 128-byte-swizzled
// K-major layout (8-row atoms of 1024 bytes, 16-byte chunk c of row r stored
// at chunk c ^ (r % 8)), two stages deep.  One elected thread issues four
// tcgen05.mma (M=128, N=NT, K=16) per block and commits them to the stage's
// mbarrier; the stage is refilled only after that mbarrier completes.  The
// accumulator lives in NT tensor-memory columns (lane = tile row); the four
// warps read their 32 lanes with tcgen05.ld and run the epilogue:
//   EPI_FWD  bias + ReLU -> bf16 row-major and (optionally) transposed copies
//   EPI_BWD  ReLU mask of the previous activation -> bf16 row-major / transposed
//   EPI_F32  FP32 tile (split-K partials of weight gradients)
// Every mbarrier wait is bounded (2 s of %globaltimer); on expiry the kernel
// sets an error flag, waits once more (bounded) for its own MMAs, frees its
// tensor memory and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/bgt.h"
#include "../../include/bgt_mlp.h"

namespace bgt {
namespace mlp {

typedef __nv_bfloat16 bf16;

constexpr int BM = 128;
constexpr int BK = 64;
constexpr int THREADS = 128;
constexpr int H = BGT_MLP_HIDDEN;
constexpr int IN = BGT_MLP_IN;
constexpr int KSPLIT = 128;  // samples per split-K chunk of a weight gradient

// flat parameter layout
constexpr int64_t OFF_W1 = 0;
constexpr int64_t OFF_B1 = OFF_W1 + (int64_t)H * IN;
constexpr int64_t OFF_W2 = OFF_B1 + H;
constexpr int64_t OFF_B2 = OFF_W2 + (int64_t)H * H;
constexpr int64_t OFF_W3 = OFF_B2 + H;
constexpr int64_t OFF_B3 = OFF_W3 + (int64_t)H * H;
constexpr int64_t OFF_W4 = OFF_B3 + H;
constexpr int64_t OFF_B4 = OFF_W4 + H;
constexpr int64_t N_PARAMS = OFF_B4 + 1;
static_assert(N_PARAMS == BGT_MLP_N_PARAMS, "parameter layout");

enum { EPI_FWD = 0, EPI_BWD = 1, EPI_F32 = 2 };

// ---------------------------------------------------------------------------
// PTX wrappers

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// Wait for the phase of `parity` to complete; false after limit_ns.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > limit_ns) return false;
  }
  return true;
}

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(dst_smem), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// D[tmem] (+)= A[smem desc] . B[smem desc]^T, kind::f16 (bf16 in, f32 accumulate)
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// arrive (once) on `bar` when every MMA this thread issued so far has completed
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
               : "memory");
}
// 32 consecutive FP32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// Shared-memory matrix descriptor, K-major, 128-byte swizzle: start address
// (>> 4), leading byte offset 1 (unused for swizzled K-major), stride byte
// offset 1024 B between 8-row atoms, descriptor version 1, layout type 2.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
// Instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), A and
// B BF16 (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at 24.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// ---------------------------------------------------------------------------
// GEMM

struct Epi {
  const float* bias;        // EPI_FWD: [N]
  bf16* out;                // EPI_FWD / EPI_BWD: row-major [M][ldo]
  int64_t ldo;
  bf16* out_t;              // optional transposed copy [N][ldt]
  int64_t ldt;
  const bf16* mask;         // EPI_BWD: previous activation, row-major [M][ldm]
  int64_t ldm;
  float* out_f32;           // EPI_F32: [gridDim.y][M][N]
};

// rows x 64 bf16 block of a row-major matrix into swizzled shared memory
template <int ROWS>
__device__ __forceinline__ void load_block(uint32_t s_base, const bf16* g, int64_t ld, int64_t row0, int64_t k0,
                                           int tid) {
#pragma unroll 4
  for (int idx = tid; idx < ROWS * 8; idx += THREADS) {
    const int r = idx >> 3, c = idx & 7;
    const uint32_t dst = s_base + (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((c ^ (r & 7)) << 4));
    cp_async16(dst, g + (row0 + r) * ld + k0 + c * 8);
  }
}

__device__ int g_gemm_error;

template <int NT, int EPI>
__global__ void __launch_bounds__(THREADS, 1)
    gemm_kernel(const bf16* __restrict__ A, int64_t lda, const bf16* __restrict__ B, int64_t ldb, int k_blocks,
                Epi ep, int* err, uint64_t wait_ns, int skip_mma) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ uint32_t tmem_slot;
  constexpr uint32_t A_BYTES = BM * BK * 2;
  constexpr uint32_t B_BYTES = NT * BK * 2;
  constexpr uint32_t IDESC = idesc_bf16(BM, NT);
  const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
  const uint32_t sA0 = base, sB0 = base + A_BYTES, sA1 = base + A_BYTES + B_BYTES, sB1 = sA1 + A_BYTES;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t row0 = (int64_t)blockIdx.x * BM;
  const int64_t kbase = (int64_t)blockIdx.y * k_blocks * BK;
  const uint32_t bar0 = smem_u32(&bars[0]), bar1 = smem_u32(&bars[1]);

  if (warp == 0) {
    tmem_alloc(smem_u32(&tmem_slot), NT);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(bar0, 1);
    mbar_init(bar1, 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  bool ok = true;
  load_block<BM>(sA0, A, lda, row0, kbase, tid);
  load_block<NT>(sB0, B, ldb, 0, kbase, tid);
  cp_async_commit();
  for (int kb = 0; kb < k_blocks; kb++) {
    const int s = kb & 1;
    if (kb + 1 < k_blocks) {
      const int s1 = (kb + 1) & 1;
      if (kb >= 1) {
        // the MMAs of block kb-1 read stage s1: wait before refilling it
        // (the outcome is made CTA-uniform before anyone leaves the loop)
        const bool w = mbar_wait(s1 ? bar1 : bar0, ((kb - 1) >> 1) & 1, wait_ns);
        if (!__syncthreads_and(w)) {
          ok = false;
          break;
        }
      }
      load_block<BM>(s1 ? sA1 : sA0, A, lda, row0, kbase + (int64_t)(kb + 1) * BK, tid);
      load_block<NT>(s1 ? sB1 : sB0, B, ldb, 0, kbase + (int64_t)(kb + 1) * BK, tid);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    fence_proxy_async();
    __syncthreads();
    // skip_mma (tests only): no MMA and no commit are issued, so the
    // mbarrier waits run out with nothing outstanding
    if (tid == 0 && !skip_mma) {
      tc_fence_after();
      const uint32_t a_s = s ? sA1 : sA0, b_s = s ? sB1 : sB0;
#pragma unroll
      for (int k = 0; k < BK / 16; k++) {
        // K step of 16 bf16 = 32 bytes inside the 128-byte swizzle atom
        mma_bf16(tmem, sw128_desc(a_s + k * 32), sw128_desc(b_s + k * 32), IDESC, (kb > 0 || k > 0) ? 1u : 0u);
      }
      mma_commit(s ? bar1 : bar0);
    }
  }
  cp_async_wait<0>();
  const int last = k_blocks - 1;
  const uint32_t last_bar = (last & 1) ? bar1 : bar0;
  if (ok) ok = mbar_wait(last_bar, (last >> 1) & 1, wait_ns);
  ok = __syncthreads_and(ok);  // tcgen05.ld below is warp-collective
  if (!ok) {
    atomicExch(err, 1);
    // bounded second wait for the MMAs in flight before tensor memory is freed
    mbar_wait(last_bar, (last >> 1) & 1, wait_ns);
  }
  tc_fence_after();
  __syncwarp();
  if (ok) {
    const int64_t row = row0 + warp * 32 + lane;
    const uint32_t t_row = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int c0 = 0; c0 < NT; c0 += 32) {
      uint32_t r[32];
      tmem_ld32(t_row + c0, r);
      float v[32];
#pragma unroll
      for (int j = 0; j < 32; j++) v[j] = __uint_as_float(r[j]);
      if (EPI == EPI_F32) {
        float4* dst = reinterpret_cast<float4*>(ep.out_f32 + ((int64_t)blockIdx.y * gridDim.x * BM + row) * NT + c0);
#pragma unroll
        for (int q = 0; q < 8; q++) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
      } else {
        if (EPI == EPI_FWD) {
#pragma unroll
          for (int j = 0; j < 32; j++) v[j] = fmaxf(v[j] + ep.bias[c0 + j], 0.0f);
        } else {
          const uint4* mp = reinterpret_cast<const uint4*>(ep.mask + row * ep.ldm + c0);
#pragma unroll
          for (int q = 0; q < 4; q++) {
            uint4 u = mp[q];
            const bf16* h = reinterpret_cast<const bf16*>(&u);
#pragma unroll
            for (int j = 0; j < 8; j++)
              if (!(__bfloat162float(h[j]) > 0.0f)) v[8 * q + j] = 0.0f;
          }
        }
        uint4 pk[4];
        bf16* ph = reinterpret_cast<bf16*>(pk);
#pragma unroll
        for (int j = 0; j < 32; j++) ph[j] = __float2bfloat16_rn(v[j]);
        uint4* dst = reinterpret_cast<uint4*>(ep.out + row * ep.ldo + c0);
#pragma unroll
        for (int q = 0; q < 4; q++) dst[q] = pk[q];
        if (ep.out_t) {
#pragma unroll
          for (int j = 0; j < 32; j++) ep.out_t[(int64_t)(c0 + j) * ep.ldt + row] = ph[j];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, NT);
}

template <int NT>
constexpr int gemm_smem() {
  return 2 * (BM * BK * 2 + NT * BK * 2) + 1024;
}

template <int NT, int EPI>
static cudaError_t launch_gemm(const bf16* A, int64_t lda, const bf16* B, int64_t ldb, int m_tiles, int splits,
                               int k_blocks, const Epi& ep, int* err, cudaStream_t st,
                               uint64_t wait_ns = 2000000000ull, int skip_mma = 0) {
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    cudaError_t e =
        cudaFuncSetAttribute(gemm_kernel<NT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, gemm_smem<NT>());
    if (e != cudaSuccess) return e;
    attr_set[dev & 63] = true;
  }
  gemm_kernel<NT, EPI><<<dim3(m_tiles, splits), THREADS, gemm_smem<NT>(), st>>>(A, lda, B, ldb, k_blocks, ep, err, wait_ns,
                                                                              skip_mma);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// CUDA-core kernels

// output layer, probability, loss and its gradient; one warp per sample
__global__ void head_kernel(const bf16* __restrict__ A3, int64_t n, const float* __restrict__ w4,
                            const float* __restrict__ b4, const float* __restrict__ label, float inv_batch,
                            float* __restrict__ prob, float* __restrict__ dlogit, bf16* __restrict__ dz3,
                            bf16* __restrict__ dz3_t, int64_t ldt, float* __restrict__ loss_acc) {
  const int64_t s = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (s >= n) return;
  const uint4 u = *reinterpret_cast<const uint4*>(A3 + s * H + lane * 8);
  const bf16* a = reinterpret_cast<const bf16*>(&u);
  float w[8], av[8];
  float acc = 0.0f;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    w[j] = __bfloat162float(__float2bfloat16_rn(w4[lane * 8 + j]));
    av[j] = __bfloat162float(a[j]);
    acc += av[j] * w[j];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  const float z = acc + b4[0];
  const float p = 1.0f / (1.0f + expf(-z));
  if (prob && lane == 0) prob[s] = p;
  if (!label) return;
  const float y = label[s];
  const float g = (p - y) * inv_batch;
  if (lane == 0) {
    dlogit[s] = g;
    // binary cross-entropy in the softplus form
    const float l = fmaxf(z, 0.0f) - z * y + log1pf(expf(-fabsf(z)));
    atomicAdd(loss_acc, l * inv_batch);
  }
  uint4 out;
  bf16* o = reinterpret_cast<bf16*>(&out);
#pragma unroll
  for (int j = 0; j < 8; j++) o[j] = __float2bfloat16_rn(av[j] > 0.0f ? g * w[j] : 0.0f);
  *reinterpret_cast<uint4*>(dz3 + s * H + lane * 8) = out;
#pragma unroll
  for (int j = 0; j < 8; j++) dz3_t[(int64_t)(lane * 8 + j) * ldt + s] = o[j];
}

// partial[c][j] = sum over rows s of chunk c of w[s] * M[s][j] (w = 1 if NULL)
__global__ void colsum_kernel(const bf16* __restrict__ M, int64_t ldm, const float* __restrict__ w, int64_t n,
                              int rows_per_chunk, int ncols, float* __restrict__ partial) {
  const int j = threadIdx.x;
  const int64_t c = blockIdx.x;
  if (j >= ncols) return;
  const int64_t s0 = c * rows_per_chunk, s1 = min(n, s0 + rows_per_chunk);
  float acc = 0.0f;
  for (int64_t s = s0; s < s1; s++) acc += (w ? w[s] : 1.0f) * __bfloat162float(M[s * ldm + j]);
  partial[c * ncols + j] = acc;
}

// out[j] = sum_c partial[c][j], j < count
__global__ void reduce_kernel(const float* __restrict__ partial, int64_t n_chunks, int64_t count,
                              float* __restrict__ out) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= count) return;
  float acc = 0.0f;
  for (int64_t c = 0; c < n_chunks; c++) acc += partial[c * count + j];
  out[j] = acc;
}

// sum of the first n floats into out[0] (one block)
__global__ void sum_kernel(const float* __restrict__ x, int64_t n, float* __restrict__ out) {
  __shared__ float sh[256];
  float acc = 0.0f;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) acc += x[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = sh[0];
}

// Xt[k][s] = X[s][k]
__global__ void transpose_in_kernel(const bf16* __restrict__ X, int64_t n, bf16* __restrict__ Xt, int64_t ldt) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  for (int k = 0; k < IN; k++) Xt[(int64_t)k * ldt + s] = X[s * IN + k];
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float bc1,
                            float bc2) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// bf16 weights for the GEMMs: W (row-major [out][in]) and, for the hidden
// layers, W^T ([in][out]) for the backward pass
__global__ void pack_kernel(const float* __restrict__ p, bf16* __restrict__ w1, bf16* __restrict__ w2,
                            bf16* __restrict__ w2t, bf16* __restrict__ w3, bf16* __restrict__ w3t) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < (int64_t)H * IN) w1[i] = __float2bfloat16_rn(p[OFF_W1 + i]);
  if (i < (int64_t)H * H) {
    const int64_t o = i / H, k = i % H;
    const bf16 a = __float2bfloat16_rn(p[OFF_W2 + i]), b = __float2bfloat16_rn(p[OFF_W3 + i]);
    w2[i] = a;
    w3[i] = b;
    w2t[k * H + o] = a;
    w3t[k * H + o] = b;
  }
}

__global__ void features_kernel(const double* __restrict__ vec0, const double* __restrict__ vec, int64_t n,
                                int64_t stride, const int32_t* __restrict__ var, const double* __restrict__ table,
                                const float* __restrict__ mean, const float* __restrict__ inv_std,
                                float* __restrict__ raw, bf16* __restrict__ x) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* T = table + (int64_t)(var ? var[i] : 0) * BGT_MLP_VARIANT_COLS;
  double f[BGT_MLP_FEATURES];
  for (int k = 0; k < 6; k++) f[k] = vec0[k * stride + i] - T[k];
  for (int k = 0; k < 16; k++) f[6 + k] = T[14 + k];
  for (int k = 0; k < 6; k++) f[22 + k] = vec[k * stride + i] - T[k];
  const double dp = f[27];
  const double xb = f[22] - T[6] * dp, pxb = f[23] - T[7] * dp;
  const double yb = f[24] - T[8] * dp, pyb = f[25] - T[9] * dp;
  const double ba = T[10], aa = T[11], bb = T[12], ab = T[13];
  const double ja = 0.5 * ((1 + aa * aa) / ba * xb * xb + 2 * aa * xb * pxb + ba * pxb * pxb);
  const double jb = 0.5 * ((1 + ab * ab) / bb * yb * yb + 2 * ab * yb * pyb + bb * pyb * pyb);
  f[28] = sqrt(fmax(ja, 0.0));
  f[29] = sqrt(fmax(jb, 0.0));
  if (raw)
    for (int k = 0; k < BGT_MLP_FEATURES; k++) raw[i * BGT_MLP_FEATURES + k] = (float)f[k];
  if (x) {
    uint4 pk[IN / 8];
    bf16* h = reinterpret_cast<bf16*>(pk);
    for (int k = 0; k < IN; k++)
      h[k] = __float2bfloat16_rn(k < BGT_MLP_FEATURES ? ((float)f[k] - mean[k]) * inv_std[k] : 0.0f);
    uint4* dst = reinterpret_cast<uint4*>(x + i * IN);
    for (int q = 0; q < IN / 8; q++) dst[q] = pk[q];
  }
}

}  // namespace mlp
}  // namespace bgt

using namespace bgt::mlp;

struct bgt_mlp {
  int device = 0;
  int32_t max_batch = 0;
  std::string err;
  int64_t launches = 0;
  int64_t step = 0;
  float* params = nullptr;   // FP32 master
  float* grads = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  float* partial = nullptr;  // split-K / column-sum partials
  float* scalars = nullptr;  // [0] loss
  int* d_err = nullptr;
  bf16 *w1 = nullptr, *w2 = nullptr, *w2t = nullptr, *w3 = nullptr, *w3t = nullptr;
  bf16 *xt = nullptr, *a1 = nullptr, *a1t = nullptr, *a2 = nullptr, *a2t = nullptr, *a3 = nullptr;
  bf16 *dz1 = nullptr, *dz1t = nullptr, *dz2 = nullptr, *dz2t = nullptr, *dz3 = nullptr, *dz3t = nullptr;
  float* dlogit = nullptr;
  std::vector<void*> allocs;
};

static int mlp_err(bgt_mlp* m, int code, const std::string& msg) {
  if (m) m->err = msg;
  return code;
}

#define MCU(m, call)                                                                          \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return mlp_err((m), BGT_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

template <class T>
static cudaError_t mlp_alloc(bgt_mlp* m, T** p, size_t count) {
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e == cudaSuccess) m->allocs.push_back((void*)*p);
  return e;
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// splitmix64 -> uniform in [-1, 1)
static double mix_uniform(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * (1.0 / 4503599627370496.0) - 1.0;
}

static int pack_weights(bgt_mlp* m, cudaStream_t st) {
  pack_kernel<<<(H * H + 255) / 256, 256, 0, st>>>(m->params, m->w1, m->w2, m->w2t, m->w3, m->w3t);
  m->launches++;
  MCU(m, cudaGetLastError());
  return 0;
}

extern "C" {

int bgt_mlp_create(bgt_mlp** out, int32_t max_batch, uint64_t seed, int32_t device) {
  if (!out || max_batch <= 0 || max_batch % 128) return BGT_EINVAL;
  *out = nullptr;
  bgt_mlp* m = new bgt_mlp();
  m->device = device;
  m->max_batch = max_batch;
  cudaError_t e = cudaSetDevice(device);
  const int64_t B = max_batch;
  const int64_t n_split = B / KSPLIT;
  const int64_t partial = std::max<int64_t>(n_split * 2 * BM * H, (B / 128 + 1) * H);
  if (e == cudaSuccess) e = mlp_alloc(m, &m->params, N_PARAMS);
  if (e == cudaSuccess) e = mlp_alloc(m, &m->grads, N_PARAMS);
  if (e == cudaSuccess) e = mlp_alloc(m, &m->adam_m, N_PARAMS);
  if (e == cudaSuccess) e = mlp_alloc(m, &m->adam_v, N_PARAMS);
  if (e == cudaSuccess) e = mlp_alloc(m, &m->partial, partial);
  if (e == cudaSuccess) e = mlp_alloc(m, &m->scalars, 8);
  if (e == cudaSuccess) e = mlp_alloc(m, &m->d_err, 1);
  if (e == cudaSuccess) e = mlp_alloc(m, &m->w1, (size_t)H * IN);
  bf16** hh[] = {&m->w2, &m->w2t, &m->w3, &m->w3t};
  for (auto p : hh)
    if (e == cudaSuccess) e = mlp_alloc(m, p, (size_t)H * H);
  if (e == cudaSuccess) e = mlp_alloc(m, &m->xt, (size_t)IN * B);
  bf16** acts[] = {&m->a1, &m->a1t, &m->a2, &m->a2t, &m->a3, &m->dz1, &m->dz1t, &m->dz2, &m->dz2t, &m->dz3, &m->dz3t};
  for (auto p : acts)
    if (e == cudaSuccess) e = mlp_alloc(m, p, (size_t)H * B);
  if (e == cudaSuccess) e = mlp_alloc(m, &m->dlogit, B);
  if (e == cudaSuccess) e = cudaMemset(m->d_err, 0, sizeof(int));
  if (e != cudaSuccess) {
    fprintf(stderr, "bgt_mlp_create: %s\n", cudaGetErrorString(e));
    bgt_mlp_destroy(m);
    return BGT_ENOMEM;
  }
  // He-uniform weights, zero biases; the padded input columns stay zero
  std::vector<float> p(N_PARAMS, 0.0f);
  uint64_t s = seed;
  const double lim1 = std::sqrt(6.0 / BGT_MLP_FEATURES), limh = std::sqrt(6.0 / H);
  for (int o = 0; o < H; o++)
    for (int k = 0; k < BGT_MLP_FEATURES; k++) p[OFF_W1 + o * IN + k] = (float)(lim1 * mix_uniform(s));
  for (int64_t i = 0; i < (int64_t)H * H; i++) p[OFF_W2 + i] = (float)(limh * mix_uniform(s));
  for (int64_t i = 0; i < (int64_t)H * H; i++) p[OFF_W3 + i] = (float)(limh * mix_uniform(s));
  for (int i = 0; i < H; i++) p[OFF_W4 + i] = (float)(std::sqrt(3.0 / H) * mix_uniform(s));
  *out = m;
  return bgt_mlp_set_params(m, p.data());
}

int bgt_mlp_destroy(bgt_mlp* m) {
  if (!m) return 0;
  for (void* p : m->allocs) cudaFree(p);
  delete m;
  return 0;
}

const char* bgt_mlp_last_error(const bgt_mlp* m) { return m ? m->err.c_str() : "null handle"; }
int64_t bgt_mlp_launch_count(const bgt_mlp* m) { return m ? m->launches : 0; }

int bgt_mlp_get_params(bgt_mlp* m, float* params) {
  if (!m || !params) return BGT_EINVAL;
  MCU(m, cudaSetDevice(m->device));
  MCU(m, cudaDeviceSynchronize());
  MCU(m, cudaMemcpy(params, m->params, N_PARAMS * sizeof(float), cudaMemcpyDeviceToHost));
  return 0;
}

int bgt_mlp_set_params(bgt_mlp* m, const float* params) {
  if (!m || !params) return BGT_EINVAL;
  MCU(m, cudaSetDevice(m->device));
  MCU(m, cudaMemcpy(m->params, params, N_PARAMS * sizeof(float), cudaMemcpyHostToDevice));
  MCU(m, cudaMemset(m->adam_m, 0, N_PARAMS * sizeof(float)));
  MCU(m, cudaMemset(m->adam_v, 0, N_PARAMS * sizeof(float)));
  m->step = 0;
  int rc = pack_weights(m, 0);
  if (rc) return rc;
  MCU(m, cudaDeviceSynchronize());
  return 0;
}

}  // extern "C"

// forward pass of n rows (n % 128 == 0, n <= max_batch when training) from
// X bf16 [n][64]; training keeps the transposed copies for the weight
// gradients and runs the loss head with labels
static int forward_rows(bgt_mlp* m, const bf16* X, int64_t n, bool training, const float* label, float inv_batch,
                        float* prob, cudaStream_t st) {
  const int tiles = (int)(n / BM);
  const int64_t ldt = m->max_batch;
  Epi e{};
  e.bias = m->params + OFF_B1;
  e.out = m->a1;
  e.ldo = H;
  e.out_t = training ? m->a1t : nullptr;
  e.ldt = ldt;
  MCU(m, (launch_gemm<256, EPI_FWD>(X, IN, m->w1, IN, tiles, 1, IN / BK, e, m->d_err, st)));
  e.bias = m->params + OFF_B2;
  e.out = m->a2;
  e.out_t = training ? m->a2t : nullptr;
  MCU(m, (launch_gemm<256, EPI_FWD>(m->a1, H, m->w2, H, tiles, 1, H / BK, e, m->d_err, st)));
  e.bias = m->params + OFF_B3;
  e.out = m->a3;
  e.out_t = nullptr;
  MCU(m, (launch_gemm<256, EPI_FWD>(m->a2, H, m->w3, H, tiles, 1, H / BK, e, m->d_err, st)));
  const int64_t threads = n * 32;
  head_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
      m->a3, n, m->params + OFF_W4, m->params + OFF_B4, label, inv_batch, prob, m->dlogit, m->dz3, m->dz3t, ldt,
      m->scalars);
  m->launches += 4;
  MCU(m, cudaGetLastError());
  return 0;
}

static int check_error_flag(bgt_mlp* m) {
  int flag = 0;
  MCU(m, cudaMemcpy(&flag, m->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) return mlp_err(m, BGT_ETIMEOUT, "tensor-core GEMM: mbarrier wait timed out");
  return 0;
}

// gradients of the mean loss over one batch into m->grads
static int backward_batch(bgt_mlp* m, const bf16* X, const float* label, int32_t batch, cudaStream_t st) {
  const int64_t B = batch, ldt = m->max_batch;
  const int tiles = (int)(B / BM);
  MCU(m, cudaMemsetAsync(m->scalars, 0, sizeof(float), st));
  transpose_in_kernel<<<(unsigned)((B + 255) / 256), 256, 0, st>>>(X, B, m->xt, ldt);
  m->launches++;
  int rc = forward_rows(m, X, B, true, label, 1.0f / (float)B, nullptr, st);
  if (rc) return rc;
  // dZ2 = (dZ3 . W3) * relu'(A2), dZ1 = (dZ2 . W2) * relu'(A1)
  Epi e{};
  e.ldo = H;
  e.ldt = ldt;
  e.ldm = H;
  e.out = m->dz2;
  e.out_t = m->dz2t;
  e.mask = m->a2;
  MCU(m, (launch_gemm<256, EPI_BWD>(m->dz3, H, m->w3t, H, tiles, 1, H / BK, e, m->d_err, st)));
  e.out = m->dz1;
  e.out_t = m->dz1t;
  e.mask = m->a1;
  MCU(m, (launch_gemm<256, EPI_BWD>(m->dz2, H, m->w2t, H, tiles, 1, H / BK, e, m->d_err, st)));
  // weight gradients dW = dZ^T . A_prev, split over the batch
  const int splits = (int)(B / KSPLIT);
  Epi f{};
  f.out_f32 = m->partial;
  struct G {
    const bf16* dzt;
    const bf16* at;
    int64_t off;
    int nt;
  } gs[3] = {{m->dz3t, m->a2t, OFF_W3, 256}, {m->dz2t, m->a1t, OFF_W2, 256}, {m->dz1t, m->xt, OFF_W1, 64}};
  for (const G& g : gs) {
    if (g.nt == 256)
      MCU(m, (launch_gemm<256, EPI_F32>(g.dzt, ldt, g.at, ldt, H / BM, splits, KSPLIT / BK, f, m->d_err, st)));
    else
      MCU(m, (launch_gemm<64, EPI_F32>(g.dzt, ldt, g.at, ldt, H / BM, splits, KSPLIT / BK, f, m->d_err, st)));
    const int64_t count = (int64_t)H * g.nt;
    reduce_kernel<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(m->partial, splits, count, m->grads + g.off);
    m->launches += 2;
  }
  // bias gradients (column sums of dZ), output layer w4 = sum dlogit * A3, b4 = sum dlogit
  const int chunks = (int)(B / 128);
  struct C2 {
    const bf16* mat;
    const float* w;
    int64_t off;
  } cs[4] = {{m->dz1, nullptr, OFF_B1}, {m->dz2, nullptr, OFF_B2}, {m->dz3, nullptr, OFF_B3}, {m->a3, m->dlogit, OFF_W4}};
  for (const C2& c : cs) {
    colsum_kernel<<<chunks, 256, 0, st>>>(c.mat, H, c.w, B, 128, H, m->partial);
    reduce_kernel<<<1, 256, 0, st>>>(m->partial, chunks, H, m->grads + c.off);
    m->launches += 2;
  }
  sum_kernel<<<1, 256, 0, st>>>(m->dlogit, B, m->grads + OFF_B4);
  m->launches++;
  MCU(m, cudaGetLastError());
  return 0;
}

static int check_batch(bgt_mlp* m, const uint16_t* d_x, const float* d_label, int32_t batch) {
  if (!m || !d_x || !d_label) return BGT_EINVAL;
  if (batch <= 0 || batch % 128 || batch > m->max_batch)
    return mlp_err(m, BGT_EINVAL, "batch must be a positive multiple of 128 and <= max_batch");
  if (!aligned16(d_x)) return mlp_err(m, BGT_EINVAL, "d_x must be 16-byte aligned");
  return 0;
}

extern "C" {

int bgt_mlp_forward(bgt_mlp* m, const uint16_t* d_x, int64_t n, float* d_prob, void* stream) {
  if (!m || !d_x || !d_prob || n < 0) return BGT_EINVAL;
  if (n % 128) return mlp_err(m, BGT_EINVAL, "n must be a multiple of 128 (pad the input rows)");
  if (!aligned16(d_x)) return mlp_err(m, BGT_EINVAL, "d_x must be 16-byte aligned");
  MCU(m, cudaSetDevice(m->device));
  cudaStream_t st = (cudaStream_t)stream;
  const bf16* X = reinterpret_cast<const bf16*>(d_x);
  for (int64_t r0 = 0; r0 < n; r0 += m->max_batch) {
    const int64_t rows = std::min<int64_t>(m->max_batch, n - r0);
    int rc = forward_rows(m, X + r0 * IN, rows, false, nullptr, 0.0f, d_prob + r0, st);
    if (rc) return rc;
  }
  return 0;
}

int bgt_mlp_gradients(bgt_mlp* m, const uint16_t* d_x, const float* d_label, int32_t batch, float* d_grad,
                      float* loss, void* stream) {
  int rc = check_batch(m, d_x, d_label, batch);
  if (rc) return rc;
  MCU(m, cudaSetDevice(m->device));
  cudaStream_t st = (cudaStream_t)stream;
  rc = backward_batch(m, reinterpret_cast<const bf16*>(d_x), d_label, batch, st);
  if (rc) return rc;
  if (d_grad) MCU(m, cudaMemcpyAsync(d_grad, m->grads, N_PARAMS * sizeof(float), cudaMemcpyDeviceToDevice, st));
  if (loss) {
    MCU(m, cudaMemcpyAsync(loss, m->scalars, sizeof(float), cudaMemcpyDeviceToHost, st));
    MCU(m, cudaStreamSynchronize(st));
    return check_error_flag(m);
  }
  return 0;
}

int bgt_mlp_train_step(bgt_mlp* m, const uint16_t* d_x, const float* d_label, int32_t batch, float lr, float* loss,
                       void* stream) {
  int rc = check_batch(m, d_x, d_label, batch);
  if (rc) return rc;
  MCU(m, cudaSetDevice(m->device));
  cudaStream_t st = (cudaStream_t)stream;
  rc = backward_batch(m, reinterpret_cast<const bf16*>(d_x), d_label, batch, st);
  if (rc) return rc;
  m->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float bc1 = 1.0f - (float)std::pow((double)b1, (double)m->step);
  const float bc2 = 1.0f - (float)std::pow((double)b2, (double)m->step);
  adam_kernel<<<(unsigned)((N_PARAMS + 255) / 256), 256, 0, st>>>(m->params, m->grads, m->adam_m, m->adam_v,
                                                                    N_PARAMS, lr, b1, b2, 1e-8f, bc1, bc2);
  m->launches++;
  MCU(m, cudaGetLastError());
  rc = pack_weights(m, st);
  if (rc) return rc;
  if (loss) {
    MCU(m, cudaMemcpyAsync(loss, m->scalars, sizeof(float), cudaMemcpyDeviceToHost, st));
    MCU(m, cudaStreamSynchronize(st));
    return check_error_flag(m);
  }
  return 0;
}

int bgt_mlp_features(const double* d_vec0, const double* d_vec, int64_t n, int64_t stride, const int32_t* d_variant,
                     const double* d_table, int32_t n_variants, const float* d_mean, const float* d_inv_std,
                     float* d_raw, uint16_t* d_x, void* stream) {
  if (!d_vec0 || !d_vec || !d_table || n < 0 || stride < n || n_variants <= 0) return BGT_EINVAL;
  if (d_x && (!d_mean || !d_inv_std || !aligned16(d_x))) return BGT_EINVAL;
  if (n == 0) return 0;
  features_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      d_vec0, d_vec, n, stride, d_variant, d_table, d_mean, d_inv_std, d_raw, reinterpret_cast<bf16*>(d_x));
  return cudaGetLastError() == cudaSuccess ? 0 : BGT_ECUDA;
}

static int gemm_bf16(const uint16_t* d_a, int64_t lda, const uint16_t* d_b, int64_t ldb, int32_t m, int32_t n,
                     int32_t k, float* d_c, void* stream, uint64_t wait_ns, int skip_mma) {
  if (!d_a || !d_b || !d_c || m <= 0 || m % BM || (n != 64 && n != 256) || k <= 0 || k % BK) return BGT_EINVAL;
  if (lda < k || ldb < k || lda % 8 || ldb % 8 || !aligned16(d_a) || !aligned16(d_b) || !aligned16(d_c))
    return BGT_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  int* d_err = nullptr;
  if (cudaGetSymbolAddress((void**)&d_err, g_gemm_error) != cudaSuccess) return BGT_ECUDA;
  if (cudaMemsetAsync(d_err, 0, sizeof(int), st) != cudaSuccess) return BGT_ECUDA;
  Epi e{};
  e.out_f32 = d_c;
  const bf16* A = reinterpret_cast<const bf16*>(d_a);
  const bf16* B = reinterpret_cast<const bf16*>(d_b);
  cudaError_t ce = (n == 256)
                       ? launch_gemm<256, EPI_F32>(A, lda, B, ldb, m / BM, 1, k / BK, e, d_err, st, wait_ns, skip_mma)
                       : launch_gemm<64, EPI_F32>(A, lda, B, ldb, m / BM, 1, k / BK, e, d_err, st, wait_ns, skip_mma);
  if (ce != cudaSuccess) return BGT_ECUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return BGT_ECUDA;
  int flag = 0;
  if (cudaMemcpy(&flag, d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return BGT_ECUDA;
  return flag ? BGT_ETIMEOUT : 0;
}

int bgt_mlp_gemm_bf16(const uint16_t* d_a, int64_t lda, const uint16_t* d_b, int64_t ldb, int32_t m, int32_t n,
                      int32_t k, float* d_c, void* stream) {
  return gemm_bf16(d_a, lda, d_b, ldb, m, n, k, d_c, stream, 2000000000ull, 0);
}

int bgt_mlp_gemm_bf16_wait_test(const uint16_t* d_a, int64_t lda, const uint16_t* d_b, int64_t ldb, int32_t m,
                                int32_t n, int32_t k, float* d_c, uint32_t wait_limit_us, void* stream) {
  if (wait_limit_us == 0) return BGT_EINVAL;
  return gemm_bf16(d_a, lda, d_b, ldb, m, n, k, d_c, stream, (uint64_t)wait_limit_us * 1000ull, 1);
}

}  // extern "C"
