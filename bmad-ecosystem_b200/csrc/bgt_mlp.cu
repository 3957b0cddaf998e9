// bgt_mlp.cu -- survival classifier for pruning dynamic-aperture scans:
// feature extraction from tracked particles, a 64-256-256-256-1 MLP whose
// hidden layers are tcgen05 tensor-core GEMMs (BF16 operands, FP32
// accumulators in tensor memory), the output layer / loss / Adam on CUDA
// cores.  C ABI in include/bgt_mlp.h.  No counterpart in the reference.
//
// GEMM kernel (gemm_kernel<NT, EPI, BRES>): C = A[M][K] . B[NT][K]^T with
// both operands K-major (row-major, K contiguous), in 128 x NT output tiles
// (NT = 256, or 64 for the first layer's weight gradient), optionally split
// over K (weight gradients over the batch: each split writes its own FP32
// partial tile).  Persistent: min(tiles, SMs) CTAs walk the tiles in a
// static round robin.  BRES (one split, K <= 256: the forward and
// backward-data layers, where B is the layer's weights): B is loaded into
// shared memory once per CTA and only A streams through the ring.  Ten
// warps, each with one job:
//   warp 0     TMA producer: one lane issues cp.async.bulk.tensor loads of
//              the 128 x 64 block of A and the NT x 64 block of B into a
//              ring of shared-memory stages (128-byte swizzle, the canonical
//              K-major layout the MMA reads), completing on the stage's
//              "full" mbarrier;
//   warp 1     MMA issuer: owns the tensor memory; one lane waits for a full
//              stage, issues four tcgen05.mma (M=128, N=NT, K=16) into the
//              tile's accumulator and commits them to the stage's "empty"
//              mbarrier (the producer refills it when they complete); after
//              the tile's last block it commits to the accumulator's "full"
//              mbarrier;
//   warps 2-9  epilogue: each warp owns the 32 tensor-memory lanes (tile
//              rows) of its warp index mod 4 and half of the columns; it
//              reads 64 FP32 columns at a time with tcgen05.ld, applies the
//              layer's epilogue (bias from shared memory; the ReLU mask
//              requested before the tensor-memory load), writes each 32 x 32
//              block into its swizzled shared-memory staging buffer and
//              stores it with a TMA tensor store.
// The accumulator is double-buffered in tensor memory (2 x NT columns), so
// the epilogue of one tile runs while the MMAs of the next tile do.
// Epilogues:
//   EPI_FWD  bias + ReLU -> bf16 row-major and (optionally) a transposed copy
//   EPI_BWD  ReLU mask of the previous activation -> bf16 row-major / transposed
//   EPI_F32  FP32 tile (the test GEMM; split-K partials of weight gradients)
// Every TMA load is a plain per-CTA load of this GPU's own memory: each CTA
// loads its own tiles, none is shared across a cluster.
// Every mbarrier wait is bounded (%globaltimer, 2 s by default).  A role
// whose wait runs out sets the error flag and leaves its loop; the roles
// waiting on it then run out too.  Before the tensor memory is freed the MMA
// lane waits (bounded) for its own MMAs and the producer for its own loads,
// so nothing is in flight when the CTA exits.
#include <cuda.h>
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
#ifndef BGT_GEMM_EPI_WARPS
#define BGT_GEMM_EPI_WARPS 8
#endif
constexpr int EPI_WARPS = BGT_GEMM_EPI_WARPS;  // 4 or 8: one or two warps per tensor-memory lane quarter
constexpr int THREADS = 64 + 32 * EPI_WARPS;   // producer warp, MMA warp, epilogue warps
constexpr int H = BGT_MLP_HIDDEN;
constexpr int IN = BGT_MLP_IN;
constexpr int KSPLIT = 128;  // fewest samples per split-K chunk of a weight gradient

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

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
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

// TMA: 2-D tile load into this CTA's shared memory, completing on an
// mbarrier, and 2-D tile store from shared memory in a bulk group
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int32_t x, int32_t y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int32_t x, int32_t y, uint32_t src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(src)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// at most N of this thread's store groups still reading shared memory
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;\n" ::"n"(N) : "memory");
}
// all of this thread's store groups complete
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void prefetch_map(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
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

// 64 consecutive FP32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, uint32_t (&r)[64]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, "
      "%32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, "
      "%48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
        "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
        "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
        "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
        "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// Shared-memory matrix descriptor, K-major, 128-byte swizzle: start address
// (>> 4), leading byte offset 1 (unused for swizzled K-major), stride byte
// offset 1024 B between 8-row atoms, descriptor version 1, layout type 2.
// The TMA's 128-byte swizzle writes exactly this layout: row r of a block
// at r * 128 bytes, its 16-byte chunk c at chunk c ^ (r % 8).
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
  const float* bias;   // EPI_FWD: [N]
  bf16* out_t;         // optional transposed copy [N][ldt] (EPI_FWD / EPI_BWD)
  int64_t ldt;
  const bf16* mask;    // EPI_BWD: previous activation, row-major [M][ldm]
  int64_t ldm;
};

// Shared memory of one CTA: [stationary B: K <= 256, one split only]
// [ring of STAGES stages: A block, and the B block when B is not stationary]
// [one 32 x 32 output staging buffer per epilogue warp] + alignment slack.
template <int NT, bool BRES>
struct GemmCfg {
  static constexpr uint32_t A_BYTES = BM * BK * 2;
  static constexpr uint32_t B_BYTES = NT * BK * 2;
  static constexpr int BRES_BLOCKS = 4;  // K blocks of a stationary B (K <= 256)
  static constexpr uint32_t BRES_BYTES = BRES ? BRES_BLOCKS * B_BYTES : 0;
  static constexpr uint32_t STAGE_BYTES = BRES ? A_BYTES : A_BYTES + B_BYTES;
  static constexpr uint32_t EPI_BUF = 4096;  // 32 x 32 FP32 (or bf16) output block
  static constexpr uint32_t EPI_BYTES = EPI_WARPS * EPI_BUF;
  static constexpr uint32_t TMEM_COLS = 2 * NT;
  static constexpr int COLS_PER_WARP = NT / (EPI_WARPS / 4);  // accumulator columns one epilogue warp drains
  // as many stages as fit (at most 6), leaving 2 KB for the static shared
  // memory and 1 KB of alignment slack
  static constexpr int STAGES_FIT = (int)((232448u - 2048u - EPI_BYTES - BRES_BYTES) / STAGE_BYTES);
  static constexpr int STAGES = STAGES_FIT < 6 ? STAGES_FIT : 6;
  static constexpr int SMEM = BRES_BYTES + STAGES * STAGE_BYTES + EPI_BYTES + 1024;
};
static_assert(EPI_WARPS == 4 || EPI_WARPS == 8, "epilogue warps");
static_assert(GemmCfg<256, false>::STAGES >= 4 && GemmCfg<256, true>::STAGES >= 4 &&
                  GemmCfg<64, false>::COLS_PER_WARP >= 32,
              "GEMM configuration");
static_assert(GemmCfg<256, false>::SMEM <= 230400 && GemmCfg<256, true>::SMEM <= 230400, "shared memory per CTA");

__device__ int g_gemm_error;

// Tile t of a (m_tiles x splits) grid: rows mt * 128, K blocks [kb0, kb1)
// of split sp.  Every split has at least one K block (host check).
struct TileIdx {
  int mt, sp, kb0, kb1;
};
__device__ __forceinline__ TileIdx tile_of(int t, int m_tiles, int splits, int kb_total) {
  TileIdx r;
  r.mt = t % m_tiles;
  r.sp = t / m_tiles;
  r.kb0 = (int)((int64_t)r.sp * kb_total / splits);
  r.kb1 = (int)((int64_t)(r.sp + 1) * kb_total / splits);
  return r;
}

// BRES: B (the layer's weights in the forward and backward-data GEMMs) is
// loaded into shared memory once per CTA and stays there for all its tiles;
// only A streams through the ring.  Needs one split and K <= 256.
template <int NT, int EPI, bool BRES>
__global__ void __launch_bounds__(THREADS, 1)
    gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                const __grid_constant__ CUtensorMap tmC, int m_tiles, int splits, int kb_total, Epi ep, int* err,
                uint64_t wait_ns, int skip_mma) {
  using C = GemmCfg<NT, BRES>;
  constexpr int S = C::STAGES;
  constexpr uint32_t IDESC = idesc_bf16(BM, NT);
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[S], empty_bar[S], acc_full[2], acc_empty[2], done_bar, bres_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ __align__(16) float bias_s[EPI == EPI_FWD ? NT : 1];
  const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
  uint8_t* base_ptr = smem_raw + (base - smem_u32(smem_raw));
  const uint32_t ring = base + C::BRES_BYTES;  // stage s at ring + s * STAGE_BYTES
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n_tiles = m_tiles * splits;

  if (warp == 1) {
    tmem_alloc(smem_u32(&tmem_slot), C::TMEM_COLS);
    tmem_relinquish();
  }
  // Launched as a programmatic dependent of the previous kernel on the
  // stream: everything above runs while that kernel drains; no global
  // memory is touched before the previous grid has completed and its writes
  // are visible.  Then this grid lets the next one begin its own launch.
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  if (EPI == EPI_FWD) {
    for (int j = tid; j < NT; j += THREADS) bias_s[j] = ep.bias[j];
  }
  if (tid == 0) {
    for (int s = 0; s < S; s++) {
      mbar_init(smem_u32(&full_bar[s]), 1);
      mbar_init(smem_u32(&empty_bar[s]), 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(smem_u32(&acc_full[b]), 1);
      mbar_init(smem_u32(&acc_empty[b]), EPI_WARPS);  // one arrival per epilogue warp
    }
    mbar_init(smem_u32(&done_bar), 1);
    mbar_init(smem_u32(&bres_bar), 1);
    fence_mbar_init();
    prefetch_map(&tmA);
    prefetch_map(&tmB);
    prefetch_map(&tmC);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  bool ok = true;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      if (BRES) {
        // the stationary B: all its K blocks on one barrier
        mbar_arrive_expect_tx(smem_u32(&bres_bar), (uint32_t)kb_total * C::B_BYTES);
        for (int kb = 0; kb < kb_total; kb++)
          tma_load_2d(base + (uint32_t)kb * C::B_BYTES, &tmB, kb * BK, 0, smem_u32(&bres_bar));
      }
      int it = 0;  // ring loads issued
      for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
        const TileIdx ti = tile_of(t, m_tiles, splits, kb_total);
        for (int kb = ti.kb0; kb < ti.kb1; kb++) {
          const int s = it % S;
          const uint32_t ph = (uint32_t)(it / S) & 1u;
          // the stage's previous MMAs are done (the first pass waits on the
          // phase before the barrier's first, which counts as complete)
          if (!mbar_wait(smem_u32(&empty_bar[s]), ph ^ 1u, wait_ns)) {
            ok = false;
            break;
          }
          const uint32_t sa = ring + (uint32_t)s * C::STAGE_BYTES;
          const uint32_t fb = smem_u32(&full_bar[s]);
          mbar_arrive_expect_tx(fb, C::STAGE_BYTES);
          tma_load_2d(sa, &tmA, kb * BK, ti.mt * BM, fb);
          if (!BRES) tma_load_2d(sa + C::A_BYTES, &tmB, kb * BK, 0, fb);
          it++;
        }
      }
      // every load issued has landed before the CTA can exit (bounded)
      for (int s = 0; s < S && s < it; s++) {
        const int last = it - 1 - ((it - 1 - s) % S);  // the last load into stage s
        mbar_wait(smem_u32(&full_bar[s]), (uint32_t)(last / S) & 1u, wait_ns);
      }
      if (BRES) mbar_wait(smem_u32(&bres_bar), 0u, wait_ns);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      int it = 0, tc = 0;
      bool issued = false;
      if (BRES && !mbar_wait(smem_u32(&bres_bar), 0u, wait_ns)) ok = false;
      for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x, tc++) {
        const TileIdx ti = tile_of(t, m_tiles, splits, kb_total);
        const int b = tc & 1;
        const uint32_t tph = (uint32_t)(tc >> 1) & 1u;
        // the epilogue has drained this accumulator buffer
        if (!mbar_wait(smem_u32(&acc_empty[b]), tph ^ 1u, wait_ns)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(b * NT);
        for (int kb = ti.kb0; kb < ti.kb1; kb++, it++) {
          const int s = it % S;
          if (!mbar_wait(smem_u32(&full_bar[s]), (uint32_t)(it / S) & 1u, wait_ns)) {
            ok = false;
            break;
          }
          tc_fence_after();
          // skip_mma (tests only): no MMA and no commit are issued, so the
          // other roles' waits run out with nothing outstanding
          if (!skip_mma) {
            const uint32_t sa = ring + (uint32_t)s * C::STAGE_BYTES;
            const uint32_t sb = BRES ? base + (uint32_t)kb * C::B_BYTES : sa + C::A_BYTES;
#pragma unroll
            for (int k = 0; k < BK / 16; k++) {
              // K step of 16 bf16 = 32 bytes inside the 128-byte swizzle atom
              mma_bf16(d, sw128_desc(sa + k * 32), sw128_desc(sb + k * 32), IDESC,
                       (kb > ti.kb0 || k > 0) ? 1u : 0u);
            }
            mma_commit(smem_u32(&empty_bar[s]));
            issued = true;
          }
        }
        if (!ok) break;
        if (!skip_mma) mma_commit(smem_u32(&acc_full[b]));
      }
      // every MMA issued has completed before tensor memory is freed (bounded)
      if (issued) {
        mma_commit(smem_u32(&done_bar));
        mbar_wait(smem_u32(&done_bar), 0u, wait_ns);
      }
    }
  } else {
    // ---------------- epilogue ----------------
    const int q = warp & 3;  // tensor-memory lanes 32q .. 32q + 31 = tile rows
    const int col0 = ((warp - 2) >> 2) * C::COLS_PER_WARP;  // this warp's accumulator columns
    constexpr int GROUP = C::COLS_PER_WARP >= 64 ? 64 : 32;  // columns per tensor-memory load
    const uint32_t buf = ring + (uint32_t)S * C::STAGE_BYTES + (uint32_t)(warp - 2) * C::EPI_BUF;
    uint8_t* buf_ptr = base_ptr + (buf - base);
    int tc = 0;
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, tc++) {
      const TileIdx ti = tile_of(t, m_tiles, splits, kb_total);
      const int b = tc & 1;
      const int64_t row = (int64_t)ti.mt * BM + q * 32 + lane;  // this lane's output row
      const bool w = mbar_wait(smem_u32(&acc_full[b]), (uint32_t)(tc >> 1) & 1u, wait_ns);
      if (!__all_sync(0xffffffffu, w)) {
        ok = false;
        break;
      }
      tc_fence_after();
      // row of the 32 x 32 store box in the output map
      const int32_t ybox = (EPI == EPI_F32 ? ti.sp * m_tiles * BM : 0) + ti.mt * BM + q * 32;
      const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * NT);
#pragma unroll 1
      for (int g0 = col0; g0 < col0 + C::COLS_PER_WARP; g0 += GROUP) {
        // EPI_BWD: the ReLU mask of this group's columns, requested before
        // the tensor-memory load so the two latencies overlap
        uint4 mk[GROUP / 8];
        if (EPI == EPI_BWD) {
          const uint4* mp = reinterpret_cast<const uint4*>(ep.mask + row * ep.ldm + g0);
#pragma unroll
          for (int c = 0; c < GROUP / 8; c++) mk[c] = mp[c];
        }
        uint32_t r[64];
        if (GROUP == 64) {
          tmem_ld64(taddr + g0, r);
        } else {
          tmem_ld32(taddr + g0, *reinterpret_cast<uint32_t(*)[32]>(r));
        }
        if (g0 + GROUP == col0 + C::COLS_PER_WARP) {
          // this warp's part of the accumulator buffer is read: the next
          // tile's MMAs may overwrite it
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(smem_u32(&acc_empty[b]));
        }
#pragma unroll
        for (int h = 0; h < GROUP / 32; h++) {
          const int c0 = g0 + 32 * h;
          float v[32];
#pragma unroll
          for (int j = 0; j < 32; j++) v[j] = __uint_as_float(r[32 * h + j]);
          // the staging buffer's previous store has finished reading it
          if (lane == 0) bulk_wait_read<0>();
          __syncwarp();
          if (EPI == EPI_F32) {
            // 32 rows x 128 bytes, 128-byte swizzle: chunk c of row r at c ^ (r % 8)
#pragma unroll
            for (int c = 0; c < 8; c++)
              *reinterpret_cast<float4*>(buf_ptr + lane * 128 + ((c ^ (lane & 7)) << 4)) =
                  make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
          } else {
            if (EPI == EPI_FWD) {
#pragma unroll
              for (int c = 0; c < 8; c++) {
                const float4 bb = *reinterpret_cast<const float4*>(&bias_s[c0 + 4 * c]);
                v[4 * c] = fmaxf(v[4 * c] + bb.x, 0.0f);
                v[4 * c + 1] = fmaxf(v[4 * c + 1] + bb.y, 0.0f);
                v[4 * c + 2] = fmaxf(v[4 * c + 2] + bb.z, 0.0f);
                v[4 * c + 3] = fmaxf(v[4 * c + 3] + bb.w, 0.0f);
              }
            } else {
#pragma unroll
              for (int c = 0; c < 4; c++) {
                const bf16* hh = reinterpret_cast<const bf16*>(&mk[4 * h + c]);
#pragma unroll
                for (int j = 0; j < 8; j++)
                  if (!(__bfloat162float(hh[j]) > 0.0f)) v[8 * c + j] = 0.0f;
              }
            }
            uint4 pk[4];
            bf16* ph = reinterpret_cast<bf16*>(pk);
#pragma unroll
            for (int j = 0; j < 32; j++) ph[j] = __float2bfloat16_rn(v[j]);
            // 32 rows x 64 bytes, 64-byte swizzle: chunk c of row r at c ^ ((r / 2) % 4)
#pragma unroll
            for (int c = 0; c < 4; c++)
              *reinterpret_cast<uint4*>(buf_ptr + lane * 64 + ((c ^ ((lane >> 1) & 3)) << 4)) = pk[c];
            if (ep.out_t) {
#pragma unroll
              for (int j = 0; j < 32; j++) ep.out_t[(int64_t)(c0 + j) * ep.ldt + row] = ph[j];
            }
          }
          fence_proxy_async();
          __syncwarp();
          if (lane == 0) {
            tma_store_2d(&tmC, c0, ybox, buf);
            bulk_commit();
          }
        }
      }
    }
    if (lane == 0) bulk_wait_all();
  }
  if (!ok) atomicExch(err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, C::TMEM_COLS);
  }
}

// ---------------------------------------------------------------------------
// Tensor maps (driver entry point, resolved once through the runtime)

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = []() -> EncodeTiledFn {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// 2-D map of a row-major matrix: `rows` rows of `cols` elements, `ld`
// elements apart; boxes of box_rows x box_cols
static bool make_map(CUtensorMap* map, CUtensorMapDataType dt, size_t esize, const void* ptr, uint64_t cols,
                     uint64_t rows, uint64_t ld, uint32_t box_cols, uint32_t box_rows, CUtensorMapSwizzle sw) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return false;
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {ld * esize};
  const cuuint32_t box[2] = {box_cols, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return enc(map, dt, 2, const_cast<void*>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static int sm_count() {
  int dev = 0, n = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 148;
}

template <int NT, int EPI, bool BRES>
static cudaError_t launch_gemm_kernel(const CUtensorMap& ma, const CUtensorMap& mb, const CUtensorMap& mc, int m_tiles,
                                      int splits, int kb_total, const Epi& ep, int* err, cudaStream_t st,
                                      uint64_t wait_ns, int skip_mma) {
  using C = GemmCfg<NT, BRES>;
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    cudaError_t e =
        cudaFuncSetAttribute(gemm_kernel<NT, EPI, BRES>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
    if (e != cudaSuccess) return e;
    attr_set[dev & 63] = true;
  }
  const int grid = std::min(m_tiles * splits, sm_count());
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(THREADS);
  cfg.dynamicSmemBytes = C::SMEM;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, gemm_kernel<NT, EPI, BRES>, ma, mb, mc, m_tiles, splits, kb_total, ep, err,
                            wait_ns, skip_mma);
}

// C = A . B^T over K = k: A [a_rows][lda] bf16 (a_rows a multiple of 128),
// B [NT][ldb] bf16, k a multiple of 64 split into `splits` chunks of whole
// 64-blocks.  Output: EPI_F32 -> out FP32 [splits][a_rows][NT];
// EPI_FWD / EPI_BWD -> out bf16 [a_rows][ldo] (columns 0..NT-1).  With one
// split and K <= 256 the kernel keeps B stationary in shared memory.
template <int NT, int EPI>
static cudaError_t launch_gemm(const bf16* A, int64_t lda, int64_t a_rows, const bf16* B, int64_t ldb, int64_t k,
                               int splits, void* out, int64_t ldo, const Epi& ep, int* err, cudaStream_t st,
                               uint64_t wait_ns = 2000000000ull, int skip_mma = 0) {
  const int m_tiles = (int)(a_rows / BM);
  const int kb_total = (int)(k / BK);
  if (m_tiles <= 0 || kb_total <= 0 || splits <= 0 || splits > kb_total || a_rows % BM || k % BK)
    return cudaErrorInvalidValue;
  CUtensorMap ma, mb, mc;
  bool good = make_map(&ma, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, A, (uint64_t)k, (uint64_t)a_rows, (uint64_t)lda,
                       BK, BM, CU_TENSOR_MAP_SWIZZLE_128B) &&
              make_map(&mb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, B, (uint64_t)k, (uint64_t)NT, (uint64_t)ldb, BK, NT,
                       CU_TENSOR_MAP_SWIZZLE_128B);
  if (EPI == EPI_F32)
    good = good && make_map(&mc, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, out, (uint64_t)NT,
                            (uint64_t)splits * (uint64_t)a_rows, (uint64_t)ldo, 32, 32, CU_TENSOR_MAP_SWIZZLE_128B);
  else
    good = good && make_map(&mc, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, out, (uint64_t)NT, (uint64_t)a_rows,
                            (uint64_t)ldo, 32, 32, CU_TENSOR_MAP_SWIZZLE_64B);
  if (!good) return cudaErrorInvalidValue;
  if (splits == 1 && kb_total <= GemmCfg<NT, true>::BRES_BLOCKS)
    return launch_gemm_kernel<NT, EPI, true>(ma, mb, mc, m_tiles, splits, kb_total, ep, err, st, wait_ns, skip_mma);
  return launch_gemm_kernel<NT, EPI, false>(ma, mb, mc, m_tiles, splits, kb_total, ep, err, st, wait_ns, skip_mma);
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
  const int64_t ldt = m->max_batch;
  Epi e{};
  e.bias = m->params + OFF_B1;
  e.out_t = training ? m->a1t : nullptr;
  e.ldt = ldt;
  MCU(m, (launch_gemm<256, EPI_FWD>(X, IN, n, m->w1, IN, IN, 1, m->a1, H, e, m->d_err, st)));
  e.bias = m->params + OFF_B2;
  e.out_t = training ? m->a2t : nullptr;
  MCU(m, (launch_gemm<256, EPI_FWD>(m->a1, H, n, m->w2, H, H, 1, m->a2, H, e, m->d_err, st)));
  e.bias = m->params + OFF_B3;
  e.out_t = nullptr;
  MCU(m, (launch_gemm<256, EPI_FWD>(m->a2, H, n, m->w3, H, H, 1, m->a3, H, e, m->d_err, st)));
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
  MCU(m, cudaMemsetAsync(m->scalars, 0, sizeof(float), st));
  transpose_in_kernel<<<(unsigned)((B + 255) / 256), 256, 0, st>>>(X, B, m->xt, ldt);
  m->launches++;
  int rc = forward_rows(m, X, B, true, label, 1.0f / (float)B, nullptr, st);
  if (rc) return rc;
  // dZ2 = (dZ3 . W3) * relu'(A2), dZ1 = (dZ2 . W2) * relu'(A1)
  Epi e{};
  e.ldt = ldt;
  e.ldm = H;
  e.out_t = m->dz2t;
  e.mask = m->a2;
  MCU(m, (launch_gemm<256, EPI_BWD>(m->dz3, H, B, m->w3t, H, H, 1, m->dz2, H, e, m->d_err, st)));
  e.out_t = m->dz1t;
  e.mask = m->a1;
  MCU(m, (launch_gemm<256, EPI_BWD>(m->dz2, H, B, m->w2t, H, H, 1, m->dz1, H, e, m->d_err, st)));
  // weight gradients dW = dZ^T . A_prev over the batch, split into one
  // chunk per CTA of a full wave (at least KSPLIT samples per chunk: the
  // partial buffer holds max_batch / KSPLIT chunks); the FP32 partials are
  // summed in a fixed order, so the gradients are deterministic
  const int splits = (int)std::max<int64_t>(1, std::min<int64_t>(B / KSPLIT, sm_count() / (H / BM)));
  Epi f{};
  struct G {
    const bf16* dzt;
    const bf16* at;
    int64_t off;
    int nt;
  } gs[3] = {{m->dz3t, m->a2t, OFF_W3, 256}, {m->dz2t, m->a1t, OFF_W2, 256}, {m->dz1t, m->xt, OFF_W1, 64}};
  for (const G& g : gs) {
    if (g.nt == 256)
      MCU(m, (launch_gemm<256, EPI_F32>(g.dzt, ldt, H, g.at, ldt, B, splits, m->partial, 256, f, m->d_err, st)));
    else
      MCU(m, (launch_gemm<64, EPI_F32>(g.dzt, ldt, H, g.at, ldt, B, splits, m->partial, 64, f, m->d_err, st)));
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
  const bf16* A = reinterpret_cast<const bf16*>(d_a);
  const bf16* B = reinterpret_cast<const bf16*>(d_b);
  cudaError_t ce = (n == 256)
                       ? launch_gemm<256, EPI_F32>(A, lda, m, B, ldb, k, 1, d_c, n, e, d_err, st, wait_ns, skip_mma)
                       : launch_gemm<64, EPI_F32>(A, lda, m, B, ldb, k, 1, d_c, n, e, d_err, st, wait_ns, skip_mma);
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
