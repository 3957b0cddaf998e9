// bgt_track.cu -- host side of the FP64 tracker: the handle, the launch
// dispatch and the C ABI declared in include/bgt.h.  The element-table
// compiler is in bgt_compile.h, the kernel in bgt_kernel.cuh (instances in
// bgt_track_kernels.cu).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/bgt.h"
#include "bgt_compile.h"
#include "bgt_kernel.cuh"

// ===========================================================================
// Handle and C ABI

using namespace bgt;

// Resources of one call.  A call takes a context from its handle's pool (a
// new one when all are busy) and returns it when the call returns, so calls
// that run at the same time on one handle -- from OpenMP threads, as the
// reference calls track1 (bmad/multiparticle/beam_utils.f90:69-74) -- never
// share a stream, staging buffers or the kernel's tile counter.  `done`
// marks the end of the GPU work the context's last call enqueued; the next
// call orders its own stream after it before reusing the device scratch.
struct CallCtx {
  cudaStream_t st = nullptr;     // library-owned stream (host-buffer calls)
  cudaEvent_t done = nullptr;
  bool used = false;             // `done` has been recorded
  int32_t* d_scratch = nullptr;  // [0] tile counter, [1] error flag, [2] status read-back
  // device staging of host-buffer calls
  double* d_vec6 = nullptr;
  double* d_beta = nullptr;
  int32_t* d_i32 = nullptr;  // state, ixe, ixt, slot map, tile variant
  uint64_t* d_t = nullptr;   // particle times (binary128), cap of them
  int64_t cap = 0, cap_slots = 0, cap_tiles = 0;
  // pinned host staging of host-buffer calls
  unsigned char* h_pin = nullptr;
  size_t pin_bytes = 0;
  // device-buffer calls: grouping by variant (slot map, tile variant; per
  // variant first index / count / first slot (int64) plus a check flag)
  int32_t* d_grp = nullptr;
  int64_t* d_grp_v = nullptr;
  int64_t grp_cap_slots = 0, grp_cap_tiles = 0;
};

struct bgt_handle {
  int device = 0;
  int num_sms = 148;
  int32_t n_ele = 0, n_variants = 0;
  bgt_species sp{};
  Glob G{};
  int32_t table_dw = 0;
  std::vector<double> h_tables;
  std::vector<int64_t> h_table_off;
  double* d_tables = nullptr;
  int64_t* d_table_off = nullptr;
  int32_t* d_status = nullptr;  // sticky error flag of device-buffer calls (bgt_device_status)
  bool rare = false;            // some record needs the RARE kernels
  std::atomic<int64_t> launches{0};
  std::mutex mu;  // guards tuning and the context pool
  bgt_tuning tuning{128, 4, 0, 0, 0, 0, 0};
  std::vector<CallCtx*> pool, idle;
};

// Error messages are per thread: concurrent calls never overwrite each
// other's message.
static thread_local std::string t_err;

static int set_err(bgt_handle*, int code, const std::string& msg) {
  t_err = msg;
  return code;
}

#define CU(h, call)                                                                              \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return set_err((h), BGT_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));        \
  } while (0)

// Makes `dev` current for the scope of a call and restores the caller's
// current device on every return path.
struct DeviceGuard {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit DeviceGuard(int dev) {
    if ((err = cudaGetDevice(&prev)) != cudaSuccess) return;
    if (prev != dev) err = cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

static void free_ctx(CallCtx* c) {
  if (!c) return;
  if (c->st) cudaStreamDestroy(c->st);
  if (c->done) cudaEventDestroy(c->done);
  cudaFree(c->d_scratch);
  cudaFree(c->d_vec6);
  cudaFree(c->d_beta);
  cudaFree(c->d_i32);
  cudaFree(c->d_t);
  cudaFree(c->d_grp);
  cudaFree(c->d_grp_v);
  if (c->h_pin) cudaFreeHost(c->h_pin);
  delete c;
}

// A context of the handle's pool for this call (the handle's device current).
static int acquire_ctx(bgt_handle* h, CallCtx** out) {
  *out = nullptr;
  {
    std::lock_guard<std::mutex> g(h->mu);
    if (!h->idle.empty()) {
      *out = h->idle.back();
      h->idle.pop_back();
      return 0;
    }
  }
  CallCtx* c = new CallCtx();
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaMalloc(&c->d_scratch, 64)) != cudaSuccess ||
      (e = cudaMemsetAsync(c->d_scratch, 0, 64, c->st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(c->st)) != cudaSuccess) {
    free_ctx(c);
    return set_err(h, BGT_ECUDA, std::string("call context: ") + cudaGetErrorString(e));
  }
  std::lock_guard<std::mutex> g(h->mu);
  h->pool.push_back(c);
  *out = c;
  return 0;
}

// One call's lease on a context: `use(st)` orders stream st after the
// context's previous work; the destructor marks the end of this call's work
// on st and returns the context to the pool.
struct CtxLease {
  bgt_handle* h;
  CallCtx* c = nullptr;
  cudaStream_t st = nullptr;
  explicit CtxLease(bgt_handle* hh) : h(hh) {}
  int acquire() { return acquire_ctx(h, &c); }
  cudaError_t use(cudaStream_t s) {
    st = s;
    return c->used && s != c->st ? cudaStreamWaitEvent(s, c->done, 0) : cudaSuccess;
  }
  ~CtxLease() {
    if (!c) return;
    if (cudaEventRecord(c->done, st ? st : c->st) == cudaSuccess) c->used = true;
    std::lock_guard<std::mutex> g(h->mu);
    h->idle.push_back(c);
  }
};

static bgt_tuning get_tuning_locked(bgt_handle* h) {
  std::lock_guard<std::mutex> g(h->mu);
  return h->tuning;
}

// Dynamic shared memory of a launch: the table (unless read from global
// memory), the compaction stage (9 rows of BLOCK doubles, 11 with the
// particle times of the RARE instances) and the quadrupole memo.
static size_t smem_bytes(const bgt_handle* h, int block, bool compact, bool gtab, bool rare) {
  size_t b = gtab ? 0 : (size_t)h->table_dw * 8;
  if (compact) b += (size_t)(rare ? 11 : 9) * block * 8;
  b += (size_t)QMEMO_CLASSES * 13 * block * 8;
  return b;
}

namespace bgt {
TrackKernelGroup track_kernel_group_0();
TrackKernelGroup track_kernel_group_1();
TrackKernelGroup track_kernel_group_2();
TrackKernelGroup track_kernel_group_3();
TrackKernelGroup track_kernel_group_4();
TrackKernelGroup track_kernel_group_5();
TrackKernelGroup track_kernel_group_6();
TrackKernelGroup track_kernel_group_7();
TrackKernelGroup track_kernel_group_8();
TrackKernelGroup track_kernel_group_9();
TrackKernelGroup track_kernel_group(int g) {
  static TrackKernelGroup (*const groups[N_KERNEL_GROUPS])() = {
      track_kernel_group_0, track_kernel_group_1, track_kernel_group_2, track_kernel_group_3,
      track_kernel_group_4, track_kernel_group_5, track_kernel_group_6, track_kernel_group_7,
      track_kernel_group_8, track_kernel_group_9};
  return groups[g]();
}
}  // namespace bgt

// The compiled kernel for a shape, table mode and feature set, or nullptr.
static LaunchFn find_track_kernel(int block, int minb, int tmode, bool rare) {
  for (int g = 0; g < N_KERNEL_GROUPS; g++) {
    const TrackKernelGroup grp = track_kernel_group(g);
    for (int i = 0; i < grp.n; i++) {
      const TrackKernel& k = grp.kernels[i];
      if (k.block == block && k.minb == minb && k.tmode == tmode && k.rare == rare) return k.launch;
    }
  }
  return nullptr;
}

// Fill every kernel group's copy of the multipole coefficient tables on the
// current device, once per device (the values never change).
static cudaError_t upload_multipole_tables() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> g(mu);
  if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
  static double cm[BGT_MAXPOLE_DEV + 1][BGT_MAXPOLE_DEV + 1], cm0[BGT_MAXPOLE_DEV + 1][BGT_MAXPOLE_DEV + 1];
  host::c_multi_tables(cm, cm0);
  for (int gi = 0; gi < N_KERNEL_GROUPS; gi++) {
    e = track_kernel_group(gi).upload_cm(&cm[0][0], &cm0[0][0], sizeof(cm));
    if (e != cudaSuccess) return e;
  }
  if (dev >= 0 && dev < 64) done[dev] = true;
  return cudaSuccess;
}

// Wait bound of the staging mbarrier.
static uint64_t wait_ns_of(const bgt_tuning& t) {
  return t.wait_limit_us > 0 ? (uint64_t)t.wait_limit_us * 1000ull : 2000000000ull;
}

// The kernel instance for a tuning and a shared-memory need, with the
// placement of the table it implies; 0 or an error code.
static int pick_kernel(bgt_handle* h, const bgt_tuning& tun, bool compact, bool rare, LaunchFn* fn,
                       size_t* smem) {
  const int block = tun.threads_per_block;
  const bool fits = smem_bytes(h, block, compact, false, rare) <= SMEM_LIMIT;
  if (tun.table_mode == 1 && !fits)
    return set_err(h, BGT_ETOOLARGE, "element table does not fit in shared memory (table_mode 1)");
  const bool gtab = tun.table_mode >= 2 || !fits;
  const bool warp_sched = tun.table_mode == 3;
  *smem = smem_bytes(h, block, compact, gtab, rare);
  if (*smem > SMEM_LIMIT) return set_err(h, BGT_ETOOLARGE, "tracking state does not fit in shared memory");
  *fn = find_track_kernel(block, tun.blocks_per_sm, gtab ? (warp_sched ? 2 : 1) : 0, rare);
  if (!*fn) {
    if (gtab)
      return set_err(h, BGT_ETOOLARGE,
                     "element table read from global memory: tuning must be (128: 3,4,5) or (256: 2,3)");
    return set_err(h, BGT_EINVAL,
                   "tuning (threads_per_block, blocks_per_sm) must be one of (64: 8,10,12,16), "
                   "(128: 4,5,6,8), (256: 2,3,4)");
  }
  return 0;
}

// Enqueue tracking of slots on `st` with the call context's tile counter
// and error flag.
static int enqueue_track(bgt_handle* h, const bgt_tuning& tun, CallCtx* c, KArgs a, int64_t n_tiles,
                         cudaStream_t st) {
  LaunchFn launch = nullptr;
  size_t smem = 0;
  // the RARE instances also carry the particle time
  const bool rare = h->rare || a.t != nullptr;
  int rc = pick_kernel(h, tun, a.compact_every > 0, rare, &launch, &smem);
  if (rc) return rc;
  int64_t grid = (int64_t)h->num_sms * std::max(1, tun.blocks_per_sm);
  if (grid > n_tiles) grid = n_tiles;
  if (grid < 1) grid = 1;
  a.tile_counter = c->d_scratch;
  a.error_flag = c->d_scratch + 1;
  a.wait_ns = wait_ns_of(tun);
  a.skip_table_copy = tun.test_skip_table_copy;
  CU(h, cudaMemsetAsync(c->d_scratch, 0, sizeof(int32_t), st));
  const cudaError_t e = launch(a, (int)grid, smem, st);
  if (e != cudaSuccess) return set_err(h, BGT_ECUDA, std::string("track_kernel launch: ") + cudaGetErrorString(e));
  h->launches++;
  return 0;
}

static KArgs base_args(bgt_handle* h, const bgt_tuning& tun) {
  KArgs a{};
  a.tables = h->d_tables;
  a.table_off_dw = h->d_table_off;
  a.table_dw = h->table_dw;
  a.n_rec = h->n_ele;
  a.rec_begin = 0;
  a.rec_end = h->n_ele;
  a.G = h->G;
  a.compact_every = tun.compact_every;
  return a;
}

// Tuning as bgt_set_tuning normalises it; 0 or BGT_EINVAL with the message.
static int normalise_tuning(bgt_handle* h, bgt_tuning* n) {
  if (n->threads_per_block == 0) n->threads_per_block = 128;
  if (n->blocks_per_sm == 0) n->blocks_per_sm = 4;
  if (n->threads_per_block != 64 && n->threads_per_block != 128 && n->threads_per_block != 256)
    return set_err(h, BGT_EINVAL, "threads_per_block must be 64, 128 or 256");
  if (n->compact_every < 0 || n->turns_per_launch < 0 || n->wait_limit_us < 0)
    return set_err(h, BGT_EINVAL, "negative tuning value");
  if (n->table_mode < 0 || n->table_mode > 3) return set_err(h, BGT_EINVAL, "table_mode must be 0, 1, 2 or 3");
  if (n->test_skip_table_copy != 0 && n->test_skip_table_copy != 1)
    return set_err(h, BGT_EINVAL, "test_skip_table_copy must be 0 or 1");
  return 0;
}

extern "C" {

int bgt_create(bgt_handle** out, const bgt_element* eles, int32_t n_ele, int32_t n_variants,
               const bgt_species* species, int32_t device) {
  if (!out || !eles || !species || n_ele <= 0 || n_variants <= 0)
    return set_err(nullptr, BGT_EINVAL, "bgt_create: invalid argument");
  *out = nullptr;
  bgt_handle* h = new bgt_handle();
  h->device = device;
  h->n_ele = n_ele;
  h->n_variants = n_variants;
  h->sp = *species;
  double p0c = eles[0].p0c;
  h->G.mc2 = species->mass;
  h->G.mc2sq = species->mass * species->mass;
  h->G.p0c = p0c;
  h->G.mal = species->max_aperture_limit;
  h->G.ap_on = species->aperture_limit_on;
  h->G.charge = species->charge;
  h->G.abs_time = species->absolute_time_tracking ? 1 : 0;
  h->G.abs_ref_shift = species->absolute_time_ref_shift ? 1 : 0;
  std::vector<double> all;
  std::string msg;
  int rc = host::compile_tables(eles, n_ele, n_variants, *species, QMEMO_CLASSES, all, h->h_table_off,
                                h->table_dw, h->rare, msg);
  if (rc) {
    delete h;
    // no handle to carry the message: print it once so the caller sees why
    fprintf(stderr, "bgt_create: %s\n", msg.c_str());
    return set_err(nullptr, rc, msg);
  }
  h->h_tables = all;
  DeviceGuard dg(device);
  cudaError_t e = dg.err;
  if (e != cudaSuccess ||
      (e = cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess ||
      (e = cudaMalloc(&h->d_tables, all.size() * 8)) != cudaSuccess ||
      (e = cudaMalloc(&h->d_table_off, h->h_table_off.size() * 8)) != cudaSuccess ||
      (e = cudaMalloc(&h->d_status, 64)) != cudaSuccess ||
      (e = cudaMemcpy(h->d_tables, all.data(), all.size() * 8, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(h->d_table_off, h->h_table_off.data(), h->h_table_off.size() * 8, cudaMemcpyHostToDevice)) !=
          cudaSuccess ||
      (e = cudaMemset(h->d_status, 0, 64)) != cudaSuccess || (e = upload_multipole_tables()) != cudaSuccess) {
    fprintf(stderr, "bgt_create: CUDA error: %s\n", cudaGetErrorString(e));
    bgt_destroy(h);
    return set_err(nullptr, BGT_ECUDA, std::string("bgt_create: ") + cudaGetErrorString(e));
  }
  *out = h;
  return 0;
}

int bgt_destroy(bgt_handle* h) {
  if (!h) return 0;
  DeviceGuard dg(h->device);
  for (CallCtx* c : h->pool) {
    if (c->st) cudaStreamSynchronize(c->st);
    free_ctx(c);
  }
  cudaFree(h->d_tables);
  cudaFree(h->d_table_off);
  cudaFree(h->d_status);
  delete h;
  return 0;
}

const char* bgt_last_error(const bgt_handle*) { return t_err.c_str(); }

int bgt_table_info(const bgt_handle* h, int64_t* table_bytes, int32_t* n_records) {
  if (!h) return set_err(nullptr, BGT_EINVAL, "null handle");
  if (table_bytes) *table_bytes = (int64_t)h->table_dw * 8;
  if (n_records) *n_records = h->n_ele;
  return 0;
}

int bgt_set_tuning(bgt_handle* h, const bgt_tuning* t) {
  if (!h || !t) return set_err(h, BGT_EINVAL, "bgt_set_tuning: invalid argument");
  bgt_tuning n = *t;
  int rc = normalise_tuning(h, &n);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(h->mu);
  h->tuning = n;
  return 0;
}

int bgt_get_tuning(const bgt_handle* h, bgt_tuning* t) {
  if (!h || !t) return set_err(nullptr, BGT_EINVAL, "bgt_get_tuning: invalid argument");
  *t = get_tuning_locked(const_cast<bgt_handle*>(h));
  return 0;
}

int64_t bgt_kernel_launch_count(const bgt_handle* h) { return h ? h->launches.load() : -1; }

// Track device-resident particles for turns [turn0, turn0 + n_turns) in
// segments of tuning.turns_per_launch turns (one persistent launch each).
// The call's error flag is cleared once, the tile counter per launch.
static int track_device_impl(bgt_handle* h, const bgt_tuning& tun, CallCtx* c, int32_t* status, double* d_vec6,
                             int64_t n_stride, double* d_beta, uint64_t* d_t, int32_t* d_state, int32_t* d_ixe,
                             int32_t* d_ixt,
                             const int32_t* d_slot, const int32_t* d_tile_var, int64_t n, int64_t n_slots,
                             int32_t turn0, int32_t n_turns, int32_t rec_begin, int32_t rec_end, cudaStream_t st) {
  KArgs a = base_args(h, tun);
  a.vec6 = d_vec6;
  a.n_stride = n_stride;
  a.beta = d_beta;
  a.t = d_t;
  a.G.track_time = d_t ? 1 : 0;
  a.state = d_state;
  a.ix_ele_lost = d_ixe;
  a.ix_turn_lost = d_ixt;
  a.slot_particle = d_slot;
  a.tile_variant = d_tile_var;
  a.n = n;
  a.n_slots = n_slots;
  a.rec_begin = rec_begin;
  a.rec_end = rec_end;
  a.status = status;
  CU(h, cudaMemsetAsync(c->d_scratch + 1, 0, sizeof(int32_t), st));
  int64_t n_tiles = (n_slots + tun.threads_per_block - 1) / tun.threads_per_block;
  int32_t seg = tun.turns_per_launch > 0 ? tun.turns_per_launch : n_turns;
  for (int32_t t = 0; t < n_turns; t += seg) {
    a.turn0 = turn0 + t;
    a.n_turns = std::min(seg, n_turns - t);
    int rc = enqueue_track(h, tun, c, a, n_tiles, st);
    if (rc) return rc;
  }
  return 0;
}

// Per-variant particle counts of a variant-sorted device array, with a check
// that ids are in range (bad bit 1) and non-decreasing (bad bit 2).
__global__ void variant_count_kernel(const int32_t* var, int64_t n, int32_t n_var, int64_t* first, int64_t* count,
                                     int32_t* bad) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int32_t v = var[i];
  if (v < 0 || v >= n_var) {
    atomicOr(bad, 1);
    return;
  }
  if (i > 0 && var[i - 1] > v) atomicOr(bad, 2);
  if (i == 0 || var[i - 1] != v) first[v] = i;
  atomicAdd((unsigned long long*)&count[v], 1ull);
}

// slot of particle i: its variant's first slot + its rank inside the variant
__global__ void variant_slot_kernel(const int32_t* var, int64_t n, const int64_t* first, const int64_t* slot0,
                                    int32_t* slot) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int32_t v = var[i];
  slot[slot0[v] + (i - first[v])] = (int32_t)i;
}

int bgt_track_turns_device(bgt_handle* h, double* d_vec6, double* d_beta, void* d_t, int32_t* d_state,
                           int32_t* d_ix_ele_lost, int32_t* d_ix_turn_lost, const int32_t* d_variant, int64_t n,
                           int32_t turn0, int32_t n_turns, void* stream) {
  if (!h || !d_vec6 || !d_beta || !d_state || !d_ix_ele_lost || n < 0 || n_turns < 0)
    return set_err(h, BGT_EINVAL, "bgt_track_turns_device: invalid argument");
  if (h->G.abs_time && !d_t)
    return set_err(h, BGT_EINVAL, "bgt_track_turns_device: absolute time tracking needs the particle times t");
  uint64_t* tq = static_cast<uint64_t*>(d_t);
  if (n == 0 || n_turns == 0) return 0;
  if (n > INT32_MAX) return set_err(h, BGT_EINVAL, "bgt_track_turns_device: n exceeds 2^31 - 1");
  DeviceGuard dg(h->device);
  CU(h, dg.err);
  const bgt_tuning tun = get_tuning_locked(h);
  cudaStream_t st = (cudaStream_t)stream;
  CtxLease L(h);
  int rc = L.acquire();
  if (rc) return rc;
  CallCtx* c = L.c;
  CU(h, L.use(st));
  if (!d_variant || h->n_variants == 1)
    return track_device_impl(h, tun, c, h->d_status, d_vec6, n, d_beta, tq, d_state, d_ix_ele_lost,
                             d_ix_turn_lost, nullptr, nullptr, n, n, turn0, n_turns, 0, h->n_ele, st);
  // Group by variant into tile-aligned slot ranges.  The variant ids must be
  // sorted (non-decreasing); the per-variant counts are read back once.
  const int32_t nv = h->n_variants;
  const int block = tun.threads_per_block;
  if (!c->d_grp_v) CU(h, cudaMalloc(&c->d_grp_v, ((size_t)3 * nv + 1) * 8));
  int64_t* d_first = c->d_grp_v;
  int64_t* d_count = d_first + nv;
  int64_t* d_slot0 = d_count + nv;
  int32_t* d_bad = (int32_t*)(d_slot0 + nv);
  CU(h, cudaMemsetAsync(d_first, 0, ((size_t)3 * nv + 1) * 8, st));
  variant_count_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_variant, n, nv, d_first, d_count, d_bad);
  h->launches++;
  std::vector<int64_t> cnt((size_t)nv + 1);
  CU(h, cudaMemcpyAsync(cnt.data(), d_count, (size_t)nv * 8, cudaMemcpyDeviceToHost, st));
  int32_t bad = 0;
  CU(h, cudaMemcpyAsync(&bad, d_bad, 4, cudaMemcpyDeviceToHost, st));
  CU(h, cudaStreamSynchronize(st));
  if (bad & 1) return set_err(h, BGT_EINVAL, "bgt_track_turns_device: variant id out of range");
  if (bad & 2) return set_err(h, BGT_EINVAL, "bgt_track_turns_device: variant ids must be sorted");
  std::vector<int64_t> slot0(nv);
  std::vector<int32_t> tvar;
  int64_t s = 0;
  for (int32_t v = 0; v < nv; v++) {
    slot0[v] = s;
    int64_t tiles = (cnt[v] + block - 1) / block;
    for (int64_t t = 0; t < tiles; t++) tvar.push_back(v);
    s += tiles * block;
  }
  const int64_t n_slots = s, n_tiles = (int64_t)tvar.size();
  if (n_slots > c->grp_cap_slots || n_tiles > c->grp_cap_tiles) {
    CU(h, cudaStreamSynchronize(st));
    cudaFree(c->d_grp);
    c->d_grp = nullptr;
    c->grp_cap_slots = std::max(n_slots, c->grp_cap_slots);
    c->grp_cap_tiles = std::max(n_tiles, c->grp_cap_tiles);
    CU(h, cudaMalloc(&c->d_grp, (size_t)(c->grp_cap_slots + c->grp_cap_tiles) * 4));
  }
  int32_t* d_slot = c->d_grp;
  int32_t* d_tvar = d_slot + c->grp_cap_slots;
  CU(h, cudaMemcpyAsync(d_slot0, slot0.data(), (size_t)nv * 8, cudaMemcpyHostToDevice, st));
  CU(h, cudaMemcpyAsync(d_tvar, tvar.data(), (size_t)n_tiles * 4, cudaMemcpyHostToDevice, st));
  CU(h, cudaMemsetAsync(d_slot, 0xff, (size_t)n_slots * 4, st));
  variant_slot_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_variant, n, d_first, d_slot0, d_slot);
  h->launches++;
  // (copies from pageable host memory return once the data is staged, so
  // slot0 and tvar may go out of scope before the copies complete)
  return track_device_impl(h, tun, c, h->d_status, d_vec6, n, d_beta, tq, d_state, d_ix_ele_lost, d_ix_turn_lost,
                           d_slot, d_tvar, n, n_slots, turn0, n_turns, 0, h->n_ele, st);
}

// Reads and clears the handle's device error flag after `stream` completes.
__global__ void take_status_kernel(int32_t* status, int32_t* out) { *out = atomicExch(status, 0); }

int bgt_device_status(bgt_handle* h, void* stream) {
  if (!h) return set_err(nullptr, BGT_EINVAL, "null handle");
  DeviceGuard dg(h->device);
  CU(h, dg.err);
  cudaStream_t st = (cudaStream_t)stream;
  CtxLease L(h);
  int rc = L.acquire();
  if (rc) return rc;
  CU(h, L.use(st));
  take_status_kernel<<<1, 1, 0, st>>>(h->d_status, L.c->d_scratch + 2);
  h->launches++;
  int32_t flag = 0;
  CU(h, cudaMemcpyAsync(&flag, L.c->d_scratch + 2, 4, cudaMemcpyDeviceToHost, st));
  CU(h, cudaStreamSynchronize(st));
  if (flag) return set_err(h, BGT_ETIMEOUT, "element-table staging did not complete on the device");
  return 0;
}

// Grow a context's device staging buffers.
static int ensure_staging(bgt_handle* h, CallCtx* c, int64_t n, int64_t n_slots, int64_t n_tiles, bool with_t) {
  if (n <= c->cap && n_slots <= c->cap_slots && n_tiles <= c->cap_tiles && (!with_t || c->d_t)) return 0;
  CU(h, cudaStreamSynchronize(c->st));
  cudaFree(c->d_vec6);
  cudaFree(c->d_beta);
  cudaFree(c->d_i32);
  cudaFree(c->d_t);
  c->d_vec6 = nullptr;
  c->d_beta = nullptr;
  c->d_i32 = nullptr;
  c->d_t = nullptr;
  c->cap = std::max(n, c->cap);
  c->cap_slots = std::max(n_slots, c->cap_slots);
  c->cap_tiles = std::max(n_tiles, c->cap_tiles);
  CU(h, cudaMalloc(&c->d_vec6, (size_t)c->cap * 6 * 8));
  CU(h, cudaMalloc(&c->d_beta, (size_t)c->cap * 8));
  CU(h, cudaMalloc(&c->d_i32, (size_t)(3 * c->cap + c->cap_slots + c->cap_tiles) * 4));
  if (with_t) CU(h, cudaMalloc(&c->d_t, (size_t)c->cap * 16));
  return 0;
}

// Grow a context's pinned host staging buffer.
static int ensure_pinned(bgt_handle* h, CallCtx* c, size_t bytes) {
  if (bytes <= c->pin_bytes) return 0;
  CU(h, cudaStreamSynchronize(c->st));
  if (c->h_pin) cudaFreeHost(c->h_pin);
  c->h_pin = nullptr;
  c->pin_bytes = 0;
  CU(h, cudaMallocHost(&c->h_pin, bytes));
  c->pin_bytes = bytes;
  return 0;
}

// Host-buffer tracking shared by bgt_track_turns and bgt_track_elements: the
// particles go through the context's pinned staging buffer to its device
// buffers on its own stream; the call waits for that stream only.
// Copies between the caller's (pageable) host buffers and the pinned
// staging buffer.  One core copies pageable memory at a few GB/s, well below
// the host link, so large calls split the bytes evenly over up to 8 threads.
struct HostCopy {
  void* dst;
  const void* src;
  size_t bytes;
};
static void host_copies(const std::vector<HostCopy>& jobs) {
  size_t total = 0;
  for (const HostCopy& j : jobs) total += j.bytes;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int nt = (int)std::min<size_t>(std::min(8u, hw), total / ((size_t)4 << 20));
  auto piece = [&](int k, int parts) {
    const size_t lo = total * k / parts, hi = total * (k + 1) / parts;
    size_t off = 0;
    for (const HostCopy& j : jobs) {
      const size_t a = std::max(lo, off), b = std::min(hi, off + j.bytes);
      if (a < b) memcpy((char*)j.dst + (a - off), (const char*)j.src + (a - off), b - a);
      off += j.bytes;
    }
  };
  if (nt <= 1) {
    piece(0, 1);
    return;
  }
  std::vector<std::thread> th;
  for (int k = 1; k < nt; k++) {
    try {
      th.emplace_back(piece, k, nt);
    } catch (...) {
      piece(k, nt);  // no thread available: this one copies the piece
    }
  }
  piece(0, nt);
  for (std::thread& t : th) t.join();
}

static int track_host(bgt_handle* h, double* vec6, double* beta, void* t, int32_t* state, int32_t* ixe, int32_t* ixt,
                      const int32_t* variant, int64_t n, int32_t turn0, int32_t n_turns, int32_t rec_begin,
                      int32_t rec_end) {
  if (!h || !vec6 || !beta || !state || !ixe || n < 0) return set_err(h, BGT_EINVAL, "invalid argument");
  if (h->G.abs_time && !t) return set_err(h, BGT_EINVAL, "absolute time tracking needs the particle times t");
  if (n == 0 || n_turns == 0) return 0;
  if (n > INT32_MAX) return set_err(h, BGT_EINVAL, "n exceeds 2^31 - 1");
  DeviceGuard dg(h->device);
  CU(h, dg.err);
  const bgt_tuning tun = get_tuning_locked(h);
  const int block = tun.threads_per_block;
  // group particles by variant into tile-aligned slot ranges
  std::vector<int32_t> slot_map, tile_var;
  int64_t n_slots = n;
  bool multi = variant && h->n_variants > 1;
  if (multi) {
    std::vector<int64_t> count(h->n_variants, 0);
    for (int64_t i = 0; i < n; i++) {
      if (variant[i] < 0 || variant[i] >= h->n_variants) return set_err(h, BGT_EINVAL, "variant out of range");
      count[variant[i]]++;
    }
    std::vector<int64_t> start(h->n_variants, 0);
    int64_t s = 0;
    for (int v = 0; v < h->n_variants; v++) {
      start[v] = s;
      int64_t tiles = (count[v] + block - 1) / block;
      for (int64_t t = 0; t < tiles; t++) tile_var.push_back(v);
      s += tiles * block;
    }
    n_slots = s;
    slot_map.assign(n_slots, -1);
    std::vector<int64_t> fill = start;
    for (int64_t i = 0; i < n; i++) slot_map[fill[variant[i]]++] = (int32_t)i;
  } else if (variant && h->n_variants == 1) {
    for (int64_t i = 0; i < n; i++)
      if (variant[i] != 0) return set_err(h, BGT_EINVAL, "variant out of range");
  }
  int64_t n_tiles = (n_slots + block - 1) / block;
  CtxLease L(h);
  int rc = L.acquire();
  if (rc) return rc;
  CallCtx* c = L.c;
  cudaStream_t st = c->st;
  CU(h, L.use(st));
  if ((rc = ensure_staging(h, c, n, n_slots, n_tiles, t != nullptr))) return rc;
  // pinned layout: times [n][16 B] (when tracked), vec6 [6][n], beta [n],
  // state/ixe/ixt [n] each, slot map, tile variants, error flag
  const size_t b_t = t ? (size_t)n * 16 : 0;
  const size_t b_v = (size_t)n * 6 * 8, b_b = (size_t)n * 8, b_i = (size_t)n * 4;
  const size_t b_slot = multi ? (size_t)n_slots * 4 : 0, b_tv = multi ? tile_var.size() * 4 : 0;
  if ((rc = ensure_pinned(h, c, b_t + b_v + b_b + 3 * b_i + b_slot + b_tv + 16))) return rc;
  unsigned char* p_time = c->h_pin;
  unsigned char* p = c->h_pin + b_t;
  double* p_v = (double*)p;
  double* p_b = (double*)(p + b_v);
  int32_t* p_s = (int32_t*)(p + b_v + b_b);
  int32_t* p_e = p_s + n;
  int32_t* p_t = p_e + n;
  int32_t* p_slot = p_t + n;
  int32_t* p_tv = p_slot + (multi ? n_slots : 0);
  int32_t* p_flag = p_tv + (multi ? tile_var.size() : 0);
  host_copies({{p_time, t, b_t},
               {p_v, vec6, b_v},
               {p_b, beta, b_b},
               {p_s, state, b_i},
               {p_e, ixe, b_i},
               {p_t, ixt, ixt ? b_i : 0},
               {p_slot, slot_map.data(), b_slot},
               {p_tv, tile_var.data(), b_tv}});
  int32_t* d_state = c->d_i32;
  int32_t* d_ixe = d_state + c->cap;
  int32_t* d_ixt = d_ixe + c->cap;
  int32_t* d_slot = d_ixt + c->cap;
  int32_t* d_tvar = d_slot + c->cap_slots;
  if (t) CU(h, cudaMemcpyAsync(c->d_t, p_time, b_t, cudaMemcpyHostToDevice, st));
  CU(h, cudaMemcpy2DAsync(c->d_vec6, c->cap * 8, p_v, n * 8, n * 8, 6, cudaMemcpyHostToDevice, st));
  CU(h, cudaMemcpyAsync(c->d_beta, p_b, b_b, cudaMemcpyHostToDevice, st));
  CU(h, cudaMemcpyAsync(d_state, p_s, b_i, cudaMemcpyHostToDevice, st));
  CU(h, cudaMemcpyAsync(d_ixe, p_e, b_i, cudaMemcpyHostToDevice, st));
  if (ixt) CU(h, cudaMemcpyAsync(d_ixt, p_t, b_i, cudaMemcpyHostToDevice, st));
  if (multi) {
    CU(h, cudaMemcpyAsync(d_slot, p_slot, b_slot, cudaMemcpyHostToDevice, st));
    CU(h, cudaMemcpyAsync(d_tvar, p_tv, b_tv, cudaMemcpyHostToDevice, st));
  }
  rc = track_device_impl(h, tun, c, nullptr, c->d_vec6, c->cap, c->d_beta, t ? c->d_t : nullptr, d_state, d_ixe,
                         ixt ? d_ixt : nullptr,
                         multi ? d_slot : nullptr, multi ? d_tvar : nullptr, n, n_slots, turn0, n_turns, rec_begin,
                         rec_end, st);
  if (rc) {
    cudaStreamSynchronize(st);
    return rc;
  }
  CU(h, cudaMemcpyAsync(p_flag, c->d_scratch + 1, 4, cudaMemcpyDeviceToHost, st));
  if (t) CU(h, cudaMemcpyAsync(p_time, c->d_t, b_t, cudaMemcpyDeviceToHost, st));
  CU(h, cudaMemcpy2DAsync(p_v, n * 8, c->d_vec6, c->cap * 8, n * 8, 6, cudaMemcpyDeviceToHost, st));
  CU(h, cudaMemcpyAsync(p_b, c->d_beta, b_b, cudaMemcpyDeviceToHost, st));
  CU(h, cudaMemcpyAsync(p_s, d_state, b_i, cudaMemcpyDeviceToHost, st));
  CU(h, cudaMemcpyAsync(p_e, d_ixe, b_i, cudaMemcpyDeviceToHost, st));
  if (ixt) CU(h, cudaMemcpyAsync(p_t, d_ixt, b_i, cudaMemcpyDeviceToHost, st));
  CU(h, cudaStreamSynchronize(st));
  if (*p_flag) return set_err(h, BGT_ETIMEOUT, "element-table staging did not complete");
  host_copies({{t, p_time, b_t},
               {vec6, p_v, b_v},
               {beta, p_b, b_b},
               {state, p_s, b_i},
               {ixe, p_e, b_i},
               {ixt, p_t, ixt ? b_i : 0}});
  return 0;
}

int bgt_track_turns(bgt_handle* h, double* vec6, double* beta, void* t, int32_t* state, int32_t* ix_ele_lost,
                    int32_t* ix_turn_lost, const int32_t* variant, int64_t n, int32_t turn0, int32_t n_turns) {
  if (!h) return set_err(nullptr, BGT_EINVAL, "null handle");
  return track_host(h, vec6, beta, t, state, ix_ele_lost, ix_turn_lost, variant, n, turn0, n_turns, 0, h->n_ele);
}

int bgt_track_elements(bgt_handle* h, double* vec6, double* beta, void* t, int32_t* state, int32_t* ix_ele_lost,
                       const int32_t* variant, int64_t n, int32_t e_begin, int32_t e_end) {
  if (!h) return set_err(nullptr, BGT_EINVAL, "null handle");
  if (e_begin < 0 || e_end > h->n_ele || e_begin >= e_end) return set_err(h, BGT_EINVAL, "bad element range");
  return track_host(h, vec6, beta, t, state, ix_ele_lost, nullptr, variant, n, 0, 1, e_begin, e_end);
}

}  // extern "C"

// ===========================================================================
// Dynamic-aperture polar grid (bmad/modules/dynamic_aperture_mod.f90:27-207,
// 284-398 with the bisection replaced by a fixed grid of radii).

namespace bgt {

struct DAArgs {
  const double* ref;  // [(v*n_delta + d)*6 + c]
  const double* cs;   // [a] = (cos(angle_a), sin(angle_a)), host-evaluated
  int32_t n_var, n_delta, n_angle, n_radius;
  double a0, da, dr, y_scale;
  int32_t block;
  int64_t per_var, slots_per_var;
  double p0c, mc2;
  double* vec6;
  int64_t stride;
  double* beta;
  int32_t* state;
  int32_t* ixe;
  int32_t* ixt;
  int32_t* slot;
  uint64_t* t;  // particle times (absolute time tracking) or nullptr
};

// particle index p = ((v*n_delta + d)*n_angle + a)*n_radius + r
__global__ void da_init_kernel(DAArgs A, int64_t n) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int32_t r = (int32_t)(i % A.n_radius);
  int64_t q = i / A.n_radius;
  int32_t a = (int32_t)(q % A.n_angle);
  q /= A.n_angle;
  int32_t d = (int32_t)(q % A.n_delta);
  int32_t v = (int32_t)(q / A.n_delta);
  const double* ref = A.ref + ((int64_t)v * A.n_delta + d) * 6;
  double rad = A.dr * r;
  double x1 = A.cs[2 * a] * rad;
  double y1 = A.cs[2 * a + 1] * rad * A.y_scale;
  A.vec6[0 * A.stride + i] = ref[0] + x1;
  A.vec6[1 * A.stride + i] = ref[1];
  A.vec6[2 * A.stride + i] = ref[2] + y1;
  A.vec6[3 * A.stride + i] = ref[3];
  A.vec6[4 * A.stride + i] = ref[4];
  A.vec6[5 * A.stride + i] = ref[5];
  double pc = (1 + ref[5]) * A.p0c;
  A.beta[i] = pc / sqrt(pc * pc + A.mc2 * A.mc2);
  A.state[i] = ALIVE;
  A.ixe[i] = -1;
  A.ixt[i] = -1;
  if (A.t) {
    // init_coord.f90:222: t = ref_time - z / (beta c_light), ref_time = 0
    // at the scan's starting element
    const qp::Q t0 = qp::from_double(0.0 - A.vec6[4 * A.stride + i] / (A.beta[i] * C_LIGHT));
    A.t[2 * i] = t0.lo;
    A.t[2 * i + 1] = t0.hi;
  }
  // slot of this particle: variant-major, padded per variant; inside a
  // variant radius-major ((d * n_radius + r) * n_angle + a), so that a warp
  // (and a CTA) holds probes of one or few radii across the angles -- they
  // are lost at similar turns, and warps of a CTA finish together instead of
  // idling at the end-of-tile barrier.  Results do not depend on the slot.
  int64_t within = ((int64_t)d * A.n_radius + r) * A.n_angle + a;
  A.slot[(int64_t)v * A.slots_per_var + within] = (int32_t)i;
}

__global__ void da_tile_var_kernel(int32_t* tvar, int64_t tiles_per_var, int64_t n_tiles) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < n_tiles) tvar[t] = (int32_t)(t / tiles_per_var);
}

__global__ void da_reduce_kernel(const int32_t* state, const int32_t* ixt, int64_t n_rays, int32_t n_radius,
                                 double dr, int32_t turn0, int32_t n_turns, double* da_radius,
                                 int32_t* survive) {
  int64_t ray = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (ray >= n_rays) return;
  int64_t base = ray * n_radius;
  int32_t first_lost = n_radius;
  for (int32_t r = 0; r < n_radius; r++) {
    int32_t s = state[base + r];
    if (s != ALIVE && first_lost == n_radius) first_lost = r;
    if (survive) survive[base + r] = (s == ALIVE) ? n_turns : (ixt[base + r] - turn0);
  }
  int32_t last_ok = first_lost - 1;
  da_radius[ray] = last_ok < 0 ? 0.0 : dr * last_ok;
}

// FP64 fused multiply-add throughput probe: 8 independent chains per thread.
__global__ void fp64_peak_kernel(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x * 1e-9, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
         x7 = x0 + 7;
  for (int i = 0; i < iters; i++) {
    x0 = fma(x0, a, b);
    x1 = fma(x1, a, b);
    x2 = fma(x2, a, b);
    x3 = fma(x3, a, b);
    x4 = fma(x4, a, b);
    x5 = fma(x5, a, b);
    x6 = fma(x6, a, b);
    x7 = fma(x7, a, b);
  }
  double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 12345.678) out[0] = s;  // keeps the chains live
}

}  // namespace bgt

extern "C" {

int bgt_da_scan_grid(bgt_handle* h, const double* ref_orbit, int32_t n_variants_used, int32_t n_delta,
                     int32_t n_angle, double angle_min, double angle_max, int32_t n_radius, double r_max,
                     double y_scale, int32_t n_turns, double* da_radius, int32_t* survive_turns) {
  if (!h || !ref_orbit || !da_radius || n_variants_used <= 0 || n_variants_used > h->n_variants || n_delta <= 0 ||
      n_angle <= 0 || n_radius <= 1 || n_turns <= 0)
    return set_err(h, BGT_EINVAL, "bgt_da_scan_grid: invalid argument");
  DeviceGuard dg(h->device);
  CU(h, dg.err);
  const bgt_tuning tun = get_tuning_locked(h);
  const int block = tun.threads_per_block;
  DAArgs A{};
  A.n_var = n_variants_used;
  A.n_delta = n_delta;
  A.n_angle = n_angle;
  A.n_radius = n_radius;
  A.a0 = angle_min;
  A.da = n_angle > 1 ? (angle_max - angle_min) / (n_angle - 1) : 0.0;
  A.dr = r_max / (n_radius - 1);
  A.y_scale = y_scale;
  A.per_var = (int64_t)n_delta * n_angle * n_radius;
  int64_t tiles_per_var = (A.per_var + block - 1) / block;
  A.slots_per_var = tiles_per_var * block;
  int64_t n = A.per_var * n_variants_used;
  int64_t n_slots = A.slots_per_var * n_variants_used;
  int64_t n_tiles = tiles_per_var * n_variants_used;
  if (n > INT32_MAX) return set_err(h, BGT_EINVAL, "bgt_da_scan_grid: more than 2^31 - 1 probes");
  A.p0c = h->G.p0c;
  A.mc2 = h->G.mc2;
  CtxLease L(h);
  int rc = L.acquire();
  if (rc) return rc;
  CallCtx* c = L.c;
  cudaStream_t st = c->st;
  CU(h, L.use(st));
  const bool with_t = h->G.abs_time != 0;
  if ((rc = ensure_staging(h, c, n, n_slots, n_tiles, with_t))) return rc;
  int32_t* d_state = c->d_i32;
  int32_t* d_ixe = d_state + c->cap;
  int32_t* d_ixt = d_ixe + c->cap;
  int32_t* d_slot = d_ixt + c->cap;
  int32_t* d_tvar = d_slot + c->cap_slots;
  int64_t n_rays = (int64_t)n_variants_used * n_delta * n_angle;
  // ray directions: angle_j = j * delta_angle + min_angle
  // (dynamic_aperture_mod.f90:88-95), cos/sin by the host C library
  std::vector<double> cs(2 * (size_t)n_angle);
  for (int j = 0; j < n_angle; j++) {
    double ang = (n_angle == 1) ? (angle_min + angle_max) / 2 : j * A.da + angle_min;
    cs[2 * j] = cos(ang);
    cs[2 * j + 1] = sin(ang);
  }
  // per-call device buffers: ray directions, reference orbits, radii,
  // survival turns (one allocation)
  const size_t b_cs = cs.size() * 8, b_ref = (size_t)n_variants_used * n_delta * 6 * 8, b_da = (size_t)n_rays * 8;
  const size_t b_surv = survive_turns ? (size_t)n * 4 : 0;
  unsigned char* d_buf = nullptr;
  CU(h, cudaMalloc(&d_buf, b_cs + b_ref + b_da + b_surv));
  struct Free {
    unsigned char* p;
    cudaStream_t st;
    ~Free() {
      cudaStreamSynchronize(st);
      cudaFree(p);
    }
  } free_buf{d_buf, st};
  double* d_cs = (double*)d_buf;
  double* d_ref = (double*)(d_buf + b_cs);
  double* d_da = (double*)(d_buf + b_cs + b_ref);
  int32_t* d_surv = survive_turns ? (int32_t*)(d_buf + b_cs + b_ref + b_da) : nullptr;
  CU(h, cudaMemcpyAsync(d_cs, cs.data(), b_cs, cudaMemcpyHostToDevice, st));
  CU(h, cudaMemcpyAsync(d_ref, ref_orbit, b_ref, cudaMemcpyHostToDevice, st));
  CU(h, cudaMemsetAsync(d_slot, 0xff, (size_t)n_slots * 4, st));
  A.cs = d_cs;
  A.ref = d_ref;
  A.vec6 = c->d_vec6;
  A.stride = c->cap;
  A.beta = c->d_beta;
  A.state = d_state;
  A.ixe = d_ixe;
  A.ixt = d_ixt;
  A.slot = d_slot;
  A.t = with_t ? c->d_t : nullptr;
  A.block = block;
  da_init_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(A, n);
  da_tile_var_kernel<<<(unsigned)((n_tiles + 255) / 256), 256, 0, st>>>(d_tvar, tiles_per_var, n_tiles);
  h->launches += 2;
  rc = track_device_impl(h, tun, c, nullptr, c->d_vec6, c->cap, c->d_beta, A.t, d_state, d_ixe, d_ixt, d_slot,
                         d_tvar, n, n_slots, 0, n_turns, 0, h->n_ele, st);
  if (rc) return rc;
  da_reduce_kernel<<<(unsigned)((n_rays + 127) / 128), 128, 0, st>>>(d_state, d_ixt, n_rays, n_radius, A.dr, 0,
                                                                     n_turns, d_da, d_surv);
  h->launches++;
  int32_t flag = 0;
  CU(h, cudaMemcpyAsync(&flag, c->d_scratch + 1, 4, cudaMemcpyDeviceToHost, st));
  CU(h, cudaMemcpyAsync(da_radius, d_da, b_da, cudaMemcpyDeviceToHost, st));
  if (survive_turns) CU(h, cudaMemcpyAsync(survive_turns, d_surv, b_surv, cudaMemcpyDeviceToHost, st));
  CU(h, cudaStreamSynchronize(st));
  if (flag) return set_err(h, BGT_ETIMEOUT, "element-table staging did not complete");
  return 0;
}

// Measured FP64 FMA throughput of the current device in TFLOP/s (2 flops per
// FMA).  Measurement helper for roofline reporting; no reference counterpart.
int bgt_fp64_peak_tflops(int32_t device, double* tflops) {
  if (!tflops) return BGT_EINVAL;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return BGT_ECUDA;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  double* d_out = nullptr;
  if (cudaMalloc(&d_out, 8) != cudaSuccess) return BGT_ECUDA;
  const int threads = 256, blocks = sms * 8, iters = 1 << 14;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  fp64_peak_kernel<<<blocks, threads>>>(d_out, iters, 0.999999, 1e-9);
  cudaEventRecord(t0);
  const int reps = 5;
  for (int r = 0; r < reps; r++) fp64_peak_kernel<<<blocks, threads>>>(d_out, iters, 0.999999, 1e-9);
  cudaEventRecord(t1);
  cudaEventSynchronize(t1);
  float ms = 0;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaFree(d_out);
  if (cudaGetLastError() != cudaSuccess) return BGT_ECUDA;
  double flops = 2.0 * 8.0 * iters * (double)threads * blocks * reps;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return 0;
}

}  // extern "C"

// ===========================================================================
// Allocation-free tracking entry point.
//
// For callers that cannot allocate device memory from inside this library:
// hosts whose framework owns the device memory (a caching allocator that has
// reserved the GPU, so a cudaMalloc here could fail or fragment its pool) and
// loops that must not allocate per call.  The element table, the tile
// counter and the error flag live in one file-scope device array instead of
// handle-owned cudaMalloc buffers; the caller passes the particle arrays.
//
// The array holds BGT_NOALLOC_SCRATCH_BYTES on every GPU that loads this
// library, until the process exits.  Tables larger than that are rejected.
// Every call uses the same array and leaves its contents behind: calls that
// overlap on the GPU (different streams, or threads) race and must be
// serialised by the caller.  The first call on a device resolves the array's
// address (cudaGetSymbolAddress), zeroes its header and uploads the
// multipole coefficient tables; make that first call before any stream
// capture.

#define BGT_NOALLOC_SCRATCH_BYTES (256 * 1024)

namespace bgt {

// [0..3] tile counter, [4..7] error flag (int32); [16..23] table offset of
// the single variant (int64, always 0); table from byte 256 on
static __device__ __align__(256) unsigned char g_noalloc_scratch[BGT_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kNoallocMaxDevices = 64;
std::atomic<unsigned char*> g_noalloc_ptr[kNoallocMaxDevices];
std::mutex g_noalloc_setup_mu;
}  // namespace

}  // namespace bgt

extern "C" int bgt_track_turns_device_noalloc(const bgt_element* eles, int32_t n_ele, const bgt_species* species,
                                              double* d_vec6, double* d_beta, int32_t* d_state,
                                              int32_t* d_ix_ele_lost, int32_t* d_ix_turn_lost, int64_t n,
                                              int32_t turn0, int32_t n_turns, const bgt_tuning* tuning,
                                              int32_t device, void* stream, int32_t* d_status, char* err,
                                              int32_t err_len) {
  auto fail = [&](int code, const std::string& msg) {
    if (err && err_len > 0) {
      snprintf(err, (size_t)err_len, "%s", msg.c_str());
    }
    return code;
  };
  if (!eles || !species || n_ele <= 0 || !d_vec6 || !d_beta || !d_state || !d_ix_ele_lost || n < 0 ||
      n_turns < 0 || device < 0 || device >= bgt::kNoallocMaxDevices)
    return fail(BGT_EINVAL, "bgt_track_turns_device_noalloc: invalid argument");
  if (n > INT32_MAX) return fail(BGT_EINVAL, "bgt_track_turns_device_noalloc: n exceeds 2^31 - 1");
  // the launch shape is checked before anything is enqueued
  bgt_tuning t = tuning ? *tuning : bgt_tuning{128, 4, 0, 0, 0, 0, 0};
  if (t.threads_per_block == 0) t.threads_per_block = 128;
  if (t.blocks_per_sm == 0) t.blocks_per_sm = 4;
  if (!((t.threads_per_block == 128 && t.blocks_per_sm == 4) || (t.threads_per_block == 256 && t.blocks_per_sm == 2)))
    return fail(BGT_EINVAL, "bgt_track_turns_device_noalloc: tuning must be (128, 4) or (256, 2)");
  if (t.compact_every < 0 || t.turns_per_launch < 0 || t.wait_limit_us < 0 ||
      (t.test_skip_table_copy != 0 && t.test_skip_table_copy != 1))
    return fail(BGT_EINVAL, "bgt_track_turns_device_noalloc: invalid tuning value");
  if (species->absolute_time_tracking)
    return fail(BGT_EUNSUPPORTED, "bgt_track_turns_device_noalloc: absolute time tracking needs the particle times, "
                                  "which only the handle entry points carry");
  if (n == 0 || n_turns == 0) return 0;
  DeviceGuard dg(device);
  cudaError_t ce = dg.err;
  if (ce != cudaSuccess) return fail(BGT_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(ce));

  // one-time set-up on this device (this device current)
  if (!bgt::g_noalloc_ptr[device].load(std::memory_order_acquire)) {
    std::lock_guard<std::mutex> g(bgt::g_noalloc_setup_mu);
    if (!bgt::g_noalloc_ptr[device].load(std::memory_order_acquire)) {
      void* p = nullptr;
      ce = cudaGetSymbolAddress(&p, bgt::g_noalloc_scratch);
      if (ce != cudaSuccess) return fail(BGT_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(ce));
      if ((ce = cudaMemset(p, 0, 256)) != cudaSuccess)
        return fail(BGT_ECUDA, std::string("scratch header: ") + cudaGetErrorString(ce));
      if ((ce = upload_multipole_tables()) != cudaSuccess)
        return fail(BGT_ECUDA, std::string("coefficient upload: ") + cudaGetErrorString(ce));
      bgt::g_noalloc_ptr[device].store(static_cast<unsigned char*>(p), std::memory_order_release);
    }
  }
  unsigned char* base = bgt::g_noalloc_ptr[device].load(std::memory_order_acquire);

  // compile the table on the host (same records as bgt_create, one variant)
  std::vector<double> tab((size_t)(n_ele + (n_ele % 2)), 0.0);
  std::unordered_map<std::string, int32_t> pool;
  std::string msg;
  bool rare = false;
  const double p0c = eles[0].p0c;
  for (int e = 0; e < n_ele; e++) {
    std::vector<double> rec;
    int rc = bgt::host::compile_element(eles[e], *species, p0c, rec, msg);
    if (rc) return fail(rc, msg);
    bgt::RecHdr* rh = reinterpret_cast<bgt::RecHdr*>(rec.data());
    rh->ix_ele = 0;
    if (bgt::host::record_is_rare(rh)) rare = true;
    if (rh->kind == bgt::K_QUAD) rh->aux0 = -1;  // no quad memo classes on this path
    std::string key(reinterpret_cast<const char*>(rec.data()), rec.size() * sizeof(double));
    auto it = pool.find(key);
    int32_t off;
    if (it != pool.end()) {
      off = it->second;
    } else {
      off = (int32_t)tab.size();
      tab.insert(tab.end(), rec.begin(), rec.end());
      pool.emplace(std::move(key), off);
    }
    int32_t* s = reinterpret_cast<int32_t*>(tab.data()) + 2 * e;
    s[0] = off;
    s[1] = eles[e].ix_ele;
  }
  if (tab.size() % 2) tab.push_back(0.0);
  const size_t table_bytes = tab.size() * sizeof(double);
  if (256 + table_bytes > BGT_NOALLOC_SCRATCH_BYTES)
    return fail(BGT_ETOOLARGE, "bgt_track_turns_device_noalloc: element table needs " +
                                   std::to_string(table_bytes) + " bytes, the scratch array holds " +
                                   std::to_string(BGT_NOALLOC_SCRATCH_BYTES - 256));
  // The table is staged in shared memory when it fits, else read in place
  // from the scratch array (global memory, CTA tiles), as bgt_create's
  // tables are.
  const int block = t.threads_per_block;
  const size_t state_smem = (t.compact_every > 0 ? (size_t)9 * block * 8 : 0) +
                            (size_t)bgt::QMEMO_CLASSES * 13 * block * 8;
  const bool gtab = state_smem + table_bytes > SMEM_LIMIT;
  const size_t smem = state_smem + (gtab ? 0 : table_bytes);
  const LaunchFn launch = find_track_kernel(block, t.blocks_per_sm, gtab ? 1 : 0, rare);
  if (!launch) return fail(BGT_EINVAL, "bgt_track_turns_device_noalloc: no kernel instance for this tuning");
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);

  cudaStream_t st = (cudaStream_t)stream;
  int32_t* d_counter = reinterpret_cast<int32_t*>(base);
  double* d_table = reinterpret_cast<double*>(base + 256);
  int64_t* d_table_off = reinterpret_cast<int64_t*>(base + 16);
  // (a copy from pageable host memory returns once the data is staged, so
  // `tab` may go out of scope before the copy completes)
  if ((ce = cudaMemcpyAsync(d_table, tab.data(), table_bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail(BGT_ECUDA, std::string("table upload: ") + cudaGetErrorString(ce));

  bgt::KArgs a{};
  a.vec6 = d_vec6;
  a.beta = d_beta;
  a.state = d_state;
  a.ix_ele_lost = d_ix_ele_lost;
  a.ix_turn_lost = d_ix_turn_lost;
  a.n = n;
  a.n_stride = n;
  a.n_slots = n;
  a.tables = d_table;
  a.table_off_dw = d_table_off;
  a.table_dw = (int32_t)tab.size();
  a.rec_begin = 0;
  a.rec_end = n_ele;
  a.n_rec = n_ele;
  a.compact_every = t.compact_every;
  a.tile_counter = d_counter;
  a.error_flag = d_counter + 1;
  a.status = nullptr;
  a.wait_ns = wait_ns_of(t);
  a.skip_table_copy = t.test_skip_table_copy;
  a.G.mc2 = species->mass;
  a.G.mc2sq = species->mass * species->mass;
  a.G.p0c = p0c;
  a.G.mal = species->max_aperture_limit;
  a.G.ap_on = species->aperture_limit_on;
  a.G.charge = species->charge;
  const int64_t n_tiles = (n + block - 1) / block;
  int64_t grid = std::min<int64_t>((int64_t)sms * t.blocks_per_sm, n_tiles);
  if (grid < 1) grid = 1;
  // the counter and error flag must start at zero for every call
  if ((ce = cudaMemsetAsync(d_counter, 0, 2 * sizeof(int32_t), st)) != cudaSuccess)
    return fail(BGT_ECUDA, std::string("scratch clear: ") + cudaGetErrorString(ce));
  const int32_t seg = t.turns_per_launch > 0 ? t.turns_per_launch : n_turns;
  for (int32_t k = 0; k < n_turns; k += seg) {
    a.turn0 = turn0 + k;
    a.n_turns = std::min(seg, n_turns - k);
    if (k > 0 && (ce = cudaMemsetAsync(d_counter, 0, sizeof(int32_t), st)) != cudaSuccess)
      return fail(BGT_ECUDA, std::string("scratch clear: ") + cudaGetErrorString(ce));
    ce = launch(a, (int)grid, smem, st);
    if (ce != cudaSuccess) return fail(BGT_ECUDA, std::string("track_kernel launch: ") + cudaGetErrorString(ce));
  }
  // the call's error flag (1 = a table-staging wait ran out) for the caller
  if (d_status &&
      (ce = cudaMemcpyAsync(d_status, d_counter + 1, sizeof(int32_t), cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
    return fail(BGT_ECUDA, std::string("status copy: ") + cudaGetErrorString(ce));
  return 0;
}
