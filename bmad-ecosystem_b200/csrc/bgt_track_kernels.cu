// bgt_track_kernels.cu -- explicit instances of track_kernel, one group per
// compilation: build.py compiles this file once per group with
// -DBGT_KERNEL_GROUP=0..9, so the groups compile in parallel.
//
// Groups 0-4 hold the RARE = false kernels, 5-9 the RARE = true ones, each
// over the same shapes:
//   table in shared memory (TMODE 0): 64 x (8, 10, 12, 16), 128 x (4, 5, 6, 8),
//     256 x (2, 3, 4) threads x resident CTAs per SM (register caps 128, 102,
//     85 and 64 per thread through __launch_bounds__);
//   table in global memory, CTA tiles (TMODE 1) and warp tiles (TMODE 2):
//     128 x (3, 4, 5), 256 x (2, 3) -- 128 x 3 (170 registers, no spills) for
//     small long-lived sets where one particle's turn latency sets the time.
#include "bgt_kernel.cuh"

#ifndef BGT_KERNEL_GROUP
#error "compile with -DBGT_KERNEL_GROUP=<0..9>"
#endif

#define BGT_RARE (BGT_KERNEL_GROUP >= 5)
#if BGT_KERNEL_GROUP % 5 == 0
#define BGT_SHAPES X(64, 8, 0) X(64, 10, 0) X(64, 12, 0) X(64, 16, 0)
#elif BGT_KERNEL_GROUP % 5 == 1
#define BGT_SHAPES X(128, 4, 0) X(128, 5, 0) X(128, 6, 0) X(128, 8, 0)
#elif BGT_KERNEL_GROUP % 5 == 2
#define BGT_SHAPES X(256, 2, 0) X(256, 3, 0) X(256, 4, 0)
#elif BGT_KERNEL_GROUP % 5 == 3
#define BGT_SHAPES X(128, 3, 1) X(128, 4, 1) X(128, 5, 1) X(256, 2, 1) X(256, 3, 1)
#else
#define BGT_SHAPES X(128, 3, 2) X(128, 4, 2) X(128, 5, 2) X(256, 2, 2) X(256, 3, 2)
#endif

#define BGT_CAT2(a, b) a##b
#define BGT_CAT(a, b) BGT_CAT2(a, b)

namespace bgt {

static const TrackKernel kGroupKernels[] = {
#define X(b, m, t) {b, m, t, BGT_RARE, &launch_track<b, m, t, BGT_RARE>},
    BGT_SHAPES
#undef X
};

static cudaError_t upload_cm(const double* cm, const double* cm0, size_t bytes) {
  if (bytes != sizeof(c_cm) || bytes != sizeof(c_cm0)) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemcpyToSymbol(c_cm, cm, bytes);
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_cm0, cm0, bytes);
  return e;
}

TrackKernelGroup BGT_CAT(track_kernel_group_, BGT_KERNEL_GROUP)() {
  return {kGroupKernels, (int)(sizeof(kGroupKernels) / sizeof(kGroupKernels[0])), upload_cm};
}

}  // namespace bgt
