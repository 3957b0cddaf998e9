/*
 * bgt_mlp.h -- C ABI of the survival classifier that prunes dynamic-aperture
 * scans (libbgt.so).  No counterpart in the reference: Bmad's
 * dynamic_aperture program (bsim/dynamic_aperture, driven by
 * bmad/modules/dynamic_aperture_mod.f90:27-398) tracks every probe to the
 * full turn count; these entry points let a caller retire probes that a
 * network trained on the tracker's own survive/lost labels marks as certain,
 * and keep the plain FP64 tracker for every uncertain or audited probe.
 *
 * Network: 64 inputs (30 features used, the rest zero) -> 256 -> 256 -> 256
 * (ReLU) -> 1 (sigmoid), BF16 weights and activations, FP32 accumulation.
 * The three hidden layers run as tcgen05 tensor-core GEMMs with accumulators
 * in tensor memory; the output layer, loss and optimiser run on CUDA cores.
 *
 * Device buffers are caller-owned; every call is asynchronous on `stream`
 * (a cudaStream_t, NULL = legacy default stream) unless it returns host data.
 * Return codes are those of bgt.h (0 = success, negative = error).
 */
#ifndef BGT_MLP_H
#define BGT_MLP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BGT_MLP_IN 64         /* padded input width (bf16) */
#define BGT_MLP_FEATURES 30   /* features actually used */
#define BGT_MLP_HIDDEN 256
/* flat FP32 parameter vector: W1[256][64], b1[256], W2[256][256], b2[256],
 * W3[256][256], b3[256], w4[256], b4 */
#define BGT_MLP_N_PARAMS 148481
/* per-variant optics/error table row used by bgt_mlp_features: closed orbit
 * (6), eta_x, etap_x, eta_y, etap_y, beta_a, alpha_a, beta_b, alpha_b,
 * error summary (16) */
#define BGT_MLP_VARIANT_COLS 30

typedef struct bgt_mlp bgt_mlp;

/* Network state on `device`, buffers for training batches of up to
 * max_batch samples (a multiple of 128), weights from a seeded He-uniform
 * draw. */
int bgt_mlp_create(bgt_mlp** out, int32_t max_batch, uint64_t seed, int32_t device);
int bgt_mlp_destroy(bgt_mlp* m);
const char* bgt_mlp_last_error(const bgt_mlp* m);
int64_t bgt_mlp_launch_count(const bgt_mlp* m);

/* FP32 master parameters, BGT_MLP_N_PARAMS floats (host arrays).  Setting
 * them also resets the optimiser moments. */
int bgt_mlp_get_params(bgt_mlp* m, float* params);
int bgt_mlp_set_params(bgt_mlp* m, const float* params);

/* p(lost) for n samples: d_x bf16 [n][64] row-major, n a multiple of 128;
 * d_prob float [n]. */
int bgt_mlp_forward(bgt_mlp* m, const uint16_t* d_x, int64_t n, float* d_prob, void* stream);

/* Gradient of the mean binary cross-entropy over one batch (batch <= max_batch,
 * a multiple of 128; labels 1 = lost, 0 = survived) into d_grad (device,
 * BGT_MLP_N_PARAMS floats, may be NULL to keep it internal).  If loss is not
 * NULL the call synchronises and writes the batch loss. */
int bgt_mlp_gradients(bgt_mlp* m, const uint16_t* d_x, const float* d_label, int32_t batch, float* d_grad,
                      float* loss, void* stream);

/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on one batch. */
int bgt_mlp_train_step(bgt_mlp* m, const uint16_t* d_x, const float* d_label, int32_t batch, float lr,
                       float* loss, void* stream);

/* Classifier inputs from tracked particles.  d_vec0 / d_vec: FP64 SoA
 * [6][stride] coordinates at the start and after the early turns;
 * d_variant int32 [n]; d_table FP64 [n_variants][BGT_MLP_VARIANT_COLS].
 * Features: start coordinates - closed orbit (6), error summary (16),
 * current coordinates - closed orbit (6), sqrt of the two linear actions
 * (2, dispersion removed with the current pz).  d_raw (optional) receives
 * float [n][30]; d_x (optional) receives bf16 [n][64] of
 * (raw - mean) * inv_std, zero padded (d_mean, d_inv_std float [30]). */
int bgt_mlp_features(const double* d_vec0, const double* d_vec, int64_t n, int64_t stride, const int32_t* d_variant,
                     const double* d_table, int32_t n_variants, const float* d_mean, const float* d_inv_std,
                     float* d_raw, uint16_t* d_x, void* stream);

/* The tensor-core GEMM the network is built from, exposed for testing:
 * C[m][n] (float, row-major) = A[m][k] . B[n][k]^T with bf16 A, B (row-major,
 * leading dimensions lda, ldb in elements); m a multiple of 128, n 64 or 256,
 * k a multiple of 64. */
int bgt_mlp_gemm_bf16(const uint16_t* d_a, int64_t lda, const uint16_t* d_b, int64_t ldb, int32_t m, int32_t n,
                      int32_t k, float* d_c, void* stream);

/* Test of the GEMM's bounded mbarrier waits: the same launch with no MMA and
 * no commit issued, so every wait runs out after wait_limit_us (> 0) with
 * nothing outstanding; the kernel frees its tensor memory and returns, and
 * the call reports BGT_ETIMEOUT.  d_c is not written. */
int bgt_mlp_gemm_bf16_wait_test(const uint16_t* d_a, int64_t lda, const uint16_t* d_b, int64_t ldb, int32_t m,
                                int32_t n, int32_t k, float* d_c, uint32_t wait_limit_us, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BGT_MLP_H */
