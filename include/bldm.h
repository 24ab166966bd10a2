/*
 * bldm.h — C ABI of the B200-native multiplicative-update Best Latent
 * Decomposition solver (libbldm.so).
 *
 * The reference (eozd/bnmf-algs) exposes this path as C++ templates only:
 *
 *   template <typename T, typename Scalar>
 *   tensor_t<T, 3> bld::bld_mult(const matrix_t<T>& X, size_t z,
 *                               const alloc_model::Params<Scalar>& params,
 *                               size_t max_iter = 1000,
 *                               bool use_psi_appr = false,
 *                               double eps = 1e-50);
 *   (src/bld/bld_mult/bld_mult.hpp:82-86; bld_mult_cuda at :225-229 has the
 *   same signature)
 *
 * These entry points are what that template binds to (see the header-only
 * C++14 mirror bnmf-algs_b200/cpp/bnmf_algs_b200/bld_mult.hpp).  Plain
 * pointers and sizes only.  Layouts are row-major like the reference's
 * matrix_t / tensor_t (src/defs.hpp:40-52): X(i,j) at i*y+j and S(i,j,k) at
 * (i*y+j)*z+k.  Every function returns a bldm_status.
 */
#ifndef BLDM_H_
#define BLDM_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference reports argument errors with BNMF_ASSERT
 * (src/defs.hpp:12-20), which throws std::invalid_argument in test builds;
 * the C++ mirror maps BLDM_ERR_BAD_ARG and BLDM_ERR_NEG_X to that exception
 * and every other failure to std::runtime_error. */
typedef enum bldm_status {
    BLDM_OK = 0,
    BLDM_ERR_BAD_ARG = 1,     /* null pointer, size mismatch (alpha != x, beta != z) */
    BLDM_ERR_NEG_X = 2,       /* X has a negative or NaN entry (check_bld_params) */
    BLDM_ERR_OOM = 3,         /* device allocation failed */
    BLDM_ERR_CUDA = 4,        /* a CUDA runtime call or launch failed */
    BLDM_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up */
    BLDM_ERR_NO_DEVICE = 6,   /* no usable CUDA device */
    BLDM_ERR_UNSUPPORTED = 7, /* batch/server: z beyond the fused kernels' range; a tuning
                                 the shape cannot take */
    BLDM_ERR_BUSY = 8,        /* serving: no slot or memory for the request now */
    BLDM_ERR_NOT_FOUND = 9,   /* serving: unknown request id */
    BLDM_ERR_TOO_LARGE = 10   /* the shape's scratch exceeds a fixed scratch area */
} bldm_status;

/* Digamma selection.
 *   BLDM_PSI_EXACT       — exact digamma everywhere: bld::bld_mult with
 *                          use_psi_appr=false (bld_mult.hpp:119-120).
 *   BLDM_PSI_APPR        — util::psi_appr everywhere (use_psi_appr=true).
 *   BLDM_PSI_LEGACY_CUDA — bld::bld_mult_cuda with use_psi_appr=false: its
 *                          grad_plus kernel always uses psi_appr
 *                          (cuda_src/bld_mult/bld_mult_cuda_kernels.cu:116)
 *                          while grad_minus uses the exact digamma
 *                          (bld_mult.hpp:286,309). */
typedef enum bldm_psi_mode {
    BLDM_PSI_EXACT = 0,
    BLDM_PSI_APPR = 1,
    BLDM_PSI_LEGACY_CUDA = 2
} bldm_psi_mode;

/* Storage precision of S and X on the device. */
typedef enum bldm_dtype { BLDM_F64 = 0, BLDM_F32 = 1 } bldm_dtype;

/* alloc_model::Params<Scalar> (src/alloc_model/alloc_model_params.hpp:25-84):
 * Gamma shape a and rate b, Dirichlet parameters alpha (length x) and beta
 * (length z).  a and b are not used by bld_mult itself; they are carried for
 * log_marginal_S. */
typedef struct bldm_params {
    double a;
    double b;
    const double* alpha;
    size_t n_alpha;
    const double* beta;
    size_t n_beta;
} bldm_params;

/* Per-call statistics (optional output; pass NULL to skip). */
typedef struct bldm_stats {
    double device_ms;       /* device time of the iterations (CUDA events) */
    double total_ms;        /* host wall time of the whole call */
    uint64_t iterations;    /* iterations run */
    uint64_t kernel_launches; /* kernels launched by the call */
    double rel_change;      /* ||S_last - S_prev||_1 / ||S_last||_1 (batch/server) */
    /* Row-sum conservation of the result, max_ij |sum_k S(i,j,k) - X(i,j)| /
     * max(X(i,j), 1), computed on the device after the last iteration.  The
     * reference's tests check S_ij+ against X after a solve
     * (test/bld/bld_mult/test_bld_mult.cpp:67-71,80-84); the update uses the
     * pre-update sums (bld_mult_funcs.hpp:307-327), so it is zero only at the
     * fixed point and is reported rather than enforced. */
    double conservation_residual;
} bldm_stats;

/* ------------------------------------------------------------------------
 * Drop-in host-buffer solve.
 *
 * Replaces bld::bld_mult_cuda (src/bld/bld_mult/bld_mult.hpp:225-324) and,
 * with BLDM_PSI_EXACT, bld::bld_mult (bld_mult.hpp:82-150).  X (x*y) and the
 * result S_out (x*y*z) are HOST buffers (pinned memory makes the copies
 * faster but is not required).  S0 (x*y*z, host) is the initial allocation
 * tensor; when NULL it is drawn on the device as S(i,j,:) = X(i,j) *
 * Dirichlet(1_z) from a counter-based generator seeded with `seed` (the
 * reference's init_S, bld_mult_funcs.hpp:36-74, is GSL-seeded and
 * thread-count dependent).  The call is synchronous.  Device buffers are
 * kept in a per-device cache between calls of the same shape (release them
 * with bldm_release_cache).
 *
 * _f64: FP64 storage and arithmetic.  _f32: FP32 storage and arithmetic with
 * Kahan-compensated axis sums; X and S are FP32 host buffers.
 * ---------------------------------------------------------------------- */
int bldm_solve_f64(const double* X, size_t x, size_t y, size_t z,
                   const bldm_params* params, size_t max_iter, int psi_mode,
                   double eps, const double* S0, uint64_t seed, double* S_out,
                   bldm_stats* stats);
int bldm_solve_f32(const float* X, size_t x, size_t y, size_t z,
                   const bldm_params* params, size_t max_iter, int psi_mode,
                   double eps, const float* S0, uint64_t seed, float* S_out,
                   bldm_stats* stats);

/* Free the device buffers cached by bldm_solve_* on the current device. */
int bldm_release_cache(void);

/* ------------------------------------------------------------------------
 * Device-buffer plan.  For callers that keep X and S resident in HBM
 * (serving, frameworks).  A plan owns the solver's workspace for one shape.
 * d_X (x*y), d_S (x*y*z) are device buffers of the plan's dtype, 16-byte
 * aligned and allocated in multiples of 16 bytes (cudaMalloc and the torch
 * caching allocator both satisfy this); d_alpha (x) and d_beta (z) are FP64
 * device buffers.  d_S holds S0 on entry and the solution on return.  Work
 * is enqueued on `stream` (a cudaStream_t; NULL = legacy default stream) and
 * the call returns without synchronising; bldm_plan_check asynchronously
 * surfaces a device-side error once the stream has drained.
 * ---------------------------------------------------------------------- */
typedef struct bldm_plan bldm_plan;

int bldm_plan_create(bldm_plan** plan, size_t x, size_t y, size_t z, int dtype);

/* Launch knobs of the fused sweep; 0 = chosen by the library.  stages: depth
 * of the shared-memory ring of bulk-copied row segments (2..8); ctas_per_sm:
 * resident sweep CTAs per SM (1 or 2); row_ranges: row ranges the rows of a
 * band of columns are split into (one CTA each).  The reference has no
 * counterpart (its kernels use fixed 32x32 / 16x16x4 blocks,
 * cuda_src/bld_mult/bld_mult_cuda_funcs.cu:18-24); the autotuner sets them.
 * skip_zero_rows = 1: an update maps every fiber with X == 0 to zero, so once
 * the first update of a run has stored those zeros, the later updates neither
 * read nor write the rows of a band whose X segment is all zero, nor store
 * the zeros of single fibers with X == 0 again.  The result is bitwise the
 * same; the work scales with the rows that hold nonzeros.  Off by default:
 * the plain path streams all of S each iteration as the reference does. */
typedef struct bldm_tuning {
    int stages;
    int ctas_per_sm;
    int row_ranges;
    int skip_zero_rows;
} bldm_tuning;
int bldm_plan_create_tuned(bldm_plan** plan, size_t x, size_t y, size_t z, int dtype,
                           const bldm_tuning* tuning);
int bldm_plan_get_tuning(const bldm_plan* plan, bldm_tuning* out);
int bldm_plan_destroy(bldm_plan* plan);
/* Bytes of device workspace the plan holds (partials, digamma tables). */
int bldm_plan_workspace_bytes(const bldm_plan* plan, size_t* bytes);
int bldm_plan_run(bldm_plan* plan, const void* d_X, const double* d_alpha,
                  const double* d_beta, void* d_S, size_t max_iter,
                  int psi_mode, double eps, void* stream);
/* The same solve as bldm_plan_run without allocating anything.  No counterpart
 * in the reference.  For callers that cannot allocate device memory while they
 * solve: cudaMalloc/cudaFree may synchronise the device (too slow for a
 * latency-bound serving loop), and a raw allocation can fail with out-of-memory
 * in a process whose device memory another allocator (a framework's caching
 * allocator, a server's up-front reservation) already holds.  The solver's
 * scratch comes from a fixed 32 MiB array in the library's device data, held on
 * every GPU where the library's device code is loaded until the process exits;
 * shapes whose scratch exceeds it return BLDM_ERR_TOO_LARGE (1024x1024x64 FP64
 * needs 22.5 MB).  The caller passes device buffers as for bldm_plan_run (dtype
 * is BLDM_F64 or BLDM_F32).  The first call on a device looks up the array's
 * device address on that device and keeps it for later calls (make that first
 * call before any stream capture); after cudaDeviceReset, or anything else
 * that unloads the library's device code from that device, the kept address no
 * longer belongs to the new context, so do not call this entry point on that
 * device again in the same process.  All calls on a device share the array,
 * and calls that overlap on the GPU race.  Synchronises `stream` before
 * returning and reports a device-side error as BLDM_ERR_TIMEOUT. */
int bldm_solve_device_noalloc(const void* d_X, const double* d_alpha,
                              const double* d_beta, void* d_S, size_t x, size_t y,
                              size_t z, int dtype, size_t max_iter, int psi_mode,
                              double eps, void* stream);
/* Synchronises `stream` and reports a device-side error recorded by the
 * plan's kernels (BLDM_ERR_TIMEOUT) or a CUDA error. */
int bldm_plan_check(bldm_plan* plan, void* stream);
/* Row-sum conservation residual max_ij |sum_k S(i,j,k) - X(i,j)| / max(X(i,j), 1)
 * of device buffers of the plan's shape and dtype, computed on the device (one
 * read of S, FP64 sums) behind the work queued on `stream`; synchronises
 * `stream`.  The check the reference's tests make after a solve
 * (test/bld/bld_mult/test_bld_mult.cpp:67-71,80-84). */
int bldm_plan_conservation(bldm_plan* plan, const void* d_X, const void* d_S, void* stream,
                           double* residual);
/* Draw the seeded initial S on the device (see bldm_solve_f64). */
int bldm_plan_init_S(bldm_plan* plan, const void* d_X, void* d_S, uint64_t seed,
                     void* stream);
/* Run `iters` iterations with CUDA events around every launch of the fused
 * update kernel and report its mean duration (ms) and the mean duration of
 * one whole iteration (ms).  Used to place the kernel on the HBM roofline. */
int bldm_plan_profile(bldm_plan* plan, const void* d_X, const double* d_alpha,
                      const double* d_beta, void* d_S, size_t iters,
                      int psi_mode, double eps, void* stream,
                      double* update_kernel_ms, double* iteration_ms);
/* Kernels launched by the plan since creation. */
int bldm_plan_launch_count(const bldm_plan* plan, uint64_t* count);

/* Row-sharded solve (for one instance larger than a GPU's memory): shard g
 * of G holds rows [i0, i1) of X, S and alpha in a plan of (i1-i0) x y x z.
 * Only the sums over rows cross shards: S_+jk (y*z) and sum_i alpha_eph(i,k)
 * (z), packed in a device buffer `red` of bldm_plan_shard_red_size doubles.
 * One iteration: bldm_plan_shard_update (the shard's update sweep; red gets
 * the shard's sums), an in-place sum of red over the shards (an all-reduce,
 * e.g. NCCL), bldm_plan_shard_finish (the digamma tables from the global
 * sums).  Start with bldm_plan_shard_sums (the sums of the initial S), the
 * all-reduce and bldm_plan_shard_finish.  With one shard the iterations are
 * bitwise those of bldm_plan_run.  The reference has no sharded solver; the
 * exchange step is the one its CUDA driver performs on the host
 * (src/bld/bld_mult/bld_mult.hpp:289-312) over the whole tensor. */
int bldm_plan_shard_red_size(const bldm_plan* plan, size_t* n_doubles);
int bldm_plan_shard_sums(bldm_plan* plan, const void* d_S, const double* d_alpha, double* d_red,
                         int psi_mode, void* stream);
int bldm_plan_shard_update(bldm_plan* plan, const void* d_X, void* d_S, const double* d_alpha,
                           double* d_red, int psi_mode, double eps, void* stream);
int bldm_plan_shard_finish(bldm_plan* plan, const double* d_beta, const double* d_red,
                           int psi_mode, void* stream);
/* ------------------------------------------------------------------------
 * Per-stage device functions.  Each mirrors one function of the reference's
 * CUDA host side so that every formula can be checked against the CPU
 * restatement on its own (the reference's test strategy,
 * test/bld/bld_mult/test_bld_mult_cuda_funcs.cpp).  All pointers are FP64
 * device buffers, row-major, unpadded; work goes to `stream`.
 * ---------------------------------------------------------------------- */
/* cuda::tensor_sums (cuda_src/tensor_ops.cu:10-55): S_pjk (y*z), S_ipk
 * (x*z), S_ijp (x*y). */
int bldm_tensor_sums_f64(const double* d_S, size_t x, size_t y, size_t z,
                         double* d_pjk, double* d_ipk, double* d_ijp,
                         void* stream);
/* update_grad_plus_cuda (cuda_src/bld_mult/bld_mult_cuda_funcs.cu:8-33):
 * gp(i,j,k) = psi(beta_eph(j,k)) - psi(S(i,j,k)+1).  appr != 0 selects
 * psi_appr (the reference kernel always does). */
int bldm_update_grad_plus_f64(const double* d_S, const double* d_beta_eph,
                              size_t x, size_t y, size_t z, int appr,
                              double* d_grad_plus, void* stream);
/* update_grad_minus (bld_mult_funcs.hpp:205-229; host-side in the
 * reference): gm(i,k) = psi(sum_i alpha_eph(i,k)) - psi(alpha_eph(i,k)). */
int bldm_update_grad_minus_f64(const double* d_alpha_eph, size_t x, size_t z,
                               int appr, double* d_grad_minus, void* stream);
/* update_nom_cuda (bld_mult_cuda_funcs.cu:36-61):
 * nom(i,j) = sum_k S(i,j,k) Xr(i,j) gm(i,k). */
int bldm_update_nom_f64(const double* d_X_reciprocal, const double* d_grad_minus,
                        const double* d_S, size_t x, size_t y, size_t z,
                        double* d_nom, void* stream);
/* update_denom_cuda (bld_mult_cuda_funcs.cu:64-88):
 * denom(i,j) = sum_k S(i,j,k) Xr(i,j) gp(i,j,k). */
int bldm_update_denom_f64(const double* d_X_reciprocal, const double* d_grad_plus,
                          const double* d_S, size_t x, size_t y, size_t z,
                          double* d_denom, void* stream);
/* update_S_cuda (bld_mult_cuda_funcs.cu:91-120), with the caller's eps (the
 * reference kernel hard-codes 1e-50, bld_mult_cuda_kernels.cu:209). */
int bldm_update_S_f64(const double* d_X, const double* d_nom,
                      const double* d_denom, const double* d_grad_minus,
                      const double* d_grad_plus, const double* d_S_ijp,
                      size_t x, size_t y, size_t z, double eps, double* d_S,
                      void* stream);
/* util::psi_appr / exact digamma over an array: appr == 0 exact, 1 psi_appr,
 * 2 psi_appr as evaluated inside the fused sweep (same function, batched
 * form with Newton-Raphson reciprocals and a table logarithm). */
int bldm_psi_f64(const double* d_in, size_t n, int appr, double* d_out, void* stream);
/* FP32 digamma for FP32 storage: mode 0 the form that tabulates psi(alpha_eph)
 * and psi(beta_eph) (IEEE division, libm logarithm), mode 1 the form the
 * fused FP32 sweep evaluates for psi(S+1) (three-step rational shift,
 * Newton-Raphson reciprocal, hardware logarithm).  The reference evaluates
 * util::psi_appr (src/util/util.hpp:440-514) in the storage type. */
int bldm_psi_f32(const float* d_in, size_t n, float* d_out, void* stream);
int bldm_psi_f32_mode(const float* d_in, size_t n, int mode, float* d_out, void* stream);

/* alloc_model::log_marginal_S (src/alloc_model/alloc_model_funcs.hpp:573-586)
 * of a device tensor, computed on the device in FP64.  d_S is FP64 or FP32
 * per dtype; alpha (x) and beta (z) are HOST arrays. */
int bldm_log_marginal_S(const void* d_S, int dtype, size_t x, size_t y, size_t z,
                        const double* alpha, const double* beta, double a,
                        double b, double* result, void* stream);

/* bld::bld_fact (src/bld/bld_fact.hpp:36-80): W (x*z), H (z*y) and L (y)
 * from a BLD solution S, W(i,k) = (alpha_i + S_i+k - 1) / (sum over i of the
 * same + eps), H(k,j) = (beta_k + S_+jk - 1) / (sum over k of the same + eps),
 * L(j) = (a + S_+j+ - 1) / (b + 1 + eps).  Device tensors of the storage
 * dtype, row-major; params' alpha and beta are host arrays.  The sums are
 * reduced in FP64.  Synchronises `stream`. */
int bldm_bld_fact(const void* d_S, int dtype, size_t x, size_t y, size_t z,
                  const bldm_params* params, double eps, void* d_W, void* d_H, void* d_L,
                  void* stream);
/* The same on host FP64 arrays (the reference's interface; copies in and out). */
int bldm_bld_fact_f64(const double* S, size_t x, size_t y, size_t z, const bldm_params* params,
                      double eps, double* W, double* H, double* L);

/* alloc_model::bnmf_priors (src/alloc_model/alloc_model_funcs.hpp:461-502) on
 * the device: L_j ~ Gamma(a, scale b) (GSL's gsl_ran_gamma parameterisation,
 * as the reference), each column of W (x*z) ~ Dirichlet(alpha), each column of
 * H (z*y) ~ Dirichlet(beta).  Device outputs of the storage dtype; params'
 * alpha and beta are host arrays.  The draws come from a counter-based stream
 * of `seed` (the reference's GSL stream is not reproduced).  Synchronises
 * `stream`. */
int bldm_bnmf_priors(size_t x, size_t y, size_t z, const bldm_params* params, uint64_t seed,
                     int dtype, void* d_W, void* d_H, void* d_L, void* stream);
/* alloc_model::sample_S (alloc_model_funcs.hpp:523-552): S_ijk ~
 * Poisson(W_ik H_kj L_j), device tensors of the storage dtype. */
int bldm_sample_S(const void* d_W, const void* d_H, const void* d_L, size_t x, size_t y,
                  size_t z, uint64_t seed, int dtype, void* d_S, void* stream);
/* X_ij ~ Poisson(sum_k W_ik H_kj L_j), the distribution of sum_k S_ijk, drawn
 * directly (no counterpart in the reference, which sums a sampled S). */
int bldm_sample_X(const void* d_W, const void* d_H, const void* d_L, size_t x, size_t y,
                  size_t z, uint64_t seed, int dtype, void* d_X, void* stream);

/* ------------------------------------------------------------------------
 * Batched solver: many independent instances of different shapes (x, y, z
 * each) solved together.  No counterpart in the reference, which solves one
 * instance per call.  An instance's tiling depends only on its own shape and
 * its class's launch shape, so its result does not depend on the other
 * instances of the batch; it agrees with bldm_plan_run's to rounding (the
 * partial sums are grouped by tile).  One iteration of every instance is one
 * fused-sweep launch and one finalize launch per lane-shape class (instances
 * whose z maps to the same kernel), each class running its iterations on its
 * own forked stream; with use_graph the whole run is captured once per
 * (iters, psi_mode, eps) into a CUDA graph and replayed.  A class's tiles run
 * heaviest first by the work their X implies (rows with a nonzero, passes
 * with a nonzero); the order changes no result.
 * rows_per_tile (0 = 64) is the default tile height (rows of S per CTA tile)
 * of every class; bldm_batch_autotune picks it and the stage-ring depth per
 * class from timed probe runs on the batch's own data.
 * X, S0 and S_out are host FP64 arrays (converted for BLDM_F32 storage).
 * ---------------------------------------------------------------------- */
typedef struct bldm_batch bldm_batch;
int bldm_batch_create(bldm_batch** batch, int dtype, size_t n, const size_t* xs,
                      const size_t* ys, const size_t* zs, int rows_per_tile);
int bldm_batch_destroy(bldm_batch* batch);
/* Instance idx's data; S0 NULL draws the seeded initial S on the device.
 * The next bldm_batch_run first rebuilds the launch tables in the tile order
 * of the X values set (host work on that call only). */
int bldm_batch_set(bldm_batch* batch, size_t idx, const double* X, const double* alpha,
                   const double* beta, const double* S0, uint64_t seed);
/* Runs `iters` iterations of every instance from its current S (asynchronous
 * on `stream`; use_graph needs a non-NULL stream). */
int bldm_batch_run(bldm_batch* batch, size_t iters, int psi_mode, double eps,
                   int use_graph, void* stream);
int bldm_batch_check(bldm_batch* batch, void* stream);
/* Launch form of bldm_batch_run.  persistent = 0 (the default): per iteration,
 * one sweep launch per lane-shape class (the classes side by side on forked
 * streams) and one finalize launch for all instances.  persistent = 1: one
 * persistent launch per class runs every iteration of every instance of the
 * class from an ordered work queue; each tile finalizes its share of its
 * instance in its epilogue and an instance moves to its next iteration as soon
 * as its own previous one is complete (no grid-wide barrier, no per-iteration
 * launches).  Classes whose fibers need more than two chunks per lane always
 * use the default form.  The two forms agree to rounding (the sum of alpha_eph
 * over rows is grouped by row blocks in one and by tile row ranges in the
 * other); each is deterministic.  On batches of many small instances the
 * default form is faster: a class of small instances is bound by the latency
 * of its iterations, and only the side-by-side launches of the default form
 * overlap the classes.  wait_limit_s bounds each device-side dependency wait
 * of the persistent form (> 0, <= 60; default 1); when one runs out the run
 * stops and bldm_batch_check reports BLDM_ERR_TIMEOUT.  stall_test = 1 is for
 * tests of that failure path only: instance 0's first-iteration tiles then
 * wait for the completion of that same iteration, so the wait runs out.  No
 * counterpart in the reference. */
int bldm_batch_set_launch_mode(bldm_batch* batch, int persistent, double wait_limit_s,
                               int stall_test);
/* 1 when bldm_batch_run uses the persistent form for this batch. */
int bldm_batch_get_launch_mode(const bldm_batch* batch, int* persistent);
/* Instance idx's S (x*y*z) and the relative change sum|S_n - S_{n-1}| /
 * sum|S_n| of the run's last iteration; either output may be NULL. */
int bldm_batch_get(bldm_batch* batch, size_t idx, double* S_out, double* rel_change);
/* Row-sum conservation residual (as bldm_plan_conservation) of every
 * instance's current S, residuals[n], in one device launch behind `stream`;
 * synchronises `stream`. */
int bldm_batch_conservation(bldm_batch* batch, double* residuals, void* stream);
/* Device buffers of instance idx (storage dtype), for device-resident callers. */
int bldm_batch_device_ptrs(bldm_batch* batch, size_t idx, void** d_X, void** d_S);
int bldm_batch_info(const bldm_batch* batch, size_t* n_classes, size_t* device_bytes,
                    uint64_t* launches);

/* Launch shape of one lane-shape class of a batch. */
typedef struct bldm_batch_class {
    int vec;              /* elements per lane access */
    int lanes_per_fiber;  /* lanes sharing one (i,j) fiber */
    int chunks;           /* vec-element chunks per lane and fiber */
    int multirow;         /* 1: narrow rows, several rows per stage */
    int rows_per_tile;    /* tile height: rows of S per CTA tile */
    int stages;           /* bulk-copy ring depth (row segments of S in flight per CTA) */
    size_t tiles;         /* CTA tiles per sweep launch */
    size_t instances;     /* instances of the batch in this class */
} bldm_batch_class;
/* Class idx (< n_classes of bldm_batch_info) as the last build laid it out. */
int bldm_batch_class_info(const bldm_batch* batch, size_t idx, bldm_batch_class* out);
/* Sets the launch shape of the class with c's (vec, lanes_per_fiber, chunks,
 * multirow); rows_per_tile >= 32 (0 = the batch default), stages >= 2 or 0
 * (= as deep as shared memory allows).  Re-tiles and rebuilds the batch. */
int bldm_batch_set_class(bldm_batch* batch, const bldm_batch_class* c);
/* Autotuner: for each class, largest first, tries tile heights
 * {32, 64, 128, 256, 512} and stage depths {2, 3, 4, 6, 8}, timing
 * probe_iters iterations of the whole batch (CUDA events, best of three) in
 * the steady state of a run (from the S after one update, skipping zero rows
 * from the first probe iteration on), and keeps a change when the batch gets
 * at least 3% faster.  S is saved on the device and restored afterwards, so the
 * call does not change the solution.  Call after bldm_batch_set of every
 * instance.
 * default_ms / tuned_ms (nullable): probe time before and after. */
int bldm_batch_autotune(bldm_batch* batch, size_t probe_iters, int psi_mode, double eps,
                        void* stream, double* default_ms, double* tuned_ms);

/* ------------------------------------------------------------------------
 * Serving loop with continuous batching.  No counterpart in the reference.
 * A worker thread admits submitted requests while a slot (max_active) and
 * device memory (memory_budget bytes, 0 = 80% of the free memory at create,
 * and the device's current free memory) allow, keeps each request's X, S and
 * tables on the device, runs iters_per_round iterations of all active
 * requests per round in shared launches, and retires a request when the
 * relative change of S (sum|S_n - S_{n-1}| / sum|S_n| over its last
 * iteration) falls below tol or it has run max_iter iterations (rounded up to
 * a whole round).  Newly admitted requests get their axis sums on their own
 * before joining the round; the others carry theirs over from the previous
 * round.  Retirement runs on another thread and stream per lane, so the rounds go on
 * meanwhile: it copies S to the host (in the storage type; fetch converts to
 * FP64), computes log_marginal_S on the device (FP64) and frees the request's
 * device memory.  Requests of at least large_elements S elements are served
 * in a second lane with its own worker and a lower-priority stream, so that
 * the rounds of small requests do not wait for the large ones'.  A request's
 * result does not depend on the other requests being served.
 * ---------------------------------------------------------------------- */
typedef struct bldm_server bldm_server;
typedef struct bldm_server_config {
    int dtype;               /* BLDM_F64 or BLDM_F32 storage */
    int psi_mode;            /* bldm_psi_mode */
    double eps;              /* the reference's eps (1e-50) */
    double tol;              /* retire when the relative change of S < tol */
    size_t max_iter;         /* iteration cap per request */
    size_t iters_per_round;  /* iterations between admission/retirement points */
    size_t max_active;       /* concurrent requests on the device */
    size_t memory_budget;    /* device bytes for requests; 0 = 80% of free */
    int rows_per_tile;       /* 0 = 64 */
    size_t large_elements;   /* requests with x*y*z >= this are served in a second
                                lane (own worker thread and lower-priority stream);
                                0 = 2^25, SIZE_MAX = one lane */
} bldm_server_config;
typedef struct bldm_request_stats {
    double queue_ms;         /* submit -> admission */
    double latency_ms;       /* submit -> result ready */
    uint64_t iterations;
    double rel_change;       /* relative change of S at retirement */
    double log_marginal;     /* log_marginal_S of the result (FP64) */
    int status;              /* bldm_status of the request */
    double conservation_residual; /* as bldm_stats, computed at retirement */
} bldm_request_stats;
typedef struct bldm_server_stats {
    uint64_t submitted, completed, failed, rounds, iterations;
    size_t active, queued, bytes_in_use, bytes_peak, budget;
    double gpu_ms;           /* device time of the rounds (CUDA events) */
    double host_ms;          /* worker time between rounds (admission, tables) */
    size_t retiring;         /* requests finished on the device, results in flight */
    double gpu_ms_large;     /* the large-request lane's part of gpu_ms (the two
                                lanes' rounds overlap, so gpu_ms may exceed wall time) */
    double retire_ms;        /* retirement threads' time (waiting for the round, result
                                copies, log-marginal) */
} bldm_server_stats;
int bldm_server_create(bldm_server** server, const bldm_server_config* config);
/* Stops the worker; requests still active or queued are dropped. */
int bldm_server_destroy(bldm_server* server);
/* Queues a request (X host x*y, copied); BLDM_ERR_TOO_LARGE if it can never
 * fit the memory budget. */
int bldm_server_submit(bldm_server* server, const double* X, size_t x, size_t y, size_t z,
                       const bldm_params* params, uint64_t seed, uint64_t* request_id);
/* state: 0 queued, 1 active, 2 done, 3 failed. */
int bldm_server_poll(bldm_server* server, uint64_t request_id, int* state);
/* Blocks until the request is done or failed (BLDM_ERR_BUSY on timeout). */
int bldm_server_wait(bldm_server* server, uint64_t request_id, double timeout_s);
/* Copies the result (x*y*z FP64 host; may be NULL) and stats, then forgets
 * the request; returns the request's status. */
int bldm_server_fetch(bldm_server* server, uint64_t request_id, double* S_out,
                      bldm_request_stats* stats);
int bldm_server_cancel(bldm_server* server, uint64_t request_id);
int bldm_server_get_stats(bldm_server* server, bldm_server_stats* stats);

/* Library version string. */
const char* bldm_version(void);

#ifdef __cplusplus
}
#endif

#endif /* BLDM_H_ */
