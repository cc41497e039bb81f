/*
 * ccmpred_b200.h -- C ABI of libccmpred_b200.so, a B200 (sm_100a) implementation
 * of CCMpred's pseudo-likelihood objective + gradient.
 *
 * Two layers:
 *
 *  1. The reference's own backend triple, drop-in compatible with
 *     include/evaluate_cuda.h:8-17 (evaluate_cuda/init_cuda/destroy_cuda, the
 *     libconjugrad evaluate callback with DEVICE x and g) and, for host
 *     pointers, the shape of include/evaluate_cpu.h:21-30 (evaluate_b200 etc.).
 *     `instance` points at a struct with the layout of the reference's
 *     `userdata` (include/ccmpred.h:39-92), declared here as ccm_userdata.
 *     As in the reference (CHECK_ERR, include/evaluate_cuda_kernels.h:9), these
 *     print the error and exit(EXIT_FAILURE) on failure.
 *
 *  2. A context API (ccm_*) with explicit sizes and status codes, one context
 *     per alignment, no process globals, one CUDA stream per context.
 *
 * Parameter vector layout (both layers): the reference's padded layout,
 * include/ccmpred.h:1-17 with PADDING on (N_ALPHA_PAD = 32):
 *   x[a*L + j]                          single field V(j,a), a < 20
 *   x[nsingle .. nsingle_padded)        padding (gradient written as 0)
 *   x[nsingle_padded + ((b*L+k)*32 + a)*L + j]   coupling W(b,k,a,j)
 * with nsingle = 20 L and nsingle_padded = nsingle + 32 - nsingle % 32
 * (src/ccmpred.c:388-390); nvar_padded = nsingle_padded + 21*32*L*L.
 * The gradient is the reference's: the coupling part is the derivative along
 * the tied direction W(b,k,a,j) = W(a,j,b,k) with zeroed self-edge blocks
 * (src/evaluate_cpu.c:131-163).
 */
#ifndef CCMPRED_B200_H
#define CCMPRED_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define CCM_API __attribute__((visibility("default")))
#else
#define CCM_API
#endif

#define CCM_N_ALPHA 21
#define CCM_N_ALPHA_PAD 32

/* status codes of the ccm_* API */
#define CCM_OK 0
#define CCM_ERR_INVALID (-1)      /* bad argument (sizes, null pointers, nvar mismatch) */
#define CCM_ERR_CUDA (-2)         /* a CUDA runtime call failed; see ccm_last_error() */
#define CCM_ERR_NOMEM (-3)        /* device allocation failed */
#define CCM_ERR_DEVICE (-4)       /* a kernel reported a bounded-wait timeout */
#define CCM_ERR_UNSUPPORTED (-5)  /* no sm_100 device / unsupported option */

/* evaluation paths */
#define CCM_PATH_TC_BF16X2 0 /* tcgen05, W and R split into hi+lo bf16, f32 accumulate */
#define CCM_PATH_TC_BF16X3 1 /* tcgen05, three bf16 terms (hi+mid+lo) */
#define CCM_PATH_SIMT_F32 2  /* plain FP32 CUDA-core path (no tensor cores) */
#define CCM_PATH_SIMT_F64 3  /* FP64 CUDA-core path (gradient checks) */
#define CCM_PATH_TC_I8X3 4   /* tcgen05 kind::i8: W and R as three 8-bit fixed-point digits
                                (21 fractional bits), exact s32 accumulation */
#define CCM_PATH_TC_I8SP 5   /* CCM_PATH_TC_I8X3 with the forward on 2:4-sparse tcgen05.mma.sp
                                (the one-hot operand compressed); the same exact sums */

/* gradient conventions */
#define CCM_GRADIENT_TIED 0    /* the reference's g: coupling part along the tied direction
                                  W(b,k,a,j) = W(a,j,b,k), self-edge blocks zeroed, 2 lambda2 W
                                  (src/evaluate_cpu.c:131-163) */
#define CCM_GRADIENT_PARTIAL 1 /* true partial derivatives of f w.r.t. every entry of x: untied
                                  G2 + lambda2 W, self blocks included (gradient checks, autograd) */

typedef struct ccm_context ccm_context;

typedef struct ccm_options {
	float lambda_single; /* default 0.01 (src/ccmpred.c:222) */
	float lambda_pair;   /* default 0.2 * (L - 1) (src/ccmpred.c:224,502-503) */
	int path;            /* CCM_PATH_* ; default CCM_PATH_TC_I8SP */
	int device;          /* CUDA device ordinal; default 0 */
	void *stream;        /* cudaStream_t to run on, or NULL for a private stream that is
	                        ordered with the legacy default stream */
	int gradient;        /* CCM_GRADIENT_*; default CCM_GRADIENT_TIED */
	int max_sms;         /* upper bound on the SMs the tensor-core kernels of this context
	                        occupy (rounded down to CTA pairs); 0 = the whole GPU.  Contexts
	                        that run side by side on one GPU (the batch solver) each take a
	                        share, so that their persistent kernels stay resident together. */
	size_t mem_limit;    /* cap on the device memory of this context, in bytes; 0 = none.
	                        The context counts what it allocates (its buffers, the
	                        optimizer state of ccm_conjugrad_gpu while a solve runs, the
	                        staging buffers of ccm_evaluate_host); an allocation beyond
	                        the cap fails with CCM_ERR_NOMEM instead of taking memory
	                        that other users of the GPU hold. */
} ccm_options;

/* Result of the last evaluation, as kept on the device. */
typedef struct ccm_result {
	double fx;     /* f = data term + regulariser */
	double f_data; /* sum_n w_n sum_j (lse - logit of observed state) */
	double reg;    /* lambda1 sum V^2 + 0.5 lambda2 sum W^2 over all padded slots */
	int status;    /* device error bits, 0 when clean */
	int pad;
} ccm_result;

/* Reference `userdata` (include/ccmpred.h:39-92), float build. */
typedef struct ccm_userdata {
	unsigned char *msa;       /* N x L row-major, states 0..20 */
	float *weights;           /* N sequence weights (filled by init_cuda/init_b200) */
	int ncol;                 /* L */
	int nrow;                 /* N */
	int nsingle;              /* 20 L */
	int nvar;                 /* 20 L + 441 L^2 (unpadded count) */
	void *extra;              /* backend state (a ccm_context*) */
	float lambda_single;
	float lambda_pair;
	float reweighting_threshold;
	void *meta_steps;
} ccm_userdata;

/* ---------------------------------------------------------------- sizes */
CCM_API long long ccm_nsingle_padded(int ncol);
CCM_API long long ccm_nvar_padded(int ncol);

/* ---------------------------------------------------------------- context API */
CCM_API void ccm_options_default(ccm_options *opt, int ncol);

/* Upload the alignment and weights, allocate all device state for `path`.
 * weights == NULL means uniform weights 1.0 (src/reweighting.c:61-67); weights
 * must be finite (any magnitude: the integer paths scale the residuals by the
 * smallest power of two at or above the largest weight).  States above 20 are rejected with
 * CCM_ERR_INVALID.  Replaces init_cuda (src/evaluate_cuda.c:77-139) without
 * process globals. */
CCM_API int ccm_create(ccm_context **ctx, const unsigned char *msa, int ncol, int nrow,
               const float *weights, const ccm_options *opt);
CCM_API int ccm_destroy(ccm_context *ctx);

/* f and g at x; x and g are DEVICE pointers of nvar_padded floats (the
 * conjugrad_gpu convention, src/evaluate_cuda.c:23-74).  g is overwritten.
 * Blocks until the result is on the host; *fx receives f in FP64. */
CCM_API int ccm_evaluate(ccm_context *ctx, const float *d_x, float *d_g, long long nvar_padded,
                 double *fx);

/* Same, enqueued on the context stream without a host synchronisation; the
 * result stays on the device (ccm_result_device) for device-side consumers. */
CCM_API int ccm_evaluate_async(ccm_context *ctx, const float *d_x, float *d_g, long long nvar_padded);

/* Same with HOST x and g (the evaluate_cpu convention, src/evaluate_cpu.c:16-166):
 * copies x in, evaluates, copies g out.  Where the padding states a in [21, 32)
 * of x's coupling block are all zero bits (always on the reference's CLI path),
 * they and g's padding states (then zero) do not cross PCIe: the host checks
 * them while the rest is copied and writes g's as zeros. */
CCM_API int ccm_evaluate_host(ccm_context *ctx, const float *x, float *g, long long nvar_padded,
                      double *fx);
/* Bytes the last ccm_evaluate_host copied host -> device and device -> host. */
CCM_API int ccm_host_copy_bytes(const ccm_context *ctx, long long *h2d, long long *d2h);

/* FP64 evaluation (CCM_PATH_SIMT_F64 contexts): double x and g on the device. */
CCM_API int ccm_evaluate_f64(ccm_context *ctx, const double *d_x, double *d_g, long long nvar_padded,
                     double *fx);

/* Device pointer to the ccm_result written by the last evaluation. */
CCM_API const ccm_result *ccm_result_device(const ccm_context *ctx);
/* Copy the last ccm_result to the host (synchronises the context stream). */
CCM_API int ccm_get_result(ccm_context *ctx, ccm_result *out);

/* Sequence weights held by the context (N floats, host). */
CCM_API int ccm_get_weights(const ccm_context *ctx, float *w);

/* The stream the context runs on (cudaStream_t). */
CCM_API void *ccm_stream(const ccm_context *ctx);

/* Identity-threshold sequence reweighting on the GPU, bit-exact with the
 * serial reference calculate_weights (src/reweighting.c:9-58): integer
 * identity counts, idthres = (int)ceil(threshold * (float)ncol),
 * w_i = (float)(1.0 / (count_i - 1)) with self counted twice. */
CCM_API int ccm_calculate_weights(const unsigned char *msa, int ncol, int nrow, float threshold,
                          float *w, int device);

/* Instrumentation.  ccm_profile_begin records CUDA events on the context
 * stream around every kernel of the next max_evals evaluations;
 * ccm_profile_end synchronises and returns, per kernel position in the
 * launch sequence, the summed device time in ms (tensor-core path: prep,
 * forward, backward, finalize; SIMT path: rows, pairs, single, sym,
 * finalize), the number of kernels per evaluation and of evaluations seen. */
CCM_API int ccm_profile_begin(ccm_context *ctx, int max_evals);
CCM_API int ccm_profile_end(ccm_context *ctx, double *kernel_ms, int max_kernels, int *n_kernels,
                            int *n_evals);
/* Number of kernels this context has launched (evaluations only). */
CCM_API long long ccm_launch_count(const ccm_context *ctx);

/* Diagnostics for tests: copy an internal device buffer of a tensor-core
 * context to host memory `dst` (`bytes` long).  Split-bf16 paths: which = 0:
 * one-hot O (Npad x S bf16); 1..3: Wperm split terms (S x S bf16); 4..6: R split
 * terms (Npad x S bf16); 7: single-field data gradient (20 L float).  Integer
 * paths: 0: one-hot (Npad x S bytes, values 1); 1..3: digits of W (S x S bytes;
 * CCM_PATH_TC_I8SP: KP x SW bytes in the forward's tiled storage); 4..6: digits
 * of R (Npad x S bytes); 7: as above; 8: column maxima of |W| (21 L float bits);
 * CCM_PATH_TC_I8SP only: 9: compressed one-hot (Npad x KP/2 bytes, tiled),
 * 10: its 2:4 metadata (Npad x KP/8 bytes, tiled).  With dst == NULL returns the
 * buffer size in bytes; otherwise 0 or a negative status. */
CCM_API long long ccm_debug_copy(ccm_context *ctx, int which, void *dst, long long bytes);

/* Diagnostics for tests of the bounded waits.  cycles > 0: in the next
 * evaluations of the integer paths, the forward kernel's epilogue waits, with a
 * budget of `cycles` SM clock cycles, on a barrier that no thread arrives on
 * instead of on its accumulator tile.  The wait runs out; the kernel records the
 * timeout, drains its in-flight copies and MMAs, frees its tensor memory and
 * returns, and the evaluation reports CCM_ERR_DEVICE.  cycles = 0 restores
 * normal evaluations; the context stays usable.  No counterpart in the
 * reference (which has no bounded waits). */
CCM_API int ccm_debug_set_wait_limit(ccm_context *ctx, long long cycles);

/* Integer paths: a device-side solve (ccm_conjugrad_gpu, ccm_solve_batch) whose
 * x0 has zero padding states (a in [21, 32) of every coupling row; always so on
 * the reference's CLI path) keeps them zero and skips them in every vector pass
 * (allow = 1, the default).  allow = 0 makes the solve visit every element, for
 * comparisons; results agree up to the summation order of the FP64 dots. */
CCM_API int ccm_debug_set_cg_skip_padding(ccm_context *ctx, int allow);

/* Allocation-free sequence reweighting.  No counterpart in the reference.
 *
 * For callers that must not allocate device memory: a process whose memory
 * pool or framework already owns (nearly) all of the GPU's memory, so that a
 * cudaMalloc would fail or force the pool to give memory back, or a pipeline
 * that cannot afford the device-wide synchronisation that cudaFree implies.
 * Same result as ccm_calculate_weights (bit-exact with the reference's serial
 * calculate_weights), but with DEVICE pointers: d_msa (nrow x ncol states)
 * in, d_w (nrow floats) out, enqueued on `stream` (a cudaStream_t, NULL for
 * the legacy default stream) on the current device, without a host
 * synchronisation.  It calls no cudaMalloc, cudaFree or other allocating
 * routine: its only scratch, one int count per sequence, is a fixed array
 * compiled into the library (1 MiB, nrow <= 262144; larger nrow is rejected
 * with CCM_ERR_INVALID).  Every GPU that loads the library keeps that array
 * until the process exits.  Every call looks up the array's device address in
 * the calling thread's current context (cudaGetSymbolAddress, which allocates
 * nothing once the library's module is loaded there: the first call in a
 * context loads it, so make that call before any stream capture) and enqueues a
 * memset and two kernels.  All calls share the array and it keeps the last
 * call's counts (each call clears what it uses first): calls that overlap on
 * the GPU race on it and must be serialised by the caller (one stream, or
 * events between streams). */
CCM_API int ccm_calculate_weights_noalloc(const unsigned char *d_msa, int ncol, int nrow,
                                          float threshold, float *d_w, void *stream);

/* Description of the last error on this host thread. */
CCM_API const char *ccm_last_error(void);

/* Path used by init_cuda/init_b200 (CCM_PATH_*); default CCM_PATH_TC_I8SP. */
CCM_API void ccm_set_default_path(int path);

/* ---------------------------------------------------------------- optimizer */
/* Device-side nonlinear conjugate gradient over a context's evaluation; the
 * replacement of libconjugrad's conjugrad_gpu (src/ccmpred.c:632-648, absent
 * from the reference checkout; the libconjugrad names themselves are in
 * conjugrad.h).  Parameters as set at src/ccmpred.c:526-534 (the defaults are
 * the reference's float values); FP64 line-search tests and dot products,
 * float vectors on the device.  The line search, the direction update and the
 * stopping test run on the device: without a progress callback the whole solve
 * is one CUDA-graph launch (conditional WHILE/IF nodes), with one the host
 * waits once per iteration to call it. */
typedef struct ccm_cg_params {
	int max_iterations;   /* -n, default 250 (src/ccmpred.c:222) */
	int k;                /* -k, default 5: convergence window */
	int max_linesearch;   /* 5 */
	int pad;
	double epsilon;       /* -e, default 0.01: stop when (f_{i-k} - f_i)/|f_i| < epsilon */
	double alpha_mul;     /* 0.5: backtracking factor */
	double ftol;          /* 1e-4: sufficient-decrease constant */
	double wolfe;         /* 0.2: curvature constant (g_t.s >= wolfe g.s); <= 0 turns the
	                         curvature test off */
	double min_gnorm;     /* stop when ||g|| <= min_gnorm; 0 (default) = off */
} ccm_cg_params;

typedef struct ccm_cg_result {
	int status;       /* CCM_CG_* */
	int iterations;
	int evaluations;
	int pad;
	double fx;        /* f at the returned x */
	double gnorm;     /* ||g|| at the returned x */
} ccm_cg_result;

#define CCM_CG_SUCCESS 0
#define CCM_CG_ALREADY_MINIMIZED 1
#define CCM_CG_STOPPED 2
#define CCM_CG_ERR_MAXITER (-1023)
#define CCM_CG_ERR_LINESEARCH (-1022)
#define CCM_CG_ERR_NONFINITE (-1021)

/* Progress callback with the signature of the reference's progress()
 * (src/ccmpred.c:50-61); x and g are device pointers.  Non-zero stops the run. */
typedef int (*ccm_progress_t)(void *instance, const float *x, const float *g, const float fx,
                              const float xnorm, const float gnorm, const float step, int n, int k,
                              int ls);

CCM_API void ccm_cg_params_default(ccm_cg_params *p);
/* Minimise f starting from the DEVICE vector d_x (nvar_padded floats, updated
 * in place).  Returns CCM_OK with the optimizer outcome in *result, or a
 * CCM_ERR_* status when the device or an argument fails. */
CCM_API int ccm_conjugrad_gpu(ccm_context *ctx, float *d_x, long long n,
                              const ccm_cg_params *params, ccm_progress_t progress, void *instance,
                              ccm_cg_result *result);

/* Same with a HOST x (copied to the device, optimised, copied back). */
CCM_API int ccm_conjugrad_host(ccm_context *ctx, float *x, long long n,
                               const ccm_cg_params *params, ccm_progress_t progress,
                               void *instance, ccm_cg_result *result);

/* ---------------------------------------------------------------- batched solves */
/* Many alignments of different sizes solved to convergence concurrently on
 * one GPU (no reference counterpart: the reference runs one alignment per
 * process).  Alignments are taken largest-first.  Default (waves = 0): host
 * worker threads each take the next alignment, create its context on their own
 * stream and run its whole device-side solve (initial evaluation, CG iterations
 * in conditional graph nodes, contact scores) as one graph launch.  waves = 1:
 * alignments are admitted in waves under a device-memory budget and the solves
 * of a wave go into ONE graph as independent branches, launched once per wave
 * (a wave lasts as long as its slowest solve, so on B200 it measured a few per
 * cent slower than the threads on the 256-alignment batch). */
typedef struct ccm_msa_desc {
	const unsigned char *msa;   /* nrow x ncol states 0..20, host memory */
	int ncol;
	int nrow;
	int path;                   /* CCM_PATH_* for this alignment, or -1: the batch's
	                               path (ccmpred_b200.autotune picks one per size) */
	int pad;
} ccm_msa_desc;

typedef struct ccm_batch_params {
	float reweighting_threshold; /* 0.8 */
	float lambda_single;         /* 0.01 */
	float lambda_pair_factor;    /* 0.2: lambda_pair = factor * (L - 1) */
	int path;                    /* CCM_PATH_* */
	int workers;                 /* concurrent solves (threads / streams), default 8 */
	int device;
	int use_apc;                 /* contact maps with APC (1) or raw Frobenius norms (0) */
	int sms_per_worker;          /* max_sms of every worker's contexts; 0 = no limit
	                                (default; on B200 the 256-alignment batch ran
	                                fastest with no limit) */
	int waves;                   /* 0 (default): host worker threads; 1: one graph
	                                launch per wave of alignments */
	int wave_max;                /* most alignments in one wave (default 64) */
	size_t wave_bytes;           /* device memory of one wave (estimated from the
	                                alignments' sizes); 0 = 60 % of the free memory */
	ccm_cg_params cg;            /* optimizer settings for every alignment */
} ccm_batch_params;

typedef struct ccm_batch_result {
	int status;        /* CCM_CG_* of the solve, or a CCM_ERR_* code */
	int iterations;
	int evaluations;
	int pad;
	double fx;
	double seconds;    /* wall time of this alignment's solve (of its wave, with waves) */
} ccm_batch_result;

CCM_API void ccm_batch_params_default(ccm_batch_params *p);
/* results[i] for msas[i]; contact_maps may be NULL or hold n pointers (each
 * NULL or ncol*ncol floats) that receive the APC-corrected maps. */
CCM_API int ccm_solve_batch(int n, const ccm_msa_desc *msas, const ccm_batch_params *params,
                            ccm_batch_result *results, float **contact_maps);

/* Devices (src/ccmpred.c:400-478 device selection and memory report). */
CCM_API int ccm_device_count(void);
CCM_API int ccm_device_info(int device, char *name, int name_len, size_t *mem_free,
                            size_t *mem_total);

/* ---------------------------------------------------------------- host-side drop-in pieces */
/* Bit-identical restatements (float, same operation order) of the reference's
 * host code around the evaluation. */

/* src/ccmpred.c:90-131 init_bias: x = 0 except V(j,a) = log f_a - log f_gap with
 * pseudocount 1; x holds nvar_padded floats. */
CCM_API void ccm_init_bias(const unsigned char *msa, int ncol, int nrow, float *x);
/* src/util.c:16-64 sum_submatrices (L x L map); returns the coupling norm the
 * reference prints as "xnorm". */
CCM_API double ccm_sum_submatrices(const float *x, float *out, int ncol);
/* The same L x L map (without the xnorm) from a DEVICE x into a DEVICE out,
 * enqueued on `stream` (a cudaStream_t, NULL for the legacy default stream);
 * equal to ccm_sum_submatrices bit for bit.  For callers that keep x on the
 * GPU after ccm_conjugrad_gpu: only L*L floats need to come back to the host. */
CCM_API int ccm_sum_submatrices_gpu(const float *d_x, float *d_out, int ncol, void *stream);
/* src/util.c:66-108 apc, in place. */
CCM_API void ccm_apc(float *mat, int ncol);
/* src/util.c:110-140 normalize, in place; CCM_ERR_INVALID on a constant map. */
CCM_API int ccm_normalize(float *mat, int ncol);
/* src/io.c:20-28 write_matrix ("%.20e\t"). */
CCM_API int ccm_write_matrix(const char *path, const float *mat, int ncol, int nrow);
/* src/io.c:31-60 write_raw. */
CCM_API int ccm_write_raw(const char *path, const float *x, int ncol);
/* src/io.c:62-103 read_raw (fills both symmetric halves; x not cleared). */
CCM_API int ccm_read_raw(const char *path, float *x, int ncol);
/* src/sequence.c:48-80 read_msa (PSICOV); NULL with *ncol = -1 for a3m/FASTA
 * input.  Free the result with ccm_free. */
CCM_API unsigned char *ccm_read_msa(const char *path, int *ncol, int *nrow);
CCM_API void ccm_free(void *p);

/* ---------------------------------------------------------------- reference triple */
/* Drop-in for include/evaluate_cuda.h:8-17: device x and g, nvar = nvar_padded,
 * returns f (src/evaluate_cuda.c:23-74).  init_cuda computes the weights on the
 * GPU (threshold < 1) or uses uniform weights (src/evaluate_cuda.c:105-125) and,
 * unlike the reference, also fills ud->weights on the host. */
CCM_API float evaluate_cuda(void *instance, const float *x, float *g, const int nvar);
CCM_API int init_cuda(void *instance);
CCM_API int destroy_cuda(void *instance);

/* Host-pointer backend with the shape of include/evaluate_cpu.h:21-30. */
CCM_API float evaluate_b200(void *instance, const float *x, float *g, const int nvar);
CCM_API int init_b200(void *instance);
CCM_API int destroy_b200(void *instance);

#ifdef __cplusplus
}
#endif

#endif /* CCMPRED_B200_H */
