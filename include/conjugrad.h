/*
 * conjugrad.h -- the optimizer interface of libccmpred_b200.so under the names
 * the reference's driver calls (src/ccmpred.c:526-534, 619-647): the entry
 * points of libconjugrad, the nonlinear conjugate-gradient library that the
 * reference takes as a git submodule (lib/libconjugrad, .gitmodules:1-3).  That
 * library is absent from the reference checkout; everything below is what its
 * callers in the reference use, so that src/ccmpred.c compiles unchanged
 * against this header and links against libccmpred_b200.so:
 *
 *   conjugrad_float_t        float (the reference's default CONJUGRAD_FLOAT=32,
 *                            CMakeLists.txt:57-59)
 *   F0 ... F2, FInf          float constants (src/ccmpred.c:222-227 and
 *                            src/evaluate_cpu.c:42,153,157).  FInf is NaN: the
 *                            reference marks "lambda_pair not given" with it and
 *                            tests isnan (src/ccmpred.c:226,500)
 *   fexp, flog, fdexp, fdlog expf / logf (src/ccmpred.c:124-126,
 *                            src/evaluate_cpu.c:81-91)
 *   conjugrad_evaluate_t     the evaluate callback (include/evaluate_cuda.h:8-13)
 *   conjugrad_progress_t     the progress callback (src/ccmpred.c:50-61)
 *   conjugrad_parameter_t    the fields set at src/ccmpred.c:526-534
 *   status codes             src/ccmpred.c:653-659
 *
 * The optimizer is this library's own (the rules of libconjugrad are not
 * available): Polak-Ribiere+ directions, a line search on sufficient decrease
 * (ftol) and the curvature condition (wolfe), FP64 dot products, the
 * reference's stopping rule over the last k iterations (epsilon).  See
 * ccmpred_b200/csrc/ccm_cg.cu.
 */
#ifndef CCMPRED_B200_CONJUGRAD_H
#define CCMPRED_B200_CONJUGRAD_H

#include <math.h>

typedef float conjugrad_float_t;

#define F0 0.0f
#define F001 0.01f
#define F02 0.2f
#define F05 0.5f
#define F08 0.8f
#define F1 1.0f
#define F2 2.0f
#define FInf NAN

#define fexp expf
#define flog logf
#define fdexp expf
#define fdlog logf

/* return values of conjugrad / conjugrad_gpu */
#define CONJUGRAD_SUCCESS 0
#define CONJUGRAD_ALREADY_MINIMIZED 1
#define CONJUGRADERR_UNKNOWN (-1024)
#define CONJUGRADERR_MAXIMUMITERATION (-1023)
#define CONJUGRADERR_MAXIMUMLINESEARCH (-1022)

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define CONJUGRAD_API __attribute__((visibility("default")))
#else
#define CONJUGRAD_API
#endif

/* f at x, gradient into g (overwritten); n = nvar_padded.  Host pointers for
 * conjugrad, device pointers for conjugrad_gpu. */
typedef conjugrad_float_t (*conjugrad_evaluate_t)(void *instance, const conjugrad_float_t *x,
                                                  conjugrad_float_t *g, const int n);

/* Called once per iteration; a non-zero return stops the optimizer. */
typedef int (*conjugrad_progress_t)(void *instance, const conjugrad_float_t *x,
                                    const conjugrad_float_t *g, const conjugrad_float_t fx,
                                    const conjugrad_float_t xnorm, const conjugrad_float_t gnorm,
                                    const conjugrad_float_t step, int n, int k, int ls);

typedef struct {
	int max_linesearch;          /* trials per line search (src/ccmpred.c:530: 5) */
	int max_iterations;          /* -n */
	int k;                       /* -k: window of the stopping rule */
	conjugrad_float_t epsilon;   /* -e: stop when (f_{i-k} - f_i) / |f_i| < epsilon */
	conjugrad_float_t ftol;      /* sufficient-decrease constant (1e-4) */
	conjugrad_float_t wolfe;     /* curvature constant (0.2) */
	conjugrad_float_t alpha_mul; /* backtracking factor (0.5) */
	conjugrad_float_t min_gnorm; /* stop when ||g|| <= min_gnorm (0: off) */
} conjugrad_parameter_t;

/* A parameter block with this library's defaults, from malloc: the caller
 * releases it with free() (src/ccmpred.c:765). */
CONJUGRAD_API conjugrad_parameter_t *conjugrad_init(void);

/* Minimise from the HOST vector x (n floats, updated in place); *fx receives f
 * at the returned x.  The callback gets host pointers.  Vector arithmetic runs
 * on the host in FP64 accumulation (the callback decides where f and g are
 * computed: evaluate_b200 runs them on the GPU, the reference's evaluate_cpu on
 * the CPU). */
CONJUGRAD_API int conjugrad(int n, conjugrad_float_t *x, conjugrad_float_t *fx,
                            conjugrad_evaluate_t proc_evaluate,
                            conjugrad_progress_t proc_progress, void *instance,
                            conjugrad_parameter_t *param);

/* Minimise from the DEVICE vector d_x (n floats on the current device, updated
 * in place).  With this library's evaluate_cuda as the callback and an instance
 * set up by its init_cuda, the whole solve runs as the fused device CG of
 * ccm_conjugrad_gpu on that context; any other callback is called with device
 * pointers once per line-search trial (the vector operations, dot products and
 * line-search decisions stay on the device; the trial point is complete when
 * the callback is called, and g must be complete when it returns, as the
 * reference's evaluate_cuda guarantees by synchronising). */
CONJUGRAD_API int conjugrad_gpu(int n, conjugrad_float_t *d_x, conjugrad_float_t *fx,
                                conjugrad_evaluate_t proc_evaluate,
                                conjugrad_progress_t proc_progress, void *instance,
                                conjugrad_parameter_t *param);

/* Host vectors of n floats (64-byte aligned) and their release. */
CONJUGRAD_API conjugrad_float_t *conjugrad_malloc(int n);
CONJUGRAD_API void conjugrad_free(conjugrad_float_t *x);

#ifdef __cplusplus
}
#endif

#endif /* CCMPRED_B200_CONJUGRAD_H */
