/*
 * oracle/conjugrad.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A stand-in for the header of libconjugrad, the optimizer library that the
 * reference includes as a git submodule (lib/libconjugrad, .gitmodules:1-3)
 * and that is absent from the reference checkout.  It exists so that the
 * reference's own C sources (src/evaluate_cpu.c, src/evaluate_cpu_omp.c,
 * src/reweighting.c, src/util.c, src/io.c, src/sequence.c, src/ccmpred.c and
 * the CUDA path src/evaluate_cuda.c + src/evaluate_cuda_kernels.cu) compile
 * unmodified, in place, into the reference oracle under oracle/_ref/.
 *
 * Everything here is inferred from how the reference uses the header:
 *   - conjugrad_float_t is float (CONJUGRAD_FLOAT=32, CMakeLists.txt:57-59)
 *   - F0 ... FInf constants (src/evaluate_cpu.c:42,153,157; src/ccmpred.c:222-227)
 *   - fexp/flog (src/evaluate_cpu.c:81-91) and fdexp/fdlog
 *     (src/evaluate_cuda_kernels.cu:83-97).  The meaning of these macros in
 *     libconjugrad is unknown; this shim maps them to expf/logf.
 *   - conjugrad_malloc(n) allocates n conjugrad_float_t (src/evaluate_cpu.c:174)
 *   - the evaluate/progress callback types and the parameter struct fields
 *     (src/ccmpred.c:50-61, 526-534) and the status codes (src/ccmpred.c:653-659).
 *
 * Nothing under ccmpred_b200/ includes this file.
 */
#ifndef CCM_ORACLE_CONJUGRAD_SHIM_H
#define CCM_ORACLE_CONJUGRAD_SHIM_H

#include <math.h>
#include <stdlib.h>

#ifndef CONJUGRAD_FLOAT
#define CONJUGRAD_FLOAT 32
#endif

#if CONJUGRAD_FLOAT == 32
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
#else
typedef double conjugrad_float_t;
#define F0 0.0
#define F001 0.01
#define F02 0.2
#define F05 0.5
#define F08 0.8
#define F1 1.0
#define F2 2.0
#define FInf NAN
#define fexp exp
#define flog log
#define fdexp exp
#define fdlog log
#endif

#define CONJUGRAD_SUCCESS 0
#define CONJUGRAD_ALREADY_MINIMIZED 1
#define CONJUGRADERR_UNKNOWN -1024
#define CONJUGRADERR_MAXIMUMITERATION -1023
#define CONJUGRADERR_MAXIMUMLINESEARCH -1022

#ifdef __cplusplus
extern "C" {
#endif

typedef conjugrad_float_t (*conjugrad_evaluate_t)(
	void *instance, const conjugrad_float_t *x, conjugrad_float_t *g, const int n);

typedef int (*conjugrad_progress_t)(
	void *instance, const conjugrad_float_t *x, const conjugrad_float_t *g,
	const conjugrad_float_t fx, const conjugrad_float_t xnorm,
	const conjugrad_float_t gnorm, const conjugrad_float_t step,
	int n, int k, int ls);

typedef struct {
	int max_linesearch;
	int max_iterations;
	int k;
	conjugrad_float_t epsilon;
	conjugrad_float_t ftol;
	conjugrad_float_t wolfe;
	conjugrad_float_t alpha_mul;
	conjugrad_float_t min_gnorm;
} conjugrad_parameter_t;

conjugrad_parameter_t *conjugrad_init(void);

int conjugrad(int n, conjugrad_float_t *x, conjugrad_float_t *fx,
	conjugrad_evaluate_t proc_evaluate, conjugrad_progress_t proc_progress,
	void *instance, conjugrad_parameter_t *param);

int conjugrad_gpu(int n, conjugrad_float_t *d_x, conjugrad_float_t *fx,
	conjugrad_evaluate_t proc_evaluate, conjugrad_progress_t proc_progress,
	void *instance, conjugrad_parameter_t *param);

conjugrad_float_t *conjugrad_malloc(int n);
void conjugrad_free(conjugrad_float_t *x);

#ifdef __cplusplus
}
#endif

#endif
