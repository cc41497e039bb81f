/*
 * oracle/ref_glue.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Linked into oracle/_ref/libccmref.so next to the reference's own C sources
 * (compiled in place from the reference checkout by oracle/Makefile).  It
 * provides
 *   - the few libconjugrad symbols that the reference sources link against
 *     (conjugrad_init, conjugrad_malloc/free; conjugrad/conjugrad_gpu are
 *     never called through this library and return CONJUGRADERR_UNKNOWN), and
 *   - path-based wrappers around the FILE*-based reference functions
 *     read_msa (src/sequence.c:48), write_matrix (src/io.c:20) and
 *     write_raw (src/io.c:31), so that tests can drive them through ctypes,
 *   - a constructor for the reference `userdata` struct (include/ccmpred.h:39-92).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * the resulting library, as the checker and the timed CPU baseline.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "conjugrad.h"
#include "ccmpred.h"
#include "io.h"
#include "sequence.h"

conjugrad_parameter_t *conjugrad_init(void) {
	conjugrad_parameter_t *p = (conjugrad_parameter_t *)calloc(1, sizeof(conjugrad_parameter_t));
	return p;
}

conjugrad_float_t *conjugrad_malloc(int n) {
	void *p = NULL;
	if (posix_memalign(&p, 64, sizeof(conjugrad_float_t) * (size_t)n) != 0) {
		return NULL;
	}
	return (conjugrad_float_t *)p;
}

void conjugrad_free(conjugrad_float_t *x) { free(x); }

int conjugrad(int n, conjugrad_float_t *x, conjugrad_float_t *fx,
	conjugrad_evaluate_t e, conjugrad_progress_t p, void *inst,
	conjugrad_parameter_t *param) {
	(void)n; (void)x; (void)fx; (void)e; (void)p; (void)inst; (void)param;
	return CONJUGRADERR_UNKNOWN;
}

int conjugrad_gpu(int n, conjugrad_float_t *x, conjugrad_float_t *fx,
	conjugrad_evaluate_t e, conjugrad_progress_t p, void *inst,
	conjugrad_parameter_t *param) {
	(void)n; (void)x; (void)fx; (void)e; (void)p; (void)inst; (void)param;
	return CONJUGRADERR_UNKNOWN;
}

/* userdata with the fields that src/ccmpred.c:504-515 fills in. */
userdata *ref_userdata_new(unsigned char *msa, int ncol, int nrow,
	float lambda_single, float lambda_pair, float threshold) {
	userdata *ud = (userdata *)calloc(1, sizeof(userdata));
	if (!ud) return NULL;
	ud->msa = msa;
	ud->ncol = ncol;
	ud->nrow = nrow;
	ud->nsingle = ncol * (N_ALPHA - 1);
	ud->nvar = ud->nsingle + ncol * ncol * N_ALPHA * N_ALPHA;
	ud->lambda_single = lambda_single;
	ud->lambda_pair = lambda_pair;
	ud->reweighting_threshold = threshold;
	ud->weights = conjugrad_malloc(nrow);
	return ud;
}

float *ref_userdata_weights(userdata *ud) { return ud->weights; }
void *ref_userdata_extra(userdata *ud) { return ud->extra; }

void ref_userdata_free(userdata *ud) {
	if (!ud) return;
	conjugrad_free(ud->weights);
	free(ud);
}

int ref_sizeof_userdata(void) { return (int)sizeof(userdata); }

unsigned char *ref_read_msa_path(const char *path, int *ncol, int *nrow) {
	FILE *f = fopen(path, "r");
	if (!f) return NULL;
	unsigned char *msa = read_msa(f, ncol, nrow);
	fclose(f);
	return msa;
}

void ref_free(void *p) { free(p); }

int ref_write_matrix_path(const char *path, float *mat, int ncol, int nrow) {
	FILE *f = fopen(path, "w");
	if (!f) return 1;
	write_matrix(f, mat, ncol, nrow);
	fclose(f);
	return 0;
}

int ref_write_raw_path(const char *path, float *x, int ncol) {
	FILE *f = fopen(path, "w");
	if (!f) return 1;
	write_raw(f, x, ncol);
	fclose(f);
	return 0;
}
