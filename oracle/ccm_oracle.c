/*
 * oracle/ccm_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A CPU restatement of the reference's pseudo-likelihood hot path, written
 * for checking the CUDA product path.  It is compiled to oracle/libccmoracle.so
 * and loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg; nothing under ccmpred_b200/ links or loads it.
 *
 * Pinned against the reference itself: tests/test_oracle.py compares every
 * function here with the reference's own compiled sources (oracle/_ref/,
 * built by oracle/Makefile) and with the committed golden vectors under
 * tests/golden/ that were generated from them.
 *
 * Layout (include/ccmpred.h:1-17 with PADDING on, CMakeLists.txt:37-40,71-73):
 *   x = [ V(j,a) at a*L + j, a < 20 | zero padding up to nsingle_padded |
 *         W(b,k,a,j) at ((b*L + k)*32 + a)*L + j ]
 *   nsingle = 20 L, nsingle_padded = nsingle + 32 - nsingle % 32
 *   (src/ccmpred.c:388-390), nvar_padded = nsingle_padded + 21*32*L*L.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define Q 21
#define QPAD 32

static inline long nsingle_padded_of(int L) {
	long ns = (long)L * (Q - 1);
	return ns + QPAD - (ns % QPAD);
}

long oracle_nvar_padded(int L) {
	return nsingle_padded_of(L) + (long)L * L * Q * QPAD;
}

long oracle_nsingle_padded(int L) { return nsingle_padded_of(L); }

/*
 * f and g of the L2-regularised pseudo-log-likelihood, in double precision.
 * Follows src/evaluate_cpu.c:16-166 step by step:
 *   logits PC(a,j) = V(j,a)[a<20] + sum_k W(X_nk,k,a,j)      (:56-75, k == j included)
 *   lse_j = log sum_a exp PC(a,j), P = exp(PC - lse)           (:78-93)
 *   f += w_n (lse_j - PC(X_nj, j))                              (:100)
 *   G1(j,a) += w_n (P(a,j) - [X_nj == a]), a < 20              (:102-110)
 *   G2(b,k,a,j) += w_n [X_nk == b] (P(a,j) - [X_nj == a])     (:112-126)
 *   g2 = G2 + G2^T over a,b < 21 (:131-140), self blocks zeroed (:142-149)
 *   reg: lambda1 sum V^2 + 0.5 lambda2 sum over ALL padded W slots,
 *        g += 2 lambda1 V, g += 2 lambda2 W (:151-163).
 * Loop order is rearranged for OpenMP (rows in parallel for the logits, the
 * coupling scatter parallel over k); every output is accumulated by one
 * thread in a fixed order, so results do not depend on the thread count.
 * P is kept for all rows: N * 21 * L doubles of scratch.
 */
double oracle_evaluate_f64(const unsigned char *msa, const double *w, int L, int N,
	double lambda_single, double lambda_pair, const double *x, double *g) {

	const long nsp = nsingle_padded_of(L);
	const long nvarp = oracle_nvar_padded(L);
	const long QL = (long)Q * L;
	const double *x1 = x;
	const double *x2 = x + nsp;
	double *g1 = g;
	double *g2l = g + nsp;

	double *P = (double *)malloc(sizeof(double) * (size_t)N * QL);
	double *fn = (double *)malloc(sizeof(double) * (size_t)N);
	double *G2 = (double *)calloc((size_t)QL * QL, sizeof(double));
	if (!P || !fn || !G2) { free(P); free(fn); free(G2); return NAN; }

	memset(g, 0, sizeof(double) * (size_t)nvarp);

	#pragma omp parallel for schedule(dynamic, 16)
	for (int n = 0; n < N; n++) {
		double *pc = P + (size_t)n * QL;          /* pc[a*L + j] */
		for (int a = 0; a < Q - 1; a++)
			for (int j = 0; j < L; j++) pc[a * L + j] = x1[a * L + j];
		for (int j = 0; j < L; j++) pc[(Q - 1) * L + j] = 0.0;
		for (int k = 0; k < L; k++) {
			int b = msa[(size_t)n * L + k];
			const double *row = x2 + ((long)b * L + k) * QPAD * L;
			for (long c = 0; c < QL; c++) pc[c] += row[c];
		}
		double fsum = 0.0;
		for (int j = 0; j < L; j++) {
			double m = -INFINITY;
			for (int a = 0; a < Q; a++) if (pc[a * L + j] > m) m = pc[a * L + j];
			double s = 0.0;
			for (int a = 0; a < Q; a++) s += exp(pc[a * L + j] - m);
			double lse = m + log(s);
			int xj = msa[(size_t)n * L + j];
			fsum += w[n] * (lse - pc[xj * L + j]);
			for (int a = 0; a < Q; a++) pc[a * L + j] = exp(pc[a * L + j] - lse);
		}
		fn[n] = fsum;
	}

	double fx = 0.0;
	for (int n = 0; n < N; n++) fx += fn[n];

	/* single-field gradient, parallel over columns */
	#pragma omp parallel for
	for (int j = 0; j < L; j++) {
		for (int n = 0; n < N; n++) {
			const double *p = P + (size_t)n * QL;
			int xj = msa[(size_t)n * L + j];
			if (xj < Q - 1) g1[xj * L + j] -= w[n];
			for (int a = 0; a < Q - 1; a++) g1[a * L + j] += w[n] * p[a * L + j];
		}
	}

	/* coupling gradient G2 (unpadded, rows b*L+k, cols a*L+j), parallel over k */
	#pragma omp parallel for schedule(dynamic, 1)
	for (int k = 0; k < L; k++) {
		for (int n = 0; n < N; n++) {
			const unsigned char *xn = msa + (size_t)n * L;
			int b = xn[k];
			double wn = w[n];
			double *gr = G2 + ((long)b * L + k) * QL;
			const double *p = P + (size_t)n * QL;
			for (long c = 0; c < QL; c++) gr[c] += wn * p[c];
			for (int j = 0; j < L; j++) gr[(long)xn[j] * L + j] -= wn;
		}
	}

	/* symmetrise into the padded layout, zero self blocks */
	#pragma omp parallel for
	for (int b = 0; b < Q; b++)
		for (int k = 0; k < L; k++)
			for (int a = 0; a < Q; a++)
				for (int j = 0; j < L; j++) {
					double v = (k == j) ? 0.0
						: G2[((long)b * L + k) * QL + (long)a * L + j]
						+ G2[((long)a * L + j) * QL + (long)b * L + k];
					g2l[(((long)b * L + k) * QPAD + a) * L + j] = v;
				}

	double reg = 0.0;
	for (long v = 0; v < (long)L * (Q - 1); v++) {
		reg += lambda_single * x[v] * x[v];
		g[v] += 2.0 * lambda_single * x[v];
	}
	for (long v = nsp; v < nvarp; v++) {
		reg += 0.5 * lambda_pair * x[v] * x[v];
		g[v] += 2.0 * lambda_pair * x[v];
	}
	fx += reg;

	free(P); free(fn); free(G2);
	return fx;
}

/*
 * Sequence weights, following src/reweighting.c:9-58 run serially (the
 * reference's OpenMP loop races on w[i]++, src/reweighting.c:37-40):
 *   idthres = (int)ceil(threshold * ncol) with the product taken in float
 *   (float * uint64 -> float, :10); count_i = #{j : ids(i,j) > idthres}
 *   over the i <= j triangle, so i == j is counted twice (:14-41);
 *   w_i = 1 / (count_i - 1) computed in double and stored as float (:43-45).
 * Identity counts are integers; the result is bit-exact.
 */
void oracle_calculate_weights(const unsigned char *msa, int L, int N, float threshold, float *w_out) {
	float thr_prod = threshold * (float)(uint64_t)L;
	int idthres = (int)ceil(thr_prod);
	int *cnt = (int *)calloc((size_t)N, sizeof(int));
	#pragma omp parallel for schedule(dynamic, 8)
	for (int i = 0; i < N; i++) {
		const unsigned char *a = msa + (size_t)i * L;
		int c = 0;
		for (int j = 0; j < N; j++) {
			const unsigned char *b = msa + (size_t)j * L;
			int ids = 0;
			for (int k = 0; k < L; k++) ids += (a[k] == b[k]);
			if (ids > idthres) c += (i == j) ? 2 : 1;
		}
		cnt[i] = c;
	}
	for (int i = 0; i < N; i++) {
		float cf = (float)cnt[i];
		w_out[i] = (float)(1. / (cf - 1));
	}
	free(cnt);
}

/*
 * FP64 host restatement of the device conjugate gradient of
 * ccmpred_b200/csrc/ccm_cg.cu with the rules of ccm_cg_rules.cuh (the
 * optimizer itself is this project's; the reference's libconjugrad is absent,
 * so this is the checker of the device loop, not of libconjugrad), written
 * here as a plain loop over FP64 vectors:
 *   s0 = -g0, alpha0 = 1/||g0||;
 *   a trial x_t = x + alpha s meets (A) f_t <= f + ftol alpha g.s and
 *   (C) g_t.s >= wolfe g.s (wolfe <= 0: C always holds);
 *   A and C, or A with fewer than two trials left: take the step;
 *   A without C and two trials left: remember alpha, try the secant step
 *   alpha g.s / (g.s - g_t.s) kept in [1.5, 16] alpha (alpha / alpha_mul when
 *   g_t.s <= g.s);
 *   not A after such an expansion: retreat to the remembered alpha (taken);
 *   not A otherwise: safeguarded quadratic backtracking in [0.1, alpha_mul] alpha;
 *   max_ls trials without a step: restart along -g once (fresh budget), then fail;
 *   Polak-Ribiere+ beta, steepest descent when s is not a descent direction;
 *   next alpha = 2 (f_old - f_new) / -(g.s_new) (1/||g|| if that is not positive);
 *   stop when i >= k and (f_{i-k} - f_i)/|f_i| < eps.
 * f_hist receives f after every iteration (f_hist[0] = f(x0)); returns the
 * status code (0 success, -1023 max iterations, -1022 line search failed).
 */
static double dot(const double *a, const double *b, long n) {
	double s = 0.0;
	for (long i = 0; i < n; i++) s += a[i] * b[i];
	return s;
}

int oracle_conjugrad_f64(const unsigned char *msa, const double *w, int L, int N,
	double lambda_single, double lambda_pair, double *x, int max_iter, int kwin,
	int max_ls, double alpha_mul, double ftol, double wolfe, double eps,
	double *f_hist, int *iterations, int *evaluations) {
	const long n = oracle_nvar_padded(L);
	double *g = (double *)malloc(sizeof(double) * n);
	double *gt = (double *)malloc(sizeof(double) * n);
	double *xt = (double *)malloc(sizeof(double) * n);
	double *s = (double *)malloc(sizeof(double) * n);
	double f = oracle_evaluate_f64(msa, w, L, N, lambda_single, lambda_pair, x, g);
	int evals = 1, status = -1023, it = 0, steepest = 1;
	f_hist[0] = f;
	double gg = dot(g, g, n);
	for (long i = 0; i < n; i++) s[i] = -g[i];
	double gs = -gg;
	double alpha = 1.0 / sqrt(gg);
	for (int k = 1; k <= max_iter; k++) {
		int ok = 0, ls = 0, retreat = 0;
		double ft = 0.0, good = 0.0;
		for (;;) {
			for (long i = 0; i < n; i++) xt[i] = x[i] + alpha * s[i];
			ft = oracle_evaluate_f64(msa, w, L, N, lambda_single, lambda_pair, xt, gt);
			evals++;
			ls++;
			const int suff = isfinite(ft) && ft <= f + ftol * alpha * gs;
			const double gts = dot(gt, s, n);
			const int curv = wolfe <= 0.0 || gts >= wolfe * gs;
			if (retreat) {
				ok = suff;
			} else if (suff && (curv || ls + 2 > max_ls)) {
				ok = 1;
			} else if (suff) {
				good = alpha;
				if (gts > gs) {
					const double r = gs / (gs - gts);
					alpha = alpha * (r < 1.5 ? 1.5 : (r > 16.0 ? 16.0 : r));
				} else {
					alpha = alpha / alpha_mul;
				}
			} else if (good > 0.0) {
				alpha = good;
				retreat = 1;
			} else {
				double den = 2.0 * (ft - f - gs * alpha);
				double aq = (isfinite(ft) && den > 0.0) ? -gs * alpha * alpha / den : alpha_mul * alpha;
				aq = fmin(aq, alpha_mul * alpha);
				alpha = fmax(aq, 0.1 * alpha);
			}
			if (ok) break;
			if (ls >= max_ls) {
				if (steepest) break;
				for (long i = 0; i < n; i++) s[i] = -g[i];
				gs = -gg;
				alpha = 1.0 / sqrt(gg);
				steepest = 1;
				ls = 0;
				good = 0.0;
				retreat = 0;
			}
		}
		if (!ok) { status = -1022; break; }
		double ggnew = dot(gt, gt, n), gtg = dot(gt, g, n), gts_old = dot(gt, s, n);
		double beta = (ggnew - gtg) / gg;
		if (!(beta > 0.0)) beta = 0.0;
		double gs_new = -ggnew + beta * gts_old;
		if (!(gs_new < 0.0)) {
			beta = 0.0;
			gs_new = -ggnew;
		}
		steepest = beta == 0.0;
		for (long i = 0; i < n; i++) { x[i] = xt[i]; s[i] = beta * s[i] - gt[i]; g[i] = gt[i]; }
		double anext = 2.0 * (f - ft) / -gs_new;
		if (!(anext > 0.0) || !isfinite(anext)) anext = 1.0 / sqrt(ggnew);
		alpha = anext;
		gs = gs_new;
		f = ft;
		gg = ggnew;
		f_hist[k] = f;
		it = k;
		if (k >= kwin && (f_hist[k - kwin] - f) / fabs(f) < eps) { status = 0; break; }
	}
	*iterations = it;
	*evaluations = evals;
	free(g); free(gt); free(xt); free(s);
	return status;
}
