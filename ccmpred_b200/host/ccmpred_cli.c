/*
 * ccmpred -- command-line driver over libccmpred_b200.so.
 *
 * Keeps the reference's command line and outputs (src/ccmpred.c:183-770):
 *   ccmpred [options] input.aln output.mat
 *   -n NUMITER  maximum CG iterations (default 250, src/ccmpred.c:222)
 *   -e EPSILON  convergence: relative decrease over the last K iterations (0.01)
 *   -k LASTK    K of the convergence test (5)
 *   -i INIFILE  warm start from a raw file (src/io.c:62-103)
 *   -r RAWFILE  write the raw parameters (src/io.c:31-60)
 *   -w IDTHRES  sequence reweighting identity threshold (0.8)
 *   -l LFACTOR  pairwise regularisation lambda_pair = LFACTOR * (L - 1) (0.2)
 *   -A          disable average product correction
 *   -R          re-normalise the output matrix to [0,1]
 *   -d DEVICE   CUDA device (default 0)
 *   -t THREADS  accepted for compatibility; this program evaluates on the GPU
 * The evaluation, the weights and the optimizer run on the GPU; the output
 * matrix is the APC-corrected Frobenius norm map written with "%.20e\t".
 */
#include <getopt.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ccmpred_b200.h"

static int progress(void *instance, const float *x, const float *g, const float fx,
                    const float xnorm, const float gnorm, const float step, int n, int k, int ls) {
	(void)instance; (void)x; (void)g; (void)n;
	printf("%-4d\t%-4d\t%-8g\t%-8g\t%-8.8g\t%-3.3g\n", k, ls, fx, xnorm, gnorm, step);
	fflush(stdout);
	return 0;
}

static void usage(const char *exe, int long_usage) {
	printf("Usage: %s [options] input.aln output.mat\n\n", exe);
	if (long_usage) {
		printf("Options:\n");
		printf("\t-d DEVICE \tCalculate on CUDA device number DEVICE [default: 0]\n");
		printf("\t-t THREADS\tAccepted for compatibility (evaluation runs on the GPU)\n");
		printf("\t-n NUMITER\tCompute a maximum of NUMITER operations [default: 250]\n");
		printf("\t-e EPSILON\tSet convergence criterion for minimum decrease in the last K iterations to EPSILON [default: 0.01]\n");
		printf("\t-k LASTK  \tSet K parameter for convergence criterion to LASTK [default: 5]\n");
		printf("\n");
		printf("\t-i INIFILE\tRead initial weights from INIFILE\n");
		printf("\t-r RAWFILE\tStore raw prediction matrix in RAWFILE\n");
		printf("\n");
		printf("\t-w IDTHRES\tSet sequence reweighting identity threshold to IDTHRES [default: 0.8]\n");
		printf("\t-l LFACTOR\tSet pairwise regularization coefficients to LFACTOR * (L-1) [default: 0.2]\n");
		printf("\t-A        \tDisable average product correction (APC)\n");
		printf("\t-R        \tRe-normalize output matrix to [0,1]\n");
		printf("\t-h        \tDisplay help\n\n");
	}
	exit(1);
}

static void die(const char *msg) {
	fprintf(stderr, "\nERROR: %s\n\n", msg);
	exit(1);
}

int main(int argc, char **argv) {
	char *rawfilename = NULL, *initfilename = NULL;
	int numiter = 250, use_apc = 1, use_normalization = 0, conjugrad_k = 5, device = 0;
	float lambda_single = 0.01f, lambda_pair_factor = 0.2f, reweighting_threshold = 0.8f;
	/* float, as the reference holds it (src/ccmpred.c:229,312,529): the stopping test
	 * then uses the same threshold as the reference's own driver does */
	float conjugrad_eps = 0.01f;
	int opt;
	while ((opt = getopt(argc, argv, "r:i:n:w:k:e:l:d:t:ARh?")) != -1) {
		switch (opt) {
			case 'r': rawfilename = optarg; break;
			case 'i': initfilename = optarg; break;
			case 'n': numiter = atoi(optarg); break;
			case 'w': reweighting_threshold = (float)atof(optarg); break;
			case 'l': lambda_pair_factor = (float)atof(optarg); break;
			case 'k': conjugrad_k = atoi(optarg); break;
			case 'e': conjugrad_eps = (float)atof(optarg); break;
			case 'd': device = atoi(optarg); break;
			case 't': break;
			case 'A': use_apc = 0; break;
			case 'R': use_normalization = 1; break;
			default: usage(argv[0], 1);
		}
	}
	if (argc - optind != 2) usage(argv[0], 0);
	const char *msafilename = argv[optind], *matfilename = argv[optind + 1];

	FILE *probe = fopen(msafilename, "r");
	if (!probe) {
		printf("Cannot open %s!\n\n", msafilename);
		return 2;
	}
	fclose(probe);
	int ncol = 0, nrow = 0;
	unsigned char *msa = ccm_read_msa(msafilename, &ncol, &nrow);
	if (!msa) {
		if (ncol == -1) {
			printf("ERROR: The alignment file seems to be in a3m or fasta format!\n"
			       "Please reformat the alignment to PSICOV format!\n\n");
			exit(100);
		}
		die("Cannot read the alignment");
	}

	printf(" _____ _____ _____               _ \n");
	printf("|     |     |     |___ ___ ___ _| |\n");
	printf("|   --|   --| | | | . |  _| -_| . |\n");
	printf("|_____|_____|_|_|_|  _|_| |___|___|\n");
	printf("                  |_|              \n\n");

	int ndev = ccm_device_count();
	if (ndev == 0) die("No CUDA devices available; this program evaluates on the GPU");
	if (device < 0 || device >= ndev) {
		printf("Error: %d is not a valid device number. Please choose a number between 0 and %d\n",
		       device, ndev - 1);
		exit(1);
	}
	char name[256];
	size_t mem_free = 0, mem_total = 0;
	if (ccm_device_info(device, name, sizeof(name), &mem_free, &mem_total) != CCM_OK)
		die(ccm_last_error());
	printf("Found %d CUDA devices, using device #%d: %s\n", ndev, device, name);
	printf("Total GPU RAM:  %17zu\nFree GPU RAM:   %17zu\n", mem_total, mem_free);

	const long long nvar_padded = ccm_nvar_padded(ncol);
	const int nvar = ncol * 20 + ncol * ncol * 21 * 21;
	float *x = (float *)malloc(sizeof(float) * (size_t)nvar_padded);
	if (!x) die("ERROR: Not enough memory to allocate variables!");
	float lambda_pair = lambda_pair_factor * (ncol - 1);

	if (initfilename == NULL) {
		ccm_init_bias(msa, ncol, nrow, x);
	} else {
		memset(x, 0, sizeof(float) * (size_t)nvar_padded);
		if (ccm_read_raw(initfilename, x, ncol) != CCM_OK) die("Cannot read the initial raw file");
	}

	float *weights = (float *)malloc(sizeof(float) * (size_t)nrow);
	if (reweighting_threshold < 1.0f) {
		if (ccm_calculate_weights(msa, ncol, nrow, reweighting_threshold, weights, device) != CCM_OK)
			die(ccm_last_error());
		float wsum = 0, wmin = weights[0], wmax = weights[0];
		for (int i = 0; i < nrow; i++) {
			wsum += weights[i];
			if (weights[i] > wmax) wmax = weights[i];
			if (weights[i] < wmin) wmin = weights[i];
		}
		printf("Reweighted %d sequences with threshold %.1f to Beff=%g weight mean=%g, min=%g, max=%g\n",
		       nrow, reweighting_threshold, wsum, wsum / nrow, wmin, wmax);
	} else {
		for (int i = 0; i < nrow; i++) weights[i] = 1.0f;
		printf("Using uniform weights on %d sequences\n", nrow);
	}

	ccm_options o;
	ccm_options_default(&o, ncol);
	o.lambda_single = lambda_single;
	o.lambda_pair = lambda_pair;
	o.device = device;
	const char *path = getenv("CCM_PATH");
	if (path && strcmp(path, "tc_bf16x2") == 0) o.path = CCM_PATH_TC_BF16X2;
	if (path && strcmp(path, "tc_bf16x3") == 0) o.path = CCM_PATH_TC_BF16X3;
	if (path && strcmp(path, "simt_f32") == 0) o.path = CCM_PATH_SIMT_F32;
	if (path && strcmp(path, "tc_i8x3") == 0) o.path = CCM_PATH_TC_I8X3;
	ccm_context *ctx = NULL;
	if (ccm_create(&ctx, msa, ncol, nrow, weights, &o) != CCM_OK) die(ccm_last_error());

	ccm_cg_params param;
	ccm_cg_params_default(&param);
	param.max_iterations = numiter;
	param.epsilon = conjugrad_eps;
	param.k = conjugrad_k;

	printf("\nWill optimize %d %ld-bit variables\n\n", nvar, (long)sizeof(float) * 8);
	printf("iter\teval\tf(x)    \t\xe2\x95\x91x\xe2\x95\x91     \t\xe2\x95\x91g\xe2\x95\x91     \tstep\n");

	ccm_cg_result res;
	if (ccm_conjugrad_host(ctx, x, nvar_padded, &param, progress, NULL, &res) != CCM_OK)
		die(ccm_last_error());
	const int ret = res.status;
	printf("\n");
	printf("%s with status code %d - ", (ret < 0 ? "Exit" : "Done"), ret);
	if (ret == CCM_CG_SUCCESS) printf("Success!\n");
	else if (ret == CCM_CG_ALREADY_MINIMIZED) printf("Already minimized!\n");
	else if (ret == CCM_CG_ERR_MAXITER) printf("Maximum number of iterations reached.\n");
	else printf("Unknown status code!\n");
	printf("\nFinal fx = %f\n\n", res.fx);

	FILE *out = fopen(matfilename, "w");
	if (out == NULL) {
		printf("Cannot open %s for writing!\n\n", matfilename);
		return 3;
	}
	fclose(out);
	if (rawfilename != NULL) {
		printf("Writing raw output to %s\n", rawfilename);
		if (ccm_write_raw(rawfilename, x, ncol) != CCM_OK) {
			printf("Cannot open %s for writing!\n\n", rawfilename);
			return 4;
		}
	}
	float *outmat = (float *)malloc(sizeof(float) * (size_t)ncol * ncol);
	const double xnorm = ccm_sum_submatrices(x, outmat, ncol);
	printf("xnorm = %g\n", xnorm);
	if (use_apc) ccm_apc(outmat, ncol);
	if (use_normalization && ccm_normalize(outmat, ncol) != CCM_OK)
		die("Cannot normalise a constant contact map");
	if (ccm_write_matrix(matfilename, outmat, ncol, ncol) != CCM_OK) {
		printf("Cannot open %s for writing!\n\n", matfilename);
		return 3;
	}
	ccm_destroy(ctx);
	free(outmat);
	free(x);
	free(weights);
	ccm_free(msa);
	printf("Output can be found in %s\n", matfilename);
	return 0;
}
