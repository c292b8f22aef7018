/*
 * smooth — drop-in for petenez/pfc's smoothing tool (demos/honey/smooth.c)
 * with the transforms on the GPU through include/pfc_b200.h:
 *
 *   smooth <input data file> <output data file> <kernel spread sigma>
 *
 * The field is convolved with the Gaussian whose Fourier transform is
 * exp(-k^2 / (2 sigma^2)) (smooth.c:81-121) and written as the reference does
 * (smooth.c:126-143): "%d %d %lf %lf" header, then "%.12e" per value.
 * The reference divides by the sum of the real-space kernel, which is exactly 1
 * (only k = 0 survives the sum and G(0) = 1); that division is omitted.
 * Environment: PFC_B200_PRECISION fp64 (default) or fp32, PFC_B200_DEVICE.
 * Differences: a data file with fewer values than its header announces is an
 * error (exit 1) instead of being read as whatever fscanf left in memory.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "nio.h"
#include "pfc_b200.h"

int main(int argc, char** argv) {
	if (argc == 1) {
		printf("smooth convolves PFC data with a Gaussian on a B200 GPU. It takes the names of the input and "
		       "output data files and the spread of the smoothing kernel in reciprocal units:\n\n"
		       "smooth [input data file] [output data file] [smoothing kernel spread]\n");
		return 0;
	}
	if (argc != 4) {
		fprintf(stderr, "smooth takes three arguments: input file, output file, kernel spread\n");
		return 1;
	}
	size_t len = 0;
	char* buf = nio_slurp(argv[1], &len);
	if (!buf) {
		printf("Input file not found!\n");
		return 1;
	}
	char* q = buf;
	char* end;
	const long W = strtol(q, &end, 10);
	q = end;
	const long H = strtol(q, &end, 10);
	q = end;
	const double dx = strtod(q, &end);
	q = end;
	const double dy = strtod(q, &end);
	if (end == q || W < 1 || H < 1) {
		fprintf(stderr, "%s: bad header\n", argv[1]);
		return 1;
	}
	q = end;
	const size_t n = (size_t)W * (size_t)H;
	double* f = (double*)malloc(sizeof(double) * n);
	if (nio_parse_values(q, buf + len, f, n)) {
		fprintf(stderr, "%s: fewer than %ld values\n", argv[1], W * H);
		return 1;
	}
	free(buf);

	const char* de = getenv("PFC_B200_DEVICE");
	if (de && pfcg_set_device(atoi(de))) {
		fprintf(stderr, "%s\n", pfcg_last_error(NULL));
		return 1;
	}
	const char* pe0 = getenv("PFC_B200_PRECISION");
	if (!pfcg_size_supported_for((int)W, (int)H, 1, (pe0 && strcmp(pe0, "fp32") == 0) ? PFCG_FP32 : PFCG_FP64)) {
		fprintf(stderr, "grid size not supported by pfc_b200 (see pfcg_size_supported_for).\n");
		return 42;
	}
	/* one field; only sigma matters for the smoothing */
	pfcg_params p;
	memset(&p, 0, sizeof(p));
	p.U = 1;
	p.W[0] = 1;
	p.c = 1.0;
	p.dt = 1.0;
	p.sigma = atof(argv[3]);
	p.alpha[0][0] = -0.25;
	p.beta[0][0] = 1.0;
	p.nu2[0][0] = 1.0;
	p.omega[0][0] = 1.0;
	const char* pe = getenv("PFC_B200_PRECISION");
	const pfcg_prec prec = (pe && strcmp(pe, "fp32") == 0) ? PFCG_FP32 : PFCG_FP64;
	pfcg_handle* h = NULL;
	double* out = (double*)malloc(sizeof(double) * n);
	int rc = pfcg_create(&p, (int)W, (int)H, dx, dy, prec, &h);
	if (!rc) rc = pfcg_upload(h, f);
	if (!rc) rc = pfcg_smooth(h, 0, out);
	if (rc) {
		fprintf(stderr, "%s\n", pfcg_last_error(h));
		return 43;
	}
	pfcg_destroy(h);
	FILE* o = fopen(argv[2], "w");
	if (!o) {
		fprintf(stderr, "cannot write %s\n", argv[2]);
		return 1;
	}
	fprintf(o, "%ld %ld %lf %lf\n", W, H, dx, dy);
	nio_write_values(o, 12, out, n);
	fclose(o);
	free(f);
	free(out);
	return 0;
}
