/*
 * fields — drop-in for petenez/pfc's orientation / deformation tool
 * (src/fields.c) with the transforms on the GPU through pfcg_fields:
 *
 *   fields density.n orientation.phi fold sk sb
 *   fields density.n orientation.phi deformation.chi fold sk sb power
 *
 * Same arguments, messages and output formats as the reference (fields.c:
 * 365-419): the orientation file holds "%e %e" (real, imaginary) per point,
 * the deformation file "%e" per point, both after a "%d %d %lf %lf" header.
 * Differences: fold must be even (the reference's method works only for even
 * folds and says so); a data file with fewer values than its header announces
 * is "Error: Invalid data." instead of being read as whatever fscanf left.
 * Environment: PFC_B200_DEVICE.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "nio.h"
#include "pfc_b200.h"

static void help(void) {
	printf("fields computes the orientation field, and optionally the deformation field, of a density field "
	       "describing a periodic system such as a polycrystal, on a B200 GPU (method: Hirvonen et al., Physical "
	       "Review Materials 2, 103603 (2018)).\n\n"
	       "fields density.n orientation.phi [order of rotational symmetry] [spread of complex-valued kernel] "
	       "[spread of Gaussian smoothing kernel]\n\n"
	       "fields density.n orientation.phi deformation.chi [order of rotational symmetry] [spread of complex-valued "
	       "kernel] [spread of Gaussian smoothing kernel] [tunable exponent for deformation field]\n\n"
	       "The order of rotational symmetry must be even (2 stripes, 4 square, 6 hexagonal or honeycomb); the input "
	       "field should have a characteristic wave number close to 1.\n");
}

static int write_header(FILE* f, int W, int H, double dx, double dy) { return fprintf(f, "%d %d %lf %lf\n", W, H, dx, dy); }

int main(int argc, char** argv) {
	if (argc == 1) {
		help();
		return 0;
	}
	if (argc != 6 && argc != 8) {
		printf("Error: Invalid syntax.\n");
		return 1;
	}
	const int deform = argc == 8;
	const char* name_n = argv[1];
	const char* name_phi = argv[2];
	const char* name_chi = deform ? argv[3] : NULL;
	const int base = deform ? 4 : 3;
	const int fold = atoi(argv[base]);
	const double sk = atof(argv[base + 1]), sb = atof(argv[base + 2]);
	const double power = deform ? atof(argv[7]) : 0.0;

	size_t len = 0;
	char* buf = nio_slurp(name_n, &len);
	if (!buf) {
		printf("Error: Input file not found.\n");
		return 1;
	}
	char* q = buf;
	char* end;
	const long W = strtol(q, &end, 10);
	const int ok1 = end != q;
	q = end;
	const long H = strtol(q, &end, 10);
	const int ok2 = end != q;
	q = end;
	const double dx = strtod(q, &end);
	const int ok3 = end != q;
	q = end;
	const double dy = strtod(q, &end);
	const int ok4 = end != q;
	q = end;
	if (!(ok1 && ok2 && ok3 && ok4) || W < 1 || H < 1) {
		printf("Error: Invalid data.\n");
		return 1;
	}
	const size_t n = (size_t)W * (size_t)H;
	double* p = (double*)malloc(sizeof(double) * n);
	if (nio_parse_values(q, buf + len, p, n)) {
		printf("Error: Invalid data.\n");
		return 1;
	}
	free(buf);
	const char* de = getenv("PFC_B200_DEVICE");
	if (de && pfcg_set_device(atoi(de))) {
		fprintf(stderr, "%s\n", pfcg_last_error(NULL));
		return 1;
	}
	if (!pfcg_size_supported_for((int)W, (int)H, 2, PFCG_FP64)) {
		fprintf(stderr, "grid size not supported by pfc_b200 (see pfcg_size_supported_for).\n");
		return 42;
	}
	double* psi = (double*)malloc(sizeof(double) * 2 * n);
	double* chi = deform ? (double*)malloc(sizeof(double) * n) : NULL;
	const int rc = pfcg_fields(p, (int)W, (int)H, dx, dy, fold, sk, sb, power, psi, chi);
	if (rc) {
		fprintf(stderr, "%s\n", pfcg_last_error(NULL));
		return rc == PFCG_EARG ? 1 : 43;
	}
	FILE* f = fopen(name_phi, "w");
	if (!f) {
		fprintf(stderr, "cannot write %s\n", name_phi);
		return 1;
	}
	write_header(f, (int)W, (int)H, dx, dy);
	nio_write_pairs(f, 6, psi, psi + n, n);
	fclose(f);
	if (deform) {
		f = fopen(name_chi, "w");
		if (!f) {
			fprintf(stderr, "cannot write %s\n", name_chi);
			return 1;
		}
		write_header(f, (int)W, (int)H, dx, dy);
		nio_write_values(f, 6, chi, n);
		fclose(f);
	}
	free(p);
	free(psi);
	free(chi);
	return 0;
}
