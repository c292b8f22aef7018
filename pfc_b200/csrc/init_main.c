/*
 * pfc-init — the reference's initial-state builder (src/PFCInit.java, run as
 * `java -jar pfc-init.jar <input file>`) for the steps that build the states
 * of the relaxation workloads, with the Voronoi step on the GPU through
 * include/pfc_b200.h:
 *
 *   pfc-init <input file>
 *
 * The input is read as PFCInit.java:270-290 reads it: whitespace-separated
 * tokens, a token starting with '#' ends its line. Steps (labels):
 *   D Nx Ny dx dy         dimensions and discretisation (:304-315)
 *   S seed                java.util.Random seed (:318-322)
 *   L file type i0 j0 dNx dNy i1 j1   load part of a saved field (:325-386)
 *   V N, then N grains of x y type sym a nave amp namp tx1 ty1 theta xr yr tx2 ty2
 *                         Voronoi grains (:389-462), on the GPU (pfcg_init_voronoi)
 *   T nave famp           transform (:649-667)
 *   O file prec           output (:670-686), Java's "%.{prec}e" (pfcg_write_n_pfcinit)
 * Messages and exit codes are the reference's. The circular (C) and polygon (P)
 * grains are not built here; an input using them stops with exit code 1.
 * Without S, the reference seeds from the clock; so does this tool.
 */
#include <ctype.h>
#include <errno.h>
#include <limits.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "nio.h"
#include "pfc_b200.h"

static char** tok;
static int ntok;

static void die(void) { exit(1); }

/* Integer.parseInt: optional sign, decimal digits, int range (PFCInit.java:12-21) */
static int s2i(const char* s) {
	const char* c = s;
	if (*c == '+' || *c == '-') c++;
	int ok = *c != '\0';
	for (const char* d = c; *d; d++)
		if (!isdigit((unsigned char)*d)) ok = 0;
	errno = 0;
	const long v = ok ? strtol(s, NULL, 10) : 0;
	if (!ok || errno || v < INT_MIN || v > INT_MAX) {
		printf("Error: Invalid input file. Integer expected instead of \"%s\".\n", s);
		die();
	}
	return (int)v;
}

/* Double.parseDouble (PFCInit.java:23-32): the whole token, an optional
 * trailing type letter f/F/d/D allowed as Java does */
static double s2d(const char* s) {
	char* end;
	errno = 0;
	const double v = strtod(s, &end);
	if (end != s && (end[0] == 'f' || end[0] == 'F' || end[0] == 'd' || end[0] == 'D') && end[1] == '\0') end++;
	if (end == s || *end != '\0') {
		printf("Error: Invalid input file. Decimal number expected instead of \"%s\".\n", s);
		die();
	}
	return v;
}

/* the tokens of the input file, comments removed (PFCInit.java:270-290) */
static void read_tokens(const char* path) {
	size_t len = 0;
	char* buf = nio_slurp(path, &len);
	if (!buf) {
		printf("Error: Input file \"%s\" not found.\n", path);
		die();
	}
	int cap = 256;
	tok = (char**)malloc(sizeof(char*) * cap);
	char* p = buf;
	while (*p) {
		char* line = p;
		char* nl = strchr(p, '\n');
		if (nl) *nl = '\0';
		p = nl ? nl + 1 : p + strlen(p);
		char* save = NULL;
		for (char* w = strtok_r(line, " \t\r\f\v", &save); w; w = strtok_r(NULL, " \t\r\f\v", &save)) {
			if (w[0] == '#') break;
			if (ntok == cap) tok = (char**)realloc(tok, sizeof(char*) * (cap *= 2));
			tok[ntok++] = w;
		}
	}
}

static const char* next(int* k) {
	if (*k >= ntok) {
		printf("Error: Invalid input file. Unexpected end of input.\n");
		die();
	}
	return tok[(*k)++];
}

static int wrapi(int i, int n) {
	while (i < 0) i += n;
	while (i >= n) i -= n;
	return i;
}

int main(int argc, char** argv) {
	if (argc != 2) {
		printf("This is a tool for constructing 2D density fields for PFC calculations (a B200 build of the "
		       "reference's pfc-init for the steps D, S, L, V, T and O). The program expects one argument "
		       "specifying an input file.\n");
		return 0;
	}
	read_tokens(argv[1]);
	const char* de = getenv("PFC_B200_DEVICE");
	if (de && pfcg_set_device(atoi(de))) {
		fprintf(stderr, "%s\n", pfcg_last_error(NULL));
		return 1;
	}
	long long rng = pfcg_java_random_seed((long long)time(NULL) ^ (long long)clock());
	int Nx = -1, Ny = -1;
	double dx = 0.0, dy = 0.0;
	double* arr = NULL;
	int k = 0;
	while (k < ntok) {
		const char* lab = next(&k);
		if (!strcmp(lab, "D")) {
			Nx = s2i(next(&k));
			Ny = s2i(next(&k));
			dx = s2d(next(&k));
			dy = s2d(next(&k));
			free(arr);
			arr = (double*)calloc((size_t)(Nx > 0 ? Nx : 1) * (size_t)(Ny > 0 ? Ny : 1), sizeof(double));
		} else if (!strcmp(lab, "S")) {
			rng = pfcg_java_random_seed(s2i(next(&k)));
		} else if (!strcmp(lab, "L")) {
			const char* name = next(&k);
			const int type = s2i(next(&k));
			if (type == 2) {
				/* the reference skips the step's remaining tokens only by failing on them (:331-334) */
				printf("Warning: Phantom type used for the system from data file \"%s\".\n", name);
				continue;
			}
			if (type < 0 || type > 2)
				printf("Warning: Invalid type used for the system from data file \"%s\". Defaulting to overwrite.\n",
				       name);
			size_t len = 0;
			char* buf = nio_slurp(name, &len);
			if (!buf) {
				printf("Error: Data file \"%s\" not found.\n", name);
				die();
			}
			char* q = buf;
			char* end;
			const long Nx2 = strtol(q, &end, 10);
			q = end;
			const long Ny2 = strtol(q, &end, 10);
			q = end;
			const double dx2 = strtod(q, &end);
			q = end;
			const double dy2 = strtod(q, &end);
			q = end;
			if (dx2 != dx || dy2 != dy)
				printf("Warning: System from data file \"%s\" has incompatible discretization.\n", name);
			const int i0 = wrapi(s2i(next(&k)), (int)Nx2);
			const int j0 = wrapi(s2i(next(&k)), (int)Ny2);
			const int dNx = s2i(next(&k));
			const int dNy = s2i(next(&k));
			const int i1 = wrapi(s2i(next(&k)), Nx);
			const int j1 = wrapi(s2i(next(&k)), Ny);
			double* arr2 = (double*)malloc(sizeof(double) * (size_t)Nx2 * (size_t)Ny2);
			if (Nx2 < 1 || Ny2 < 1 || nio_parse_values(q, buf + len, arr2, (size_t)Nx2 * (size_t)Ny2)) {
				printf("Error: Invalid data file \"%s\".\n", name);
				die();
			}
			free(buf);
			/* the reference warns about an invalid type but still uses it (:335-337, :380) */
			const double t = (double)type;
			for (int j = 0; j < dNy; j++) {
				const int js = wrapi(j0 + j, (int)Ny2), jt = wrapi(j1 + j, Ny);
				for (int i = 0; i < dNx; i++) {
					const int is = wrapi(i0 + i, (int)Nx2), it = wrapi(i1 + i, Nx);
					arr[(size_t)jt * Nx + it] = t * arr[(size_t)jt * Nx + it] + arr2[(size_t)js * Nx2 + is];
				}
			}
			free(arr2);
		} else if (!strcmp(lab, "V")) {
			const int N = s2i(next(&k));
			pfcg_grain* g = (pfcg_grain*)calloc(N > 0 ? N : 1, sizeof(pfcg_grain));
			for (int n = 0; n < N; n++) {
				g[n].x = s2d(next(&k));
				g[n].y = s2d(next(&k));
				g[n].type = s2i(next(&k));
				g[n].sym = s2i(next(&k));
				g[n].a = s2d(next(&k));
				g[n].nave = s2d(next(&k));
				g[n].amp = s2d(next(&k));
				g[n].namp = s2d(next(&k));
				g[n].tx1 = s2d(next(&k));
				g[n].ty1 = s2d(next(&k));
				g[n].theta_deg = s2d(next(&k));
				g[n].xr = s2d(next(&k));
				g[n].yr = s2d(next(&k));
				g[n].tx2 = s2d(next(&k));
				g[n].ty2 = s2d(next(&k));
				if (g[n].type < 0 || g[n].type > 2) {
					printf("Warning: Invalid type used for a Voronoi grain. Defaulting to overwrite.\n");
					g[n].type = 0;
				}
				if (g[n].type != 2 && g[n].sym != 3 && g[n].sym != 4 && g[n].sym != 6) {
					printf("Error: Invalid lattice symmetry specified. Only triangular, square and hexagonal "
					       "symmetries are supported.\n");
					die();
				}
				if (g[n].type == 2) g[n].sym = 3; /* never evaluated */
			}
			if (N > 0 && arr && pfcg_init_voronoi(arr, Nx, Ny, dx, dy, N, g, &rng, NULL)) {
				fprintf(stderr, "%s\n", pfcg_init_last_error());
				return 1;
			}
			free(g);
		} else if (!strcmp(lab, "T")) {
			const double nave = s2d(next(&k));
			const double famp = s2d(next(&k));
			double nave0 = 0.0;
			const size_t n = (size_t)Nx * Ny;
			for (size_t i = 0; i < n; i++) nave0 += arr[i];
			nave0 *= 1.0 / Nx / Ny;
			for (size_t i = 0; i < n; i++) arr[i] = (arr[i] - nave0) * famp + nave;
		} else if (!strcmp(lab, "O")) {
			const char* name = next(&k);
			const int prec = s2i(next(&k));
			if (pfcg_write_n_pfcinit(name, Nx, Ny, dx, dy, arr, prec)) {
				printf("Error: cannot write \"%s\".\n", name);
				die();
			}
		} else if (!strcmp(lab, "C") || !strcmp(lab, "P")) {
			printf("Error: step \"%s\" is not supported by this build of pfc-init (D, S, L, V, T and O are).\n", lab);
			die();
		} else {
			printf("Error: Invalid input file. Label expected instead of \"%s\".\n", lab);
			die();
		}
	}
	free(arr);
	return 0;
}
