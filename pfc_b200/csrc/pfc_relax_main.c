/*
 * pfc-relax — drop-in command-line driver for the B200 relaxation library.
 *
 *   pfc-relax <input.in>
 *
 * Same command line, .in grammar, .n/.f/.out formats, printed lines and exit
 * codes as petenez/pfc's pfc-relax (demos/honey/pfc-relax.c, line numbers
 * below), with the hot path (step, evaluate, optimize, update_AB) running on
 * the GPU through include/pfc_b200.h. Host code only; one process, one GPU.
 *
 * Environment (no command-line flags, to keep the reference's syntax):
 *   PFC_B200_PRECISION  fp64 (default, the reference's precision) or fp32
 *   PFC_B200_DEVICE     CUDA device index (default 0)
 *   PFC_B200_CHECK_ONLY 1: parse the .in and .n files, print a summary, exit
 *                       (no GPU is touched); 2: also write each input field
 *                       back with the output writer to <field file>.check
 * The .n files are parsed and formatted by all OpenMP threads (OMP_NUM_THREADS);
 * the bytes are those of one strtod / fprintf("%.*e\n") per value in order.
 */
#include <ctype.h>
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "nio.h"
#include "pfc_b200.h"

#define LINE 8192

/* ------------------------------------------------------------- errors ---- */

/* The reference's fail() messages and codes (pfc-relax.c:242-411): scripts
 * see the same text on stdout and the same exit status. */
static const char* const MESSAGES[] = {
	"Error: Input file not found.",
	"Error: Invalid multicharacter label found.",
	"Error: Failed to read an input data file name.",
	"Error: Input data file not found.",
	"Error: Invalid input data file header.",
	"Error: Invalid mismatching dimensions of input data files.",
	"Error: Invalid number of output data files specified.",
	"Error: Failed to read an output data file name.",
	"Error: Failed to read the free energy density output data file name.",
	"Error: Invalid parameters for writing output.",
	"Error: Invalid write steps specified.",
	"Error: Failed to read the number of density fields.",
	"Error: Mismatching numbers of input data files and density fields specified.",
	"Error: Label for parameters lambda not found.",
	"Error: Invalid syntax for parameters lambda.",
	"Error:  Label for parameters alpha not found.",
	"Error: Invalid syntax for parameters alpha.",
	"Error:  Label for parameters beta not found.",
	"Error: Invalid syntax for parameters beta.",
	"Error:  Label for parameters gamma not found.",
	"Error: Invalid syntax for parameters gamma.",
	"Error: Label for parameters delta not found.",
	"Error: Invalid syntax for parameters delta.",
	"Error: Label for parameters epsilon not found.",
	"Error: Invalid syntax for parameters epsilon.",
	"Error: Label for parameters sigma not found.",
	"Error: Invalid syntax for parameters sigma.",
	"Error: Label for parameters 1/nu not found.",
	"Error: Invalid syntax for parameters 1/nu.",
	"Error: Label for parameters omega not found.",
	"Error: Invalid syntax for parameters omega.",
	"Error: Label for parameters phi not found.",
	"Error: Invalid syntax for parameters phi.",
	"Error: Label for parameters 1/mu not found.",
	"Error: Invalid syntax for parameters 1/mu.",
	"Error: Invalid parameters for relaxation.",
	"Error: Invalid label found.",
	"Error: Input data file not found.",
	"Error: Invalid data in data file.",
	"Error: Not a number value detected.",
	"Error: An error occurred while reading the input file.",
	"Error: Invalid syntax.",
};

/* codes beyond the reference's: limits of pfc_b200 and device errors */
#define E_UNSUPPORTED 42
#define E_DEVICE 43

static void die(int code) {
	if (code >= 0 && code <= 41) printf("%s\n", MESSAGES[code]);
	fflush(stdout);
	exit(code);
}

static void die_msg(int code, const char* msg) {
	printf("Error: %s\n", msg);
	fflush(stdout);
	exit(code);
}

/* -------------------------------------------------------------- config ---- */

typedef struct {
	char input[LINE];
	int U;
	int Nx, Ny;
	char* innames[PFCG_MAX_U + 64];
	char* outnames[PFCG_MAX_U + 64];
	char* fname; /* free-energy density output, or NULL */
	int Tprint, Twrite, pprint, pwrite;
	int* twrite; /* write steps, nwrite of them */
	int nwrite;
	double c, dx, dy, dt;
	int tend, Topt, xopt, yopt;
	pfcg_params p;
	int have_params;
} Config;

static int count_words(const char* line) {
	int n = 0, off = 0;
	char w[LINE];
	while (sscanf(line, "%s%n", w, &off) == 1) {
		n++;
		line += off;
	}
	return n;
}

static void read_line(FILE* in, char* line) {
	if (fgets(line, LINE, in) == NULL) die(40);
}

/* skips tokens until `label` (pfc-relax.c:552-554 and the same loops for
 * every model label; tokens in between, comments included, are skipped) */
static void seek_label(FILE* in, const char* label, int code) {
	char tok[LINE];
	for (;;) {
		if (fscanf(in, " %s", tok) != 1) die(code);
		if (strcmp(tok, label) == 0) return;
	}
}

/* U rows of the upper triangle (v from u, or from u+1 when strict), pfc-relax.c:565-572 */
static void read_triangle(FILE* in, Config* s, double m[PFCG_MAX_U][PFCG_MAX_U], int strict, int code) {
	char line[LINE];
	const int U = s->U;
	for (int u = 0; u < U - strict; u++) {
		read_line(in, line);
		const char* q = line;
		int off = 0;
		for (int v = u + strict; v < U; v++) {
			if (sscanf(q, " %lf%n", &m[u][v], &off) != 1) die(code);
			q += off;
		}
	}
}

static void parse_I(FILE* in, Config* s) {
	char line[LINE], word[LINE];
	const char* q;
	int off = 0;
	/* input data files: their count defines U (pfc-relax.c:445-472) */
	read_line(in, line);
	const int prevU = s->U;
	s->U += count_words(line);
	if (s->U > PFCG_MAX_U) die_msg(E_UNSUPPORTED, "more than 4 density fields are not supported by pfc_b200.");
	q = line;
	s->Nx = s->Ny = -1;
	for (int u = 0; u < s->U; u++) {
		if (sscanf(q, "%s%n", word, &off) != 1) die(2);
		q += off;
		free(s->innames[u]);
		s->innames[u] = strdup(word);
		FILE* f = fopen(word, "r");
		if (!f) die(3);
		int nx, ny;
		double a, b;
		if (fscanf(f, "%d %d %lf %lf", &nx, &ny, &a, &b) != 4) die(4);
		if ((s->Nx > 0 && s->Nx != nx) || (s->Ny > 0 && s->Ny != ny)) die(5);
		s->Nx = nx;
		s->Ny = ny;
		fclose(f);
	}
	(void)prevU;
	/* output data files and the optional free-energy file (:475-499) */
	read_line(in, line);
	const int V = count_words(line);
	if (V < s->U || V > s->U + 1) die(6);
	q = line;
	for (int u = 0; u < s->U; u++) {
		if (sscanf(q, "%s%n", word, &off) != 1) die(7);
		q += off;
		free(s->outnames[u]);
		s->outnames[u] = strdup(word);
	}
	s->fname = NULL;
	if (V > s->U) {
		if (sscanf(q, "%s", word) != 1) die(8);
		s->fname = strdup(word);
	}
	/* write parameters: "Tprint Twrite pprint pwrite" or "Tprint [ t... ] pprint pwrite" (:502-537) */
	s->Twrite = -1;
	read_line(in, line);
	const int N = count_words(line);
	if (N == 4) {
		if (sscanf(line, " %d %d %d %d", &s->Tprint, &s->Twrite, &s->pprint, &s->pwrite) != 4) die(9);
	} else if (N >= 6) {
		const int M = N - 5;
		free(s->twrite);
		s->twrite = (int*)malloc(sizeof(int) * M);
		s->nwrite = M;
		q = line;
		if (sscanf(q, "%d%n", &s->Tprint, &off) != 1) die(9);
		q += off;
		if (sscanf(q, "%s%n", word, &off) != 1 || strcmp(word, "[") != 0) die(9);
		q += off;
		for (int k = 0; k < M; k++) {
			if (sscanf(q, "%d%n", &s->twrite[k], &off) != 1) die(9);
			q += off;
		}
		for (int k = 1; k < M; k++)
			if (s->twrite[k] <= s->twrite[k - 1]) die(10);
		if (sscanf(q, "%s%n", word, &off) != 1 || strcmp(word, "]") != 0) die(9);
		q += off;
		if (sscanf(q, "%d %d", &s->pprint, &s->pwrite) != 2) die(9);
	} else {
		die(9);
	}
}

static void parse_M(FILE* in, Config* s) {
	char line[LINE], word[LINE];
	int V = 0, off = 0;
	read_line(in, line);
	if (sscanf(line, "%d", &V) != 1) die(11);
	if (V != s->U) die(12);
	pfcg_params* p = &s->p;
	memset(p, 0, sizeof(*p));
	p->U = s->U;
	const int U = s->U;
	/* lambda (:551-558) */
	seek_label(in, "l", 13);
	for (int u = 0; u < U; u++) {
		read_line(in, line);
		if (sscanf(line, " %lf", &p->lambda[u]) != 1) die(14);
	}
	seek_label(in, "a", 15);
	read_triangle(in, s, p->alpha, 0, 16);
	seek_label(in, "b", 17);
	read_triangle(in, s, p->beta, 0, 18);
	seek_label(in, "g", 19);
	read_triangle(in, s, p->gamma, 0, 20);
	seek_label(in, "d", 21);
	for (int u = 0; u < U; u++) {
		read_line(in, line);
		if (sscanf(line, " %lf", &p->delta[u]) != 1) die(22);
	}
	seek_label(in, "e", 23);
	read_triangle(in, s, p->epsilon, 1, 24);
	seek_label(in, "s", 25);
	read_line(in, line);
	if (sscanf(line, " %lf", &p->sigma) != 1) die(26);
	/* 1/nu: the count of values per row defines W[u]; stored as nu^2 (:635-659) */
	seek_label(in, "n", 27);
	for (int u = 0; u < U; u++) {
		read_line(in, line);
		const int W = count_words(line);
		if (W > PFCG_MAX_W) die_msg(E_UNSUPPORTED, "more than 4 modes per density field are not supported by pfc_b200.");
		p->W[u] = W;
		const char* q = line;
		for (int w = 0; w < W; w++) {
			double x;
			if (sscanf(q, "%lf%n", &x, &off) != 1) die(28);
			p->nu2[u][w] = 1.0 / x / x;
			q += off;
		}
	}
	seek_label(in, "o", 29);
	for (int u = 0; u < U; u++) {
		read_line(in, line);
		const char* q = line;
		for (int w = 0; w < p->W[u]; w++) {
			if (sscanf(q, "%lf%n", &p->omega[u][w], &off) != 1) die(30);
			q += off;
		}
	}
	seek_label(in, "p", 31);
	for (int u = 0; u < U; u++) {
		read_line(in, line);
		const char* q = line;
		for (int w = 0; w < p->W[u]; w++) {
			if (sscanf(q, "%lf%n", &p->phi[u][w], &off) != 1) die(32);
			q += off;
		}
	}
	/* 1/mu: stored as mu^2, 0 where beta is 0 (:689-704) */
	seek_label(in, "m", 33);
	for (int u = 0; u < U - 1; u++) {
		read_line(in, line);
		const char* q = line;
		for (int v = u + 1; v < U; v++) {
			double x;
			if (sscanf(q, " %lf%n", &x, &off) != 1) die(34);
			p->mu2[u][v] = (p->beta[u][v] == 0.0) ? 0.0 : 1.0 / x / x;
			q += off;
		}
	}
	(void)word;
	s->have_params = 1;
}

static void parse_R(FILE* in, Config* s) {
	char line[LINE];
	read_line(in, line);
	if (sscanf(line, "%lf %d %lf %lf %lf %d %d %d", &s->c, &s->tend, &s->dx, &s->dy, &s->dt, &s->Topt, &s->xopt,
	           &s->yopt) != 8)
		die(35);
	/* write interval -> write steps 0, Twrite, 2 Twrite, ... (:712-718) */
	if (s->Twrite > 0) {
		const int n = s->tend / s->Twrite + 1;
		free(s->twrite);
		s->twrite = (int*)malloc(sizeof(int) * n);
		s->nwrite = n;
		for (int k = 0; k < n; k++) s->twrite[k] = s->Twrite * k;
	}
}

/* read_input, pfc-relax.c:414-726 */
static void read_input(Config* s) {
	FILE* in = fopen(s->input, "r");
	if (!in) die(0);
	char tok[LINE], line[LINE];
	while (fscanf(in, " %s", tok) > 0) {
		if (tok[0] == '#') {
			read_line(in, line); /* comment: rest of the line */
		} else if (strlen(tok) > 1) {
			die(1);
		} else if (tok[0] == 'I') {
			parse_I(in, s);
		} else if (tok[0] == 'M') {
			parse_M(in, s);
		} else if (tok[0] == 'R') {
			parse_R(in, s);
		} else {
			die(36);
		}
	}
	fclose(in);
}

/* ---------------------------------------------------------------- data ---- */


/* read_data, pfc-relax.c:729-764: header "Nx Ny dx dy", then Nx*Ny values
 * y-major, whitespace separated (the reference's fscanf(" %lf ")). */
static void read_data(const Config* s, double* fields) {
	const size_t npts = (size_t)s->Nx * s->Ny;
	for (int u = 0; u < s->U; u++) {
		size_t len = 0;
		char* buf = nio_slurp(s->innames[u], &len);
		if (!buf) die(37);
		char* q = buf;
		char* end;
		/* header: two ints, two doubles */
		for (int k = 0; k < 4; k++) {
			errno = 0;
			if (k < 2) {
				long v = strtol(q, &end, 10);
				(void)v;
			} else {
				double v = strtod(q, &end);
				(void)v;
			}
			if (end == q) die(4);
			q = end;
		}
		if (nio_parse_values(q, buf + len, fields + u * npts, npts)) die(38);
		free(buf);
	}
}

/* file name with the first '#' replaced by the step (pfc-relax.c:787-793) */
static void step_name(const char* pattern, int t, char* out, size_t n) {
	const char* x = strchr(pattern, '#');
	if (!x) snprintf(out, n, "%s", pattern);
	else snprintf(out, n, "%.*s%d%s", (int)(x - pattern), pattern, t, x + 1);
}

/* header "%d %d %.*lf %.*lf\n" then "%.*e\n" per value (pfc-relax.c:800-806) */
static void write_field(const char* path, int Nx, int Ny, int prec, double dx, double dy, const double* v) {
	FILE* f = fopen(path, "w");
	if (!f) {
		fprintf(stderr, "cannot write %s\n", path);
		return;
	}
	fprintf(f, "%d %d %.*lf %.*lf\n", Nx, Ny, prec, dx, prec, dy);
	nio_write_values(f, prec, v, (size_t)Nx * Ny);
	fclose(f);
}

/* print_output, pfc-relax.c:862-898 */
static void print_output(const Config* s, int t, time_t t0, double dx, double dy, double fave, const double* nave) {
	char line[LINE];
	int n = snprintf(line, sizeof(line), "%d %d %.*lf %.*lf %.*lf ", t, (int)(time(NULL) - t0), s->pprint, dx,
	                 s->pprint, dy, s->pprint, fave);
	for (int u = 0; u < s->U; u++) n += snprintf(line + n, sizeof(line) - n, "%.*lf ", s->pprint, nave[u]);
	printf("%s\n", line);
	fflush(stdout);
	char out[LINE];
	const size_t L = strlen(s->input);
	if (L >= 3 && strcmp(s->input + L - 3, ".in") == 0) snprintf(out, sizeof(out), "%.*s.out", (int)(L - 3 < sizeof(out) - 5 ? L - 3 : sizeof(out) - 5), s->input);
	else snprintf(out, sizeof(out), "%.*s.out", (int)(sizeof(out) - 5), s->input);
	FILE* f = fopen(out, t == 0 ? "w" : "a");
	if (f) {
		fprintf(f, "%s\n", line);
		fclose(f);
	}
}

/* ---------------------------------------------------------------- relax --- */

static void check(int rc, pfcg_handle* h) {
	if (rc == 0) return;
	if (rc == PFCG_NAN) die(39);
	char msg[LINE];
	snprintf(msg, sizeof(msg), "GPU relaxation failed (%d): %s", rc, pfcg_last_error(h));
	die_msg(E_DEVICE, msg);
}

int main(int argc, char** argv) {
	if (argc == 1) {
		printf("pfc-relax relaxes phase field crystal (PFC) systems of one or more density fields on a B200 GPU. "
		       "It takes one argument, an input file that names the input and output data files and gives the "
		       "model parameters (labels I, M and R) and the relaxation parameters, in the format of petenez/pfc's "
		       "pfc-relax. Dynamics are conserved or nonconserved; the system size can be optimised to remove "
		       "strain. Environment: PFC_B200_PRECISION=fp64|fp32, PFC_B200_DEVICE=<index>.\n");
		return 0;
	}
	if (argc != 2) die(41);

	Config s;
	memset(&s, 0, sizeof(s));
	const time_t t0 = time(NULL);
	snprintf(s.input, sizeof(s.input), "%s", argv[1]);
	read_input(&s);
	if (!s.have_params) die(11);

	const char* co = getenv("PFC_B200_CHECK_ONLY");
	const size_t npts = (size_t)s.Nx * s.Ny;
	double* fields = (double*)malloc(sizeof(double) * npts * s.U);
	read_data(&s, fields);
	if (co && (co[0] == '1' || co[0] == '2')) {
		printf("ok U=%d Nx=%d Ny=%d tend=%d Tprint=%d nwrite=%d c=%g dt=%g dx=%g dy=%g Topt=%d\n", s.U, s.Nx, s.Ny, s.tend,
		       s.Tprint, s.nwrite, s.c, s.dt, s.dx, s.dy, s.Topt);
		/* 2: also write every input field back with the output writer, to <input name>.check */
		if (co[0] == '2')
			for (int u = 0; u < s.U; u++) {
				char name[LINE + 8];
				snprintf(name, sizeof(name), "%s.check", s.innames[u]);
				write_field(name, s.Nx, s.Ny, s.pwrite, s.dx, s.dy, fields + u * npts);
			}
		return 0;
	}
	const char* pe = getenv("PFC_B200_PRECISION");
	const pfcg_prec prec = (pe && strcmp(pe, "fp32") == 0) ? PFCG_FP32 : PFCG_FP64;
	if (!pfcg_size_supported(s.Nx, s.Ny))
		die_msg(E_UNSUPPORTED, "grid size not supported by pfc_b200 (need even sizes 8..8192 with prime factors 2, 3, 5, 7).");
	if (!pfcg_size_supported_for(s.Nx, s.Ny, s.U, prec))
		die_msg(E_UNSUPPORTED, prec == PFCG_FP64 ? "grid size not supported by pfc_b200 in FP64 for this many fields "
		                                           "(see pfcg_size_supported_for; PFC_B200_PRECISION=fp32 supports more)."
		                                         : "grid size not supported by pfc_b200 for this many fields.");
	const char* de = getenv("PFC_B200_DEVICE");
	check(pfcg_set_device(de ? atoi(de) : 0), NULL);

	s.p.c = s.c;
	s.p.dt = s.dt;
	pfcg_handle* h = NULL;
	check(pfcg_create(&s.p, s.Nx, s.Ny, s.dx, s.dy, prec, &h), NULL);
	check(pfcg_upload(h, fields), h);

	double* fdens = s.fname ? (double*)malloc(sizeof(double) * npts) : NULL;
	int have_f = 0;
	double fave = 0.0, nave[PFCG_MAX_U] = {0};
	double d = 0.0001; /* relax(), :1296 */
	double dx = s.dx, dy = s.dy;
	int nw = 0;
	for (int t = 0; t <= s.tend;) {
		check(pfcg_set_time(h, t), h);
		if (s.Topt > 0 && t > 0 && t % s.Topt == 0) {
			if (fdens) {
				/* the reference's f(r) after optimize is the one of its last sampled box (:1260-1267) */
				const double tx = dx + (s.yopt ? 0.0 : (s.xopt ? d : 0.0));
				const double ty = dy + (s.yopt ? d : 0.0);
				check(pfcg_set_box(h, tx, ty), h);
				check(pfcg_evaluate(h, &fave, nave, fdens), h);
				check(pfcg_set_box(h, dx, dy), h);
				have_f = 1;
			}
			check(pfcg_optimize(h, s.xopt, s.yopt, &d), h);
			check(pfcg_get_box(h, &dx, &dy), h);
		}
		if (s.Tprint > 0 && t % s.Tprint == 0) {
			check(pfcg_evaluate(h, &fave, nave, fdens), h);
			if (fdens) have_f = 1;
			print_output(&s, t, t0, dx, dy, fave, nave);
		}
		if (nw < s.nwrite && t == s.twrite[nw]) {
			check(pfcg_download(h, fields), h);
			char name[LINE];
			for (int u = 0; u < s.U; u++) {
				step_name(s.outnames[u], t, name, sizeof(name));
				write_field(name, s.Nx, s.Ny, s.pwrite, dx, dy, fields + u * npts);
			}
			if (fdens) {
				if (!have_f) check(pfcg_evaluate(h, &fave, nave, fdens), h);
				have_f = 1;
				step_name(s.fname, t, name, sizeof(name));
				write_field(name, s.Nx, s.Ny, s.pwrite, dx, dy, fdens);
			}
			nw++;
		}
		if (t >= s.tend) break;
		/* step to the next event in one call */
		int next = s.tend;
		if (s.Tprint > 0 && (t / s.Tprint + 1) * s.Tprint < next) next = (t / s.Tprint + 1) * s.Tprint;
		if (s.Topt > 0 && (t / s.Topt + 1) * s.Topt < next) next = (t / s.Topt + 1) * s.Topt;
		if (nw < s.nwrite && s.twrite[nw] > t && s.twrite[nw] < next) next = s.twrite[nw];
		check(pfcg_step(h, next - t), h);
		t = next;
	}
	pfcg_destroy(h);
	free(fields);
	free(fdens);
	return 0;
}
