/*
 * Timing harness around the reference solver (test/baseline infrastructure).
 *
 * The reference source file (demos/honey/pfc-relax.c, path given by REF_SRC at
 * compile time) is #included unchanged, with its main() renamed, and linked
 * against the one-rank FFTW/MPI shim in oracle/shim/. This harness then calls
 * the reference's own functions in the order its initialize() and relax() do
 * (pfc-relax.c:960-965, 1293-1313), except that the density fields come from a
 * raw float64 file instead of read_data()'s text parser, so that a bounded
 * window of step() calls can be timed without minutes of %lf parsing:
 *
 *   pfc-relax-bench <input.in> <fields.bin> <warmup steps> <timed steps>
 *
 * fields.bin holds U*Ny*Nx little-endian doubles, component-major, y-major.
 * The .n files named in input.in only need their header line (read_input
 * reads nothing else from them, pfc-relax.c:463-470).
 * Prints one JSON line: steps, seconds, threads and a checksum of the result.
 */
#define main pfc_reference_main
#include REF_SRC
#undef main

#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static double now_s(void) {
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int main(int argc, char** argv) {
	if (argc != 5) {
		fprintf(stderr, "usage: %s <input.in> <fields.bin> <warmup> <steps>\n", argv[0]);
		return 2;
	}
	struct S s;
	memset(&s, 0, sizeof(s));
	s.r = 0;
	s.R = 1;
	s.t0 = (int)time(NULL);
	strncpy(s.input, argv[1], BUFSIZ - 1);
	read_input(&s);
	allocate_data(&s);
	plan_FFTs(&s);

	FILE* fb = fopen(argv[2], "rb");
	if (!fb) { fprintf(stderr, "cannot open %s\n", argv[2]); return 3; }
	const int Nxp = 2 * (s.Nx / 2 + 1);
	for (int u = 0; u < s.U; u++)
		for (int j = 0; j < s.Ny; j++)
			if (fread(s.m[u] + (size_t)Nxp * j, sizeof(double), (size_t)s.Nx, fb) != (size_t)s.Nx) {
				fprintf(stderr, "short read in %s\n", argv[2]);
				return 3;
			}
	fclose(fb);
	update_AB(&s);

	const int W = atoi(argv[3]);
	const int K = atoi(argv[4]);
	s.t = 0;
	for (int k = 0; k < W; k++, s.t++) step(&s);
	const double t0 = now_s();
	for (int k = 0; k < K; k++, s.t++) step(&s);
	const double t1 = now_s();

	double sum = 0.0;
	for (int j = 0; j < s.Ny; j++)
		for (int i = 0; i < s.Nx; i++) sum += s.m[0][(size_t)Nxp * j + i];
	int threads = 1;
#ifdef _OPENMP
	threads = omp_get_max_threads();
#endif
	printf("{\"steps\": %d, \"seconds\": %.6f, \"threads\": %d, \"Nx\": %d, \"Ny\": %d, \"U\": %d, \"checksum\": %.17g}\n",
	       K, t1 - t0, threads, s.Nx, s.Ny, s.U, sum);
	return 0;
}
