/*
 * fft64 — double-precision FFTs for the CPU oracle. Test infrastructure only;
 * see fft64.h for the contract and the algorithm reference.
 */
#include "fft64.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define FFT64_PI 3.14159265358979323846264338327950288

struct fft64_plan1d {
	int n;
	int nstage;
	int radix[64];
	fft64_cplx* tw; /* exp(-2 pi i k / n), k = 0..n-1 */
};

/* ---------------------------------------------------------------- plans -- */

#define FFT64_CACHE 64
static fft64_plan1d* cache[FFT64_CACHE];
static int ncache = 0;

static fft64_plan1d* plan_new(int n) {
	fft64_plan1d* p = (fft64_plan1d*)calloc(1, sizeof(*p));
	p->n = n;
	int m = n;
	/* radix order: 4s first, then one 2, then odd primes */
	while (m % 4 == 0) { p->radix[p->nstage++] = 4; m /= 4; }
	while (m % 2 == 0) { p->radix[p->nstage++] = 2; m /= 2; }
	for (int f = 3; m > 1; f += 2) {
		while (m % f == 0) { p->radix[p->nstage++] = f; m /= f; }
	}
	p->tw = (fft64_cplx*)malloc(sizeof(fft64_cplx) * (size_t)n);
	for (int k = 0; k < n; k++) {
		double a = -2.0 * FFT64_PI * (double)k / (double)n;
		p->tw[k] = cos(a) + I * sin(a);
	}
	return p;
}

const fft64_plan1d* fft64_plan1d_get(int n) {
	for (int i = 0; i < ncache; i++)
		if (cache[i]->n == n) return cache[i];
	fft64_plan1d* p = plan_new(n);
	if (ncache < FFT64_CACHE) cache[ncache++] = p;
	return p;
}

/* ------------------------------------------------------------ 1-D DFT --- */

static inline fft64_cplx twv(const fft64_plan1d* p, int sign, int k) {
	fft64_cplx w = p->tw[k];
	return sign < 0 ? w : conj(w);
}

/* multiply by sign*i */
static inline fft64_cplx mul_si(fft64_cplx z, int sign) {
	return sign < 0 ? cimag(z) - I * creal(z) : -cimag(z) + I * creal(z);
}

/* One Stockham stage: radix R, Ns = product of earlier radices. */
static void stage(const fft64_plan1d* p, int sign, int R, int Ns, const fft64_cplx* in, fft64_cplx* out) {
	const int n = p->n;
	const int nR = n / R;
	const int tstep = n / (Ns * R);
	fft64_cplx v[64];
	for (int j = 0; j < nR; j++) {
		const int jm = j % Ns;
		const int idxD = (j / Ns) * Ns * R + jm;
		for (int r = 0; r < R; r++) {
			fft64_cplx x = in[j + r * nR];
			if (r && jm) x *= twv(p, sign, r * jm * tstep);
			v[r] = x;
		}
		if (R == 2) {
			fft64_cplx a = v[0], b = v[1];
			out[idxD] = a + b;
			out[idxD + Ns] = a - b;
		} else if (R == 4) {
			fft64_cplx a0 = v[0] + v[2], a1 = v[0] - v[2];
			fft64_cplx b0 = v[1] + v[3], b1 = mul_si(v[1] - v[3], sign);
			out[idxD] = a0 + b0;
			out[idxD + Ns] = a1 + b1;
			out[idxD + 2 * Ns] = a0 - b0;
			out[idxD + 3 * Ns] = a1 - b1;
		} else {
			/* direct DFT of length R using the plan's table: exp(s 2 pi i rs/R) */
			const int step = n / R;
			for (int s = 0; s < R; s++) {
				fft64_cplx acc = v[0];
				for (int r = 1; r < R; r++) acc += v[r] * twv(p, sign, ((r * s) % R) * step);
				out[idxD + s * Ns] = acc;
			}
		}
	}
}

/* Large prime factors (> 64) fall back to a full direct DFT. */
static void direct_dft(const fft64_plan1d* p, int sign, fft64_cplx* x, fft64_cplx* work) {
	const int n = p->n;
	for (int k = 0; k < n; k++) {
		fft64_cplx acc = 0;
		for (int j = 0; j < n; j++) acc += x[j] * twv(p, sign, (int)(((long long)j * k) % n));
		work[k] = acc;
	}
	memcpy(x, work, sizeof(fft64_cplx) * (size_t)n);
}

void fft64_1d(const fft64_plan1d* p, int sign, fft64_cplx* x, fft64_cplx* work) {
	for (int s = 0; s < p->nstage; s++)
		if (p->radix[s] > 64) { direct_dft(p, sign, x, work); return; }
	fft64_cplx* a = x;
	fft64_cplx* b = work;
	int Ns = 1;
	for (int s = 0; s < p->nstage; s++) {
		const int R = p->radix[s];
		stage(p, sign, R, Ns, a, b);
		Ns *= R;
		fft64_cplx* t = a; a = b; b = t;
	}
	if (a != x) memcpy(x, a, sizeof(fft64_cplx) * (size_t)p->n);
}

/* ------------------------------------------------------------ 2-D ------- */

void fft64_prepare_2d(int Ny, int Nx) {
	fft64_plan1d_get(Nx);
	fft64_plan1d_get(Ny);
}

static int nthreads(void) {
#ifdef _OPENMP
	return omp_get_max_threads();
#else
	return 1;
#endif
}
static int tid(void) {
#ifdef _OPENMP
	return omp_get_thread_num();
#else
	return 0;
#endif
}

/* blocked transpose: src rows x cols (ld_src) -> dst cols x rows (ld_dst) */
static void transpose(const fft64_cplx* src, int rows, int cols, ptrdiff_t ld_src, fft64_cplx* dst, ptrdiff_t ld_dst) {
	const int B = 32;
#pragma omp parallel for collapse(2) schedule(static)
	for (int r0 = 0; r0 < rows; r0 += B)
		for (int c0 = 0; c0 < cols; c0 += B) {
			int r1 = r0 + B < rows ? r0 + B : rows;
			int c1 = c0 + B < cols ? c0 + B : cols;
			for (int r = r0; r < r1; r++)
				for (int c = c0; c < c1; c++) dst[(ptrdiff_t)c * ld_dst + r] = src[(ptrdiff_t)r * ld_src + c];
		}
}

void fft64_r2c_2d_tr(int Ny, int Nx, const double* in, ptrdiff_t in_stride, fft64_cplx* out) {
	const int H = Nx / 2 + 1;
	const fft64_plan1d* px = fft64_plan1d_get(Nx);
	const fft64_plan1d* py = fft64_plan1d_get(Ny);
	fft64_cplx* T = (fft64_cplx*)malloc(sizeof(fft64_cplx) * (size_t)H * (size_t)Ny);
	const int nt = nthreads();
	const int wl = (Nx > Ny ? Nx : Ny);
	fft64_cplx* wbuf = (fft64_cplx*)malloc(sizeof(fft64_cplx) * (size_t)wl * 2 * (size_t)nt);

	/* rows, two real rows per complex transform */
	const int npair = (Ny + 1) / 2;
#pragma omp parallel for schedule(static)
	for (int pr = 0; pr < npair; pr++) {
		fft64_cplx* z = wbuf + (size_t)tid() * 2 * wl;
		fft64_cplx* w = z + wl;
		const int y0 = 2 * pr, y1 = 2 * pr + 1;
		const double* a = in + (ptrdiff_t)y0 * in_stride;
		if (y1 < Ny) {
			const double* b = in + (ptrdiff_t)y1 * in_stride;
			for (int x = 0; x < Nx; x++) z[x] = a[x] + I * b[x];
		} else {
			for (int x = 0; x < Nx; x++) z[x] = a[x];
		}
		fft64_1d(px, -1, z, w);
		fft64_cplx* ta = T + (size_t)y0 * H;
		fft64_cplx* tb = (y1 < Ny) ? T + (size_t)y1 * H : NULL;
		for (int k = 0; k < H; k++) {
			fft64_cplx zk = z[k];
			fft64_cplx zc = conj(z[(Nx - k) % Nx]);
			ta[k] = 0.5 * (zk + zc);
			if (tb) tb[k] = -0.5 * I * (zk - zc);
		}
	}
	/* transpose T[y][k] -> out[k][y] (T is a separate buffer, so aliasing of in/out is fine) */
	transpose(T, Ny, H, H, out, Ny);
	free(T);
	/* columns */
#pragma omp parallel for schedule(static)
	for (int k = 0; k < H; k++) {
		fft64_cplx* w = wbuf + (size_t)tid() * 2 * wl;
		fft64_1d(py, -1, out + (size_t)k * Ny, w);
	}
	free(wbuf);
}

void fft64_c2r_2d_tr(int Ny, int Nx, const fft64_cplx* in, double* out, ptrdiff_t out_stride) {
	const int H = Nx / 2 + 1;
	const fft64_plan1d* px = fft64_plan1d_get(Nx);
	const fft64_plan1d* py = fft64_plan1d_get(Ny);
	fft64_cplx* C = (fft64_cplx*)malloc(sizeof(fft64_cplx) * (size_t)H * (size_t)Ny);
	fft64_cplx* T = (fft64_cplx*)malloc(sizeof(fft64_cplx) * (size_t)H * (size_t)Ny);
	memcpy(C, in, sizeof(fft64_cplx) * (size_t)H * (size_t)Ny);
	const int nt = nthreads();
	const int wl = (Nx > Ny ? Nx : Ny);
	fft64_cplx* wbuf = (fft64_cplx*)malloc(sizeof(fft64_cplx) * (size_t)wl * 2 * (size_t)nt);
	/* inverse along y for every kx column */
#pragma omp parallel for schedule(static)
	for (int k = 0; k < H; k++) {
		fft64_cplx* w = wbuf + (size_t)tid() * 2 * wl;
		fft64_1d(py, +1, C + (size_t)k * Ny, w);
	}
	transpose(C, H, Ny, Ny, T, H);
	free(C);
	const int npair = (Ny + 1) / 2;
	const int even = (Nx % 2 == 0);
#pragma omp parallel for schedule(static)
	for (int pr = 0; pr < npair; pr++) {
		fft64_cplx* z = wbuf + (size_t)tid() * 2 * wl;
		fft64_cplx* w = z + wl;
		const int y0 = 2 * pr, y1 = 2 * pr + 1;
		const fft64_cplx* A = T + (size_t)y0 * H;
		const fft64_cplx* B = (y1 < Ny) ? T + (size_t)y1 * H : NULL;
		for (int k = 0; k < H; k++) {
			fft64_cplx a = A[k], b = B ? B[k] : 0;
			if (k == 0 || (even && k == Nx / 2)) { a = creal(a); b = creal(b); }
			z[k] = a + I * b;
			if (k > 0 && Nx - k >= H) z[Nx - k] = conj(a) + I * conj(b);
		}
		fft64_1d(px, +1, z, w);
		double* oa = out + (ptrdiff_t)y0 * out_stride;
		for (int x = 0; x < Nx; x++) oa[x] = creal(z[x]);
		if (B) {
			double* ob = out + (ptrdiff_t)y1 * out_stride;
			for (int x = 0; x < Nx; x++) ob[x] = cimag(z[x]);
		}
	}
	free(T);
	free(wbuf);
}
