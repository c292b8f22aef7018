/*
 * One-rank implementation of the FFTW-MPI / MPI subset declared in
 * fftw3-mpi.h, over oracle/fft64.c. Test infrastructure only.
 */
#include "fftw3-mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../fft64.h"

struct pfc_shim_plan {
	int kind; /* 0 = r2c, 1 = c2r, 2 = complex forward, 3 = complex backward */
	int n0, n1; /* rows (y), columns (x) of the real array */
	void* in;
	void* out;
	unsigned flags;
};

int MPI_Init(int* argc, char*** argv) { (void)argc; (void)argv; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_rank(MPI_Comm comm, int* rank) { (void)comm; *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm comm, int* size) { (void)comm; *size = 1; return 0; }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return 0; }
int MPI_Abort(MPI_Comm comm, int code) {
	(void)comm;
	fflush(stdout);
	fflush(stderr);
	exit(code);
}
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm) {
	(void)op; (void)comm;
	if (sendbuf != MPI_IN_PLACE) {
		size_t sz = (type == MPI_DOUBLE) ? sizeof(double) : sizeof(int);
		const char* s = (const char*)sendbuf;
		char* d = (char*)recvbuf;
		for (size_t i = 0; i < sz * (size_t)count; i++) d[i] = s[i];
	}
	return 0;
}

void fftw_mpi_init(void) {}
void fftw_mpi_cleanup(void) {}

ptrdiff_t fftw_mpi_local_size_2d_transposed(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm comm, ptrdiff_t* local_n0,
                                            ptrdiff_t* local_0_start, ptrdiff_t* local_n1, ptrdiff_t* local_1_start) {
	(void)comm;
	*local_n0 = n0;
	*local_0_start = 0;
	*local_n1 = n1;
	*local_1_start = 0;
	return n0 * n1;
}

ptrdiff_t fftw_mpi_local_size_2d(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm comm, ptrdiff_t* local_n0, ptrdiff_t* local_0_start) {
	(void)comm;
	*local_n0 = n0;
	*local_0_start = 0;
	return n0 * n1;
}

static fftw_plan mkplan(int kind, ptrdiff_t n0, ptrdiff_t n1, void* in, void* out, unsigned flags) {
	(void)flags;
	fftw_plan p = (fftw_plan)malloc(sizeof(*p));
	p->kind = kind;
	p->n0 = (int)n0;
	p->n1 = (int)n1;
	p->in = in;
	p->out = out;
	fft64_prepare_2d((int)n0, (int)n1);
	return p;
}

fftw_plan fftw_mpi_plan_dft_r2c_2d(ptrdiff_t n0, ptrdiff_t n1, double* in, fftw_complex* out, MPI_Comm comm, unsigned flags) {
	(void)comm;
	return mkplan(0, n0, n1, in, out, flags);
}

fftw_plan fftw_mpi_plan_dft_c2r_2d(ptrdiff_t n0, ptrdiff_t n1, fftw_complex* in, double* out, MPI_Comm comm, unsigned flags) {
	(void)comm;
	return mkplan(1, n0, n1, in, out, flags);
}

fftw_plan fftw_mpi_plan_dft_2d(ptrdiff_t n0, ptrdiff_t n1, fftw_complex* in, fftw_complex* out, MPI_Comm comm, int sign,
                               unsigned flags) {
	(void)comm;
	fftw_plan p = mkplan(sign < 0 ? 2 : 3, n0, n1, in, out, flags);
	p->flags = flags;
	fft64_plan1d_get((int)n0);
	fft64_plan1d_get((int)n1);
	return p;
}

/* complex 2-D: rows [n0][n1] <-> transposed spectrum [n1][n0] (documented FFTW-MPI layouts) */
static void c2c_2d(const fftw_plan p) {
	const int n0 = p->n0, n1 = p->n1;
	const size_t n = (size_t)n0 * n1;
	fft64_cplx* in = (fft64_cplx*)p->in;
	fft64_cplx* out = (fft64_cplx*)p->out;
	fft64_cplx* t = (fft64_cplx*)malloc(sizeof(fft64_cplx) * n);
	const int sign = p->kind == 2 ? -1 : +1;
	const int tin = (p->flags & FFTW_MPI_TRANSPOSED_IN) != 0, tout = (p->flags & FFTW_MPI_TRANSPOSED_OUT) != 0;
	const fft64_plan1d* p0 = fft64_plan1d_get(n0);
	const fft64_plan1d* p1 = fft64_plan1d_get(n1);
	/* t = input as [n0][n1] */
	if (tin) {
		for (int i = 0; i < n1; i++)
			for (int j = 0; j < n0; j++) t[(size_t)j * n1 + i] = in[(size_t)i * n0 + j];
	} else {
		memcpy(t, in, sizeof(fft64_cplx) * n);
	}
	fft64_cplx* w = (fft64_cplx*)malloc(sizeof(fft64_cplx) * (n0 > n1 ? n0 : n1));
	fft64_cplx* col = (fft64_cplx*)malloc(sizeof(fft64_cplx) * n0);
	for (int j = 0; j < n0; j++) fft64_1d(p1, sign, t + (size_t)j * n1, w);
	for (int i = 0; i < n1; i++) {
		for (int j = 0; j < n0; j++) col[j] = t[(size_t)j * n1 + i];
		fft64_1d(p0, sign, col, w);
		for (int j = 0; j < n0; j++) t[(size_t)j * n1 + i] = col[j];
	}
	if (tout) {
		for (int i = 0; i < n1; i++)
			for (int j = 0; j < n0; j++) out[(size_t)i * n0 + j] = t[(size_t)j * n1 + i];
	} else {
		memcpy(out, t, sizeof(fft64_cplx) * n);
	}
	free(col);
	free(w);
	free(t);
}

void fftw_execute(const fftw_plan p) {
	if (p->kind >= 2) {
		c2c_2d(p);
		return;
	}
	const ptrdiff_t stride = 2 * (p->n1 / 2 + 1);
	if (p->kind == 0)
		fft64_r2c_2d_tr(p->n0, p->n1, (const double*)p->in, stride, (fft64_cplx*)p->out);
	else
		fft64_c2r_2d_tr(p->n0, p->n1, (const fft64_cplx*)p->in, (double*)p->out, stride);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }

void* fftw_malloc(size_t n) {
	void* p = NULL;
	if (posix_memalign(&p, 64, n ? n : 1) != 0) return NULL;
	return p;
}
void fftw_free(void* p) { free(p); }
double* fftw_alloc_real(size_t n) { return (double*)fftw_malloc(n * sizeof(double)); }
fftw_complex* fftw_alloc_complex(size_t n) { return (fftw_complex*)fftw_malloc(n * sizeof(fftw_complex)); }
