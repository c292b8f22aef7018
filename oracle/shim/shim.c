/*
 * One-rank implementation of the FFTW-MPI / MPI subset declared in
 * fftw3-mpi.h, over oracle/fft64.c. Test infrastructure only.
 */
#include "fftw3-mpi.h"

#include <stdio.h>
#include <stdlib.h>

#include "../fft64.h"

struct pfc_shim_plan {
	int kind; /* 0 = r2c, 1 = c2r */
	int n0, n1; /* rows (y), columns (x) of the real array */
	void* in;
	void* out;
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

void fftw_execute(const fftw_plan p) {
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
