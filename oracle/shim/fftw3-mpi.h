/*
 * Minimal stand-in for <fftw3-mpi.h> (and the MPI names it pulls in), so the
 * reference solver pfc-relax.c (and smooth.c) compiles unchanged with gcc on a
 * machine that has neither FFTW nor MPI. Test infrastructure only: this header
 * and shim.c are built into the oracle binaries under oracle/_ref/ and nothing
 * in the product includes them.
 *
 * Only the public API names and documented semantics that the reference calls
 * are provided (pfc-relax.c:24, 166, 196-239, 248-408, 1120-1121, 1395-1430;
 * smooth.c:18-19, 49, 73-75, 86, 102-103, 113), for ONE rank:
 *   - fftw_mpi_local_size_2d_transposed returns the whole grid as the local slab;
 *   - r2c / c2r 2-D plans with FFTW_MPI_TRANSPOSED_OUT / _IN run oracle/fft64.c;
 *   - MPI_Allreduce with MPI_IN_PLACE is the identity, MPI_Abort exits with the code.
 * No FFTW or MPI code is used or reproduced.
 */
#ifndef PFC_ORACLE_SHIM_FFTW3_MPI_H
#define PFC_ORACLE_SHIM_FFTW3_MPI_H

#include <complex.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- MPI subset ---- */
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_DOUBLE ((MPI_Datatype)1)
#define MPI_INT ((MPI_Datatype)2)
#define MPI_SUM ((MPI_Op)1)
#define MPI_MIN ((MPI_Op)2)
#define MPI_MAX ((MPI_Op)3)
#define MPI_IN_PLACE ((void*)1)

int MPI_Init(int* argc, char*** argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);

/* ---- FFTW subset ---- */
typedef double _Complex fftw_complex;
typedef struct pfc_shim_plan* fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MPI_TRANSPOSED_IN (1U << 29)
#define FFTW_MPI_TRANSPOSED_OUT (1U << 30)
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)

void fftw_mpi_init(void);
void fftw_mpi_cleanup(void);
ptrdiff_t fftw_mpi_local_size_2d_transposed(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm comm, ptrdiff_t* local_n0,
                                            ptrdiff_t* local_0_start, ptrdiff_t* local_n1, ptrdiff_t* local_1_start);
ptrdiff_t fftw_mpi_local_size_2d(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm comm, ptrdiff_t* local_n0, ptrdiff_t* local_0_start);
fftw_plan fftw_mpi_plan_dft_r2c_2d(ptrdiff_t n0, ptrdiff_t n1, double* in, fftw_complex* out, MPI_Comm comm, unsigned flags);
fftw_plan fftw_mpi_plan_dft_c2r_2d(ptrdiff_t n0, ptrdiff_t n1, fftw_complex* in, double* out, MPI_Comm comm, unsigned flags);
/* complex 2-D transform; FFTW_MPI_TRANSPOSED_OUT (forward) leaves [n1][n0],
 * FFTW_MPI_TRANSPOSED_IN (backward) takes [n1][n0]; unnormalised */
fftw_plan fftw_mpi_plan_dft_2d(ptrdiff_t n0, ptrdiff_t n1, fftw_complex* in, fftw_complex* out, MPI_Comm comm, int sign,
                               unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void* fftw_malloc(size_t n);
void fftw_free(void* p);
double* fftw_alloc_real(size_t n);
fftw_complex* fftw_alloc_complex(size_t n);

#ifdef __cplusplus
}
#endif

#endif
