/*
 * fft64 — double-precision FFTs for the CPU oracle (test infrastructure only).
 *
 * This is NOT part of the product. It exists so that
 *   (1) the reference solver source (pfc-relax.c) can be compiled on a machine
 *       without FFTW, through the FFTW/MPI subset in oracle/shim/, and
 *   (2) the C restatement in oracle/pfc_oracle.c has an FP64 transform.
 *
 * Algorithm: mixed-radix Stockham autosort (Govindaraju et al., "High
 * performance discrete Fourier transforms on graphics processors", SC 2008),
 * radices 4, 2, 3, 5, 7 plus a direct DFT for any other prime factor, so every
 * length is accepted. Twiddles are computed directly in double from the index
 * (no recurrences).
 *
 * The 2-D real transforms reproduce the data layout of FFTW-MPI's
 * fftw_mpi_plan_dft_r2c_2d / c2r_2d with FFTW_MPI_TRANSPOSED_OUT / _IN on one
 * rank, which is what pfc-relax.c relies on (pfc-relax.c:227-235):
 *   real array:    Ny rows, row stride Nxp = 2*(Nx/2+1) doubles, x fastest;
 *   complex array: (Nx/2+1) x Ny, index Ny*kx + ky (transposed), unnormalised.
 * Order of work matches FFTW-MPI's transposed plans: r2c along x, then the
 * complex transform along y; c2r does the inverse y transform first and then
 * the x c2r, in which the imaginary parts of the kx=0 and (even Nx) kx=Nx/2
 * entries are ignored.
 */
#ifndef PFC_ORACLE_FFT64_H
#define PFC_ORACLE_FFT64_H

#include <complex.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double _Complex fft64_cplx;

typedef struct fft64_plan1d fft64_plan1d;

/* Returns a cached plan for complex length n (n >= 1). Not thread safe:
 * call before entering parallel regions. */
const fft64_plan1d* fft64_plan1d_get(int n);

/* In-place complex DFT of x (length n). sign = -1 forward, +1 backward,
 * unnormalised. work must hold n elements. */
void fft64_1d(const fft64_plan1d* p, int sign, fft64_cplx* x, fft64_cplx* work);

/* 2-D real-to-complex, output transposed ([kx][ky], ky fastest), unnormalised.
 * in: Ny rows of Nx doubles at row stride in_stride (doubles).
 * out: (Nx/2+1)*Ny complex. in and out may alias. */
void fft64_r2c_2d_tr(int Ny, int Nx, const double* in, ptrdiff_t in_stride, fft64_cplx* out);

/* 2-D complex-to-real, input transposed, unnormalised.
 * in: (Nx/2+1)*Ny complex; out: Ny rows of Nx doubles at row stride out_stride.
 * in and out may alias. */
void fft64_c2r_2d_tr(int Ny, int Nx, const fft64_cplx* in, double* out, ptrdiff_t out_stride);

/* Prepares the plans the 2-D transforms of this size use (call once, serially). */
void fft64_prepare_2d(int Ny, int Nx);

#ifdef __cplusplus
}
#endif

#endif
