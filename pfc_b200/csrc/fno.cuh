// Internal entry points of the warm-start network used by the relaxation handle.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

struct pfcg_fno;

// Tiled network application on a device FP64 grid of two fields (y-major,
// field-major, d_in != d_out), with the input's field means restored in FP64.
// Ordered after prior work on st; st waits for it.
int fno_apply_device(pfcg_fno* f, const double* d_in, double* d_out, int Nx, int Ny, cudaStream_t st);

// A device scratch grid of at least n doubles owned by the network object.
int fno_scratch_grid(pfcg_fno* f, size_t n, double** out);

const char* fno_error(const pfcg_fno* f);
