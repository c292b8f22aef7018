// Kernel interfaces of the B200 relaxation path (implemented in kernels_impl.cuh,
// instantiated by kernels_f32*.cu and kernels_f64.cu, and in kernels_common.cu).
//
// Data layout in HBM for a system of U fields on an Nx x Ny grid, H = Nx/2+1:
//
//   spec[u]  spectral state N^_u / (Nx Ny) without its k = 0 entry, complex,
//            [kx][ky] with ky fastest (the reference's TRANSPOSED_OUT order,
//            pfc-relax.c:227-228, index Ny*kx + ky). Entry (0,0) is kept 0.
//   mean[u]  the k = 0 entry (the mean density), FP64.
//   work[u]  the mixed (kx, y) representation between the two passes, complex,
//            tiled by R rows: element (kx, y) at ((y/R)*H + kx)*R + y%R, so one
//            row tile is contiguous for the x-pass and CC adjacent columns of
//            one tile are contiguous for the y-pass.
//
// One time step is two kernels:
//   x-pass (one CTA per R-row tile, all U fields): c2r along x of work,
//     + mean -> real field m, nonlinear term NL(m) (pfc-relax.c:1188-1209),
//     r2c along x -> work. Sum of NL (FP64) and a NaN flag are reduced on the way.
//   y-pass (one CTA per CC columns, all U fields): forward FFT along y of work
//     -> M^, k-space coupling and ETD1 update with A, B computed on the fly
//     (pfc-relax.c:1215-1244, 901-958) against spec, write spec, inverse FFT
//     along y -> work. The k = 0 entry is updated in FP64 from the NL sum, and
//     the kx = 0 and kx = Nx/2 columns are projected onto their Hermitian part.
// Pairs of real rows (or of fields) share one complex transform of length Nx.
#pragma once

#include <cuda_runtime.h>

#include "fft_core.cuh"

namespace pfcg {

constexpr int MAXU = 4;
constexpr int MAXW = 4;
constexpr int MAX_CH = 8;     // real rows (channels) per x-pass CTA; odd counts pad with a zero channel
constexpr int MAX_TRIAL = 5;  // box sizes per Parseval reduction

struct Model {
	int U;
	int W[MAXU];
	double c;  // 0 nonconserved, 1 conserved (normalised as pfc-relax.c:930)
	double sigma, dt;
	double lambda[MAXU], delta[MAXU];
	double alpha[MAXU][MAXU], beta[MAXU][MAXU], gamma[MAXU][MAXU], epsilon[MAXU][MAXU], mu2[MAXU][MAXU];
	double nu2[MAXU][MAXW], omega[MAXU][MAXW], phi[MAXU][MAXW];
	int scheme; // SCHEME_ETD1 (the reference's update) or SCHEME_SEMI (linear part implicit)
};

// Time integrators of the k-space update N' = A N + B M (M the nonlinear and
// coupling terms, x = o a dt with o = c - 1 - c k^2 and a the linear operator):
//   SCHEME_ETD1  A = exp(x), B = (A - 1) / a, the reference's (pfc-relax.c:946-953)
//   SCHEME_SEMI  A = 1 / (1 - x), B = o dt / (1 - x): the linear part implicit,
//                the rest explicit, i.e. N' = (N - dt k^2 M) / (1 + dt k^2 a) for
//                conserved dynamics. Same fixed points as ETD1.
enum Scheme { SCHEME_ETD1 = 0, SCHEME_SEMI = 1 };

struct Geom {
	int Nx, Ny, H;
	int R;      // rows per tile
	int CC;     // columns per y-pass CTA
	double dx, dy;
	double dkx, dky;  // 2 pi / (dx Nx), 2 pi / (dy Ny), pfc-relax.c:916-917
};

enum XMode { XP_STEP = 0, XP_EVAL = 1, XP_C2R = 2, XP_R2C = 3 };
enum YMode { YP_STEP = 0, YP_INIT = 1, YP_WEIGHT = 2 };
// k-space weights of YP_WEIGHT: P_u(k), the model's G(k), (mu2 - k^2)^2, and
// for the orientation / deformation fields a Gaussian of runtime spread
// (W_GS), one part of the complex orientation kernel applied to the field pair
// (W_OR) and a Gaussian-smoothed derivative (W_DG)
enum WKind { W_ONE = 0, W_P = 1, W_G = 2, W_Q = 3, W_GS = 4, W_OR = 5, W_DG = 6 };

// Model constants of the y-pass update in the transform precision, filled on
// the host (host_step_k): as kernel parameters the instructions that use them
// read them straight from the constant bank, with no conversion and no
// register held across the update.
template <typename T> struct StepK {
	T invN, cc, dt, ag;
	int semi;
	int W[MAXU];
	T alpha[MAXU], betad[MAXU];
	T nu2[MAXU][MAXW], omega[MAXU][MAXW], phi[MAXU][MAXW];
	T beta[MAXU][MAXU], eps[MAXU][MAXU], mu2[MAXU][MAXU];
	T dkx, dky;
};
template <typename T> StepK<T> host_step_k(const Model& m, const Geom& g);

template <typename T> struct XArgs {
	cplx<T>* work;          // U arrays at stride wstride
	long long wstride;
	const double* off;      // per-field value added after c2r / subtracted before r2c (the mean)
	double* real;           // XP_C2R output / XP_R2C input: U fields of Ny*Nx doubles
	double* acc;            // FP64 accumulators of the modes that add atomically (see part)
	int* flag;              // NaN flag
	const cplx<T>* tw;      // twiddles of length Nx
	const cplx<T>* twct;    // per-pass twiddle table of the specialised kernels
	FftPlan plan;
	int sb;                 // channel pairs per FFT call
	Model m;
	Geom g;
	// STEP: the block sums of the nonlinear term go to part[tile * U + u] (the
	// y-pass adds them in a fixed order, so a step is bit-reproducible); EVAL:
	// the 1 + U sums to part[tile * (1 + U) + i] (added by launch_sum_parts);
	// nullptr: atomically into acc
	double* part;
};

// Parameters of one k-space weight (YP_WEIGHT), resolved on the host so the
// kernel never indexes the model by a runtime field index.
struct WParams {
	int W;
	double nu2[MAXW], omega[MAXW], phi[MAXW];
	double mu2;
	double gs;   // W_GS, W_DG: Gaussian exp(-k^2 / (2 gs^2))
	double sk;   // W_OR: radial spread of the kernel exp(-(|k| - 1)^2 / (2 sk^2))
	int fold;    // W_OR: angular order, exp(i fold atan2(ky, kx)) (even)
	int part;    // W_OR: 0 -> Kr s0 - Ki s1, 1 -> Ki s0 + Kr s1 (s0, s1 the two fields)
	int dir;     // W_DG: 0 -> i kx, 1 -> i ky
};

template <typename T> struct YArgs {
	cplx<T>* work;          // in/out (YP_STEP, YP_INIT) or out (YP_WEIGHT)
	long long wstride;
	cplx<T>* spec;          // U arrays at stride sstride
	long long sstride;
	double* mean;           // U, updated in place by YP_STEP at k = 0
	double* acc;            // without part: FP64 sum of NL per field (read and cleared by YP_STEP)
	const cplx<T>* tw;      // twiddles of length Ny
	const cplx<T>* twct;    // per-pass twiddle table of the specialised kernels
	FftPlan plan;
	int sb;                 // sequences per FFT call
	Model m;
	Geom g;
	int wkind, wsrc;        // YP_WEIGHT: weight kind and source field
	WParams wp;             // YP_WEIGHT: parameters of the weight
	int regio;              // STEP, specialised kernels: first/last transform pass to/from global memory
	// STEP with register ends: a CUtensorMap (device memory) over `work` viewed as
	// [field][tile][kx][row] with boxes (R rows, CC columns, tma_tiles tiles, 1
	// field), through which the forward transform's input columns arrive by TMA;
	// nullptr = plain loads. tma_tiles divides Ny / R.
	const void* tmap;
	int tma_tiles;
	unsigned tma_extra;     // bytes the wait expects beyond the loads (0; > 0 only to test the time-out)
	unsigned long long tma_timeout_ns; // bound of that wait
	int* flag;              // bit 1: a bounded device wait ran out (PFCG_ETIMEOUT)
	StepK<T> k;             // STEP: the update's constants
	const double* part;     // STEP: the x-pass's per-tile sums of the nonlinear term (nullptr: acc)
	int nparts;             //   and their number of tiles
};

// Flag bits of the step kernels' status word
constexpr int FLAG_NAN = 1;
constexpr int FLAG_TIMEOUT = 2;

struct LaunchCfg {
	int grid, block, smem;
	int spec;  // 1: the compile-time specialised STEP kernel for this shape (2: never the fused y-pass)
};

// Shapes of the compile-time specialised STEP kernels (kernels_impl.cuh):
// rows per x-pass tile and columns per y-pass CTA for length 2048 / 4096.
int spec_rows(bool fp64, int U, int N);
int spec_cols(bool fp64, int U, int N);
// threads and shared-memory bytes of those kernels
int spec_x_threads(bool fp64, int U, int N);
int spec_y_threads(bool fp64, int U, int N, bool fused);
int spec_x_smem(bool fp64, int U, int N);
int spec_y_smem(bool fp64, int U, int N);
int spec_twiddles(bool fp64, int N);
// 1 if that y-pass reads its input columns straight from memory (TMA-capable)
int spec_y_regio(bool fp64, int U, int N);

// Host-side launchers; return cudaGetLastError().
template <typename T> cudaError_t launch_xpass(int mode, const XArgs<T>& a, const LaunchCfg& c, cudaStream_t s);
template <typename T> cudaError_t launch_ypass(int mode, const YArgs<T>& a, const LaunchCfg& c, cudaStream_t s);

// One batched STEP pass (pass 0 = x, 1 = y) over per-problem arguments in
// device memory (XArgs<T> or YArgs<T> array) and per-block (problem, tile or
// column group) tables of nblk blocks. launch_ct_batch: every block's problem
// has U fields and length N, which has specialised kernels (launch shape c of
// those problems); launch_generic_batch: the runtime-plan kernels, any sizes.
// nblk = 0 only prepares the kernels' shared-memory limits (call it before
// capturing a graph).
template <typename T> void prepare_batch_kernels();
template <typename T>
cudaError_t launch_ct_batch(int pass, int U, int N, const void* probs, const int* bp, const int* bl, int nblk,
                            const LaunchCfg& c, cudaStream_t s);
template <typename T>
cudaError_t launch_generic_batch(int pass, const void* probs, const int* bp, const int* bl, int nblk, int threads,
                                 int smem, cudaStream_t s);

// Parseval sums for up to MAX_TRIAL box sizes: out[t] = ... With part
// (MAX_TRIAL * KSPACE_MAX_BLOCKS doubles) the blocks' sums are added in a fixed
// order; without it they are added to out atomically.
constexpr int KSPACE_MAX_BLOCKS = 148 * 8;
template <typename T>
cudaError_t launch_kspace_energy(const cplx<T>* spec, long long sstride, const Model& m, const Geom& g, int ntrial,
                                 const double* dxs, const double* dys, double* out, double* part, cudaStream_t s);

// out[i] = sum over p < nparts of part[p * nv + i] in a fixed order (i < nv)
cudaError_t launch_sum_parts(const double* part, int nparts, int nv, double* out, cudaStream_t s);

// Deterministic FP64 means of U real fields (npts each): per-block partial
// sums into part[U * nblocks], then one block per field adds them in order.
cudaError_t launch_field_means(const double* real, int U, long long npts, double* part, int nblocks, double* mean,
                               cudaStream_t s);

// f(r) assembly for write_energy: f = sum of local terms of m plus gradient /
// smoothing couplings from the precomputed real fields (kernels_common.cu).
cudaError_t launch_energy_density(const double* m, const double* pn, const double* eta, const double* q, int npair,
                                  const Model& mod, long long npts, double* f, cudaStream_t s);

// orientation / deformation fields: a *= s and b *= s; out = (sum of the
// squares of the four fields of g4)^(power/2); acc += r / max(r) (part: nparts
// doubles of scratch)
cudaError_t launch_fields_mul(double* a, double* b, const double* s, long long n, cudaStream_t st);
cudaError_t launch_fields_gradpow(const double* g4, long long n, double power, double* out, cudaStream_t st);
cudaError_t launch_scaled_acc(double* acc, const double* r, long long n, double* part, int nparts, cudaStream_t st);

// elements per thread and main radix of the runtime-plan kernels; main radix
// of the kernels specialised on the length N
int max_elems_per_thread(bool fp64);
int max_radix(bool fp64);
int ct_radix(bool fp64, int N);

} // namespace pfcg
