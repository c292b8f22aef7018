/*
 * pfc_b200.h — C ABI of the B200 spectral relaxation library (libpfc_b200.so).
 *
 * The reference (petenez/pfc, pfc-relax.c) has no library API: its hot path is
 * the set of functions relax() calls between the host parser and FFTW-MPI.
 * Each entry point below replaces one of those functions (cited per entry).
 * Line numbers refer to demos/honey/pfc-relax.c, the copy the oracle is built
 * from; src/pfc-relax.c lacks its line 499, so subtract 1 from lines >= 500 there.
 *
 * Conventions
 *  - Plain C types only; the caller owns every host buffer it passes.
 *  - The library owns device memory, one CUDA stream and its graphs per handle.
 *    One handle per host thread; handles are independent (no global state).
 *  - Real fields cross the boundary unpadded, y-major: value (x=i, y=j) of
 *    component u is at fields[(u*Ny + j)*Nx + i] — the order of the .n files
 *    (pfc-relax.c:748-755, 803-809).
 *  - Return value: 0 = success; positive = the reference's fail() code for the
 *    same condition (pfc-relax.c:242-411), e.g. 39 = NaN detected; negative =
 *    a library error (PFCG_E*), with a message from pfcg_last_error().
 */
#ifndef PFC_B200_H
#define PFC_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PFCG_MAX_U 4 /* density fields per system */
#define PFCG_MAX_W 4 /* modes per density field */

/* error codes (library-side; positive codes are the reference's fail() codes) */
#define PFCG_OK 0
#define PFCG_NAN 39         /* pfc-relax.c:402-404, "Not a number value detected." */
#define PFCG_EARG (-1)      /* invalid argument */
#define PFCG_ECUDA (-2)     /* CUDA runtime error */
#define PFCG_ESIZE (-3)     /* grid size not supported (see pfcg_size_supported) */
#define PFCG_ENOMEM (-4)    /* device allocation failed */
#define PFCG_ETIMEOUT (-5)  /* a bounded device-side wait ran out */
#define PFCG_ENODEV (-6)    /* no CUDA device / not an sm_100 device */

typedef enum { PFCG_FP32 = 0, PFCG_FP64 = 1 } pfcg_prec;

/* Model parameters, stored the way pfc-relax.c's read_input leaves them in
 * struct S (pfc-relax.c:34-120, 542-705):
 *   nu2[u][w] = 1/(1/nu)^2 (:655), mu2[u][v] = 1/(1/mu)^2, or 0 when beta[u][v]
 *   == 0 (:699-700). Matrices are read in their upper triangle (v >= u; v > u
 *   for epsilon and mu2). c is the raw input value: 0 = nonconserved, any other
 *   value = conserved (:930). */
typedef struct pfcg_params {
	int U;
	int W[PFCG_MAX_U];
	double c;
	double sigma;
	double dt;
	double lambda[PFCG_MAX_U];
	double delta[PFCG_MAX_U];
	double alpha[PFCG_MAX_U][PFCG_MAX_U];
	double beta[PFCG_MAX_U][PFCG_MAX_U];
	double gamma[PFCG_MAX_U][PFCG_MAX_U];
	double epsilon[PFCG_MAX_U][PFCG_MAX_U];
	double mu2[PFCG_MAX_U][PFCG_MAX_U];
	double nu2[PFCG_MAX_U][PFCG_MAX_W];
	double omega[PFCG_MAX_U][PFCG_MAX_W];
	double phi[PFCG_MAX_U][PFCG_MAX_W];
} pfcg_params;

typedef struct pfcg_handle pfcg_handle;

/* 1 if an Nx x Ny grid has a supported shape (both even, 8 <= N <= 8192,
 * N = 2^a 3^b 5^c 7^d), else 0: a necessary condition. The reference accepts
 * any size through FFTW; sizes outside this set are rejected with PFCG_ESIZE
 * instead of falling back to a CPU path. */
int pfcg_size_supported(int Nx, int Ny);

/* 1 if pfcg_create accepts an Nx x Ny grid of U fields in precision prec, else
 * 0 (no device work). Beyond the shape rules above, a transform of length N
 * runs in one CTA: a radix-r pass needs N/r <= 512 * floor(16/r) butterflies
 * (so 8192 with factors 2 only, 7168 with a 7, 7680 with a 3 or 5), and the U
 * fields of one column (y-pass) or the channel pairs of one row (x-pass) must
 * fit in shared memory (e.g. FP64 with U = 2 up to Ny of about 5600). */
int pfcg_size_supported_for(int Nx, int Ny, int U, pfcg_prec prec);

/* Creates a relaxation of U = p->U fields on an Nx x Ny grid with spacing dx, dy.
 * Replaces initialize() minus read_data: allocate_data (:162-193), plan_FFTs
 * (:196-239) and update_AB (:901-958). prec selects the FFT/pointwise precision;
 * reductions, the k=0 (mean) mode and the box optimisation are FP64 in both. */
int pfcg_create(const pfcg_params* p, int Nx, int Ny, double dx, double dy, pfcg_prec prec, pfcg_handle** out);

/* Uploads the real fields (U*Ny*Nx doubles, layout above) as the state at time
 * t = 0. Replaces read_data (:729-764) filling m[u], plus the first spectral
 * synchronisation step() does at t = 0 (:1179-1185). */
int pfcg_upload(pfcg_handle* h, const double* fields);

/* Downloads the current real fields (U*Ny*Nx doubles). Replaces the m[u] that
 * write_data prints (:803-809). */
int pfcg_download(pfcg_handle* h, double* fields);

/* As pfcg_upload / pfcg_download, with the fields in DEVICE memory (for data
 * that is generated or consumed on the GPU). */
int pfcg_upload_device(pfcg_handle* h, const double* d_fields);
int pfcg_download_device(pfcg_handle* h, double* d_fields);

/* Seeded two-field heterostructure initial state, generated on the device
 * (the one-mode approximation and periodic Voronoi grains of the reference's
 * initial-state builder, src/PFCInit.java:46-93 and :389-462). Each region
 * belongs to one field, which carries mean[u] + amp[u] * OMA(r, sym,
 * lattice[u]) there, rotated by the grain's angle; the other field sits at its
 * mean. grains > 0: Voronoi grains with centres, angles in [0, max_angle_deg)
 * and fields drawn from the seed; grains <= 0: vertical stripes of
 * stripe_width columns, shifted by stripe_offset >= 0 columns, field
 * ((x + offset) / width) % 2, unrotated. noise * N(0, 1) is added to both
 * fields. d_fields: DEVICE, 2 x Ny x Nx doubles. No counterpart in the
 * reference's C code (its states come from pfc-init.jar). */
typedef struct pfcg_hetero {
	int grains;
	int stripe_width, stripe_offset;
	int sym; /* 3 triangular, 4 square, 6 honeycomb */
	double mean[2], amp[2], lattice[2];
	double noise;
	double max_angle_deg;
	unsigned seed;
} pfcg_hetero;
int pfcg_init_hetero(double* d_fields, int Nx, int Ny, double dx, double dy, const pfcg_hetero* s, void* stream);
const char* pfcg_init_last_error(void);

/* One grain of the reference builder's Voronoi step "V" (src/PFCInit.java:389-462,
 * fields in its input order): centre (x, y) (wrapped into the box), write type
 * (0 overwrite, 1 superpose, 2 phantom: the point is left as it is), lattice
 * symmetry (3 triangular, 4 square, 6 honeycomb), length scale a, average
 * density nave, amplitude amp, noise amplitude namp, and the placement tx1,
 * ty1, theta (degrees), rotation axis xr, yr, tx2, ty2. */
typedef struct pfcg_grain {
	double x, y;
	int type, sym;
	double a, nave, amp, namp;
	double tx1, ty1, theta_deg, xr, yr, tx2, ty2;
} pfcg_grain;

/* The Voronoi step on one field (Ny*Nx doubles, y-major; DEVICE or HOST memory,
 * told apart by cudaPointerGetAttributes), read and written in place: each
 * point takes the grain whose centre is nearest under periodic boundaries
 * (closest(), src/PFCInit.java:68-93) and becomes
 * type * old + nave + amp * OMA(r') + 2 namp (U - 0.5) (:444-458), OMA the
 * one-mode lattice of :46-66. U is java.util.Random's nextDouble, drawn once
 * per non-phantom point in row-major order as the Java loop does; *rng is the
 * generator's 48-bit state (pfcg_java_random_seed(seed) for new Random(seed)),
 * advanced past the draws on return, so consecutive steps continue one
 * sequence. Allocates and frees its own scratch; synchronises `stream`. */
int pfcg_init_voronoi(double* field, int Nx, int Ny, double dx, double dy, int ngrains, const pfcg_grain* grains,
                      long long* rng, void* stream);

/* The 48-bit state of java.util.Random(seed) (its documented initial scramble). */
long long pfcg_java_random_seed(long long seed);

/* Writes a density field as the reference builder's output step "O" does
 * (src/PFCInit.java:670-686): "Nx Ny " then dx and dy in Java's "%.{prec}e",
 * then the Nx*Ny values (y-major) one per line in the same format. Java's
 * Formatter rounds the shortest round-trip decimal digits half-up where C's
 * printf rounds the exact binary value (ties to even), so the two differ on
 * values whose shortest digits end in a 5 just past the last printed digit;
 * this writer follows Java (exactly for prec <= 13). HOST memory; returns 0, or
 * PFCG_EARG when the file cannot be written. */
int pfcg_write_n_pfcinit(const char* path, int Nx, int Ny, double dx, double dy, const double* field, int prec);

/* Sets the grid spacing and rebuilds the linear operators. Replaces update_AB
 * (:901-958) after a change of s->dx, s->dy. */
int pfcg_set_box(pfcg_handle* h, double dx, double dy);
int pfcg_get_box(const pfcg_handle* h, double* dx, double* dy);

/* Time integration scheme of pfcg_step (and of a batch's steps, which pick up
 * the change at their next pfcg_batch_step). PFCG_SCHEME_ETD1, the default, is
 * the reference's exponential update N' = A N + B M with A = exp(o a dt),
 * B = (A - 1)/a (update_AB, pfc-relax.c:947-953, applied in step :1238).
 * PFCG_SCHEME_SEMI_IMPLICIT treats the linear part implicitly and the rest
 * explicitly: N' = (N + dt o M) / (1 - dt o a), i.e. for conserved dynamics
 * (o = -k^2) N' = (N - dt k^2 M) / (1 + dt k^2 a(k)); it has the same fixed
 * points but no counterpart in the reference. Returns PFCG_EARG for an unknown
 * scheme. */
#define PFCG_SCHEME_ETD1 0
#define PFCG_SCHEME_SEMI_IMPLICIT 1
int pfcg_set_scheme(pfcg_handle* h, int scheme);
int pfcg_get_scheme(const pfcg_handle* h, int* scheme);

/* Relaxation step counter t used for the every-100-steps resynchronisation of
 * the spectral state (:1179-1185). pfcg_upload sets t = 0, pfcg_step advances it. */
int pfcg_set_time(pfcg_handle* h, int t);
int pfcg_get_time(const pfcg_handle* h, int* t);

/* Advances nsteps semi-implicit (ETD1) steps. Replaces step() (:1134-1248)
 * called nsteps times. Returns 39 if a NaN appeared in the field (the
 * reference checks m[0][0] at :1176; this checks every point). Steps, like
 * pfcg_evaluate and pfcg_optimize, are bit-reproducible for a given library
 * build and device: every sum over CTAs is added in a fixed order. */
int pfcg_step(pfcg_handle* h, int nsteps);

/* Computes <f> and <n_u> of the current state, and the free-energy density f(r)
 * (Ny*Nx doubles) when f != NULL. Replaces evaluate() (:988-1131). The gradient
 * coupling uses mu2 as intended; the reference reads nu2 there (:1020), which
 * only matters when some beta[u][v] != 0 with u < v. */
int pfcg_evaluate(pfcg_handle* h, double* fave, double* nave, double* f);

/* One box-size optimisation. Replaces optimize() (:1251-1290): samples <f> at
 * dx, dx -/+ d and dy -/+ d, moves to the parabola vertex with the change
 * clamped to a quarter lattice constant, rebuilds the operators and adapts d.
 * *d is the sampling step (in/out; relax() starts it at 1e-4, :1296). */
int pfcg_optimize(pfcg_handle* h, int xopt, int yopt, double* d);

/* Field u of the current state smoothed by the model's kernel
 * G(k) = exp(-k^2 / (2 sigma^2)) (sigma of pfcg_params), written to out (HOST,
 * Ny*Nx doubles). Replaces the smooth tool (demos/honey/smooth.c:81-121:
 * r2c, multiply by G, c2r, normalise by the sum of the real-space kernel,
 * which is exactly 1 since G(0) = 1). */
int pfcg_smooth(pfcg_handle* h, int u, double* out);

/* Orientation and deformation fields of a density field (Nx*Ny doubles, HOST),
 * replacing the fields tool (src/fields.c): psi (HOST, 2*Ny*Nx doubles: the
 * real plane, then the imaginary plane) is the complex orientation field,
 * (density - min) convolved with exp(-(|k|-1)^2 / (2 sk^2)) exp(i fold
 * atan2(ky, kx)), times (density - min), smoothed by exp(-k^2 / (2 sb^2)) and
 * normalised to max |psi| = 1 (fields.c:103-200); chi (HOST, Ny*Nx, or NULL to
 * skip it) is the deformation field, the sum over Gaussian scales 1/2, 1/4, ...
 * (while 4 pi/sqrt(3) times the scale index stays below half the box) of the
 * maximum-normalised smoothing of |grad psi_unnormalised|^power
 * (fields.c:218-320). fold must be even (the reference's method works only
 * for even folds). Transforms in FP64. Uses the current device. */
int pfcg_fields(const double* density, int Nx, int Ny, double dx, double dy, int fold, double sk, double sb,
                double power, double* psi, double* chi);

/* Makes `device` the CUDA device that later pfcg_create calls on this host
 * thread use (one process per GPU). No counterpart in the reference, whose
 * ranks are MPI processes (pfc-relax.c:1395-1401). */
int pfcg_set_device(int device);

/* Per-kernel timing with CUDA events on the handle's stream (off by default).
 * pfcg_profile_read returns, for each kernel kind k (0 = x-pass step, 1 = y-pass
 * step, 2 = everything else), the summed milliseconds and launch counts since
 * profiling was switched on. No counterpart in the reference (it prints only
 * wall seconds, pfc-relax.c:881). */
int pfcg_set_profiling(pfcg_handle* h, int on);
int pfcg_profile_read(pfcg_handle* h, double* ms, long long* launches, int nkinds);

/* Measures the launch shapes the runtime-plan kernels can take for this
 * handle's size (rows per x-pass tile, columns per y-pass group) over nsteps
 * steps each and keeps the fastest; results are cached per (precision, U, Nx,
 * Ny) for the process. Call before pfcg_upload: the timing steps run on the
 * handle's buffers, which are cleared afterwards. Sizes with compile-time
 * specialised kernels (FP32: 256, 384, 512, 768, 1024, 1536, 2048, 4096; FP64: 2048,
 * 4096) keep their fixed shape. No counterpart in
 * the reference (FFTW_MEASURE planning, pfc-relax.c:227-231, is the nearest). */
int pfcg_autotune(pfcg_handle* h, int nsteps);

/* Many independent relaxations (sizes, fields and parameters may differ)
 * stepped together. The problems fall into classes: one per (U, N) with
 * N = Nx = Ny a length with specialised kernels (pfcg_autotune lists them), in
 * their fixed launch shape, and one for all other problems, on the
 * runtime-plan kernels. A step of a class is two kernel launches (a batched
 * x-pass and a batched y-pass over per-problem tables); pfcg_batch_step
 * captures nsteps steps into one CUDA graph (cached per nsteps), each class a
 * chain of its own that runs beside the others, and launches it.
 * pfcg_batch_launches reports 2 * classes * nsteps kernels per graph launch. Problem i is an ordinary handle (pfcg_batch_problem) for upload,
 * evaluate, optimize and download; do not step it on its own while the batch is
 * in use. params is an array of nprob structs; autotune != 0 runs
 * pfcg_autotune on every problem first. No counterpart in the reference, which
 * relaxes one system per process. */
typedef struct pfcg_batch pfcg_batch;
int pfcg_batch_create(int nprob, const pfcg_params* params, const int* Nx, const int* Ny, const double* dx,
                      const double* dy, pfcg_prec prec, int autotune, pfcg_batch** out);
pfcg_handle* pfcg_batch_problem(pfcg_batch* b, int i);
int pfcg_batch_step(pfcg_batch* b, int nsteps); /* 39 if any problem saw a NaN */
int pfcg_batch_launches(const pfcg_batch* b, int nsteps, long long* kernels, long long* graph_launches);
int pfcg_batch_stream(const pfcg_batch* b, void** stream); /* the cudaStream_t the batch launches on, for timing */
void pfcg_batch_destroy(pfcg_batch* b);

/* ---- Learned warm start. No counterpart in the reference. ----
 * A Fourier neural operator on T x T periodic tiles of two fields (T a power
 * of two in [32, 512]): a per-point lift of the two fields to C channels, L
 * layers z = W v + b + K v (K: complex C x C weights on the retained Fourier
 * modes kx = 0..MODES_X-1, ky = -MODES_Y/2..MODES_Y/2-1 of the tile; GELU after
 * every layer but the last), and a per-point projection whose output is added
 * to the input fields. Kernels read BF16 weights and accumulate in FP32; the
 * FP32 master weights are what set/get_params and Adam see.
 * Parameter layout (floats): P[C][2], p[C]; per layer W[C][C], b[C],
 * Re R[C][C][MODES_Y][MODES_X], Im R[...] (R indexed [in][out][ky row][kx],
 * ky rows 0..MODES_Y/2-1 = ky 0.., the rest = ky -MODES_Y/2..-1); Q[2][C], q[2]. */
#define PFCG_FNO_LAYERS 4
#define PFCG_FNO_CHANNELS 32
#define PFCG_FNO_MODES_X 8
#define PFCG_FNO_MODES_Y 16
#define PFCG_FNO_PARAMS 1052962
typedef struct pfcg_fno pfcg_fno;
size_t pfcg_fno_param_count(void);
/* max_batch tiles per launch sequence; memory grows as max_batch * T^2 * 1.9 KB. */
int pfcg_fno_create(int tile, int max_batch, pfcg_fno** out);
int pfcg_fno_set_params(pfcg_fno* f, const float* host_params); /* also resets Adam */
int pfcg_fno_get_params(pfcg_fno* f, float* host_params);
/* DEVICE tensors [batch][2][T][T] FP32 (x-fastest). */
int pfcg_fno_forward(pfcg_fno* f, const float* d_in, float* d_out, int batch);
/* Mean-square error of the output against d_target over all batch points and
 * both fields, and its gradient (kept on the device for pfcg_fno_adam_step;
 * copied to host_grad when it is not NULL). */
int pfcg_fno_loss_grad(pfcg_fno* f, const float* d_in, const float* d_target, int batch, double* loss,
                       float* host_grad);
int pfcg_fno_adam_step(pfcg_fno* f, float lr, float beta1, float beta2, float eps);
/* The network on a periodic DEVICE grid of two FP64 fields (2 x Ny x Nx,
 * d_in != d_out): tiles of T points whose central T/2 x T/2 block is kept
 * (T/4 points of periodic halo on each side); each field's mean is then
 * restored to the input's in FP64, since the relaxation conserves it.
 * stream: cudaStream_t the call is ordered on (NULL = default stream). */
int pfcg_fno_apply(pfcg_fno* f, const double* d_in, double* d_out, int Nx, int Ny, void* stream);
/* Replaces the handle's fields (U = 2) by the network's proposal, in place on
 * the device; the step count is kept. */
int pfcg_warmstart(pfcg_handle* h, pfcg_fno* f);
int pfcg_fno_stream(const pfcg_fno* f, void** stream);
int pfcg_fno_launch_count(const pfcg_fno* f, long long* count);
const char* pfcg_fno_last_error(const pfcg_fno* f); /* NULL: last failed create */
void pfcg_fno_destroy(pfcg_fno* f);

/* Bytes of the static device workspace of pfcg_relax_noalloc. */
#define PFCG_NOALLOC_SCRATCH_BYTES (32u << 20)

/* One relaxation of nsteps steps without any device allocation. No counterpart
 * in the reference: it exists for callers that cannot call cudaMalloc, such as
 * a host application that hands out all device memory from its own pool and
 * forbids other allocations, or a loop that must not pay cudaMalloc's implicit
 * device synchronisation.
 * fields: DEVICE memory, U*Ny*Nx doubles in the layout above; it holds the
 *   initial fields on entry and the relaxed fields on return. The caller
 *   allocates it; the call itself allocates nothing.
 * stream: a cudaStream_t (NULL = the default stream); the call returns after it
 *   has synchronised with that stream.
 * Transforms run in FP32 (means and reductions in FP64), as PFCG_FP32, on the
 * runtime-plan step kernels only: the kernels specialised on a length need
 * per-pass twiddle tables that this call does not build, so at those lengths a
 * step costs more than through a handle (512^2 U=1: about 59 us against 24 us
 * on a B200).
 * The workspace is a file-scope array of PFCG_NOALLOC_SCRATCH_BYTES (32 MiB)
 * that every GPU loading the library holds until exit; grids needing more,
 * about 2 * U * (Nx/2+1) * Ny * 8 bytes plus 32 * Ny bytes and a few KB, are
 * rejected with PFCG_ESIZE. Every call looks up the array's address on the
 * current device (cudaGetSymbolAddress, which allocates nothing). The first
 * call on a device also sets kernel attributes (cudaFuncSetAttribute); make
 * that first call before any stream capture begins. All calls share the one
 * array and it keeps the last call's contents (the call clears what must start
 * at zero), so calls that overlap on the GPU (other streams, other host
 * threads) race.
 * Returns 0, 39 on NaN, or a negative PFCG_E* code (pfcg_last_error(NULL)). */
int pfcg_relax_noalloc(const pfcg_params* p, int Nx, int Ny, double dx, double dy, int nsteps, double* fields,
                       void* stream);

/* The CUDA stream the handle launches on (a cudaStream_t), for timing. */
int pfcg_stream(const pfcg_handle* h, void** stream);

/* Number of kernel launches the handle has issued so far. */
int pfcg_launch_count(const pfcg_handle* h, long long* count);

/* Last error message of the handle (or of the last failed pfcg_create when h is NULL). */
const char* pfcg_last_error(const pfcg_handle* h);

void pfcg_destroy(pfcg_handle* h);

#ifdef __cplusplus
}
#endif

#endif
