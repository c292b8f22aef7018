// C ABI of libpfc_b200.so (declared in include/pfc_b200.h): handle life
// cycle, launch-shape selection and the host side of evaluate / optimize.
//
// Reference correspondence (demos/honey/pfc-relax.c):
//   pfcg_create     allocate_data :162-193, plan_FFTs :196-239, update_AB :901-958
//   pfcg_upload     read_data's m[u] :729-764 + first resync in step :1179-1185
//   pfcg_step       step :1134-1248 (x-pass + y-pass kernels per step)
//   pfcg_evaluate   evaluate :988-1131 (local terms in real space, gradient and
//                   smoothing terms by Parseval in k space)
//   pfcg_optimize   optimize :1251-1290
//   pfcg_download   the m[u] written by write_data :767-815
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/pfc_b200.h"
#include "fno.cuh"
#include "kernels.cuh"

using namespace pfcg;

namespace {

constexpr int ACC_NL = 0;     // U doubles: sum of the nonlinear term of the current step
constexpr int ACC_EVAL = 8;   // 1 + U doubles: sum of local energy density, sums of m_u
constexpr int ACC_TRIAL = 16; // MAX_TRIAL doubles: Parseval sums per box size
constexpr int ACC_N = 24;
constexpr int OFFS_N = 32;    // per-field offsets for the f(r) fields
constexpr int MAX_THREADS = 512;
// doubles of a handle's block-sum slots: a step's U per row tile, evaluate's
// 1 + U per row tile (Ny tiles at most) or its MAX_TRIAL per Parseval block
size_t nlpart_elems(int Ny) {
	return std::max((size_t)(MAXU + 1) * Ny, (size_t)MAX_TRIAL * KSPACE_MAX_BLOCKS);
}
constexpr double PI = 3.14159265358979323846264338327;

thread_local std::string g_err;

} // namespace

struct pfcg_handle {
	int dev = 0;
	pfcg_prec prec = PFCG_FP64;
	Model model{};
	Geom geom{};
	int U = 0, Nx = 0, Ny = 0, H = 0;
	int t = 0;
	cudaStream_t stream = nullptr;
	size_t celem = 0; // bytes of one complex element
	void* spec = nullptr;
	void* work = nullptr;
	void* work1 = nullptr;
	void* twx = nullptr;
	void* twy = nullptr;
	double* mean = nullptr;
	double* acc = nullptr;
	double* offs = nullptr;
	int* flag = nullptr;
	int* h_flag = nullptr;
	double* h_buf = nullptr; // pinned: ACC_N accumulators, MAXU means, OFFS_N offsets
	FftPlan px{}, py{};
	LaunchCfg cx{}, cy{}, cx1{}, cy1{};
	LaunchCfg cxs{}, cys{}; // STEP kernels (possibly compile-time specialised)
	void* twctx = nullptr;  // per-pass twiddle tables of the specialised kernels
	void* twcty = nullptr;
	int sbx = 1, sby = 1, sbx1 = 1, sby1 = 1;
	double* d_real = nullptr;   // U*Ny*Nx doubles
	double* d_fields = nullptr; // f(r) work fields
	double* d_part = nullptr;   // partial sums of the field means
	double* nlpart = nullptr;   // per-block sums added in a fixed order: of the nonlinear term in a step (U per
	                            // row tile), of evaluate's local terms (1 + U per tile) and Parseval sums
	int regio = 1;              // y-pass register ends (PFCG_YPASS_REGIO=0: load/store phases through shared memory)
	void* tmap = nullptr;       // device copy of the y-pass's TMA tensor map over `work` (null: plain loads)
	int tma_tiles = 0;          // row tiles per TMA box
	// Test hook of the bounded wait (PFCG_TMA_TEST_STALL=<bytes> when the handle is created): the
	// wait expects that many bytes more than the loads bring, so it runs out after 1 ms and the
	// step reports PFCG_ETIMEOUT; no load or store changes.
	unsigned tma_extra = 0;
	unsigned long long tma_timeout_ns = 1000000000ull;
	long long launches = 0;
	// per-kernel timing (pfcg_set_profiling)
	bool profiling = false;
	// STEP_GRAPH steps captured as one CUDA graph and replayed by do_steps, for
	// the arguments in sgraph_key (recaptured when the box, scheme or launch
	// shapes change); stepped_plain: a step has run outside capture (the
	// kernels' attributes are set)
	cudaGraphExec_t sgraph = nullptr;
	std::vector<unsigned char> sgraph_key;
	bool stepped_plain = false;
	std::vector<cudaEvent_t> ev;     // event pairs, recorded around launches
	std::vector<int> ev_kind;
	double prof_ms[3] = {0, 0, 0};
	long long prof_n[3] = {0, 0, 0};
	std::string err;
};

namespace {

// wave-number steps of the current box, pfc-relax.c:916-917
void set_dk(pfcg_handle* h) {
	h->geom.dkx = 2.0 * PI / (h->geom.dx * h->Nx);
	h->geom.dky = 2.0 * PI / (h->geom.dy * h->Ny);
}

int fail(pfcg_handle* h, int code, const std::string& msg) {
	if (h) h->err = msg;
	else g_err = msg;
	return code;
}

int cuda_fail(pfcg_handle* h, const char* what, cudaError_t e) {
	return fail(h, PFCG_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(h, call)                                                                                                    \
	do {                                                                                                           \
		cudaError_t e_ = (call);                                                                               \
		if (e_ != cudaSuccess) return cuda_fail(h, #call, e_);                                                 \
	} while (0)

bool factor_ok(int n) {
	if (n < 1) return false;
	for (int f : {2, 3, 5, 7})
		while (n % f == 0) n /= f;
	return n == 1;
}

// n = RM^nmain * rtail * 3^n3 * 5^n5 * 7^n7, rtail in {1,2,4,8} below RM
bool make_plan(int n, int rmain, FftPlan* p) {
	if (!factor_ok(n)) return false;
	int m = n, k2 = 0;
	p->n = n;
	p->n3 = p->n5 = p->n7 = 0;
	while (m % 2 == 0) { m /= 2; k2++; }
	while (m % 3 == 0) { m /= 3; p->n3++; }
	while (m % 5 == 0) { m /= 5; p->n5++; }
	while (m % 7 == 0) { m /= 7; p->n7++; }
	const int lg = (rmain == 16) ? 4 : 3;
	p->nmain = k2 / lg;
	p->rtail = 1 << (k2 % lg);
	return true;
}

// threads one fft_batch over P sequences needs (0 if more than MAX_THREADS)
int threads_for(const FftPlan& p, int P, int maxe) {
	auto need = [&](int R) {
		const long long bfly = (long long)P * p.n / R;
		const int nb = maxe / R;
		return (int)((bfly + nb - 1) / nb);
	};
	int nt = 32;
	if (p.nmain > 0) nt = std::max(nt, need(maxe));
	if (p.rtail > 1) nt = std::max(nt, need(p.rtail));
	if (p.n3) nt = std::max(nt, need(3));
	if (p.n5) nt = std::max(nt, need(5));
	if (p.n7) nt = std::max(nt, need(7));
	nt = (nt + 31) / 32 * 32;
	return nt <= MAX_THREADS ? nt : 0;
}

// largest sub-batch (<= S) whose FFT fits in MAX_THREADS threads; 0 if none
int sub_batch(const FftPlan& p, int S, int maxe, int* nt) {
	for (int sb = S; sb >= 1; sb--) {
		const int t = threads_for(p, sb, maxe);
		if (t) { *nt = t; return sb; }
	}
	return 0;
}

template <typename T> int padded_host(int n) { return padded_len<T>(n); }

int padded(int n, bool fp64) { return fp64 ? padded_host<double>(n) : padded_host<float>(n); }

bool x_tile_ok(const pfcg_handle* h, int r) {
	const bool fp64 = h->prec == PFCG_FP64;
	const size_t budget = fp64 ? 200 * 1024 : 150 * 1024;
	if (h->Ny % r) return false;
	const int CH = h->U * r;
	if (CH > MAX_CH) return false;
	const int P = (CH + 1) / 2;
	if ((size_t)P * padded(h->Nx, fp64) * h->celem > budget) return false;
	int nt;
	return sub_batch(h->px, P, max_elems_per_thread(fp64), &nt) > 0;
}

bool y_group_ok(const pfcg_handle* h, int c) {
	const bool fp64 = h->prec == PFCG_FP64;
	const size_t budget = fp64 ? 200 * 1024 : 150 * 1024;
	const int S = h->U * c;
	if ((size_t)S * padded(h->Ny, fp64) * h->celem > budget) return false;
	int nt;
	return sub_batch(h->py, S, max_elems_per_thread(fp64), &nt) > 0;
}

// launch shapes of the runtime-plan kernels for row tile R and column group CC
void set_generic_configs(pfcg_handle* h, int R, int CC) {
	const bool fp64 = h->prec == PFCG_FP64;
	const int maxe = max_elems_per_thread(fp64);
	const int U = h->U;
	h->geom.R = R;
	h->geom.CC = CC;
	int nt;
	const int P = (U * R + 1) / 2;
	h->sbx = sub_batch(h->px, P, maxe, &nt);
	h->cx = {h->Ny / R, nt, (int)(P * padded(h->Nx, fp64) * h->celem)};
	const int P1 = (R + 1) / 2;
	h->sbx1 = sub_batch(h->px, P1, maxe, &nt);
	h->cx1 = {h->Ny / R, nt, (int)(P1 * padded(h->Nx, fp64) * h->celem)};
	const int S = U * CC;
	h->sby = sub_batch(h->py, S, maxe, &nt);
	h->cy = {(h->H + CC - 1) / CC, nt, (int)(S * padded(h->Ny, fp64) * h->celem)};
	h->sby1 = sub_batch(h->py, CC, maxe, &nt);
	h->cy1 = {(h->H + CC - 1) / CC, nt, (int)(CC * padded(h->Ny, fp64) * h->celem)};
	h->cxs = h->cx;
	h->cys = h->cy;
}

// Chooses the row tile R (x-pass) and column group CC (y-pass): the shape of
// the compile-time specialised kernels where the size has one, otherwise the
// largest sizes that fit shared memory and still give two CTAs per SM
// (pfcg_autotune can replace this guess by measurement).
int choose_layout(pfcg_handle* h, int nsm) {
	const bool fp64 = h->prec == PFCG_FP64;
	const int want = 2 * nsm;
	const int U = h->U;
	int R = 0;
	// PFCG_GENERIC_KERNELS=1 in the environment disables the specialised kernels (A/B checks)
	const char* gen = std::getenv("PFCG_GENERIC_KERNELS");
	const bool allow_spec = !(gen && gen[0] == '1');
	const int rs = allow_spec ? spec_rows(fp64, U, h->Nx) : 0;
	if (rs && h->Ny % rs == 0) R = rs;
	for (int r : {8, 4, 2, 1}) {
		if (R) break;
		if (!x_tile_ok(h, r)) continue;
		R = r;
		if (h->Ny / r >= want) break;
	}
	if (!R) return fail(h, PFCG_ESIZE, "no x-pass tile fits shared memory for this Nx");
	int CC = 0;
	const bool yspec = allow_spec && spec_cols(fp64, U, h->Ny) && spec_rows(fp64, U, h->Ny) == R;
	if (yspec) CC = spec_cols(fp64, U, h->Ny);
	for (int c : {4, 2, 1}) {
		if (CC) break;
		if (!y_group_ok(h, c)) continue;
		CC = c;
		if ((h->H + c - 1) / c >= want) break;
	}
	if (!CC) return fail(h, PFCG_ESIZE, "no y-pass column group fits shared memory for this Ny");
	set_generic_configs(h, R, CC);
	if (rs && R == rs) h->cxs = {h->Ny / R, spec_x_threads(fp64, U, h->Nx), spec_x_smem(fp64, U, h->Nx), 1};
	if (yspec) {
		// The specialised y-pass keeps the update between the two transforms in
		// shared memory by default (measured faster at 4096^2 U=2: 0.299 vs 0.328 ms);
		// PFCG_YPASS_FUSED=1 selects the register-fused variant.
		const char* fu = std::getenv("PFCG_YPASS_FUSED");
		const bool fused = fu && fu[0] == '1';
		h->cys = {(h->H + CC - 1) / CC, spec_y_threads(fp64, U, h->Ny, fused), spec_y_smem(fp64, U, h->Ny), fused ? 1 : 2};
		const char* ri = std::getenv("PFCG_YPASS_REGIO");
		h->regio = (ri && ri[0] == '0') ? 0 : 1;
	}
	return 0;
}

// Per-pass twiddle table of a compile-time length N (the layout of fft_core.cuh's
// CtPlan): passes of radix rmain with the tail radix second; pass p > 0 contributes
// entries [q * Ns + jm] = exp(-2 pi i r_q jm / (Ns R)) with r_q = q + 1, or for
// radix 16 r_q in {1, 2, 3, 4, 8, 12} (ct_twiddle makes the other powers).
template <typename T> int upload_ct_twiddles(pfcg_handle* h, int N, int rmain, void** dst) {
	// N = rmain^A * tail; the tail radix is the second pass (fft_core.cuh, CtPlan)
	std::vector<int> radix;
	int rest = N;
	while (rest % rmain == 0) {
		radix.push_back(rmain);
		rest /= rmain;
	}
	if (rest > 1) radix.insert(radix.begin() + (radix.empty() ? 0 : 1), rest);
	std::vector<cplx<T>> tab;
	int Ns = 1;
	for (size_t p = 0; p < radix.size(); p++) {
		const int R = radix[p];
		static const int pow16[6] = {1, 2, 3, 4, 8, 12};
		const int nq = R == 16 ? 6 : R - 1;
		if (p > 0)
			for (int q = 0; q < nq; q++)
				for (int jm = 0; jm < Ns; jm++) {
					const int r = R == 16 ? pow16[q] : q + 1;
					const double a = -2.0 * PI * (double)r * (double)jm / ((double)Ns * R);
					cplx<T> w;
					w.x = (T)std::cos(a);
					w.y = (T)std::sin(a);
					tab.push_back(w);
				}
		Ns *= R;
	}
	if ((int)tab.size() != spec_twiddles(h->prec == PFCG_FP64, N)) return fail(h, PFCG_ESIZE, "twiddle table size mismatch");
	CK(h, cudaMalloc(dst, sizeof(cplx<T>) * tab.size()));
	CK(h, cudaMemcpy(*dst, tab.data(), sizeof(cplx<T>) * tab.size(), cudaMemcpyHostToDevice));
	return 0;
}

template <typename T> int upload_twiddles(pfcg_handle* h, int n, void** dst) {
	std::vector<cplx<T>> tw(n);
	for (int k = 0; k < n; k++) {
		const double a = -2.0 * PI * (double)k / (double)n;
		tw[k].x = (T)std::cos(a);
		tw[k].y = (T)std::sin(a);
	}
	CK(h, cudaMalloc(dst, sizeof(cplx<T>) * n));
	CK(h, cudaMemcpy(*dst, tw.data(), sizeof(cplx<T>) * n, cudaMemcpyHostToDevice));
	return 0;
}

// The y-pass's TMA tensor map (FP32 specialised y-pass with register ends):
// `work` as a 4-D tensor of 8-byte complex elements [field][tile][kx][row] with
// boxes of (R rows, CC columns, tb tiles, 1 field). A box starts on a 16-byte
// multiple (R * 8 bytes, a multiple of 16, is the innermost extent) and lands
// on a 128-byte multiple of shared memory. PFCG_TMA=0 in the environment keeps
// the plain loads. Without a driver entry point the plain loads are used.
int setup_tma(pfcg_handle* h) {
	const char* env = std::getenv("PFCG_TMA");
	if (env && env[0] == '0') return 0;
	if (h->prec != PFCG_FP32 || !h->cys.spec || h->cys.spec == 1 || !h->regio || h->U > 2) return 0;
	if (!spec_y_regio(false, h->U, h->Ny)) return 0;
	const int R = h->geom.R, CC = h->geom.CC, ntile = h->Ny / R;
	const size_t el = sizeof(float2);
	if ((R * el) % 16 != 0 || CC > 256 || R > 256) return 0;
	int tb = 0;
	for (int t = std::min(256, ntile); t >= 1; t--)
		if (ntile % t == 0 && (t * CC * R * el) % 128 == 0) {
			tb = t;
			break;
		}
	if (!tb) return 0;
	static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
	if (!encode) {
		cudaDriverEntryPointQueryResult q;
		void* fn = nullptr;
		if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn) {
			cudaGetLastError();
			return 0;
		}
		encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
	}
	CUtensorMap tm;
	cuuint64_t dims[4] = {(cuuint64_t)R, (cuuint64_t)h->H, (cuuint64_t)ntile, (cuuint64_t)h->U};
	cuuint64_t strides[3] = {(cuuint64_t)(R * el), (cuuint64_t)h->H * R * el, (cuuint64_t)h->H * h->Ny * el};
	cuuint32_t box[4] = {(cuuint32_t)R, (cuuint32_t)CC, (cuuint32_t)tb, 1};
	cuuint32_t es[4] = {1, 1, 1, 1};
	if (encode(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, h->work, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
	           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
	    CUDA_SUCCESS)
		return 0;
	CK(h, cudaMalloc(&h->tmap, sizeof(CUtensorMap)));
	CK(h, cudaMemcpy(h->tmap, &tm, sizeof(CUtensorMap), cudaMemcpyHostToDevice));
	h->tma_tiles = tb;
	const char* stall = std::getenv("PFCG_TMA_TEST_STALL");
	if (stall && std::atoi(stall) > 0) {
		h->tma_extra = (unsigned)std::atoi(stall) & ~15u;
		h->tma_timeout_ns = 1000000ull;
	}
	return 0;
}

Model to_model(const pfcg_params* p) {
	Model m{};
	m.U = p->U;
	for (int u = 0; u < MAXU; u++) {
		m.W[u] = u < p->U ? p->W[u] : 0;
		m.lambda[u] = p->lambda[u];
		m.delta[u] = p->delta[u];
		for (int v = 0; v < MAXU; v++) {
			m.alpha[u][v] = p->alpha[u][v];
			m.beta[u][v] = p->beta[u][v];
			m.gamma[u][v] = p->gamma[u][v];
			m.epsilon[u][v] = p->epsilon[u][v];
			m.mu2[u][v] = p->mu2[u][v];
		}
		for (int w = 0; w < MAXW; w++) {
			m.nu2[u][w] = p->nu2[u][w];
			m.omega[u][w] = p->omega[u][w];
			m.phi[u][w] = p->phi[u][w];
		}
	}
	m.c = (p->c != 0.0) ? 1.0 : 0.0; // pfc-relax.c:930
	m.sigma = p->sigma;
	m.dt = p->dt;
	return m;
}

double P_host(const Model& m, int u, double k2) {
	double P = 1.0;
	for (int w = 0; w < m.W[u]; w++) {
		const double q = m.nu2[u][w] - k2;
		P *= m.omega[u][w] * q * q + m.phi[u][w];
	}
	return P;
}

// k = 0 term of the Parseval sum (the mean is held outside the spectrum)
double k0_energy(const Model& m, const double* mean) {
	double e = 0.0;
	for (int u = 0; u < m.U; u++) {
		e += 0.5 * m.beta[u][u] * P_host(m, u, 0.0) * mean[u] * mean[u];
		for (int v = u + 1; v < m.U; v++)
			e += (m.beta[u][v] * m.mu2[u][v] * m.mu2[u][v] + m.epsilon[u][v]) * mean[u] * mean[v];
	}
	return e;
}

template <typename T> XArgs<T> xargs(pfcg_handle* h) {
	XArgs<T> a{};
	a.work = (cplx<T>*)h->work;
	a.wstride = (long long)h->H * h->Ny;
	a.off = h->mean;
	a.real = h->d_real;
	a.acc = h->acc;
	a.flag = h->flag;
	a.tw = (const cplx<T>*)h->twx;
	a.twct = (const cplx<T>*)h->twctx;
	a.plan = h->px;
	a.sb = h->sbx;
	a.m = h->model;
	a.g = h->geom;
	a.part = h->nlpart;
	return a;
}

template <typename T> YArgs<T> yargs(pfcg_handle* h) {
	YArgs<T> a{};
	a.work = (cplx<T>*)h->work;
	a.wstride = (long long)h->H * h->Ny;
	a.spec = (cplx<T>*)h->spec;
	a.sstride = (long long)h->H * h->Ny;
	a.mean = h->mean;
	a.acc = h->acc + ACC_NL;
	a.tw = (const cplx<T>*)h->twy;
	a.twct = (const cplx<T>*)h->twcty;
	a.plan = h->py;
	a.sb = h->sby;
	a.m = h->model;
	a.g = h->geom;
	a.regio = h->regio;
	a.tmap = h->tmap;
	a.tma_tiles = h->tma_tiles;
	a.tma_extra = h->tma_extra;
	a.tma_timeout_ns = h->tma_timeout_ns;
	a.flag = h->flag;
	a.k = host_step_k<T>(h->model, h->geom);
	a.part = h->nlpart;
	a.nparts = h->Ny / h->geom.R;
	return a;
}

constexpr int MEAN_BLOCKS = 296;

// Event pair around a launch when profiling; kind 0 = x-pass step, 1 = y-pass step, 2 = other.
struct ProfScope {
	pfcg_handle* h;
	int kind;
	cudaEvent_t b = nullptr, e = nullptr;
	ProfScope(pfcg_handle* h_, int k) : h(h_), kind(k) {
		if (!h->profiling) return;
		cudaEventCreate(&b);
		cudaEventCreate(&e);
		cudaEventRecord(b, h->stream);
	}
	~ProfScope() {
		if (!b) return;
		cudaEventRecord(e, h->stream);
		h->ev.push_back(b);
		h->ev.push_back(e);
		h->ev_kind.push_back(kind);
	}
};

void profile_collect(pfcg_handle* h) {
	if (h->ev.empty()) return;
	cudaStreamSynchronize(h->stream);
	for (size_t i = 0; i < h->ev_kind.size(); i++) {
		float ms = 0.f;
		cudaEventElapsedTime(&ms, h->ev[2 * i], h->ev[2 * i + 1]);
		h->prof_ms[h->ev_kind[i]] += ms;
		h->prof_n[h->ev_kind[i]]++;
		cudaEventDestroy(h->ev[2 * i]);
		cudaEventDestroy(h->ev[2 * i + 1]);
	}
	h->ev.clear();
	h->ev_kind.clear();
}

int ensure_real(pfcg_handle* h) {
	if (!h->d_real) CK(h, cudaMalloc(&h->d_real, sizeof(double) * (size_t)h->U * h->Nx * h->Ny));
	return 0;
}

template <typename T> int run_xpass(pfcg_handle* h, int mode, const XArgs<T>& a, const LaunchCfg& c) {
	h->launches++;
	ProfScope ps(h, mode == XP_STEP ? 0 : 2);
	CK(h, launch_xpass<T>(mode, a, c, h->stream));
	return 0;
}
template <typename T> int run_ypass(pfcg_handle* h, int mode, const YArgs<T>& a, const LaunchCfg& c) {
	h->launches++;
	ProfScope ps(h, mode == YP_STEP ? 1 : 2);
	CK(h, launch_ypass<T>(mode, a, c, h->stream));
	return 0;
}

// Spectral state from the real fields in d_real (device): FP64 means, then the
// forward transforms of the fluctuations.
template <typename T> int spectral_from_real(pfcg_handle* h) {
	const size_t npts = (size_t)h->Nx * h->Ny;
	int rc = 0;
	// the mean (k = 0 mode) in FP64, by a fixed-order reduction on the device
	h->launches += 2;
	{
		ProfScope ps(h, 2);
		CK(h, launch_field_means(h->d_real, h->U, (long long)npts, h->d_part, MEAN_BLOCKS, h->mean, h->stream));
	}
	XArgs<T> xa = xargs<T>(h);
	rc = run_xpass<T>(h, XP_R2C, xa, h->cx);
	if (rc) return rc;
	YArgs<T> ya = yargs<T>(h);
	rc = run_ypass<T>(h, YP_INIT, ya, h->cy);
	if (rc) return rc;
	CK(h, cudaStreamSynchronize(h->stream));
	return 0;
}

template <typename T> int do_upload(pfcg_handle* h, const double* fields, cudaMemcpyKind kind) {
	int rc = ensure_real(h);
	if (rc) return rc;
	CK(h, cudaMemcpyAsync(h->d_real, fields, sizeof(double) * h->U * (size_t)h->Nx * h->Ny, kind, h->stream));
	rc = spectral_from_real<T>(h);
	if (rc) return rc;
	h->t = 0;
	return 0;
}

// Real fields -> network proposal -> spectral state, all on the device.
template <typename T> int do_warmstart(pfcg_handle* h, pfcg_fno* f) {
	int rc = ensure_real(h);
	if (rc) return rc;
	XArgs<T> xa = xargs<T>(h);
	rc = run_xpass<T>(h, XP_C2R, xa, h->cx);
	if (rc) return rc;
	const size_t n = 2 * (size_t)h->Nx * h->Ny;
	double* tmp = nullptr;
	if (fno_scratch_grid(f, n, &tmp) || fno_apply_device(f, h->d_real, tmp, h->Nx, h->Ny, h->stream))
		return fail(h, PFCG_ECUDA, std::string("warm start: ") + fno_error(f));
	CK(h, cudaMemcpyAsync(h->d_real, tmp, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
	return spectral_from_real<T>(h);
}

template <typename T> int do_download(pfcg_handle* h, double* fields, cudaMemcpyKind kind) {
	int rc = ensure_real(h);
	if (rc) return rc;
	XArgs<T> xa = xargs<T>(h);
	rc = run_xpass<T>(h, XP_C2R, xa, h->cx);
	if (rc) return rc;
	CK(h, cudaMemcpyAsync(fields, h->d_real, sizeof(double) * h->U * (size_t)h->Nx * h->Ny, kind, h->stream));
	CK(h, cudaStreamSynchronize(h->stream));
	return 0;
}

// Steps per captured step graph. A short step is launch-bound (512^2: two
// kernels of about 5 us each), and one graph launch for 2 * STEP_GRAPH
// kernels removes most of the per-launch cost; PFCG_STEP_GRAPH=0 launches
// every kernel from the host.
constexpr int STEP_GRAPH = 16;

bool step_graphs_on() {
	static const int on = [] {
		const char* e = std::getenv("PFCG_STEP_GRAPH");
		return (e && e[0] == '0') ? 0 : 1;
	}();
	return on != 0;
}

// Captures STEP_GRAPH steps with these arguments into h->sgraph; on any
// failure leaves h->sgraph empty, so that the caller launches the steps itself.
template <typename T> void capture_steps(pfcg_handle* h, const XArgs<T>& xa, const YArgs<T>& ya,
                                         const std::vector<unsigned char>& key) {
	if (h->sgraph) cudaGraphExecDestroy(h->sgraph);
	h->sgraph = nullptr;
	h->sgraph_key.clear();
	if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
		cudaGetLastError();
		return;
	}
	bool ok = true;
	for (int i = 0; i < STEP_GRAPH && ok; i++)
		ok = launch_xpass<T>(XP_STEP, xa, h->cxs, h->stream) == cudaSuccess &&
		     launch_ypass<T>(YP_STEP, ya, h->cys, h->stream) == cudaSuccess;
	cudaGraph_t g = nullptr;
	const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
	if (ok && e == cudaSuccess && g && cudaGraphInstantiate(&h->sgraph, g, 0) == cudaSuccess) h->sgraph_key = key;
	else h->sgraph = nullptr;
	if (g) cudaGraphDestroy(g);
	cudaGetLastError();
}

template <typename T> int do_steps(pfcg_handle* h, int nsteps) {
	XArgs<T> xa = xargs<T>(h);
	xa.acc = h->acc + ACC_NL;
	YArgs<T> ya = yargs<T>(h);
	// The reference resynchronises the spectral state every 100 steps and after
	// evaluate (pfc-relax.c:1179-1185, 1125-1130); the y-pass does the same
	// projection every step, so no separate pass is needed.
	int s = 0;
	if (step_graphs_on() && !h->profiling && nsteps >= STEP_GRAPH) {
		if (!h->stepped_plain) {
			// the first step of a handle runs plainly (it sets the kernels' attributes)
			int rc = run_xpass<T>(h, XP_STEP, xa, h->cxs);
			if (!rc) rc = run_ypass<T>(h, YP_STEP, ya, h->cys);
			if (rc) return rc;
			h->t++;
			s = 1;
			h->stepped_plain = true;
		}
		std::vector<unsigned char> key(sizeof xa + sizeof ya + 2 * sizeof(LaunchCfg));
		std::memcpy(key.data(), &xa, sizeof xa);
		std::memcpy(key.data() + sizeof xa, &ya, sizeof ya);
		std::memcpy(key.data() + sizeof xa + sizeof ya, &h->cxs, sizeof(LaunchCfg));
		std::memcpy(key.data() + sizeof xa + sizeof ya + sizeof(LaunchCfg), &h->cys, sizeof(LaunchCfg));
		if (!h->sgraph || key != h->sgraph_key) capture_steps<T>(h, xa, ya, key);
		if (h->sgraph)
			for (; s + STEP_GRAPH <= nsteps; s += STEP_GRAPH) {
				CK(h, cudaGraphLaunch(h->sgraph, h->stream));
				h->launches += 2 * STEP_GRAPH;
				h->t += STEP_GRAPH;
			}
	}
	for (; s < nsteps; s++) {
		int rc = run_xpass<T>(h, XP_STEP, xa, h->cxs);
		if (rc) return rc;
		rc = run_ypass<T>(h, YP_STEP, ya, h->cys);
		if (rc) return rc;
		h->t++;
		h->stepped_plain = true;
	}
	CK(h, cudaMemcpyAsync(h->h_flag, h->flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
	CK(h, cudaStreamSynchronize(h->stream));
	if (*h->h_flag & FLAG_TIMEOUT) return fail(h, PFCG_ETIMEOUT, "a bounded device-side wait ran out (y-pass TMA load)");
	if (*h->h_flag) return fail(h, PFCG_NAN, "Not a number value detected.");
	return 0;
}

// local part (real space) and Parseval part for ntrial box sizes; returns
// host pointers to the accumulators (valid until the next call)
template <typename T> int eval_sums(pfcg_handle* h, int ntrial, const double* dxs, const double* dys, bool local) {
	CK(h, cudaMemsetAsync(h->acc + ACC_EVAL, 0, sizeof(double) * 16, h->stream));
	if (local) {
		XArgs<T> xa = xargs<T>(h);
		xa.acc = h->acc + ACC_EVAL;
		int rc = run_xpass<T>(h, XP_EVAL, xa, h->cx);
		if (rc) return rc;
		// the row tiles' sums, added in a fixed order
		CK(h, launch_sum_parts(h->nlpart, h->cx.grid, 1 + h->U, h->acc + ACC_EVAL, h->stream));
		h->launches++;
	}
	h->launches += 2;
	ProfScope ps(h, 2);
	CK(h, launch_kspace_energy<T>((const cplx<T>*)h->spec, (long long)h->H * h->Ny, h->model, h->geom, ntrial, dxs, dys,
	                              h->acc + ACC_TRIAL, h->nlpart, h->stream));
	CK(h, cudaMemcpyAsync(h->h_buf, h->acc, sizeof(double) * ACC_N, cudaMemcpyDeviceToHost, h->stream));
	CK(h, cudaMemcpyAsync(h->h_buf + ACC_N, h->mean, sizeof(double) * h->U, cudaMemcpyDeviceToHost, h->stream));
	CK(h, cudaStreamSynchronize(h->stream));
	return 0;
}

// Field u convolved with the smoothing kernel G(k) = exp(-k^2 / (2 sigma^2)) of
// the handle's model, in real space: c2r(G * N_u) plus the FP64 mean (G(0) = 1).
template <typename T> int do_smooth(pfcg_handle* h, int u, double* out, cudaMemcpyKind kind) {
	int rc = ensure_real(h);
	if (rc) return rc;
	if (!h->work1) CK(h, cudaMalloc(&h->work1, h->celem * (size_t)h->H * h->Ny));
	CK(h, cudaMemcpyAsync(h->offs, h->mean + u, sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
	YArgs<T> ya = yargs<T>(h);
	ya.work = (cplx<T>*)h->work1;
	ya.sb = h->sby1;
	ya.wkind = W_G;
	ya.wsrc = u;
	ya.wp = WParams{};
	rc = run_ypass<T>(h, YP_WEIGHT, ya, h->cy1);
	if (rc) return rc;
	XArgs<T> x1 = xargs<T>(h);
	x1.work = (cplx<T>*)h->work1;
	x1.m.U = 1;
	x1.sb = h->sbx1;
	x1.off = h->offs;
	x1.real = h->d_real;
	rc = run_xpass<T>(h, XP_C2R, x1, h->cx1);
	if (rc) return rc;
	CK(h, cudaMemcpyAsync(out, h->d_real, sizeof(double) * (size_t)h->Nx * h->Ny, kind, h->stream));
	CK(h, cudaStreamSynchronize(h->stream));
	return 0;
}

// out = c2r(w(k) * spectrum) + offset for one weight of YP_WEIGHT (device out, Ny*Nx)
template <typename T> int weighted_c2r(pfcg_handle* h, int kind, int src, const WParams& wp, double offset, double* out) {
	if (!h->work1) CK(h, cudaMalloc(&h->work1, h->celem * (size_t)h->H * h->Ny));
	CK(h, cudaStreamSynchronize(h->stream)); // the pinned offset slot is free again
	double* ho = h->h_buf + ACC_N + MAXU;
	ho[0] = offset;
	CK(h, cudaMemcpyAsync(h->offs, ho, sizeof(double), cudaMemcpyHostToDevice, h->stream));
	YArgs<T> ya = yargs<T>(h);
	ya.work = (cplx<T>*)h->work1;
	ya.sb = h->sby1;
	ya.wkind = kind;
	ya.wsrc = src;
	ya.wp = wp;
	int rc = run_ypass<T>(h, YP_WEIGHT, ya, h->cy1);
	if (rc) return rc;
	XArgs<T> x1 = xargs<T>(h);
	x1.work = (cplx<T>*)h->work1;
	x1.m.U = 1;
	x1.sb = h->sbx1;
	x1.off = h->offs;
	x1.real = out;
	return run_xpass<T>(h, XP_C2R, x1, h->cx1);
}

// the FP64 means of the current state, on the host
int host_means(pfcg_handle* h, double* m) {
	CK(h, cudaMemcpyAsync(m, h->mean, sizeof(double) * h->U, cudaMemcpyDeviceToHost, h->stream));
	CK(h, cudaStreamSynchronize(h->stream));
	return 0;
}

template <typename T> int energy_field(pfcg_handle* h, double* f_host) {
	const long long npts = (long long)h->Nx * h->Ny;
	const int U = h->U;
	const int npair = U * (U - 1) / 2;
	const int nf = 3 * U + npair + 1;
	if (!h->d_fields) CK(h, cudaMalloc(&h->d_fields, sizeof(double) * npts * nf));
	if (!h->work1) CK(h, cudaMalloc(&h->work1, h->celem * (size_t)h->H * h->Ny));
	double* mf = h->d_fields;
	double* pn = mf + U * npts;
	double* eta = pn + U * npts;
	double* q = eta + U * npts;
	double* f = q + npair * npts;
	const double* hm = h->h_buf + ACC_N; // means, fetched by eval_sums
	double* ho = h->h_buf + ACC_N + MAXU;
	// offsets = weight at k = 0 times the mean
	int k = 0;
	for (int u = 0; u < U; u++) ho[k++] = P_host(h->model, u, 0.0) * hm[u];
	for (int u = 0; u < U; u++) ho[k++] = hm[u];
	for (int u = 0; u < U; u++)
		for (int v = u + 1; v < U; v++) ho[k++] = h->model.mu2[u][v] * h->model.mu2[u][v] * hm[v];
	CK(h, cudaMemcpyAsync(h->offs, ho, sizeof(double) * k, cudaMemcpyHostToDevice, h->stream));

	XArgs<T> xa = xargs<T>(h);
	xa.real = mf;
	int rc = run_xpass<T>(h, XP_C2R, xa, h->cx);
	if (rc) return rc;

	auto weighted = [&](int kind, int src, int u, int v, double* out, int oi) -> int {
		YArgs<T> ya = yargs<T>(h);
		ya.work = (cplx<T>*)h->work1;
		ya.sb = h->sby1;
		ya.wkind = kind;
		ya.wsrc = src;
		ya.wp = WParams{};
		ya.wp.W = h->model.W[u];
		for (int w = 0; w < MAXW; w++) {
			ya.wp.nu2[w] = h->model.nu2[u][w];
			ya.wp.omega[w] = h->model.omega[u][w];
			ya.wp.phi[w] = h->model.phi[u][w];
		}
		ya.wp.mu2 = (v >= 0) ? h->model.mu2[u][v] : 0.0;
		int r = run_ypass<T>(h, YP_WEIGHT, ya, h->cy1);
		if (r) return r;
		XArgs<T> x1 = xargs<T>(h);
		x1.work = (cplx<T>*)h->work1;
		x1.m.U = 1;
		x1.sb = h->sbx1;
		x1.off = h->offs + oi;
		x1.real = out;
		return run_xpass<T>(h, XP_C2R, x1, h->cx1);
	};
	k = 0;
	for (int u = 0; u < U; u++, k++)
		if ((rc = weighted(W_P, u, u, -1, pn + u * npts, k))) return rc;
	for (int u = 0; u < U; u++, k++)
		if ((rc = weighted(W_G, u, u, -1, eta + u * npts, k))) return rc;
	int pair = 0;
	for (int u = 0; u < U; u++)
		for (int v = u + 1; v < U; v++, pair++, k++)
			if ((rc = weighted(W_Q, v, u, v, q + pair * npts, k))) return rc;
	h->launches++;
	CK(h, launch_energy_density(mf, pn, eta, q, npair, h->model, npts, f, h->stream));
	CK(h, cudaMemcpyAsync(f_host, f, sizeof(double) * npts, cudaMemcpyDeviceToHost, h->stream));
	CK(h, cudaStreamSynchronize(h->stream));
	return 0;
}

template <typename T> int do_evaluate(pfcg_handle* h, double* fave, double* nave, double* f) {
	const double dx = h->geom.dx, dy = h->geom.dy;
	int rc = eval_sums<T>(h, 1, &dx, &dy, true);
	if (rc) return rc;
	const double N = (double)h->Nx * h->Ny;
	const double* acc = h->h_buf;
	const double* hm = h->h_buf + ACC_N;
	const double Q = acc[ACC_TRIAL] + k0_energy(h->model, hm);
	if (fave) *fave = acc[ACC_EVAL] / N + Q;
	// <n_u> is the k = 0 mode, held in FP64 (the reference sums n over the grid,
	// pfc-relax.c:1114, which is the same number up to rounding)
	if (nave)
		for (int u = 0; u < h->U; u++) nave[u] = hm[u];
	if (f) {
		rc = energy_field<T>(h, f);
		if (rc) return rc;
	}
	return 0;
}

template <typename T> int do_optimize(pfcg_handle* h, int xopt, int yopt, double* d) {
	const double dx0 = h->geom.dx, dy0 = h->geom.dy;
	const double dxs[5] = {dx0, dx0 - *d, dx0 + *d, dx0, dx0};
	const double dys[5] = {dy0, dy0, dy0, dy0 - *d, dy0 + *d};
	int idx[5], n = 0;
	double tx[5], ty[5];
	for (int i = 0; i < 5; i++) {
		if (xopt == 0 && (i == 1 || i == 2)) continue;
		if (yopt == 0 && (i == 3 || i == 4)) continue;
		idx[n] = i;
		tx[n] = dxs[i];
		ty[n] = dys[i];
		n++;
	}
	int rc = eval_sums<T>(h, n, tx, ty, true);
	if (rc) return rc;
	const double N = (double)h->Nx * h->Ny;
	const double* acc = h->h_buf;
	const double k0 = k0_energy(h->model, h->h_buf + ACC_N);
	double fs[5] = {0, 0, 0, 0, 0};
	for (int i = 0; i < n; i++) fs[idx[i]] = acc[ACC_EVAL] / N + acc[ACC_TRIAL + i] + k0;
	// the reference leaves s->dx, s->dy at the last sampled size (:1260-1267)
	double dx = tx[n - 1], dy = ty[n - 1];
	if (xopt != 0) dx = (*d * (fs[1] - fs[2]) + 2.0 * dxs[0] * (-2.0 * fs[0] + fs[1] + fs[2])) / (2.0 * (fs[1] - 2.0 * fs[0] + fs[2]));
	if (yopt != 0) dy = (*d * (fs[3] - fs[4]) + 2.0 * dys[0] * (-2.0 * fs[0] + fs[3] + fs[4])) / (2.0 * (fs[3] - 2.0 * fs[0] + fs[4]));
	const double l0 = 4.0 * PI / std::sqrt(3.0);
	const double dw = h->Nx * (dx - dxs[0]);
	const double dh = h->Ny * (dy - dys[0]);
	const double dr = std::sqrt(dw * dw + dh * dh);
	double x = 0.25 * l0;
	if (dr > x) {
		x /= dr;
		dx = x * dx + (1.0 - x) * dxs[0];
		dy = x * dy + (1.0 - x) * dys[0];
	}
	h->geom.dx = dx;
	h->geom.dy = dy;
	set_dk(h);
	const double ddx = dx - dxs[0], ddy = dy - dys[0];
	const double ddr = std::sqrt(ddx * ddx + ddy * ddy);
	if (ddr < *d) *d *= 0.5;
	else *d *= 2.0;
	if (*d < 1.0e-6) *d *= 2.0;
	return 0;
}

} // namespace

extern "C" {

int pfcg_size_supported(int Nx, int Ny) {
	if (Nx < 8 || Ny < 8 || Nx > 8192 || Ny > 8192) return 0;
	if (Nx % 2 || Ny % 2) return 0;
	return factor_ok(Nx) && factor_ok(Ny);
}

int pfcg_size_supported_for(int Nx, int Ny, int U, pfcg_prec prec) {
	if (!pfcg_size_supported(Nx, Ny) || U < 1 || U > PFCG_MAX_U || (prec != PFCG_FP32 && prec != PFCG_FP64)) return 0;
	// the layout checks pfcg_create makes, on a handle that is never allocated;
	// the smallest tile and column group fit whenever any does
	pfcg_handle h;
	h.prec = prec;
	h.U = U;
	h.Nx = Nx;
	h.Ny = Ny;
	h.H = Nx / 2 + 1;
	h.celem = prec == PFCG_FP64 ? sizeof(double2) : sizeof(float2);
	if (!make_plan(Nx, max_radix(prec == PFCG_FP64), &h.px) || !make_plan(Ny, max_radix(prec == PFCG_FP64), &h.py))
		return 0;
	return x_tile_ok(&h, 1) && y_group_ok(&h, 1);
}

int pfcg_create(const pfcg_params* p, int Nx, int Ny, double dx, double dy, pfcg_prec prec, pfcg_handle** out) {
	if (!out) return fail(nullptr, PFCG_EARG, "out is NULL");
	*out = nullptr;
	if (!p) return fail(nullptr, PFCG_EARG, "params is NULL");
	if (p->U < 1 || p->U > PFCG_MAX_U) return fail(nullptr, PFCG_EARG, "U out of range 1..4");
	for (int u = 0; u < p->U; u++)
		if (p->W[u] < 0 || p->W[u] > PFCG_MAX_W) return fail(nullptr, PFCG_EARG, "W[u] out of range 0..4");
	if (prec != PFCG_FP32 && prec != PFCG_FP64) return fail(nullptr, PFCG_EARG, "unknown precision");
	if (!pfcg_size_supported(Nx, Ny))
		return fail(nullptr, PFCG_ESIZE, "grid size not supported (need even 8..8192 with factors 2,3,5,7)");

	int dev = 0;
	cudaError_t e = cudaGetDevice(&dev);
	if (e != cudaSuccess) return fail(nullptr, PFCG_ENODEV, std::string("no CUDA device: ") + cudaGetErrorString(e));
	cudaDeviceProp prop;
	e = cudaGetDeviceProperties(&prop, dev);
	if (e != cudaSuccess) return fail(nullptr, PFCG_ENODEV, cudaGetErrorString(e));
	if (prop.major != 10) return fail(nullptr, PFCG_ENODEV, "libpfc_b200 is built for sm_100a (B200) only");

	pfcg_handle* h = new pfcg_handle();
	h->dev = dev;
	h->prec = prec;
	h->model = to_model(p);
	h->U = p->U;
	h->Nx = Nx;
	h->Ny = Ny;
	h->H = Nx / 2 + 1;
	h->geom.Nx = Nx;
	h->geom.Ny = Ny;
	h->geom.H = h->H;
	h->geom.dx = dx;
	h->geom.dy = dy;
	set_dk(h);
	const bool fp64 = prec == PFCG_FP64;
	h->celem = fp64 ? sizeof(double2) : sizeof(float2);
	const int rmain = max_radix(fp64);
	int rc = 0;
	if (!make_plan(Nx, rmain, &h->px) || !make_plan(Ny, rmain, &h->py)) rc = fail(h, PFCG_ESIZE, "bad factorisation");
	if (!rc) rc = choose_layout(h, prop.multiProcessorCount);
	auto bail = [&](int code) {
		g_err = h->err;
		pfcg_destroy(h);
		return code;
	};
	if (rc) return bail(rc);
	const size_t nspec = (size_t)h->H * Ny;
#define CKC(call)                                                                                                      \
	do {                                                                                                           \
		cudaError_t e_ = (call);                                                                               \
		if (e_ != cudaSuccess) return bail(cuda_fail(h, #call, e_));                                           \
	} while (0)
	CKC(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
	CKC(cudaMalloc(&h->spec, h->celem * nspec * h->U));
	CKC(cudaMalloc(&h->work, h->celem * nspec * h->U));
	CKC(cudaMalloc(&h->mean, sizeof(double) * MAXU));
	CKC(cudaMalloc(&h->acc, sizeof(double) * ACC_N));
	CKC(cudaMalloc(&h->offs, sizeof(double) * OFFS_N));
	CKC(cudaMalloc(&h->flag, sizeof(int)));
	CKC(cudaMalloc(&h->d_part, sizeof(double) * MAXU * MEAN_BLOCKS));
	CKC(cudaMalloc(&h->nlpart, sizeof(double) * nlpart_elems(Ny)));
	CKC(cudaMallocHost(&h->h_flag, sizeof(int)));
	CKC(cudaMallocHost(&h->h_buf, sizeof(double) * (ACC_N + MAXU + OFFS_N)));
	CKC(cudaMemset(h->spec, 0, h->celem * nspec * h->U));
	CKC(cudaMemset(h->work, 0, h->celem * nspec * h->U));
	CKC(cudaMemset(h->mean, 0, sizeof(double) * MAXU));
	CKC(cudaMemset(h->acc, 0, sizeof(double) * ACC_N));
	CKC(cudaMemset(h->flag, 0, sizeof(int)));
	CKC(cudaMemset(h->nlpart, 0, sizeof(double) * nlpart_elems(Ny)));
#undef CKC
	rc = fp64 ? upload_twiddles<double>(h, Nx, &h->twx) : upload_twiddles<float>(h, Nx, &h->twx);
	if (!rc) rc = fp64 ? upload_twiddles<double>(h, Ny, &h->twy) : upload_twiddles<float>(h, Ny, &h->twy);
	if (!rc && h->cxs.spec)
		rc = fp64 ? upload_ct_twiddles<double>(h, Nx, ct_radix(true, Nx), &h->twctx)
		          : upload_ct_twiddles<float>(h, Nx, ct_radix(false, Nx), &h->twctx);
	if (!rc && h->cys.spec)
		rc = fp64 ? upload_ct_twiddles<double>(h, Ny, ct_radix(true, Ny), &h->twcty)
		          : upload_ct_twiddles<float>(h, Ny, ct_radix(false, Ny), &h->twcty);
	if (!rc) rc = setup_tma(h);
	if (rc) return bail(rc);
	*out = h;
	return 0;
}

void pfcg_destroy(pfcg_handle* h) {
	if (!h) return;
	if (h->stream) cudaStreamSynchronize(h->stream);
	cudaFree(h->spec);
	cudaFree(h->work);
	cudaFree(h->work1);
	cudaFree(h->twx);
	cudaFree(h->twy);
	cudaFree(h->twctx);
	cudaFree(h->twcty);
	cudaFree(h->tmap);
	cudaFree(h->mean);
	cudaFree(h->acc);
	cudaFree(h->offs);
	cudaFree(h->flag);
	cudaFree(h->d_real);
	cudaFree(h->d_fields);
	cudaFree(h->d_part);
	cudaFree(h->nlpart);
	for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
	if (h->h_flag) cudaFreeHost(h->h_flag);
	if (h->h_buf) cudaFreeHost(h->h_buf);
	if (h->sgraph) cudaGraphExecDestroy(h->sgraph);
	if (h->stream) cudaStreamDestroy(h->stream);
	delete h;
}

int pfcg_upload(pfcg_handle* h, const double* fields) {
	if (!h || !fields) return fail(h, PFCG_EARG, "NULL argument");
	return h->prec == PFCG_FP64 ? do_upload<double>(h, fields, cudaMemcpyHostToDevice)
	                            : do_upload<float>(h, fields, cudaMemcpyHostToDevice);
}

int pfcg_upload_device(pfcg_handle* h, const double* d_fields) {
	if (!h || !d_fields) return fail(h, PFCG_EARG, "NULL argument");
	return h->prec == PFCG_FP64 ? do_upload<double>(h, d_fields, cudaMemcpyDeviceToDevice)
	                            : do_upload<float>(h, d_fields, cudaMemcpyDeviceToDevice);
}

int pfcg_download(pfcg_handle* h, double* fields) {
	if (!h || !fields) return fail(h, PFCG_EARG, "NULL argument");
	return h->prec == PFCG_FP64 ? do_download<double>(h, fields, cudaMemcpyDeviceToHost)
	                            : do_download<float>(h, fields, cudaMemcpyDeviceToHost);
}

int pfcg_download_device(pfcg_handle* h, double* d_fields) {
	if (!h || !d_fields) return fail(h, PFCG_EARG, "NULL argument");
	return h->prec == PFCG_FP64 ? do_download<double>(h, d_fields, cudaMemcpyDeviceToDevice)
	                            : do_download<float>(h, d_fields, cudaMemcpyDeviceToDevice);
}

// fields.c (write_phi :103-216, write_chi :218-343) on a two-field handle whose
// fields are the real and imaginary parts of the complex field z
static int fields_impl(pfcg_handle* h, const double* density, int fold, double sk, double sb, double power, double* psi,
                       double* chi) {
	const long long n = (long long)h->Nx * h->Ny;
	std::vector<double> host(2 * n, 0.0);
	double mn = density[0];
	for (long long i = 1; i < n; i++) mn = density[i] < mn ? density[i] : mn;
	for (long long i = 0; i < n; i++) host[i] = density[i] - mn;
	double *d_s = nullptr, *d_g = nullptr, *d_part = nullptr;
	auto cleanup = [&]() {
		cudaFree(d_s);
		cudaFree(d_g);
		cudaFree(d_part);
	};
	constexpr int NPART = 296;
	int rc = 0;
	double m[2];
	WParams wp{};
	do {
		if (cudaMalloc(&d_s, sizeof(double) * n) != cudaSuccess || cudaMalloc(&d_g, sizeof(double) * 4 * n) != cudaSuccess ||
		    cudaMalloc(&d_part, sizeof(double) * NPART) != cudaSuccess) {
			rc = fail(h, PFCG_ENOMEM, "fields: device allocation failed");
			break;
		}
		if (cudaMemcpy(d_s, host.data(), sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess) {
			rc = fail(h, PFCG_ECUDA, "fields: copy failed");
			break;
		}
		// z = (density - min) convolved with the complex orientation kernel
		if ((rc = do_upload<double>(h, host.data(), cudaMemcpyHostToDevice))) break;
		if ((rc = host_means(h, m))) break;
		const double k0 = std::exp(-0.5 / (sk * sk)); // the kernel at k = 0
		wp.sk = sk;
		wp.fold = fold;
		wp.part = 0;
		if ((rc = weighted_c2r<double>(h, W_OR, 0, wp, k0 * m[0], h->d_real))) break;
		wp.part = 1;
		if ((rc = weighted_c2r<double>(h, W_OR, 0, wp, k0 * m[1], h->d_real + n))) break;
		// times (density - min), then Gaussian smoothing with spread sb
		if (launch_fields_mul(h->d_real, h->d_real + n, d_s, n, h->stream) != cudaSuccess) {
			rc = fail(h, PFCG_ECUDA, "fields: kernel launch failed");
			break;
		}
		h->launches++;
		if ((rc = spectral_from_real<double>(h))) break;
		if ((rc = host_means(h, m))) break;
		wp = WParams{};
		wp.gs = sb;
		if ((rc = weighted_c2r<double>(h, W_GS, 0, wp, m[0], d_g))) break;
		if ((rc = weighted_c2r<double>(h, W_GS, 1, wp, m[1], d_g + n))) break;
		if (cudaMemcpyAsync(psi, d_g, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
		    cudaStreamSynchronize(h->stream) != cudaSuccess) {
			rc = fail(h, PFCG_ECUDA, "fields: copy failed");
			break;
		}
		double mx = 0.0;
		for (long long i = 0; i < n; i++) mx = std::max(mx, std::hypot(psi[i], psi[n + i]));
		const double inv = 1.0 / mx;
		for (long long i = 0; i < 2 * n; i++) psi[i] *= inv;
		if (!chi) break;
		// deformation: |grad z|^power of the smoothed z, summed over Gaussian scales 1/2, 1/4, ...
		for (int k = 0; k < 4; k++) {
			wp = WParams{};
			wp.gs = sb;
			wp.dir = k / 2;
			if ((rc = weighted_c2r<double>(h, W_DG, k % 2, wp, 0.0, d_g + k * n))) break;
		}
		if (rc) break;
		if (launch_fields_gradpow(d_g, n, power, h->d_real, h->stream) != cudaSuccess ||
		    cudaMemsetAsync(h->d_real + n, 0, sizeof(double) * n, h->stream) != cudaSuccess) {
			rc = fail(h, PFCG_ECUDA, "fields: kernel launch failed");
			break;
		}
		h->launches++;
		if ((rc = spectral_from_real<double>(h))) break;
		if ((rc = host_means(h, m))) break;
		double* acc = d_g + n;
		if (cudaMemsetAsync(acc, 0, sizeof(double) * n, h->stream) != cudaSuccess) {
			rc = fail(h, PFCG_ECUDA, "fields: memset failed");
			break;
		}
		const double l0 = 4.0 * PI / std::sqrt(3.0);
		const double L = std::min(h->Nx * h->geom.dx, h->Ny * h->geom.dy);
		for (int sc = 2; l0 * sc < 0.5 * L; sc *= 2) {
			wp = WParams{};
			wp.gs = 1.0 / sc;
			if ((rc = weighted_c2r<double>(h, W_GS, 0, wp, m[0], d_g))) break;
			if (launch_scaled_acc(acc, d_g, n, d_part, NPART, h->stream) != cudaSuccess) {
				rc = fail(h, PFCG_ECUDA, "fields: kernel launch failed");
				break;
			}
			h->launches += 2;
		}
		if (rc) break;
		if (cudaMemcpyAsync(chi, acc, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
		    cudaStreamSynchronize(h->stream) != cudaSuccess)
			rc = fail(h, PFCG_ECUDA, "fields: copy failed");
	} while (0);
	cleanup();
	return rc;
}

int pfcg_fields(const double* density, int Nx, int Ny, double dx, double dy, int fold, double sk, double sb,
                double power, double* psi, double* chi) {
	if (!density || !psi) return fail(nullptr, PFCG_EARG, "NULL argument");
	if (fold <= 0 || fold % 2) return fail(nullptr, PFCG_EARG, "the orientation kernel needs an even, positive fold");
	if (!(sk > 0) || !(sb > 0)) return fail(nullptr, PFCG_EARG, "kernel spreads must be positive");
	pfcg_params p;
	std::memset(&p, 0, sizeof(p));
	p.U = 2;
	p.c = 1.0;
	p.dt = 1.0;
	p.sigma = 1.0;
	for (int u = 0; u < 2; u++) {
		p.W[u] = 1;
		p.alpha[u][u] = -0.25;
		p.beta[u][u] = 1.0;
		p.nu2[u][0] = 1.0;
		p.omega[u][0] = 1.0;
	}
	pfcg_handle* h = nullptr;
	int rc = pfcg_create(&p, Nx, Ny, dx, dy, PFCG_FP64, &h);
	if (rc) return rc;
	rc = fields_impl(h, density, fold, sk, sb, power, psi, chi);
	if (rc) g_err = h->err;
	pfcg_destroy(h);
	return rc;
}

int pfcg_smooth(pfcg_handle* h, int u, double* out) {
	if (!h || !out) return fail(h, PFCG_EARG, "NULL argument");
	if (u < 0 || u >= h->U) return fail(h, PFCG_EARG, "field index out of range");
	return h->prec == PFCG_FP64 ? do_smooth<double>(h, u, out, cudaMemcpyDeviceToHost)
	                            : do_smooth<float>(h, u, out, cudaMemcpyDeviceToHost);
}

int pfcg_warmstart(pfcg_handle* h, pfcg_fno* f) {
	if (!h || !f) return fail(h, PFCG_EARG, "NULL argument");
	if (h->U != 2) return fail(h, PFCG_EARG, "the warm-start network takes two fields");
	return h->prec == PFCG_FP64 ? do_warmstart<double>(h, f) : do_warmstart<float>(h, f);
}

int pfcg_set_box(pfcg_handle* h, double dx, double dy) {
	if (!h) return PFCG_EARG;
	h->geom.dx = dx;
	h->geom.dy = dy;
	set_dk(h);
	return 0;
}

int pfcg_set_scheme(pfcg_handle* h, int scheme) {
	if (!h) return PFCG_EARG;
	if (scheme != PFCG_SCHEME_ETD1 && scheme != PFCG_SCHEME_SEMI_IMPLICIT)
		return fail(h, PFCG_EARG, "unknown time integration scheme");
	h->model.scheme = scheme == PFCG_SCHEME_SEMI_IMPLICIT ? SCHEME_SEMI : SCHEME_ETD1;
	return 0;
}

int pfcg_get_scheme(const pfcg_handle* h, int* scheme) {
	if (!h || !scheme) return PFCG_EARG;
	*scheme = h->model.scheme == SCHEME_SEMI ? PFCG_SCHEME_SEMI_IMPLICIT : PFCG_SCHEME_ETD1;
	return 0;
}

int pfcg_get_box(const pfcg_handle* h, double* dx, double* dy) {
	if (!h || !dx || !dy) return PFCG_EARG;
	*dx = h->geom.dx;
	*dy = h->geom.dy;
	return 0;
}

int pfcg_set_time(pfcg_handle* h, int t) {
	if (!h) return PFCG_EARG;
	h->t = t;
	return 0;
}

int pfcg_get_time(const pfcg_handle* h, int* t) {
	if (!h || !t) return PFCG_EARG;
	*t = h->t;
	return 0;
}

int pfcg_step(pfcg_handle* h, int nsteps) {
	if (!h || nsteps < 0) return fail(h, PFCG_EARG, "bad argument");
	if (nsteps == 0) return 0;
	return h->prec == PFCG_FP64 ? do_steps<double>(h, nsteps) : do_steps<float>(h, nsteps);
}

int pfcg_evaluate(pfcg_handle* h, double* fave, double* nave, double* f) {
	if (!h) return PFCG_EARG;
	return h->prec == PFCG_FP64 ? do_evaluate<double>(h, fave, nave, f) : do_evaluate<float>(h, fave, nave, f);
}

int pfcg_optimize(pfcg_handle* h, int xopt, int yopt, double* d) {
	if (!h || !d) return fail(h, PFCG_EARG, "NULL argument");
	return h->prec == PFCG_FP64 ? do_optimize<double>(h, xopt, yopt, d) : do_optimize<float>(h, xopt, yopt, d);
}

int pfcg_set_device(int device) {
	cudaError_t e = cudaSetDevice(device);
	if (e != cudaSuccess) return fail(nullptr, PFCG_ENODEV, cudaGetErrorString(e));
	return 0;
}

int pfcg_set_profiling(pfcg_handle* h, int on) {
	if (!h) return PFCG_EARG;
	profile_collect(h);
	h->profiling = on != 0;
	for (int k = 0; k < 3; k++) { h->prof_ms[k] = 0; h->prof_n[k] = 0; }
	return 0;
}

int pfcg_profile_read(pfcg_handle* h, double* ms, long long* launches, int nkinds) {
	if (!h || nkinds < 0) return PFCG_EARG;
	profile_collect(h);
	for (int k = 0; k < nkinds && k < 3; k++) {
		if (ms) ms[k] = h->prof_ms[k];
		if (launches) launches[k] = h->prof_n[k];
	}
	return 0;
}

int pfcg_stream(const pfcg_handle* h, void** stream) {
	if (!h || !stream) return PFCG_EARG;
	*stream = (void*)h->stream;
	return 0;
}

int pfcg_launch_count(const pfcg_handle* h, long long* count) {
	if (!h || !count) return PFCG_EARG;
	*count = h->launches;
	return 0;
}

const char* pfcg_last_error(const pfcg_handle* h) { return h ? h->err.c_str() : g_err.c_str(); }

} // extern "C"

// --------------------------------------------------------------- autotune ---
namespace {

// measured (R, CC) per (precision, U, Nx, Ny), shared by every handle of the process
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, std::pair<int, int>> g_tune;

template <typename T> int time_steps(pfcg_handle* h, int nsteps, float* ms) {
	XArgs<T> xa = xargs<T>(h);
	xa.acc = h->acc + ACC_NL;
	YArgs<T> ya = yargs<T>(h);
	cudaEvent_t e0, e1;
	CK(h, cudaEventCreate(&e0));
	CK(h, cudaEventCreate(&e1));
	int rc = 0;
	for (int s = 0; s < nsteps + 2 && !rc; s++) {
		if (s == 2) cudaEventRecord(e0, h->stream);
		rc = run_xpass<T>(h, XP_STEP, xa, h->cxs);
		if (!rc) rc = run_ypass<T>(h, YP_STEP, ya, h->cys);
	}
	cudaEventRecord(e1, h->stream);
	cudaEventSynchronize(e1);
	cudaEventElapsedTime(ms, e0, e1);
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	return rc;
}

} // namespace

extern "C" int pfcg_autotune(pfcg_handle* h, int nsteps) {
	if (!h || nsteps < 1) return fail(h, PFCG_EARG, "bad argument");
	if (h->cxs.spec || h->cys.spec) return 0; // the specialised kernels have a fixed shape
	const auto key = std::make_tuple((int)h->prec, h->U, h->Nx, h->Ny);
	{
		std::lock_guard<std::mutex> lk(g_tune_mu);
		auto it = g_tune.find(key);
		if (it != g_tune.end()) {
			set_generic_configs(h, it->second.first, it->second.second);
			return 0;
		}
	}
	float best = 1e30f;
	int bR = h->geom.R, bC = h->geom.CC;
	for (int r : {8, 4, 2, 1}) {
		if (!x_tile_ok(h, r)) continue;
		for (int c : {4, 2, 1}) {
			if (!y_group_ok(h, c)) continue;
			set_generic_configs(h, r, c);
			float ms = 0.f;
			const int rc = h->prec == PFCG_FP64 ? time_steps<double>(h, nsteps, &ms) : time_steps<float>(h, nsteps, &ms);
			if (rc) return rc;
			if (ms < best) { best = ms; bR = r; bC = c; }
		}
	}
	set_generic_configs(h, bR, bC);
	// the timing steps ran on whatever the buffers held: start clean
	const size_t nspec = (size_t)h->H * h->Ny * h->U;
	CK(h, cudaMemsetAsync(h->spec, 0, h->celem * nspec, h->stream));
	CK(h, cudaMemsetAsync(h->work, 0, h->celem * nspec, h->stream));
	CK(h, cudaMemsetAsync(h->mean, 0, sizeof(double) * MAXU, h->stream));
	CK(h, cudaMemsetAsync(h->acc, 0, sizeof(double) * ACC_N, h->stream));
	CK(h, cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream));
	CK(h, cudaStreamSynchronize(h->stream));
	std::lock_guard<std::mutex> lk(g_tune_mu);
	g_tune[key] = {bR, bC};
	return 0;
}

// ------------------------------------------------------------------ batch ---
// Problems of a batch that run the same kernels: one length N = Nx = Ny and
// field count U with specialised kernels, or (ct = false) every other problem,
// on the runtime-plan kernels. A class's blocks are a contiguous range of the
// batch's block tables, and its steps form one chain of the step graph on its
// own stream, independent of the other classes' chains.
struct BatchClass {
	bool ct = false;
	int U = 0, N = 0;
	LaunchCfg cx{}, cy{};      // ct: the specialised launch shapes of its problems
	int threads = 0, smem = 0; // runtime-plan class: the largest of its problems'
	int xoff = 0, xn = 0, yoff = 0, yn = 0;
	cudaStream_t stream = nullptr;
	cudaEvent_t done = nullptr;
};

struct pfcg_batch {
	pfcg_prec prec = PFCG_FP32;
	std::vector<pfcg_handle*> h;
	cudaStream_t stream = nullptr;
	cudaEvent_t fork = nullptr;
	void* d_xargs = nullptr;
	void* d_yargs = nullptr;
	int* d_blk = nullptr; // x problem, x local, y problem, y local tables
	int* d_flags = nullptr;
	int* h_flags = nullptr;
	int xblocks = 0, yblocks = 0;
	std::vector<BatchClass> cls;
	std::map<int, cudaGraphExec_t> graphs;
	std::vector<unsigned char> hargs; // host copy of the x and y argument arrays last uploaded
	std::string err;
};

// whether a batch problem runs the specialised kernels (decided at creation)
static bool batch_ct(const pfcg_handle* h) { return h->cxs.spec && h->cys.spec && h->Nx == h->Ny && h->U <= 2; }

namespace {

// per-problem kernel arguments of a batch from the problems' handles
template <typename T> void batch_args(pfcg_batch* b, std::vector<XArgs<T>>& xa, std::vector<YArgs<T>>& ya) {
	const int n = (int)b->h.size();
	xa.assign(n, XArgs<T>{});
	ya.assign(n, YArgs<T>{});
	for (int i = 0; i < n; i++) {
		pfcg_handle* h = b->h[i];
		xa[i] = xargs<T>(h);
		xa[i].acc = h->acc + ACC_NL;
		xa[i].flag = b->d_flags + i;
		ya[i] = yargs<T>(h);
		ya[i].flag = b->d_flags + i; // NaN and wait time-out of problem i
	}
}

// Re-uploads the argument arrays the step graphs read when a problem's box or
// scheme changed since the last upload (pfcg_optimize / pfcg_set_box /
// pfcg_set_scheme on a problem handle), ordered on the batch stream.
template <typename T> int batch_refresh_args(pfcg_batch* b) {
	std::vector<XArgs<T>> xa;
	std::vector<YArgs<T>> ya;
	batch_args<T>(b, xa, ya);
	const size_t bx = sizeof(XArgs<T>) * xa.size(), by = sizeof(YArgs<T>) * ya.size();
	std::vector<unsigned char> cur(bx + by);
	memcpy(cur.data(), xa.data(), bx);
	memcpy(cur.data() + bx, ya.data(), by);
	if (cur == b->hargs) return 0;
	cudaError_t e = cudaMemcpyAsync(b->d_xargs, xa.data(), bx, cudaMemcpyHostToDevice, b->stream);
	if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_yargs, ya.data(), by, cudaMemcpyHostToDevice, b->stream);
	if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
	if (e != cudaSuccess) {
		b->err = std::string("batch arguments: ") + cudaGetErrorString(e);
		return PFCG_ECUDA;
	}
	b->hargs.swap(cur);
	return 0;
}

template <typename T> int batch_build(pfcg_batch* b) {
	const int n = (int)b->h.size();
	auto bfail = [&](cudaError_t e, const char* what) {
		b->err = std::string(what) + ": " + cudaGetErrorString(e);
		return PFCG_ECUDA;
	};
	std::vector<XArgs<T>> xa;
	std::vector<YArgs<T>> ya;
	batch_args<T>(b, xa, ya);
	// classes: one per (U, N) with specialised kernels, one for the rest
	std::map<std::pair<int, int>, int> key;
	std::vector<std::vector<int>> members;
	int generic = -1;
	for (int i = 0; i < n; i++) {
		pfcg_handle* h = b->h[i];
		int c;
		if (batch_ct(h)) {
			auto it = key.find({h->U, h->Nx});
			if (it == key.end()) {
				c = (int)b->cls.size();
				key[{h->U, h->Nx}] = c;
				BatchClass k;
				k.ct = true;
				k.U = h->U;
				k.N = h->Nx;
				k.cx = h->cxs;
				k.cy = h->cys;
				b->cls.push_back(k);
				members.emplace_back();
			} else {
				c = it->second;
			}
		} else {
			if (generic < 0) {
				generic = (int)b->cls.size();
				b->cls.push_back(BatchClass{});
				b->cls.back().threads = 32;
				members.emplace_back();
			}
			c = generic;
			BatchClass& k = b->cls[c];
			k.threads = std::max(k.threads, std::max(h->cx.block, h->cy.block));
			k.smem = std::max(k.smem, std::max(h->cx.smem, h->cy.smem));
		}
		members[c].push_back(i);
	}
	// blocks of the largest problems first, so the tail of a launch is short
	auto work = [&](int i) { return (long long)b->h[i]->Nx * b->h[i]->Ny * b->h[i]->U; };
	std::vector<int> xp, xl, yp, yl;
	for (size_t c = 0; c < b->cls.size(); c++) {
		BatchClass& k = b->cls[c];
		std::vector<int>& m = members[c];
		std::stable_sort(m.begin(), m.end(), [&](int a, int d) { return work(a) > work(d); });
		k.xoff = (int)xp.size();
		k.yoff = (int)yp.size();
		for (int i : m) {
			const pfcg_handle* h = b->h[i];
			const int gx = k.ct ? h->cxs.grid : h->cx.grid, gy = k.ct ? h->cys.grid : h->cy.grid;
			for (int t = 0; t < gx; t++) { xp.push_back(i); xl.push_back(t); }
			for (int g = 0; g < gy; g++) { yp.push_back(i); yl.push_back(g); }
		}
		k.xn = (int)xp.size() - k.xoff;
		k.yn = (int)yp.size() - k.yoff;
		cudaError_t e = cudaStreamCreateWithFlags(&k.stream, cudaStreamNonBlocking);
		if (e == cudaSuccess) e = cudaEventCreateWithFlags(&k.done, cudaEventDisableTiming);
		// the kernels' shared-memory limits are set here, outside any capture
		for (int pass = 0; pass < 2 && e == cudaSuccess; pass++)
			e = k.ct ? launch_ct_batch<T>(pass, k.U, k.N, nullptr, nullptr, nullptr, 0, pass ? k.cy : k.cx, k.stream)
			         : launch_generic_batch<T>(pass, nullptr, nullptr, nullptr, 0, k.threads, k.smem, k.stream);
		if (e != cudaSuccess) return bfail(e, "batch class");
	}
	b->xblocks = (int)xp.size();
	b->yblocks = (int)yp.size();
	cudaError_t e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
	if (e != cudaSuccess) return bfail(e, "cudaEventCreate");
	if ((e = cudaMalloc(&b->d_xargs, sizeof(XArgs<T>) * n)) != cudaSuccess) return bfail(e, "cudaMalloc");
	if ((e = cudaMalloc(&b->d_yargs, sizeof(YArgs<T>) * n)) != cudaSuccess) return bfail(e, "cudaMalloc");
	if ((e = cudaMalloc(&b->d_blk, sizeof(int) * (2 * xp.size() + 2 * yp.size()))) != cudaSuccess) return bfail(e, "cudaMalloc");
	cudaMemcpy(b->d_xargs, xa.data(), sizeof(XArgs<T>) * n, cudaMemcpyHostToDevice);
	cudaMemcpy(b->d_yargs, ya.data(), sizeof(YArgs<T>) * n, cudaMemcpyHostToDevice);
	b->hargs.resize(sizeof(XArgs<T>) * n + sizeof(YArgs<T>) * n);
	memcpy(b->hargs.data(), xa.data(), sizeof(XArgs<T>) * n);
	memcpy(b->hargs.data() + sizeof(XArgs<T>) * n, ya.data(), sizeof(YArgs<T>) * n);
	int* q = b->d_blk;
	cudaMemcpy(q, xp.data(), sizeof(int) * xp.size(), cudaMemcpyHostToDevice);
	cudaMemcpy(q + xp.size(), xl.data(), sizeof(int) * xl.size(), cudaMemcpyHostToDevice);
	cudaMemcpy(q + 2 * xp.size(), yp.data(), sizeof(int) * yp.size(), cudaMemcpyHostToDevice);
	if ((e = cudaMemcpy(q + 2 * xp.size() + yp.size(), yl.data(), sizeof(int) * yl.size(), cudaMemcpyHostToDevice)) !=
	    cudaSuccess)
		return bfail(e, "cudaMemcpy");
	return 0;
}

// nsteps steps of every class, each class a chain on its own stream forked
// from and joined back into the batch stream (which is capturing a graph).
template <typename T> int batch_launch_steps(pfcg_batch* b, int nsteps) {
	const int* q = b->d_blk;
	const int* xp = q;
	const int* xl = q + b->xblocks;
	const int* yp = q + 2 * b->xblocks;
	const int* yl = yp + b->yblocks;
	cudaError_t e = cudaEventRecord(b->fork, b->stream);
	for (BatchClass& k : b->cls) {
		if (e == cudaSuccess) e = cudaStreamWaitEvent(k.stream, b->fork, 0);
		for (int s = 0; s < nsteps && e == cudaSuccess; s++) {
			if (k.ct) {
				e = launch_ct_batch<T>(0, k.U, k.N, b->d_xargs, xp + k.xoff, xl + k.xoff, k.xn, k.cx, k.stream);
				if (e == cudaSuccess)
					e = launch_ct_batch<T>(1, k.U, k.N, b->d_yargs, yp + k.yoff, yl + k.yoff, k.yn, k.cy, k.stream);
			} else {
				e = launch_generic_batch<T>(0, b->d_xargs, xp + k.xoff, xl + k.xoff, k.xn, k.threads, k.smem, k.stream);
				if (e == cudaSuccess)
					e = launch_generic_batch<T>(1, b->d_yargs, yp + k.yoff, yl + k.yoff, k.yn, k.threads, k.smem, k.stream);
			}
		}
		// joined even after an error, so that the capture can end
		cudaEventRecord(k.done, k.stream);
		cudaStreamWaitEvent(b->stream, k.done, 0);
	}
	if (e != cudaSuccess) {
		b->err = std::string("batch step: ") + cudaGetErrorString(e);
		return PFCG_ECUDA;
	}
	return 0;
}

} // namespace

extern "C" {

int pfcg_batch_create(int nprob, const pfcg_params* params, const int* Nx, const int* Ny, const double* dx,
                      const double* dy, pfcg_prec prec, int autotune, pfcg_batch** out) {
	if (!out || nprob < 1 || !params || !Nx || !Ny || !dx || !dy) return fail(nullptr, PFCG_EARG, "bad argument");
	*out = nullptr;
	pfcg_batch* b = new pfcg_batch();
	b->prec = prec;
	auto bail = [&](int rc) {
		if (!b->err.empty()) g_err = b->err;
		pfcg_batch_destroy(b);
		return rc;
	};
	for (int i = 0; i < nprob; i++) {
		pfcg_handle* h = nullptr;
		const int rc = pfcg_create(&params[i], Nx[i], Ny[i], dx[i], dy[i], prec, &h);
		if (rc) return bail(rc);
		b->h.push_back(h);
		// sizes with specialised kernels run them in their fixed shape; the
		// others run the runtime-plan kernels, in the shape the autotuner picks
		if (batch_ct(h)) continue;
		h->cxs = h->cx;
		h->cys = h->cy;
		if (autotune) {
			const int r2 = pfcg_autotune(h, 5);
			if (r2) {
				b->err = h->err;
				return bail(r2);
			}
		}
	}
	cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
	if (e == cudaSuccess) e = cudaMalloc(&b->d_flags, sizeof(int) * nprob);
	if (e == cudaSuccess) e = cudaMemset(b->d_flags, 0, sizeof(int) * nprob);
	if (e == cudaSuccess) e = cudaMallocHost(&b->h_flags, sizeof(int) * nprob);
	if (e != cudaSuccess) {
		b->err = cudaGetErrorString(e);
		return bail(PFCG_ECUDA);
	}
	const int rc = prec == PFCG_FP64 ? batch_build<double>(b) : batch_build<float>(b);
	if (rc) return bail(rc);
	*out = b;
	return 0;
}

pfcg_handle* pfcg_batch_problem(pfcg_batch* b, int i) {
	if (!b || i < 0 || i >= (int)b->h.size()) return nullptr;
	return b->h[i];
}

int pfcg_batch_step(pfcg_batch* b, int nsteps) {
	if (!b || nsteps < 0) return fail(nullptr, PFCG_EARG, "bad argument");
	if (nsteps == 0) return 0;
	// every problem's own stream must be idle (uploads are synchronous)
	auto it = b->graphs.find(nsteps);
	if (it == b->graphs.end()) {
		cudaGraph_t g;
		cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
		if (e != cudaSuccess) { b->err = cudaGetErrorString(e); g_err = b->err; return PFCG_ECUDA; }
		const int rc = b->prec == PFCG_FP64 ? batch_launch_steps<double>(b, nsteps) : batch_launch_steps<float>(b, nsteps);
		e = cudaStreamEndCapture(b->stream, &g);
		if (rc) { g_err = b->err; return rc; }
		if (e != cudaSuccess) { b->err = cudaGetErrorString(e); g_err = b->err; return PFCG_ECUDA; }
		cudaGraphExec_t ge;
		e = cudaGraphInstantiate(&ge, g, 0);
		cudaGraphDestroy(g);
		if (e != cudaSuccess) { b->err = cudaGetErrorString(e); g_err = b->err; return PFCG_ECUDA; }
		it = b->graphs.emplace(nsteps, ge).first;
	}
	const int ra = b->prec == PFCG_FP64 ? batch_refresh_args<double>(b) : batch_refresh_args<float>(b);
	if (ra) { g_err = b->err; return ra; }
	cudaError_t e = cudaGraphLaunch(it->second, b->stream);
	const int n = (int)b->h.size();
	if (e == cudaSuccess) e = cudaMemcpyAsync(b->h_flags, b->d_flags, sizeof(int) * n, cudaMemcpyDeviceToHost, b->stream);
	if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
	if (e != cudaSuccess) { b->err = cudaGetErrorString(e); g_err = b->err; return PFCG_ECUDA; }
	for (pfcg_handle* h : b->h) {
		h->t += nsteps;
		h->launches += 2 * nsteps;
	}
	for (int i = 0; i < n; i++)
		if (b->h_flags[i] & FLAG_TIMEOUT) {
			g_err = "a bounded device-side wait ran out (y-pass TMA load)";
			return PFCG_ETIMEOUT;
		}
	for (int i = 0; i < n; i++)
		if (b->h_flags[i]) { g_err = "Not a number value detected."; return PFCG_NAN; }
	return 0;
}

int pfcg_batch_stream(const pfcg_batch* b, void** stream) {
	if (!b || !stream) return PFCG_EARG;
	*stream = (void*)b->stream;
	return 0;
}

int pfcg_batch_launches(const pfcg_batch* b, int nsteps, long long* kernels, long long* graph_launches) {
	if (!b) return PFCG_EARG;
	if (kernels) *kernels = 2LL * nsteps * (long long)b->cls.size();
	if (graph_launches) *graph_launches = 1;
	return 0;
}

void pfcg_batch_destroy(pfcg_batch* b) {
	if (!b) return;
	if (b->stream) cudaStreamSynchronize(b->stream);
	for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
	for (pfcg_handle* h : b->h) pfcg_destroy(h);
	for (BatchClass& k : b->cls) {
		if (k.stream) cudaStreamDestroy(k.stream);
		if (k.done) cudaEventDestroy(k.done);
	}
	if (b->fork) cudaEventDestroy(b->fork);
	cudaFree(b->d_xargs);
	cudaFree(b->d_yargs);
	cudaFree(b->d_blk);
	cudaFree(b->d_flags);
	if (b->h_flags) cudaFreeHost(b->h_flags);
	if (b->stream) cudaStreamDestroy(b->stream);
	delete b;
}

} // extern "C"

// --------------------------------------------------------------- no-alloc ---
// pfcg_relax_noalloc: a whole relaxation call (upload, steps, download) whose
// device workspace lives in the file-scope array below instead of cudaMalloc'd
// memory. Every GPU that loads this library holds the array until the process
// exits. In host code g_noalloc_scratch names a host-side stand-in, not device
// memory: every call looks up its device address on the current device with
// cudaGetSymbolAddress (a host-side query that allocates nothing), so no
// address is cached across calls, contexts or host threads.

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[PFCG_NOALLOC_SCRATCH_BYTES];

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

// exp(-2 pi i k / n) in FP32 from a double-precision sincospi
__global__ void noalloc_twiddles_kernel(float2* tw, int n) {
	for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		double sn, cs;
		sincospi(-2.0 * (double)k / (double)n, &sn, &cs);
		tw[k] = make_float2((float)cs, (float)sn);
	}
}

// workspace bytes a call of this size needs (FP32 transforms)
size_t noalloc_bytes(int U, int Nx, int Ny) {
	const size_t nspec = (size_t)(Nx / 2 + 1) * Ny;
	return 2 * align256(sizeof(float2) * nspec * U)       // spectral state, mixed workspace
	       + align256(sizeof(double) * MAXU)               // means
	       + align256(sizeof(double) * ACC_N)              // accumulators
	       + align256(sizeof(int))                         // NaN flag
	       + align256(sizeof(double) * MAXU * MEAN_BLOCKS) // partial sums of the means
	       + align256(sizeof(double) * MAXU * Ny)          // per-tile sums of the nonlinear term
	       + align256(sizeof(float2) * Nx) + align256(sizeof(float2) * Ny);
}

} // namespace

extern "C" int pfcg_relax_noalloc(const pfcg_params* p, int Nx, int Ny, double dx, double dy, int nsteps, double* fields,
                                  void* stream) {
	if (!p || !fields || nsteps < 0) return fail(nullptr, PFCG_EARG, "NULL argument or negative step count");
	if (p->U < 1 || p->U > PFCG_MAX_U) return fail(nullptr, PFCG_EARG, "U out of range 1..4");
	for (int u = 0; u < p->U; u++)
		if (p->W[u] < 0 || p->W[u] > PFCG_MAX_W) return fail(nullptr, PFCG_EARG, "W[u] out of range 0..4");
	if (!pfcg_size_supported(Nx, Ny))
		return fail(nullptr, PFCG_ESIZE, "grid size not supported (need even 8..8192 with factors 2,3,5,7)");
	const size_t need = noalloc_bytes(p->U, Nx, Ny);
	if (need > (size_t)PFCG_NOALLOC_SCRATCH_BYTES)
		return fail(nullptr, PFCG_ESIZE,
		            "grid too large for pfcg_relax_noalloc: needs " + std::to_string(need) + " bytes of its " +
		                std::to_string((size_t)PFCG_NOALLOC_SCRATCH_BYTES) + "-byte static workspace");
	int dev = 0;
	cudaError_t e = cudaGetDevice(&dev);
	if (e != cudaSuccess) return fail(nullptr, PFCG_ENODEV, cudaGetErrorString(e));
	cudaDeviceProp prop;
	e = cudaGetDeviceProperties(&prop, dev);
	if (e != cudaSuccess) return fail(nullptr, PFCG_ENODEV, cudaGetErrorString(e));
	if (prop.major != 10) return fail(nullptr, PFCG_ENODEV, "libpfc_b200 is built for sm_100a (B200) only");
	// the array's address on the current device, looked up on every call
	void* scratch = nullptr;
	e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
	if (e != cudaSuccess || !scratch)
		return fail(nullptr, PFCG_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));

	// host-side description of the relaxation; no device memory is allocated
	pfcg_handle h;
	h.dev = dev;
	h.prec = PFCG_FP32;
	h.model = to_model(p);
	h.U = p->U;
	h.Nx = Nx;
	h.Ny = Ny;
	h.H = Nx / 2 + 1;
	h.geom.Nx = Nx;
	h.geom.Ny = Ny;
	h.geom.H = h.H;
	h.geom.dx = dx;
	h.geom.dy = dy;
	set_dk(&h);
	h.celem = sizeof(float2);
	h.stream = (cudaStream_t)stream;
	int rc = 0;
	if (!make_plan(Nx, max_radix(false), &h.px) || !make_plan(Ny, max_radix(false), &h.py))
		rc = fail(&h, PFCG_ESIZE, "bad factorisation");
	if (!rc) rc = choose_layout(&h, prop.multiProcessorCount);
	if (rc) return fail(nullptr, rc, h.err);
	// the runtime-plan STEP kernels (the specialised ones need per-pass tables)
	h.cxs = h.cx;
	h.cys = h.cy;

	unsigned char* base = (unsigned char*)scratch;
	const size_t nspec = (size_t)h.H * Ny;
	size_t off = 0;
	auto carve = [&](size_t bytes) {
		void* q = base + off;
		off += align256(bytes);
		return q;
	};
	h.spec = carve(sizeof(float2) * nspec * h.U);
	h.work = carve(sizeof(float2) * nspec * h.U);
	h.mean = (double*)carve(sizeof(double) * MAXU);
	h.acc = (double*)carve(sizeof(double) * ACC_N);
	h.flag = (int*)carve(sizeof(int));
	h.d_part = (double*)carve(sizeof(double) * MAXU * MEAN_BLOCKS);
	h.nlpart = (double*)carve(sizeof(double) * MAXU * Ny);
	h.twx = carve(sizeof(float2) * Nx);
	h.twy = carve(sizeof(float2) * Ny);
	h.d_real = fields; // the caller's buffer is both input and output

	auto done = [&](int code) {
		// the handle's pointers are views of the static workspace: nothing to free
		h.spec = h.work = h.twx = h.twy = nullptr;
		h.mean = h.acc = h.d_part = h.nlpart = nullptr;
		h.flag = nullptr;
		h.d_real = nullptr;
		return code ? fail(nullptr, code, h.err) : 0;
	};
#define CKN(call)                                                                                                      \
	do {                                                                                                           \
		cudaError_t e_ = (call);                                                                               \
		if (e_ != cudaSuccess) return done(cuda_fail(&h, #call, e_));                                          \
	} while (0)

	// the workspace keeps the previous call's contents: clear what must start at zero
	CKN(cudaMemsetAsync(h.acc, 0, sizeof(double) * ACC_N, h.stream));
	CKN(cudaMemsetAsync(h.flag, 0, sizeof(int), h.stream));
	noalloc_twiddles_kernel<<<(Nx + 255) / 256, 256, 0, h.stream>>>((float2*)h.twx, Nx);
	CKN(cudaGetLastError());
	noalloc_twiddles_kernel<<<(Ny + 255) / 256, 256, 0, h.stream>>>((float2*)h.twy, Ny);
	CKN(cudaGetLastError());

	// upload (means, r2c along x, FFT along y), steps, download
	CKN(launch_field_means(fields, h.U, (long long)Nx * Ny, h.d_part, MEAN_BLOCKS, h.mean, h.stream));
	XArgs<float> xa = xargs<float>(&h);
	YArgs<float> ya = yargs<float>(&h);
	if ((rc = run_xpass<float>(&h, XP_R2C, xa, h.cx))) return done(rc);
	if ((rc = run_ypass<float>(&h, YP_INIT, ya, h.cy))) return done(rc);
	xa.acc = h.acc + ACC_NL;
	for (int s = 0; s < nsteps; s++) {
		if ((rc = run_xpass<float>(&h, XP_STEP, xa, h.cxs))) return done(rc);
		if ((rc = run_ypass<float>(&h, YP_STEP, ya, h.cys))) return done(rc);
	}
	xa.acc = h.acc;
	if ((rc = run_xpass<float>(&h, XP_C2R, xa, h.cx))) return done(rc);
	int nan = 0;
	CKN(cudaMemcpyAsync(&nan, h.flag, sizeof(int), cudaMemcpyDeviceToHost, h.stream));
	CKN(cudaStreamSynchronize(h.stream));
#undef CKN
	if (nan) {
		h.err = "Not a number value detected.";
		return done(PFCG_NAN);
	}
	return done(0);
}
