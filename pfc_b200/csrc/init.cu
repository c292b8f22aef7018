// Seeded two-field heterostructure initial states, generated on the device.
//
// Restates the one-mode approximation (src/PFCInit.java:46-66, OMA) and the
// periodic nearest-centre Voronoi assignment (src/PFCInit.java:68-93 closest,
// :389-462 the "V" step) of the reference's initial-state builder for two
// density fields: each region (a Voronoi grain, or a vertical stripe) belongs
// to one field, which carries mean + amp * OMA(r rotated by the grain's angle)
// there; the other field sits at its mean. White noise is added to both.
// Random numbers are counter based (splitmix64 finaliser of seed, stream and
// index; Box-Muller normals over consecutive word pairs), so every value
// depends only on (seed, stream, index): grain k takes uniforms 4k..4k+3 of
// stream 1 (x, y, angle, field), the noise of field u is stream 3 + u at the
// point's y-major index. Distances and rotations use explicitly rounded FP64
// operations so that region labels match a restatement with the same
// operation order bit for bit.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/pfc_b200.h"

namespace {

constexpr double PI = 3.141592653589793238462643383279502884;
constexpr double TWO53_INV = 1.0 / 9007199254740992.0;

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
	unsigned long long z = x + 0x9E3779B97F4A7C15ull;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}

__device__ __forceinline__ unsigned long long rng_key(unsigned seed, int stream) {
	return ((unsigned long long)(seed & 0xFFFFFFu) << 32) + ((unsigned long long)(stream & 0xFF) << 56);
}

__device__ __forceinline__ double uniform01(unsigned long long key, unsigned long long k) {
	return (double)(splitmix64(key + k) >> 11) * TWO53_INV;
}

__device__ __forceinline__ double normal01(unsigned long long key, unsigned long long k) {
	const unsigned long long a = splitmix64(key + 2 * k), b = splitmix64(key + 2 * k + 1);
	const double u1 = ((double)(a >> 11) + 1.0) * TWO53_INV;
	const double u2 = (double)(b >> 11) * TWO53_INV;
	return sqrt(-2.0 * log(u1)) * cos(2.0 * PI * u2);
}

__device__ double oma(double x, double y, int sym, double a) {
	const double q = 2.0 * PI / a;
	if (sym == 4) return cos(q * x) * cos(q * y);
	const double qx = q, qy = q / sqrt(3.0);
	if (sym == 3) return cos(qx * x) * cos(qy * y) + 0.5 * cos(2.0 * qy * y);
	return -2.0 * cos(qx * x - qy * y) - 2.0 * cos(2.0 * qy * y) - 2.0 * cos(-qx * x - qy * y) +
	       cos(-qx * x - 3.0 * qy * y) + cos(2.0 * qx * x) + cos(-qx * x + 3.0 * qy * y);
}

// periodic minimum image of d in a box of length W
__device__ __forceinline__ double wrap(double d, double W) {
	return d > 0.5 * W ? __dsub_rn(d, W) : (d < -0.5 * W ? __dadd_rn(d, W) : d);
}

__global__ void hetero_kernel(double* __restrict__ out, int Nx, int Ny, double dx, double dy, pfcg_hetero s,
                              double angle_scale) {
	const long long n = (long long)Nx * Ny;
	const unsigned long long kg = rng_key(s.seed, 1);
	const double W = __dmul_rn((double)Nx, dx), H = __dmul_rn((double)Ny, dy);
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
		const int j = (int)(t / Nx), i = (int)(t - (long long)j * Nx);
		const double X = __dmul_rn((double)i, dx), Y = __dmul_rn((double)j, dy);
		int phase;
		double xr = X, yr = Y;
		if (s.grains <= 0) {
			phase = ((i + s.stripe_offset) / s.stripe_width) & 1;
		} else {
			double best = INFINITY;
			int lab = 0;
			for (int g = 0; g < s.grains; g++) {
				const double cx = __dmul_rn(__dmul_rn(uniform01(kg, 4ull * g), (double)Nx), dx);
				const double cy = __dmul_rn(__dmul_rn(uniform01(kg, 4ull * g + 1), (double)Ny), dy);
				const double ddx = wrap(__dsub_rn(X, cx), W), ddy = wrap(__dsub_rn(Y, cy), H);
				const double d2 = __dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy));
				if (d2 < best) {
					best = d2;
					lab = g;
				}
			}
			const double theta = __dmul_rn(uniform01(kg, 4ull * lab + 2), angle_scale);
			phase = uniform01(kg, 4ull * lab + 3) >= 0.5 ? 1 : 0;
			const double c = cos(-theta), sn = sin(-theta);
			xr = __dsub_rn(__dmul_rn(X, c), __dmul_rn(Y, sn));
			yr = __dadd_rn(__dmul_rn(X, sn), __dmul_rn(Y, c));
		}
		for (int u = 0; u < 2; u++) {
			double v = s.mean[u];
			if (phase == u) v = s.mean[u] + s.amp[u] * oma(xr, yr, s.sym, s.lattice[u]);
			if (s.noise != 0.0) v += s.noise * normal01(rng_key(s.seed, 3 + u), (unsigned long long)t);
			out[(long long)u * n + t] = v;
		}
	}
}

// ------------------------------------------------------------------ V step --
// The reference builder's Voronoi step (src/PFCInit.java:389-462) for one
// density field: every point takes the periodic-nearest grain centre
// (closest(), :68-93, first minimum wins); a phantom grain (type 2) leaves the
// point alone, otherwise the point becomes type * old + nave + amp * OMA(r') +
// 2 namp (U - 0.5), with r' the point moved by -(tx2 + xr, ty2 + yr), rotated
// by -theta, moved by (xr - tx1, yr - ty1) (:448-456). Arithmetic follows the
// Java expressions' order with explicit FP64 roundings (no contraction), so
// only the cosines can differ from the JVM's in the last bit.
//
// U is java.util.Random.nextDouble() (the Java API documentation's generator:
// 48-bit linear congruential x' = 0x5DEECE66D x + 11 mod 2^48, next(b) = the top
// b bits, nextDouble = (next(26) 2^27 + next(27)) 2^-53), drawn once per
// non-phantom point in row-major order whatever namp is, as the Java loop
// does. Point p's draw is number 2 c(p) of the sequence, c(p) the count of
// non-phantom points before it (a prefix sum); the state is jumped there by
// the LCG's closed form (repeated squaring of the affine map).

constexpr unsigned long long LCG_A = 0x5DEECE66Dull, LCG_C = 0xBull, LCG_MASK = (1ull << 48) - 1;

// state advanced by n steps: x_n = A^n x + C (A^n - 1)/(A - 1), by squaring
__host__ __device__ inline unsigned long long lcg_jump(unsigned long long x, unsigned long long n) {
	unsigned long long a = LCG_A, c = LCG_C, A = 1, C = 0;
	while (n) {
		if (n & 1) {
			A = (A * a) & LCG_MASK;
			C = (C * a + c) & LCG_MASK;
		}
		c = ((a + 1) * c) & LCG_MASK;
		a = (a * a) & LCG_MASK;
		n >>= 1;
	}
	return (A * x + C) & LCG_MASK;
}

__device__ __forceinline__ double java_next_double(unsigned long long& x) {
	x = (x * LCG_A + LCG_C) & LCG_MASK;
	const unsigned long long hi = x >> (48 - 26);
	x = (x * LCG_A + LCG_C) & LCG_MASK;
	const unsigned long long lo = x >> (48 - 27);
	return (double)((hi << 27) + lo) * (1.0 / 9007199254740992.0);
}

// OMA of src/PFCInit.java:46-66 with the Java expression's roundings
__device__ double oma_java(double x, double y, int sym, double a) {
	const double q = __ddiv_rn(2.0 * PI, a);
	if (sym == 4) return __dmul_rn(cos(__dmul_rn(q, x)), cos(__dmul_rn(q, y)));
	const double qx = q, qy = __ddiv_rn(q, sqrt(3.0));
	if (sym == 3)
		return __dadd_rn(__dmul_rn(cos(__dmul_rn(qx, x)), cos(__dmul_rn(qy, y))),
		                 __dmul_rn(0.5, cos(__dmul_rn(__dmul_rn(2.0, qy), y))));
	const double qxx = __dmul_rn(qx, x), qyy = __dmul_rn(qy, y);
	double r = __dmul_rn(-2.0, cos(__dsub_rn(qxx, qyy)));
	r = __dsub_rn(r, __dmul_rn(2.0, cos(__dmul_rn(__dmul_rn(2.0, qy), y))));
	r = __dsub_rn(r, __dmul_rn(2.0, cos(__dsub_rn(-qxx, qyy))));
	r = __dadd_rn(r, cos(__dsub_rn(-qxx, __dmul_rn(__dmul_rn(3.0, qy), y))));
	r = __dadd_rn(r, cos(__dmul_rn(__dmul_rn(2.0, qx), x)));
	r = __dadd_rn(r, cos(__dadd_rn(-qxx, __dmul_rn(__dmul_rn(3.0, qy), y))));
	return r;
}

struct GrainDev {
	double x, y, a, nave, amp, namp, tx1, ty1, theta, xr, yr, tx2, ty2;
	int type, sym;
};

// pass 1: nearest grain of every point and whether it draws a random number
__global__ void voronoi_label_kernel(const GrainDev* __restrict__ g, int ng, int Nx, int Ny, double dx, double dy,
                                     int* __restrict__ label, unsigned* __restrict__ draws) {
	const long long n = (long long)Nx * Ny;
	const double W = __dmul_rn((double)Nx, dx), H = __dmul_rn((double)Ny, dy);
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
		const int j = (int)(t / Nx), i = (int)(t - (long long)j * Nx);
		const double u = __dmul_rn((double)i, dx), v = __dmul_rn((double)j, dy);
		int best = 0;
		double d2 = 0.0;
		for (int m = 0; m < ng; m++) {
			double ddx = __dsub_rn(u, g[m].x);
			if (ddx > 0.5 * W) ddx = __dsub_rn(ddx, W);
			else if (ddx < -0.5 * W) ddx = __dadd_rn(ddx, W);
			double ddy = __dsub_rn(v, g[m].y);
			if (ddy > 0.5 * H) ddy = __dsub_rn(ddy, H);
			else if (ddy < -0.5 * H) ddy = __dadd_rn(ddy, H);
			const double e = __dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy));
			if (m == 0 || e < d2) {
				best = m;
				d2 = e;
			}
		}
		label[t] = best;
		draws[t] = g[best].type == 2 ? 0u : 1u;
	}
}

// exclusive prefix sum of draws in place, per block of SCAN_B points, block totals to tot
constexpr int SCAN_T = 256, SCAN_PER = 16, SCAN_B = SCAN_T * SCAN_PER;
__global__ void __launch_bounds__(SCAN_T) scan_block_kernel(unsigned* __restrict__ v, long long n,
                                                            unsigned long long* __restrict__ tot) {
	__shared__ unsigned long long part[SCAN_T];
	const long long base = (long long)blockIdx.x * SCAN_B + (long long)threadIdx.x * SCAN_PER;
	unsigned loc[SCAN_PER];
	unsigned long long s = 0;
	for (int k = 0; k < SCAN_PER; k++) {
		loc[k] = base + k < n ? v[base + k] : 0u;
		s += loc[k];
	}
	part[threadIdx.x] = s;
	__syncthreads();
	for (int o = 1; o < SCAN_T; o <<= 1) {
		const unsigned long long add = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0ull;
		__syncthreads();
		part[threadIdx.x] += add;
		__syncthreads();
	}
	unsigned long long run = part[threadIdx.x] - s;
	for (int k = 0; k < SCAN_PER; k++) {
		if (base + k < n) v[base + k] = (unsigned)run;
		run += loc[k];
	}
	if (threadIdx.x == SCAN_T - 1) tot[blockIdx.x] = part[SCAN_T - 1];
}

// pass 2: the grain value of every non-phantom point
__global__ void voronoi_value_kernel(double* __restrict__ out, const GrainDev* __restrict__ g, int Nx, int Ny,
                                     double dx, double dy, const int* __restrict__ label,
                                     const unsigned* __restrict__ draws, const unsigned long long* __restrict__ boff,
                                     unsigned long long rng) {
	const long long n = (long long)Nx * Ny;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
		const GrainDev& q = g[label[t]];
		if (q.type == 2) continue;
		const int j = (int)(t / Nx), i = (int)(t - (long long)j * Nx);
		const double u = __dsub_rn(__dsub_rn(__dmul_rn((double)i, dx), q.tx2), q.xr);
		const double v = __dsub_rn(__dsub_rn(__dmul_rn((double)j, dy), q.ty2), q.yr);
		const double sn = sin(-q.theta), cs = cos(-q.theta);
		const double rx = __dsub_rn(__dadd_rn(__dsub_rn(__dmul_rn(u, cs), __dmul_rn(v, sn)), q.xr), q.tx1);
		const double ry = __dsub_rn(__dadd_rn(__dadd_rn(__dmul_rn(u, sn), __dmul_rn(v, cs)), q.yr), q.ty1);
		unsigned long long x = lcg_jump(rng, 2ull * (boff[t / SCAN_B] + draws[t]));
		const double U = java_next_double(x);
		double r = __dadd_rn(__dmul_rn((double)q.type, out[t]), q.nave);
		r = __dadd_rn(r, __dmul_rn(q.amp, oma_java(rx, ry, q.sym, q.a)));
		r = __dadd_rn(r, __dmul_rn(__dmul_rn(2.0, q.namp), __dsub_rn(U, 0.5)));
		out[t] = r;
	}
}

thread_local std::string g_init_err;

} // namespace

extern "C" {

int pfcg_init_hetero(double* d_fields, int Nx, int Ny, double dx, double dy, const pfcg_hetero* s, void* stream) {
	if (!d_fields || !s) {
		g_init_err = "NULL argument";
		return PFCG_EARG;
	}
	if (Nx < 1 || Ny < 1 || (s->grains <= 0 && (s->stripe_width < 1 || s->stripe_offset < 0)) || s->grains > 4096 ||
	    (s->sym != 3 && s->sym != 4 && s->sym != 6)) {
		g_init_err = "invalid grid, stripe width or offset, grain count or symmetry";
		return PFCG_EARG;
	}
	const double angle_scale = s->max_angle_deg * (PI / 180.0);
	cudaStream_t st = (cudaStream_t)stream;
	const long long n = (long long)Nx * Ny;
	const int grid = (int)((n + 255) / 256 > 148 * 8 ? 148 * 8 : (n + 255) / 256);
	hetero_kernel<<<grid, 256, 0, st>>>(d_fields, Nx, Ny, dx, dy, *s, angle_scale);
	cudaError_t e = cudaGetLastError();
	if (e == cudaSuccess) e = cudaStreamSynchronize(st);
	if (e != cudaSuccess) {
		g_init_err = std::string("hetero_kernel: ") + cudaGetErrorString(e);
		return PFCG_ECUDA;
	}
	return 0;
}

int pfcg_init_voronoi(double* d_field, int Nx, int Ny, double dx, double dy, int ngrains, const pfcg_grain* grains,
                      long long* rng, void* stream) {
	if (!d_field || !grains || !rng || Nx < 1 || Ny < 1 || ngrains < 1 || ngrains > (1 << 20)) {
		g_init_err = "NULL argument or empty grid / grain list";
		return PFCG_EARG;
	}
	const long long n = (long long)Nx * Ny;
	if (n > 0xFFFFFFFFll) {
		g_init_err = "grid too large";
		return PFCG_EARG;
	}
	const double W = (double)Nx * dx, H = (double)Ny * dy;
	std::vector<GrainDev> g(ngrains);
	for (int k = 0; k < ngrains; k++) {
		const pfcg_grain& s = grains[k];
		if (s.sym != 3 && s.sym != 4 && s.sym != 6) {
			g_init_err = "grain symmetry must be 3, 4 or 6";
			return PFCG_EARG;
		}
		GrainDev& d = g[k];
		// centres wrapped into the box as w(double, double) does (src/PFCInit.java:40-44)
		double x = s.x, y = s.y;
		while (x < 0) x += W;
		while (x >= W) x -= W;
		while (y < 0) y += H;
		while (y >= H) y -= H;
		d.x = x;
		d.y = y;
		d.type = (s.type < 0 || s.type > 2) ? 0 : s.type; // the reference's "defaulting to overwrite"
		d.sym = s.sym;
		d.a = s.a;
		d.nave = s.nave;
		d.amp = s.amp;
		d.namp = s.namp;
		d.tx1 = s.tx1;
		d.ty1 = s.ty1;
		d.theta = s.theta_deg / 180.0 * PI;
		d.xr = s.xr;
		d.yr = s.yr;
		d.tx2 = s.tx2;
		d.ty2 = s.ty2;
	}
	cudaStream_t st = (cudaStream_t)stream;
	const long long nb = (n + SCAN_B - 1) / SCAN_B;
	// a host field goes through a device copy
	cudaPointerAttributes pa;
	const bool on_dev = cudaPointerGetAttributes(&pa, d_field) == cudaSuccess &&
	                    (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged);
	cudaGetLastError();
	double* host_field = on_dev ? nullptr : d_field;
	if (!on_dev) {
		d_field = nullptr;
		cudaError_t ea = cudaMalloc(&d_field, sizeof(double) * n);
		if (ea == cudaSuccess) ea = cudaMemcpyAsync(d_field, host_field, sizeof(double) * n, cudaMemcpyHostToDevice, st);
		if (ea != cudaSuccess) {
			cudaFree(d_field);
			g_init_err = std::string("pfcg_init_voronoi: ") + cudaGetErrorString(ea);
			return PFCG_ECUDA;
		}
	}
	GrainDev* dg = nullptr;
	int* label = nullptr;
	unsigned* draws = nullptr;
	unsigned long long* tot = nullptr;
	cudaError_t e = cudaMalloc(&dg, sizeof(GrainDev) * ngrains);
	if (e == cudaSuccess) e = cudaMalloc(&label, sizeof(int) * n);
	if (e == cudaSuccess) e = cudaMalloc(&draws, sizeof(unsigned) * n);
	if (e == cudaSuccess) e = cudaMalloc(&tot, sizeof(unsigned long long) * nb);
	std::vector<unsigned long long> htot(nb);
	if (e == cudaSuccess) e = cudaMemcpyAsync(dg, g.data(), sizeof(GrainDev) * ngrains, cudaMemcpyHostToDevice, st);
	const int grid = (int)((n + 255) / 256 > 148 * 8 ? 148 * 8 : (n + 255) / 256);
	if (e == cudaSuccess) {
		voronoi_label_kernel<<<grid, 256, 0, st>>>(dg, ngrains, Nx, Ny, dx, dy, label, draws);
		e = cudaGetLastError();
	}
	if (e == cudaSuccess) {
		scan_block_kernel<<<(unsigned)nb, SCAN_T, 0, st>>>(draws, n, tot);
		e = cudaGetLastError();
	}
	// block offsets: the exclusive sum of the block totals, on the host (n / 4096 values)
	if (e == cudaSuccess) e = cudaMemcpyAsync(htot.data(), tot, sizeof(unsigned long long) * nb, cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess) e = cudaStreamSynchronize(st);
	unsigned long long total = 0;
	if (e == cudaSuccess) {
		for (long long b = 0; b < nb; b++) {
			const unsigned long long c = htot[b];
			htot[b] = total;
			total += c;
		}
		e = cudaMemcpyAsync(tot, htot.data(), sizeof(unsigned long long) * nb, cudaMemcpyHostToDevice, st);
	}
	const unsigned long long r0 = (unsigned long long)*rng & LCG_MASK;
	if (e == cudaSuccess) {
		voronoi_value_kernel<<<grid, 256, 0, st>>>(d_field, dg, Nx, Ny, dx, dy, label, draws, tot, r0);
		e = cudaGetLastError();
	}
	if (e == cudaSuccess && host_field)
		e = cudaMemcpyAsync(host_field, d_field, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess) e = cudaStreamSynchronize(st);
	if (host_field) cudaFree(d_field);
	cudaFree(dg);
	cudaFree(label);
	cudaFree(draws);
	cudaFree(tot);
	if (e != cudaSuccess) {
		g_init_err = std::string("pfcg_init_voronoi: ") + cudaGetErrorString(e);
		return PFCG_ECUDA;
	}
	*rng = (long long)lcg_jump(r0, 2ull * total);
	return 0;
}

long long pfcg_java_random_seed(long long seed) { return (long long)(((unsigned long long)seed ^ LCG_A) & LCG_MASK); }

const char* pfcg_init_last_error(void) { return g_init_err.c_str(); }

} // extern "C"
