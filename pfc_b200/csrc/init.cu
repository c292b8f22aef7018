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

const char* pfcg_init_last_error(void) { return g_init_err.c_str(); }

} // extern "C"
