// Precision-independent kernels and helpers of the B200 relaxation path.
#include "kernels_impl.cuh"

namespace pfcg {

int max_elems_per_thread(bool fp64) { (void)fp64; return RT_MAXE; }
int max_radix(bool fp64) { (void)fp64; return RT_MAXE; }
int ct_radix(bool fp64, int N) { return fp64 ? ct_maxe<double>(N) : ct_maxe<float>(N); }

// 0 where the size has no specialised kernel (Spec in kernels_impl.cuh)
int spec_rows(bool fp64, int U, int N) { return fp64 ? Spec<double>::xr(U, N) : Spec<float>::xr(U, N); }
int spec_cols(bool fp64, int U, int N) { return fp64 ? Spec<double>::ycc(U, N) : Spec<float>::ycc(U, N); }

template <typename T> static int ct_twn(int N) {
	constexpr int M = FftCfg<T>::MAXE;
	switch (N) {
	case 4096: return CtPlan<4096, M>::TWN;
	case 2048: return CtPlan<2048, M>::TWN;
	}
	if constexpr (M == 16) {
		switch (N) {
		case 384: return CtPlan<384, ct_maxe<T>(384)>::TWN;
		case 1536: return CtPlan<1536, M>::TWN;
		case 1024: return CtPlan<1024, M>::TWN;
		case 768: return CtPlan<768, M>::TWN;
		case 512: return CtPlan<512, M>::TWN;
		case 256: return CtPlan<256, M>::TWN;
		}
	}
	return 0;
}
int spec_twiddles(bool fp64, int N) { return fp64 ? ct_twn<double>(N) : ct_twn<float>(N); }

// whether the specialised y-pass (not the register-fused variant) of this
// shape takes its first transform's input straight from memory (register
// ends, the path that can load by TMA)
template <typename T, int U, int N> static bool y_regio() {
	constexpr int CC = Spec<T>::ycc(U, N), R = Spec<T>::xr(U, N);
	using C = YCfg<T, U, N, CC, R, false>;
	constexpr int M = C::MAXE;
	return C::NSUB == C::S && C::S * (N / M) == C::NT && CtPlan<N, M>::FUSABLE;
}
template <typename T, int U> static bool y_regio_n(int N) {
	switch (N) {
	case 4096: return y_regio<T, U, 4096>();
	case 2048: return y_regio<T, U, 2048>();
	}
	if constexpr (sizeof(T) == 4) {
		switch (N) {
		case 1536: return y_regio<T, U, 1536>();
		case 1024: return y_regio<T, U, 1024>();
		case 768: return y_regio<T, U, 768>();
		case 512: return y_regio<T, U, 512>();
		case 384: return y_regio<T, U, 384>();
		case 256: return y_regio<T, U, 256>();
		}
	}
	return false;
}
int spec_y_regio(bool fp64, int U, int N) {
	if (U == 1) return fp64 ? y_regio_n<double, 1>(N) : y_regio_n<float, 1>(N);
	if (U == 2) return fp64 ? y_regio_n<double, 2>(N) : y_regio_n<float, 2>(N);
	return 0;
}

int spec_x_threads(bool fp64, int U, int N) {
	const int maxe = ct_radix(fp64, N);
	const int P = (U * spec_rows(fp64, U, N) + 1) / 2;
	return P * N / maxe <= MAXNT ? P * N / maxe : MAXNT;
}
int spec_y_threads(bool fp64, int U, int N, bool fused) {
	// fused y-pass: one thread per (field, column, butterfly); otherwise as many
	// sequences per FFT call as fit MAXNT threads
	const int maxe = ct_radix(fp64, N);
	const int S = U * spec_cols(fp64, U, N);
	if (fused && U <= 2 && S * N / maxe <= MAXNT) return S * N / maxe;
	if (S * N / maxe <= MAXNT) return S * N / maxe;
	return MAXNT;
}
int spec_x_smem(bool fp64, int U, int N) {
	const int P = (U * spec_rows(fp64, U, N) + 1) / 2;
	const int ce = fp64 ? 16 : 8;
	const int ld = fp64 ? padded_len<double>(N) : padded_len<float>(N);
	return (P * ld + spec_twiddles(fp64, N)) * ce;
}
int spec_y_smem(bool fp64, int U, int N) {
	const int S = U * spec_cols(fp64, U, N);
	const int ce = fp64 ? 16 : 8;
	const int ld = fp64 ? padded_len<double>(N) : padded_len<float>(N);
	return (S * ld + spec_twiddles(fp64, N)) * ce;
}

// ------------------------------------------------------ energy density --
template <int U>
__global__ void energy_density_kernel(const double* __restrict__ mf, const double* __restrict__ pn,
                                      const double* __restrict__ eta, const double* __restrict__ q, const Model m,
                                      long long npts, double* __restrict__ f) {
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npts; i += (long long)gridDim.x * blockDim.x) {
		double fv = 0.0;
		int pair = 0;
#pragma unroll
		for (int u = 0; u < U; u++) {
			const double nu = mf[u * npts + i], nunu = nu * nu;
			fv += m.lambda[u] * nu + 0.5 * m.alpha[u][u] * nunu + 0.5 * m.beta[u][u] * nu * pn[u * npts + i] +
			      (1.0 / 3.0) * m.gamma[u][u] * nu * nunu + 0.25 * m.delta[u] * nunu * nunu;
#pragma unroll
			for (int v = u + 1; v < U; v++, pair++) {
				const double nv = mf[v * npts + i];
				fv += m.alpha[u][v] * nu * nv + m.beta[u][v] * nu * q[pair * npts + i] +
				      0.5 * m.gamma[u][v] * (nunu * nv + nu * nv * nv) + m.epsilon[u][v] * eta[u * npts + i] * eta[v * npts + i];
			}
		}
		f[i] = fv;
	}
}

cudaError_t launch_energy_density(const double* mf, const double* pn, const double* eta, const double* q, int npair,
                                  const Model& mod, long long npts, double* f, cudaStream_t s) {
	(void)npair;
	int grid = (int)((npts + 255) / 256);
	if (grid > 148 * 16) grid = 148 * 16;
	switch (mod.U) {
	case 1: energy_density_kernel<1><<<grid, 256, 0, s>>>(mf, pn, eta, q, mod, npts, f); break;
	case 2: energy_density_kernel<2><<<grid, 256, 0, s>>>(mf, pn, eta, q, mod, npts, f); break;
	case 3: energy_density_kernel<3><<<grid, 256, 0, s>>>(mf, pn, eta, q, mod, npts, f); break;
	case 4: energy_density_kernel<4><<<grid, 256, 0, s>>>(mf, pn, eta, q, mod, npts, f); break;
	default: return cudaErrorInvalidValue;
	}
	return cudaGetLastError();
}

// ------------------------------------------------------------ field means --
__global__ void __launch_bounds__(256) partial_sums_kernel(const double* __restrict__ real, long long npts,
                                                            double* __restrict__ part) {
	const int u = blockIdx.y;
	const double* f = real + u * npts;
	double s = 0.0;
	for (long long i = blockIdx.x * 256LL + threadIdx.x; i < npts; i += (long long)gridDim.x * 256) s += f[i];
	__shared__ double red[256];
	red[threadIdx.x] = s;
	__syncthreads();
	for (int o = 128; o; o >>= 1) {
		if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
		__syncthreads();
	}
	if (threadIdx.x == 0) part[u * gridDim.x + blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(256) finish_means_kernel(const double* __restrict__ part, int nblocks, long long npts,
                                                            double* __restrict__ mean) {
	const int u = blockIdx.x;
	double s = 0.0;
	for (int i = threadIdx.x; i < nblocks; i += 256) s += part[u * nblocks + i];
	__shared__ double red[256];
	red[threadIdx.x] = s;
	__syncthreads();
	for (int o = 128; o; o >>= 1) {
		if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
		__syncthreads();
	}
	if (threadIdx.x == 0) mean[u] = red[0] / (double)npts;
}

// out[i] = sum over p of part[p * nv + i], p in a fixed order (one block per i)
__global__ void __launch_bounds__(256) sum_parts_kernel(const double* __restrict__ part, int nparts, int nv,
                                                         double* __restrict__ out) {
	const int i = blockIdx.x;
	double s = 0.0;
	for (int p = threadIdx.x; p < nparts; p += 256) s += part[(long long)p * nv + i];
	__shared__ double red[256];
	red[threadIdx.x] = s;
	__syncthreads();
	for (int o = 128; o; o >>= 1) {
		if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
		__syncthreads();
	}
	if (threadIdx.x == 0) out[i] = red[0];
}

cudaError_t launch_sum_parts(const double* part, int nparts, int nv, double* out, cudaStream_t s) {
	sum_parts_kernel<<<nv, 256, 0, s>>>(part, nparts, nv, out);
	return cudaGetLastError();
}

cudaError_t launch_field_means(const double* real, int U, long long npts, double* part, int nblocks, double* mean,
                               cudaStream_t s) {
	partial_sums_kernel<<<dim3(nblocks, U), 256, 0, s>>>(real, npts, part);
	cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess) return e;
	finish_means_kernel<<<U, 256, 0, s>>>(part, nblocks, npts, mean);
	return cudaGetLastError();
}

} // namespace pfcg

// ------------------------------------------------- orientation / deformation --
namespace pfcg {
namespace {
__global__ void fields_mul_kernel(double* __restrict__ a, double* __restrict__ b, const double* __restrict__ s,
                                  long long n) {
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
		a[i] *= s[i];
		b[i] *= s[i];
	}
}

__global__ void fields_gradpow_kernel(const double* __restrict__ g, long long n, double power, double* __restrict__ out) {
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
		const double u2 = g[i] * g[i] + g[n + i] * g[n + i], v2 = g[2 * n + i] * g[2 * n + i] + g[3 * n + i] * g[3 * n + i];
		out[i] = pow(u2 + v2, 0.5 * power);
	}
}

// per-block maxima, then one block takes the maximum of those in a fixed order
__global__ void max_partials_kernel(const double* __restrict__ x, long long n, double* __restrict__ part) {
	__shared__ double red[32];
	double m = -INFINITY;
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		m = fmax(m, x[i]);
	for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
	__syncthreads();
	if (threadIdx.x < 32) {
		m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : -INFINITY;
		for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
		if (threadIdx.x == 0) part[blockIdx.x] = m;
	}
}

// acc += r / max(r), the maximum taken from the partials
__global__ void scaled_acc_kernel(double* __restrict__ acc, const double* __restrict__ r, const double* __restrict__ part,
                                  int nparts, long long n) {
	__shared__ double m;
	if (threadIdx.x == 0) {
		double v = -INFINITY;
		for (int k = 0; k < nparts; k++) v = fmax(v, part[k]);
		m = v;
	}
	__syncthreads();
	const double inv = 1.0 / m;
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		acc[i] += r[i] * inv;
}

int grid_of(long long n) { return (int)((n + 255) / 256 > 148 * 8 ? 148 * 8 : (n + 255) / 256); }
} // namespace

cudaError_t launch_fields_mul(double* a, double* b, const double* s, long long n, cudaStream_t st) {
	fields_mul_kernel<<<grid_of(n), 256, 0, st>>>(a, b, s, n);
	return cudaGetLastError();
}
cudaError_t launch_fields_gradpow(const double* g4, long long n, double power, double* out, cudaStream_t st) {
	fields_gradpow_kernel<<<grid_of(n), 256, 0, st>>>(g4, n, power, out);
	return cudaGetLastError();
}
cudaError_t launch_scaled_acc(double* acc, const double* r, long long n, double* part, int nparts, cudaStream_t st) {
	max_partials_kernel<<<nparts, 256, 0, st>>>(r, n, part);
	scaled_acc_kernel<<<grid_of(n), 256, 0, st>>>(acc, r, part, nparts, n);
	return cudaGetLastError();
}

} // namespace pfcg

namespace pfcg {

template <typename T> StepK<T> host_step_k(const Model& m, const Geom& g) {
	StepK<T> k{};
	k.invN = (T)(1.0 / ((double)g.Nx * (double)g.Ny));
	k.cc = (T)m.c;
	k.dt = (T)m.dt;
	k.ag = (T)(-0.5 / m.sigma / m.sigma);
	k.semi = m.scheme == SCHEME_SEMI;
	for (int u = 0; u < MAXU; u++) {
		k.W[u] = m.W[u];
		k.alpha[u] = (T)m.alpha[u][u];
		k.betad[u] = (T)m.beta[u][u];
		for (int w = 0; w < MAXW; w++) {
			k.nu2[u][w] = (T)m.nu2[u][w];
			k.omega[u][w] = (T)m.omega[u][w];
			k.phi[u][w] = (T)m.phi[u][w];
		}
		for (int v = 0; v < MAXU; v++) {
			k.beta[u][v] = (T)m.beta[u][v];
			k.eps[u][v] = (T)m.epsilon[u][v];
			k.mu2[u][v] = (T)m.mu2[u][v];
		}
	}
	k.dkx = (T)g.dkx;
	k.dky = (T)g.dky;
	return k;
}

template StepK<float> host_step_k<float>(const Model&, const Geom&);
template StepK<double> host_step_k<double>(const Model&, const Geom&);

} // namespace pfcg
