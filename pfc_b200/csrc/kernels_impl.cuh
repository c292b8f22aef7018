// Kernels of the B200 relaxation path; see kernels.cuh for the data layout.
// Included by kernels_f32.cu / kernels_f64.cu, which instantiate one precision
// each, by kernels_f32_<N>.cu, which instantiate the FP32 kernels specialised on
// one length N below 2048, and by kernels_common.cu for the
// precision-independent parts.
//
// Reference correspondence (demos/honey/pfc-relax.c):
//   xpass XP_STEP   nonlinear part in real space          :1188-1209
//                   (c2r of :1246 and r2c of :1212 fused around it, x direction)
//   ypass YP_STEP   k-space coupling + ETD1 update          :1215-1244
//                   with A, B of update_AB                  :901-958
//                   (y direction of the r2c :1212 and c2r :1246 fused around it)
//   hermitian_column   spectral resynchronisation (in the y-pass) :1179-1185
//   xpass XP_EVAL + kspace_energy   evaluate()              :988-1131
//   energy_density  f(r) written by write_energy            :1094-1118, :817-859
#pragma once

#include <math.h>
#include <stdlib.h>
#include <stdio.h>

#include <type_traits>

#include "kernels.cuh"

namespace pfcg {

// Elements a thread holds during one FFT pass (and the largest radix):
// 16 in FP32, 8 in FP64, so the butterfly inputs take 32 registers either way.
// Elements per thread (= main radix) of the compile-time specialised kernels
template <typename T> struct FftCfg;
template <> struct FftCfg<float> { static constexpr int MAXE = 16; };
template <> struct FftCfg<double> { static constexpr int MAXE = 8; };
// and of the runtime-plan kernels, in both precisions: 16 elements per thread
// let 512 threads hold one 8192-point sequence (and 7168 / 7680 with a factor 7 / 5)
constexpr int RT_MAXE = 16;
// Main radix (elements per thread) of the kernels specialised on the length N:
// FftCfg's, except FP32 384 = 8 * 6 * 8, which has no radix-16 form with
// radix-16 first and last passes.
template <typename T> __host__ __device__ constexpr int ct_maxe(int N) {
	return (sizeof(T) == 4 && N == 384) ? 8 : FftCfg<T>::MAXE;
}
constexpr int MAXNT = 512; // threads per CTA of the FFT kernels



// --------------------------------------------------------------- helpers --

// The block's sums of v: with store, written to dst (one CTA per slot, so the
// result does not depend on the order CTAs finish in); otherwise added
// atomically. Both trees are fixed: shuffles within each warp, then warp 0 over
// the warps in order.
template <int NV> __device__ __forceinline__ void block_reduce_put(double (&v)[NV], double* dst, bool store) {
	__shared__ double red[32][NV > 0 ? NV : 1];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
	for (int i = 0; i < NV; i++)
#pragma unroll
		for (int o = 16; o; o >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
	if (lane == 0)
#pragma unroll
		for (int i = 0; i < NV; i++) red[warp][i] = v[i];
	__syncthreads();
	if (warp == 0) {
#pragma unroll
		for (int i = 0; i < NV; i++) {
			double x = lane < nw ? red[lane][i] : 0.0;
#pragma unroll
			for (int o = 16; o; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
			if (lane == 0) {
				if (store) dst[i] = x;
				else atomicAdd(dst + i, x);
			}
		}
	}
}

template <typename T> __device__ __forceinline__ T expT(T x);
template <> __device__ __forceinline__ float expT<float>(float x) { return expf(x); }
template <> __device__ __forceinline__ double expT<double>(double x) { return exp(x); }

// B = (exp(x) - 1)/a as pfc-relax.c:952 computes it (FP64 path; FP32 uses phi1f).
template <typename T> __device__ __forceinline__ T etd_b(T A, T x, T a) { return (A - (T)1) / a; }

// P_u(k^2) = prod_w (omega (nu2 - k2)^2 + phi), pfc-relax.c:943-947. Callers
// pass a u that is a compile-time constant after unrolling, so nothing indexes
// the parameter struct dynamically (that would copy it to local memory).
template <typename T> __device__ __forceinline__ T P_of(const Model& m, int u, T k2) {
	T P = (T)1;
#pragma unroll
	for (int w = 0; w < MAXW; w++) {
		if (w < m.W[u]) {
			T q = (T)m.nu2[u][w] - k2;
			P *= (T)m.omega[u][w] * q * q + (T)m.phi[u][w];
		}
	}
	return P;
}

__device__ __forceinline__ double k2_of(int kx, int ky, const Geom& g, double dx, double dy) {
	const double dkx = 2.0 * 3.14159265358979323846264338327 / (dx * g.Nx);
	const double dky = 2.0 * 3.14159265358979323846264338327 / (dy * g.Ny);
	const double kxv = kx * dkx;
	const double kyv = (ky < g.Ny / 2 ? ky : ky - g.Ny) * dky;
	return kxv * kxv + kyv * kyv;
}

// k^2 of the current box with the wave-number steps precomputed on the host
template <typename T> __device__ __forceinline__ T k2_step(int kx, int ky, int Ny, T dkx, T dky) {
	const T kxv = (T)kx * dkx;
	const T kyv = (T)(ky < Ny / 2 ? ky : ky - Ny) * dky;
	return kxv * kxv + kyv * kyv;
}

// phi1(x) = (exp(x) - 1) / x given A = exp(x): Taylor series to x^6 / 7! for
// |x| < 1/4 (remainder < 2e-9), the quotient otherwise (relative error below
// 3e-7 in FP32). B = (A - 1)/a = o dt phi1(x) with x = o a dt, which is also
// the reference's a = 0 case (pfc-relax.c:951-952). The quotient is the
// correctly rounded division: __fdividef (2 ulp) was 0.4 % faster per step but
// moved the relaxed 4096^2 heterostructure's FP32 energy from 1.6e-7 to 2.6e-6
// of the FP64 one (the box optimisation picked other trial sizes).
__device__ __forceinline__ float phi1f(float x, float A) {
	if (fabsf(x) < 0.25f)
		return 1.f + x * (0.5f + x * (1.f / 6.f + x * (1.f / 24.f + x * (1.f / 120.f + x * (1.f / 720.f + x * (1.f / 5040.f))))));
	return (A - 1.f) / x;
}

// Launch shapes of the kernels specialised on a compile-time length NC (NC = 0:
// runtime length and plan). P / S resident sequences, NSUB per FFT call, NT threads.
template <typename T, int U, int NC, int RC> struct XCfg {
	static constexpr bool CT = NC > 0;
	static constexpr int MAXE = CT ? ct_maxe<T>(NC) : RT_MAXE;
	static constexpr int P = CT ? (U * RC + 1) / 2 : 1;
	static constexpr int LD = NC + (NC >> Pad<T>::SHIFT) + 1;
	static constexpr int NSUB = CT ? (P * NC / MAXE <= MAXNT ? P : MAXNT * MAXE / NC) : 1;
	static constexpr int NT = CT ? NSUB * NC / MAXE : MAXNT;
	static constexpr int MINB = (CT && sizeof(T) == 4) ? 2 : 1;
	static constexpr int TWN = CT ? CtPlan<NC, MAXE>::TWN : 0;
};

template <typename T, int U, int NC, int CCC, int RC, bool FUSEDK = true> struct YCfg {
	static constexpr bool CT = NC > 0;
	static constexpr int MAXE = CT ? ct_maxe<T>(NC) : RT_MAXE;
	static constexpr int S = CT ? U * CCC : 1;
	static constexpr int LD = NC + (NC >> Pad<T>::SHIFT) + 1;
	static constexpr bool FUSED = FUSEDK && CT && CtPlan<(CT ? NC : 256), MAXE>::FUSABLE && U <= 2 &&
	                              U * CCC * (CT ? NC : 256) / MAXE <= MAXNT;
	static constexpr int NSUB = CT ? (FUSED ? S : (S * NC / MAXE <= MAXNT ? S : MAXNT * MAXE / NC)) : 1;
	// fused: thread t holds butterfly t mod N/MAXE of column t / (N/MAXE) for every field
	static constexpr int NT = CT ? (FUSED ? U * CCC * NC / MAXE : NSUB * NC / MAXE) : MAXNT;
	static constexpr int MINB = (CT && sizeof(T) == 4) ? 2 : 1;
	static constexpr int TWN = CT ? CtPlan<NC, MAXE>::TWN : 0;
};

// ETD coefficients of one (kx, ky) entry (pfc-relax.c:940-955 and the coupling
// terms of :1215-1244): A_u = exp(o a_u dt) and B_u (FP32: o dt phi1(o a_u dt);
// FP64: the reference's (A - 1)/a, o dt at a = 0) for every field, and the
// coupling coefficient beta_uv (mu2_uv - k2)^2 + eps_uv G^2 of every pair u < v.
template <typename T, int U> __host__ __device__ constexpr int npairs() { return U * (U - 1) / 2 > 0 ? U * (U - 1) / 2 : 1; }
template <typename T, int U>
__device__ __forceinline__ void entry_coef(const StepK<T>& K, T k2, T (&A)[U], T (&Bn)[U],
                                           T (&cu)[npairs<T, U>()]) {
	if constexpr (U > 1) {
		const T G = expT<T>(K.ag * k2);
		const T G2 = G * G;
		int p = 0;
#pragma unroll
		for (int u = 0; u < U - 1; u++)
#pragma unroll
			for (int v = u + 1; v < U; v++) {
				T d2 = K.mu2[u][v] - k2;
				d2 *= d2;
				cu[p++] = K.beta[u][v] * d2 + K.eps[u][v] * G2;
			}
	}
	const T o = K.cc - (T)1 - K.cc * k2;
#pragma unroll
	for (int u = 0; u < U; u++) {
		T P = (T)1;
#pragma unroll
		for (int w = 0; w < MAXW; w++)
			if (w < K.W[u]) {
				const T q = K.nu2[u][w] - k2;
				P *= K.omega[u][w] * q * q + K.phi[u][w];
			}
		const T av = K.alpha[u] + K.betad[u] * P;
		const T x = o * av * K.dt;
		if (K.semi) {
			A[u] = (T)1 / ((T)1 - x);
			Bn[u] = o * K.dt * A[u];
			continue;
		}
		A[u] = expT<T>(x);
		if constexpr (sizeof(T) == 4) Bn[u] = o * K.dt * phi1f(x, A[u]);
		else Bn[u] = (av == (T)0) ? o * K.dt : etd_b<T>(A[u], x, av);
	}
}

// k^2 of entry (kx, ky) as the y-pass STEP computes it
template <typename T>
__device__ __forceinline__ T step_k2(int kx, int ky, int Ny, T dkxT, T dkyT, const Geom& g) {
	if constexpr (sizeof(T) == 4) return k2_step<T>(kx, ky, Ny, dkxT, dkyT);
	else return (T)k2_of(kx, ky, g, g.dx, g.dy);
}

// Hermitian projection of one resident column (kx = 0 or kx = Nx/2): entry ky
// and entry Ny - ky become (a + conj b)/2 and its conjugate, self-conjugate
// entries become real. Writes shared memory and the spectral state. This is
// the reference's resynchronisation N^ = FFT(c2r(N^)) (pfc-relax.c:1179-1185)
// restricted to the only columns where it is not the identity, done every
// step: their anti-Hermitian part is invisible to c2r and is not acted on by
// the nonlinear term, so between resyncs it grows like A(k)^t for every
// unstable k (x1.28 per step for epsilon = -0.25, dt = 1), which overflows in FP32.
template <typename T>
__device__ __forceinline__ void hermitian_column(cplx<T>* col, cplx<T>* spec_col, int Ny, int tid, int nt) {
	const int half = Ny / 2;
	for (int base = 0; base <= half; base += nt) {
		const int j = base + tid;
		cplx<T> p = mk<T>((T)0, (T)0);
		const int jn = (Ny - j) % Ny;
		if (j <= half) {
			const cplx<T> a = col[pad<T>(j)], b = col[pad<T>(jn)];
			p = mk<T>((T)0.5 * (a.x + b.x), (T)0.5 * (a.y - b.y));
		}
		__syncthreads();
		if (j <= half) {
			col[pad<T>(j)] = p;
			spec_col[j] = p;
			if (jn != j) {
				col[pad<T>(jn)] = cconj(p);
				spec_col[jn] = cconj(p);
			}
		}
		__syncthreads();
	}
}

// ------------------------------------------------ fused step pipelines --
// Specialised lengths whose first and last FFT pass have the same radix keep
// each thread's elements in registers from the last pass of one transform to
// the first pass of the next (fft_core.cuh, RegBlock), so the pointwise work
// between two transforms costs no shared-memory round trip and no barrier.

template <typename T, int U, int N> __device__ __forceinline__ T pick(const T (&a)[N], int u) {
	T r = a[0];
#pragma unroll
	for (int k = 1; k < U; k++)
		if (u == k) r = a[k];
	return r;
}

// k = 0 in FP64: mean' = A(0) mean + B(0) (sum NL + couplings),
// pfc-relax.c:1215-1244 at k = 0. The sum of the nonlinear term is that of the
// x-pass's per-tile sums, added by the whole CTA in a fixed order (thread t
// takes tiles t, t + nt, ..., then a fixed tree), or the atomically summed
// accumulator, which is cleared for the next step. Called by every thread of
// the CTA that holds column kx = 0.
template <typename T, int U> __device__ __forceinline__ void ypass_mean_update(const YArgs<T>& a, int tid, int nt) {
	__shared__ double red[32][U];
	double s[U];
#pragma unroll
	for (int u = 0; u < U; u++) s[u] = 0.0;
	if (a.part) {
		for (int i = tid; i < a.nparts; i += nt)
#pragma unroll
			for (int u = 0; u < U; u++) s[u] += a.part[(long long)i * U + u];
		const int lane = tid & 31, warp = tid >> 5, nwp = (nt + 31) >> 5;
#pragma unroll
		for (int u = 0; u < U; u++)
#pragma unroll
			for (int o = 16; o; o >>= 1) s[u] += __shfl_down_sync(0xffffffffu, s[u], o);
		if (lane == 0)
#pragma unroll
			for (int u = 0; u < U; u++) red[warp][u] = s[u];
		__syncthreads();
		if (tid == 0)
#pragma unroll
			for (int u = 0; u < U; u++) {
				s[u] = 0.0;
				for (int w = 0; w < nwp; w++) s[u] += red[w][u];
			}
	}
	if (tid != 0) return;
	const double NxNy = (double)a.g.Nx * (double)a.g.Ny;
	double mean0[U], Mk[U];
#pragma unroll
	for (int u = 0; u < U; u++) { mean0[u] = a.mean[u]; Mk[u] = a.part ? s[u] : a.acc[u]; }
#pragma unroll
	for (int u = 0; u < U - 1; u++)
#pragma unroll
		for (int v = u + 1; v < U; v++) {
			const double d2 = a.m.mu2[u][v] * a.m.mu2[u][v];
			const double cu = a.m.beta[u][v] * d2 + a.m.epsilon[u][v];
			Mk[u] += cu * mean0[v] * NxNy;
			Mk[v] += cu * mean0[u] * NxNy;
		}
#pragma unroll
	for (int u = 0; u < U; u++) {
		const double P0 = P_of<double>(a.m, u, 0.0);
		const double av = a.m.alpha[u][u] + a.m.beta[u][u] * P0;
		const double o = a.m.c - 1.0;
		double A, B;
		if (a.m.scheme == SCHEME_SEMI) {
			A = 1.0 / (1.0 - o * av * a.m.dt);
			B = o * a.m.dt * A / NxNy;
		} else {
			A = exp(o * av * a.m.dt);
			B = ((av == 0.0) ? o * a.m.dt : (A - 1.0) / av) / NxNy;
		}
		a.mean[u] = A * mean0[u] + B * Mk[u];
		if (!a.part) a.acc[u] = 0.0;
	}
}

// x-pass STEP: Y tile -> (Hermitian pairs) -> inverse FFT, its last pass into
// registers -> + mean, NaN check, NL, FP64 sum of NL -> forward FFT from
// registers -> unpack -> Z tile. U in {1, 2}; pair p holds row p (U = 2: the
// two fields as real and imaginary part) or rows 2p, 2p + 1 (U = 1).
// Per-pass twiddle table of a specialised kernel into shared memory: all of a
// thread's loads first, then its stores, so that the table's L2 latency is paid
// once (callers issue their own global loads before it).
template <typename T, int TWN, int NT>
__device__ __forceinline__ void copy_twiddles(cplx<T>* tws, const cplx<T>* __restrict__ src, int tid) {
	constexpr int TPT = (TWN + NT - 1) / NT;
	cplx<T> t[TPT];
#pragma unroll
	for (int j = 0; j < TPT; j++) {
		const int i = tid + j * NT;
		if (TWN % NT == 0 || i < TWN) t[j] = src[i];
	}
#pragma unroll
	for (int j = 0; j < TPT; j++) {
		const int i = tid + j * NT;
		if (TWN % NT == 0 || i < TWN) tws[i] = t[j];
	}
}

template <typename T, int U, int NC, int RC, int P, int NT, int MAXE>
__device__ __forceinline__ void xpass_step_fused(const XArgs<T>& a, cplx<T>* sm, cplx<T>* tws, int tile, int tid,
                                                 bool load_tw) {
	using PL = CtPlan<NC, MAXE>;
	using RB = RegBlock<NC, MAXE, P, NT, T>;
	constexpr int LD = NC + (NC >> Pad<T>::SHIFT) + 1;
	constexpr int H = NC / 2 + 1;
	constexpr int CH = U * RC;
	const long long tofs = (long long)tile * H * RC;
	// Hermitian-extended pair spectra (as in the runtime kernel); the loop is
	// unrolled so that all of a thread's loads are in flight together
	constexpr int KIT = (H + NT - 1) / NT;
#pragma unroll
	for (int it = 0; it < KIT; it++) {
		const int k = tid + it * NT;
		if (k >= H) break;
		cplx<T> y[CH];
		if constexpr (sizeof(T) == 4 && RC == 2) {
			// both rows of a field at k are one 16-byte word
#pragma unroll
			for (int u = 0; u < U; u++) {
				const float4 q = *reinterpret_cast<const float4*>(a.work + u * a.wstride + tofs + (long long)k * RC);
				y[u] = mk<T>(q.x, q.y);
				y[U + u] = mk<T>(q.z, q.w);
			}
		} else {
#pragma unroll
			for (int c = 0; c < CH; c++) y[c] = a.work[(c % U) * a.wstride + tofs + (long long)k * RC + c / U];
		}
		const bool selfc = (k == 0) || (2 * k == NC);
#pragma unroll
		for (int p = 0; p < P; p++) {
			cplx<T> A = y[2 * p], B = y[2 * p + 1];
			if (selfc) { A.y = (T)0; B.y = (T)0; }
			sm[p * LD + pad<T>(k)] = mk<T>(A.x - B.y, A.y + B.x);
			if (k > 0 && 2 * k < NC) sm[p * LD + pad<T>(NC - k)] = mk<T>(A.x + B.y, B.x - A.y);
		}
	}
	if (load_tw) copy_twiddles<T, CtPlan<NC, MAXE>::TWN, NT>(tws, a.twct, tid);
	__syncthreads();
	// inverse transform: all passes but the last in shared memory, the last into registers
	ct_pass<NC, PL::radix(0), PL::ns(0), PL::twoff(0), P, NT, +1, T>(sm, tws, tid);
	ct_middle<NC, MAXE, P, NT, +1, T>(sm, tws, tid);
	RB rb;
	ct_last_to_regs<NC, MAXE, P, NT, +1, T>(sm, tws, rb, tid);
	// nonlinear term in registers, pfc-relax.c:1188-1209
	T offT[U], lam[U], del[U], gam[U][U], alp[U][U];
#pragma unroll
	for (int u = 0; u < U; u++) {
		offT[u] = (T)a.off[u];
		lam[u] = (T)a.m.lambda[u];
		del[u] = (T)a.m.delta[u];
#pragma unroll
		for (int v = 0; v < U; v++) { gam[u][v] = (T)a.m.gamma[u][v]; alp[u][v] = (T)a.m.alpha[u][v]; }
	}
	T accT[U];
#pragma unroll
	for (int u = 0; u < U; u++) accT[u] = (T)0;
	bool nan = false;
#pragma unroll
	for (int i = 0; i < RB::NB; i++)
#pragma unroll
		for (int r = 0; r < MAXE; r++) {
			cplx<T>& z = rb.v[i][r];
			if constexpr (U == 2) {
				const T m0 = z.x + offT[0], m1 = z.y + offT[1];
				nan |= (m0 != m0) | (m1 != m1);
				const T mc0 = alp[0][1] * m1 + (T)0.5 * gam[0][1] * ((T)2 * m0 * m1 + m1 * m1);
				const T mc1 = alp[0][1] * m0 + (T)0.5 * gam[0][1] * ((T)2 * m1 * m0 + m0 * m0);
				const T q0 = m0 * m0, q1 = m1 * m1;
				const T nl0 = lam[0] + gam[0][0] * q0 + del[0] * m0 * q0 + mc0;
				const T nl1 = lam[1] + gam[1][1] * q1 + del[1] * m1 * q1 + mc1;
				accT[0] += nl0;
				accT[1] += nl1;
				z = mk<T>(nl0, nl1);
			} else {
				const T m0 = z.x + offT[0], m1 = z.y + offT[0];
				nan |= (m0 != m0) | (m1 != m1);
				const T q0 = m0 * m0, q1 = m1 * m1;
				const T nl0 = lam[0] + gam[0][0] * q0 + del[0] * m0 * q0;
				const T nl1 = lam[0] + gam[0][0] * q1 + del[0] * m1 * q1;
				accT[0] += nl0 + nl1;
				z = mk<T>(nl0, nl1);
			}
		}
	// forward transform: first pass from registers, the rest in shared memory
	ct_first_from_regs<NC, MAXE, P, NT, -1, T>(sm, rb, tid);
	ct_middle<NC, MAXE, P, NT, -1, T>(sm, tws, tid);
	ct_pass<NC, MAXE, PL::ns(PL::NPASS - 1), PL::twoff(PL::NPASS - 1), P, NT, -1, T>(sm, tws, tid);
	if (nan) atomicOr(a.flag, 1);
	// split the pairs and store the Z tile
	const T half = (T)0.5;
	for (int k = tid; k < H; k += NT) {
		const int km = (k == 0) ? 0 : NC - k;
		cplx<T> zz[2 * P];
#pragma unroll
		for (int p = 0; p < P; p++) {
			const cplx<T> Ck = sm[p * LD + pad<T>(k)];
			const cplx<T> Cm = sm[p * LD + pad<T>(km)];
			zz[2 * p] = mk<T>(half * (Ck.x + Cm.x), half * (Ck.y - Cm.y));
			zz[2 * p + 1] = mk<T>(half * (Ck.y + Cm.y), half * (Cm.x - Ck.x));
		}
		if constexpr (sizeof(T) == 4 && RC == 2) {
#pragma unroll
			for (int u = 0; u < U; u++)
				*reinterpret_cast<float4*>(a.work + u * a.wstride + tofs + (long long)k * RC) =
				    make_float4(zz[u].x, zz[u].y, zz[U + u].x, zz[U + u].y);
		} else {
#pragma unroll
			for (int c = 0; c < CH; c++) a.work[(c % U) * a.wstride + tofs + (long long)k * RC + c / U] = zz[c];
		}
	}
	double acc[U];
#pragma unroll
	for (int u = 0; u < U; u++) acc[u] = (double)accT[u];
	block_reduce_put<U>(acc, a.part ? a.part + (long long)tile * U : a.acc, a.part != nullptr);
}

// y-pass STEP: Z columns from global straight into the first forward pass ->
// forward FFT, last pass into registers -> coupling + ETD1 update in registers
// -> Hermitian fix of the kx = 0 and kx = Nx/2 columns (their CTAs only) ->
// inverse FFT from registers, last pass into registers -> Y columns to global.
// One butterfly of one field per thread, NT = U * CC * N/MAXE. With two fields
// the PairMap puts them in lanes l and l ^ 16 at the same points: each thread
// reads only its own field's spectral state and gets the other one by a
// shuffle, so no thread reads an entry another thread writes.
template <typename T, int U, int NC, int CCC, int RC, int S, int NT, int MAXE>
__device__ __forceinline__ void ypass_step_fused(const YArgs<T>& a, cplx<T>* sm, const cplx<T>* tws, int kx0, int ncol,
                                                 int tid) {
	using MAP = typename std::conditional<U == 2, PairMap<NC, MAXE, CCC>, StdMap<NC, MAXE, S, NT>>::type;
	using RB = RegBlock<NC, MAXE, S, NT, T, MAP>;
	static_assert(RB::NB == 1 && NT == U * CCC * (NC / MAXE), "one butterfly per thread");
	constexpr int LD = NC + (NC >> Pad<T>::SHIFT) + 1;
	constexpr int NR = NC / MAXE;
	const int Nx = a.g.Nx, H = a.g.H;
	const long long tileH = (long long)H * RC;
	const int p = MAP::seq(tid, 0);
	const int u = p / CCC, c = p % CCC;
	const int j = MAP::bj(tid, 0);
	const int kx = kx0 + c;
	const bool live = c < ncol;
	RB rb;
	// Z column: element y at work[u][y / RC][kx][y % RC]
	{
		const cplx<T>* src = a.work + u * a.wstride + (long long)kx * RC;
#pragma unroll
		for (int r = 0; r < MAXE; r++) {
			const int y = j + r * NR;
			rb.v[0][r] = live ? src[(long long)(y / RC) * tileH + y % RC] : mk<T>((T)0, (T)0);
		}
	}
	ct_first_from_regs<NC, MAXE, S, NT, -1, T, MAP>(sm, rb, tid);
	ct_middle<NC, MAXE, S, NT, -1, T>(sm, tws, tid);
	ct_last_to_regs<NC, MAXE, S, NT, -1, T, MAP>(sm, tws, rb, tid);

	// update, pfc-relax.c:1215-1244 (A, B of update_AB, :901-958, recomputed);
	// the field's own constants, selected once
	const StepK<T>& K = a.k;
	const T dkxT = K.dkx, dkyT = K.dky;
	const T alpha = pick<T, U>(K.alpha, u), betad = pick<T, U>(K.betad, u);
	const int W = pick<int, U>(K.W, u);
	T nu2[MAXW], om[MAXW], ph[MAXW];
#pragma unroll
	for (int w = 0; w < MAXW; w++) {
		nu2[w] = K.nu2[0][w];
		om[w] = K.omega[0][w];
		ph[w] = K.phi[0][w];
		if constexpr (U > 1)
			if (u == 1) { nu2[w] = K.nu2[1][w]; om[w] = K.omega[1][w]; ph[w] = K.phi[1][w]; }
	}
	// no store to the spectral state inside this loop, so the compiler may issue
	// its loads as early as registers allow
	const cplx<T>* spec_in = a.spec + u * a.sstride + (long long)kx * NC;
#pragma unroll
	for (int r = 0; r < MAXE; r++) {
		const int ky = j + r * NR;
		const cplx<T> Nown = live ? spec_in[ky] : mk<T>((T)0, (T)0);
		const T k2 = k2_step<T>(kx, ky, NC, dkxT, dkyT);
		cplx<T> M = cscale(rb.v[0][r], K.invN);
		if constexpr (U > 1) {
			cplx<T> Noth;
			Noth.x = __shfl_xor_sync(0xffffffffu, Nown.x, 16);
			Noth.y = __shfl_xor_sync(0xffffffffu, Nown.y, 16);
			const T G = expT<T>(K.ag * k2);
			T d2 = K.mu2[0][1] - k2;
			d2 *= d2;
			const T cu = K.beta[0][1] * d2 + K.eps[0][1] * G * G;
			M = cadd(M, cscale(Noth, cu));
		}
		T Pk = (T)1;
#pragma unroll
		for (int w = 0; w < MAXW; w++)
			if (w < W) {
				const T q = nu2[w] - k2;
				Pk *= om[w] * q * q + ph[w];
			}
		const T av = alpha + betad * Pk;
		const T o = K.cc - (T)1 - K.cc * k2;
		const T x = o * av * K.dt;
		T A, Bn;
		if (K.semi) {
			A = (T)1 / ((T)1 - x);
			Bn = o * K.dt * A;
		} else {
			A = expT<T>(x);
			if constexpr (sizeof(T) == 4) Bn = o * K.dt * phi1f(x, A);
			else Bn = (av == (T)0) ? o * K.dt : etd_b<T>(A, x, av);
		}
		cplx<T> nn = cadd(cscale(Nown, A), cscale(M, Bn));
		if (kx == 0 && ky == 0) nn = mk<T>((T)0, (T)0);
		rb.v[0][r] = nn;
	}
	if (live) {
		cplx<T>* spec_out = a.spec + u * a.sstride + (long long)kx * NC;
#pragma unroll
		for (int r = 0; r < MAXE; r++) spec_out[j + r * NR] = rb.v[0][r];
	}
	// kx = 0 and (even Nx) kx = Nx/2: Hermitian projection needs ky and -ky together
	const int kn = (Nx % 2 == 0) ? Nx / 2 : -1;
	const bool has0 = (kx0 == 0);
	const bool hasn = (kn >= kx0 && kn < kx0 + ncol);
	if (has0 || hasn) {
		__syncthreads();
#pragma unroll
		for (int r = 0; r < MAXE; r++) sm[p * LD + pad<T>(j + r * NR)] = rb.v[0][r];
		__syncthreads();
#pragma unroll
		for (int v = 0; v < U; v++) {
			if (has0) hermitian_column<T>(sm + (v * CCC) * LD, a.spec + v * a.sstride, NC, tid, NT);
			if (hasn)
				hermitian_column<T>(sm + (v * CCC + (kn - kx0)) * LD, a.spec + v * a.sstride + (long long)kn * NC, NC, tid,
				                    NT);
		}
#pragma unroll
		for (int r = 0; r < MAXE; r++) rb.v[0][r] = sm[p * LD + pad<T>(j + r * NR)];
	}
	ct_first_from_regs<NC, MAXE, S, NT, +1, T, MAP>(sm, rb, tid);
	ct_middle<NC, MAXE, S, NT, +1, T>(sm, tws, tid);
	ct_last_to_regs<NC, MAXE, S, NT, +1, T, MAP>(sm, tws, rb, tid);
	if (live) {
		cplx<T>* dst = a.work + u * a.wstride + (long long)kx * RC;
#pragma unroll
		for (int r = 0; r < MAXE; r++) {
			const int y = j + r * NR;
			dst[(long long)(y / RC) * tileH + y % RC] = rb.v[0][r];
		}
	}
	if (kx0 == 0) ypass_mean_update<T, U>(a, tid, NT);
}

// ----------------------------------------------------------------- x-pass --

// Body of the x-pass for row tile `tile`; called by xpass_kernel (one problem)
// and by xpass_batch_kernel (many problems in one launch).
// (in the fused instantiations the code after the early return is unreachable,
// which is intended)
#pragma nv_diag_suppress 128
template <typename T, int U, int MODE, int NC, int RC>
__device__ __forceinline__ void xpass_body(const XArgs<T>& a, const int tile, const bool load_tw = true) {
	using C = XCfg<T, U, NC, RC>;
	constexpr int MAXE = C::MAXE;
	extern __shared__ __align__(128) unsigned char smem_raw[];
	cplx<T>* sm = reinterpret_cast<cplx<T>*>(smem_raw);
	const int Nx = C::CT ? NC : a.g.Nx;
	const int Ny = a.g.Ny;
	const int H = Nx / 2 + 1;
	const int R = C::CT ? RC : a.g.R;
	const int CH = U * R;
	const int P = (CH + 1) >> 1;
	const int ld = C::CT ? C::LD : padded_len<T>(Nx);
	const int y0 = tile * R;
	const int tid = threadIdx.x;
	const int nt = C::CT ? C::NT : (int)blockDim.x;
	const long long tofs = (long long)tile * H * R;
	cplx<T>* tws = sm + (C::CT ? C::P * C::LD : 0);
	constexpr bool XFUSED = MODE == XP_STEP && C::CT && CtPlan<(C::CT ? NC : 256), MAXE>::FUSABLE && C::NSUB == C::P &&
	                        U <= 2 && (U * RC) % 2 == 0;
	if constexpr (C::CT && !XFUSED) {
		if (load_tw) copy_twiddles<T, C::TWN, C::NT>(tws, a.twct, tid);
	}
	if constexpr (XFUSED) {
		// the fused pass copies the twiddles after issuing its tile loads
		xpass_step_fused<T, U, NC, RC, C::P, C::NT, MAXE>(a, sm, tws, tile, tid, load_tw);
		return;
	}

	double off[U];
#pragma unroll
	for (int u = 0; u < U; u++) off[u] = a.off ? a.off[u] : 0.0;

	if constexpr (MODE == XP_R2C) {
		// real rows (minus their mean) -> pairs of channels in one complex sequence
		for (int x = tid; x < Nx; x += nt) {
#pragma unroll
			for (int p = 0; p < MAX_CH / 2; p++) {
				if (p < P) {
					const int c0 = 2 * p, c1 = 2 * p + 1;
					const int u0 = c0 % U, r0 = c0 / U, u1 = c1 % U, r1 = c1 / U;
					const double v0 = a.real[((long long)u0 * Ny + y0 + r0) * Nx + x] - (a.off ? a.off[u0] : 0.0);
					const double v1 = (c1 < CH) ? a.real[((long long)u1 * Ny + y0 + r1) * Nx + x] - (a.off ? a.off[u1] : 0.0) : 0.0;
					sm[p * ld + pad<T>(x)] = mk<T>((T)v0, (T)v1);
				}
			}
		}
	} else {
		// Hermitian-extended spectra of channel pairs: C = A + iB on 0..Nx/2,
		// conj(A) + i conj(B) on Nx/2+1..Nx-1; imaginary parts of the kx = 0 and
		// kx = Nx/2 entries are dropped like a c2r transform does.
		for (int k = tid; k < H; k += nt) {
			cplx<T> y[MAX_CH];
#pragma unroll
			for (int c = 0; c < MAX_CH; c++) {
				y[c] = mk<T>((T)0, (T)0);
				if (c < CH) {
					const int u = c % U, r = c / U;
					y[c] = a.work[u * a.wstride + tofs + (long long)k * R + r];
				}
			}
			const bool selfc = (k == 0) || (2 * k == Nx);
#pragma unroll
			for (int p = 0; p < MAX_CH / 2; p++) {
				if (p < P) {
					cplx<T> A = y[2 * p], B = y[2 * p + 1];
					if (selfc) { A.y = (T)0; B.y = (T)0; }
					sm[p * ld + pad<T>(k)] = mk<T>(A.x - B.y, A.y + B.x);
					if (k > 0 && 2 * k < Nx) sm[p * ld + pad<T>(Nx - k)] = mk<T>(A.x + B.y, B.x - A.y);
				}
			}
		}
		__syncthreads();
		if constexpr (C::CT) fft_ct<NC, MAXE, C::P, C::NSUB, C::NT, +1, T>(sm, tws, tid);
		else fft_batches<+1, MAXE, T>(sm, ld, P, a.sb, a.plan, a.tw, tid, nt);
	}

	if constexpr (MODE == XP_STEP || MODE == XP_EVAL || MODE == XP_C2R) {
		constexpr int NACC = (MODE == XP_EVAL) ? 1 + U : U;
		double acc[NACC];
#pragma unroll
		for (int i = 0; i < NACC; i++) acc[i] = 0.0;
		bool nan = false;
		T lam[U], del[U], gam[U][U], alp[U][U], offT[U];
#pragma unroll
		for (int u = 0; u < U; u++) {
			offT[u] = (T)off[u];
			lam[u] = (T)a.m.lambda[u];
			del[u] = (T)a.m.delta[u];
#pragma unroll
			for (int v = 0; v < U; v++) { gam[u][v] = (T)a.m.gamma[u][v]; alp[u][v] = (T)a.m.alpha[u][v]; }
		}
		for (int x = tid; x < Nx; x += nt) {
			T z[MAX_CH];
#pragma unroll
			for (int p = 0; p < MAX_CH / 2; p++) {
				if (p < P) {
					const cplx<T> v = sm[p * ld + pad<T>(x)];
					z[2 * p] = v.x;
					z[2 * p + 1] = v.y;
				}
			}
#pragma unroll
			for (int r = 0; r < MAX_CH / U; r++) {
				if (r < R) {
					if constexpr (MODE == XP_STEP) {
						T mv[U], mc[U];
#pragma unroll
						for (int u = 0; u < U; u++) {
							mv[u] = z[r * U + u] + offT[u];
							nan |= (mv[u] != mv[u]);
							mc[u] = (T)0;
						}
#pragma unroll
						for (int u = 0; u < U - 1; u++)
#pragma unroll
							for (int v = u + 1; v < U; v++) {
								mc[u] += alp[u][v] * mv[v] + (T)0.5 * gam[u][v] * ((T)2 * mv[u] * mv[v] + mv[v] * mv[v]);
								mc[v] += alp[u][v] * mv[u] + (T)0.5 * gam[u][v] * ((T)2 * mv[v] * mv[u] + mv[u] * mv[u]);
							}
#pragma unroll
						for (int u = 0; u < U; u++) {
							const T m2 = mv[u] * mv[u];
							const T nl = lam[u] + gam[u][u] * m2 + del[u] * mv[u] * m2 + mc[u];
							z[r * U + u] = nl;
							acc[u] += (double)nl;
						}
					} else if constexpr (MODE == XP_EVAL) {
						double mv[U];
#pragma unroll
						for (int u = 0; u < U; u++) mv[u] = (double)z[r * U + u] + off[u];
						double f = 0.0;
#pragma unroll
						for (int u = 0; u < U; u++) {
							const double n1 = mv[u], n2 = n1 * n1;
							f += a.m.lambda[u] * n1 + 0.5 * a.m.alpha[u][u] * n2 + (1.0 / 3.0) * a.m.gamma[u][u] * n1 * n2 +
							     0.25 * a.m.delta[u] * n2 * n2;
#pragma unroll
							for (int v = u + 1; v < U; v++) {
								const double nv = mv[v];
								f += a.m.alpha[u][v] * n1 * nv + 0.5 * a.m.gamma[u][v] * (n2 * nv + n1 * nv * nv);
							}
							acc[1 + u] += n1;
						}
						acc[0] += f;
					} else {
#pragma unroll
						for (int u = 0; u < U; u++)
							a.real[((long long)u * Ny + y0 + r) * Nx + x] = (double)z[r * U + u] + off[u];
					}
				}
			}
			if constexpr (MODE == XP_STEP) {
#pragma unroll
				for (int p = 0; p < MAX_CH / 2; p++)
					if (p < P) sm[p * ld + pad<T>(x)] = mk<T>(z[2 * p], (2 * p + 1 < CH) ? z[2 * p + 1] : (T)0);
			}
		}
		if constexpr (MODE == XP_STEP) {
			if (nan) atomicOr(a.flag, 1);
			block_reduce_put<NACC>(acc, a.part ? a.part + (long long)tile * U : a.acc, a.part != nullptr);
		} else if constexpr (MODE == XP_EVAL) {
			block_reduce_put<NACC>(acc, a.part ? a.part + (long long)tile * NACC : a.acc, a.part != nullptr);
		}
	}

	if constexpr (MODE == XP_STEP || MODE == XP_R2C) {
		__syncthreads();
		if constexpr (C::CT) fft_ct<NC, MAXE, C::P, C::NSUB, C::NT, -1, T>(sm, tws, tid);
		else fft_batches<-1, MAXE, T>(sm, ld, P, a.sb, a.plan, a.tw, tid, nt);
		// split each pair: Za = (C[k] + conj C[-k]) / 2, Zb = (C[k] - conj C[-k]) / (2i)
		const T half = (T)0.5;
		for (int k = tid; k < H; k += nt) {
			const int km = (k == 0) ? 0 : Nx - k;
			cplx<T> zz[MAX_CH];
#pragma unroll
			for (int p = 0; p < MAX_CH / 2; p++) {
				if (p < P) {
					const cplx<T> Ck = sm[p * ld + pad<T>(k)];
					const cplx<T> Cm = sm[p * ld + pad<T>(km)];
					zz[2 * p] = mk<T>(half * (Ck.x + Cm.x), half * (Ck.y - Cm.y));
					zz[2 * p + 1] = mk<T>(half * (Ck.y + Cm.y), half * (Cm.x - Ck.x));
				}
			}
#pragma unroll
			for (int c = 0; c < MAX_CH; c++) {
				if (c < CH) {
					const int u = c % U, r = c / U;
					a.work[u * a.wstride + tofs + (long long)k * R + r] = zz[c];
				}
			}
		}
	}
}
#pragma nv_diag_default 128

// ----------------------------------------------------------------- y-pass --



// Row tiles blockIdx.x, + gridDim.x, ... < ntiles: a grid of fewer CTAs than
// tiles keeps each CTA resident over several tiles, loading the per-pass
// twiddle table of the specialised kernels once.
template <typename T, int U, int MODE, int NC, int RC>
__global__ void __launch_bounds__(XCfg<T, U, NC, RC>::NT, XCfg<T, U, NC, RC>::MINB)
    xpass_kernel(const XArgs<T> a, int ntiles) {
	// programmatic dependent launch (pdl_launch): the previous kernel's results
	// are complete and visible after this wait; a plain launch returns at once
	asm volatile("griddepcontrol.wait;" ::: "memory");
	asm volatile("griddepcontrol.launch_dependents;");
	for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
		if (t != (int)blockIdx.x) __syncthreads(); // the previous tile's readers of shared memory are done
		xpass_body<T, U, MODE, NC, RC>(a, t, t == (int)blockIdx.x);
	}
}

// Body of the y-pass for column group `grp`; called by ypass_kernel and by
// ypass_batch_kernel.
// ------------------------------------------------------ TMA column loads --
// The y-pass's input columns are R-row pieces of every row tile of `work`
// (16 bytes per tile and column at 4096^2 U=2 FP32), a gather that costs the
// load/store unit one request per 16 bytes. The tensor memory accelerator
// moves them instead: thread 0 issues one cp.async.bulk.tensor per box of
// tma_tiles tiles and field, the boxes land in shared memory as
// [field][tile][column][row] (so field u, column c, row y of a column group
// is at u * Ny * CC + ((y / R) * CC + c) * R + y % R), and the CTA waits on an
// mbarrier. The wait is bounded: after tma_timeout_ns (1 s) of polling it
// records FLAG_TIMEOUT and goes on, and the step returns PFCG_ETIMEOUT. The tensor map
// covers only this GPU's own `work` buffer and no load uses multicast.

__device__ __forceinline__ void tma_bar_init(unsigned bar) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void tma_expect(unsigned bar, unsigned bytes) {
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load4(unsigned dst, const void* tmap, int c0, int c1, int c2, int c3, unsigned bar) {
	asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
	             "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
	             : "memory");
}

// polls phase `parity` of the mbarrier for at most `limit_ns` (%globaltimer); false on time-out
__device__ __forceinline__ bool tma_wait(unsigned bar, unsigned parity, unsigned long long limit_ns) {
	unsigned long long t0;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
	for (;;) {
		unsigned done;
		asm volatile("{ .reg .pred q; mbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2; selp.u32 %0, 1, 0, q; }"
		             : "=r"(done)
		             : "r"(bar), "r"(parity)
		             : "memory");
		if (done) return true;
		unsigned long long t;
		asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
		if (t - t0 > limit_ns) return false;
	}
}

template <typename T, int U, int MODE, int NC, int CCC, int RC, bool FUSEDK = true>
__device__ __forceinline__ void ypass_body(const YArgs<T>& a, const int grp, const bool load_tw = true, const int iter = 0) {
	using C = YCfg<T, U, NC, CCC, RC, FUSEDK>;
	constexpr int MAXE = C::MAXE;
	extern __shared__ __align__(128) unsigned char smem_raw[];
	cplx<T>* sm = reinterpret_cast<cplx<T>*>(smem_raw);
	const int Nx = a.g.Nx, H = a.g.H;
	const int Ny = C::CT ? NC : a.g.Ny;
	const int R = C::CT ? RC : a.g.R;
	const int CC = C::CT ? CCC : a.g.CC;
	const int S = U * CC;
	const int ld = C::CT ? C::LD : padded_len<T>(Ny);
	const int kx0 = grp * CC;
	const int ncol = min(CC, H - kx0);
	const int ntile = Ny / R;
	const long long tileH = (long long)H * R;
	const int chunk = CC * R;
	const int tid = threadIdx.x;
	const int nt = C::CT ? C::NT : (int)blockDim.x;
	cplx<T>* tws = sm + (C::CT ? C::S * C::LD : 0);
	// (copying the twiddles after the register-end loads instead, as the
	// x-pass does, measured 2 % slower here)
	if constexpr (C::CT) {
		if (load_tw)
			for (int i = tid; i < C::TWN; i += C::NT) tws[i] = a.twct[i];
	}

	if constexpr (MODE == YP_STEP && C::FUSED && FUSEDK) {
		ypass_step_fused<T, U, NC, CCC, RC, C::S, C::NT, MAXE>(a, sm, tws, kx0, ncol, tid);
		return;
	}
	if constexpr (MODE == YP_STEP && C::CT) {
		// this group's spectral-state columns into L2 now, so that the update's
		// loads after the forward transform find them there: one 128-byte line
		// per prefetch, all inside the live columns
		constexpr int LPC = NC * (int)sizeof(cplx<T>) / 128; // lines per column
		for (int i = tid; i < U * ncol * LPC; i += C::NT) {
			const int u = i / (ncol * LPC), rest = i % (ncol * LPC);
			const char* line = reinterpret_cast<const char*>(a.spec + u * a.sstride + (long long)kx0 * NC) + rest * 128;
			asm volatile("prefetch.global.L2 [%0];" ::"l"(line));
		}
	}

	// Register ends (STEP, one butterfly per thread per pass): the forward
	// transform's first pass takes its inputs straight from global memory and
	// the inverse transform's last pass stores straight to it, which saves the
	// shared-memory round trip and barrier of a separate load and store phase.
	constexpr int NCX = C::CT ? NC : 256;
	using PLX = CtPlan<NCX, MAXE>;
	constexpr bool REGIO = C::CT && MODE == YP_STEP && !(C::FUSED && FUSEDK) && C::NSUB == C::S &&
	                       C::S * (NCX / MAXE) == C::NT && PLX::FUSABLE;
	using RBY = RegBlock<NCX, MAXE, C::S, C::NT, T>;
	constexpr int CCX = C::CT ? CCC : 1;
	// global address of element y of resident sequence p (field p / CCC, column p % CCC)
	auto gaddr = [&](int p, int y) -> long long {
		return (long long)(p / CCX) * a.wstride + (long long)(y / R) * tileH + (long long)(kx0 + p % CCX) * R +
		       y % R;
	};
	bool regio = false;
	if constexpr (REGIO) {
		if (a.regio) {
			regio = true;
			RBY rb;
			if (a.tmap) {
				__shared__ __align__(8) unsigned long long tbar;
				const unsigned bar = (unsigned)__cvta_generic_to_shared(&tbar);
				if (iter == 0) {
					if (tid == 0) tma_bar_init(bar);
					__syncthreads();
				}
				constexpr int NTILE = NCX / RC;
				if (tid == 0) {
					const int tb = a.tma_tiles;
					// earlier generic accesses to the buffer before the async-proxy writes
					asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
					tma_expect(bar, (unsigned)(U * NCX * CCX * sizeof(cplx<T>)) + a.tma_extra);
					for (int u = 0; u < U; u++)
						for (int t0 = 0; t0 < NTILE; t0 += tb)
							tma_load4((unsigned)__cvta_generic_to_shared(sm + (u * NTILE + t0) * CCX * RC), a.tmap, 0, kx0,
							          t0, u, bar);
				}
				if (!tma_wait(bar, (unsigned)(iter & 1), a.tma_timeout_ns) && tid == 0) atomicOr(a.flag, FLAG_TIMEOUT);
#pragma unroll
				for (int i = 0; i < RBY::NB; i++) {
					const int p = RBY::seq(tid, i);
#pragma unroll
					for (int r = 0; r < MAXE; r++) {
						const int y = RBY::pos(tid, i, r);
						rb.v[i][r] = sm[((p / CCX) * NTILE + y / RC) * CCX * RC + (p % CCX) * RC + y % RC];
					}
				}
			} else {
#pragma unroll
				for (int i = 0; i < RBY::NB; i++) {
					const int p = RBY::seq(tid, i);
					const bool live = p % CCX < ncol;
#pragma unroll
					for (int r = 0; r < MAXE; r++)
						rb.v[i][r] = live ? a.work[gaddr(p, RBY::pos(tid, i, r))] : mk<T>((T)0, (T)0);
				}
			}
			ct_first_from_regs<NCX, MAXE, C::S, C::NT, -1, T>(sm, rb, tid);
			ct_middle<NCX, MAXE, C::S, C::NT, -1, T>(sm, tws, tid);
			ct_pass<NCX, PLX::radix(PLX::NPASS - 1), PLX::ns(PLX::NPASS - 1), PLX::twoff(PLX::NPASS - 1), C::S, C::NT,
			        -1, T>(sm, tws, tid);
		}
	}

	if constexpr (MODE != YP_WEIGHT) if (!regio) {
		if constexpr (C::CT && ((NC / RC) * CCC * RC) % C::NT == 0) {
			// every load of the tile in flight before the first shared-memory store
			constexpr int CH = CCC * RC;
			constexpr int PER = (NC / RC) * CH / C::NT;
			cplx<T> v[U][PER];
#pragma unroll
			for (int u = 0; u < U; u++) {
				const cplx<T>* src = a.work + u * a.wstride + (long long)kx0 * RC;
#pragma unroll
				for (int i = 0; i < PER; i++) {
					const int e = tid + i * C::NT;
					const int t = e / CH, rem = e % CH;
					v[u][i] = (rem / RC < ncol) ? src[t * tileH + rem] : mk<T>((T)0, (T)0);
				}
			}
#pragma unroll
			for (int u = 0; u < U; u++)
#pragma unroll
				for (int i = 0; i < PER; i++) {
					const int e = tid + i * C::NT;
					const int t = e / CH, rem = e % CH;
					sm[(u * CCC + rem / RC) * C::LD + pad<T>(t * RC + rem % RC)] = v[u][i];
				}
		} else {
#pragma unroll
			for (int u = 0; u < U; u++) {
				const cplx<T>* src = a.work + u * a.wstride + (long long)kx0 * R;
				for (int e = tid; e < ntile * chunk; e += nt) {
					const int t = e / chunk, rem = e - t * chunk;
					const int c = rem / R, r = rem - c * R;
					cplx<T> v = mk<T>((T)0, (T)0);
					if (c < ncol) v = src[t * tileH + rem];
					sm[(u * CC + c) * ld + pad<T>(t * R + r)] = v;
				}
			}
		}
		__syncthreads();
		if constexpr (C::CT) fft_ct<NC, MAXE, C::S, C::NSUB, C::NT, -1, T>(sm, tws, tid);
		else fft_batches<-1, MAXE, T>(sm, ld, S, a.sb, a.plan, a.tw, tid, nt);
	}

	const double dx = a.g.dx, dy = a.g.dy;
	if constexpr (MODE == YP_STEP) {
		// model constants in the transform precision, once per CTA
		const StepK<T>& K = a.k;
		const T dkxT = K.dkx, dkyT = K.dky;
		// update of one (kx, ky) entry for all fields with its coefficients
		// (A, B, couplings of k^2), pfc-relax.c:1215-1244
		auto apply = [&](int c, int kx, int ky, const cplx<T>(&Nv)[U], const T(&A)[U], const T(&Bn)[U],
		                 const T(&cu)[npairs<T, U>()]) {
			cplx<T> Mv[U];
#pragma unroll
			for (int u = 0; u < U; u++) Mv[u] = cscale(sm[(u * CC + c) * ld + pad<T>(ky)], K.invN);
			if constexpr (U > 1) {
				int p = 0;
#pragma unroll
				for (int u = 0; u < U - 1; u++)
#pragma unroll
					for (int v = u + 1; v < U; v++, p++) {
						Mv[u] = cadd(Mv[u], cscale(Nv[v], cu[p]));
						Mv[v] = cadd(Mv[v], cscale(Nv[u], cu[p]));
					}
			}
			const bool origin = (kx == 0 && ky == 0);
#pragma unroll
			for (int u = 0; u < U; u++) {
				cplx<T> nn = cadd(cscale(Nv[u], A[u]), cscale(Mv[u], Bn[u]));
				if (origin) nn = mk<T>((T)0, (T)0);
				// streaming (evict-first) accesses for the spectral state, read
				// and written once per step, leave L2 to `work`, which the next
				// pass reads back
				__stcs(a.spec + u * a.sstride + (long long)kx * Ny + ky, nn);
				sm[(u * CC + c) * ld + pad<T>(ky)] = nn;
			}
		};
		auto update = [&](int c, int kx, int ky, const cplx<T>(&Nv)[U]) {
			T A[U], Bn[U], cu[npairs<T, U>()];
			entry_coef<T, U>(K, step_k2<T>(kx, ky, Ny, dkxT, dkyT, a.g), A, Bn, cu);
			apply(c, kx, ky, Nv, A, Bn, cu);
		};
		if constexpr (C::CT && (CCC * NC / 2) % C::NT == 0) {
			// entries ky and NC - ky have the same k^2 (signed wave numbers ky and
			// -ky), so each thread takes such pairs and evaluates the coefficients
			// once for both; ky = 0 is paired with the self-mirrored NC / 2 and
			// evaluates them twice
			constexpr int HALF = NC / 2;
			constexpr int PH = CCC * HALF / C::NT;
			cplx<T> Nv[PH][2][U];
#pragma unroll
			for (int i = 0; i < PH; i++) {
				const int h = tid + i * C::NT;
				const int c = h / HALF, kb = h % HALF;
				const int ky2 = kb ? NC - kb : HALF;
				const long long col = (long long)(kx0 + c) * NC;
#pragma unroll
				for (int u = 0; u < U; u++) {
					Nv[i][0][u] = (c < ncol) ? __ldcs(a.spec + u * a.sstride + col + kb) : mk<T>((T)0, (T)0);
					Nv[i][1][u] = (c < ncol) ? __ldcs(a.spec + u * a.sstride + col + ky2) : mk<T>((T)0, (T)0);
				}
			}
#pragma unroll
			for (int i = 0; i < PH; i++) {
				const int h = tid + i * C::NT;
				const int c = h / HALF, kb = h % HALF;
				const int kx = kx0 + c;
				if (c < ncol) {
					T A[U], Bn[U], cu[npairs<T, U>()];
					entry_coef<T, U>(K, step_k2<T>(kx, kb, NC, dkxT, dkyT, a.g), A, Bn, cu);
					apply(c, kx, kb, Nv[i][0], A, Bn, cu);
					if (kb == 0) entry_coef<T, U>(K, step_k2<T>(kx, HALF, NC, dkxT, dkyT, a.g), A, Bn, cu);
					apply(c, kx, kb ? NC - kb : HALF, Nv[i][1], A, Bn, cu);
				}
			}
		} else if constexpr (C::CT && (CCC * NC) % C::NT == 0) {
			// every thread owns PER entries: issue all spectral-state loads first
			constexpr int PER = CCC * NC / C::NT;
			cplx<T> Nv[PER][U];
#pragma unroll
			for (int i = 0; i < PER; i++) {
				const int e = tid + i * C::NT;
				const int c = e / NC, ky = e % NC;
				const int kx = kx0 + c;
#pragma unroll
				for (int u = 0; u < U; u++)
					Nv[i][u] = (c < ncol) ? a.spec[u * a.sstride + (long long)kx * NC + ky] : mk<T>((T)0, (T)0);
			}
#pragma unroll
			for (int i = 0; i < PER; i++) {
				const int e = tid + i * C::NT;
				const int c = e / NC, ky = e % NC;
				if (c < ncol) update(c, kx0 + c, ky, Nv[i]);
			}
		} else {
			for (int e = tid; e < CC * Ny; e += nt) {
				const int c = e / Ny, ky = e - c * Ny;
				if (c >= ncol) continue;
				const int kx = kx0 + c;
				cplx<T> Nv[U];
#pragma unroll
				for (int u = 0; u < U; u++) Nv[u] = a.spec[u * a.sstride + (long long)kx * Ny + ky];
				update(c, kx, ky, Nv);
			}
		}
		if (kx0 == 0) ypass_mean_update<T, U>(a, tid, nt);
	} else if constexpr (MODE == YP_INIT) {
		const T invN = (T)(1.0 / ((double)Nx * (double)Ny));
		for (int e = tid; e < CC * Ny; e += nt) {
			const int c = e / Ny, ky = e - c * Ny;
			if (c >= ncol) continue;
			const int kx = kx0 + c;
			const long long si = (long long)kx * Ny + ky;
#pragma unroll
			for (int u = 0; u < U; u++) {
				cplx<T> nn = cscale(sm[(u * CC + c) * ld + pad<T>(ky)], invN);
				if (kx == 0 && ky == 0) nn = mk<T>((T)0, (T)0);
				a.spec[u * a.sstride + si] = nn;
				sm[(u * CC + c) * ld + pad<T>(ky)] = nn;
			}
		}
	} else {
		// YP_WEIGHT (U == 1): w(k) * spec[src] -> sm, with the weight's
		// parameters in a.wp (field index resolved on the host)
		const double ag = -0.5 / a.m.sigma / a.m.sigma;
		const cplx<T>* src = a.spec + a.wsrc * a.sstride;
		for (int e = tid; e < CC * Ny; e += nt) {
			const int c = e / Ny, ky = e - c * Ny;
			const int kx = kx0 + c;
			cplx<T> nn = mk<T>((T)0, (T)0);
			if (c < ncol && !(kx == 0 && ky == 0)) {
				const double k2 = k2_of(kx, ky, a.g, dx, dy);
				double w = 1.0;
				if (a.wkind == W_P) {
#pragma unroll
					for (int q = 0; q < MAXW; q++)
						if (q < a.wp.W) {
							const double d = a.wp.nu2[q] - k2;
							w *= a.wp.omega[q] * d * d + a.wp.phi[q];
						}
				} else if (a.wkind == W_G) {
					w = exp(ag * k2);
				} else if (a.wkind == W_Q) {
					const double d = a.wp.mu2 - k2;
					w = d * d;
				} else if (a.wkind == W_GS || a.wkind == W_DG) {
					w = exp(-0.5 * k2 / (a.wp.gs * a.wp.gs));
				}
				const long long si = (long long)kx * Ny + ky;
				if (a.wkind == W_OR) {
					// orientation kernel K = exp(-(|k| - 1)^2 / (2 sk^2)) exp(i fold phi),
					// fields.c:143-153; real and imaginary parts are even in k
					// for even fold, so each part maps the field pair to a real field
					const double kxv = kx * a.g.dkx;
					const double kyv = (ky < Ny / 2 ? ky : ky - Ny) * a.g.dky;
					const double q = sqrt(k2) - 1.0;
					const double rad = exp(-0.5 * q * q / (a.wp.sk * a.wp.sk));
					double sn, cs;
					sincos(a.wp.fold * atan2(kyv, kxv), &sn, &cs);
					const T kr = (T)(rad * cs), ki = (T)(rad * sn);
					const cplx<T> s0 = a.spec[si], s1 = a.spec[a.sstride + si];
					nn = a.wp.part == 0 ? csub(cscale(s0, kr), cscale(s1, ki)) : cadd(cscale(s0, ki), cscale(s1, kr));
				} else if (a.wkind == W_DG) {
					// i k_dir G(k) times the field (fields.c:260-271 on the smoothed spectrum)
					const double kd = a.wp.dir == 0 ? kx * a.g.dkx : (ky < Ny / 2 ? ky : ky - Ny) * a.g.dky;
					const cplx<T> v = src[si];
					const T f = (T)(kd * w);
					nn = mk<T>(-f * v.y, f * v.x);
				} else {
					nn = cscale(src[si], (T)w);
				}
			}
			sm[c * ld + pad<T>(ky)] = nn;
		}
	}

	if constexpr (MODE == YP_STEP || MODE == YP_INIT) {
		// kx = 0 and (even Nx) kx = Nx/2 columns: keep them exactly Hermitian
		const bool has0 = (kx0 == 0);
		const int kn = (Nx % 2 == 0) ? Nx / 2 : -1;
		const bool hasn = (kn >= kx0 && kn < kx0 + ncol);
		if (has0 || hasn) {
			__syncthreads();
#pragma unroll
			for (int u = 0; u < U; u++) {
				if (has0) hermitian_column<T>(sm + (u * CC) * ld, a.spec + u * a.sstride, Ny, tid, nt);
				if (hasn)
					hermitian_column<T>(sm + (u * CC + (kn - kx0)) * ld, a.spec + u * a.sstride + (long long)kn * Ny, Ny,
					                    tid, nt);
			}
		}
	}
	__syncthreads();
	if constexpr (REGIO) {
		if (regio) {
			ct_pass<NCX, PLX::radix(0), PLX::ns(0), PLX::twoff(0), C::S, C::NT, +1, T>(sm, tws, tid);
			ct_middle<NCX, MAXE, C::S, C::NT, +1, T>(sm, tws, tid);
			RBY rb;
			ct_last_to_regs<NCX, MAXE, C::S, C::NT, +1, T>(sm, tws, rb, tid);
#pragma unroll
			for (int i = 0; i < RBY::NB; i++) {
				const int p = RBY::seq(tid, i);
				if (p % CCX < ncol) {
#pragma unroll
					for (int r = 0; r < MAXE; r++) a.work[gaddr(p, RBY::pos(tid, i, r))] = rb.v[i][r];
				}
			}
			return;
		}
	}
	if constexpr (C::CT) fft_ct<NC, MAXE, C::S, C::NSUB, C::NT, +1, T>(sm, tws, tid);
	else fft_batches<+1, MAXE, T>(sm, ld, S, a.sb, a.plan, a.tw, tid, nt);

#pragma unroll
	for (int u = 0; u < U; u++) {
		cplx<T>* dst = a.work + u * a.wstride + (long long)kx0 * R;
		for (int e = tid; e < ntile * chunk; e += nt) {
			const int t = e / chunk, rem = e - t * chunk;
			const int c = rem / R, r = rem - c * R;
			if (c < ncol) dst[t * tileH + rem] = sm[(u * CC + c) * ld + pad<T>(t * R + r)];
		}
	}
}

// ------------------------------------------------------- Parseval energy --
// <f> gradient/coupling part in k space, for several box sizes at once:
//   sum over the half spectrum with weight 1 (kx = 0, Nx/2) or 2 of
//   1/2 beta_uu P_u |N_u|^2 + sum_{u<v} (beta_uv (mu2_uv - k2)^2 + eps_uv G^2) Re(N_u conj N_v),
// which equals the mean over the grid of the beta and epsilon terms of
// pfc-relax.c:1101-1111 (Parseval; N^ normalised by 1/(Nx Ny)).
struct Trials {
	double dx[MAX_TRIAL], dy[MAX_TRIAL];
};

template <typename T, int U>
__global__ void __launch_bounds__(256) kspace_energy_kernel(const cplx<T>* __restrict__ spec, long long sstride, const Model m,
                                                           const Geom g, int ntrial, const Trials tr, double* out,
                                                           double* part) {
	double acc[MAX_TRIAL];
#pragma unroll
	for (int t = 0; t < MAX_TRIAL; t++) acc[t] = 0.0;
	const long long total = (long long)g.H * g.Ny;
	const double ag = -1.0 / m.sigma / m.sigma; // G^2 = exp(-k2 / sigma^2)
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
		const int kx = (int)(i / g.Ny), ky = (int)(i - (long long)kx * g.Ny);
		const double wgt = (kx == 0 || 2 * kx == g.Nx) ? 1.0 : 2.0;
		double nr[U], ni[U];
#pragma unroll
		for (int u = 0; u < U; u++) {
			const cplx<T> v = spec[u * sstride + i];
			nr[u] = (double)v.x;
			ni[u] = (double)v.y;
		}
#pragma unroll
		for (int t = 0; t < MAX_TRIAL; t++) {
			if (t < ntrial) {
				const double k2 = k2_of(kx, ky, g, tr.dx[t], tr.dy[t]);
				double e = 0.0;
#pragma unroll
				for (int u = 0; u < U; u++) e += 0.5 * m.beta[u][u] * P_of<double>(m, u, k2) * (nr[u] * nr[u] + ni[u] * ni[u]);
				if constexpr (U > 1) {
					const double G2 = exp(ag * k2);
#pragma unroll
					for (int u = 0; u < U - 1; u++)
#pragma unroll
						for (int v = u + 1; v < U; v++) {
							const double d = m.mu2[u][v] - k2;
							e += (m.beta[u][v] * d * d + m.epsilon[u][v] * G2) * (nr[u] * nr[v] + ni[u] * ni[v]);
						}
				}
				acc[t] += wgt * e;
			}
		}
	}
	block_reduce_put<MAX_TRIAL>(acc, part ? part + (long long)blockIdx.x * MAX_TRIAL : out, part != nullptr);
}

// -------------------------------------------------------------- launchers --

template <typename T, int U, int MODE, int NC, int CCC, int RC, bool FUSEDK = true>
__global__ void __launch_bounds__(YCfg<T, U, NC, CCC, RC, FUSEDK>::NT, YCfg<T, U, NC, CCC, RC, FUSEDK>::MINB)
    ypass_kernel(const YArgs<T> a, int ngroups) {
	asm volatile("griddepcontrol.wait;" ::: "memory"); // as in xpass_kernel
	asm volatile("griddepcontrol.launch_dependents;");
	// column groups blockIdx.x, + gridDim.x, ... (as the x-pass's tiles)
	for (int g = blockIdx.x; g < ngroups; g += gridDim.x) {
		if (g != (int)blockIdx.x) __syncthreads();
		ypass_body<T, U, MODE, NC, CCC, RC, FUSEDK>(a, g, g == (int)blockIdx.x, (g - (int)blockIdx.x) / (int)gridDim.x);
	}
}

// ------------------------------------------------------------------ batch --
// Many independent relaxations of runtime sizes in one launch: block b runs
// tile (x-pass) or column group (y-pass) blk_local[b] of problem blk_prob[b],
// whose arguments sit in global memory. Launched with the largest thread count
// and shared memory any problem needs; the runtime-plan bodies use whatever
// threads they get.
template <typename T>
__global__ void __launch_bounds__(MAXNT, 1)
    xpass_batch_kernel(const XArgs<T>* __restrict__ probs, const int* __restrict__ blk_prob,
                       const int* __restrict__ blk_local) {
	const XArgs<T>& a = probs[blk_prob[blockIdx.x]];
	const int local = blk_local[blockIdx.x];
	switch (a.m.U) {
	case 1: xpass_body<T, 1, XP_STEP, 0, 0>(a, local); break;
	case 2: xpass_body<T, 2, XP_STEP, 0, 0>(a, local); break;
	case 3: xpass_body<T, 3, XP_STEP, 0, 0>(a, local); break;
	case 4: xpass_body<T, 4, XP_STEP, 0, 0>(a, local); break;
	}
}

template <typename T>
__global__ void __launch_bounds__(MAXNT, 1)
    ypass_batch_kernel(const YArgs<T>* __restrict__ probs, const int* __restrict__ blk_prob,
                       const int* __restrict__ blk_local) {
	const YArgs<T>& a = probs[blk_prob[blockIdx.x]];
	const int local = blk_local[blockIdx.x];
	switch (a.m.U) {
	case 1: ypass_body<T, 1, YP_STEP, 0, 0, 0>(a, local); break;
	case 2: ypass_body<T, 2, YP_STEP, 0, 0, 0>(a, local); break;
	case 3: ypass_body<T, 3, YP_STEP, 0, 0, 0>(a, local); break;
	case 4: ypass_body<T, 4, YP_STEP, 0, 0, 0>(a, local); break;
	}
}

// Raises the dynamic shared-memory limit of a kernel once per device.
// Batched STEP passes of the kernels specialised on a length: every block of
// the launch belongs to a problem of that length and field count (one launch
// per such class of a batch), so the body is the single-problem one.
template <typename T, int U, int MODE, int NC, int RC>
__global__ void __launch_bounds__(XCfg<T, U, NC, RC>::NT, XCfg<T, U, NC, RC>::MINB)
    xpass_ct_batch_kernel(const XArgs<T>* __restrict__ probs, const int* __restrict__ blk_prob,
                          const int* __restrict__ blk_local) {
	xpass_body<T, U, MODE, NC, RC>(probs[blk_prob[blockIdx.x]], blk_local[blockIdx.x]);
}

template <typename T, int U, int MODE, int NC, int CCC, int RC, bool FUSEDK>
__global__ void __launch_bounds__(YCfg<T, U, NC, CCC, RC, FUSEDK>::NT, YCfg<T, U, NC, CCC, RC, FUSEDK>::MINB)
    ypass_ct_batch_kernel(const YArgs<T>* __restrict__ probs, const int* __restrict__ blk_prob,
                          const int* __restrict__ blk_local) {
	ypass_body<T, U, MODE, NC, CCC, RC, FUSEDK>(probs[blk_prob[blockIdx.x]], blk_local[blockIdx.x]);
}

template <typename K> static void smem_attr(K k, unsigned long long& mask) {
	int dev = 0;
	cudaGetDevice(&dev);
	const unsigned long long bit = 1ull << (dev & 63);
	if (!(mask & bit)) {
		int optin = 0;
		cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
		cudaFuncAttributes fa;
		cudaFuncGetAttributes(&fa, k);
		cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
		mask |= bit;
	}
}

// Grid of the compile-time specialised FP64 kernels: as many CTAs as fit on the
// device at once (cached per kernel), each looping over several tiles or column
// groups, so the 64 KB twiddle table loads once per CTA (1.8 % more steps/s at
// 4096^2; the FP32 kernels measured 4.7 % slower this way and keep one CTA per
// tile). PFCG_PERSISTENT=0 launches one CTA per tile in FP64 too.
template <typename K> static int resident_grid(K k, const LaunchCfg& c, int& resident) {
	if (resident == 0) {
		const char* e = getenv("PFCG_PERSISTENT");
		int dev = 0, sms = 0, per = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, c.block, c.smem);
		resident = (e && e[0] == '0') || per < 1 || sms < 1 ? -1 : per * sms;
	}
	return resident > 0 && resident < c.grid ? resident : c.grid;
}

// Launch of the x- and y-pass kernels as programmatic dependent launches: the
// next pass's CTAs may be scheduled while the last wave of the previous one
// drains, and each kernel waits for the previous kernel's completion and
// memory (griddepcontrol.wait, its first statement) before touching anything
// that kernel writes. PFCG_PDL=0 launches them plainly. Persistent grids (one
// CTA per resident slot, the FP64 specialised kernels) launch plainly too:
// with every slot taken there is no drain to overlap, and dependent launches
// measured 2 % slower there (1.041 against 1.019 ms per 4096^2 U=2 FP64 step).
static bool pdl_on() {
	static const int on = [] {
		const char* e = std::getenv("PFCG_PDL");
		return (e && e[0] == '0') ? 0 : 1;
	}();
	return on != 0;
}

template <typename K, typename A>
static cudaError_t pdl_launch(K k, int grid, int block, int smem, cudaStream_t s, const A& a, int n) {
	if (!pdl_on() || grid < n) {
		k<<<grid, block, smem, s>>>(a, n);
		return cudaGetLastError();
	}
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3(grid);
	cfg.blockDim = dim3(block);
	cfg.dynamicSmemBytes = smem;
	cfg.stream = s;
	cudaLaunchAttribute at[1];
	at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	at[0].val.programmaticStreamSerializationAllowed = 1;
	cfg.attrs = at;
	cfg.numAttrs = 1;
	return cudaLaunchKernelEx(&cfg, k, a, n);
}

template <typename T, int U, int MODE, int NC, int RC>
static cudaError_t xlaunch(const XArgs<T>& a, const LaunchCfg& c, cudaStream_t s) {
	auto k = xpass_kernel<T, U, MODE, NC, RC>;
	static unsigned long long mask = 0;
	static int resident = 0;
	smem_attr(k, mask);
	const int grid = NC > 0 && std::is_same<T, double>::value ? resident_grid(k, c, resident) : c.grid;
	return pdl_launch(k, grid, c.block, c.smem, s, a, c.grid);
}

// Compile-time specialisations of the STEP kernels: (length, rows per tile,
// columns per y-pass CTA) for the sizes the workloads use; other sizes and
// modes run the runtime-plan kernels.
template <typename T, int U, int MODE, int NC, int CCC, int RC, bool FUSEDK = true>
static cudaError_t ylaunch(const YArgs<T>& a, const LaunchCfg& c, cudaStream_t s) {
	auto k = ypass_kernel<T, U, MODE, NC, CCC, RC, FUSEDK>;
	static unsigned long long mask = 0;
	static int resident = 0;
	smem_attr(k, mask);
	const int grid = NC > 0 && std::is_same<T, double>::value ? resident_grid(k, c, resident) : c.grid;
	return pdl_launch(k, grid, c.block, c.smem, s, a, c.grid);
}

template <typename T> struct Spec;
// Rows per x-pass tile (xr) and columns per y-pass group (ycc) of the kernels
// specialised on a compile-time length N, 0 where there is none. The row tile
// is also the layout of `work` for the runtime-plan modes (evaluate, c2r, r2c),
// so U * xr stays within MAX_CH: an FP32 x-pass CTA runs U * xr * N / (2 M)
// threads for the main radix M = ct_maxe (512 at N = 4096 and 2048, N / 4
// below with M = 16, 192 at N = 384). A y-pass CTA runs U * ycc * N / M
// threads: 512, or 384 at N = 384, 768 and 1536 (8^2 * 6, 16^2 * 3, 16^2 * 6).
template <> struct Spec<float> {
	static constexpr int x1(int N) {
		return N == 4096 ? 4 : (N == 2048 || N == 1536 || N == 1024 || N == 768 || N == 512 || N == 384 || N == 256) ? 8 : 0;
	}
	static constexpr int y1(int N) {
		return N == 4096 ? 2 : N == 2048 || N == 1536 ? 4 : N == 1024 || N == 768 || N == 384 ? 8 : N == 512 ? 16 : N == 256 ? 32 : 0;
	}
	static constexpr int xr(int U, int N) { return U == 1 ? x1(N) : U == 2 ? x1(N) / 2 : 0; }
	static constexpr int ycc(int U, int N) { return U == 1 ? y1(N) : U == 2 ? y1(N) / 2 : 0; }
};
template <> struct Spec<double> {
	static constexpr int xr(int U, int N) {
		return N == 4096 ? (U == 1 ? 2 : U == 2 ? 1 : 0) : N == 2048 ? (U == 1 ? 4 : U == 2 ? 2 : 0) : 0;
	}
	static constexpr int ycc(int U, int N) {
		return N == 4096 ? (U == 1 ? 1 : U == 2 ? 1 : 0) : N == 2048 ? (U == 1 ? 2 : U == 2 ? 1 : 0) : 0;
	}
};

template <typename T, int U> static bool x_is_spec(const XArgs<T>& a) {
	return Spec<T>::xr(U, a.g.Nx) > 0 && a.g.R == Spec<T>::xr(U, a.g.Nx);
}
template <typename T, int U> static bool y_is_spec(const YArgs<T>& a) {
	return Spec<T>::ycc(U, a.g.Ny) > 0 && a.g.CC == Spec<T>::ycc(U, a.g.Ny) && a.g.R == Spec<T>::xr(U, a.g.Ny);
}

// STEP passes of the specialised kernels of length N. The FP32 lengths below
// 2048 are instantiated in kernels_f32_<N>.cu, one file each, so that they
// compile in parallel.
template <typename T, int U, int N> cudaError_t ct_xstep(const XArgs<T>& a, const LaunchCfg& c, cudaStream_t s) {
	return xlaunch<T, U, XP_STEP, N, Spec<T>::xr(U, N)>(a, c, s);
}
template <typename T, int U, int N> cudaError_t ct_ystep(const YArgs<T>& a, const LaunchCfg& c, cudaStream_t s) {
	// c.spec: 1 = specialised (fused where possible), 2 = specialised, never fused
	if (c.spec == 2) return ylaunch<T, U, YP_STEP, N, Spec<T>::ycc(U, N), Spec<T>::xr(U, N), false>(a, c, s);
	return ylaunch<T, U, YP_STEP, N, Spec<T>::ycc(U, N), Spec<T>::xr(U, N)>(a, c, s);
}

// Batched STEP passes over nblk blocks of problems of length N (nblk = 0 only
// sets the kernel's shared-memory limit, which must not happen under capture).
template <typename T, int U, int N>
cudaError_t ct_xbatch(const XArgs<T>* probs, const int* bp, const int* bl, int nblk, const LaunchCfg& c, cudaStream_t s) {
	auto k = xpass_ct_batch_kernel<T, U, XP_STEP, N, Spec<T>::xr(U, N)>;
	static unsigned long long mask = 0;
	smem_attr(k, mask);
	if (nblk > 0) k<<<nblk, c.block, c.smem, s>>>(probs, bp, bl);
	return cudaGetLastError();
}
template <typename T, int U, int N>
cudaError_t ct_ybatch(const YArgs<T>* probs, const int* bp, const int* bl, int nblk, const LaunchCfg& c, cudaStream_t s) {
	constexpr int CC = Spec<T>::ycc(U, N), R = Spec<T>::xr(U, N);
	static unsigned long long m1 = 0, m2 = 0;
	if (c.spec == 2) {
		auto k = ypass_ct_batch_kernel<T, U, YP_STEP, N, CC, R, false>;
		smem_attr(k, m2);
		if (nblk > 0) k<<<nblk, c.block, c.smem, s>>>(probs, bp, bl);
	} else {
		auto k = ypass_ct_batch_kernel<T, U, YP_STEP, N, CC, R, true>;
		smem_attr(k, m1);
		if (nblk > 0) k<<<nblk, c.block, c.smem, s>>>(probs, bp, bl);
	}
	return cudaGetLastError();
}

#ifndef PFCG_CT_TU
#define PFCG_CT_TU 0
#endif
#define PFCG_CT_DECL(EXT, U, N)                                                                                        \
	EXT template cudaError_t ct_xstep<float, U, N>(const XArgs<float>&, const LaunchCfg&, cudaStream_t);               \
	EXT template cudaError_t ct_ystep<float, U, N>(const YArgs<float>&, const LaunchCfg&, cudaStream_t);               \
	EXT template cudaError_t ct_xbatch<float, U, N>(const XArgs<float>*, const int*, const int*, int, const LaunchCfg&,  \
	                                                cudaStream_t);                                                     \
	EXT template cudaError_t ct_ybatch<float, U, N>(const YArgs<float>*, const int*, const int*, int, const LaunchCfg&,  \
	                                                cudaStream_t);
#if PFCG_CT_TU != 256
PFCG_CT_DECL(extern, 1, 256)
PFCG_CT_DECL(extern, 2, 256)
#endif
#if PFCG_CT_TU != 384
PFCG_CT_DECL(extern, 1, 384)
PFCG_CT_DECL(extern, 2, 384)
#endif
#if PFCG_CT_TU != 512
PFCG_CT_DECL(extern, 1, 512)
PFCG_CT_DECL(extern, 2, 512)
#endif
#if PFCG_CT_TU != 768
PFCG_CT_DECL(extern, 1, 768)
PFCG_CT_DECL(extern, 2, 768)
#endif
#if PFCG_CT_TU != 1024
PFCG_CT_DECL(extern, 1, 1024)
PFCG_CT_DECL(extern, 2, 1024)
#endif
#if PFCG_CT_TU != 1536
PFCG_CT_DECL(extern, 1, 1536)
PFCG_CT_DECL(extern, 2, 1536)
#endif
#if PFCG_CT_TU != 2048
PFCG_CT_DECL(extern, 1, 2048)
PFCG_CT_DECL(extern, 2, 2048)
#endif
#if PFCG_CT_TU != 4096
PFCG_CT_DECL(extern, 1, 4096)
PFCG_CT_DECL(extern, 2, 4096)
#endif

template <typename T, int U> static cudaError_t ct_xdispatch(const XArgs<T>& a, const LaunchCfg& c, cudaStream_t s) {
	switch (a.g.Nx) {
	case 4096: return ct_xstep<T, U, 4096>(a, c, s);
	case 2048: return ct_xstep<T, U, 2048>(a, c, s);
	}
	if constexpr (std::is_same<T, float>::value) {
		switch (a.g.Nx) {
		case 1536: return ct_xstep<T, U, 1536>(a, c, s);
		case 1024: return ct_xstep<T, U, 1024>(a, c, s);
		case 768: return ct_xstep<T, U, 768>(a, c, s);
		case 512: return ct_xstep<T, U, 512>(a, c, s);
		case 384: return ct_xstep<T, U, 384>(a, c, s);
		case 256: return ct_xstep<T, U, 256>(a, c, s);
		}
	}
	return cudaErrorInvalidValue;
}
template <typename T, int U> static cudaError_t ct_ydispatch(const YArgs<T>& a, const LaunchCfg& c, cudaStream_t s) {
	switch (a.g.Ny) {
	case 4096: return ct_ystep<T, U, 4096>(a, c, s);
	case 2048: return ct_ystep<T, U, 2048>(a, c, s);
	}
	if constexpr (std::is_same<T, float>::value) {
		switch (a.g.Ny) {
		case 1536: return ct_ystep<T, U, 1536>(a, c, s);
		case 1024: return ct_ystep<T, U, 1024>(a, c, s);
		case 768: return ct_ystep<T, U, 768>(a, c, s);
		case 512: return ct_ystep<T, U, 512>(a, c, s);
		case 384: return ct_ystep<T, U, 384>(a, c, s);
		case 256: return ct_ystep<T, U, 256>(a, c, s);
		}
	}
	return cudaErrorInvalidValue;
}

// One launch of the batched STEP pass (pass 0 = x, 1 = y) of the class of
// problems with U fields and length N; cudaErrorInvalidValue where the size
// has no specialised kernel.
template <typename T, int U>
static cudaError_t ct_batch_u(int pass, int N, const void* probs, const int* bp, const int* bl, int nblk,
                              const LaunchCfg& c, cudaStream_t s) {
#define PFCG_CT_CASE(NN)                                                                                              \
	case NN:                                                                                                           \
		return pass == 0 ? ct_xbatch<T, U, NN>((const XArgs<T>*)probs, bp, bl, nblk, c, s)                            \
		                 : ct_ybatch<T, U, NN>((const YArgs<T>*)probs, bp, bl, nblk, c, s);
	switch (N) {
		PFCG_CT_CASE(4096)
		PFCG_CT_CASE(2048)
	}
	if constexpr (std::is_same<T, float>::value) {
		switch (N) {
			PFCG_CT_CASE(1536)
			PFCG_CT_CASE(1024)
			PFCG_CT_CASE(768)
			PFCG_CT_CASE(512)
			PFCG_CT_CASE(384)
			PFCG_CT_CASE(256)
		}
	}
#undef PFCG_CT_CASE
	return cudaErrorInvalidValue;
}
template <typename T>
cudaError_t launch_ct_batch(int pass, int U, int N, const void* probs, const int* bp, const int* bl, int nblk,
                            const LaunchCfg& c, cudaStream_t s) {
	if (U == 1) return ct_batch_u<T, 1>(pass, N, probs, bp, bl, nblk, c, s);
	if (U == 2) return ct_batch_u<T, 2>(pass, N, probs, bp, bl, nblk, c, s);
	return cudaErrorInvalidValue;
}
template <typename T>
cudaError_t launch_generic_batch(int pass, const void* probs, const int* bp, const int* bl, int nblk, int threads,
                                 int smem, cudaStream_t s) {
	prepare_batch_kernels<T>();
	if (nblk <= 0) return cudaGetLastError();
	if (pass == 0) xpass_batch_kernel<T><<<nblk, threads, smem, s>>>((const XArgs<T>*)probs, bp, bl);
	else ypass_batch_kernel<T><<<nblk, threads, smem, s>>>((const YArgs<T>*)probs, bp, bl);
	return cudaGetLastError();
}

template <typename T, int U> static cudaError_t xlaunch_mode(int mode, const XArgs<T>& a, const LaunchCfg& c, cudaStream_t s) {
	switch (mode) {
	case XP_STEP:
		if constexpr (U <= 2)
			if (c.spec && x_is_spec<T, U>(a)) return ct_xdispatch<T, U>(a, c, s);
		return xlaunch<T, U, XP_STEP, 0, 0>(a, c, s);
	case XP_EVAL: return xlaunch<T, U, XP_EVAL, 0, 0>(a, c, s);
	case XP_C2R: return xlaunch<T, U, XP_C2R, 0, 0>(a, c, s);
	case XP_R2C: return xlaunch<T, U, XP_R2C, 0, 0>(a, c, s);
	}
	return cudaErrorInvalidValue;
}

template <typename T> cudaError_t launch_xpass(int mode, const XArgs<T>& a, const LaunchCfg& c, cudaStream_t s) {
	switch (a.m.U) {
	case 1: return xlaunch_mode<T, 1>(mode, a, c, s);
	case 2: return xlaunch_mode<T, 2>(mode, a, c, s);
	case 3: return xlaunch_mode<T, 3>(mode, a, c, s);
	case 4: return xlaunch_mode<T, 4>(mode, a, c, s);
	}
	return cudaErrorInvalidValue;
}


template <typename T, int U> static cudaError_t ystep(const YArgs<T>& a, const LaunchCfg& c, cudaStream_t s) {
	if (c.spec && y_is_spec<T, U>(a)) return ct_ydispatch<T, U>(a, c, s);
	return ylaunch<T, U, YP_STEP, 0, 0, 0>(a, c, s);
}

template <typename T> cudaError_t launch_ypass(int mode, const YArgs<T>& a, const LaunchCfg& c, cudaStream_t s) {
	if (mode == YP_WEIGHT) return ylaunch<T, 1, YP_WEIGHT, 0, 0, 0>(a, c, s);
	if (mode == YP_STEP) {
		switch (a.m.U) {
		case 1: return ystep<T, 1>(a, c, s);
		case 2: return ystep<T, 2>(a, c, s);
		case 3: return ylaunch<T, 3, YP_STEP, 0, 0, 0>(a, c, s);
		case 4: return ylaunch<T, 4, YP_STEP, 0, 0, 0>(a, c, s);
		}
	}
	if (mode == YP_INIT) {
		switch (a.m.U) {
		case 1: return ylaunch<T, 1, YP_INIT, 0, 0, 0>(a, c, s);
		case 2: return ylaunch<T, 2, YP_INIT, 0, 0, 0>(a, c, s);
		case 3: return ylaunch<T, 3, YP_INIT, 0, 0, 0>(a, c, s);
		case 4: return ylaunch<T, 4, YP_INIT, 0, 0, 0>(a, c, s);
		}
	}
	return cudaErrorInvalidValue;
}

template <typename T> void prepare_batch_kernels() {
	static unsigned long long mx = 0, my = 0;
	smem_attr(xpass_batch_kernel<T>, mx);
	smem_attr(ypass_batch_kernel<T>, my);
}

template <typename T>
cudaError_t launch_kspace_energy(const cplx<T>* spec, long long sstride, const Model& m, const Geom& g, int ntrial,
                                 const double* dxs, const double* dys, double* out, double* part, cudaStream_t s) {
	Trials tr;
	for (int t = 0; t < MAX_TRIAL; t++) {
		tr.dx[t] = t < ntrial ? dxs[t] : 1.0;
		tr.dy[t] = t < ntrial ? dys[t] : 1.0;
	}
	const long long total = (long long)g.H * g.Ny;
	int grid = (int)((total + 255) / 256);
	if (grid > KSPACE_MAX_BLOCKS) grid = KSPACE_MAX_BLOCKS;
	switch (m.U) {
	case 1: kspace_energy_kernel<T, 1><<<grid, 256, 0, s>>>(spec, sstride, m, g, ntrial, tr, out, part); break;
	case 2: kspace_energy_kernel<T, 2><<<grid, 256, 0, s>>>(spec, sstride, m, g, ntrial, tr, out, part); break;
	case 3: kspace_energy_kernel<T, 3><<<grid, 256, 0, s>>>(spec, sstride, m, g, ntrial, tr, out, part); break;
	case 4: kspace_energy_kernel<T, 4><<<grid, 256, 0, s>>>(spec, sstride, m, g, ntrial, tr, out, part); break;
	default: return cudaErrorInvalidValue;
	}
	cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess || !part) return e;
	return launch_sum_parts(part, grid, MAX_TRIAL, out, s);
}


} // namespace pfcg
