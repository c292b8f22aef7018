// Shared-memory mixed-radix FFT building blocks for sm_100a.
//
// One CTA transforms a batch of P complex sequences of length N that sit in
// shared memory. Each pass is one radix-R Stockham autosort stage (Govindaraju
// et al., "High performance discrete Fourier transforms on graphics
// processors", SC 2008): butterfly j of a sequence reads x[j + r*N/R]
// (r = 0..R-1, consecutive threads read consecutive words), multiplies by the
// twiddle W^(r * (j mod Ns) * N/(Ns*R)), does a length-R DFT in registers and
// writes y[(j/Ns)*Ns*R + (j mod Ns) + r*Ns]. The output comes out in natural
// order, so no bit reversal is needed.
//
// The pass is done in place: every thread first loads all the butterflies it
// owns into registers, the CTA synchronises, then every thread writes. A
// thread owns at most MAXE/R butterflies of a pass (MAXE elements).
//
// Shared memory is padded by one element every 128 bytes (pad()) so the
// strided writes of the first passes do not hit one bank.
//
// Twiddles come from a per-length table tw[k] = exp(-2 pi i k / N) that the host
// computes in double precision and stores in the transform precision; the
// backward transform uses the conjugate.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pfcg {

template <typename T> struct cplx_t;
template <> struct cplx_t<float> { using type = float2; };
template <> struct cplx_t<double> { using type = double2; };
template <typename T> using cplx = typename cplx_t<T>::type;

template <typename T> __host__ __device__ __forceinline__ cplx<T> mk(T x, T y) { cplx<T> r; r.x = x; r.y = y; return r; }
template <typename V> __host__ __device__ __forceinline__ V cadd(V a, V b) { V r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename V> __host__ __device__ __forceinline__ V csub(V a, V b) { V r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename V> __host__ __device__ __forceinline__ V cmul(V a, V b) {
	V r;
	r.x = a.x * b.x - a.y * b.y;
	r.y = a.x * b.y + a.y * b.x;
	return r;
}
template <typename V> __host__ __device__ __forceinline__ V cconj(V a) { a.y = -a.y; return a; }
template <typename V, typename T> __host__ __device__ __forceinline__ V cscale(V a, T s) { a.x *= s; a.y *= s; return a; }
// a * (sign * i)
template <int SIGN, typename V> __host__ __device__ __forceinline__ V cmul_si(V a) {
	V r;
	if (SIGN < 0) { r.x = a.y; r.y = -a.x; }
	else { r.x = -a.y; r.y = a.x; }
	return r;
}

// Padded shared-memory index: one spare element after every 128 bytes.
template <typename T> struct Pad;
template <> struct Pad<float> { static constexpr int SHIFT = 4; };
template <> struct Pad<double> { static constexpr int SHIFT = 3; };
template <typename T> __device__ __host__ __forceinline__ int pad(int i) { return i + (i >> Pad<T>::SHIFT); }
template <typename T> __host__ __device__ inline int padded_len(int n) { return n + (n >> Pad<T>::SHIFT) + 1; }

// ---------------------------------------------------------------- DFTs ---
// In-register DFT of length R: v'[k] = sum_r v[r] exp(SIGN 2 pi i r k / R).

template <int SIGN, typename T> __host__ __device__ __forceinline__ void dft2(cplx<T>* v) {
	cplx<T> a = v[0], b = v[1];
	v[0] = cadd(a, b);
	v[1] = csub(a, b);
}

template <int SIGN, typename T> __host__ __device__ __forceinline__ void dft4(cplx<T>* v) {
	cplx<T> a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
	cplx<T> b0 = cadd(v[1], v[3]), b1 = cmul_si<SIGN>(csub(v[1], v[3]));
	v[0] = cadd(a0, b0);
	v[1] = cadd(a1, b1);
	v[2] = csub(a0, b0);
	v[3] = csub(a1, b1);
}

// length 8 as 2 x 4: inner DFT4 on even/odd halves, twiddle by exp(SIGN 2 pi i k/8)
template <int SIGN, typename T> __host__ __device__ __forceinline__ void dft8(cplx<T>* v) {
	const T h = (T)0.70710678118654752440084436210485; // 1/sqrt(2)
	cplx<T> e[4] = {v[0], v[2], v[4], v[6]};
	cplx<T> o[4] = {v[1], v[3], v[5], v[7]};
	dft4<SIGN, T>(e);
	dft4<SIGN, T>(o);
	// o[k] *= exp(SIGN 2 pi i k / 8)
	o[1] = mk<T>(h * (o[1].x - SIGN * o[1].y), h * (o[1].y + SIGN * o[1].x));
	o[2] = cmul_si<SIGN>(o[2]);
	o[3] = mk<T>(h * (-o[3].x - SIGN * o[3].y), h * (-o[3].y + SIGN * o[3].x));
#pragma unroll
	for (int k = 0; k < 4; k++) {
		v[k] = cadd(e[k], o[k]);
		v[k + 4] = csub(e[k], o[k]);
	}
}

// length 16 as 4 x 4 (four DFT4 on stride-4 subsequences, twiddles, four DFT4)
template <int SIGN, typename T> __host__ __device__ __forceinline__ void dft16(cplx<T>* v) {
	const T c1 = (T)0.92387953251128675612818318939679;  // cos(pi/8)
	const T s1 = (T)0.38268343236508977172845998403040;  // sin(pi/8)
	const T h = (T)0.70710678118654752440084436210485;   // cos(pi/4)
	cplx<T> a[4][4];
#pragma unroll
	for (int q = 0; q < 4; q++) {
#pragma unroll
		for (int r = 0; r < 4; r++) a[q][r] = v[4 * r + q];
		dft4<SIGN, T>(a[q]);
	}
	// a[q][k] *= exp(SIGN 2 pi i q k / 16), q, k in 0..3
	// q=1: k=1 (c1,s1), k=2 (h,h), k=3 (s1,c1)
	// q=2: k=1 (h,h), k=2 i, k=3 (-h,h)
	// q=3: k=1 (s1,c1), k=2 (-h,h), k=3 (-c1,-s1)
	const T cs[4][4][2] = {
		{{1, 0}, {1, 0}, {1, 0}, {1, 0}},
		{{1, 0}, {c1, s1}, {h, h}, {s1, c1}},
		{{1, 0}, {h, h}, {0, 1}, {-h, h}},
		{{1, 0}, {s1, c1}, {-h, h}, {-c1, -s1}},
	};
#pragma unroll
	for (int q = 1; q < 4; q++)
#pragma unroll
		for (int k = 1; k < 4; k++) {
			cplx<T> w = mk<T>(cs[q][k][0], SIGN * cs[q][k][1]);
			a[q][k] = cmul(a[q][k], w);
		}
#pragma unroll
	for (int k = 0; k < 4; k++) {
		cplx<T> b[4] = {a[0][k], a[1][k], a[2][k], a[3][k]};
		dft4<SIGN, T>(b);
#pragma unroll
		for (int s = 0; s < 4; s++) v[k + 4 * s] = b[s];
	}
}

template <int SIGN, typename T> __host__ __device__ __forceinline__ void dft3(cplx<T>* v) {
	const T c = (T)-0.5;
	const T s = (T)SIGN * (T)0.86602540378443864676372317075294; // SIGN sin(2 pi/3)
	cplx<T> t1 = cadd(v[1], v[2]);
	cplx<T> t2 = csub(v[1], v[2]);
	cplx<T> a = v[0];
	v[0] = cadd(a, t1);
	cplx<T> m1 = mk<T>(a.x + c * t1.x, a.y + c * t1.y);
	cplx<T> m2 = mk<T>(-s * t2.y, s * t2.x); // i s t2
	v[1] = cadd(m1, m2);
	v[2] = csub(m1, m2);
}

// Length 6 = 2 x 3 by the prime-factor (Good-Thomas) index map, which needs no
// twiddles: input n = (3 n1 + 2 n2) mod 6, output k = (3 k1 + 4 k2) mod 6, and
// exp(SIGN 2 pi i n k / 6) = (-1)^(n1 k1) exp(SIGN 2 pi i n2 k2 / 3).
template <int SIGN, typename T> __host__ __device__ __forceinline__ void dft6(cplx<T>* v) {
	cplx<T> b0[3] = {v[0], v[2], v[4]}; // k1 = 0: sums over n1
	cplx<T> b1[3] = {v[0], v[2], v[4]}; // k1 = 1: differences
	const cplx<T> o[3] = {v[3], v[5], v[1]};
#pragma unroll
	for (int n2 = 0; n2 < 3; n2++) {
		b0[n2] = cadd(b0[n2], o[n2]);
		b1[n2] = csub(b1[n2], o[n2]);
	}
	dft3<SIGN, T>(b0);
	dft3<SIGN, T>(b1);
	v[0] = b0[0];
	v[4] = b0[1];
	v[2] = b0[2];
	v[3] = b1[0];
	v[1] = b1[1];
	v[5] = b1[2];
}

template <int SIGN, typename T> __host__ __device__ __forceinline__ void dft5(cplx<T>* v) {
	const T c1 = (T)0.30901699437494742410229341718282;  // cos(2pi/5)
	const T c2 = (T)-0.80901699437494742410229341718282; // cos(4pi/5)
	const T s1 = (T)SIGN * (T)0.95105651629515357211643933337938; // sin(2pi/5)
	const T s2 = (T)SIGN * (T)0.58778525229247312916870595463907; // sin(4pi/5)
	cplx<T> a = v[0];
	cplx<T> p1 = cadd(v[1], v[4]), m1 = csub(v[1], v[4]);
	cplx<T> p2 = cadd(v[2], v[3]), m2 = csub(v[2], v[3]);
	v[0] = cadd(a, cadd(p1, p2));
	cplx<T> r1 = mk<T>(a.x + c1 * p1.x + c2 * p2.x, a.y + c1 * p1.y + c2 * p2.y);
	cplx<T> r2 = mk<T>(a.x + c2 * p1.x + c1 * p2.x, a.y + c2 * p1.y + c1 * p2.y);
	// i*(s1 m1 + s2 m2), i*(s2 m1 - s1 m2)
	cplx<T> i1 = mk<T>(-(s1 * m1.y + s2 * m2.y), s1 * m1.x + s2 * m2.x);
	cplx<T> i2 = mk<T>(-(s2 * m1.y - s1 * m2.y), s2 * m1.x - s1 * m2.x);
	v[1] = cadd(r1, i1);
	v[4] = csub(r1, i1);
	v[2] = cadd(r2, i2);
	v[3] = csub(r2, i2);
}

template <int SIGN, typename T> __host__ __device__ __forceinline__ void dft7(cplx<T>* v) {
	const T c1 = (T)0.62348980185873353052500488400424;   // cos(2pi/7)
	const T c2 = (T)-0.22252093395631440428890256449680;  // cos(4pi/7)
	const T c3 = (T)-0.90096886790241912623610231950745;  // cos(6pi/7)
	const T s1 = (T)SIGN * (T)0.78183148246802980870844452667406; // sin(2pi/7)
	const T s2 = (T)SIGN * (T)0.97492791218182360701813168299393; // sin(4pi/7)
	const T s3 = (T)SIGN * (T)0.43388373911755812047576833284836; // sin(6pi/7)
	cplx<T> a = v[0];
	cplx<T> p1 = cadd(v[1], v[6]), m1 = csub(v[1], v[6]);
	cplx<T> p2 = cadd(v[2], v[5]), m2 = csub(v[2], v[5]);
	cplx<T> p3 = cadd(v[3], v[4]), m3 = csub(v[3], v[4]);
	v[0] = cadd(a, cadd(p1, cadd(p2, p3)));
	// k=1: c1 c2 c3 / s1 s2 s3 ; k=2: c2 c3(=cos 12pi/7 = c2? ) -> use cos(2pi*2r/7)
	// cos(2pi*k*r/7) for r=1..3: k=1: c1,c2,c3 ; k=2: c2,c3,c1 ; k=3: c3,c1,c2
	// sin(2pi*k*r/7):            k=1: s1,s2,s3 ; k=2: s2,-s3,-s1 ; k=3: s3,-s1,s2
	cplx<T> r1 = mk<T>(a.x + c1 * p1.x + c2 * p2.x + c3 * p3.x, a.y + c1 * p1.y + c2 * p2.y + c3 * p3.y);
	cplx<T> r2 = mk<T>(a.x + c2 * p1.x + c3 * p2.x + c1 * p3.x, a.y + c2 * p1.y + c3 * p2.y + c1 * p3.y);
	cplx<T> r3 = mk<T>(a.x + c3 * p1.x + c1 * p2.x + c2 * p3.x, a.y + c3 * p1.y + c1 * p2.y + c2 * p3.y);
	T j1x = s1 * m1.x + s2 * m2.x + s3 * m3.x, j1y = s1 * m1.y + s2 * m2.y + s3 * m3.y;
	T j2x = s2 * m1.x - s3 * m2.x - s1 * m3.x, j2y = s2 * m1.y - s3 * m2.y - s1 * m3.y;
	T j3x = s3 * m1.x - s1 * m2.x + s2 * m3.x, j3y = s3 * m1.y - s1 * m2.y + s2 * m3.y;
	cplx<T> i1 = mk<T>(-j1y, j1x), i2 = mk<T>(-j2y, j2x), i3 = mk<T>(-j3y, j3x);
	v[1] = cadd(r1, i1);
	v[6] = csub(r1, i1);
	v[2] = cadd(r2, i2);
	v[5] = csub(r2, i2);
	v[3] = cadd(r3, i3);
	v[4] = csub(r3, i3);
}

template <int R, int SIGN, typename T> __host__ __device__ __forceinline__ void dft(cplx<T>* v) {
	if constexpr (R == 2) dft2<SIGN, T>(v);
	else if constexpr (R == 3) dft3<SIGN, T>(v);
	else if constexpr (R == 4) dft4<SIGN, T>(v);
	else if constexpr (R == 5) dft5<SIGN, T>(v);
	else if constexpr (R == 6) dft6<SIGN, T>(v);
	else if constexpr (R == 7) dft7<SIGN, T>(v);
	else if constexpr (R == 8) dft8<SIGN, T>(v);
	else if constexpr (R == 16) dft16<SIGN, T>(v);
}

// ---------------------------------------------------------------- plans --

// A transform length n = RMAIN^nmain * rtail * 3^n3 * 5^n5 * 7^n7 with
// rtail in {1, 2, 4, 8} (< RMAIN), done as runs of one radix each: nmain
// passes of RMAIN, one of rtail, then the odd radices. A loop body holding a
// single radix keeps register allocation tight; the host fills the counts.
struct FftPlan {
	int n;
	int nmain;
	int rtail;
	int n3, n5, n7;
};

// ---------------------------------------------------------------- passes -

// One Stockham pass over P sequences (sequence p starts at buf + p*ld, padded
// indexing inside a sequence). nthreads threads take part, thread index t.
// Only the butterfly inputs are live across the barrier; twiddles are read
// after it, so a thread needs about MAXE complex registers plus one DFT's
// temporaries.
template <int R, int SIGN, int MAXE, typename T>
__device__ __forceinline__ void stockham_pass(cplx<T>* buf, int ld, int P, int n, int Ns,
                                              const cplx<T>* __restrict__ tw, int t, int nthreads) {
	constexpr int NB = MAXE / R;
	static_assert(NB >= 1, "MAXE too small for radix");
	const int nR = n / R;
	const int total = P * nR;
	cplx<T> v[NB][R];
#pragma unroll
	for (int i = 0; i < NB; i++) {
		const int b = t + i * nthreads;
		if (b < total) {
			const int p = b / nR;
			const int j = b - p * nR;
			const cplx<T>* in = buf + p * ld;
#pragma unroll
			for (int r = 0; r < R; r++) v[i][r] = in[pad<T>(j + r * nR)];
		}
	}
	__syncthreads();
	const int tstep = n / (Ns * R);
#pragma unroll
	for (int i = 0; i < NB; i++) {
		const int b = t + i * nthreads;
		if (b < total) {
			const int p = b / nR;
			const int j = b - p * nR;
			const int jm = j % Ns;
			if (jm > 0) {
				const cplx<T>* twj = tw + jm * tstep;
#pragma unroll
				for (int r = 1; r < R; r++) {
					cplx<T> w = __ldg(twj + (r - 1) * jm * tstep);
					if (SIGN > 0) w.y = -w.y;
					v[i][r] = cmul(v[i][r], w);
				}
			}
			dft<R, SIGN, T>(v[i]);
			cplx<T>* out = buf + p * ld;
			const int d0 = (j - jm) * R + jm;
#pragma unroll
			for (int r = 0; r < R; r++) out[pad<T>(d0 + r * Ns)] = v[i][r];
		}
	}
	__syncthreads();
}

// Full transform of P sequences of length plan.n in place in shared memory.
// RMAIN = MAXE; requires ceil(P * n / (R * nthreads)) <= MAXE / R for each radix R.
template <int SIGN, int MAXE, typename T>
__device__ __forceinline__ void fft_batch(cplx<T>* buf, int ld, int P, const FftPlan& plan,
                                          const cplx<T>* __restrict__ tw, int t, int nthreads) {
	constexpr int RM = MAXE;
	const int n = plan.n;
	int Ns = 1;
	for (int s = 0; s < plan.nmain; s++) {
		stockham_pass<RM, SIGN, MAXE, T>(buf, ld, P, n, Ns, tw, t, nthreads);
		Ns *= RM;
	}
	if constexpr (RM > 8) {
		if (plan.rtail == 8) { stockham_pass<8, SIGN, MAXE, T>(buf, ld, P, n, Ns, tw, t, nthreads); Ns *= 8; }
	}
	if (plan.rtail == 4) { stockham_pass<4, SIGN, MAXE, T>(buf, ld, P, n, Ns, tw, t, nthreads); Ns *= 4; }
	else if (plan.rtail == 2) { stockham_pass<2, SIGN, MAXE, T>(buf, ld, P, n, Ns, tw, t, nthreads); Ns *= 2; }
	for (int s = 0; s < plan.n3; s++) { stockham_pass<3, SIGN, MAXE, T>(buf, ld, P, n, Ns, tw, t, nthreads); Ns *= 3; }
	for (int s = 0; s < plan.n5; s++) { stockham_pass<5, SIGN, MAXE, T>(buf, ld, P, n, Ns, tw, t, nthreads); Ns *= 5; }
	for (int s = 0; s < plan.n7; s++) { stockham_pass<7, SIGN, MAXE, T>(buf, ld, P, n, Ns, tw, t, nthreads); Ns *= 7; }
}

// Transforms S resident sequences in sub-batches of at most SB (so that the
// thread count needed by one fft_batch call stays within the CTA).
template <int SIGN, int MAXE, typename T>
__device__ __forceinline__ void fft_batches(cplx<T>* buf, int ld, int S, int SB, const FftPlan& plan,
                                            const cplx<T>* __restrict__ tw, int t, int nthreads) {
	for (int b0 = 0; b0 < S; b0 += SB) {
		const int nb = (S - b0) < SB ? (S - b0) : SB;
		fft_batch<SIGN, MAXE, T>(buf + b0 * ld, ld, nb, plan, tw, t, nthreads);
	}
}

// ------------------------------------------------- compile-time lengths --
// Power-of-two lengths known at compile time: N = RM^A * RT. All index math
// folds to shifts and masks; twiddles come from a per-pass table in shared
// memory laid out [q * Ns + jm] (consecutive threads read consecutive words):
// for radix R < 16 entry q is w^(q+1), w = exp(-2 pi i jm / (Ns R)); for radix
// 16 only w^1, w^2, w^3, w^4, w^8, w^12 are stored and the other nine powers
// are products of two of them (ct_twiddle), which cuts the table and its
// shared-memory reads by 60 % for one extra complex product per power.

// N = RM^A * RT with RM^(A+1) not dividing N; RT (1 = none) is one of the
// radices dft() has (2, 3, 4, 6, 8 for the lengths used). The tail radix, when
// there is one, is pass 1 (second), so that the first and the last pass both
// have radix RM: the last pass then leaves in each thread exactly the elements
// the next transform's first pass needs (fused below).
__host__ __device__ constexpr int ct_count(int n, int r) { return (n > 0 && n % r == 0) ? 1 + ct_count(n / r, r) : 0; }
__host__ __device__ constexpr int ct_ipow(int b, int e) { return e == 0 ? 1 : b * ct_ipow(b, e - 1); }
template <int N, int RM> struct CtPlan {
	static constexpr int A = ct_count(N, RM);          // passes of radix RM
	static constexpr int RT = N / ct_ipow(RM, A);      // tail radix (1 = none)
	static_assert(N == 0 || RT == 1 || RT == 2 || RT == 3 || RT == 4 || RT == 6 || RT == 8, "no DFT for this tail radix");
	static constexpr int NPASS = A + (RT > 1 ? 1 : 0);
	static constexpr bool FUSABLE = A >= 2;            // first and last pass both radix RM
	__host__ __device__ static constexpr int radix(int p) { return (RT > 1 && p == 1) ? RT : RM; }
	__host__ __device__ static constexpr int ns(int p) { return p == 0 ? 1 : ns(p - 1) * radix(p - 1); }
	// twiddle-table offset of pass p (pass 0 has none)
	// table entries per butterfly position of a pass of radix r (ct_twiddle)
	__host__ __device__ static constexpr int twcnt(int r) { return r == 16 ? 6 : r - 1; }
	__host__ __device__ static constexpr int twoff(int p) { return p <= 1 ? 0 : twoff(p - 1) + twcnt(radix(p - 1)) * ns(p - 1); }
	static constexpr int TWN = twoff(NPASS);
};

// v[r] *= w^r for r = 1 .. R-1, w = exp(SIGN 2 pi i jm / (NS R)); twj points at
// the pass's table entry for jm (layout above).
template <int R, int NS, int SIGN, typename T>
__host__ __device__ __forceinline__ void ct_twiddle(cplx<T>* v, const cplx<T>* twj) {
	if constexpr (R == 16) {
		cplx<T> b[6]; // w^1, w^2, w^3, w^4, w^8, w^12
#pragma unroll
		for (int q = 0; q < 6; q++) {
			b[q] = twj[q * NS];
			if (SIGN > 0) b[q].y = -b[q].y;
		}
		v[1] = cmul(v[1], b[0]);
		v[2] = cmul(v[2], b[1]);
		v[3] = cmul(v[3], b[2]);
		v[4] = cmul(v[4], b[3]);
		v[8] = cmul(v[8], b[4]);
		v[12] = cmul(v[12], b[5]);
#pragma unroll
		for (int hi = 0; hi < 3; hi++) {
			const cplx<T> h = hi == 0 ? b[3] : hi == 1 ? b[4] : b[5]; // w^4, w^8, w^12
			const int base = 4 * (hi + 1);
			v[base + 1] = cmul(v[base + 1], cmul(h, b[0]));
			v[base + 2] = cmul(v[base + 2], cmul(h, b[1]));
			v[base + 3] = cmul(v[base + 3], cmul(h, b[2]));
		}
	} else {
#pragma unroll
		for (int r = 1; r < R; r++) {
			cplx<T> w = twj[(r - 1) * NS];
			if (SIGN > 0) w.y = -w.y;
			v[r] = cmul(v[r], w);
		}
	}
}

// pad(a + m * P) = pad(a) + m * (P + 1) for the padding period P = 2^SHIFT:
// strides that are multiples of P become constant offsets from one padded base.
template <int N, int R, int NS, int TWO, int NSEQ, int NT, int SIGN, typename T>
__device__ __forceinline__ void ct_pass(cplx<T>* buf, const cplx<T>* tws, int t) {
	constexpr int LD = N + (N >> Pad<T>::SHIFT) + 1;
	constexpr int NR = N / R;
	constexpr int TOTAL = NSEQ * NR;
	constexpr int NB = (TOTAL + NT - 1) / NT;
	constexpr int PP = 1 << Pad<T>::SHIFT;
	cplx<T> v[NB][R];
#pragma unroll
	for (int i = 0; i < NB; i++) {
		const int b = t + i * NT;
		if (TOTAL % NT == 0 || b < TOTAL) {
			const int p = b / NR, j = b % NR;
			const cplx<T>* in = buf + p * LD;
			if constexpr (NR % PP == 0) {
				const int pj = pad<T>(j);
#pragma unroll
				for (int r = 0; r < R; r++) v[i][r] = in[pj + r * (NR + NR / PP)];
			} else {
#pragma unroll
				for (int r = 0; r < R; r++) v[i][r] = in[pad<T>(j + r * NR)];
			}
		}
	}
	__syncthreads();
#pragma unroll
	for (int i = 0; i < NB; i++) {
		const int b = t + i * NT;
		if (TOTAL % NT == 0 || b < TOTAL) {
			const int p = b / NR, j = b % NR;
			const int jm = j % NS;
			if constexpr (NS > 1) ct_twiddle<R, NS, SIGN, T>(v[i], tws + TWO + jm);
			dft<R, SIGN, T>(v[i]);
			cplx<T>* out = buf + p * LD;
			const int d0 = (j - jm) * R + jm;
			if constexpr (NS % PP == 0) {
				const int pd = pad<T>(d0);
#pragma unroll
				for (int r = 0; r < R; r++) out[pd + r * (NS + NS / PP)] = v[i][r];
			} else if constexpr (NS == 1 && R <= PP && PP % R == 0) {
				// d0 = j * R: the R outputs never cross a padding period
				const int pd = pad<T>(d0);
#pragma unroll
				for (int r = 0; r < R; r++) out[pd + r] = v[i][r];
			} else {
#pragma unroll
				for (int r = 0; r < R; r++) out[pad<T>(d0 + r * NS)] = v[i][r];
			}
		}
	}
	__syncthreads();
}

template <int N, int RM, int P, int NSEQ, int NT, int SIGN, typename T>
__device__ __forceinline__ void ct_passes(cplx<T>* buf, const cplx<T>* tws, int t) {
	using PL = CtPlan<N, RM>;
	if constexpr (P < PL::NPASS) {
		ct_pass<N, PL::radix(P), PL::ns(P), PL::twoff(P), NSEQ, NT, SIGN, T>(buf, tws, t);
		ct_passes<N, RM, P + 1, NSEQ, NT, SIGN, T>(buf, tws, t);
	}
}

template <int N, int RM, int P, int NSEQ, int NT, int SIGN, typename T>
__device__ __forceinline__ void ct_middle_from(cplx<T>* buf, const cplx<T>* tws, int t) {
	using PL = CtPlan<N, RM>;
	if constexpr (P < PL::NPASS - 1) {
		ct_pass<N, PL::radix(P), PL::ns(P), PL::twoff(P), NSEQ, NT, SIGN, T>(buf, tws, t);
		ct_middle_from<N, RM, P + 1, NSEQ, NT, SIGN, T>(buf, tws, t);
	}
}

// ------------------------------------------------------ fused first/last --
// In a pass of radix RM, butterfly b = t + i*NT of the NSEQ sequences handles
// sequence p = b / (N/RM) at positions j + r*N/RM (j = b mod N/RM): the first
// pass (Ns = 1) reads them and the last pass (Ns = N/RM) writes them. RegBlock
// holds one thread's elements between the two, so pointwise work and global
// loads/stores can act on them in registers.
// Thread-to-butterfly maps of a fused pass: StdMap is b = t + i*NT;
// PairMap (two fields of CC columns, one butterfly per thread) puts field 0
// in lanes 0-15 and field 1 in lanes 16-31 of each warp at the same butterfly,
// so lane l and lane l ^ 16 hold the two fields at the same points.
template <int N, int RM, int NSEQ, int NT> struct StdMap {
	static constexpr int NR = N / RM;
	static constexpr int NB = (NSEQ * NR + NT - 1) / NT;
	static_assert((NSEQ * NR) % NT == 0, "whole butterflies per thread");
	__device__ __forceinline__ static int seq(int t, int i) { return (t + i * NT) / NR; }
	__device__ __forceinline__ static int bj(int t, int i) { return (t + i * NT) % NR; }
};

template <int N, int RM, int CC> struct PairMap {
	static constexpr int NR = N / RM;
	static constexpr int NB = 1;
	__device__ __forceinline__ static int field(int t) { return (t >> 4) & 1; }
	__device__ __forceinline__ static int rest(int t) { return ((t >> 5) << 4) | (t & 15); }
	__device__ __forceinline__ static int col(int t) { return rest(t) / NR; }
	__device__ __forceinline__ static int seq(int t, int) { return field(t) * CC + col(t); }
	__device__ __forceinline__ static int bj(int t, int) { return rest(t) % NR; }
};

template <int N, int RM, int NSEQ, int NT, typename T, typename MAP = StdMap<N, RM, NSEQ, NT>> struct RegBlock {
	static constexpr int NR = N / RM;
	static constexpr int NB = MAP::NB;
	cplx<T> v[NB][RM];
	__device__ __forceinline__ static int seq(int t, int i) { return MAP::seq(t, i); }
	__device__ __forceinline__ static int pos(int t, int i, int r) { return MAP::bj(t, i) + r * NR; }
};

// first pass of a transform (Ns = 1) from registers to shared memory
template <int N, int RM, int NSEQ, int NT, int SIGN, typename T, typename MAP = StdMap<N, RM, NSEQ, NT>>
__device__ __forceinline__ void ct_first_from_regs(cplx<T>* buf, RegBlock<N, RM, NSEQ, NT, T, MAP>& rb, int t) {
	constexpr int LD = N + (N >> Pad<T>::SHIFT) + 1;
	constexpr int PP = 1 << Pad<T>::SHIFT;
#pragma unroll
	for (int i = 0; i < MAP::NB; i++) dft<RM, SIGN, T>(rb.v[i]);
	__syncthreads(); // earlier readers of buf are done
#pragma unroll
	for (int i = 0; i < MAP::NB; i++) {
		const int p = MAP::seq(t, i), j = MAP::bj(t, i);
		cplx<T>* out = buf + p * LD;
		const int d0 = j * RM;
		if constexpr (RM <= PP && PP % RM == 0) {
			const int pd = pad<T>(d0);
#pragma unroll
			for (int r = 0; r < RM; r++) out[pd + r] = rb.v[i][r];
		} else {
#pragma unroll
			for (int r = 0; r < RM; r++) out[pad<T>(d0 + r)] = rb.v[i][r];
		}
	}
	__syncthreads();
}

// last pass of a transform (Ns = N/RM) from shared memory into registers
template <int N, int RM, int NSEQ, int NT, int SIGN, typename T, typename MAP = StdMap<N, RM, NSEQ, NT>>
__device__ __forceinline__ void ct_last_to_regs(const cplx<T>* buf, const cplx<T>* tws,
                                               RegBlock<N, RM, NSEQ, NT, T, MAP>& rb, int t) {
	using PL = CtPlan<N, RM>;
	constexpr int LD = N + (N >> Pad<T>::SHIFT) + 1;
	constexpr int NR = N / RM;
	constexpr int NS = NR;
	constexpr int TWO = PL::twoff(PL::NPASS - 1);
	constexpr int PP = 1 << Pad<T>::SHIFT;
	static_assert(PL::ns(PL::NPASS - 1) == NS, "last pass of radix RM");
#pragma unroll
	for (int i = 0; i < MAP::NB; i++) {
		const int p = MAP::seq(t, i), j = MAP::bj(t, i);
		const cplx<T>* in = buf + p * LD;
		if constexpr (NR % PP == 0) {
			const int pj = pad<T>(j);
#pragma unroll
			for (int r = 0; r < RM; r++) rb.v[i][r] = in[pj + r * (NR + NR / PP)];
		} else {
#pragma unroll
			for (int r = 0; r < RM; r++) rb.v[i][r] = in[pad<T>(j + r * NR)];
		}
	}
	// no barrier needed here: the caller works on registers and the next write
	// to this buffer is preceded by one
#pragma unroll
	for (int i = 0; i < MAP::NB; i++) {
		const int j = MAP::bj(t, i); // jm = j since Ns = N/RM
		ct_twiddle<RM, NS, SIGN, T>(rb.v[i], tws + TWO + j);
		dft<RM, SIGN, T>(rb.v[i]);
	}
}

// the passes strictly between the first and the last, shared memory to shared memory
template <int N, int RM, int NSEQ, int NT, int SIGN, typename T>
__device__ __forceinline__ void ct_middle(cplx<T>* buf, const cplx<T>* tws, int t) {
	ct_middle_from<N, RM, 1, NSEQ, NT, SIGN, T>(buf, tws, t);
}

// NSEQ resident sequences of compile-time length N (stride padded_len(N)),
// transformed NSUB at a time by NT threads.
template <int N, int RM, int NSEQ, int NSUB, int NT, int SIGN, typename T>
__device__ __forceinline__ void fft_ct(cplx<T>* buf, const cplx<T>* tws, int t) {
	constexpr int LD = N + (N >> Pad<T>::SHIFT) + 1;
#pragma unroll 1
	for (int b0 = 0; b0 < NSEQ; b0 += NSUB) ct_passes<N, RM, 0, NSUB, NT, SIGN, T>(buf + b0 * LD, tws, t);
}

} // namespace pfcg
