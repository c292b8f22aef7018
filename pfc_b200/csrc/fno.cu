// Fourier neural operator warm start: forward, backward, Adam and tiled apply.
//
// Network (fixed shape; two fields on a T x T periodic tile):
//   v0 = P x + p                            lift, 2 -> C channels per pixel
//   z_l = W_l v_l + b_l + K_l v_l,  v_{l+1} = gelu(z_l)  (l < L-1), v_L = z_{L-1}
//   y = x + Q v_L + q                       projection C -> 2, added to the input
// K_l v = irfft2 of R_l (complex C x C per retained mode) times rfft2(v) on the
// retained modes kx in [0, MX), ky in {0..MY/2-1} u {T-MY/2..T-1}; all other
// modes are dropped. The truncated transforms are direct sums against
// twiddle matrices (dft_x, idft_x, dft_y_fwd, dft_y_inv); the adjoint of each
// linear step is another of these kernels, which is how the backward pass is
// built:
//   idft_x^T = dft_x with the inverse's per-mode weights, dft_y_fwd^T =
//   dft_y_inv, mix^T = mix with conj(R) transposed, dft_x^T = idft_x.
// Activations and sums are FP32; the kernels read a BF16 copy of the FP32
// master weights, which Adam updates.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/pfc_b200.h"
#include "fno.cuh"

namespace {

constexpr int C = PFCG_FNO_CHANNELS;
constexpr int L = PFCG_FNO_LAYERS;
constexpr int MX = PFCG_FNO_MODES_X;
constexpr int MY = PFCG_FNO_MODES_Y;
constexpr int NK = MX * MY; // retained modes per channel pair

// parameter layout, in floats: P [C][2], p [C], per layer {W [C][C], b [C],
// Rr [C][C][NK], Ri [C][C][NK]} with R indexed [in][out][ky-row][kx], Q [2][C], q [2]
constexpr size_t OFF_P = 0;
constexpr size_t OFF_PB = OFF_P + C * 2;
constexpr size_t OFF_L0 = OFF_PB + C;
constexpr size_t LAYER = C * C + C + 2 * (size_t)C * C * NK;
constexpr size_t OFF_Q = OFF_L0 + L * LAYER;
constexpr size_t OFF_QB = OFF_Q + 2 * C;
constexpr size_t NPARAM = OFF_QB + 2;
static_assert(NPARAM == PFCG_FNO_PARAMS, "parameter count");

__host__ __device__ constexpr size_t off_W(int l) { return OFF_L0 + l * LAYER; }
__host__ __device__ constexpr size_t off_b(int l) { return off_W(l) + C * C; }
__host__ __device__ constexpr size_t off_Rr(int l) { return off_b(l) + C; }
__host__ __device__ constexpr size_t off_Ri(int l) { return off_Rr(l) + (size_t)C * C * NK; }

constexpr int MAXT = 512; // largest tile (twiddle table in shared memory)

__device__ __forceinline__ float wld(const __nv_bfloat16* w, size_t i) { return __bfloat162float(w[i]); }

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float z) {
	return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * __expf(-0.5f * z * z);
}

// wave number of retained row k along y
__device__ __forceinline__ int ky_of(int k, int T) { return k < MY / 2 ? k : T - MY + k; }

template <typename A> __device__ __forceinline__ A warp_sum(A a) {
	for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
	return a;
}

// ------------------------------------------------------------- kernels ---

// tw[j] = (cos, sin)(2 pi j / T), from FP64
__global__ void twiddle_kernel(float2* tw, int T) {
	for (int j = threadIdx.x + blockIdx.x * blockDim.x; j < T; j += blockDim.x * gridDim.x) {
		double s, c;
		sincospi(2.0 * j / (double)T, &s, &c);
		tw[j] = make_float2((float)c, (float)s);
	}
}

// v0[b][c][p] = P[c][0] x[b][0][p] + P[c][1] x[b][1][p] + p[c]
__global__ void lift_fwd(const float* __restrict__ x, const __nv_bfloat16* __restrict__ w, float* __restrict__ v, int B,
                         int npix) {
	__shared__ float Ps[3 * C];
	for (int i = threadIdx.x; i < 3 * C; i += blockDim.x) Ps[i] = wld(w, OFF_P + i);
	__syncthreads();
	const long long n = (long long)B * npix;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
		const long long b = t / npix;
		const int p = (int)(t - b * npix);
		const float x0 = x[(b * 2) * npix + p], x1 = x[(b * 2 + 1) * npix + p];
		float* vb = v + b * C * npix + p;
#pragma unroll 8
		for (int c = 0; c < C; c++) vb[(long long)c * npix] = Ps[2 * c] * x0 + Ps[2 * c + 1] * x1 + Ps[2 * C + c];
	}
}

// ------------------------------------------- tensor-core channel products --
// The per-pixel channel contractions (z = W v, dv = W^T dz, dW = dz v^T) are
// GEMMs with a 32 x 32 weight or result and the pixels as the long dimension;
// they run on the tensor cores as mma.sync m16n8k16 with BF16 operands and
// FP32 accumulation. An FP32 operand is split into a BF16 high part and a
// BF16 remainder (x = hi + lo to about 2^-16 relative) and the products that
// matter are summed: with the BF16 weights, which are exact, W hi + W lo; with
// two FP32 operands, hi hi + hi lo + lo hi. Fragment layouts are those of the
// PTX ISA for m16n8k16: g = lane / 4, t = lane % 4; A (16 x 16, row major)
// holds rows g, g + 8 and columns 2t, 2t + 1, 2t + 8, 2t + 9; B (16 x 8) holds
// rows 2t, 2t + 1, 2t + 8, 2t + 9 of column g; the accumulator holds rows g,
// g + 8 and columns 2t, 2t + 1.

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
	asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
	             "{%0,%1,%2,%3};\n"
	             : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
	             : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// two FP32 values (the lower index first) as BF16 pairs: high parts and remainders
__device__ __forceinline__ void split2(float x0, float x1, uint32_t& hi, uint32_t& lo) {
	const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
	const float2 hf = __bfloat1622float2(h);
	const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
	hi = *reinterpret_cast<const uint32_t*>(&h);
	lo = *reinterpret_cast<const uint32_t*>(&l);
}

// two BF16 weights as one B-fragment register (the first in the low half)
__device__ __forceinline__ uint32_t pack_bf16(const __nv_bfloat16* w, size_t i0, size_t i1) {
	const unsigned short a = *reinterpret_cast<const unsigned short*>(w + i0);
	const unsigned short b = *reinterpret_cast<const unsigned short*>(w + i1);
	return (uint32_t)a | ((uint32_t)b << 16);
}

// The truncated transforms along x are GEMMs too, with the rows as the long
// dimension and a fixed matrix of twiddles as the other operand, whose
// BF16-split mma fragments are tabulated once per tile size (dft_frag_kernel):
//   dft_x:  D[row][2m + q] = sum_x in[row][x] E[x][2m + q], E = cos / -sin(2 pi m x / T)
//   idft_x: D[row][x] = sum_{m, q} in'[row][2m + q] F[2m + q][x], F = cos / -sin(2 pi m x / T),
//           in' = scale[m] (Re, Im) of the row's modes
// Fragment entry (k-step or n-tile, lane) holds the B registers of the high
// parts and of the remainders.

// fdx: [T/16 k-steps][2 n-tiles][32 lanes], fix: [T/8 n-tiles][32 lanes]
__global__ void dft_frag_kernel(const float2* __restrict__ tw, int T, uint4* __restrict__ fdx, uint4* __restrict__ fix) {
	const int nx = T / 16 * 2 * 32, ni = T / 8 * 32;
	for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nx + ni; e += gridDim.x * blockDim.x) {
		float v[4];
		if (e < nx) {
			const int lane = e & 31, nt = (e >> 5) & 1, ks = e >> 6;
			const int col = 8 * nt + (lane >> 2), m = col >> 1, q = col & 1, t = lane & 3;
			const int xs[4] = {16 * ks + 2 * t, 16 * ks + 2 * t + 1, 16 * ks + 2 * t + 8, 16 * ks + 2 * t + 9};
#pragma unroll
			for (int k = 0; k < 4; k++) {
				const float2 w = tw[(m * xs[k]) & (T - 1)];
				v[k] = q ? -w.y : w.x;
			}
		} else {
			const int f = e - nx, lane = f & 31, nt = f >> 5;
			const int x = 8 * nt + (lane >> 2), t = lane & 3;
			const float2 w0 = tw[(t * x) & (T - 1)], w4 = tw[((t + 4) * x) & (T - 1)];
			v[0] = w0.x;
			v[1] = -w0.y;
			v[2] = w4.x;
			v[3] = -w4.y;
		}
		uint32_t h0, l0, h1, l1;
		split2(v[0], v[1], h0, l0);
		split2(v[2], v[3], h1, l1);
		const uint4 r = make_uint4(h0, h1, l0, l1);
		if (e < nx) fdx[e] = r;
		else fix[e - nx] = r;
	}
}

// out[r][m] = scale[m] * sum_x in[r][x] exp(-2 pi i m x / T) for m < MX; one
// warp per 16 rows
__global__ void __launch_bounds__(256) dft_x(const float* __restrict__ in, float2* __restrict__ out,
                                             const uint4* __restrict__ fdx, const float* __restrict__ scale,
                                             long long nrows, int T) {
	const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
	const long long ntile = nrows / 16, nw = ((long long)gridDim.x * blockDim.x) >> 5;
	for (long long tile = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile < ntile; tile += nw) {
		const float* r0 = in + (tile * 16 + g) * T + 2 * t;
		const float* r8 = r0 + 8LL * T;
		float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
		for (int ks = 0; ks < T / 16; ks++) {
			const float2 x0 = *reinterpret_cast<const float2*>(r0 + 16 * ks);
			const float2 x1 = *reinterpret_cast<const float2*>(r8 + 16 * ks);
			const float2 x2 = *reinterpret_cast<const float2*>(r0 + 16 * ks + 8);
			const float2 x3 = *reinterpret_cast<const float2*>(r8 + 16 * ks + 8);
			uint32_t ah[4], al[4];
			split2(x0.x, x0.y, ah[0], al[0]);
			split2(x1.x, x1.y, ah[1], al[1]);
			split2(x2.x, x2.y, ah[2], al[2]);
			split2(x3.x, x3.y, ah[3], al[3]);
#pragma unroll
			for (int nt = 0; nt < 2; nt++) {
				const uint4 f = __ldg(fdx + (ks * 2 + nt) * 32 + lane);
				const uint32_t bh[2] = {f.x, f.y}, bl[2] = {f.z, f.w};
				mma_bf16(acc[nt], ah, bh);
				mma_bf16(acc[nt], ah, bl);
				mma_bf16(acc[nt], al, bh);
			}
		}
		// accumulator columns 2t, 2t + 1 of n-tile nt are (Re, Im) of mode 4 nt + t
#pragma unroll
		for (int nt = 0; nt < 2; nt++) {
			const int m = 4 * nt + t;
			const float sc = scale ? scale[m] : 1.f;
			out[(tile * 16 + g) * MX + m] = make_float2(acc[nt][0] * sc, acc[nt][1] * sc);
			out[(tile * 16 + g + 8) * MX + m] = make_float2(acc[nt][2] * sc, acc[nt][3] * sc);
		}
	}
}

// out[r][x] (+)= sum_m scale[m] Re(in[r][m] exp(+2 pi i m x / T)); one warp per
// 16 rows, eight points of each per n-tile
__global__ void __launch_bounds__(256) idft_x(const float2* __restrict__ in, float* __restrict__ out,
                                              const uint4* __restrict__ fix, const float* __restrict__ scale,
                                              long long nrows, int T, int accumulate) {
	const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
	const float s0 = scale ? scale[t] : 1.f, s4 = scale ? scale[t + 4] : 1.f;
	const long long ntile = nrows / 16, nw = ((long long)gridDim.x * blockDim.x) >> 5;
	for (long long tile = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile < ntile; tile += nw) {
		const long long ra = tile * 16 + g, rb = ra + 8;
		const float2 z0 = in[ra * MX + t], z1 = in[rb * MX + t], z2 = in[ra * MX + t + 4], z3 = in[rb * MX + t + 4];
		uint32_t ah[4], al[4];
		split2(s0 * z0.x, s0 * z0.y, ah[0], al[0]);
		split2(s0 * z1.x, s0 * z1.y, ah[1], al[1]);
		split2(s4 * z2.x, s4 * z2.y, ah[2], al[2]);
		split2(s4 * z3.x, s4 * z3.y, ah[3], al[3]);
		float* oa = out + ra * T + 2 * t;
		float* ob = out + rb * T + 2 * t;
		for (int nt = 0; nt < T / 8; nt++) {
			const uint4 f = __ldg(fix + nt * 32 + lane);
			const uint32_t bh[2] = {f.x, f.y}, bl[2] = {f.z, f.w};
			float d[4] = {0.f, 0.f, 0.f, 0.f};
			mma_bf16(d, ah, bh);
			mma_bf16(d, ah, bl);
			mma_bf16(d, al, bh);
			float2* pa = reinterpret_cast<float2*>(oa + 8 * nt);
			float2* pb = reinterpret_cast<float2*>(ob + 8 * nt);
			float2 va = make_float2(d[0], d[1]), vb = make_float2(d[2], d[3]);
			if (accumulate) {
				const float2 qa = *pa, qb = *pb;
				va.x += qa.x;
				va.y += qa.y;
				vb.x += qb.x;
				vb.y += qb.y;
			}
			*pa = va;
			*pb = vb;
		}
	}
}

// The truncated transforms along y, per plane of [rows][MX] complex values:
//   forward: out[k][m] = sum_y in[y][m] exp(-2 pi i ky(k) y / T), k < MY
//   inverse: out[y][m] = sum_k in[k][m] exp(+2 pi i ky(k) y / T), y < T
// are GEMMs against fixed twiddle matrices, on the tensor cores with one warp
// per plane. The twiddles are the A operand, their BF16-split fragments
// tabulated once per tile size (dfty_frag_kernel); the plane's values are the
// B operand, split per use, with three products (hi hi, hi lo, lo hi):
//   forward: D[k][2m + q] = sum_{y, c} E[k][2y + c] Z[2y + c][2m + q], (E[k][2y], E[k][2y + 1]) = (cos, sin)(2 pi ky(k) y / T)
//   inverse: D[y][2m + q] = sum_{k, c} F[y][2k + c] Z[2k + c][2m + q], (F[y][2k], F[y][2k + 1]) = (cos, -sin)(2 pi ky(k) y / T)
// with Z[2j][2m] = Re z[j][m], Z[2j + 1][2m] = Im, Z[2j][2m + 1] = Im, Z[2j + 1][2m + 1] = -Re, so that
// the accumulator pair of columns 2t, 2t + 1 is one output's (Re, Im).
static_assert(MY == 16 && MX == 8, "one m16 tile of modes and two n8 tiles of (Re, Im) columns");

// fdy: [T/8 k-steps][32 lanes][hi, lo], fiy: [T/16 m-tiles][2 k-steps][32 lanes][hi, lo];
// each uint4 holds the four A registers (rows g, g + 8 by columns 2t, 2t + 8)
__global__ void dfty_frag_kernel(const float2* __restrict__ tw, int T, uint4* __restrict__ fdy, uint4* __restrict__ fiy) {
	const int nf = T / 8 * 32, ni = T / 16 * 2 * 32;
	for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nf + ni; e += gridDim.x * blockDim.x) {
		const bool fwd = e < nf;
		const int f = fwd ? e : e - nf;
		const int lane = f & 31, g = lane >> 2, t = lane & 3;
		int rows[2], cols[2];
		if (fwd) {
			const int ks = f >> 5;
			rows[0] = g;
			rows[1] = g + 8;
			cols[0] = 8 * ks + t;
			cols[1] = cols[0] + 4;
		} else {
			const int ks = (f >> 5) & 1, mt = f >> 6;
			rows[0] = 16 * mt + g;
			rows[1] = rows[0] + 8;
			cols[0] = 8 * ks + t;
			cols[1] = cols[0] + 4;
		}
		uint32_t hi[4], lo[4];
#pragma unroll
		for (int r = 0; r < 4; r++) {
			// register r: row rows[r & 1], column pair of cols[r >> 1]
			const int row = rows[r & 1], col = cols[r >> 1];
			const int ky = ky_of(fwd ? row : col, T), y = fwd ? col : row;
			const float2 w = tw[(ky * y) & (T - 1)];
			split2(w.x, fwd ? w.y : -w.y, hi[r], lo[r]);
		}
		uint4* dst = (fwd ? fdy : fiy) + 2 * f;
		dst[0] = make_uint4(hi[0], hi[1], hi[2], hi[3]);
		dst[1] = make_uint4(lo[0], lo[1], lo[2], lo[3]);
	}
}

// the B registers of value z in the output column of parity q: (Re, Im) or (Im, -Re)
__device__ __forceinline__ void zsplit(float2 z, int q, uint32_t& hi, uint32_t& lo) {
	if (q) split2(z.y, -z.x, hi, lo);
	else split2(z.x, z.y, hi, lo);
}

// One block of four warps per plane. Forward: warp w takes the k-steps
// w, w + 4, ... and the warps' partial sums are added in shared memory in a
// fixed order. Inverse: warp w takes the m-tiles w, w + 4, ...
constexpr int DY_WARPS = 4;

__global__ void __launch_bounds__(32 * DY_WARPS) dft_y_fwd(const float2* __restrict__ in, float2* __restrict__ out,
                                                          const uint4* __restrict__ fdy, long long nplanes, int T) {
	__shared__ float red[DY_WARPS][32][8];
	const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3, q = g & 1;
	for (long long plane = blockIdx.x; plane < nplanes; plane += gridDim.x) {
		const float2* pin = in + plane * T * MX;
		float d[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
		for (int ks = wp; ks < T / 8; ks += DY_WARPS) {
			const uint4 fh = __ldg(fdy + (ks * 32 + lane) * 2), fl = __ldg(fdy + (ks * 32 + lane) * 2 + 1);
			const uint32_t ah[4] = {fh.x, fh.y, fh.z, fh.w}, al[4] = {fl.x, fl.y, fl.z, fl.w};
			const int y0 = 8 * ks + t;
#pragma unroll
			for (int nt = 0; nt < 2; nt++) {
				const int m = 4 * nt + (g >> 1);
				uint32_t bh[2], bl[2];
				zsplit(pin[y0 * MX + m], q, bh[0], bl[0]);
				zsplit(pin[(y0 + 4) * MX + m], q, bh[1], bl[1]);
				mma_bf16(d[nt], ah, bh);
				mma_bf16(d[nt], ah, bl);
				mma_bf16(d[nt], al, bh);
			}
		}
		__syncthreads(); // the previous plane's sums have been read
#pragma unroll
		for (int j = 0; j < 8; j++) red[wp][lane][j] = d[j >> 2][j & 3];
		__syncthreads();
		if (wp == 0) {
#pragma unroll
			for (int j = 0; j < 8; j++) d[j >> 2][j & 3] = red[0][lane][j] + red[1][lane][j] + red[2][lane][j] + red[3][lane][j];
			float2* pout = out + plane * MY * MX;
#pragma unroll
			for (int nt = 0; nt < 2; nt++) {
				const int m = 4 * nt + t;
				pout[g * MX + m] = make_float2(d[nt][0], d[nt][1]);
				pout[(g + 8) * MX + m] = make_float2(d[nt][2], d[nt][3]);
			}
		}
	}
}

__global__ void __launch_bounds__(32 * DY_WARPS) dft_y_inv(const float2* __restrict__ in, float2* __restrict__ out,
                                                          const uint4* __restrict__ fiy, long long nplanes, int T) {
	const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3, q = g & 1;
	for (long long plane = blockIdx.x; plane < nplanes; plane += gridDim.x) {
		const float2* pin = in + plane * MY * MX;
		// the whole plane as B fragments: two k-steps (K = 2 MY) by two n-tiles
		uint32_t bh[2][2][2], bl[2][2][2];
#pragma unroll
		for (int ks = 0; ks < 2; ks++)
#pragma unroll
			for (int nt = 0; nt < 2; nt++) {
				const int k0 = 8 * ks + t, m = 4 * nt + (g >> 1);
				zsplit(pin[k0 * MX + m], q, bh[ks][nt][0], bl[ks][nt][0]);
				zsplit(pin[(k0 + 4) * MX + m], q, bh[ks][nt][1], bl[ks][nt][1]);
			}
		float2* pout = out + plane * T * MX;
		for (int mt = wp; mt < T / 16; mt += DY_WARPS) {
			float d[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
			for (int ks = 0; ks < 2; ks++) {
				const uint4 fh = __ldg(fiy + ((mt * 2 + ks) * 32 + lane) * 2);
				const uint4 fl = __ldg(fiy + ((mt * 2 + ks) * 32 + lane) * 2 + 1);
				const uint32_t ah[4] = {fh.x, fh.y, fh.z, fh.w}, al[4] = {fl.x, fl.y, fl.z, fl.w};
#pragma unroll
				for (int nt = 0; nt < 2; nt++) {
					mma_bf16(d[nt], ah, bh[ks][nt]);
					mma_bf16(d[nt], ah, bl[ks][nt]);
					mma_bf16(d[nt], al, bh[ks][nt]);
				}
			}
			const int y0 = 16 * mt + g;
#pragma unroll
			for (int nt = 0; nt < 2; nt++) {
				const int m = 4 * nt + t;
				pout[y0 * MX + m] = make_float2(d[nt][0], d[nt][1]);
				pout[(y0 + 8) * MX + m] = make_float2(d[nt][2], d[nt][3]);
			}
		}
	}
}

// Mode mixing, per retained mode km:
//   forward: out[b][o][km] = sum_i R[i][o][km] in[b][i][km]
//   adjoint: out[b][i][km] = sum_o conj(R[i][o][km]) in[b][o][km]
// On the tensor cores, one warp per mode and 16 batch rows: D[b][2o + q] =
// sum_{i, c} A[b][2i + c] M[2i + c][2o + q] with A = (Re, Im) of the inputs
// (BF16 high parts and remainders, two products) and M the real 64 x 64 form
// of R or of conj(R)^T, whose entries are the exact BF16 weights:
//   forward: M[2i][2o] = Rr, M[2i+1][2o] = -Ri, M[2i][2o+1] = Ri, M[2i+1][2o+1] = Rr  (of R[i][o])
//   adjoint: M[2o][2i] = Rr, M[2o+1][2i] = Ri, M[2o][2i+1] = -Ri, M[2o+1][2i+1] = Rr
// (M's rows indexed by the step's input channel, its columns by the output).
// The accumulator pair of columns 2t, 2t + 1 is one output's (Re, Im).
__device__ __forceinline__ uint32_t bf16_pair(unsigned short lo, unsigned short hi) { return (uint32_t)lo | ((uint32_t)hi << 16); }

__global__ void __launch_bounds__(128) mix(const float2* __restrict__ in, float2* __restrict__ out,
                                           const __nv_bfloat16* __restrict__ w, int l, int B, int adjoint) {
	const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
	const int mtiles = (B + 15) / 16;
	const unsigned short* Rr = reinterpret_cast<const unsigned short*>(w + off_Rr(l));
	const unsigned short* Ri = reinterpret_cast<const unsigned short*>(w + off_Ri(l));
	const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
	// one warp per (n-tile of eight output columns, mode, 16 batch rows); whole
	// warps take the same items, so the mma.sync lanes stay converged
	for (long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; wid < (long long)NK * mtiles * 8;
	     wid += nw) {
		const int nt = (int)(wid & 7), km = (int)((wid >> 3) % NK), mt = (int)((wid >> 3) / NK);
		const int b0 = 16 * mt + g, b1 = b0 + 8;
		const int col = 4 * nt + (g >> 1), q = g & 1; // output channel and part of column 8 nt + g
		float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
		for (int ks = 0; ks < 4; ks++) {
			const int i0 = 8 * ks + t, i1 = i0 + 4;
			const float2 zero = make_float2(0.f, 0.f);
			const float2 z00 = b0 < B ? in[((long long)b0 * C + i0) * NK + km] : zero;
			const float2 z10 = b1 < B ? in[((long long)b1 * C + i0) * NK + km] : zero;
			const float2 z01 = b0 < B ? in[((long long)b0 * C + i1) * NK + km] : zero;
			const float2 z11 = b1 < B ? in[((long long)b1 * C + i1) * NK + km] : zero;
			uint32_t ah[4], al[4];
			split2(z00.x, z00.y, ah[0], al[0]);
			split2(z10.x, z10.y, ah[1], al[1]);
			split2(z01.x, z01.y, ah[2], al[2]);
			split2(z11.x, z11.y, ah[3], al[3]);
			uint32_t bw[2];
#pragma unroll
			for (int h = 0; h < 2; h++) {
				const int row = 8 * ks + t + 4 * h; // input channel of rows 16 ks + 2t (+8 h), + 1
				const size_t idx = adjoint ? ((size_t)col * C + row) * NK + km : ((size_t)row * C + col) * NK + km;
				const unsigned short rr = Rr[idx], ri = Ri[idx], nri = ri ^ 0x8000u;
				if (!adjoint) bw[h] = q ? bf16_pair(ri, rr) : bf16_pair(rr, nri);
				else bw[h] = q ? bf16_pair(nri, rr) : bf16_pair(rr, ri);
			}
			mma_bf16(d, ah, bw);
			mma_bf16(d, al, bw);
		}
		const int oc = 4 * nt + t;
		if (b0 < B) out[((long long)b0 * C + oc) * NK + km] = make_float2(d[0], d[1]);
		if (b1 < B) out[((long long)b1 * C + oc) * NK + km] = make_float2(d[2], d[3]);
	}
}

// dR[i][o][km] += sum_b dY[b][o][km] conj(X[b][i][km])
__global__ void mix_grad(const float2* __restrict__ X, const float2* __restrict__ dY, float* __restrict__ g, int l, int B) {
	const long long n = (long long)C * C * NK;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
		const int km = (int)(t % NK);
		const int o = (int)((t / NK) % C);
		const int i = (int)(t / ((long long)NK * C));
		float gr = 0.f, gi = 0.f;
		for (int b = 0; b < B; b++) {
			const float2 x = X[((long long)b * C + i) * NK + km];
			const float2 d = dY[((long long)b * C + o) * NK + km];
			gr += d.x * x.x + d.y * x.y;
			gi += d.y * x.x - d.x * x.y;
		}
		g[off_Rr(l) + t] += gr;
		g[off_Ri(l) + t] += gi;
	}
}

// z = W v + b + s; out = gelu(z) (act) or z. One warp per 16-pixel tile:
// D[pixel][out] = sum_in A[pixel][in] B[in][out] with A = v, B = W^T.
__global__ void __launch_bounds__(128, 4) pointwise_fwd(const float* __restrict__ v, const float* __restrict__ s,
                                                     const __nv_bfloat16* __restrict__ w, int l, float* __restrict__ z,
                                                     float* __restrict__ out, int B, int npix, int act) {
	const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
	uint32_t bw[4][2][2];
	float bias[4][2];
#pragma unroll
	for (int nt = 0; nt < 4; nt++) {
		const size_t row = off_W(l) + (size_t)(8 * nt + g) * C;
#pragma unroll
		for (int ks = 0; ks < 2; ks++) {
			bw[nt][ks][0] = pack_bf16(w, row + 16 * ks + 2 * t, row + 16 * ks + 2 * t + 1);
			bw[nt][ks][1] = pack_bf16(w, row + 16 * ks + 2 * t + 8, row + 16 * ks + 2 * t + 9);
		}
		bias[nt][0] = wld(w, off_b(l) + 8 * nt + 2 * t);
		bias[nt][1] = wld(w, off_b(l) + 8 * nt + 2 * t + 1);
	}
	const int tpi = npix / 16;
	const long long ntile = (long long)B * tpi;
	const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
	for (long long tile = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile < ntile; tile += nw) {
		const long long b = tile / tpi;
		const long long base = b * C * npix + (tile - b * tpi) * 16;
		uint32_t ah[2][4], al[2][4];
#pragma unroll
		for (int ks = 0; ks < 2; ks++) {
			const float* c0 = v + base + (long long)(16 * ks + 2 * t) * npix;
			const float* c1 = c0 + npix;
			const float* c8 = c0 + 8LL * npix;
			const float* c9 = c8 + npix;
			split2(c0[g], c1[g], ah[ks][0], al[ks][0]);
			split2(c0[g + 8], c1[g + 8], ah[ks][1], al[ks][1]);
			split2(c8[g], c9[g], ah[ks][2], al[ks][2]);
			split2(c8[g + 8], c9[g + 8], ah[ks][3], al[ks][3]);
		}
#pragma unroll
		for (int nt = 0; nt < 4; nt++) {
			const long long o0 = base + (long long)(8 * nt + 2 * t) * npix, o1 = o0 + npix;
			float d[4] = {bias[nt][0] + s[o0 + g], bias[nt][1] + s[o1 + g], bias[nt][0] + s[o0 + g + 8],
			              bias[nt][1] + s[o1 + g + 8]};
#pragma unroll
			for (int ks = 0; ks < 2; ks++) {
				mma_bf16(d, ah[ks], bw[nt][ks]);
				mma_bf16(d, al[ks], bw[nt][ks]);
			}
			if (z) {
				z[o0 + g] = d[0];
				z[o1 + g] = d[1];
				z[o0 + g + 8] = d[2];
				z[o1 + g + 8] = d[3];
			}
			out[o0 + g] = act ? gelu(d[0]) : d[0];
			out[o1 + g] = act ? gelu(d[1]) : d[1];
			out[o0 + g + 8] = act ? gelu(d[2]) : d[2];
			out[o1 + g + 8] = act ? gelu(d[3]) : d[3];
		}
	}
}

// dz = dout * g'(z) (also the gradient of the spectral branch); dv = W^T dz:
// D[pixel][in] = sum_out A[pixel][out] B[out][in] with A = dz, B = W.
__global__ void __launch_bounds__(128, 4) pointwise_bwd(const float* __restrict__ z, const float* __restrict__ dout,
                                                     const __nv_bfloat16* __restrict__ w, int l, float* __restrict__ dz,
                                                     float* __restrict__ dv, int B, int npix, int act) {
	const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
	uint32_t bw[4][2][2];
#pragma unroll
	for (int nt = 0; nt < 4; nt++) {
		const size_t col = off_W(l) + 8 * nt + g; // W[o][i = 8 nt + g] at col + o C
#pragma unroll
		for (int ks = 0; ks < 2; ks++) {
			const int o = 16 * ks + 2 * t;
			bw[nt][ks][0] = pack_bf16(w, col + (size_t)o * C, col + (size_t)(o + 1) * C);
			bw[nt][ks][1] = pack_bf16(w, col + (size_t)(o + 8) * C, col + (size_t)(o + 9) * C);
		}
	}
	const int tpi = npix / 16;
	const long long ntile = (long long)B * tpi;
	const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
	for (long long tile = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile < ntile; tile += nw) {
		const long long b = tile / tpi;
		const long long base = b * C * npix + (tile - b * tpi) * 16;
		uint32_t ah[2][4], al[2][4];
#pragma unroll
		for (int ks = 0; ks < 2; ks++) {
			float dd[8];
			const int och[4] = {16 * ks + 2 * t, 16 * ks + 2 * t + 1, 16 * ks + 2 * t + 8, 16 * ks + 2 * t + 9};
#pragma unroll
			for (int q = 0; q < 4; q++)
#pragma unroll
				for (int h = 0; h < 2; h++) {
					const long long i = base + (long long)och[q] * npix + g + 8 * h;
					const float gv = dout[i];
					const float d = act ? gv * gelu_d(z[i]) : gv;
					dz[i] = d;
					dd[2 * q + h] = d;
				}
			// a0 (g; o, o+1), a1 (g+8; o, o+1), a2 (g; o+8, o+9), a3 (g+8; o+8, o+9)
			split2(dd[0], dd[2], ah[ks][0], al[ks][0]);
			split2(dd[1], dd[3], ah[ks][1], al[ks][1]);
			split2(dd[4], dd[6], ah[ks][2], al[ks][2]);
			split2(dd[5], dd[7], ah[ks][3], al[ks][3]);
		}
#pragma unroll
		for (int nt = 0; nt < 4; nt++) {
			float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
			for (int ks = 0; ks < 2; ks++) {
				mma_bf16(d, ah[ks], bw[nt][ks]);
				mma_bf16(d, al[ks], bw[nt][ks]);
			}
			const long long i0 = base + (long long)(8 * nt + 2 * t) * npix, i1 = i0 + npix;
			dv[i0 + g] = d[0];
			dv[i1 + g] = d[1];
			dv[i0 + g + 8] = d[2];
			dv[i1 + g + 8] = d[3];
		}
	}
}

// dW[o][i] += sum_p dz[o][p] v[i][p], db[o] += sum_p dz[o][p]: D[o][i] = sum_p
// A[o][p] B[p][i] with A = dz, B = v^T, 16 pixels per step; each warp sums its
// tiles, the block adds its warps in shared memory, then one atomic per entry.
constexpr int WG_THREADS = 256;
__global__ void __launch_bounds__(WG_THREADS) weight_grad(const float* __restrict__ dz, const float* __restrict__ v,
                                                          float* __restrict__ gW, float* __restrict__ gb, int B,
                                                          int npix) {
	__shared__ float sW[C * C];
	__shared__ float sb[C];
	for (int i = threadIdx.x; i < C * C; i += blockDim.x) sW[i] = 0.f;
	if (threadIdx.x < C) sb[threadIdx.x] = 0.f;
	__syncthreads();
	const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
	float acc[2][4][4];
#pragma unroll
	for (int mt = 0; mt < 2; mt++)
#pragma unroll
		for (int nt = 0; nt < 4; nt++)
#pragma unroll
			for (int k = 0; k < 4; k++) acc[mt][nt][k] = 0.f;
	float bsum[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
	const int tpi = npix / 16;
	const long long ntile = (long long)B * tpi;
	const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
	for (long long tile = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile < ntile; tile += nw) {
		const long long b = tile / tpi;
		const long long base = b * C * npix + (tile - b * tpi) * 16 + 2 * t;
		uint32_t ah[2][4], al[2][4], bh[4][2], bl[4][2];
#pragma unroll
		for (int mt = 0; mt < 2; mt++) {
			const float* r0 = dz + base + (long long)(16 * mt + g) * npix;
			const float* r8 = r0 + 8LL * npix;
			const float2 x0 = *reinterpret_cast<const float2*>(r0), x1 = *reinterpret_cast<const float2*>(r8);
			const float2 x2 = *reinterpret_cast<const float2*>(r0 + 8), x3 = *reinterpret_cast<const float2*>(r8 + 8);
			split2(x0.x, x0.y, ah[mt][0], al[mt][0]);
			split2(x1.x, x1.y, ah[mt][1], al[mt][1]);
			split2(x2.x, x2.y, ah[mt][2], al[mt][2]);
			split2(x3.x, x3.y, ah[mt][3], al[mt][3]);
			bsum[mt][0] += (x0.x + x0.y) + (x2.x + x2.y);
			bsum[mt][1] += (x1.x + x1.y) + (x3.x + x3.y);
		}
#pragma unroll
		for (int nt = 0; nt < 4; nt++) {
			const float* r = v + base + (long long)(8 * nt + g) * npix;
			const float2 y0 = *reinterpret_cast<const float2*>(r), y1 = *reinterpret_cast<const float2*>(r + 8);
			split2(y0.x, y0.y, bh[nt][0], bl[nt][0]);
			split2(y1.x, y1.y, bh[nt][1], bl[nt][1]);
		}
#pragma unroll
		for (int mt = 0; mt < 2; mt++)
#pragma unroll
			for (int nt = 0; nt < 4; nt++) {
				mma_bf16(acc[mt][nt], ah[mt], bh[nt]);
				mma_bf16(acc[mt][nt], ah[mt], bl[nt]);
				mma_bf16(acc[mt][nt], al[mt], bh[nt]);
			}
	}
#pragma unroll
	for (int mt = 0; mt < 2; mt++)
#pragma unroll
		for (int nt = 0; nt < 4; nt++) {
			const int o = 16 * mt + g, i = 8 * nt + 2 * t;
			atomicAdd(&sW[o * C + i], acc[mt][nt][0]);
			atomicAdd(&sW[o * C + i + 1], acc[mt][nt][1]);
			atomicAdd(&sW[(o + 8) * C + i], acc[mt][nt][2]);
			atomicAdd(&sW[(o + 8) * C + i + 1], acc[mt][nt][3]);
		}
	// bias: the four lanes of a group hold disjoint pixels of the same rows
#pragma unroll
	for (int mt = 0; mt < 2; mt++)
#pragma unroll
		for (int h = 0; h < 2; h++) {
			float x = bsum[mt][h];
			x += __shfl_xor_sync(0xffffffffu, x, 1);
			x += __shfl_xor_sync(0xffffffffu, x, 2);
			if (t == 0) atomicAdd(&sb[16 * mt + g + 8 * h], x);
		}
	__syncthreads();
	for (int i = threadIdx.x; i < C * C; i += blockDim.x) atomicAdd(&gW[i], sW[i]);
	if (threadIdx.x < C) atomicAdd(&gb[threadIdx.x], sb[threadIdx.x]);
}

// y = x + Q v + q; with a target also loss += sum (y - t)^2 / n and dy = 2 (y - t) / n
__global__ void proj_fwd_loss(const float* __restrict__ x, const float* __restrict__ v, const __nv_bfloat16* __restrict__ w,
                              float* __restrict__ y, const float* __restrict__ target, float* __restrict__ dy,
                              double* __restrict__ loss, int B, int npix) {
	__shared__ float Qs[2 * C + 2];
	__shared__ double red[32];
	for (int i = threadIdx.x; i < 2 * C + 2; i += blockDim.x) Qs[i] = wld(w, OFF_Q + i);
	__syncthreads();
	const long long n = (long long)B * npix;
	const float inv = 2.f / (float)(2 * n);
	double acc = 0.0;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
		const long long b = t / npix;
		const int p = (int)(t - b * npix);
		const float* vb = v + b * C * npix + p;
		float o0 = Qs[2 * C], o1 = Qs[2 * C + 1];
#pragma unroll 8
		for (int c = 0; c < C; c++) {
			const float vv = vb[(long long)c * npix];
			o0 += Qs[c] * vv;
			o1 += Qs[C + c] * vv;
		}
		const long long i0 = b * 2 * npix + p, i1 = i0 + npix;
		const float y0 = x[i0] + o0, y1 = x[i1] + o1;
		y[i0] = y0;
		y[i1] = y1;
		if (target) {
			const float e0 = y0 - target[i0], e1 = y1 - target[i1];
			acc += (double)e0 * e0 + (double)e1 * e1;
			dy[i0] = inv * e0;
			dy[i1] = inv * e1;
		}
	}
	if (target) {
		acc = warp_sum(acc);
		if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
		__syncthreads();
		if (threadIdx.x < 32) {
			double a = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
			a = warp_sum(a);
			if (threadIdx.x == 0) atomicAdd(loss, a / (double)(2 * n));
		}
	}
}

// dv = Q^T dy
__global__ void proj_bwd(const float* __restrict__ dy, const __nv_bfloat16* __restrict__ w, float* __restrict__ dv, int B,
                         int npix) {
	__shared__ float Qs[2 * C];
	for (int i = threadIdx.x; i < 2 * C; i += blockDim.x) Qs[i] = wld(w, OFF_Q + i);
	__syncthreads();
	const long long n = (long long)B * npix;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
		const long long b = t / npix;
		const int p = (int)(t - b * npix);
		const float d0 = dy[b * 2 * npix + p], d1 = dy[b * 2 * npix + npix + p];
		float* db = dv + b * C * npix + p;
#pragma unroll 8
		for (int c = 0; c < C; c++) db[(long long)c * npix] = Qs[c] * d0 + Qs[C + c] * d1;
	}
}

// Per-channel sums over all pixels of a[b][c][p] * e[b][j][p] (j = 0, 1; e a
// two-field tensor) and of a itself. Gradients of the lift (a = dv0, e = x;
// g_ae = dP [C][2], g_a = dp [C]) and of the projection (a = v_L, e = dy;
// g_ae = dQ [2][C]). One block row per channel (blockIdx.y).
__global__ void channel_grad(const float* __restrict__ a, const float* __restrict__ e, float* __restrict__ g_ae,
                             int stride_c, int stride_j, float* __restrict__ g_a, int B, int npix) {
	__shared__ float red[3][32];
	const int c = blockIdx.y;
	const long long n = (long long)B * npix;
	float s0 = 0.f, s1 = 0.f, sa = 0.f;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
		const long long b = t / npix;
		const int p = (int)(t - b * npix);
		const float av = a[(b * C + c) * npix + p];
		s0 += av * e[(b * 2) * npix + p];
		s1 += av * e[(b * 2 + 1) * npix + p];
		sa += av;
	}
	s0 = warp_sum(s0);
	s1 = warp_sum(s1);
	sa = warp_sum(sa);
	if ((threadIdx.x & 31) == 0) {
		red[0][threadIdx.x >> 5] = s0;
		red[1][threadIdx.x >> 5] = s1;
		red[2][threadIdx.x >> 5] = sa;
	}
	__syncthreads();
	if (threadIdx.x < 32) {
		const bool in = threadIdx.x < (blockDim.x >> 5);
		s0 = warp_sum(in ? red[0][threadIdx.x] : 0.f);
		s1 = warp_sum(in ? red[1][threadIdx.x] : 0.f);
		sa = warp_sum(in ? red[2][threadIdx.x] : 0.f);
		if (threadIdx.x == 0) {
			atomicAdd(&g_ae[c * stride_c], s0);
			atomicAdd(&g_ae[c * stride_c + stride_j], s1);
			if (g_a) atomicAdd(&g_a[c], sa);
		}
	}
}

// g[j] += sum over pixels of e[b][j][p], j = 0, 1
__global__ void sum2_kernel(const float* __restrict__ e, float* __restrict__ g, int B, int npix) {
	const long long n = (long long)B * npix;
	float s0 = 0.f, s1 = 0.f;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
		const long long b = t / npix;
		const int p = (int)(t - b * npix);
		s0 += e[b * 2 * npix + p];
		s1 += e[b * 2 * npix + npix + p];
	}
	s0 = warp_sum(s0);
	s1 = warp_sum(s1);
	if ((threadIdx.x & 31) == 0) {
		atomicAdd(&g[0], s0);
		atomicAdd(&g[1], s1);
	}
}

__global__ void to_bf16(const float* __restrict__ a, __nv_bfloat16* __restrict__ b, long long n) {
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		b[i] = __float2bfloat16(a[i]);
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
		const float gi = g[i];
		const float mi = b1 * m[i] + (1.f - b1) * gi;
		const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
		m[i] = mi;
		v[i] = vi;
		p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
	}
}

// Tiles of a periodic two-field FP64 grid as FP32 network input. Tile j of the
// batch is block (first + j) of the grid's core x core blocks (row-major over
// tiles_x columns) plus halo points on each side, wrapped periodically.
__global__ void gather_tiles(const double* __restrict__ f, float* __restrict__ out, int Nx, int Ny, int T, int core,
                             int halo, int tiles_x, int first, int count) {
	const long long per = 2LL * T * T;
	const long long n = per * count;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
		const int j = (int)(t / per);
		const int r = (int)(t - (long long)j * per);
		const int u = r / (T * T), q = r - u * T * T;
		const int ty = q / T, tx = q - ty * T;
		const int tile = first + j;
		const int by = tile / tiles_x, bx = tile - by * tiles_x;
		int x = (bx * core - halo + tx) % Nx, y = (by * core - halo + ty) % Ny;
		if (x < 0) x += Nx;
		if (y < 0) y += Ny;
		out[t] = (float)f[((long long)u * Ny + y) * Nx + x];
	}
}

// Writes each tile's core block of the network output back to the grid.
__global__ void scatter_tiles(const float* __restrict__ in, double* __restrict__ f, int Nx, int Ny, int T, int core,
                              int halo, int tiles_x, int first, int count) {
	const long long per = 2LL * core * core;
	const long long n = per * count;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
		const int j = (int)(t / per);
		const int r = (int)(t - (long long)j * per);
		const int u = r / (core * core), q = r - u * core * core;
		const int cy = q / core, cx = q - cy * core;
		const int tile = first + j;
		const int by = tile / tiles_x, bx = tile - by * tiles_x;
		const int x = bx * core + cx, y = by * core + cy;
		if (x >= Nx || y >= Ny) continue;
		f[((long long)u * Ny + y) * Nx + x] =
		    (double)in[(long long)j * 2 * T * T + ((long long)u * T + halo + cy) * T + halo + cx];
	}
}

// Per-block FP64 partial sums of (out - in) for each of the two fields.
constexpr int MEAN_BLOCKS = 296;
__global__ void diff_partials(const double* __restrict__ in, const double* __restrict__ out, double* __restrict__ part,
                              long long npts) {
	__shared__ double red[2][32];
	for (int u = 0; u < 2; u++) {
		double s = 0.0;
		for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npts;
		     i += (long long)gridDim.x * blockDim.x)
			s += out[u * npts + i] - in[u * npts + i];
		s = warp_sum(s);
		if ((threadIdx.x & 31) == 0) red[u][threadIdx.x >> 5] = s;
	}
	__syncthreads();
	if (threadIdx.x < 32) {
		for (int u = 0; u < 2; u++) {
			double s = threadIdx.x < (blockDim.x >> 5) ? red[u][threadIdx.x] : 0.0;
			s = warp_sum(s);
			if (threadIdx.x == 0) part[u * gridDim.x + blockIdx.x] = s;
		}
	}
}

// out[u] -= (sum of the partials of u) / npts: gives each field back the
// input's mean (the relaxation conserves it). Fixed summation order.
__global__ void restore_means(double* __restrict__ out, const double* __restrict__ part, int nparts, long long npts) {
	__shared__ double shift[2];
	if (threadIdx.x < 2) {
		double s = 0.0;
		for (int i = 0; i < nparts; i++) s += part[threadIdx.x * nparts + i];
		shift[threadIdx.x] = s / (double)npts;
	}
	__syncthreads();
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 2 * npts;
	     i += (long long)gridDim.x * blockDim.x)
		out[i] -= shift[i >= npts];
}

int grid_for(long long n, int block) {
	long long g = (n + block - 1) / block;
	return (int)(g > 148 * 16 ? 148 * 16 : (g < 1 ? 1 : g));
}


thread_local std::string g_fno_err;

} // namespace

struct pfcg_fno {
	int T = 0, maxB = 0;
	cudaStream_t stream = nullptr;
	float* p = nullptr;          // master weights (FP32)
	__nv_bfloat16* w = nullptr;  // BF16 copy read by the kernels
	float* g = nullptr;          // gradients
	float* am = nullptr;         // Adam moments
	float* av = nullptr;
	long long adam_t = 0;
	float2* tw = nullptr;        // twiddles of the tile size
	uint4* fdx = nullptr;        // mma fragments of the truncated x transforms (dft_frag_kernel)
	uint4* fix = nullptr;
	uint4* fdy = nullptr;        // mma fragments of the truncated y transforms (dfty_frag_kernel)
	uint4* fiy = nullptr;
	float* sx = nullptr;         // per-kx weights of the truncated irfft2: (kx ? 2 : 1) / T^2
	float* v[L + 1] = {};        // layer inputs (v[L] feeds the projection)
	float* z[L] = {};            // pre-activations
	float* s = nullptr;          // spectral branch output
	float2* A = nullptr;         // [B][C][T][MX] x-transformed rows (and adjoint scratch)
	float2* X[L] = {};           // [B][C][MY][MX] retained modes of each layer input
	float2* Y = nullptr;         // [B][C][MY][MX] mixed modes
	float2* Bq = nullptr;        // [B][C][T][MX] y-inverse rows (and adjoint scratch)
	float* dv = nullptr;         // gradient scratch
	float* dv2 = nullptr;
	float* dz = nullptr;
	float* x = nullptr;          // [B][2][T][T] tile input (apply)
	float* y = nullptr;          // [B][2][T][T] network output
	float* dy = nullptr;
	double* loss = nullptr;
	double* field_tmp = nullptr; // grid-sized scratch for the warm start
	size_t field_tmp_n = 0;
	double* part = nullptr;      // mean partial sums [2][MEAN_BLOCKS]
	long long launches = 0;
	std::string err;
};

namespace {

int ffail(pfcg_fno* f, int code, const std::string& m) {
	if (f) f->err = m;
	g_fno_err = m;
	return code;
}

#define FCK(call)                                                                                                      \
	do {                                                                                                           \
		cudaError_t e_ = (call);                                                                               \
		if (e_ != cudaSuccess) return ffail(f, PFCG_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
	} while (0)

// forward pass over a batch of B tiles; with train the pre-activations are kept for backward
int forward(pfcg_fno* f, const float* x, int B, const float* target, bool train) {
	const int T = f->T, npix = T * T;
	const long long rows = (long long)B * C * T, planes = (long long)B * C;
	cudaStream_t st = f->stream;
	lift_fwd<<<grid_for((long long)B * npix, 256), 256, 0, st>>>(x, f->w, f->v[0], B, npix);
	f->launches++;
	for (int l = 0; l < L; l++) {
		dft_x<<<grid_for(rows * 2, 256), 256, 0, st>>>(f->v[l], f->A, f->fdx, nullptr, rows, T);
		dft_y_fwd<<<grid_for(planes * 32 * DY_WARPS, 32 * DY_WARPS), 32 * DY_WARPS, 0, st>>>(f->A, f->X[l], f->fdy, planes, T);
		mix<<<grid_for((long long)NK * ((B + 15) / 16) * 8 * 32, 128), 128, 0, st>>>(f->X[l], f->Y, f->w, l, B, 0);
		dft_y_inv<<<grid_for(planes * 32 * DY_WARPS, 32 * DY_WARPS), 32 * DY_WARPS, 0, st>>>(f->Y, f->Bq, f->fiy, planes, T);
		idft_x<<<grid_for(rows * 2, 256), 256, 0, st>>>(f->Bq, f->s, f->fix, f->sx, rows, T, 0);
		pointwise_fwd<<<grid_for((long long)B * npix / 16 * 32, 128), 128, 0, st>>>(f->v[l], f->s, f->w, l, train ? f->z[l] : nullptr,
		                                                                    f->v[l + 1], B, npix, l < L - 1);
		f->launches += 6;
	}
	if (target) FCK(cudaMemsetAsync(f->loss, 0, sizeof(double), st));
	proj_fwd_loss<<<grid_for((long long)B * npix, 256), 256, 0, st>>>(x, f->v[L], f->w, f->y, target, f->dy, f->loss, B,
	                                                                 npix);
	f->launches++;
	FCK(cudaGetLastError());
	return 0;
}

int backward(pfcg_fno* f, const float* x, int B) {
	const int T = f->T, npix = T * T;
	const long long rows = (long long)B * C * T, planes = (long long)B * C;
	cudaStream_t st = f->stream;
	const dim3 cg(std::min(grid_for((long long)B * npix, 256), 64), C);
	const int wg = std::min(grid_for((long long)B * npix / 16 / (WG_THREADS / 32), 1), 148 * 4);
	FCK(cudaMemsetAsync(f->g, 0, sizeof(float) * NPARAM, st));
	// projection: dQ[j][c] = sum v_L[c] dy[j], dq[j] = sum dy[j], dv_L = Q^T dy
	channel_grad<<<cg, 256, 0, st>>>(f->v[L], f->dy, f->g + OFF_Q, 1, C, nullptr, B, npix);
	sum2_kernel<<<grid_for((long long)B * npix, 256), 256, 0, st>>>(f->dy, f->g + OFF_QB, B, npix);
	proj_bwd<<<grid_for((long long)B * npix, 256), 256, 0, st>>>(f->dy, f->w, f->dv, B, npix);
	f->launches += 3;
	for (int l = L - 1; l >= 0; l--) {
		pointwise_bwd<<<grid_for((long long)B * npix / 16 * 32, 128), 128, 0, st>>>(f->z[l], f->dv, f->w, l, f->dz, f->dv2, B, npix,
		                                                                    l < L - 1);
		weight_grad<<<wg, WG_THREADS, 0, st>>>(f->dz, f->v[l], f->g + off_W(l), f->g + off_b(l), B, npix);
		// spectral branch, in reverse
		dft_x<<<grid_for(rows * 2, 256), 256, 0, st>>>(f->dz, f->Bq, f->fdx, f->sx, rows, T);
		dft_y_fwd<<<grid_for(planes * 32 * DY_WARPS, 32 * DY_WARPS), 32 * DY_WARPS, 0, st>>>(f->Bq, f->Y, f->fdy, planes, T);
		mix_grad<<<grid_for((long long)C * C * NK, 256), 256, 0, st>>>(f->X[l], f->Y, f->g, l, B);
		mix<<<grid_for((long long)NK * ((B + 15) / 16) * 8 * 32, 128), 128, 0, st>>>(f->Y, f->Bq, f->w, l, B, 1);
		dft_y_inv<<<grid_for(planes * 32 * DY_WARPS, 32 * DY_WARPS), 32 * DY_WARPS, 0, st>>>(f->Bq, f->A, f->fiy, planes, T);
		idft_x<<<grid_for(rows * 2, 256), 256, 0, st>>>(f->A, f->dv2, f->fix, nullptr, rows, T, 1);
		f->launches += 8;
		std::swap(f->dv, f->dv2);
	}
	// lift: dP[c][j] = sum dv0[c] x[j], dp[c] = sum dv0[c]
	channel_grad<<<cg, 256, 0, st>>>(f->dv, x, f->g + OFF_P, 2, 1, f->g + OFF_PB, B, npix);
	f->launches++;
	FCK(cudaGetLastError());
	return 0;
}

} // namespace

int fno_apply_device(pfcg_fno* f, const double* d_in, double* d_out, int Nx, int Ny, cudaStream_t st) {
	const int T = f->T, halo = T / 4, core = T - 2 * halo;
	const int tx = (Nx + core - 1) / core, ty = (Ny + core - 1) / core;
	const int ntiles = tx * ty;
	const cudaStream_t own = f->stream;
	cudaEvent_t ev;
	FCK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
	FCK(cudaEventRecord(ev, st));
	FCK(cudaStreamWaitEvent(own, ev, 0));
	for (int first = 0; first < ntiles; first += f->maxB) {
		const int count = std::min(f->maxB, ntiles - first);
		gather_tiles<<<grid_for(2LL * T * T * count, 256), 256, 0, own>>>(d_in, f->x, Nx, Ny, T, core, halo, tx, first,
		                                                                  count);
		f->launches++;
		int rc = forward(f, f->x, count, nullptr, false);
		if (rc) return rc;
		scatter_tiles<<<grid_for(2LL * core * core * count, 256), 256, 0, own>>>(f->y, d_out, Nx, Ny, T, core, halo, tx,
		                                                                         first, count);
		f->launches++;
	}
	const long long npts = (long long)Nx * Ny;
	diff_partials<<<MEAN_BLOCKS, 256, 0, own>>>(d_in, d_out, f->part, npts);
	restore_means<<<grid_for(2 * npts, 256), 256, 0, own>>>(d_out, f->part, MEAN_BLOCKS, npts);
	f->launches += 2;
	FCK(cudaGetLastError());
	FCK(cudaEventRecord(ev, own));
	FCK(cudaStreamWaitEvent(st, ev, 0));
	FCK(cudaEventDestroy(ev));
	return 0;
}

int fno_scratch_grid(pfcg_fno* f, size_t n, double** out) {
	if (f->field_tmp_n < n) {
		cudaFree(f->field_tmp);
		f->field_tmp = nullptr;
		f->field_tmp_n = 0;
		FCK(cudaMalloc(&f->field_tmp, sizeof(double) * n));
		f->field_tmp_n = n;
	}
	*out = f->field_tmp;
	return 0;
}

const char* fno_error(const pfcg_fno* f) { return f->err.c_str(); }

extern "C" {

size_t pfcg_fno_param_count(void) { return NPARAM; }

int pfcg_fno_create(int tile, int max_batch, pfcg_fno** out) {
	if (!out) return ffail(nullptr, PFCG_EARG, "NULL argument");
	*out = nullptr;
	if (tile < 2 * MY || tile > MAXT || (tile & (tile - 1)) != 0 || max_batch < 1)
		return ffail(nullptr, PFCG_EARG, "tile must be a power of two in [32, 512] and max_batch >= 1");
	pfcg_fno* f = new pfcg_fno();
	f->T = tile;
	f->maxB = max_batch;
	const long long npix = (long long)tile * tile;
	const size_t nv = (size_t)max_batch * C * npix;
	cudaError_t e = cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking);
	std::vector<void**> bufs;
	std::vector<size_t> sizes;
	auto add = [&](void** ptr, size_t bytes) {
		bufs.push_back(ptr);
		sizes.push_back(bytes);
	};
	// the first five (weights, gradients, moments) are cleared below
	add((void**)&f->p, sizeof(float) * NPARAM);
	add((void**)&f->w, sizeof(__nv_bfloat16) * NPARAM);
	add((void**)&f->g, sizeof(float) * NPARAM);
	add((void**)&f->am, sizeof(float) * NPARAM);
	add((void**)&f->av, sizeof(float) * NPARAM);
	add((void**)&f->tw, sizeof(float2) * tile);
	add((void**)&f->fdx, sizeof(uint4) * (tile / 16) * 2 * 32);
	add((void**)&f->fix, sizeof(uint4) * (tile / 8) * 32);
	add((void**)&f->fdy, sizeof(uint4) * (tile / 8) * 32 * 2);
	add((void**)&f->fiy, sizeof(uint4) * (tile / 16) * 2 * 32 * 2);
	add((void**)&f->sx, sizeof(float) * MX);
	for (int l = 0; l <= L; l++) add((void**)&f->v[l], sizeof(float) * nv);
	for (int l = 0; l < L; l++) add((void**)&f->z[l], sizeof(float) * nv);
	for (int l = 0; l < L; l++) add((void**)&f->X[l], sizeof(float2) * max_batch * C * NK);
	add((void**)&f->s, sizeof(float) * nv);
	add((void**)&f->A, sizeof(float2) * max_batch * C * tile * MX);
	add((void**)&f->Y, sizeof(float2) * max_batch * C * NK);
	add((void**)&f->Bq, sizeof(float2) * max_batch * C * tile * MX);
	add((void**)&f->dv, sizeof(float) * nv);
	add((void**)&f->dv2, sizeof(float) * nv);
	add((void**)&f->dz, sizeof(float) * nv);
	add((void**)&f->x, sizeof(float) * max_batch * 2 * npix);
	add((void**)&f->y, sizeof(float) * max_batch * 2 * npix);
	add((void**)&f->dy, sizeof(float) * max_batch * 2 * npix);
	add((void**)&f->loss, sizeof(double));
	add((void**)&f->part, sizeof(double) * 2 * MEAN_BLOCKS);
	for (size_t i = 0; i < bufs.size() && e == cudaSuccess; i++) e = cudaMalloc(bufs[i], sizes[i]);
	if (e != cudaSuccess) {
		pfcg_fno_destroy(f);
		return ffail(nullptr, PFCG_ENOMEM, std::string("device allocation: ") + cudaGetErrorString(e));
	}
	float sc[MX];
	for (int m = 0; m < MX; m++) sc[m] = (m == 0 ? 1.f : 2.f) / (float)npix;
	e = cudaMemcpyAsync(f->sx, sc, sizeof(sc), cudaMemcpyHostToDevice, f->stream);
	twiddle_kernel<<<1, 256, 0, f->stream>>>(f->tw, tile);
	dft_frag_kernel<<<(tile * 8 + 255) / 256, 256, 0, f->stream>>>(f->tw, tile, f->fdx, f->fix);
	dfty_frag_kernel<<<(tile * 8 + 255) / 256, 256, 0, f->stream>>>(f->tw, tile, f->fdy, f->fiy);
	f->launches += 2;
	for (size_t i = 0; i < 5 && e == cudaSuccess; i++) e = cudaMemsetAsync(*bufs[i], 0, sizes[i], f->stream);
	if (e == cudaSuccess) e = cudaStreamSynchronize(f->stream);
	if (e == cudaSuccess) e = cudaGetLastError();
	if (e != cudaSuccess) {
		pfcg_fno_destroy(f);
		return ffail(nullptr, PFCG_ECUDA, std::string("set-up: ") + cudaGetErrorString(e));
	}
	*out = f;
	return 0;
}

void pfcg_fno_destroy(pfcg_fno* f) {
	if (!f) return;
	if (f->stream) cudaStreamSynchronize(f->stream);
	void* ptrs[] = {f->p,  f->w,  f->g,  f->am, f->av,   f->tw,        f->sx,   f->s,   f->A,   f->Y,   f->Bq, f->dv,
	                f->dv2, f->dz, f->x, f->y,  f->dy,   f->loss,      f->field_tmp, f->part, f->fdx, f->fix, f->fdy, f->fiy};
	for (void* q : ptrs) cudaFree(q);
	for (int l = 0; l <= L; l++) cudaFree(f->v[l]);
	for (int l = 0; l < L; l++) {
		cudaFree(f->z[l]);
		cudaFree(f->X[l]);
	}
	if (f->stream) cudaStreamDestroy(f->stream);
	delete f;
}

int pfcg_fno_set_params(pfcg_fno* f, const float* host_params) {
	if (!f || !host_params) return ffail(f, PFCG_EARG, "NULL argument");
	FCK(cudaMemcpyAsync(f->p, host_params, sizeof(float) * NPARAM, cudaMemcpyHostToDevice, f->stream));
	to_bf16<<<grid_for(NPARAM, 256), 256, 0, f->stream>>>(f->p, f->w, NPARAM);
	f->launches++;
	FCK(cudaMemsetAsync(f->am, 0, sizeof(float) * NPARAM, f->stream));
	FCK(cudaMemsetAsync(f->av, 0, sizeof(float) * NPARAM, f->stream));
	f->adam_t = 0;
	FCK(cudaStreamSynchronize(f->stream));
	return 0;
}

int pfcg_fno_get_params(pfcg_fno* f, float* host_params) {
	if (!f || !host_params) return ffail(f, PFCG_EARG, "NULL argument");
	FCK(cudaMemcpyAsync(host_params, f->p, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, f->stream));
	FCK(cudaStreamSynchronize(f->stream));
	return 0;
}

int pfcg_fno_forward(pfcg_fno* f, const float* d_in, float* d_out, int batch) {
	if (!f || !d_in || !d_out) return ffail(f, PFCG_EARG, "NULL argument");
	if (batch < 1 || batch > f->maxB) return ffail(f, PFCG_EARG, "batch outside [1, max_batch]");
	int rc = forward(f, d_in, batch, nullptr, false);
	if (rc) return rc;
	FCK(cudaMemcpyAsync(d_out, f->y, sizeof(float) * batch * 2 * f->T * f->T, cudaMemcpyDeviceToDevice, f->stream));
	FCK(cudaStreamSynchronize(f->stream));
	return 0;
}

int pfcg_fno_loss_grad(pfcg_fno* f, const float* d_in, const float* d_target, int batch, double* loss,
                       float* host_grad) {
	if (!f || !d_in || !d_target) return ffail(f, PFCG_EARG, "NULL argument");
	if (batch < 1 || batch > f->maxB) return ffail(f, PFCG_EARG, "batch outside [1, max_batch]");
	int rc = forward(f, d_in, batch, d_target, true);
	if (!rc) rc = backward(f, d_in, batch);
	if (rc) return rc;
	if (loss) FCK(cudaMemcpyAsync(loss, f->loss, sizeof(double), cudaMemcpyDeviceToHost, f->stream));
	if (host_grad) FCK(cudaMemcpyAsync(host_grad, f->g, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, f->stream));
	FCK(cudaStreamSynchronize(f->stream));
	return 0;
}

int pfcg_fno_adam_step(pfcg_fno* f, float lr, float beta1, float beta2, float eps) {
	if (!f) return ffail(f, PFCG_EARG, "NULL argument");
	f->adam_t++;
	const float c1 = 1.f - std::pow(beta1, (float)f->adam_t), c2 = 1.f - std::pow(beta2, (float)f->adam_t);
	adam_kernel<<<grid_for(NPARAM, 256), 256, 0, f->stream>>>(f->p, f->g, f->am, f->av, NPARAM, lr, beta1, beta2, eps,
	                                                           c1, c2);
	to_bf16<<<grid_for(NPARAM, 256), 256, 0, f->stream>>>(f->p, f->w, NPARAM);
	f->launches += 2;
	FCK(cudaGetLastError());
	return 0;
}

int pfcg_fno_apply(pfcg_fno* f, const double* d_in, double* d_out, int Nx, int Ny, void* stream) {
	if (!f || !d_in || !d_out) return ffail(f, PFCG_EARG, "NULL argument");
	if (d_in == d_out) return ffail(f, PFCG_EARG, "input and output grids must be distinct");
	if (Nx < 1 || Ny < 1) return ffail(f, PFCG_EARG, "empty grid");
	cudaStream_t st = (cudaStream_t)stream;
	int rc = fno_apply_device(f, d_in, d_out, Nx, Ny, st);
	if (rc) return rc;
	FCK(cudaStreamSynchronize(st));
	return 0;
}

int pfcg_fno_stream(const pfcg_fno* f, void** stream) {
	if (!f || !stream) return PFCG_EARG;
	*stream = (void*)f->stream;
	return 0;
}

int pfcg_fno_launch_count(const pfcg_fno* f, long long* count) {
	if (!f || !count) return PFCG_EARG;
	*count = f->launches;
	return 0;
}

const char* pfcg_fno_last_error(const pfcg_fno* f) { return f ? f->err.c_str() : g_fno_err.c_str(); }

} // extern "C"
