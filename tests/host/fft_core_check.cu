// Host-side check of the in-register DFTs and the compile-time pass plans of
// pfc_b200/csrc/fft_core.cuh (their __host__ __device__ code compiled for the
// CPU): every dft<R> against a direct FP64 DFT in both directions, and for
// every specialised length the plan's radix product, tail and twiddle count.
// Prints one line per check and exits non-zero on any failure.
#include "../../pfc_b200/csrc/fft_core.cuh"

#include <cmath>
#include <cstdio>

using namespace pfcg;

static int failures = 0;

template <int R, int SIGN> static void check_dft() {
	cplx<double> v[R], ref[R];
	for (int i = 0; i < R; i++) v[i] = mk<double>(std::sin(1.3 * i + 0.2 * R), std::cos(0.7 * i * i + R));
	for (int k = 0; k < R; k++) {
		double re = 0, im = 0;
		for (int n = 0; n < R; n++) {
			const double a = SIGN * 2.0 * M_PI * n * k / R;
			re += v[n].x * std::cos(a) - v[n].y * std::sin(a);
			im += v[n].x * std::sin(a) + v[n].y * std::cos(a);
		}
		ref[k] = mk<double>(re, im);
	}
	dft<R, SIGN, double>(v);
	double err = 0;
	for (int k = 0; k < R; k++) err = std::fmax(err, std::hypot(v[k].x - ref[k].x, v[k].y - ref[k].y));
	const bool ok = err < 1e-13;
	failures += !ok;
	std::printf("dft%d sign %+d max error %.2e %s\n", R, SIGN, err, ok ? "ok" : "FAIL");
}

template <int N, int RM> static void check_plan() {
	using PL = CtPlan<N, RM>;
	int prod = 1, tw = 0;
	for (int p = 0; p < PL::NPASS; p++) {
		if (p > 0) tw += PL::twcnt(PL::radix(p)) * PL::ns(p);
		prod *= PL::radix(p);
	}
	const bool ok = prod == N && PL::FUSABLE && PL::radix(0) == RM && PL::radix(PL::NPASS - 1) == RM &&
	                tw == PL::TWN && PL::ns(PL::NPASS - 1) * RM == N;
	failures += !ok;
	std::printf("plan %d radix %d: passes %d tail %d twiddles %d %s\n", N, RM, PL::NPASS, PL::RT, PL::TWN,
	            ok ? "ok" : "FAIL");
}

// ct_twiddle on a radix-16 pass (powers 1, 2, 3, 4, 8, 12 tabulated, the rest
// as products) against the direct powers exp(SIGN 2 pi i r jm / (NS 16))
template <int NS, int SIGN> static void check_twiddle16() {
	cplx<double> tab[6 * NS];
	const int pw[6] = {1, 2, 3, 4, 8, 12};
	for (int q = 0; q < 6; q++)
		for (int jm = 0; jm < NS; jm++) {
			const double a = -2.0 * M_PI * pw[q] * jm / (NS * 16.0);
			tab[q * NS + jm] = mk<double>(std::cos(a), std::sin(a));
		}
	double err = 0;
	for (int jm = 0; jm < NS; jm++) {
		cplx<double> v[16];
		for (int r = 0; r < 16; r++) v[r] = mk<double>(1.0, 0.0);
		ct_twiddle<16, NS, SIGN, double>(v, tab + jm);
		for (int r = 1; r < 16; r++) {
			const double a = SIGN * 2.0 * M_PI * r * jm / (NS * 16.0);
			err = std::fmax(err, std::hypot(v[r].x - std::cos(a), v[r].y - std::sin(a)));
		}
	}
	const bool ok = err < 1e-14;
	failures += !ok;
	std::printf("twiddle16 NS %d sign %+d max error %.2e %s\n", NS, SIGN, err, ok ? "ok" : "FAIL");
}

int main() {
	check_twiddle16<16, -1>(); check_twiddle16<16, 1>(); check_twiddle16<256, -1>(); check_twiddle16<256, 1>();
	check_dft<2, -1>(); check_dft<2, 1>();
	check_dft<3, -1>(); check_dft<3, 1>();
	check_dft<4, -1>(); check_dft<4, 1>();
	check_dft<5, -1>(); check_dft<5, 1>();
	check_dft<6, -1>(); check_dft<6, 1>();
	check_dft<7, -1>(); check_dft<7, 1>();
	check_dft<8, -1>(); check_dft<8, 1>();
	check_dft<16, -1>(); check_dft<16, 1>();
	// FP32 (radix 16) and FP64 (radix 8) specialised lengths
	check_plan<256, 16>(); check_plan<384, 8>(); check_plan<512, 16>(); check_plan<768, 16>(); check_plan<1024, 16>();
	check_plan<1536, 16>(); check_plan<2048, 16>(); check_plan<4096, 16>();
	check_plan<2048, 8>(); check_plan<4096, 8>();
	return failures ? 1 : 0;
}
