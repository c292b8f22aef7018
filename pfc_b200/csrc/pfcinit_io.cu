// Output of the reference's initial-state builder (src/PFCInit.java:670-686,
// step "O"): the header "Nx Ny " + dx and dy in "%.{prec}e", then every value
// (y-major) on its own line in the same format, written by Java's Formatter.
//
// Java's %e and C's differ in rounding. Java (java.util.Formatter through
// FormattedFloatingDecimal) takes the shortest decimal digits that read back
// to the double and rounds those half up at prec + 1 significant digits; C
// rounds the exact binary value, ties to even. The results differ only when
// the shortest digits are exactly prec + 2 long and end in 5: the exact value
// may then lie below that 5 (C rounds down, Java up), or on it (C's tie goes
// to even). Such a value is recognised from C's own correctly rounded
// prec + 2 digit form: it ends in 5 and reads back to the value. For prec <= 13
// that form is then the shortest one: decimals of prec + 2 <= 15 significant
// digits lie more than a binary64 ulp apart (10^-15 > 2^-52 relative), so no
// two of them read back to one double, and the test is exact there.
// Host code only.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pfc_b200.h"

namespace {

// Java's String.format("%.{prec}e", v) into out; returns its length
int java_e(char* out, size_t cap, double v, int prec) {
	if (std::isnan(v)) return snprintf(out, cap, "NaN");
	if (std::isinf(v)) return snprintf(out, cap, v > 0 ? "Infinity" : "-Infinity");
	const int n = snprintf(out, cap, "%.*e", prec, v);
	if (v == 0.0 || prec > 13) return n;
	char t[64];
	snprintf(t, sizeof t, "%.*e", prec + 1, v);
	char* e = strchr(t, 'e');
	if (!e || e[-1] != '5' || strtod(t, nullptr) != v) return n;
	// the shortest digits end in that 5: round them half up, i.e. drop the 5
	// and add one unit in the last kept place
	const bool neg = t[0] == '-';
	std::string dig;
	for (const char* c = t + (neg ? 1 : 0); c < e; c++)
		if (*c != '.') dig.push_back(*c);
	dig.pop_back();
	int exp10 = atoi(e + 1);
	int k = (int)dig.size() - 1;
	while (k >= 0 && dig[k] == '9') dig[k--] = '0';
	if (k >= 0) dig[k]++;
	else {
		dig.insert(dig.begin(), '1');
		dig.pop_back();
		exp10++;
	}
	std::string r = neg ? "-" : "";
	r.push_back(dig[0]);
	if (prec > 0) {
		r.push_back('.');
		r.append(dig, 1, std::string::npos);
	}
	char ex[16];
	snprintf(ex, sizeof ex, "e%c%02d", exp10 < 0 ? '-' : '+', exp10 < 0 ? -exp10 : exp10);
	r += ex;
	return snprintf(out, cap, "%s", r.c_str());
}

} // namespace

extern "C" int pfcg_write_n_pfcinit(const char* path, int Nx, int Ny, double dx, double dy, const double* field,
                                    int prec) {
	if (!path || !field || Nx < 1 || Ny < 1 || prec < 0 || prec > 30) return PFCG_EARG;
	FILE* f = fopen(path, "wb");
	if (!f) return PFCG_EARG;
	char a[96], b[96];
	java_e(a, sizeof a, dx, prec);
	java_e(b, sizeof b, dy, prec);
	fprintf(f, "%d %d %s %s\n", Nx, Ny, a, b);
	// blocks of lines formatted in parallel, written in order
	const size_t n = (size_t)Nx * Ny, B = 1 << 16;
	const size_t nblk = (n + B - 1) / B;
	unsigned nt = std::thread::hardware_concurrency();
	if (nt < 1) nt = 1;
	if (nt > 16) nt = 16;
	bool ok = true;
	for (size_t b0 = 0; b0 < nblk && ok; b0 += nt) {
		const size_t nb = std::min<size_t>(nt, nblk - b0);
		std::vector<std::string> text(nb);
		std::vector<std::thread> th;
		for (size_t q = 0; q < nb; q++)
			th.emplace_back([&, q]() {
				const size_t lo = (b0 + q) * B, hi = std::min(n, lo + B);
				std::string& s = text[q];
				s.reserve((hi - lo) * (prec + 10));
				char buf[96];
				for (size_t i = lo; i < hi; i++) {
					const int m = java_e(buf, sizeof buf, field[i], prec);
					s.append(buf, (size_t)m);
					s.push_back('\n');
				}
			});
		for (auto& t : th) t.join();
		for (auto& s : text)
			if (fwrite(s.data(), 1, s.size(), f) != s.size()) ok = false;
	}
	if (fclose(f) != 0) ok = false;
	return ok ? 0 : PFCG_EARG;
}
