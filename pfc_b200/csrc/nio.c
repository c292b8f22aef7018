/* Multithreaded .n text I/O (nio.h). */
#include "nio.h"

#include <ctype.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* The first n whitespace-separated numbers of [q, e) into out, parsed by
 * strtod in parallel: the text is cut into one segment per thread at
 * whitespace, each thread parses its segment up to the first token that is not
 * a number, and the segments are joined in order. Returns 0, or 1 when fewer
 * than n numbers precede the first bad token or the end (the reference's
 * fscanf failure, code 38). Values after the first n are not looked at. */
int nio_parse_values(const char* q, const char* e, double* out, size_t n) {
	int nt = 1;
#ifdef _OPENMP
	nt = omp_get_max_threads();
#endif
	const size_t len = (size_t)(e - q);
	if (len < (size_t)nt * 4096) nt = 1;
	const char** cut = (const char**)malloc(sizeof(char*) * (nt + 1));
	cut[0] = q;
	cut[nt] = e;
	for (int k = 1; k < nt; k++) {
		const char* c = q + len / nt * k;
		if (c < cut[k - 1]) c = cut[k - 1];
		while (c < e && !isspace((unsigned char)*c)) c++; /* never split a token */
		cut[k] = c;
	}
	double** part = (double**)calloc(nt, sizeof(double*));
	size_t* cnt = (size_t*)calloc(nt, sizeof(size_t));
	int* bad = (int*)calloc(nt, sizeof(int));
#pragma omp parallel for schedule(static, 1) num_threads(nt)
	for (int k = 0; k < nt; k++) {
		size_t cap = 1024, m = 0;
		double* v = (double*)malloc(sizeof(double) * cap);
		const char* c = cut[k];
		char* end;
		for (;;) {
			while (c < cut[k + 1] && isspace((unsigned char)*c)) c++;
			if (c >= cut[k + 1]) break;
			const double x = strtod(c, &end);
			if (end == c) {
				bad[k] = 1;
				break;
			}
			if (m == cap) v = (double*)realloc(v, sizeof(double) * (cap *= 2));
			v[m++] = x;
			c = end;
		}
		part[k] = v;
		cnt[k] = m;
	}
	size_t got = 0;
	int fail = 0;
	for (int k = 0; k < nt && got < n; k++) {
		const size_t take = cnt[k] < n - got ? cnt[k] : n - got;
		memcpy(out + got, part[k], sizeof(double) * take);
		got += take;
		if (bad[k] && got < n) fail = 1;
		if (fail) break;
	}
	if (got < n) fail = 1;
	for (int k = 0; k < nt; k++) free(part[k]);
	free(part);
	free(cnt);
	free(bad);
	free(cut);
	return fail;
}

/* blocks of B lines are formatted in parallel, one buffer each, then written in order */
static void write_blocks(FILE* f, int prec, const double* a, const double* b, size_t n) {
	int nt = 1;
#ifdef _OPENMP
	nt = omp_get_max_threads();
#endif
	const size_t B = 1 << 15;
	const size_t per = (b ? 2 : 1) * (48 + (size_t)(prec > 0 ? prec : 0));
	char** buf = (char**)malloc(sizeof(char*) * nt);
	size_t* used = (size_t*)malloc(sizeof(size_t) * nt);
	for (int k = 0; k < nt; k++) buf[k] = (char*)malloc(B * per);
	for (size_t g0 = 0; g0 < n; g0 += B * nt) {
#pragma omp parallel for schedule(static, 1) num_threads(nt)
		for (int k = 0; k < nt; k++) {
			const size_t i0 = g0 + (size_t)k * B;
			const size_t i1 = i0 + B < n ? i0 + B : n;
			size_t pos = 0;
			for (size_t i = i0; i < i1; i++)
				pos += b ? (size_t)snprintf(buf[k] + pos, per, "%.*e %.*e\n", prec, a[i], prec, b[i])
				         : (size_t)snprintf(buf[k] + pos, per, "%.*e\n", prec, a[i]);
			used[k] = i0 < n ? pos : 0;
		}
		for (int k = 0; k < nt; k++)
			if (used[k]) fwrite(buf[k], 1, used[k], f);
	}
	for (int k = 0; k < nt; k++) free(buf[k]);
	free(buf);
	free(used);
}

void nio_write_pairs(FILE* f, int prec, const double* a, const double* b, size_t n) { write_blocks(f, prec, a, b, n); }

void nio_write_values(FILE* f, int prec, const double* v, size_t n) { write_blocks(f, prec, v, NULL, n); }

char* nio_slurp(const char* path, size_t* len) {
	FILE* f = fopen(path, "rb");
	if (!f) return NULL;
	fseek(f, 0, SEEK_END);
	long n = ftell(f);
	fseek(f, 0, SEEK_SET);
	char* buf = (char*)malloc((size_t)n + 1);
	size_t got = fread(buf, 1, (size_t)n, f);
	buf[got] = '\0';
	fclose(f);
	*len = got;
	return buf;
}
