/*
 * pfc_oracle — CPU restatement (FP64) of the pfc-relax spectral relaxation.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the GPU path is compared with;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * it. The product (libpfc_b200.so, the pfc-relax driver) never links it.
 *
 * It restates, in plain C over oracle/fft64.c, the functions of
 * demos/honey/pfc-relax.c (line numbers below refer to that file):
 *   update_AB   :901-958    linear operators A = exp(o a dt), B = (A-1)/a / (Nx Ny)
 *   step        :1134-1248  NaN check, resync every 100 steps, real-space
 *                           nonlinear term, r2c, k-space coupling + ETD1, c2r
 *   evaluate    :988-1131   free-energy density in real space, <f>, <n_u>
 *   optimize    :1251-1290  five-point box-size sampling and parabola vertex
 * with the same loop order and arithmetic, so that on one rank it agrees with
 * the reference binary built over the same FFT (oracle/_ref/) to rounding.
 *
 * One deliberate difference: evaluate() uses mu2[u][v] in the gradient
 * coupling q_uv, where the reference reads s->nu2 (:1020; out of bounds when
 * v >= W[u]). The two agree whenever beta[u][v] == 0 for all u < v; the
 * reference source with that one line corrected is built as
 * oracle/_ref/pfc-relax-mu2fix for the other cases. Set emulate_nu2 to follow
 * the reference instead (valid only when v < W[u]).
 *
 * Parity status: pinned against the reference source compiled over the
 * project FFT shim (oracle/_ref/, recipe oracle/Makefile); the FFT itself is
 * pinned against numpy.fft (tests/test_oracle.py). The reference ships no
 * golden vectors of its own.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../include/pfc_b200.h"
#include "fft64.h"

#define ORACLE_PI 3.14159265358979323846264338327

typedef struct pfco {
	pfcg_params p;
	int Nx, Ny, H, U;
	double dx, dy;
	int t;
	int emulate_nu2;
	int scheme;                /* 0 ETD1 (the reference), 1 semi-implicit (pfco_set_scheme) */
	double* m[PFCG_MAX_U];     /* real fields, Ny x Nx */
	fft64_cplx* N[PFCG_MAX_U]; /* spectral state / (Nx Ny), H x Ny transposed */
	fft64_cplx* M[PFCG_MAX_U]; /* work spectra */
	double* A[PFCG_MAX_U];
	double* B[PFCG_MAX_U];
} pfco;

static size_t npts(const pfco* o) { return (size_t)o->Nx * (size_t)o->Ny; }
static size_t nspec(const pfco* o) { return (size_t)o->H * (size_t)o->Ny; }

/* squared wave number of half-spectrum entry (i = kx index, j = ky index), :1005-1006, :1055-1057 */
static double k2_of(const pfco* o, int i, int j, double dx, double dy) {
	const double dkx = 2.0 * ORACLE_PI / (dx * o->Nx);
	const double dky = 2.0 * ORACLE_PI / (dy * o->Ny);
	double kx = i * dkx;
	double ky = (j < o->Ny / 2) ? j * dky : (j - o->Ny) * dky;
	return kx * kx + ky * ky;
}

/* multi-mode operator P_u(k) = prod_w (omega (nu2 - k2)^2 + phi), :943-947 */
static double P_of(const pfcg_params* p, int u, double k2) {
	double P = 1.0;
	for (int w = 0; w < p->W[u]; w++) {
		double q = p->nu2[u][w] - k2;
		P *= p->omega[u][w] * q * q + p->phi[u][w];
	}
	return P;
}

/* update_AB, :901-958 */
static void update_AB(pfco* o) {
	const pfcg_params* p = &o->p;
	const double inv = 1.0 / o->Nx / o->Ny;
	const double c = (p->c != 0.0) ? 1.0 : 0.0;
#pragma omp parallel for schedule(static)
	for (int i = 0; i < o->H; i++) {
		for (int j = 0; j < o->Ny; j++) {
			const double k2 = k2_of(o, i, j, o->dx, o->dy);
			const size_t ij = (size_t)o->Ny * i + j;
			for (int u = 0; u < o->U; u++) {
				const double a = p->alpha[u][u] + p->beta[u][u] * P_of(p, u, k2);
				const double om = c - 1.0 - c * k2;
				if (o->scheme == 1) {
					/* semi-implicit: (N + dt o M) / (1 - dt o a), no counterpart in the reference */
					const double den = 1.0 - om * a * p->dt;
					o->A[u][ij] = 1.0 / den;
					o->B[u][ij] = om * p->dt / den * inv;
					continue;
				}
				const double ex = exp(om * a * p->dt);
				o->A[u][ij] = ex;
				o->B[u][ij] = ((a == 0.0) ? om * p->dt : (ex - 1.0) / a) * inv;
			}
		}
	}
}

static void forward_all(pfco* o, double* const* re, fft64_cplx* const* sp, int scale) {
	const double inv = 1.0 / o->Nx / o->Ny;
	for (int u = 0; u < o->U; u++) {
		fft64_r2c_2d_tr(o->Ny, o->Nx, re[u], o->Nx, sp[u]);
		if (scale)
			for (size_t k = 0; k < nspec(o); k++) sp[u][k] *= inv;
	}
}

pfco* pfco_create(const pfcg_params* p, int Nx, int Ny, double dx, double dy) {
	if (!p || p->U < 1 || p->U > PFCG_MAX_U || Nx < 2 || Ny < 2) return NULL;
	pfco* o = (pfco*)calloc(1, sizeof(*o));
	o->p = *p;
	o->U = p->U;
	o->Nx = Nx;
	o->Ny = Ny;
	o->H = Nx / 2 + 1;
	o->dx = dx;
	o->dy = dy;
	fft64_prepare_2d(Ny, Nx);
	for (int u = 0; u < o->U; u++) {
		o->m[u] = (double*)calloc(npts(o), sizeof(double));
		o->N[u] = (fft64_cplx*)calloc(nspec(o), sizeof(fft64_cplx));
		o->M[u] = (fft64_cplx*)calloc(nspec(o), sizeof(fft64_cplx));
		o->A[u] = (double*)calloc(nspec(o), sizeof(double));
		o->B[u] = (double*)calloc(nspec(o), sizeof(double));
	}
	update_AB(o);
	return o;
}

void pfco_destroy(pfco* o) {
	if (!o) return;
	for (int u = 0; u < o->U; u++) {
		free(o->m[u]); free(o->N[u]); free(o->M[u]); free(o->A[u]); free(o->B[u]);
	}
	free(o);
}

void pfco_set_emulate_nu2(pfco* o, int on) { o->emulate_nu2 = on; }

/* Time integrator: 0 = ETD1 (update_AB, :947-953), 1 = the semi-implicit update
 * N' = (N + dt o M) / (1 - dt o a) (o = c - 1 - c k^2), which the reference does
 * not have; the restatement of the formula lives in update_AB above. */
void pfco_set_scheme(pfco* o, int scheme) {
	o->scheme = scheme;
	update_AB(o);
}

void pfco_upload(pfco* o, const double* fields) {
	for (int u = 0; u < o->U; u++) memcpy(o->m[u], fields + (size_t)u * npts(o), npts(o) * sizeof(double));
	o->t = 0;
}

void pfco_download(const pfco* o, double* fields) {
	for (int u = 0; u < o->U; u++) memcpy(fields + (size_t)u * npts(o), o->m[u], npts(o) * sizeof(double));
}

/* spectral state as interleaved (re, im), U x H x Ny */
void pfco_spectrum(const pfco* o, double* out) {
	for (int u = 0; u < o->U; u++) memcpy(out + 2 * (size_t)u * nspec(o), o->N[u], nspec(o) * sizeof(fft64_cplx));
}

void pfco_set_box(pfco* o, double dx, double dy) {
	o->dx = dx;
	o->dy = dy;
	update_AB(o);
}
void pfco_get_box(const pfco* o, double* dx, double* dy) { *dx = o->dx; *dy = o->dy; }
void pfco_set_time(pfco* o, int t) { o->t = t; }
int pfco_get_time(const pfco* o) { return o->t; }

/* step, :1134-1248 */
static int step1(pfco* o) {
	const pfcg_params* p = &o->p;
	const int U = o->U;
	if (o->m[0][0] != o->m[0][0]) return PFCG_NAN; /* :1176 */
	if (o->t % 100 == 0) forward_all(o, o->m, o->N, 1); /* :1179-1185 */

	/* nonlinear part in real space, in place, :1188-1209 */
	const size_t n = npts(o);
#pragma omp parallel for schedule(static)
	for (size_t ij = 0; ij < n; ij++) {
		double mc[PFCG_MAX_U] = {0};
		for (int u = 0; u < U - 1; u++)
			for (int v = u + 1; v < U; v++) {
				const double mu = o->m[u][ij], mv = o->m[v][ij];
				mc[u] += p->alpha[u][v] * mv + 0.5 * p->gamma[u][v] * (2.0 * mu * mv + mv * mv);
				mc[v] += p->alpha[u][v] * mu + 0.5 * p->gamma[u][v] * (2.0 * mv * mu + mu * mu);
			}
		for (int u = 0; u < U; u++) {
			const double mu = o->m[u][ij];
			const double m2 = mu * mu;
			o->m[u][ij] = p->lambda[u] + p->gamma[u][u] * m2 + p->delta[u] * mu * m2 + mc[u];
		}
	}
	forward_all(o, o->m, o->M, 0); /* :1212 */

	/* k-space coupling and ETD1 update, :1215-1244 */
	const double NxNy = (double)o->Nx * o->Ny;
	const double a = -0.5 / p->sigma / p->sigma;
#pragma omp parallel for schedule(static)
	for (int i = 0; i < o->H; i++) {
		for (int j = 0; j < o->Ny; j++) {
			const size_t ij = (size_t)o->Ny * i + j;
			const double k2 = k2_of(o, i, j, o->dx, o->dy);
			double G2 = exp(a * k2);
			G2 *= G2;
			for (int u = 0; u < U - 1; u++)
				for (int v = u + 1; v < U; v++) {
					double d2 = p->mu2[u][v] - k2;
					d2 *= d2;
					o->M[u][ij] += (p->beta[u][v] * d2 * o->N[v][ij] + p->epsilon[u][v] * G2 * o->N[v][ij]) * NxNy;
					o->M[v][ij] += (p->beta[u][v] * d2 * o->N[u][ij] + p->epsilon[u][v] * G2 * o->N[u][ij]) * NxNy;
				}
			for (int u = 0; u < U; u++) {
				o->N[u][ij] = o->A[u][ij] * o->N[u][ij] + o->B[u][ij] * o->M[u][ij];
				o->M[u][ij] = o->N[u][ij];
			}
		}
	}
	for (int u = 0; u < U; u++) fft64_c2r_2d_tr(o->Ny, o->Nx, o->M[u], o->m[u], o->Nx); /* :1246 */
	o->t++;
	return 0;
}

int pfco_step(pfco* o, int nsteps) {
	for (int s = 0; s < nsteps; s++) {
		int rc = step1(o);
		if (rc) return rc;
	}
	return 0;
}

/* evaluate, :988-1131. f may be NULL. */
void pfco_evaluate(pfco* o, double* fave_out, double* nave_out, double* f_out) {
	const pfcg_params* p = &o->p;
	const int U = o->U;
	const size_t n = npts(o), ns = nspec(o);
	/* N = FFT(m) / (Nx Ny): the reference computes this into M (:1042-1047) and
	 * restores the same value into N at the end (:1125-1130) */
	forward_all(o, o->m, o->N, 1);

	fft64_cplx* PS[PFCG_MAX_U];
	fft64_cplx* ES[PFCG_MAX_U];
	fft64_cplx* QS[PFCG_MAX_U][PFCG_MAX_U] = {{0}};
	double* pn[PFCG_MAX_U];
	double* eta[PFCG_MAX_U];
	double* q[PFCG_MAX_U][PFCG_MAX_U] = {{0}};
	for (int u = 0; u < U; u++) {
		PS[u] = (fft64_cplx*)malloc(ns * sizeof(fft64_cplx));
		ES[u] = (fft64_cplx*)malloc(ns * sizeof(fft64_cplx));
		pn[u] = (double*)malloc(n * sizeof(double));
		eta[u] = (double*)malloc(n * sizeof(double));
		for (int v = u + 1; v < U; v++) {
			QS[u][v] = (fft64_cplx*)malloc(ns * sizeof(fft64_cplx));
			q[u][v] = (double*)malloc(n * sizeof(double));
		}
	}
	/* nonlocal parts in Fourier space, :1049-1079 */
	const double a = -0.5 / p->sigma / p->sigma;
#pragma omp parallel for schedule(static)
	for (int i = 0; i < o->H; i++) {
		for (int j = 0; j < o->Ny; j++) {
			const size_t ij = (size_t)o->Ny * i + j;
			const double k2 = k2_of(o, i, j, o->dx, o->dy);
			const double G = exp(a * k2);
			for (int u = 0; u < U; u++) {
				ES[u][ij] = G * o->N[u][ij];
				for (int v = u + 1; v < U; v++) {
					const double mu2 = o->emulate_nu2 ? p->nu2[u][v] : p->mu2[u][v];
					const double d = mu2 - k2;
					QS[u][v][ij] = d * d * o->N[v][ij];
				}
				PS[u][ij] = P_of(p, u, k2) * o->N[u][ij];
			}
		}
	}
	/* back to real space, :1081-1088 */
	for (int u = 0; u < U; u++) {
		fft64_c2r_2d_tr(o->Ny, o->Nx, PS[u], pn[u], o->Nx);
		fft64_c2r_2d_tr(o->Ny, o->Nx, ES[u], eta[u], o->Nx);
		for (int v = u + 1; v < U; v++) fft64_c2r_2d_tr(o->Ny, o->Nx, QS[u][v], q[u][v], o->Nx);
	}
	/* energy density and sums, serial to keep the reference's summation order, :1091-1118 */
	double fave = 0.0;
	double nave[PFCG_MAX_U] = {0};
	const double third = 1.0 / 3.0;
	for (size_t ij = 0; ij < n; ij++) {
		double f = 0.0;
		for (int u = 0; u < U; u++) {
			const double nu = o->m[u][ij];
			const double nunu = nu * nu;
			f += p->lambda[u] * nu + 0.5 * p->alpha[u][u] * nunu + 0.5 * p->beta[u][u] * nu * pn[u][ij] +
			     third * p->gamma[u][u] * nu * nunu + 0.25 * p->delta[u] * nunu * nunu;
			for (int v = u + 1; v < U; v++) {
				const double nv = o->m[v][ij];
				const double nvnv = nv * nv;
				f += p->alpha[u][v] * nu * nv + p->beta[u][v] * nu * q[u][v][ij] +
				     0.5 * p->gamma[u][v] * (nunu * nv + nu * nvnv) + p->epsilon[u][v] * eta[u][ij] * eta[v][ij];
			}
			nave[u] += nu;
		}
		if (f_out) f_out[ij] = f;
		fave += f;
	}
	const double inv = 1.0 / o->Nx / o->Ny;
	if (fave_out) *fave_out = fave * inv;
	for (int u = 0; u < U; u++)
		if (nave_out) nave_out[u] = nave[u] * inv;
	for (int u = 0; u < U; u++) {
		free(PS[u]); free(ES[u]); free(pn[u]); free(eta[u]);
		for (int v = u + 1; v < U; v++) { free(QS[u][v]); free(q[u][v]); }
	}
}

/* optimize, :1251-1290 */
void pfco_optimize(pfco* o, int xopt, int yopt, double* d) {
	const double dx0 = o->dx, dy0 = o->dy;
	const double dxs[5] = {dx0, dx0 - *d, dx0 + *d, dx0, dx0};
	const double dys[5] = {dy0, dy0, dy0, dy0 - *d, dy0 + *d};
	double fs[5] = {0, 0, 0, 0, 0};
	for (int i = 0; i < 5; i++) {
		if (xopt == 0 && (i == 1 || i == 2)) continue;
		if (yopt == 0 && (i == 3 || i == 4)) continue;
		o->dx = dxs[i];
		o->dy = dys[i];
		pfco_evaluate(o, &fs[i], NULL, NULL);
	}
	if (xopt != 0) o->dx = (*d * (fs[1] - fs[2]) + 2.0 * dxs[0] * (-2.0 * fs[0] + fs[1] + fs[2])) / (2.0 * (fs[1] - 2.0 * fs[0] + fs[2]));
	if (yopt != 0) o->dy = (*d * (fs[3] - fs[4]) + 2.0 * dys[0] * (-2.0 * fs[0] + fs[3] + fs[4])) / (2.0 * (fs[3] - 2.0 * fs[0] + fs[4]));
	const double l0 = 4.0 * ORACLE_PI / sqrt(3.0);
	const double dw = o->Nx * (o->dx - dxs[0]);
	const double dh = o->Ny * (o->dy - dys[0]);
	const double dr = sqrt(dw * dw + dh * dh);
	double x = 0.25 * l0;
	if (dr > x) {
		x /= dr;
		o->dx = x * o->dx + (1.0 - x) * dxs[0];
		o->dy = x * o->dy + (1.0 - x) * dys[0];
	}
	update_AB(o);
	const double ddx = o->dx - dxs[0], ddy = o->dy - dys[0];
	const double ddr = sqrt(ddx * ddx + ddy * ddy);
	if (ddr < *d) *d *= 0.5;
	else *d *= 2.0;
	if (*d < 1.0e-6) *d *= 2.0;
}
