/*
 * ORACLE — test infrastructure, not product code.
 *
 * FP64 restatement of the acoustic modelling and adjoint-gradient path that hpcscan_b200
 * adds on top of the reference's propagator. Used only by tests/ as the checker.
 *
 * Forward step (the reference's computePressureWithFD, src/grid.cpp:4612-5113, with a
 * damping factor G of the absorbing sponge and an additive point source):
 *     p[n+1] = G (2 p[n] + C Lap p[n] + amp s[n] e_src) - G^2 p[n-1]
 * on the INNER points, halos held at zero; C = (v dt)^2 per point; data d[n] = p[n](receivers)
 * for n = 1..nt; p[0] = p[-1] = 0.
 *
 * Adjoint, in the variable w = C G lambda (lambda the Lagrange multipliers of the steps), for
 * k = nt..1 with w[nt+1] = w[nt+2] = 0:
 *     w[k] = G (2 w[k+1] + C Lap w[k+1] + C R^T r[k]) - G^2 w[k+2]
 * where r[k] = d[k] - dobs[k] at the receivers. With J = 1/2 sum_k |r[k]|^2 and the squared
 * slowness m = 1/v^2 (C = dt^2 / m):
 *     dJ/dm = -(C / dt^2) sum_{n=0}^{nt-1} w[n+1] Lap p[n].
 * The discrete Laplacian is symmetric on the INNER points with zero halos, which makes the
 * recursion above the exact transpose of the forward one.
 *
 * Parity unpinned by the reference: it has no adjoint. This restatement is checked in the
 * tests by a dot-product test of its own forward/adjoint pair and by central finite
 * differences of the misfit.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
	int64_t n1, n2, n3;
	int64_t s1, e1, s2, e2, s3, e3;
	int32_t dim;
	int32_t halo;
} oracle_layout;

int oracle_laplacian_f64(const oracle_layout* L, int order, const double* u, double* w,
		double inv2_1, double inv2_2, double inv2_3);

#define IDX(L, i1, i2, i3) ((i1) + (i2) * (L)->n1 + (i3) * (L)->n1 * (L)->n2)

static int64_t npoint(const oracle_layout* L) { return L->n1 * L->n2 * L->n3; }

/* out = G (2 cur + C Lap cur) - G^2 prev on INNER points (prev may alias out) */
static void step(const oracle_layout* L, int order, const double* C, const double* G,
		const double* cur, const double* prev, double* out, double* lap,
		double i1, double i2, double i3)
{
	oracle_laplacian_f64(L, order, cur, lap, i1, i2, i3);
#pragma omp parallel for collapse(2)
	for (int64_t z = L->s3; z <= L->e3; z++)
		for (int64_t y = L->s2; y <= L->e2; y++)
			for (int64_t x = L->s1; x <= L->e1; x++) {
				const int64_t ii = IDX(L, x, y, z);
				const double g = G[ii];
				out[ii] = g * (2.0 * cur[ii] + C[ii] * lap[ii]) - g * g * prev[ii];
			}
}

/* Forward modelling; traces[n * nrec + r] = p[n+1](rec[r]); snap (optional) holds
 * p[0..nt] as (nt + 1) x npoint. */
int oracle_model_forward_f64(const oracle_layout* L, int order, const double* C, const double* G,
		int64_t src, double amp, const double* wavelet, int nt, int nrec, const int64_t* rec,
		double inv2_1, double inv2_2, double inv2_3, double* traces, double* snap)
{
	const int64_t np = npoint(L);
	double* a = calloc(np, sizeof(double));   /* p[n-1], then p[n+1] */
	double* b = calloc(np, sizeof(double));   /* p[n] */
	double* lap = calloc(np, sizeof(double));
	if (!a || !b || !lap) return -1;
	if (snap) memset(snap, 0, sizeof(double) * np);
	for (int n = 0; n < nt; n++) {
		step(L, order, C, G, b, a, a, lap, inv2_1, inv2_2, inv2_3);
		a[src] += G[src] * amp * wavelet[n];
		for (int r = 0; r < nrec; r++) traces[(int64_t)n * nrec + r] = a[rec[r]];
		if (snap) memcpy(snap + (int64_t)(n + 1) * np, a, sizeof(double) * np);
		double* t = a; a = b; b = t;
	}
	free(a); free(b); free(lap);
	return 0;
}

/* Adjoint driven by res (nt x nrec, row k-1 = r[k]); w_src[n] = w[n+1](src) for n = 0..nt-1;
 * grad (optional, needs snap = p[0..nt]) accumulates -(C/dt2) sum w[n+1] Lap p[n]. */
int oracle_model_adjoint_f64(const oracle_layout* L, int order, const double* C, const double* G,
		int nt, int nrec, const int64_t* rec, double inv2_1, double inv2_2, double inv2_3,
		const double* res, int64_t src, double* w_src, const double* snap, double dt2,
		double* grad)
{
	const int64_t np = npoint(L);
	double* w2 = calloc(np, sizeof(double));  /* w[k+2], then w[k] */
	double* w1 = calloc(np, sizeof(double));  /* w[k+1] */
	double* lap = calloc(np, sizeof(double));
	if (!w2 || !w1 || !lap) return -1;
	if (grad) memset(grad, 0, sizeof(double) * np);
	for (int k = nt; k >= 1; k--) {
		step(L, order, C, G, w1, w2, w2, lap, inv2_1, inv2_2, inv2_3);
		for (int r = 0; r < nrec; r++) {
			const int64_t ii = rec[r];
			w2[ii] += C[ii] * G[ii] * res[(int64_t)(k - 1) * nrec + r];
		}
		/* now w2 = w[k] */
		if (w_src) w_src[k - 1] = w2[src];
		if (grad) {
			oracle_laplacian_f64(L, order, snap + (int64_t)(k - 1) * np, lap, inv2_1, inv2_2, inv2_3);
#pragma omp parallel for collapse(2)
			for (int64_t z = L->s3; z <= L->e3; z++)
				for (int64_t y = L->s2; y <= L->e2; y++)
					for (int64_t x = L->s1; x <= L->e1; x++) {
						const int64_t ii = IDX(L, x, y, z);
						grad[ii] -= C[ii] / dt2 * w2[ii] * lap[ii];
					}
		}
		double* t = w2; w2 = w1; w1 = t;
	}
	free(w2); free(w1); free(lap);
	return 0;
}

/* Misfit and its gradient with respect to the squared slowness. */
int oracle_model_gradient_f64(const oracle_layout* L, int order, const double* C, const double* G,
		int64_t src, double amp, const double* wavelet, int nt, int nrec, const int64_t* rec,
		double inv2_1, double inv2_2, double inv2_3, const double* dobs, double dt2,
		double* grad, double* misfit)
{
	const int64_t np = npoint(L);
	double* snap = malloc(sizeof(double) * np * (nt + 1));
	double* tr = malloc(sizeof(double) * (size_t)nt * nrec);
	if (!snap || !tr) return -1;
	int rc = oracle_model_forward_f64(L, order, C, G, src, amp, wavelet, nt, nrec, rec, inv2_1,
			inv2_2, inv2_3, tr, snap);
	double J = 0.0;
	for (int64_t i = 0; i < (int64_t)nt * nrec; i++) {
		tr[i] -= dobs[i];
		J += 0.5 * tr[i] * tr[i];
	}
	if (!rc)
		rc = oracle_model_adjoint_f64(L, order, C, G, nt, nrec, rec, inv2_1, inv2_2, inv2_3, tr,
				src, NULL, snap, dt2, grad);
	*misfit = J;
	free(snap); free(tr);
	return rc;
}
