/*
 * ORACLE — test infrastructure, not product code.
 *
 * A plain-C restatement of the hpcscan CPU reference ("Baseline" test mode)
 * for the finite-difference / acoustic-propagator hot path. It is used only by
 * tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, and
 * only as the checker. The product (hpcscan_b200) never links or calls it.
 *
 * Parity is pinned: tests/test_oracle_golden.py compares every function here
 * with grids written by the reference itself (oracle/_ref/hpcscan_fp32|fp64,
 * built unchanged from the reference sources, -writeGrid), stored as fixtures
 * in tests/golden/. Compiled with the same arithmetic flags as those binaries
 * (-O3 -mavx2, no FP contraction), the elementwise kernels are bit-identical.
 *
 * Reference citations are to files of vetienne74/hpcscan:
 *   coefficients, association order  src/fdm.h:277-545 (D2), 27-275 (D1)
 *   FD_D1_N1/N2/N3                   src/grid.cpp:3401, 3735, 4069
 *   FD_D2_N1/N2/N3                   src/grid.cpp:3232, 3566, 3900
 *   FD_LAPLACIAN                     src/grid.cpp:4235-4576
 *   updatePressure                   src/grid.cpp:4579-4609
 *   computePressureWithFD            src/grid.cpp:4612-5113
 *   applyBoundaryCondition           src/grid.cpp:3065-3229
 *   fill (constant, separable)       src/grid.cpp:1650-1826
 *   maxErr, L1Err, getSumAbsDiff,
 *   getSumAbs, getMin, getMax        src/grid.cpp:2006-2336
 *
 * Layout (src/grid.cpp:15-38): a grid is a flat array, i1 fastest,
 * idx = i1 + i2*n1 + i3*n1*n2; the stencils run over the INNER box
 * [s1,e1]x[s2,e2]x[s3,e3] (inclusive bounds, as Grid::getGridIndex returns).
 */
#include <math.h>
#include <stdint.h>
#include <float.h>

typedef struct {
	int64_t n1, n2, n3;     /* full array dimensions */
	int64_t s1, e1, s2, e2, s3, e3; /* inner box, inclusive */
	int32_t dim;            /* 1, 2 or 3 */
	int32_t halo;           /* fdOrder / 2 */
} oracle_layout;

typedef struct {
	int64_t i1s, i1e, i2s, i2e, i3s, i3e; /* inclusive box */
} oracle_box;

/* FD_D2 centred coefficients A0..A8 per order, src/fdm.h:277-545. */
static const double D2COEF[9][9] = {
	{0},
	{-2.0, 1.0},                                                       /* O2  */
	{-5./2., 4./3., -1./12.},                                          /* O4  */
	{-49./18., 3./2., -3./20., 1./90.},                                /* O6  */
	{-205./72., 8./5., -1/5., 8./315., -1/560.},                       /* O8  */
	{-5269./1800., 5./3., -5./21., 5./126., -5./1008., 1./3150.},      /* O10 */
	{-5369./1800., 12./7., -15./56., 10./189., -1./112., 2./1925., -1./16632.}, /* O12 */
	{-266681./88200., 7./4., -7./24., 7./108., -7./528., 7./3300., -7./30888., 1./84084.}, /* O14 */
	{-1077749./352800., 16./9., -14./45., 112./1485., -7./396., 112./32175., -2./3861.,
	  16./315315., -1./411840.},                                       /* O16 */
};

/* FD_D1 staggered coefficients A1..A8 per order, src/fdm.h:34-234 (index 0 unused). */
static const double D1COEF[9][9] = {
	{0},
	{0, 1.0},                                                                    /* O2  */
	{0, 9./8., -1./24.},                                                         /* O4  */
	{0, 75./64., -25./384., 3./640.},                                            /* O6  */
	{0, 1225./1024., -245./3072., 49./5120., -5./7168.},                         /* O8  */
	{0, 19845./16384., -735./8192., 567./40960., -405./229376., 35./294912.},   /* O10 */
	{0, 160083./131072., -12705./131072., 22869./1310720., -5445./1835008.,
	  847./2359296., -63./2883584.},                                             /* O12 */
	{0, 1288287./1048576., -429429./4194304., 429429./20971520., -61347./14680064.,
	  13013./18874368., -3549./46137344., 231./54525952.},                       /* O14 */
	{0, 41409225./33554432., -3578575./33554432., 3864861./167772160.,
	  -1254825./234881024., 325325./301989888., -61425./369098752., 7425./436207616.,
	  -143./167772160.},                                                         /* O16 */
};

int oracle_valid_order(int order)
{
	return (order >= 2 && order <= 16 && (order % 2) == 0) ;
}

double oracle_d2_coef(int order, int k)
{
	if (!oracle_valid_order(order) || k < 0 || k > order / 2) return 0.0 ;
	return D2COEF[order / 2][k] ;
}

#define IDX(L, i1, i2, i3) ((i1) + (i2) * (L)->n1 + (i3) * (L)->n1 * (L)->n2)

/*
 * One template body per storage/compute type T (float: Myfloat = Myfloat2 =
 * float; double: the reference's -D_STORAGE_FP64_ -D_COMPUTE_FP64_ build).
 */
#define ORACLE_DEFINE(T, SUF, MAXERRF)                                                        \
                                                                                              \
/* second derivative along one axis at linear index ii with stride st,           */          \
/* association as the src/fdm.h macros: ((A0*u + A1*(u+1 + u-1)) + A2*(...)) ... */          \
/* O2 is written (A0*u + u+1) + u-1 without A1 (src/fdm.h:286-288)             */          \
static inline T d2_##SUF(const T* u, int64_t ii, int64_t st, const T* c, int r, T inv2)      \
{                                                                                             \
	T acc = c[0] * u[ii] ;                                                                    \
	if (r == 1) return ((acc + u[ii + st]) + u[ii - st]) * inv2 ;                             \
	for (int k = 1; k <= r; k++) acc = acc + c[k] * (u[ii + k * st] + u[ii - k * st]) ;      \
	return acc * inv2 ;                                                                       \
}                                                                                             \
                                                                                              \
static void coefs_##SUF(int order, T* c)                                                     \
{                                                                                             \
	for (int k = 0; k <= order / 2; k++) c[k] = (T) D2COEF[order / 2][k] ;                   \
}                                                                                             \
                                                                                              \
/* Grid::FD_D2_N1/N2/N3: w = d2u/dxa^2 on INNER points (src/grid.cpp:3232,3566,3900) */      \
int oracle_fd_d2_##SUF(const oracle_layout* L, int axis, int order, const T* u, T* w,        \
		T inv2_1, T inv2_2, T inv2_3)                                                         \
{                                                                                             \
	if (!oracle_valid_order(order) || axis < 1 || axis > 3) return -1 ;                      \
	T c[9] ; coefs_##SUF(order, c) ;                                                          \
	const int r = order / 2 ;                                                                 \
	const int64_t st = (axis == 1) ? 1 : (axis == 2) ? L->n1 : L->n1 * L->n2 ;              \
	const T inv2 = (axis == 1) ? inv2_1 : (axis == 2) ? inv2_2 : inv2_3 ;                    \
	_Pragma("omp parallel for collapse(2)")                                                   \
	for (int64_t i3 = L->s3; i3 <= L->e3; i3++)                                               \
		for (int64_t i2 = L->s2; i2 <= L->e2; i2++)                                           \
			for (int64_t i1 = L->s1; i1 <= L->e1; i1++) {                                     \
				const int64_t ii = IDX(L, i1, i2, i3) ;                                       \
				w[ii] = d2_##SUF(u, ii, st, c, r, inv2) ;                                     \
			}                                                                                 \
	return 0 ;                                                                                \
}                                                                                             \
                                                                                              \
/* Grid::FD_D1_N1/N2/N3 (src/grid.cpp:3401,3735,4069): staggered first derivative at    */ \
/* i - 1/2 on INNER points, ((A1 (u - u-1) + A2 (u+1 - u-2)) + ...) * inv_d; O2 has no A1 */ \
/* factor (src/fdm.h:37-44)                                                            */ \
int oracle_fd_d1_##SUF(const oracle_layout* L, int axis, int order, const T* u, T* w,        \
		T inv_1, T inv_2, T inv_3)                                                            \
{                                                                                             \
	if (!oracle_valid_order(order) || axis < 1 || axis > 3) return -1 ;                      \
	const int r = order / 2 ;                                                                 \
	T c[9] ;                                                                                  \
	for (int k = 1; k <= r; k++) c[k] = (T) D1COEF[r][k] ;                                   \
	const int64_t st = (axis == 1) ? 1 : (axis == 2) ? L->n1 : L->n1 * L->n2 ;              \
	const T inv = (axis == 1) ? inv_1 : (axis == 2) ? inv_2 : inv_3 ;                        \
	_Pragma("omp parallel for collapse(2)")                                                   \
	for (int64_t i3 = L->s3; i3 <= L->e3; i3++)                                               \
		for (int64_t i2 = L->s2; i2 <= L->e2; i2++)                                           \
			for (int64_t i1 = L->s1; i1 <= L->e1; i1++) {                                     \
				const int64_t ii = IDX(L, i1, i2, i3) ;                                       \
				if (r == 1) { w[ii] = (u[ii] - u[ii - st]) * inv ; continue ; }               \
				T acc = c[1] * (u[ii] - u[ii - st]) ;                                         \
				for (int k = 2; k <= r; k++)                                                  \
					acc = acc + c[k] * (u[ii + (k - 1) * st] - u[ii - k * st]) ;              \
				w[ii] = acc * inv ;                                                           \
			}                                                                                 \
	return 0 ;                                                                                \
}                                                                                             \
                                                                                              \
/* Grid::FD_LAPLACIAN (src/grid.cpp:4235-4576); 1D is FD_D2_N1 */                            \
int oracle_laplacian_##SUF(const oracle_layout* L, int order, const T* u, T* w,              \
		T inv2_1, T inv2_2, T inv2_3)                                                         \
{                                                                                             \
	if (!oracle_valid_order(order)) return -1 ;                                              \
	if (L->dim == 1) return oracle_fd_d2_##SUF(L, 1, order, u, w, inv2_1, inv2_2, inv2_3) ;   \
	T c[9] ; coefs_##SUF(order, c) ;                                                          \
	const int r = order / 2 ;                                                                 \
	const int64_t s2 = L->n1, s3 = L->n1 * L->n2 ;                                            \
	_Pragma("omp parallel for collapse(2)")                                                   \
	for (int64_t i3 = L->s3; i3 <= L->e3; i3++)                                               \
		for (int64_t i2 = L->s2; i2 <= L->e2; i2++)                                           \
			for (int64_t i1 = L->s1; i1 <= L->e1; i1++) {                                     \
				const int64_t ii = IDX(L, i1, i2, i3) ;                                       \
				if (L->dim == 2)                                                              \
					w[ii] = d2_##SUF(u, ii, 1, c, r, inv2_1) + d2_##SUF(u, ii, s2, c, r, inv2_2) ; \
				else                                                                          \
					w[ii] = d2_##SUF(u, ii, 1, c, r, inv2_1) + d2_##SUF(u, ii, s2, c, r, inv2_2) \
					      + d2_##SUF(u, ii, s3, c, r, inv2_3) ;                                 \
			}                                                                                 \
	return 0 ;                                                                                \
}                                                                                             \
                                                                                              \
/* Grid::updatePressure: prn = 2 prc - prn + coef lapla on INNER (src/grid.cpp:4579) */      \
int oracle_update_pressure_##SUF(const oracle_layout* L, T* prn, const T* prc,              \
		const T* coef, const T* lapla)                                                        \
{                                                                                             \
	const T two = (T) 2.0 ;                                                                   \
	_Pragma("omp parallel for collapse(2)")                                                   \
	for (int64_t i3 = L->s3; i3 <= L->e3; i3++)                                               \
		for (int64_t i2 = L->s2; i2 <= L->e2; i2++)                                           \
			for (int64_t i1 = L->s1; i1 <= L->e1; i1++) {                                     \
				const int64_t ii = IDX(L, i1, i2, i3) ;                                       \
				prn[ii] = two * prc[ii] - prn[ii] + coef[ii] * lapla[ii] ;                    \
			}                                                                                 \
	return 0 ;                                                                                \
}                                                                                             \
                                                                                              \
/* Grid::computePressureWithFD (src/grid.cpp:4612-5113):                          */          \
/* prn = 2 prc - prn + coef * (D2_N1 + D2_N2 + D2_N3)(prc) on INNER                */          \
int oracle_compute_pressure_##SUF(const oracle_layout* L, int order, T* prn, const T* prc,  \
		const T* coef, T inv2_1, T inv2_2, T inv2_3)                                          \
{                                                                                             \
	if (!oracle_valid_order(order)) return -1 ;                                              \
	T c[9] ; coefs_##SUF(order, c) ;                                                          \
	const int r = order / 2 ;                                                                 \
	const T two = (T) 2.0 ;                                                                   \
	const int64_t s2 = L->n1, s3 = L->n1 * L->n2 ;                                            \
	_Pragma("omp parallel for collapse(2)")                                                   \
	for (int64_t i3 = L->s3; i3 <= L->e3; i3++)                                               \
		for (int64_t i2 = L->s2; i2 <= L->e2; i2++)                                           \
			for (int64_t i1 = L->s1; i1 <= L->e1; i1++) {                                     \
				const int64_t ii = IDX(L, i1, i2, i3) ;                                       \
				T lap ;                                                                       \
				if (L->dim == 1) lap = d2_##SUF(prc, ii, 1, c, r, inv2_1) ;                   \
				else if (L->dim == 2) lap = d2_##SUF(prc, ii, 1, c, r, inv2_1)                \
					+ d2_##SUF(prc, ii, s2, c, r, inv2_2) ;                                   \
				else lap = d2_##SUF(prc, ii, 1, c, r, inv2_1)                                 \
					+ d2_##SUF(prc, ii, s2, c, r, inv2_2) + d2_##SUF(prc, ii, s3, c, r, inv2_3) ; \
				prn[ii] = two * prc[ii] - prn[ii] + coef[ii] * lap ;                          \
			}                                                                                 \
	return 0 ;                                                                                \
}                                                                                             \
                                                                                              \
/* Grid::applyBoundaryCondition(BOUND_COND_ANTI_MIRROR) (src/grid.cpp:3065-3229).  */         \
/* Faces in the reference order I1HALO1, I1HALO2, I2HALO1, I2HALO2, I3HALO1,        */         \
/* I3HALO2; each face: boundary plane = 0, halo[k] = -inner[mirror k], over the     */         \
/* other axes' INNER ranges. Single rank: every face has no neighbour.             */         \
int oracle_apply_bc_##SUF(const oracle_layout* L, T* u)                                       \
{                                                                                             \
	const int r = L->halo ;                                                                   \
	const int64_t n1 = L->n1, n12 = L->n1 * L->n2 ;                                           \
	if (L->dim >= 1) {                                                                        \
		for (int64_t i3 = L->s3; i3 <= L->e3; i3++)                                           \
			for (int64_t i2 = L->s2; i2 <= L->e2; i2++) {                                     \
				const int64_t b = L->s1, o = i2 * n1 + i3 * n12 ;                             \
				u[b + o] = 0.0 ;                                                              \
				for (int k = 1; k <= r; k++) u[b - k + o] = -u[b + k + o] ;                   \
			}                                                                                 \
		for (int64_t i3 = L->s3; i3 <= L->e3; i3++)                                           \
			for (int64_t i2 = L->s2; i2 <= L->e2; i2++) {                                     \
				const int64_t b = L->e1, o = i2 * n1 + i3 * n12 ;                             \
				u[b + o] = 0.0 ;                                                              \
				for (int k = 1; k <= r; k++) u[b + k + o] = -u[b - k + o] ;                   \
			}                                                                                 \
	}                                                                                         \
	if (L->dim >= 2) {                                                                        \
		for (int64_t i3 = L->s3; i3 <= L->e3; i3++)                                           \
			for (int64_t i1 = L->s1; i1 <= L->e1; i1++) {                                     \
				const int64_t b = L->s2, o = i1 + i3 * n12 ;                                  \
				u[o + b * n1] = 0.0 ;                                                         \
				for (int k = 1; k <= r; k++) u[o + (b - k) * n1] = -u[o + (b + k) * n1] ;     \
			}                                                                                 \
		for (int64_t i3 = L->s3; i3 <= L->e3; i3++)                                           \
			for (int64_t i1 = L->s1; i1 <= L->e1; i1++) {                                     \
				const int64_t b = L->e2, o = i1 + i3 * n12 ;                                  \
				u[o + b * n1] = 0.0 ;                                                         \
				for (int k = 1; k <= r; k++) u[o + (b + k) * n1] = -u[o + (b - k) * n1] ;     \
			}                                                                                 \
	}                                                                                         \
	if (L->dim >= 3) {                                                                        \
		for (int64_t i2 = L->s2; i2 <= L->e2; i2++)                                           \
			for (int64_t i1 = L->s1; i1 <= L->e1; i1++) {                                     \
				const int64_t b = L->s3, o = i1 + i2 * n1 ;                                   \
				u[o + b * n12] = 0.0 ;                                                        \
				for (int k = 1; k <= r; k++) u[o + (b - k) * n12] = -u[o + (b + k) * n12] ;   \
			}                                                                                 \
		for (int64_t i2 = L->s2; i2 <= L->e2; i2++)                                           \
			for (int64_t i1 = L->s1; i1 <= L->e1; i1++) {                                     \
				const int64_t b = L->e3, o = i1 + i2 * n1 ;                                   \
				u[o + b * n12] = 0.0 ;                                                        \
				for (int k = 1; k <= r; k++) u[o + (b + k) * n12] = -u[o + (b - k) * n12] ;   \
			}                                                                                 \
	}                                                                                         \
	return 0 ;                                                                                \
}                                                                                             \
                                                                                              \
/* Grid::fill(pointType, val) (src/grid.cpp:1808) */                                          \
int oracle_fill_const_##SUF(const oracle_layout* L, T* u, const oracle_box* B, double val)    \
{                                                                                             \
	const T v = (T) val ;                                                                     \
	for (int64_t i3 = B->i3s; i3 <= B->i3e; i3++)                                             \
		for (int64_t i2 = B->i2s; i2 <= B->i2e; i2++)                                         \
			for (int64_t i1 = B->i1s; i1 <= B->i1e; i1++) u[IDX(L, i1, i2, i3)] = v ;       \
	return 0 ;                                                                                \
}                                                                                             \
                                                                                              \
/* Grid::fill(pType, f1, f2, f3, p1, p2, p3, amp) (src/grid.cpp:1650-1805): the      */        \
/* caller supplies the FP64 1-D tables; value = (T)(amp * v1[i1] * v2[i2] * v3[i3]) */        \
int oracle_fill_sep_##SUF(const oracle_layout* L, T* u, const oracle_box* B,                  \
		const double* v1, const double* v2, const double* v3, double amp)                     \
{                                                                                             \
	for (int64_t i3 = B->i3s; i3 <= B->i3e; i3++)                                             \
		for (int64_t i2 = B->i2s; i2 <= B->i2e; i2++)                                         \
			for (int64_t i1 = B->i1s; i1 <= B->i1e; i1++)                                     \
				u[IDX(L, i1, i2, i3)] = (T) (amp * v1[i1 - B->i1s] * v2[i2 - B->i2s]           \
						* v3[i3 - B->i3s]) ;                                                  \
	return 0 ;                                                                                \
}                                                                                             \
                                                                                              \
/* Grid::getSumAbs: sum |u| in FP64 (src/grid.cpp:2230) */                                   \
double oracle_sum_abs_##SUF(const oracle_layout* L, const T* u, const oracle_box* B)          \
{                                                                                             \
	double s = 0.0 ;                                                                          \
	for (int64_t i3 = B->i3s; i3 <= B->i3e; i3++)                                             \
		for (int64_t i2 = B->i2s; i2 <= B->i2e; i2++)                                         \
			for (int64_t i1 = B->i1s; i1 <= B->i1e; i1++) s += fabs((double) u[IDX(L, i1, i2, i3)]) ; \
	return s ;                                                                                \
}                                                                                             \
                                                                                              \
/* Grid::getSumAbsDiff: sum |u1 - u2| in FP64 (src/grid.cpp:2180) */                         \
double oracle_sum_abs_diff_##SUF(const oracle_layout* L, const T* u1, const T* u2,            \
		const oracle_box* B)                                                                  \
{                                                                                             \
	double s = 0.0 ;                                                                          \
	for (int64_t i3 = B->i3s; i3 <= B->i3e; i3++)                                             \
		for (int64_t i2 = B->i2s; i2 <= B->i2e; i2++)                                         \
			for (int64_t i1 = B->i1s; i1 <= B->i1e; i1++) {                                   \
				const int64_t ii = IDX(L, i1, i2, i3) ;                                       \
				s += fabs((double) u1[ii] - u2[ii]) ;                                         \
			}                                                                                 \
	return s ;                                                                                \
}                                                                                             \
                                                                                              \
/* Grid::maxErr (src/grid.cpp:2006-2055): pointwise relative error, absolute where */         \
/* |u2| < MAX_ERR_FLOAT (src/constant.h:14-20)                                      */         \
double oracle_max_err_##SUF(const oracle_layout* L, const T* u1, const T* u2,                 \
		const oracle_box* B)                                                                  \
{                                                                                             \
	double err = -FLT_MAX ;                                                                   \
	for (int64_t i3 = B->i3s; i3 <= B->i3e; i3++)                                             \
		for (int64_t i2 = B->i2s; i2 <= B->i2e; i2++)                                         \
			for (int64_t i1 = B->i1s; i1 <= B->i1e; i1++) {                                   \
				const int64_t ii = IDX(L, i1, i2, i3) ;                                       \
				double e ;                                                                    \
				if (fabsf((float) u2[ii]) < (float) (MAXERRF))                               \
					e = fabs((double) u1[ii] - u2[ii]) ;                                      \
				else e = fabs((double) u1[ii] - u2[ii]) / fabs((double) u2[ii]) ;             \
				if (e > err) err = e ;                                                        \
			}                                                                                 \
	return err ;                                                                              \
}                                                                                             \
                                                                                              \
/* Grid::getMin / getMax (src/grid.cpp:2276-2336) */                                          \
void oracle_min_max_##SUF(const oracle_layout* L, const T* u, const oracle_box* B,            \
		double* mn, double* mx)                                                               \
{                                                                                             \
	T lo = FLT_MAX, hi = -FLT_MAX ;                                                           \
	for (int64_t i3 = B->i3s; i3 <= B->i3e; i3++)                                             \
		for (int64_t i2 = B->i2s; i2 <= B->i2e; i2++)                                         \
			for (int64_t i1 = B->i1s; i1 <= B->i1e; i1++) {                                   \
				const T v = u[IDX(L, i1, i2, i3)] ;                                           \
				if (v < lo) lo = v ;                                                          \
				if (v > hi) hi = v ;                                                          \
			}                                                                                 \
	*mn = lo ; *mx = hi ;                                                                     \
}

ORACLE_DEFINE(float, f32, 1.e-5)
ORACLE_DEFINE(double, f64, 1.e-11)
