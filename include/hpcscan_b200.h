/*
 * hpcscan_b200 — C ABI of the B200 (sm_100a) implementation of the hpcscan
 * finite-difference / acoustic-propagator hot path.
 *
 * This is the boundary a hpcscan test mode binds to: the C++ class Grid_B200
 * (hpcscan_b200/host/grid_B200.cpp) subclasses the reference's Grid and
 * forwards each virtual listed below to one of these entry points; any other
 * host (Python ctypes, another C++ driver) can bind the same symbols.
 *
 * Conventions
 *  - Plain pointers and sizes only. Device pointers come from b200_malloc (or
 *    any cudaMalloc'd memory of the current device).
 *  - Every entry point returns an int status: B200_OK (0) or a negative code;
 *    b200_last_error() returns a message for the calling thread. Nothing here
 *    exits the process.
 *  - `stream` is a cudaStream_t passed as void* (NULL = the legacy default
 *    stream). Kernels are enqueued on it; entry points that return host
 *    scalars (the reductions) synchronise that stream.
 *  - A grid is one flat array, i1 fastest: idx = i1 + i2*n1 + i3*n1*n2, with
 *    the INNER box [s1,e1]x[s2,e2]x[s3,e3] (inclusive bounds) exactly as
 *    Grid::getGridIndex(INNER_POINTS) returns it (reference src/grid.cpp:15-38,
 *    2682-2843). For 1D and 2D grids the unused axes have n = 1 and s = e = 0.
 *  - Arithmetic: FP32 storage computes in FP32 and FP64 in FP64, as the
 *    reference's Myfloat/Myfloat2 builds do (src/type_def.h:22-44); FP16 and
 *    BF16 storage compute in FP32. Norms accumulate in FP64.
 *  - Field scale: a stored value s of a field with scale k stands for the
 *    physical value s*k (a power of two for 16-bit storage, 1.0 otherwise).
 */
#ifndef HPCSCAN_B200_H_
#define HPCSCAN_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------- */
#define B200_OK               0
#define B200_ERR_ARG         -1   /* invalid argument (size mismatch, bad order, bad box ...) */
#define B200_ERR_CUDA        -2   /* a CUDA runtime/driver call failed                        */
#define B200_ERR_UNSUPPORTED -3   /* valid but not supported (e.g. dtype for this operator)   */
#define B200_ERR_TIMEOUT     -4   /* a bounded device-side wait ran out                       */
#define B200_ERR_NOMEM       -5   /* device allocation failed                                 */

/* ---- storage types ------------------------------------------------------------------------ */
#define B200_F32  0
#define B200_F64  1
#define B200_F16  2
#define B200_BF16 3

/* ---- boundary conditions (reference src/type_def.h:99) ------------------------------------ */
#define B200_NO_BOUND_COND          0
#define B200_BOUND_COND_ANTI_MIRROR 1

/* Array layout of one grid: full dims and the INNER box (inclusive), dim, halo = order/2. */
typedef struct b200_layout {
	int64_t n1, n2, n3;
	int64_t s1, e1, s2, e2, s3, e3;
	int32_t dim;
	int32_t halo;
} b200_layout;

/* An index box, inclusive bounds (what Grid::getGridIndex returns for a point type). */
typedef struct b200_box {
	int64_t i1s, i1e, i2s, i2e, i3s, i3e;
} b200_box;

/* A field in device memory. */
typedef struct b200_field {
	void*   data;   /* device pointer, n1*n2*n3 elements                        */
	int32_t dtype;  /* B200_F32 / B200_F64 / B200_F16 / B200_BF16               */
	float   scale;  /* physical value = stored value * scale                    */
} b200_field;

/* ---- runtime -------------------------------------------------------------------------------
 * b200_init: select the device (reference: cudaSetDevice(rank % deviceCount) in
 * Grid_Cuda::initializeGrid, src/grid_Cuda.cu:2757-2762) and prepare the per-device state. */
int         b200_init(int device);
const char* b200_last_error(void);
int         b200_device_count(int* count);
int         b200_malloc(void** dptr, size_t bytes);
int         b200_free(void* dptr);
int         b200_memcpy_h2d(void* dst, const void* src, size_t bytes, void* stream);
int         b200_memcpy_d2h(void* dst, const void* src, size_t bytes, void* stream);
int         b200_memcpy_d2d(void* dst, const void* src, size_t bytes, void* stream);
int         b200_memset(void* dptr, int value, size_t bytes, void* stream);
int         b200_stream_sync(void* stream);
/* Copy one box of a grid between host and device (the rest untouched); replaces the
 * host<->device staging of Grid_Cuda::copyGridDeviceToHost/HostToDevice
 * (src/grid_Cuda.cu:3410-3470). elem_size = bytes per element. */
int         b200_copy_box_d2h(const b200_layout* lay, int elem_size, void* host, const void* dev,
		const b200_box* box, void* stream);
int         b200_copy_box_h2d(const b200_layout* lay, int elem_size, void* dev, const void* host,
		const b200_box* box, void* stream);

/* ---- fills ---------------------------------------------------------------------------------
 * Grid::fill(pointType, val) (src/grid.cpp:1802-1824). */
int b200_fill_const(const b200_layout* lay, b200_field u, const b200_box* box, double val,
		void* stream);

/* Grid::fill(pType, f1, f2, f3, p1, p2, p3, amp) (src/grid.cpp:1650-1805): the caller
 * supplies the three FP64 1-D tables v1[i1-i1s], v2[i2-i2s], v3[i3-i3s] (host memory);
 * u = (stored type)(amp * v1 * v2 * v3 / u.scale) over the box. */
int b200_fill_separable(const b200_layout* lay, b200_field u, const b200_box* box,
		const double* v1, const double* v2, const double* v3, double amp, void* stream);

/* Whole-array operations over n elements (every point, halos and padding included), the
 * Memory test case's Grid::fillArray, copyArray, addArray, multiplyArray and addUpdateArray
 * (src/grid.cpp:1828-1918), in the storage type's arithmetic. in2 is read by ADD and MUL
 * only, in1 by all but FILL; fields must have scale 1 (FILL excepted). */
#define B200_ARRAY_FILL       0   /* out = val        */
#define B200_ARRAY_COPY       1   /* out = in1        */
#define B200_ARRAY_ADD        2   /* out = in1 + in2  */
#define B200_ARRAY_MUL        3   /* out = in1 * in2  */
#define B200_ARRAY_ADD_UPDATE 4   /* out = out + in1  */
int b200_array_op(int op, int64_t n, b200_field out, b200_field in1, b200_field in2, double val,
		void* stream);

/* Receivers and sources of DataAcquisition (src/data_Acquisition.cpp:286-351):
 * out[i * stride] = u[idx[i]] for i < n (idx and out in device memory, out in u's storage type);
 * u[idx] = value (rounded to u's storage, divided by its scale). */
int b200_gather_points(b200_field u, const int64_t* idx, int64_t n, void* out, int64_t stride,
		void* stream);
int b200_set_point(b200_field u, int64_t idx, double value, void* stream);

/* ---- finite-difference operators (INNER points; `u` in, `w` out) ----------------------------
 * inv2_a = (1/d_a)^2 evaluated in the compute type by the caller (src/grid.cpp:3252-3258).
 * Grid::FD_D2_N1/N2/N3 (src/grid.cpp:3232, 3566, 3900); axis = 1, 2 or 3. */
int b200_fd_d2(const b200_layout* lay, int axis, int order, b200_field u, b200_field w,
		double inv2_1, double inv2_2, double inv2_3, void* stream);

/* Grid::FD_D1_N1/N2/N3 (src/grid.cpp:3401, 3735, 4069; stencils src/fdm.h:27-275): the
 * staggered first derivative at i - 1/2, w = ((A1 (u[i] - u[i-1]) + ...) * inv_a on INNER
 * points, bit-identical to the CPU path. inv_a = ONE / d_a in the compute type (src/grid.cpp:
 * 3414-3416); axis = 1..dim; the layout halo must be at least order / 2. */
int b200_fd_d1(const b200_layout* lay, int axis, int order, b200_field u, b200_field w,
		double inv_1, double inv_2, double inv_3, void* stream);

/* Grid::FD_LAPLACIAN (src/grid.cpp:4235-4576). */
int b200_laplacian(const b200_layout* lay, int order, b200_field u, b200_field w,
		double inv2_1, double inv2_2, double inv2_3, void* stream);

/* Grid::updatePressure (src/grid.cpp:4579-4609): prn = 2 prc - prn + coef*lapla, INNER. */
int b200_update_pressure(const b200_layout* lay, b200_field prn, b200_field prc, b200_field coef,
		b200_field lapla, void* stream);

/* Grid::computePressureWithFD (src/grid.cpp:4612-5113), `this` = prn:
 * prn = 2 prc - prn + coef * Laplacian(prc) on INNER points, in one pass. */
int b200_compute_pressure(const b200_layout* lay, int order, b200_field prn, b200_field prc,
		b200_field coef, double inv2_1, double inv2_2, double inv2_3, void* stream);

/* Grid::applyBoundaryCondition (src/grid.cpp:3065-3229). `faces` is a 6-bit mask of the
 * faces with no neighbour (bit 0: I1HALO1, 1: I1HALO2, 2: I2HALO1, 3: I2HALO2,
 * 4: I3HALO1, 5: I3HALO2); 0x3F for a single rank. Same result as the reference's
 * sequential face order. */
int b200_apply_boundary(const b200_layout* lay, b200_field u, int bc_type, int faces,
		void* stream);

/* Propagator_Ac2::computeWavefieldNextTimeStep for one rank (src/propagator_Ac2.cpp:366-395):
 * applyBoundaryCondition(prc) then computePressureWithFD(prn, prc), in one call. For 3-D
 * FP32/FP64 grids with at least halo + 2 inner points per axis, once selected by
 * b200_autotune_stencil or b200_set_stencil_config (op 6), the boundary condition is fused into
 * the pressure kernel (the anti-mirror values are built inside its shared-memory tiles),
 * followed by a small kernel that writes the boundary planes' zeros into prc; prn and the inner
 * points of prc end up bit-identical to the two separate calls, and prc's halo points are left
 * as they were (the next boundary condition rebuilds them before any read). Otherwise it runs
 * the boundary-condition kernels and the pressure kernel back to back. With tuning on first use
 * (b200_set_autotune) the choice is measured for each grid size of at least 2^24 inner points;
 * HPCSCAN_B200_FUSED_STEP=1 in the environment selects the fused kernel for every grid it
 * accepts. */
int b200_propagate_step(const b200_layout* lay, int order, b200_field prn, b200_field prc,
		b200_field coef, double inv2_1, double inv2_2, double inv2_3, int bc_type, void* stream);

/* ---- norms (FP64 accumulation; synchronous on `stream`) ------------------------------------
 * Grid::getSumAbs (src/grid.cpp:2229-2274). */
int b200_sum_abs(const b200_layout* lay, b200_field u, const b200_box* box, double* out,
		void* stream);
/* Grid::getSumAbsDiff (src/grid.cpp:2173-2225): sum |u1 - u2|. */
int b200_sum_abs_diff(const b200_layout* lay, b200_field u1, b200_field u2, const b200_box* box,
		double* out, void* stream);
/* Grid::L1Err (src/grid.cpp:2058-2109) in one pass: sum |u1 - u2| and sum |u2|. */
int b200_l1_sums(const b200_layout* lay, b200_field u1, b200_field u2, const b200_box* box,
		double* sum_abs_diff, double* sum_abs_ref, void* stream);
/* Grid::maxErr (src/grid.cpp:2006-2054): max over the box of |u1-u2|/|u2|, or |u1-u2|
 * where |(float)u2| < max_err_float (MAX_ERR_FLOAT, src/constant.h:14-20). */
int b200_max_err(const b200_layout* lay, b200_field u1, b200_field u2, const b200_box* box,
		double max_err_float, double* out, void* stream);
/* Grid::getMin / getMax (src/grid.cpp:2278-2334), both in one pass. */
int b200_min_max(const b200_layout* lay, b200_field u, const b200_box* box, double* mn,
		double* mx, void* stream);

/* Analytic-reference error norm without materialising the reference grid: the
 * separable field r = amp*v1*v2*v3 (rounded to u's storage type, as Grid::fill would
 * store it) replaces u2 in b200_l1_sums. This fuses the refGrid fill + getSumAbsDiff +
 * getSumAbs of TestCase_Propa::run (src/testCase_Propa.cpp:136-151) into one read of u. */
int b200_l1_sums_separable(const b200_layout* lay, b200_field u, const b200_box* box,
		const double* v1, const double* v2, const double* v3, double amp, int ref_dtype,
		double* sum_abs_diff, double* sum_abs_ref, void* stream);

/* b200_l1_sums_separable without any allocation (no counterpart in the reference, whose CPU
 * norms need no device memory). For callers that must not allocate once their time loop runs:
 * an application whose own pool holds the device memory (a cudaMalloc could fail there), or one
 * that cannot take the device-wide synchronisation of the cudaFree with which
 * b200_l1_sums_separable grows its scratch, or the pinned host buffer it allocates for results.
 * Works on a 160 KB scratch array compiled into the library, one per device: the tables of at
 * most 16384 entries (box nx + ny + nz; larger boxes are rejected with B200_ERR_UNSUPPORTED)
 * and at most 2048 partial sums. The first call on a device sets up (takes the array's device
 * address and loads the kernels) and should precede any stream capture; later calls allocate
 * and load nothing. Nothing in the scratch must start at zero: each call writes every entry it
 * reads. The scratch is shared by all calls on a device, so calls that overlap (from two host
 * threads, or on two streams) race; serialise them. Same results as b200_l1_sums_separable;
 * synchronous on `stream`. */
int b200_l1_sums_separable_noalloc(const b200_layout* lay, b200_field u, const b200_box* box,
		const double* v1, const double* v2, const double* v3, double amp, int ref_dtype,
		double* sum_abs_diff, double* sum_abs_ref, void* stream);

/* ---- acoustic modelling and adjoint gradient (no counterpart in the reference) ---------------
 * A batch of shots, each on its own 3-D FP32 grid (its own size, model, source and receivers),
 * stepped in lockstep: one launch per stencil pass for the whole batch. Per shot, with the
 * damping G = g1(i1) g2(i2) g3(i3) of an absorbing sponge and C = (v dt)^2 (the reference's
 * coef, src/propagator_Ac2.cpp:234), on the INNER points, halos held at zero:
 *   forward   p[n+1] = G (2 p[n] + C Lap p[n]) - G^2 p[n-1];  p[n+1](src) += G amp wavelet[n];
 *             traces[n][r] = p[n+1](rec[r])                     (n = 0..nt-1)
 *   adjoint   w[k] = G (2 w[k+1] + C Lap w[k+1]) - G^2 w[k+2];
 *             w[k](rec[r]) += C G (traces[k-1][r] - dobs[k-1][r])   (k = nt..1)
 *   gradient  grad += -(C / dt^2) w[n+1] Lap p[n]: with J = 1/2 sum (traces - dobs)^2 and the
 *             squared slowness m = 1/v^2, dJ/dm summed over the steps.
 * The recursion of w is the exact transpose of the forward one (the Laplacian with zero halos is
 * symmetric), so the gradient is that of the discrete misfit.
 * Each shot keeps `nslot` forward grids (`wave`, consecutive, n1*n2*n3 each) and two adjoint
 * grids (`adj`); every call names the slots it reads and writes, so a caller can keep a ring of
 * recomputed forward wavefields for checkpointing. Calls enqueue kernels on `stream` and neither
 * allocate nor synchronise (b200_batch_create allocates the batch's small device tables). The
 * receivers of a shot must be distinct points. */
typedef struct b200_shot {
	b200_layout lay;            /* 3-D, FP32, halo = order/2, n1 * 4 bytes a multiple of 16   */
	double inv2[3];             /* (1/d_a)^2                                                  */
	const float* coef;          /* C = (v dt)^2 (device)                                      */
	const float* sponge[3];     /* damping tables over n1, n2, n3 (device)                    */
	int64_t src;                /* flat index of the source point                             */
	float amp;                  /* source amplitude factor                                    */
	const float* wavelet;       /* nt source samples (device)                                 */
	int nrec;
	const int64_t* rec;         /* nrec distinct flat receiver indices (device)               */
	float* traces;              /* nt x nrec synthetic data, written by the forward steps     */
	const float* dobs;          /* nt x nrec observed data (adjoint)                          */
	float* wave;                /* nslot forward grids (device, 16-byte aligned)              */
	float* adj;                 /* 2 adjoint grids (device), or NULL                          */
	float* grad;                /* gradient of this shot (device), or NULL                    */
} b200_shot;
typedef struct b200_batch b200_batch;
#define B200_BATCH_ADJOINT  1
#define B200_BATCH_GRADIENT 2
/* Build the batch (checks every shot, encodes its tensor maps, uploads the tables). dt is the
 * common time step (the gradient factor -1/dt^2). */
int b200_batch_create(b200_batch** batch, int order, int nslot, int nshot, const b200_shot* shots,
		double dt, int flags);
int b200_batch_destroy(b200_batch* batch);
/* Forward step n of every shot: wave[sout] = G (2 wave[scur] + C Lap wave[scur]) - G^2 wave[sprev]
 * (sout may equal sprev, not scur), then the source and the receivers of row n. */
int b200_batch_forward_step(b200_batch* batch, int n, int scur, int sprev, int sout, void* stream);
/* Adjoint step k of every shot: adj[1-scur] = w[k] from adj[scur] = w[k+1], adj[1-scur] = w[k+2]. */
int b200_batch_adjoint_step(b200_batch* batch, int k, int scur, void* stream);
/* grad += -(C/dt^2) adj[sadj] Lap wave[swave] for every shot. */
int b200_batch_gradient(b200_batch* batch, int swave, int sadj, void* stream);
/* The survey gradient of a batch whose shots share one grid layout, one step, for all shots in
 * one pass without a stencil: the forward recursion gives C Lap p[n] = (p[n+1] - G amp s[n]
 * delta_src + G^2 p[n-1]) / G - 2 p[n], so
 *   grad += -(1/dt^2) sum_s w_s[n+1] (p_s[n+1] / G + G p_s[n-1] - 2 p_s[n] - amp s[n] delta_src)
 * with wave[snext] = p[n+1], wave[scur] = p[n], wave[sprev] = p[n-1] and adj[sadj] = w[n+1] of
 * every shot; `grad` is one grid of the common layout (device). The sum over the shots of their
 * b200_batch_gradient contributions, up to FP32 rounding, at 16 bytes read per shot and point
 * plus the gradient's read and write, where b200_batch_gradient reads 20 per shot. No
 * counterpart in the reference. */
int b200_batch_survey_gradient(b200_batch* batch, int n, int snext, int scur, int sprev, int sadj,
		float* grad, void* stream);
/* CTAs of one stencil pass over the whole batch. */
int b200_batch_info(const b200_batch* batch, int* ctas_per_pass);

/* ---- arithmetic mode and tuning ---------------------------------------------------------------
 * B200_ARITH_EXACT (default): every multiply and add of the stencil operators is a separately
 * rounded IEEE operation in the reference's evaluation order, so FP32/FP64 results are
 * bit-identical to the reference CPU path built without FP contraction.
 * B200_ARITH_FMA: the same expression order with fused multiply-adds (fewer instructions;
 * results differ from the reference in the last bits). Applies to the 3-D z-marching
 * pressure and Laplacian kernels. No reference counterpart. */
#define B200_ARITH_EXACT 0
#define B200_ARITH_FMA   1
int b200_set_arith_mode(int mode);
int b200_get_arith_mode(int* mode);

/* Operators for the tuning calls: 1..3 = FD_D2_N1..N3, 4 = FD_LAPLACIAN,
 * 5 = computePressureWithFD, 6 = the fused propagator step. */
#define B200_OP_FD_D2_N1     1
#define B200_OP_FD_D2_N2     2
#define B200_OP_FD_D2_N3     3
#define B200_OP_LAPLACIAN    4
#define B200_OP_PRESSURE     5
#define B200_OP_STEP         6    /* b200_propagate_step with the anti-mirror BC */

/* Tile shape (0..2 for the Laplacian, pressure and step kernels, 0 otherwise) and planes per
 * CTA (0 = heuristic) used by the 3-D kernels for (dtype, order, op); shape -1 restores the
 * untuned defaults. For op 6 a shape selects the fused step kernel (untuned, b200_propagate_step
 * runs the boundary-condition kernels and the pressure kernel). Replaces the reference's manual
 * cache-block flags -cb1/-cb2/-cb3 (src/config.cpp; src/grid_Cuda_Optim.cu:2163-2211). */
int b200_set_stencil_config(int dtype, int order, int op, int shape, int nz_chunk);
int b200_get_stencil_config(int dtype, int order, int op, int* shape, int* nz_chunk);

/* Autotuner: times every tile shape and plane-chunk candidate of the 3-D kernel for `op` on
 * scratch grids of this layout (allocated and freed here), records the fastest for later
 * launches of (dtype, order, op) and returns it. For op 6 it also times the boundary-condition
 * kernels + the tuned pressure kernel and keeps the fused kernel only if it is faster
 * (*best_shape = -1 then). Synchronous. No reference counterpart (the reference sweeps -cb
 * flags by script: script/testCase_FD_D2/cacheBlkAnalysis). */
int b200_autotune_stencil(const b200_layout* lay, int order, int dtype, int op, int reps,
		int* best_shape, int* best_chunk, double* best_ms);

/* Tuning on first use (default on; the environment variable HPCSCAN_B200_AUTOTUNE=0 turns it
 * off at start-up): the first launch of the Laplacian, pressure or fused-step kernel for a grid
 * of at least 2^24 inner points runs b200_autotune_stencil for that grid size, storage type,
 * order and operator (scratch grids of the layout's size are allocated and freed; the call
 * synchronises) and every later launch of the key uses the result. Skipped while the stream
 * is being captured, and for keys with an explicit b200_set_stencil_config. The choice of
 * shape never changes results: every shape evaluates the same expressions in the same order.
 * The role of the reference's -cb1/-cb2/-cb3 sweep (src/grid_Cuda_Optim.cu:2163-2211),
 * automatic; no reference counterpart as an entry point. */
#define B200_AUTOTUNE_OFF 0
#define B200_AUTOTUNE_ON  1
int b200_set_autotune(int mode);
int b200_get_autotune(int* mode);

/* Readies the kernels of (layout, order, dtype, op) before a timed loop: the first-use tuning
 * where it applies, else one launch of the operator on zeroed scratch grids of the layout
 * (allocated, synchronised and freed here), so that the loop's first call pays neither the
 * tuning nor the loading of its kernels. coef_dtype: the coef grid's storage (-1: dtype).
 * Synchronous. No reference counterpart. */
int b200_prepare_stencil(const b200_layout* lay, int order, int dtype, int op, int coef_dtype);

/* The launch parameters a grid of this layout gets for (dtype, order, op): tile shape, planes
 * per CTA (0 = heuristic), fused step chosen (op 6), and whether they come from a measurement
 * or an explicit setting (*measured = 1) or from the defaults (0). No device work. */
int b200_get_tuned_config(const b200_layout* lay, int order, int dtype, int op, int* shape,
		int* nz_chunk, int* fused, int* measured);

/* ---- diagnostics ----------------------------------------------------------------------------
 * Device-side error word of the library's kernels (0 = none; bit 0: a producer gave up a
 * bounded wait, bit 1: a consumer did). Synchronous; `clear` resets it. No reference
 * counterpart: the reference's CUDA modes have no device-side waits. */
int b200_device_status(int* status, int clear);

/* Which kernel family computes a stencil call with this layout/order/dtype on the current
 * device: 1 = 3-D z-marching TMA kernel, 2 = direct kernel, 0 = rejected (see
 * b200_last_error). No device work. No reference counterpart. */
int b200_stencil_route(const b200_layout* lay, int order, int dtype, int* route);

#ifdef __cplusplus
}
#endif

#endif /* HPCSCAN_B200_H_ */
