// Dispatcher, tensor maps, tuning table and autotuner of the 3-D z-marching stencil
// kernels (the kernel itself is in b200_zmarch.cuh).
//
// Tuning: for every (storage type, order, operator) the launch uses a tile shape and a
// number of planes per CTA. Defaults come from a heuristic; b200_autotune_stencil times
// every shape and chunk candidate on scratch grids of the caller's layout and records the
// fastest, which every later launch of that key uses (the reference's -cb1/-cb2/-cb3
// cache-block sweep, src/grid_Cuda_Optim.cu:2163-2211 and script/testCase_FD_D2/
// cacheBlkAnalysis, made automatic).
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "b200_zmarch.cuh"

namespace b200 {

int apply_boundary(const b200_layout* lay, const b200_field& u, int bc_type, int faces,
		cudaStream_t s);

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
		const cuuint64_t*, const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
		CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int get_encode(EncodeTiledFn* fn)
{
	static EncodeTiledFn cached = nullptr;
	if (!cached) {
		void* p = nullptr;
		cudaDriverEntryPointQueryResult q;
		int rc = cuda_error(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q),
				"cudaGetDriverEntryPoint(cuTensorMapEncodeTiled)");
		if (rc) return rc;
		if (q != cudaDriverEntryPointSuccess || !p)
			return set_error(B200_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
		cached = reinterpret_cast<EncodeTiledFn>(p);
	}
	*fn = cached;
	return B200_OK;
}

CUtensorMapDataType tma_dtype(int dtype)
{
	switch (dtype) {
	case B200_F64: return CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
	case B200_F16: return CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
	case B200_BF16: return CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
	default: return CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
	}
}

bool has_shapes(int mode)
{
	return mode == MODE_PRESSURE || mode == MODE_LAPLACIAN || mode == MODE_STEP;
}

// ---- tuning table --------------------------------------------------------------------------
struct Tuned {
	int shape = 0;
	int nz_chunk = 0;   // 0: heuristic
	bool fused = false; // MODE_STEP only: the fused kernel beat BC + pressure when tuned
};
// (dtype, R, mode, exact) and, for entries the autotuner measured, the grid's n1, n2, n3
using TuneKey = std::tuple<int, int, int, int, int64_t, int64_t, int64_t>;
std::map<TuneKey, Tuned> g_tuned;      // measured by the autotuner, per grid size
std::map<TuneKey, Tuned> g_forced;     // set by b200_set_stencil_config (any grid size)
std::mutex g_tune_mutex;
int g_arith = B200_ARITH_EXACT;
// tuning on first use: -1 = not decided yet (environment HPCSCAN_B200_AUTOTUNE, default on)
int g_autotune = -1;
std::mutex g_autotune_mutex;           // one first-use tuning at a time
// grids smaller than this (inner points) keep the defaults: their launches are too short to
// rank shapes reliably, and tuning them would cost more than it saves
constexpr int64_t kAutotuneMinPoints = int64_t(1) << 24;

TuneKey key_of(int dtype, int R, int mode, bool exact, const b200_layout* lay)
{
	return TuneKey{dtype, R, mode, exact ? 1 : 0, lay ? lay->n1 : 0, lay ? lay->n2 : 0,
	               lay ? lay->n3 : 0};
}

// Untuned defaults: the fastest shape of the pressure update measured at 512^3 on B200 for each
// storage type and half width, interleaved runs (FP32: the two-row 28x64 tiles up to R = 2, the
// 14x64 tiles with a four-plane prefetch for R = 3..4, 22x64 tiles of 11 warps with a five-plane
// prefetch for R = 5..6, the 14x64 tiles at two CTAs per SM for R = 7, the 9-warp 16x64 tiles
// for R = 8;
// FP64: 28x32 two-row tiles up to R = 2, 14x32 tiles with the four-plane prefetch for R = 3..5,
// 16x32 9-warp tiles beyond). 16-bit wavefields (pressure update only): 8-byte thread vectors
// with the z queue in FP32, 14-row tiles and the four-plane prefetch up to R = 4, 28-row
// tiles beyond (launch_16bit). The z-chunk follows the grid size (pick_nz_chunk).
Tuned default_tuning(int dtype, int R)
{
	Tuned t;
	if (dtype == B200_F64) t.shape = R <= 2 ? 0 : R <= 4 ? 1 : 2;
	else if (dtype == B200_F16 || dtype == B200_BF16) t.shape = R <= 4 ? 1 : 2;
	else t.shape = R <= 2 ? 0 : R <= 4 ? 1 : 2;
	t.nz_chunk = 0;
	return t;
}

// The launch parameters of a key: an explicit setting, else what the autotuner measured for
// this grid size, else the defaults. *measured tells whether a measured or explicit entry
// exists (false: the defaults were returned).
Tuned tuned_for(int dtype, int R, int mode, bool exact, const b200_layout* lay,
		bool* measured = nullptr)
{
	std::lock_guard<std::mutex> lock(g_tune_mutex);
	if (measured) *measured = true;
	auto f = g_forced.find(key_of(dtype, R, mode, exact, nullptr));
	if (f != g_forced.end()) return f->second;
	if (lay) {
		auto it = g_tuned.find(key_of(dtype, R, mode, exact, lay));
		if (it != g_tuned.end()) return it->second;
	}
	if (measured) *measured = false;
	return has_shapes(mode) ? default_tuning(dtype, R) : Tuned{};
}

// Times the candidates of one key on scratch grids and records the fastest (the body of
// b200_autotune_stencil, defined below).
int autotune_key(const b200_layout* lay, int order, int dtype, int op, int reps,
		int* best_shape = nullptr, int* best_chunk = nullptr, double* best_ms = nullptr);

bool autotune_enabled()
{
	if (g_autotune < 0) {
		const char* e = std::getenv("HPCSCAN_B200_AUTOTUNE");
		g_autotune = (e && e[0] == '0') ? B200_AUTOTUNE_OFF : B200_AUTOTUNE_ON;
	}
	return g_autotune == B200_AUTOTUNE_ON;
}

// HPCSCAN_B200_FUSED_STEP=1 in the environment: b200_propagate_step takes the fused kernel for
// every grid it accepts, without measuring (the way to select it from a program that cannot
// call b200_set_stencil_config, such as hpcscan's own drivers); read once.
bool fused_step_forced()
{
	static const bool forced = [] {
		const char* e = std::getenv("HPCSCAN_B200_FUSED_STEP");
		return e && e[0] == '1';
	}();
	return forced;
}

int launch(const ZLaunch& L)
{
	switch (L.mode) {
	case MODE_STEP: return zmarch_launch_step(L);
	case MODE_PRESSURE: return zmarch_launch_pressure(L);
	case MODE_LAPLACIAN: return zmarch_launch_laplacian(L);
	case MODE_D1_AXIS1:
	case MODE_D1_AXIS2:
	case MODE_D1_AXIS3: return zmarch_launch_d1(L);
	default: return zmarch_launch_d2(L);
	}
}

}  // namespace

int make_map(CUtensorMap* m, const void* base, int dtype, const b200_layout* lay, int bx, int by)
{
	EncodeTiledFn enc;
	if (int rc = get_encode(&enc)) return rc;
	const int es = dtype_size(dtype);
	const cuuint64_t dims[3] = {(cuuint64_t)lay->n1, (cuuint64_t)lay->n2, (cuuint64_t)lay->n3};
	const cuuint64_t strides[2] = {(cuuint64_t)(lay->n1 * es), (cuuint64_t)(lay->n1 * lay->n2 * es)};
	const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
	const cuuint32_t estr[3] = {1, 1, 1};
	std::memset(m, 0, sizeof(*m));
	CUresult r = enc(m, tma_dtype(dtype), 3, const_cast<void*>(base), dims, strides, box, estr,
			CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
			CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	if (r != CUDA_SUCCESS)
		return set_error(B200_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d) for box %dx%d", (int)r, bx, by);
	return B200_OK;
}

int make_map_slots(CUtensorMap* m, const void* base, const b200_layout* lay, int nslot, int bx,
		int by)
{
	EncodeTiledFn enc;
	if (int rc = get_encode(&enc)) return rc;
	const cuuint64_t es = 4;
	const cuuint64_t dims[4] = {(cuuint64_t)lay->n1, (cuuint64_t)lay->n2, (cuuint64_t)lay->n3,
	                            (cuuint64_t)nslot};
	const cuuint64_t strides[3] = {lay->n1 * es, lay->n1 * lay->n2 * es,
	                               lay->n1 * lay->n2 * lay->n3 * es};
	const cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, 1, 1};
	const cuuint32_t estr[4] = {1, 1, 1, 1};
	std::memset(m, 0, sizeof(*m));
	CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void*>(base), dims, strides,
			box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
			CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	if (r != CUDA_SUCCESS)
		return set_error(B200_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d) for a slotted grid", (int)r);
	return B200_OK;
}

bool zmarch_accepts(const b200_layout* lay, int dtype)
{
	if (lay->dim != 3) return false;
	if (dtype != B200_F32 && dtype != B200_F64 && dtype != B200_F16 && dtype != B200_BF16) return false;
	if ((lay->n1 * dtype_size(dtype)) % 16 != 0) return false;   // TMA stride rule
	if (lay->n1 > (1 << 30) || lay->n2 > (1 << 30) || lay->n3 > (1 << 30)) return false;
	return true;
}

int run_zmarch(int mode, const b200_layout* lay, int order, const b200_field& in,
		const b200_field& out, const b200_field* coef, double inv2_1, double inv2_2, double inv2_3,
		cudaStream_t s, int* handled)
{
	*handled = 0;
	if (!zmarch_accepts(lay, in.dtype)) return B200_OK;
	if (mode == MODE_STEP) {
		// the in-tile boundary condition needs mirror points that are never boundary points
		if (lay->e1 - lay->s1 + 1 < lay->halo + 2 || lay->e2 - lay->s2 + 1 < lay->halo + 2 ||
				lay->e3 - lay->s3 + 1 < lay->halo + 2)
			return B200_OK;
	}
	const bool half = in.dtype == B200_F16 || in.dtype == B200_BF16;
	if (half && mode != MODE_PRESSURE) return B200_OK;      // 16-bit: the pressure update only
	if (out.dtype != in.dtype) return B200_OK;
	if ((reinterpret_cast<uintptr_t>(in.data) | reinterpret_cast<uintptr_t>(out.data)) % 16) return B200_OK;
	if (coef) {
		if (coef->dtype != in.dtype && !(half && coef->dtype == B200_F32)) return B200_OK;
		if (coef->dtype == B200_F32 && (lay->n1 * 4) % 16) return B200_OK;
		if (reinterpret_cast<uintptr_t>(coef->data) % 16) return B200_OK;
	}
	const bool exact = !has_shapes(mode) || g_arith == B200_ARITH_EXACT;
	bool measured = false;
	Tuned t = tuned_for(in.dtype, order / 2, mode, exact, lay, &measured);
	if (!measured && has_shapes(mode) && autotune_enabled() &&
			!(mode == MODE_STEP && fused_step_forced())) {
		// first use of this (grid size, storage type, order, operator): time the candidates once
		// and keep the fastest for every later launch (not while the stream is being captured:
		// the tuning allocates and synchronises)
		const int64_t inner = (int64_t)(lay->e1 - lay->s1 + 1) * (lay->e2 - lay->s2 + 1) *
		                      (lay->e3 - lay->s3 + 1);
		cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
		cudaStreamIsCapturing(s, &cap);
		if (inner >= kAutotuneMinPoints && cap == cudaStreamCaptureStatusNone) {
			std::lock_guard<std::mutex> guard(g_autotune_mutex);
			if (int rc = autotune_key(lay, order, in.dtype, mode, 5)) {
				// could not tune (e.g. no device memory for the scratch grids): remember the
				// defaults for this key so that the next launch does not try again
				std::lock_guard<std::mutex> lock(g_tune_mutex);
				g_tuned[key_of(in.dtype, order / 2, mode, exact, lay)] = t;
				(void)rc;
			}
			t = tuned_for(in.dtype, order / 2, mode, exact, lay);
		}
	}
	if (mode == MODE_STEP && fused_step_forced()) t.fused = true;
	if (mode == MODE_STEP && !t.fused) return B200_OK;   // separate BC + pressure is faster
	*handled = 1;
	ZLaunch L;
	L.mode = mode;
	L.lay = lay;
	L.R = order / 2;
	L.in = &in;
	L.out = &out;
	L.coef = coef;
	L.inv2[0] = inv2_1;
	L.inv2[1] = inv2_2;
	L.inv2[2] = inv2_3;
	L.s = s;
	L.exact = exact;
	L.shape = t.shape;
	L.nz_chunk = t.nz_chunk;
	if (int rc = device_error_word(&L.err)) return rc;
	return launch(L);
}

}  // namespace b200

using namespace b200;

extern "C" {

int b200_set_arith_mode(int mode)
{
	if (mode != B200_ARITH_EXACT && mode != B200_ARITH_FMA)
		return set_error(B200_ERR_ARG, "arithmetic mode %d", mode);
	g_arith = mode;
	return B200_OK;
}

int b200_get_arith_mode(int* mode)
{
	if (!mode) return set_error(B200_ERR_ARG, "mode is NULL");
	*mode = g_arith;
	return B200_OK;
}

int b200_set_stencil_config(int dtype, int order, int op, int shape, int nz_chunk)
{
	if (int rc = check_order(order)) return rc;
	if (dtype != B200_F32 && dtype != B200_F64 &&
			!((dtype == B200_F16 || dtype == B200_BF16) && op == MODE_PRESSURE))
		return set_error(B200_ERR_UNSUPPORTED,
				"tuned kernels exist for FP32 and FP64, and for the 16-bit pressure update");
	if (op < MODE_D2_AXIS1 || op > MODE_STEP) return set_error(B200_ERR_ARG, "operator %d", op);
	if (shape < -1 || shape >= (has_shapes(op) ? kZShapes : 1))
		return set_error(B200_ERR_ARG, "shape %d", shape);
	if (nz_chunk < 0) return set_error(B200_ERR_ARG, "nz_chunk %d", nz_chunk);
	std::lock_guard<std::mutex> lock(g_tune_mutex);
	if (shape == -1) {   // back to the measured or default parameters
		for (int ex = 0; ex < 2; ex++) g_forced.erase(key_of(dtype, order / 2, op, ex, nullptr));
		return B200_OK;
	}
	// setting a shape for the fused step selects the fused kernel
	for (int ex = 0; ex < 2; ex++)
		g_forced[key_of(dtype, order / 2, op, ex, nullptr)] = Tuned{shape, nz_chunk, op == MODE_STEP};
	return B200_OK;
}

int b200_get_stencil_config(int dtype, int order, int op, int* shape, int* nz_chunk)
{
	if (!shape || !nz_chunk) return set_error(B200_ERR_ARG, "NULL output");
	if (int rc = check_order(order)) return rc;
	const Tuned t = tuned_for(dtype, order / 2, op, g_arith == B200_ARITH_EXACT || !has_shapes(op),
			nullptr);
	*shape = t.shape;
	*nz_chunk = t.nz_chunk;
	return B200_OK;
}

int b200_get_tuned_config(const b200_layout* lay, int order, int dtype, int op, int* shape,
		int* nz_chunk, int* fused, int* measured)
{
	if (!shape || !nz_chunk || !fused || !measured) return set_error(B200_ERR_ARG, "NULL output");
	if (int rc = check_layout(lay)) return rc;
	if (int rc = check_order(order)) return rc;
	bool m = false;
	const Tuned t = tuned_for(dtype, order / 2, op, g_arith == B200_ARITH_EXACT || !has_shapes(op),
			lay, &m);
	*shape = t.shape;
	*nz_chunk = t.nz_chunk;
	*fused = t.fused ? 1 : 0;
	*measured = m ? 1 : 0;
	return B200_OK;
}

int b200_set_autotune(int mode)
{
	if (mode != B200_AUTOTUNE_OFF && mode != B200_AUTOTUNE_ON)
		return set_error(B200_ERR_ARG, "autotune mode %d", mode);
	g_autotune = mode;
	return B200_OK;
}

int b200_get_autotune(int* mode)
{
	if (!mode) return set_error(B200_ERR_ARG, "mode is NULL");
	*mode = autotune_enabled() ? B200_AUTOTUNE_ON : B200_AUTOTUNE_OFF;
	return B200_OK;
}

int b200_autotune_stencil(const b200_layout* lay, int order, int dtype, int op, int reps,
		int* best_shape, int* best_chunk, double* best_ms)
{
	return autotune_key(lay, order, dtype, op, reps, best_shape, best_chunk, best_ms);
}

}  // extern "C"

namespace b200 {
namespace {

int autotune_key(const b200_layout* lay, int order, int dtype, int op, int reps, int* best_shape,
		int* best_chunk, double* best_ms)
{
	if (int rc = check_layout(lay)) return rc;
	if (int rc = check_order(order)) return rc;
	if (lay->halo != order / 2) return set_error(B200_ERR_ARG, "layout halo does not match order");
	if (!zmarch_accepts(lay, dtype))
		return set_error(B200_ERR_UNSUPPORTED, "layout/dtype not handled by the z-marching kernels");
	if (op < MODE_D2_AXIS1 || op > MODE_STEP) return set_error(B200_ERR_ARG, "operator %d", op);
	if (reps < 1) reps = 5;
	if (op == MODE_STEP) {
		// the fused step is compared with the boundary condition + the pressure kernel at its
		// own best parameters for this grid: tune those first
		bool have = false;
		tuned_for(dtype, order / 2, MODE_PRESSURE, !has_shapes(MODE_PRESSURE) || g_arith == B200_ARITH_EXACT,
				lay, &have);
		if (!have)
			if (int rc = autotune_key(lay, order, dtype, MODE_PRESSURE, reps)) return rc;
	}
	const size_t bytes = (size_t)npoint(lay) * dtype_size(dtype);
	void* buf[3] = {nullptr, nullptr, nullptr};
	int rc = B200_OK;
	for (int i = 0; i < 3 && !rc; i++) {
		const cudaError_t e = cudaMalloc(&buf[i], bytes);
		if (e == cudaErrorMemoryAllocation) cudaGetLastError();   // not sticky: clear it
		rc = cuda_error(e, "cudaMalloc(autotune)");
		if (!rc) rc = cuda_error(cudaMemset(buf[i], 0, bytes), "cudaMemset(autotune)");
	}
	cudaStream_t s = nullptr;
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	if (!rc) rc = cuda_error(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
	if (!rc) rc = cuda_error(cudaEventCreate(&e0), "cudaEventCreate");
	if (!rc) rc = cuda_error(cudaEventCreate(&e1), "cudaEventCreate");
	const b200_field fin{buf[0], dtype, 1.0f}, fout{buf[1], dtype, 1.0f}, fcoef{buf[2], dtype, 1.0f};
	ZLaunch L;
	L.mode = op;
	L.lay = lay;
	L.R = order / 2;
	L.in = &fin;
	L.out = &fout;
	L.coef = (op == MODE_PRESSURE || op == MODE_STEP) ? &fcoef : nullptr;
	L.inv2[0] = L.inv2[1] = L.inv2[2] = 1.0;
	L.s = s;
	L.exact = !has_shapes(op) || g_arith == B200_ARITH_EXACT;
	if (!rc) rc = device_error_word(&L.err);
	const int nz = (int)(lay->e3 - lay->s3 + 1);
	const std::vector<int> chunks = {0, 16, 32, 64, 128};
	double best = 1e300;
	Tuned win{};
	const int nshape = has_shapes(op) ? kZShapes : 1;
	for (int sh = 0; sh < nshape && !rc; sh++) {
		for (int c : chunks) {
			if (c > nz) continue;
			L.shape = sh;
			L.nz_chunk = c;
			if ((rc = launch(L))) {           // warm-up (and first-use module load)
				if (rc == B200_ERR_UNSUPPORTED) rc = B200_OK;   // shape does not fit: skip it
				break;
			}
			if ((rc = cuda_error(cudaEventRecord(e0, s), "cudaEventRecord"))) break;
			for (int r = 0; r < reps && !rc; r++) rc = launch(L);
			if (rc) break;
			if ((rc = cuda_error(cudaEventRecord(e1, s), "cudaEventRecord"))) break;
			if ((rc = cuda_error(cudaEventSynchronize(e1), "cudaEventSynchronize"))) break;
			float ms = 0.f;
			cudaEventElapsedTime(&ms, e0, e1);
			ms /= reps;
			if (ms < best) {
				best = ms;
				win = Tuned{sh, c};
			}
		}
	}
	if (!rc && op == MODE_STEP) {
		// the alternative: the boundary condition kernels + the best pressure kernel
		ZLaunch P = L;
		P.mode = MODE_PRESSURE;
		const Tuned tp = tuned_for(dtype, order / 2, MODE_PRESSURE, L.exact, lay);
		P.shape = tp.shape;
		P.nz_chunk = tp.nz_chunk;
		double sep = 1e300;
		auto run_sep = [&]() {
			int r = apply_boundary(lay, fin, B200_BOUND_COND_ANTI_MIRROR, 0x3F, s);
			return r ? r : launch(P);
		};
		if (!(rc = run_sep()) && !(rc = cuda_error(cudaEventRecord(e0, s), "cudaEventRecord"))) {
			for (int r = 0; r < reps && !rc; r++) rc = run_sep();
			if (!rc && !(rc = cuda_error(cudaEventRecord(e1, s), "cudaEventRecord")) &&
					!(rc = cuda_error(cudaEventSynchronize(e1), "cudaEventSynchronize"))) {
				float ms = 0.f;
				cudaEventElapsedTime(&ms, e0, e1);
				sep = ms / reps;
			}
		}
		win.fused = best < sep;
		if (!win.fused) best = sep;
	}
	if (e0) cudaEventDestroy(e0);
	if (e1) cudaEventDestroy(e1);
	if (s) cudaStreamDestroy(s);
	for (void* p : buf)
		if (p) cudaFree(p);
	if (rc) return rc;
	{
		std::lock_guard<std::mutex> lock(g_tune_mutex);
		g_tuned[key_of(dtype, order / 2, op, L.exact, lay)] = win;
	}
	if (best_shape) *best_shape = (op == MODE_STEP && !win.fused) ? -1 : win.shape;
	if (best_chunk) *best_chunk = win.nz_chunk;
	if (best_ms) *best_ms = best;
	return B200_OK;
}

}  // namespace
}  // namespace b200

using namespace b200;

extern "C" {

int b200_prepare_stencil(const b200_layout* lay, int order, int dtype, int op, int coef_dtype)
{
	if (int rc = check_layout(lay)) return rc;
	if (int rc = check_order(order)) return rc;
	if (lay->halo != order / 2) return set_error(B200_ERR_ARG, "layout halo does not match order");
	if (dtype_size(dtype) == 0) return set_error(B200_ERR_ARG, "dtype %d", dtype);
	if (op < MODE_D2_AXIS1 || op > MODE_STEP) return set_error(B200_ERR_ARG, "operator %d", op);
	if (coef_dtype < 0) coef_dtype = dtype;
	if (dtype_size(coef_dtype) == 0) return set_error(B200_ERR_ARG, "coef dtype %d", coef_dtype);
	const int64_t inner = (int64_t)(lay->e1 - lay->s1 + 1) * (lay->e2 - lay->s2 + 1) *
	                      (lay->e3 - lay->s3 + 1);
	const bool exact = !has_shapes(op) || g_arith == B200_ARITH_EXACT;
	if (has_shapes(op) && zmarch_accepts(lay, dtype) && autotune_enabled() &&
			inner >= kAutotuneMinPoints && coef_dtype == dtype) {
		bool have = false;
		tuned_for(dtype, order / 2, op, exact, lay, &have);
		if (!have) {
			// tuning launches every candidate kernel of the key, which loads them; a grid whose
			// scratch copies do not fit keeps the defaults (as on first use)
			std::lock_guard<std::mutex> guard(g_autotune_mutex);
			const int rc = autotune_key(lay, order, dtype, op, 5);
			if (rc == B200_ERR_NOMEM) {
				std::lock_guard<std::mutex> lock(g_tune_mutex);
				g_tuned[key_of(dtype, order / 2, op, exact, lay)] = default_tuning(dtype, order / 2);
				return B200_OK;
			}
			return rc;
		}
		return B200_OK;
	}
	// one launch of the operator on zeroed scratch grids of the layout (loads its kernels)
	const size_t n = (size_t)npoint(lay);
	void* buf[3] = {nullptr, nullptr, nullptr};
	const size_t sz[3] = {n * dtype_size(dtype), n * dtype_size(dtype), n * dtype_size(coef_dtype)};
	int rc = B200_OK;
	for (int i = 0; i < 3 && !rc; i++) {
		rc = cuda_error(cudaMalloc(&buf[i], sz[i]), "cudaMalloc(prepare)");
		if (!rc) rc = cuda_error(cudaMemset(buf[i], 0, sz[i]), "cudaMemset(prepare)");
	}
	if (!rc) {
		const b200_field u{buf[0], dtype, 1.0f}, w{buf[1], dtype, 1.0f}, c{buf[2], coef_dtype, 1.0f};
		const bool p = op == MODE_PRESSURE || op == MODE_STEP;
		if (op == MODE_STEP) {
			rc = b200_propagate_step(lay, order, w, u, c, 1.0, 1.0, 1.0, B200_BOUND_COND_ANTI_MIRROR,
					nullptr);
		} else {
			rc = run_stencil(op, lay, order, u, w, p ? &c : nullptr, 1.0, 1.0, 1.0, nullptr);
		}
		if (!rc) rc = cuda_error(cudaDeviceSynchronize(), "cudaDeviceSynchronize(prepare)");
	}
	for (void* b : buf)
		if (b) cudaFree(b);
	return rc;
}

}  // extern "C"
