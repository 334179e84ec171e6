// Acoustic modelling engine: batches of shots (each with its own grid, model, source and
// receivers) stepped forward and backward in lockstep, one launch per stencil pass for the whole
// batch, for the adjoint-state gradient of the receiver data misfit with respect to the squared
// slowness. The reference's propagator step (src/grid.cpp:4612-5113) with an absorbing sponge
// and a point source; the reference has no adjoint and no batching.
//
// Per shot, FP32 (the damping G = (g1(i1) g2(i2)) g3(i3), C = (v dt)^2):
//   forward   p[n+1] = G (2 p[n] + C Lap p[n]) - G^2 p[n-1] ; p[n+1](src) += G amp s[n]
//             traces[n] = p[n+1](receivers)
//   adjoint   w[k] = G (2 w[k+1] + C Lap w[k+1]) - G^2 w[k+2] ; w[k](rec) += C G (d[k] - dobs[k])
//   gradient  g += -(C / dt^2) w[n+1] Lap p[n]
// The stencil passes are k_zmarch_batch launches (b200_zmarch.cuh, MODE_MODEL / MODE_GRAD) over
// slotted grids: every shot keeps its forward wavefields in `nslot` consecutive grids and its
// adjoint wavefields in 2, and each call names the slots it reads and writes. No call allocates
// or synchronises, so a whole schedule can be captured in a CUDA graph.
#include <cstdlib>
#include <cstring>
#include <vector>

#include "b200_zmarch.cuh"

namespace b200 {
namespace {

// Shot data the small per-step kernels need (device copy, one per shot).
struct MShot {
	float* wave;                  // nslot x field
	float* adj;                   // 2 x field (or nullptr)
	int64_t field;                // elements per grid
	const float* coef;
	const float* g1;
	const float* g2;
	const float* g3;
	int64_t n1, n12;
	int64_t src;
	float amp;
	const float* wavelet;
	int nrec;
	const int64_t* rec;
	float* traces;
	const float* dobs;
};

__device__ __forceinline__ float damping(const MShot& m, int64_t ii)
{
	const int64_t z = ii / m.n12, r = ii - z * m.n12, y = r / m.n1, x = r - y * m.n1;
	return (m.g1[x] * m.g2[y]) * m.g3[z];
}

// The receivers of slot `slot` of every shot into row n of its traces (the source was added by
// the stencil pass). Grid (shots, receiver blocks), one thread per receiver.
__global__ void k_model_record(const MShot* __restrict__ shots, int n, int slot)
{
	const MShot& m = shots[blockIdx.x];
	const int r = blockIdx.y * blockDim.x + threadIdx.x;
	if (r >= m.nrec) return;
	m.traces[(int64_t)n * m.nrec + r] = m.wave[slot * m.field + m.rec[r]];
}

// Residual injection d[k] - dobs[k] (row k - 1) into adjoint slot `slot` at the (distinct)
// receivers. Grid (shots, receiver blocks).
__global__ void k_model_residual(const MShot* __restrict__ shots, int k, int slot)
{
	const MShot& m = shots[blockIdx.x];
	const int r = blockIdx.y * blockDim.x + threadIdx.x;
	if (r >= m.nrec) return;
	float* w = m.adj + slot * m.field;
	const int64_t row = (int64_t)(k - 1) * m.nrec;
	const int64_t ii = m.rec[r];
	const float res = m.traces[row + r] - m.dobs[row + r];
	w[ii] = fmaf(m.coef[ii] * damping(m, ii), res, w[ii]);
}

constexpr int kRecThreads = 128;

// Survey gradient of shots on one grid, one step, no stencil: the forward recursion gives
// C Lap p[n] = (p[n+1] - G amp s[n] delta_src + G^2 p[n-1]) / G - 2 p[n], so
//   grad += kscale sum_s w_s[n+1] (p_s[n+1] / G_s + G_s p_s[n-1] - 2 p_s[n] - amp_s s[n] delta_src)
// with the shots summed in batch order. One thread per 16-byte vector of four i1 points of a
// row (rows start 16-byte aligned; the vector of the first inner point may begin in the halo,
// whose lanes are read and written back unchanged), the shots' pointers staged in shared memory.
struct SurveyArgs {
	int64_t n1, n12, field;
	int x0, nvx;                // first vector's i1 (multiple of 4), vectors per row
	int s1, e1, s2, e2, s3, e3;
	int n, snext, scur, sprev, sadj, nshot;
	float kscale;
	float* grad;
};
constexpr int kSurveyMaxShots = 64;      // shots staged per pass over the table

__global__ void __launch_bounds__(256) k_survey_gradient(const MShot* __restrict__ shots, SurveyArgs a)
{
	__shared__ MShot sh[kSurveyMaxShots];
	const int ny = a.e2 - a.s2 + 1, nz = a.e3 - a.s3 + 1;
	const int64_t items = (int64_t)ny * nz * a.nvx;
	const int64_t stride = (int64_t)gridDim.x * blockDim.x;
	for (int base = 0; base < a.nshot; base += kSurveyMaxShots) {
		const int ns = min(kSurveyMaxShots, a.nshot - base);
		__syncthreads();
		for (int i = threadIdx.x; i < ns; i += blockDim.x) sh[i] = shots[base + i];
		__syncthreads();
		for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < items; t += stride) {
			const int64_t row = t / a.nvx;
			const int xv = (int)(t - row * a.nvx);
			const int z = (int)(row / ny), y = (int)(row - (int64_t)z * ny);
			const int i1 = a.x0 + 4 * xv, i2 = a.s2 + y, i3 = a.s3 + z;
			const int64_t idx = (int64_t)i3 * a.n12 + (int64_t)i2 * a.n1 + i1;
			float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
			for (int s = 0; s < ns; s++) {
				const MShot& m = sh[s];
				const float g23 = m.g2[i2] * m.g3[i3];
				const float4 g1 = *reinterpret_cast<const float4*>(m.g1 + i1);
				const float4 p1 = *reinterpret_cast<const float4*>(m.wave + a.snext * a.field + idx);
				const float4 p0 = *reinterpret_cast<const float4*>(m.wave + a.scur * a.field + idx);
				const float4 pm = *reinterpret_cast<const float4*>(m.wave + a.sprev * a.field + idx);
				const float4 w = *reinterpret_cast<const float4*>(m.adj + a.sadj * a.field + idx);
				const float G[4] = {g1.x * g23, g1.y * g23, g1.z * g23, g1.w * g23};
				const float P1[4] = {p1.x, p1.y, p1.z, p1.w}, P0[4] = {p0.x, p0.y, p0.z, p0.w};
				const float PM[4] = {pm.x, pm.y, pm.z, pm.w}, W[4] = {w.x, w.y, w.z, w.w};
				float* A = &acc.x;
#pragma unroll
				for (int e = 0; e < 4; e++) {
					if (G[e] == 0.0f) continue;            // halo lanes: G = 0 there
					float c = fmaf(G[e], PM[e], __fdiv_rn(P1[e], G[e])) - 2.0f * P0[e];
					if (idx + e == m.src) c -= m.amp * m.wavelet[a.n];
					A[e] = fmaf(W[e], c, A[e]);
				}
			}
			float4* gp = reinterpret_cast<float4*>(a.grad + idx);
			float4 g = *gp;
			float* G4 = &g.x;
			const float* A = &acc.x;
#pragma unroll
			for (int e = 0; e < 4; e++)
				if (i1 + e >= a.s1 && i1 + e <= a.e1) G4[e] = fmaf(a.kscale, A[e], G4[e]);
			*gp = g;
		}
	}
}

// Stencil passes: R and the tile shape (the pressure update's FP32 default: shape 0 up to
// R = 2, shape 1 beyond), FP32 with fused multiply-adds.
template <int R>
using ModelShape = Shape<float, R, (R <= 2 ? 0 : 1)>;
template <int R, int MODE>
using ModelCfg = ZCfg<float, R, MODE, ModelShape<R>::TX, ModelShape<R>::TY, ModelShape<R>::VY,
		ModelShape<R>::PF, false, ModelShape<R>::MINB>;

}  // namespace
}  // namespace b200

using namespace b200;

struct b200_batch {
	int R = 0;
	int nshot = 0;
	int nslot = 0;
	int ctas = 0;                   // CTAs of one stencil pass over the whole batch
	int max_nrec = 0;
	int smem[3] = {0, 0, 0};
	bool interleave = false;        // every shot has the same tiling: CTAs tile-major, shot-minor
	bool same_grid = false;         // every shot has the same layout (the survey gradient)
	b200_layout lay0{};             // the first shot's layout
	float kscale = 0.0f;            // -1 / dt^2
	ZShot* d_fwd = nullptr;         // stencil tables: forward, adjoint, gradient
	ZShot* d_adj = nullptr;
	ZShot* d_grad = nullptr;
	MShot* d_m = nullptr;
	bool has_adj = false, has_grad = false;
};

namespace {

template <int R>
int batch_tables(b200_batch* b, const b200_shot* shots, double dt, std::vector<ZShot>& fwd,
		std::vector<ZShot>& adj, std::vector<ZShot>& grad)
{
	using CF = ModelCfg<R, MODE_MODEL>;
	using CG = ModelCfg<R, MODE_GRAD>;
	static_assert(CF::TX == CG::TX && CF::TY == CG::TY && CF::BX == CG::BX && CF::BY == CG::BY,
			"one tiling for every pass");
	int rc0 = cuda_error(cudaFuncSetAttribute(k_zmarch_batch<CF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
			CF::SMEM), "cudaFuncSetAttribute(k_zmarch_batch)");
	if (!rc0)
		rc0 = cuda_error(cudaFuncSetAttribute(k_zmarch_batch<CG>,
				cudaFuncAttributeMaxDynamicSharedMemorySize, CG::SMEM),
				"cudaFuncSetAttribute(k_zmarch_batch)");
	if (rc0) return rc0;
	// one z-chunk for the batch: the longest (fewest halo re-reads) that still gives at least
	// four waves of resident CTAs over all shots
	int per_sm = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_zmarch_batch<CF>, CF::NT, CF::SMEM);
	const int64_t resident = (int64_t)(per_sm > 0 ? per_sm : 1) * num_sms();
	int chunk = 128;
	for (; chunk > 16; chunk /= 2) {
		int64_t total = 0;
		for (int i = 0; i < b->nshot; i++) {
			const b200_layout* l = &shots[i].lay;
			const int64_t x0 = l->s1 / CF::VX * CF::VX;
			total += ((l->e1 + 1 - x0 + CF::TX - 1) / CF::TX) * ((l->e2 - l->s2 + CF::TY) / CF::TY) *
			         ((l->e3 - l->s3 + chunk) / chunk);
		}
		if (total >= 4 * resident) break;
	}
	int cta = 0;
	for (int i = 0; i < b->nshot; i++) {
		const b200_shot& sh = shots[i];
		const b200_layout* lay = &sh.lay;
		ZShot z;
		std::memset(&z, 0, sizeof(z));
		ZArgs<float>& a = z.a;
		a.n1 = lay->n1;
		a.n12 = lay->n1 * lay->n2;
		a.x_start = (int)(lay->s1 / CF::VX) * CF::VX;
		a.s1 = (int)lay->s1; a.e1 = (int)lay->e1;
		a.s2 = (int)lay->s2; a.e2 = (int)lay->e2;
		a.s3 = (int)lay->s3; a.e3 = (int)lay->e3;
		a.inv2_1 = (float)sh.inv2[0];
		a.inv2_2 = (float)sh.inv2[1];
		a.inv2_3 = (float)sh.inv2[2];
		a.coef_scale = 1.0f;
		a.timeout_ns = 2000000000ull;
		if (int rc = device_error_word(&a.err)) return rc;
		a.g1 = sh.sponge[0];
		a.g2 = sh.sponge[1];
		a.g3 = sh.sponge[2];
		a.kscale = (float)(-1.0 / (dt * dt));
		{
			const int64_t sz = sh.src / (lay->n1 * lay->n2), sr = sh.src - sz * lay->n1 * lay->n2;
			a.src_z = (int)sz;
			a.src_y = (int)(sr / lay->n1);
			a.src_x = (int)(sr - (sr / lay->n1) * lay->n1);
			a.src_amp = sh.amp;
			a.wavelet = sh.wavelet;
		}
		z.ntx = (a.e1 + 1 - a.x_start + CF::TX - 1) / CF::TX;
		z.nty = (a.e2 - a.s2 + 1 + CF::TY - 1) / CF::TY;
		const int nz = a.e3 - a.s3 + 1;
		a.nz_chunk = nz < chunk ? nz : chunk;
		z.nzc = (nz + a.nz_chunk - 1) / a.nz_chunk;
		z.cta_begin = cta;
		cta += z.ntx * z.nty * z.nzc;
		const int64_t field = lay->n1 * lay->n2 * lay->n3;
		// forward: u = wave, p0 = wave (p[n-1]), p1 = coef, out = wave
		ZShot f = z;
		f.a.out = sh.wave;
		f.a.out_slot_stride = field;
		int rc = make_map_slots(&f.tm[0], sh.wave, lay, b->nslot, CF::BX, CF::BY);
		if (!rc) rc = make_map_slots(&f.tm[1], sh.wave, lay, b->nslot, CF::TX, CF::TY);
		if (!rc) rc = make_map_slots(&f.tm[2], sh.coef, lay, 1, CF::TX, CF::TY);
		if (!rc) f.tm[3] = f.tm[2];
		if (rc) return rc;
		fwd.push_back(f);
		if (b->has_adj) {
			ZShot w = z;
			w.a.out = sh.adj;
			w.a.out_slot_stride = field;
			rc = make_map_slots(&w.tm[0], sh.adj, lay, 2, CF::BX, CF::BY);
			if (!rc) rc = make_map_slots(&w.tm[1], sh.adj, lay, 2, CF::TX, CF::TY);
			if (!rc) w.tm[2] = f.tm[2];
			if (!rc) w.tm[3] = f.tm[2];
			if (rc) return rc;
			adj.push_back(w);
		}
		if (b->has_grad) {
			// gradient: u = wave (p[n]), p0 = adj (w[n+1]), p1 = coef, p2 = grad, out = grad
			ZShot g = z;
			g.a.out = sh.grad;
			g.a.out_slot_stride = 0;
			g.tm[0] = f.tm[0];
			rc = make_map_slots(&g.tm[1], sh.adj, lay, 2, CF::TX, CF::TY);
			if (!rc) g.tm[2] = f.tm[2];
			if (!rc) rc = make_map_slots(&g.tm[3], sh.grad, lay, 1, CF::TX, CF::TY);
			if (rc) return rc;
			grad.push_back(g);
		}
	}
	b->ctas = cta;
	b->interleave = true;
	for (int i = 1; i < b->nshot; i++)
		if (fwd[i].ntx != fwd[0].ntx || fwd[i].nty != fwd[0].nty || fwd[i].nzc != fwd[0].nzc ||
				fwd[i].a.nz_chunk != fwd[0].a.nz_chunk)
			b->interleave = false;
	b->smem[0] = CF::SMEM;
	b->smem[1] = CF::SMEM;
	b->smem[2] = CG::SMEM;
	return B200_OK;
}

template <int R, int MODE>
int launch_pass(const b200_batch* b, const ZShot* table, int su, int sp0, int sout, int step,
		cudaStream_t s)
{
	using Cfg = ModelCfg<R, MODE>;
	k_zmarch_batch<Cfg><<<b->ctas, Cfg::NT, Cfg::SMEM, s>>>(table, b->nshot, su, sp0, sout, step,
			b->interleave ? 1 : 0);
	return check_launch("k_zmarch_batch");
}

int dispatch_pass(const b200_batch* b, int mode, const ZShot* table, int su, int sp0, int sout,
		int step, cudaStream_t s)
{
	return dispatch_order(2 * b->R, [&](auto rt) {
		constexpr int R = decltype(rt)::value;
		if (mode == MODE_GRAD) return launch_pass<R, MODE_GRAD>(b, table, su, sp0, sout, -1, s);
		return launch_pass<R, MODE_MODEL>(b, table, su, sp0, sout, step, s);
	});
}

dim3 rec_grid(const b200_batch* b)
{
	return dim3((unsigned)b->nshot, (unsigned)((b->max_nrec + kRecThreads - 1) / kRecThreads));
}

int check_shot(const b200_shot& sh, int order, bool need_adj, bool need_grad, int i)
{
	const b200_layout* lay = &sh.lay;
	if (int rc = check_layout(lay)) return rc;
	if (lay->dim != 3) return set_error(B200_ERR_UNSUPPORTED, "shot %d: the modelling engine is 3-D", i);
	if (lay->halo != order / 2) return set_error(B200_ERR_ARG, "shot %d: halo %d for order %d", i, lay->halo, order);
	if ((lay->n1 * 4) % 16) return set_error(B200_ERR_ARG, "shot %d: n1 * 4 bytes not a multiple of 16", i);
	if (!sh.wave || !sh.coef || !sh.sponge[0] || !sh.sponge[1] || !sh.sponge[2] || !sh.wavelet)
		return set_error(B200_ERR_ARG, "shot %d: NULL wave/coef/sponge/wavelet", i);
	if ((reinterpret_cast<uintptr_t>(sh.wave) | reinterpret_cast<uintptr_t>(sh.coef)) % 16)
		return set_error(B200_ERR_ARG, "shot %d: grids must be 16-byte aligned", i);
	if (sh.nrec < 0 || (sh.nrec > 0 && (!sh.rec || !sh.traces)))
		return set_error(B200_ERR_ARG, "shot %d: receivers", i);
	const int64_t np = lay->n1 * lay->n2 * lay->n3;
	if (sh.src < 0 || sh.src >= np) return set_error(B200_ERR_ARG, "shot %d: source index", i);
	if (need_adj && (!sh.adj || !sh.dobs || reinterpret_cast<uintptr_t>(sh.adj) % 16))
		return set_error(B200_ERR_ARG, "shot %d: adjoint needs adj (16-byte aligned) and dobs", i);
	if (need_grad && (!sh.grad || reinterpret_cast<uintptr_t>(sh.grad) % 16))
		return set_error(B200_ERR_ARG, "shot %d: gradient needs grad (16-byte aligned)", i);
	return B200_OK;
}

}  // namespace

extern "C" {

int b200_batch_create(b200_batch** out, int order, int nslot, int nshot, const b200_shot* shots,
		double dt, int flags)
{
	if (!out) return set_error(B200_ERR_ARG, "batch is NULL");
	*out = nullptr;
	if (int rc = check_order(order)) return rc;
	if (nshot < 1 || !shots) return set_error(B200_ERR_ARG, "no shots");
	if (nslot < 2) return set_error(B200_ERR_ARG, "nslot %d < 2", nslot);
	if (!(dt > 0.0)) return set_error(B200_ERR_ARG, "dt %g", dt);
	const bool adj = flags & B200_BATCH_ADJOINT, grad = flags & B200_BATCH_GRADIENT;
	for (int i = 0; i < nshot; i++)
		if (int rc = check_shot(shots[i], order, adj || grad, grad, i)) return rc;
	b200_batch* b = new b200_batch;
	b->R = order / 2;
	b->nshot = nshot;
	b->nslot = nslot;
	b->has_adj = adj || grad;
	b->has_grad = grad;
	b->lay0 = shots[0].lay;
	b->kscale = (float)(-1.0 / (dt * dt));
	b->same_grid = true;
	for (int i = 1; i < nshot; i++)
		if (std::memcmp(&shots[i].lay, &shots[0].lay, sizeof(b200_layout)) != 0) b->same_grid = false;
	std::vector<ZShot> fwd, ad, gr;
	int rc = dispatch_order(order, [&](auto rt) {
		constexpr int R = decltype(rt)::value;
		return batch_tables<R>(b, shots, dt, fwd, ad, gr);
	});
	std::vector<MShot> ms(nshot);
	for (int i = 0; i < nshot && !rc; i++) {
		const b200_shot& sh = shots[i];
		MShot& m = ms[i];
		m.wave = sh.wave;
		m.adj = sh.adj;
		m.field = sh.lay.n1 * sh.lay.n2 * sh.lay.n3;
		m.coef = sh.coef;
		m.g1 = sh.sponge[0];
		m.g2 = sh.sponge[1];
		m.g3 = sh.sponge[2];
		m.n1 = sh.lay.n1;
		m.n12 = sh.lay.n1 * sh.lay.n2;
		m.src = sh.src;
		m.amp = sh.amp;
		m.wavelet = sh.wavelet;
		m.nrec = sh.nrec;
		m.rec = sh.rec;
		m.traces = sh.traces;
		m.dobs = sh.dobs;
		if (sh.nrec > b->max_nrec) b->max_nrec = sh.nrec;
	}
	auto upload = [&](auto** dst, const auto& v) -> int {
		if (v.empty()) return B200_OK;
		const size_t bytes = sizeof(v[0]) * v.size();
		int r = cuda_error(cudaMalloc(reinterpret_cast<void**>(dst), bytes), "cudaMalloc(batch)");
		if (!r) r = cuda_error(cudaMemcpy(*dst, v.data(), bytes, cudaMemcpyHostToDevice), "cudaMemcpy(batch)");
		return r;
	};
	if (!rc) rc = upload(&b->d_fwd, fwd);
	if (!rc) rc = upload(&b->d_adj, ad);
	if (!rc) rc = upload(&b->d_grad, gr);
	if (!rc) rc = upload(&b->d_m, ms);
	if (rc) {
		b200_batch_destroy(b);
		return rc;
	}
	*out = b;
	return B200_OK;
}

int b200_batch_destroy(b200_batch* b)
{
	if (!b) return B200_OK;
	cudaFree(b->d_fwd);
	cudaFree(b->d_adj);
	cudaFree(b->d_grad);
	cudaFree(b->d_m);
	delete b;
	return B200_OK;
}

int b200_batch_forward_step(b200_batch* b, int n, int scur, int sprev, int sout, void* stream)
{
	if (!b) return set_error(B200_ERR_ARG, "batch is NULL");
	if (scur < 0 || scur >= b->nslot || sprev < 0 || sprev >= b->nslot || sout < 0 ||
			sout >= b->nslot || sout == scur)
		return set_error(B200_ERR_ARG, "forward slots %d %d %d of %d", scur, sprev, sout, b->nslot);
	if (n < 0) return set_error(B200_ERR_ARG, "step %d", n);
	cudaStream_t s = as_stream(stream);
	if (int rc = dispatch_pass(b, MODE_MODEL, b->d_fwd, scur, sprev, sout, n, s)) return rc;
	if (b->max_nrec == 0) return B200_OK;
	k_model_record<<<rec_grid(b), kRecThreads, 0, s>>>(b->d_m, n, sout);
	return check_launch("k_model_record");
}

int b200_batch_adjoint_step(b200_batch* b, int k, int scur, void* stream)
{
	if (!b || !b->has_adj) return set_error(B200_ERR_ARG, "batch without adjoint wavefields");
	if (scur < 0 || scur > 1 || k < 1) return set_error(B200_ERR_ARG, "adjoint step %d slot %d", k, scur);
	cudaStream_t s = as_stream(stream);
	const int o = 1 - scur;
	if (int rc = dispatch_pass(b, MODE_MODEL, b->d_adj, scur, o, o, -1, s)) return rc;
	if (b->max_nrec == 0) return B200_OK;
	k_model_residual<<<rec_grid(b), kRecThreads, 0, s>>>(b->d_m, k, o);
	return check_launch("k_model_residual");
}

int b200_batch_gradient(b200_batch* b, int swave, int sadj, void* stream)
{
	if (!b || !b->has_grad) return set_error(B200_ERR_ARG, "batch without gradient");
	if (swave < 0 || swave >= b->nslot || sadj < 0 || sadj > 1)
		return set_error(B200_ERR_ARG, "gradient slots %d %d", swave, sadj);
	return dispatch_pass(b, MODE_GRAD, b->d_grad, swave, sadj, 0, -1, as_stream(stream));
}

int b200_batch_survey_gradient(b200_batch* b, int n, int snext, int scur, int sprev, int sadj,
		float* grad, void* stream)
{
	if (!b || !b->has_adj) return set_error(B200_ERR_ARG, "batch without adjoint wavefields");
	if (!b->same_grid) return set_error(B200_ERR_UNSUPPORTED, "survey gradient: the shots are on different grids");
	if (!grad || reinterpret_cast<uintptr_t>(grad) % 4) return set_error(B200_ERR_ARG, "grad");
	for (int sl : {snext, scur, sprev})
		if (sl < 0 || sl >= b->nslot) return set_error(B200_ERR_ARG, "survey gradient slot %d of %d", sl, b->nslot);
	if (snext == scur || scur == sprev || snext == sprev)
		return set_error(B200_ERR_ARG, "survey gradient slots must differ");
	if (sadj < 0 || sadj > 1 || n < 0) return set_error(B200_ERR_ARG, "survey gradient step %d adjoint slot %d", n, sadj);
	const b200_layout& l = b->lay0;
	SurveyArgs a;
	a.n1 = l.n1;
	a.n12 = l.n1 * l.n2;
	a.field = l.n1 * l.n2 * l.n3;
	a.s1 = (int)l.s1; a.e1 = (int)l.e1;
	a.s2 = (int)l.s2; a.e2 = (int)l.e2;
	a.s3 = (int)l.s3; a.e3 = (int)l.e3;
	a.x0 = a.s1 / 4 * 4;
	a.nvx = (a.e1 - a.x0) / 4 + 1;
	a.n = n;
	a.snext = snext; a.scur = scur; a.sprev = sprev; a.sadj = sadj;
	a.nshot = b->nshot;
	a.kscale = b->kscale;
	a.grad = grad;
	if ((l.n1 % 4) != 0) return set_error(B200_ERR_ARG, "survey gradient: n1 not a multiple of 4");
	// the vectors of a row must stay inside it: the last one ends at most at n1 - 1
	if (a.x0 + 4 * a.nvx > l.n1) return set_error(B200_ERR_ARG, "survey gradient: row vectors");
	const int64_t items = (int64_t)(l.e2 - l.s2 + 1) * (l.e3 - l.s3 + 1) * a.nvx;
	const int64_t cap = (int64_t)num_sms() * 8;
	const int64_t want = (items + 255) / 256;
	const int blocks = (int)(want < cap ? want : cap);
	k_survey_gradient<<<blocks, 256, 0, as_stream(stream)>>>(b->d_m, a);
	return check_launch("k_survey_gradient");
}

int b200_batch_info(const b200_batch* b, int* ctas_per_pass)
{
	if (!b || !ctas_per_pass) return set_error(B200_ERR_ARG, "NULL");
	*ctas_per_pass = b->ctas;
	return B200_OK;
}

}  // extern "C"
