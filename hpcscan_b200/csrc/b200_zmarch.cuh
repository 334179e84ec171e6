// 3-D z-marching stencil kernels for sm_100a: FD_D2_N1/N2/N3, FD_LAPLACIAN and
// computePressureWithFD (reference src/grid.cpp:3232-5113; the reference's best GPU form
// of the same idea is src/grid_Cuda_Optim.cu:1085-2160, plain SIMT with a __shared__ tile
// and per-plane __syncthreads).
//
// Design (one CTA = one TX x TY tile of (i1, i2) marching over a chunk of i3 planes):
//  * a producer warp streams the planes of the input grid into a ring of shared-memory
//    tiles with TMA (cp.async.bulk.tensor.3d, no cluster multicast): plane tile with the
//    x/y halos the operator needs, plus, for the pressure update, the prn and coef tiles
//    of the output plane. Full/empty mbarriers hand the slots between producer and
//    consumers; the ring runs PF planes ahead of the consumers;
//  * consumer threads own VX consecutive i1 points (16 bytes, one vector shared-memory
//    load) of VY consecutive rows and keep the 2R+1 values of each point along i3 in a
//    register queue, so every plane is read from HBM once (plus the chunk's z-halo);
//  * the x/y derivatives read the staged tile of the centre plane, which the ring keeps
//    resident for R iterations after it arrives;
//  * every operation is a separately rounded IEEE operation in the reference's order,
//    so the results are bit-identical to the reference CPU path.
// MODE_STEP fuses applyBoundaryCondition(prc, ANTI_MIRROR) into the pressure update: every
// value the stencils read is the value after the boundary condition, built from the raw
// tile (halos from mirror points in the same tile, boundary lines and planes as zero, z-halo
// planes loaded from their mirror planes). In a CTA whose planes need it, the producer warp
// rebuilds each plane in shared memory between the copy's arrival and the consumers' release,
// so the consumers run the pressure update's code unchanged. The kernel never writes prc, so
// every CTA reads the raw values; the boundary planes' zeros are written by a separate launch
// afterwards.
// Every wait on an mbarrier is bounded by a time limit: a CTA that gives up records an
// error flag (read by b200_device_status) and returns after its issued copies have landed.
//
// This header holds the kernel template and its launcher; b200_zmarch_{pressure,laplacian,
// d2}.cu instantiate them per operator and b200_stencil_zmarch.cu dispatches and tunes.
#pragma once

#include <cuda.h>

#include <cstring>
#include <utility>

#include "b200_stencil.cuh"

namespace b200 {

namespace {

// ---- PTX wrappers -------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
	return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
			: "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
			"r"(bytes)
			: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
	uint32_t ok;
	asm volatile(
			"{\n\t.reg .pred p;\n\t"
			"mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
			"selp.u32 %0, 1, 0, p;\n\t}"
			: "=r"(ok)
			: "r"(smem_u32(bar)), "r"(parity)
			: "memory");
	return ok != 0;
}

// Non-blocking: has the mbarrier phase of the given parity completed?
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity)
{
	uint32_t ok;
	asm volatile(
			"{\n\t.reg .pred p;\n\t"
			"mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
			"selp.u32 %0, 1, 0, p;\n\t}"
			: "=r"(ok)
			: "r"(smem_u32(bar)), "r"(parity)
			: "memory");
	return ok != 0;
}

// Orders this thread's earlier generic writes to shared memory before later accesses of the
// same bytes by the async proxy (the TMA copies that refill a slot).
__device__ __forceinline__ void fence_proxy_async_smem()
{
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ uint64_t global_timer_ns()
{
	uint64_t t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

// Wait for the completion of the mbarrier phase of the given parity, at most until
// `deadline` (global timer, ns). Returns false when the time ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t deadline)
{
	if (mbar_try_wait(bar, parity)) return true;
	for (uint32_t n = 1;; ++n) {
		if (mbar_try_wait(bar, parity)) return true;
		if ((n & 63u) == 0 && global_timer_ns() > deadline) return false;
	}
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* tm, int x, int y, int z,
		uint64_t* bar)
{
	asm volatile(
			"cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
			" [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
			"l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
			: "memory");
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* tm, int x, int y, int z,
		int w, uint64_t* bar)
{
	asm volatile(
			"cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
			" [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
			"l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
			: "memory");
}

// A tile load of a 3-D grid, or of slot `w` of a slotted (4-D) grid.
template <bool SLOTS>
__device__ __forceinline__ void tma_tile(void* dst, const CUtensorMap* tm, int x, int y, int z,
		int w, uint64_t* bar)
{
	if constexpr (SLOTS) tma_load_4d(dst, tm, x, y, z, w, bar);
	else tma_load_3d(dst, tm, x, y, z, bar);
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* tm)
{
	asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tm)) : "memory");
}

// ---- vector shared-memory loads (16 bytes) converted to the compute type --------------------------
template <typename S, typename C, int N>
__device__ __forceinline__ void lds_vec(const S* p, C* out)
{
	static_assert(N * sizeof(S) % 16 == 0 || N * sizeof(S) == 8, "vector of 8 or 16-byte multiples");
	if constexpr (N * sizeof(S) == 8) {
		const uint2 raw = *reinterpret_cast<const uint2*>(p);
		const S* v = reinterpret_cast<const S*>(&raw);
#pragma unroll
		for (int i = 0; i < N; i++) out[i] = Storage<S>::load(v[i]);
	} else {
#pragma unroll
		for (int b = 0; b < N * (int)sizeof(S) / 16; b++) {
			const uint4 raw = reinterpret_cast<const uint4*>(p)[b];
			const S* v = reinterpret_cast<const S*>(&raw);
#pragma unroll
			for (int i = 0; i < 16 / (int)sizeof(S); i++)
				out[b * (16 / sizeof(S)) + i] = Storage<S>::load(v[i]);
		}
	}
}

// The register queue along i3: the compute type per point, or, for 16-bit storage, the stored
// values two per register (half the registers; converted to FP32 where the stencil uses them).
template <typename S, typename C> struct ZQueueF {
	using T = C;
	static constexpr int W = 1;
	static __device__ __forceinline__ C get(const T* row, int e) { return row[e]; }
	static __device__ __forceinline__ float2 get2(const T* row, int e)
	{
		return make_float2((float)row[e], (float)row[e + 1]);
	}
	template <int N>
	static __device__ __forceinline__ void push(const S* p, T* row) { lds_vec<S, C, N>(p, row); }
};
template <typename S, typename C> struct ZQueue : ZQueueF<S, C> {};
template <> struct ZQueue<__half, float> {
	using T = __half2;
	static constexpr int W = 2;
	static __device__ __forceinline__ float get(const T* row, int e)
	{
		return (e & 1) ? __high2float(row[e >> 1]) : __low2float(row[e >> 1]);
	}
	static __device__ __forceinline__ float2 get2(const T* row, int e) { return __half22float2(row[e >> 1]); }
	template <int N>
	static __device__ __forceinline__ void push(const __half* p, T* row)
	{
#pragma unroll
		for (int b = 0; b < N / 8; b++) {
			const uint4 raw = reinterpret_cast<const uint4*>(p)[b];
			const T* v = reinterpret_cast<const T*>(&raw);
#pragma unroll
			for (int i = 0; i < 4; i++) row[b * 4 + i] = v[i];
		}
	}
};
template <> struct ZQueue<__nv_bfloat16, float> {
	using T = __nv_bfloat162;
	static constexpr int W = 2;
	static __device__ __forceinline__ float get(const T* row, int e)
	{
		return (e & 1) ? __high2float(row[e >> 1]) : __low2float(row[e >> 1]);
	}
	static __device__ __forceinline__ float2 get2(const T* row, int e) { return __bfloat1622float2(row[e >> 1]); }
	template <int N>
	static __device__ __forceinline__ void push(const __nv_bfloat16* p, T* row)
	{
#pragma unroll
		for (int b = 0; b < N / 8; b++) {
			const uint4 raw = reinterpret_cast<const uint4*>(p)[b];
			const T* v = reinterpret_cast<const T*>(&raw);
#pragma unroll
			for (int i = 0; i < 4; i++) row[b * 4 + i] = v[i];
		}
	}
};

constexpr int round_up(int v, int m) { return (v + m - 1) / m * m; }

// f(integral_constant<int, 0>) .. f(integral_constant<int, N - 1>), in order
template <typename F, int... I>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, I...>)
{
	(f(std::integral_constant<int, I>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void static_for(F&& f)
{
	static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// ---- kernel configuration -----------------------------------------------------------------------
template <typename S, int R_, int MODE_, int TX_, int TY_, int VY_, int PF_, bool EXACT_ = true,
		int MINB_ = 0, typename SC_ = S, int UQ_ = 0, int VXB_ = 16>
struct ZCfg {
	using Stor = S;
	using CoefStor = SC_;                                    // coef storage (FP32 with 16-bit waves)
	using C = typename Storage<S>::C;
	static constexpr bool EXACT = EXACT_;
	static constexpr int R = R_;
	static constexpr int MODE = MODE_;
	static constexpr int TX = TX_, TY = TY_, VY = VY_, PF = PF_;
	static constexpr int VA = 16 / sizeof(S);                // 16 bytes: the TMA alignment unit
	static constexpr int VX = VXB_ / (int)sizeof(S);         // points per thread and row
	static_assert((VXB_ == 16 || VXB_ == 8) && VX >= 1, "thread vectors of 8 or 16 bytes");
	// 16-byte vectors of 16-bit values keep the z queue packed (ZQueue); 8-byte ones keep it in
	// the compute type (ZQueueF): each value converted once, at its push
	static constexpr bool QPACK = VXB_ == 16;
	static constexpr bool BC = (MODE == MODE_STEP);          // anti-mirror BC fused in
	// operators of the Laplacian (the x, y and z stencils) and the staggered first derivatives
	static constexpr bool LAP = (MODE == MODE_LAPLACIAN || MODE == MODE_PRESSURE ||
	                             MODE == MODE_STEP || MODE == MODE_MODEL || MODE == MODE_GRAD);
	static constexpr bool D1 = (MODE == MODE_D1_AXIS1 || MODE == MODE_D1_AXIS2 ||
	                            MODE == MODE_D1_AXIS3);
	static constexpr bool XH = (MODE == MODE_D2_AXIS1 || MODE == MODE_D1_AXIS1 || LAP);
	static constexpr bool YH = (MODE == MODE_D2_AXIS2 || MODE == MODE_D1_AXIS2 || LAP);
	static constexpr bool ZQ = (MODE == MODE_D2_AXIS3 || MODE == MODE_D1_AXIS3 || LAP);
	// z stencil only: a plane is needed only while it is pushed into the register queue, so its
	// slot is released on arrival and the whole ring but one slot stays in flight
	static constexpr bool ZONLY = ZQ && !XH && !YH && !BC;
	static constexpr bool P = (MODE == MODE_PRESSURE || MODE == MODE_STEP || MODE == MODE_MODEL ||
	                           MODE == MODE_GRAD);
	// pointwise tiles of the output plane: prn + coef (pressure, model), w + C + g (gradient)
	static constexpr int NPT = (MODE == MODE_GRAD) ? 3 : 2;
	static constexpr int R4 = XH ? round_up(R, VA) : 0;     // x halo, whole 16-byte vectors
	static constexpr int RY = YH ? R : 0;
	static constexpr int RZ = ZQ ? R : 0;
	// planes per pass of the z loop (0: four, except two where four would spill registers: the
	// pressure update, fused step and modelling passes outside R = 3..6; four measured 1.3 %
	// faster than two for the pressure update at 512^3 O8 on B200)
	static constexpr int UQ = !ZQ ? 1 : UQ_ > 0 ? UQ_
	                        : ((MODE == MODE_PRESSURE || MODE == MODE_STEP || MODE == MODE_MODEL ||
	                            MODE == MODE_GRAD) && (R < 3 || R > 6))
	                                  ? 2 : 4;
	static constexpr int BX = TX + 2 * R4;
	static constexpr int BY = TY + 2 * RY;
	static constexpr int NSU = (ZONLY && 2 * PF + 4 > RZ + 1 + PF) ? 2 * PF + 4
	                                                               : RZ + 1 + PF;   // input-tile ring
	static constexpr int NSP = P ? 1 + PF : 1;               // pointwise-tile ring
	static constexpr int U_BYTES = BX * BY * (int)sizeof(S);
	static constexpr int U_STRIDE = round_up(U_BYTES, 128);
	static constexpr int PT_BYTES = TX * TY * (int)sizeof(S);
	static constexpr int PT_STRIDE = round_up(PT_BYTES, 128);
	static constexpr int CT_BYTES = TX * TY * (int)sizeof(SC_);
	static constexpr int CT_STRIDE = round_up(CT_BYTES, 128);
	// one slot of the pointwise ring: output-plane tile, coef tile, third tile (gradient)
	static constexpr int SLOT_P = PT_STRIDE + CT_STRIDE + (NPT > 2 ? PT_STRIDE : 0);
	static constexpr int SLOT_TX = PT_BYTES + CT_BYTES + (NPT > 2 ? PT_BYTES : 0);
	static constexpr int NTX = TX / VX;
	static constexpr int NC = NTX * (TY / VY);              // consumer threads
	static constexpr int NWC = NC / 32;                      // consumer warps
	static constexpr int NT = NC + 32;                       // + one producer warp
	// fused boundary condition: the producer's patch lists (phase 1: halo points from mirror
	// points, at most R columns and R rows on each side of the tile; phase 2: boundary lines)
	static constexpr int NL1 = BC ? 2 * R * BY + 2 * R * BX : 0;
	static constexpr int NL2 = BC ? 2 * BY + 2 * BX : 0;
	static_assert(!BC || (PF >= 2 && BX * BY < 0xFFFF), "fused step: patch lag and 16-bit offsets");
	static constexpr int SMEM = 128 + NSU * U_STRIDE + (P ? NSP * SLOT_P : 0) +
	                            (2 * NSU + NSP) * 8 + (BC ? NSU * 8 + (NL1 + NL2) * 4 : 0);
	// CTAs per SM the launch bounds ask for (registers follow: an SM has four sub-partitions
	// of 16K registers and spreads a CTA's warps over them). Two CTAs per SM for R <= 4 with
	// 8-warp CTAs; wider stencils keep their longer z queue in registers at one CTA per SM.
	static constexpr int MINB = MINB_ > 0 ? MINB_ : ((NT <= 256 && R <= 4) ? 2 : 1);
	static_assert(TX % VA == 0 && TY % VY == 0 && NC % 32 == 0, "tile shape");
	static_assert((MODE != MODE_MODEL && MODE != MODE_GRAD) || std::is_same_v<S, float>,
			"the modelling engine computes in FP32");
	static_assert(BX <= 256 && BY <= 256, "TMA box limit");
	static_assert((BX * sizeof(S)) % 16 == 0 && (TX * sizeof(S)) % 16 == 0, "TMA inner extent");
	static_assert((TX * sizeof(SC_)) % 16 == 0, "TMA inner extent (coef)");
};

template <typename C>
struct ZArgs {
	void* out;                 // w, or prn for the pressure update
	int64_t n1, n12;
	int x_start;               // first tile's i1 (16-byte aligned index)
	int s1, e1, s2, e2, s3, e3;
	int nz_chunk;
	C inv2_1, inv2_2, inv2_3;
	float coef_scale;
	uint64_t timeout_ns;
	unsigned int* err;         // device error word (b200_device_status)
	// modelling engine (MODE_MODEL, MODE_GRAD): damping tables G = g1 g2 g3, gradient factor
	const float* g1;
	const float* g2;
	const float* g3;
	float kscale;
	int64_t out_slot_stride;   // elements between slots of the output grid
	int src_x, src_y, src_z;   // point source of MODE_MODEL (added when the step is >= 0)
	float src_amp;
	const float* wavelet;
};


// Position in a ring of N slots: the slot index and the parity of the slot's use count
// (the mbarrier phase parity), advanced without integer division.
template <int N>
struct Ring {
	int slot = 0;
	uint32_t phase = 0;
	__device__ __forceinline__ void advance()
	{
		if (++slot == N) {
			slot = 0;
			phase ^= 1u;
		}
	}
};

// The producer warp of a fused-step CTA whose planes need the boundary condition. Lane 0 issues
// the copies as the plain producer does, except that they land on land_u; the warp rebuilds
// each landed plane in its slot (the values applyBoundaryCondition(ANTI_MIRROR) leaves in prc,
// faces in the reference's order I1, I2, I3: src/grid.cpp:3065-3229) and releases it to the
// consumers on full_u (lane 0 arrives once the warp's writes are done). One loop does both:
// copies are issued as soon as their slots are free (the plain producer's depth) and planes
// are released as soon as they land, so neither waits behind the other.
template <class Cfg, bool SLOTS>
__device__ __forceinline__ void step_patch_producer(const CUtensorMap* tm_u,
		const CUtensorMap* tm_p0, const CUtensorMap* tm_p1, const ZArgs<typename Cfg::C>& a,
		typename Cfg::Stor* su, unsigned char* sp, uint64_t* bars, int tile_x0, int tile_y0, int z0,
		int J, bool near, int slot_u, int slot_p0, uint64_t deadline)
{
	using S = typename Cfg::Stor;
	using C = typename Cfg::C;
	static_assert(Cfg::NPT == 2, "fused step: prn and coef tiles");
	constexpr int R = Cfg::R, R4 = Cfg::R4, RY = Cfg::RY, RZ = Cfg::RZ, TX = Cfg::TX;
	constexpr int BX = Cfg::BX, BY = Cfg::BY, NSU = Cfg::NSU, NSP = Cfg::NSP;
	constexpr int UE = Cfg::U_STRIDE / (int)sizeof(S);
	constexpr unsigned FULL = 0xffffffffu;
	constexpr uint32_t NEG_ZERO = 0xFFFFu;     // phase-1 source that stands for a zeroed point
	uint64_t* full_u = bars;
	uint64_t* empty_u = bars + NSU;
	uint64_t* empty_p = bars + 2 * NSU;
	uint64_t* land_u = bars + 2 * NSU + NSP;
	uint32_t* list1 = reinterpret_cast<uint32_t*>(bars + 3 * NSU + NSP);
	uint32_t* list2 = list1 + Cfg::NL1;
	const int lane = threadIdx.x & 31;
	const int xs = tile_x0 - R4, xe = tile_x0 + TX + R4 - 1;
	const int ys = tile_y0 - RY, ye = tile_y0 + Cfg::TY + RY - 1;
	if (lane == 0) {
		prefetch_tmap(tm_u);
		prefetch_tmap(tm_p0);
		prefetch_tmap(tm_p1);
	}

	// the tile's patch lists, the same for every inner plane: phase 1 writes halo points from
	// their mirror points ((dst << 16) | src; src NEG_ZERO writes -0), phase 2 zeroes the points
	// of the boundary lines
	int n1 = 0, n2 = 0;
	if (near) {
		for (int base = 0; base < Cfg::NL1; base += 32) {
			const int idx = base + lane;
			uint32_t e = 0;
			bool use = false;
			if (idx < 2 * R * BY) {
				// i1 halos: -(mirror), before any face zeroes a line
				const int side = idx / (R * BY), rem = idx % (R * BY);
				const int kk = rem / BY + 1, r = rem % BY;
				const int y = ys + r;
				const int ch = (side ? a.e1 + kk : a.s1 - kk) - xs;
				const int cm = (side ? a.e1 - kk : a.s1 + kk) - xs;
				use = y >= a.s2 && y <= a.e2 && ch >= 0 && ch < BX && cm >= 0 && cm < BX;
				e = (uint32_t)(r * BX + ch) << 16 | (uint32_t)(r * BX + cm);
			} else if (idx < Cfg::NL1) {
				// i2 halos: -(mirror), after the i1 faces zeroed their boundary columns
				const int i2 = idx - 2 * R * BY;
				const int side = i2 / (R * BX), rem = i2 % (R * BX);
				const int kk = rem / BX + 1, c = rem % BX;
				const int x = xs + c;
				const int rh = (side ? a.e2 + kk : a.s2 - kk) - ys;
				const int rm = (side ? a.e2 - kk : a.s2 + kk) - ys;
				use = x >= a.s1 && x <= a.e1 && rh >= 0 && rh < BY && rm >= 0 && rm < BY;
				e = (uint32_t)(rh * BX + c) << 16 |
				    ((x == a.s1 || x == a.e1) ? NEG_ZERO : (uint32_t)(rm * BX + c));
			}
			const unsigned m = __ballot_sync(FULL, use);
			if (use) list1[n1 + __popc(m & ((1u << lane) - 1u))] = e;
			n1 += __popc(m);
		}
		for (int base = 0; base < Cfg::NL2; base += 32) {
			const int idx = base + lane;
			uint32_t e = 0;
			bool use = false;
			if (idx < 2 * BY) {                        // boundary columns s1, e1
				const int side = idx / BY, r = idx % BY;
				const int y = ys + r, c = (side ? a.e1 : a.s1) - xs;
				use = y >= a.s2 && y <= a.e2 && c >= 0 && c < BX;
				e = (uint32_t)(r * BX + c);
			} else if (idx < Cfg::NL2) {               // boundary rows s2, e2
				const int i2 = idx - 2 * BY;
				const int side = i2 / BX, c = i2 % BX;
				const int x = xs + c, r = (side ? a.e2 : a.s2) - ys;
				use = x >= a.s1 && x <= a.e1 && r >= 0 && r < BY;
				e = (uint32_t)(r * BX + c);
			}
			const unsigned m = __ballot_sync(FULL, use);
			if (use) list2[n2 + __popc(m & ((1u << lane) - 1u))] = e;
			n2 += __popc(m);
		}
		__syncwarp();
	}
	// the inner points of the tile with its halos: a rectangle (cw x ch from (cx0, cy0))
	const int cx0 = max(xs, a.s1) - xs, cy0 = max(ys, a.s2) - ys;
	const int cw = min(xe, a.e1) - xs - cx0 + 1, ch = min(ye, a.e2) - ys - cy0 + 1;
	const int ninner = (cw > 0 && ch > 0) ? cw * ch : 0;

	// rebuild plane jj (stream index), landed, in its slot and release it to the consumers
	auto patch_plane = [&](int jj) {
		const int slot = jj % NSU;
		S* tw = su + slot * UE;
		const int pl = z0 - RZ + jj;
		bool wrote = false;
		if (pl < a.s3 || pl > a.e3) {
			// z-halo plane, loaded from its mirror plane: minus the mirror after the i1/i2 faces
			// zeroed their lines (only its inner points are read, by the z stencil)
			for (int r = cy0; r < cy0 + ch; ++r) {
				const int y = ys + r;
				const bool yline = y == a.s2 || y == a.e2;
				for (int c = cx0 + lane; c < cx0 + cw; c += 32) {
					const int x = xs + c;
					S& v = tw[r * BX + c];
					v = Storage<S>::store((yline || x == a.s1 || x == a.e1) ? -C(0) : -Storage<S>::load(v));
				}
			}
			wrote = ninner > 0;
		} else {
			for (int i = lane; i < n1; i += 32) {
				const uint32_t pe = list1[i];
				const uint32_t src = pe & 0xFFFFu;
				const C mv = src == NEG_ZERO ? C(0) : Storage<S>::load(tw[src]);
				tw[pe >> 16] = Storage<S>::store(-mv);
			}
			__syncwarp();                          // every mirror point read before lines are zeroed
			if (pl == a.s3 || pl == a.e3) {
				// boundary plane: every inner point is zero
				for (int r = cy0; r < cy0 + ch; ++r)
					for (int c = cx0 + lane; c < cx0 + cw; c += 32) tw[r * BX + c] = S(0.0f);
				wrote = true;
			} else {
				for (int i = lane; i < n2; i += 32) tw[list2[i]] = S(0.0f);
				wrote = n1 > 0 || n2 > 0;
			}
		}
		// the patch's writes before the slot is refilled by a copy (the async proxy), and before
		// lane 0's release of the plane (the warp barrier orders them before its arrival)
		if (wrote) fence_proxy_async_smem();
		__syncwarp();
		if (lane == 0) mbar_arrive(&full_u[slot]);
	};

	bool ok = true;
	int issued = 0, patched = 0;
	Ring<NSU> wu;
	Ring<NSP> wp;
	while (patched < J) {
		// every copy whose slots are free (the consumers released their previous use)
		while (issued < J) {
			const int j = issued;
			const bool pw = j >= 2 * RZ;
			bool go = true;
			if (lane == 0) {
				go = (j < NSU || mbar_test(&empty_u[wu.slot], wu.phase ^ 1u)) &&
				     (!pw || j - 2 * RZ < NSP || mbar_test(&empty_p[wp.slot], wp.phase ^ 1u));
				if (go) {
					int plane = z0 - RZ + j;           // z-halo planes come from their mirrors
					if (plane < a.s3) plane = 2 * a.s3 - plane;
					else if (plane > a.e3) plane = 2 * a.e3 - plane;
					uint64_t* bar = &land_u[wu.slot];
					mbar_arrive_expect_tx(bar, Cfg::U_BYTES + (pw ? Cfg::SLOT_TX : 0));
					tma_tile<SLOTS>(su + wu.slot * UE, tm_u, xs, ys, plane, slot_u, bar);
					if (pw) {
						const int o = j - 2 * RZ;
						unsigned char* slot = sp + wp.slot * Cfg::SLOT_P;
						tma_tile<SLOTS>(slot, tm_p0, tile_x0, tile_y0, z0 + o, slot_p0, bar);
						tma_tile<SLOTS>(slot + Cfg::PT_STRIDE, tm_p1, tile_x0, tile_y0, z0 + o, 0, bar);
					}
				}
			}
			if (!__shfl_sync(FULL, go, 0)) break;
			++issued;
			wu.advance();
			if (pw) wp.advance();
		}
		// every issued plane that has landed, oldest first
		while (patched < issued) {
			const uint32_t par = (uint32_t)(patched / NSU) & 1u;
			bool landed = false;
			if (lane == 0) landed = mbar_test(&land_u[patched % NSU], par);
			if (!__shfl_sync(FULL, landed, 0)) break;
			(void)mbar_test(&land_u[patched % NSU], par);   // every lane acquires the copy's bytes
			patch_plane(patched);
			++patched;
		}
		if (patched == J) break;
		// nothing to do: sleep in the barrier unit until the oldest copy lands or, with every
		// issued plane released, until the next slot is free (each wait bounded by the hardware's
		// own time limit; the loop then checks again)
		if (lane == 0) {
			if (patched < issued) {
				(void)mbar_try_wait(&land_u[patched % NSU], (uint32_t)(patched / NSU) & 1u);
			} else if (issued >= NSU && !mbar_test(&empty_u[wu.slot], wu.phase ^ 1u)) {
				(void)mbar_try_wait(&empty_u[wu.slot], wu.phase ^ 1u);
			} else {
				(void)mbar_try_wait(&empty_p[wp.slot], wp.phase ^ 1u);   // the pointwise slot
			}
			if (global_timer_ns() > deadline) ok = false;
		}
		if (!__shfl_sync(FULL, ok, 0)) {
			ok = false;
			break;
		}
	}
	if (!ok && lane == 0) atomicOr(a.err, 1u);
	// every issued copy lands before the CTA may retire its shared memory (the patched ones did)
	if (lane == 0) {
		const uint64_t drain = global_timer_ns() + a.timeout_ns;
		for (int jj = max(patched, issued - NSU); jj < issued; ++jj)
			mbar_wait(&land_u[jj % NSU], (uint32_t)(jj / NSU) & 1u, drain);
	}
}

// The kernel body: one CTA, tile (bx, by) of (i1, i2), z-chunk bz. tm_p[0..NPT) are the
// pointwise tiles of the output plane. SLOTS: the grids are slotted (4-D tensor maps whose
// outermost coordinate is the slot), as the modelling engine keeps its wavefields.
template <class Cfg, bool SLOTS>
__device__ __forceinline__ void zmarch_body(const CUtensorMap* tm_u, const CUtensorMap* tm_p0,
		const CUtensorMap* tm_p1, const CUtensorMap* tm_p2, const ZArgs<typename Cfg::C>& a,
		int bx, int by, int bz, int slot_u, int slot_p0, int slot_out, int step)
{
	using S = typename Cfg::Stor;
	using SC = typename Cfg::CoefStor;
	using C = typename Cfg::C;
	constexpr bool EX = Cfg::EXACT;
	using A = Arith<EX>;
	constexpr int R = Cfg::R, VX = Cfg::VX, VY = Cfg::VY, TX = Cfg::TX;
	constexpr int R4 = Cfg::R4, RY = Cfg::RY, RZ = Cfg::RZ, BX = Cfg::BX;
	constexpr int NSU = Cfg::NSU, NSP = Cfg::NSP, NC = Cfg::NC;
	constexpr int UE = Cfg::U_STRIDE / (int)sizeof(S);     // elements between input tiles

	extern __shared__ unsigned char smem_raw[];
	unsigned char* smem = reinterpret_cast<unsigned char*>(
			(reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
	S* su = reinterpret_cast<S*>(smem);
	unsigned char* sp = smem + NSU * Cfg::U_STRIDE;       // pointwise ring, Cfg::SLOT_P per slot
	constexpr int NPT = Cfg::NPT;
	uint64_t* bars = reinterpret_cast<uint64_t*>(
			smem + NSU * Cfg::U_STRIDE + (Cfg::P ? NSP * Cfg::SLOT_P : 0));
	uint64_t* full_u = bars;
	uint64_t* empty_u = bars + NSU;
	uint64_t* empty_p = bars + 2 * NSU;      // the pointwise tiles land on full_u (see the producer)
	uint64_t* land_u = bars + 2 * NSU + NSP; // fused step: where the copies land before the patch

	const int tile_x0 = a.x_start + bx * TX;
	const int tile_y0 = a.s2 + by * Cfg::TY;
	const int z0 = a.s3 + bz * a.nz_chunk;
	const int z1 = min(z0 + a.nz_chunk, a.e3 + 1);
	const int J = (z1 - z0) + 2 * RZ;          // planes this CTA streams in

	// fused boundary condition: a CTA whose tile (with halos) comes within R of an i1 or i2
	// boundary line, or whose planes include a boundary or z-halo plane, has its planes rebuilt
	// by the producer warp; the others run the pressure update as it is
	bool near = false, patch = false;
	if constexpr (Cfg::BC) {
		const int xs = tile_x0 - R4, xe = tile_x0 + TX + R4 - 1;
		const int ys = tile_y0 - RY, ye = tile_y0 + Cfg::TY + RY - 1;
		near = (xs <= a.s1 + R && xe >= a.s1 - R) || (xs <= a.e1 + R && xe >= a.e1 - R) ||
		       (ys <= a.s2 + R && ye >= a.s2 - R) || (ys <= a.e2 + R && ye >= a.e2 - R);
		patch = near || z0 - RZ <= a.s3 || z1 - 1 + RZ >= a.e3;
	}

	if (threadIdx.x == 0) {
		for (int s = 0; s < NSU; s++) {
			// one arrival completes a plane: the copy's (expect_tx), or the patching warp's lane 0
			mbar_init(&full_u[s], 1);
			mbar_init(&empty_u[s], NC);        // every consumer thread releases
			if constexpr (Cfg::BC) mbar_init(&land_u[s], 1);
		}
		for (int s = 0; s < NSP; s++) {
			mbar_init(&empty_p[s], NC);
		}
		fence_mbar_init();
	}
	__syncthreads();
	const uint64_t deadline = global_timer_ns() + a.timeout_ns;

	if (threadIdx.x >= NC) {
		if constexpr (Cfg::BC) {
			if (patch) {
				step_patch_producer<Cfg, SLOTS>(tm_u, tm_p0, tm_p1, a, su, sp, bars, tile_x0, tile_y0,
						z0, J, near, slot_u, slot_p0, deadline);
				return;
			}
		}
		// ---- producer: one thread issues every TMA copy ------------------------------------------
		if (threadIdx.x != NC) return;
		prefetch_tmap(tm_u);
		if constexpr (Cfg::P) {
			prefetch_tmap(tm_p0);
			prefetch_tmap(tm_p1);
			if constexpr (NPT > 2) prefetch_tmap(tm_p2);
		}
		int issued_u = 0;
		bool ok = true;
		Ring<NSU> wu;
		Ring<NSP> wp;
		for (int j = 0; j < J; ++j) {
			// slot reuse: wait for the consumers' previous release of this slot
			if (j >= NSU && !mbar_wait(&empty_u[wu.slot], wu.phase ^ 1u, deadline)) {
				ok = false;
				break;
			}
			// the pointwise tiles of output plane j - 2 RZ, which the consumers compute when
			// input plane j arrives, land on that plane's barrier: one wait per plane
			const bool pw = Cfg::P && j >= 2 * RZ;
			if (pw && j - 2 * RZ >= NSP && !mbar_wait(&empty_p[wp.slot], wp.phase ^ 1u, deadline)) {
				ok = false;
				break;
			}
			const int plane = z0 - RZ + j;     // (a fused step's z-halo planes: patching producer)
			uint64_t* bar = &full_u[wu.slot];
			mbar_arrive_expect_tx(bar, Cfg::U_BYTES + (pw ? Cfg::SLOT_TX : 0));
			tma_tile<SLOTS>(su + wu.slot * UE, tm_u, tile_x0 - R4, tile_y0 - RY, plane, slot_u, bar);
			issued_u = j + 1;
			wu.advance();
			if constexpr (Cfg::P) {
				if (pw) {
					const int o = j - 2 * RZ;
					unsigned char* slot = sp + wp.slot * Cfg::SLOT_P;
					tma_tile<SLOTS>(slot, tm_p0, tile_x0, tile_y0, z0 + o, slot_p0, bar);
					tma_tile<SLOTS>(slot + Cfg::PT_STRIDE, tm_p1, tile_x0, tile_y0, z0 + o, 0, bar);
					if constexpr (NPT > 2)
						tma_tile<SLOTS>(slot + Cfg::PT_STRIDE + Cfg::CT_STRIDE, tm_p2, tile_x0, tile_y0,
								z0 + o, 0, bar);
					wp.advance();
				}
			}
		}
		if (!ok) atomicOr(a.err, 1u);
		// every issued copy lands before the CTA may retire its shared memory
		const uint64_t drain = global_timer_ns() + a.timeout_ns;
		for (int j = max(0, issued_u - NSU); j < issued_u; ++j)
			mbar_wait(&full_u[j % NSU], (j / NSU) & 1, drain);
		return;
	}

	// ---- consumers ---------------------------------------------------------------------------
	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const int xl = (tid % Cfg::NTX) * VX;
	const int yl = (tid / Cfg::NTX) * VY;
	const int X = tile_x0 + xl;
	const int Y0 = tile_y0 + yl;
	// MODE_MODEL: g1(i1) g2(i2) of this thread's points, fixed along the march (points past the
	// inner box are never stored: their table reads are clamped)
	float gxy[Cfg::MODE == MODE_MODEL ? VY : 1][Cfg::MODE == MODE_MODEL ? VX : 1];
	if constexpr (Cfg::MODE == MODE_MODEL) {
#pragma unroll
		for (int v = 0; v < VY; v++) {
			const float g2 = a.g2[min(Y0 + v, a.e2)];
#pragma unroll
			for (int e = 0; e < VX; e++) gxy[v][e] = a.g1[min(X + e, a.e1)] * g2;
		}
	}
	using Q = std::conditional_t<Cfg::QPACK, ZQueue<S, C>, ZQueueF<S, C>>;
	constexpr int VQ = VX / Q::W;
	constexpr int UQ = Cfg::UQ;
	typename Q::T q[2 * RZ + UQ][VY][VQ];   // values along i3 of this thread's points
	// `alive` turns false when a bounded wait runs out: the warp then skips all work but keeps
	// the loop's barrier sequence, so no other warp is left waiting at a named barrier.
	bool alive = true;
	Ring<NSU> ru;                      // front plane j
	Ring<NSU> rc;                      // centre plane j - RZ
	rc.slot = RZ;                      // stage RZ: first centre plane (RZ < NSU, use 0)
	Ring<NSP> rp;                      // prn/coef of output plane j - 2 RZ

	// this thread's first point of output plane z0 (advanced by one plane per output plane; the
	// stores check their bounds)
	S* orow = static_cast<S*>(a.out) + X + (int64_t)Y0 * a.n1 + (int64_t)z0 * a.n12;
	if constexpr (SLOTS) orow += slot_out * a.out_slot_stride;
	// The loop runs UQ planes per pass, the pushes of a pass going to q[2 RZ + u] and the
	// queue shifted by UQ once per pass: logical q[i] of sub-step u is q[u + i].
	for (int jb = 0; jb < J; jb += UQ) {
	static_for<UQ>([&](auto uc) {
		constexpr int u = decltype(uc)::value;
		const int j = jb + u;
		if (j >= J) return;
			const int s = ru.slot;
			// lanes give up on their own (each then skips its work; no barrier follows)
			if (alive && !mbar_wait(&full_u[s], ru.phase, deadline)) alive = false;
			if constexpr (Cfg::ZQ) {
				if (alive) {
					const S* t = su + s * UE;
#pragma unroll
					for (int v = 0; v < VY; v++)
						Q::template push<VX>(t + (yl + v + RY) * BX + R4 + xl, q[u + 2 * RZ][v]);
				}
			}
			if constexpr (Cfg::ZONLY) mbar_arrive(&empty_u[s]);
			if (j >= 2 * RZ) {
				const int o = j - 2 * RZ;
				const int k = z0 + o;                     // output plane
				(void)k;
				const int sc = Cfg::ZQ ? rc.slot : s;      // slot holding plane k with its halos
				const S* t = su + sc * UE;
				const S* pt = nullptr;     // output-plane tile (prn, or w for the gradient)
				const SC* ct = nullptr;    // coef tile
				const S* gt = nullptr;     // gradient tile
				(void)pt, (void)ct, (void)gt;
				if constexpr (Cfg::P) {
					unsigned char* slot = sp + rp.slot * Cfg::SLOT_P;
					pt = reinterpret_cast<const S*>(slot);
					ct = reinterpret_cast<const SC*>(slot + Cfg::PT_STRIDE);
					gt = reinterpret_cast<const S*>(slot + Cfg::PT_STRIDE + Cfg::CT_STRIDE);
				}
				if (alive) {
					// rows of this thread's columns, plane k: (VY + 2 RY) x VX values, the centre
					// rows from the z queue
					typename Q::T yv[VY + 2 * RY][VQ];
#pragma unroll
					for (int r = 0; r < VY + 2 * RY; r++) {
						const int v = r - RY;
						if (v >= 0 && v < VY && Cfg::ZQ) {
#pragma unroll
							for (int e = 0; e < VQ; e++) yv[r][e] = q[u + RZ][v < 0 ? 0 : (v >= VY ? VY - 1 : v)][e];
						} else {
							Q::template push<VX>(t + (yl + r) * BX + R4 + xl, yv[r]);
						}
					}
#pragma unroll
					for (int v = 0; v < VY; v++) {
						C res[VX];
						// x-stencil vector of row v: left halo vectors, centre, right halo vectors
						C xv[Cfg::XH ? VX + 2 * R4 : 1];
						(void)xv;
						if constexpr (Cfg::XH) {
#pragma unroll
							for (int h = 0; h < R4 / VX; h++)
								lds_vec<S, C, VX>(t + (yl + v + RY) * BX + xl + h * VX, &xv[h * VX]);
#pragma unroll
							for (int e = 0; e < VX; e++) xv[R4 + e] = Q::get(yv[v + RY], e);
#pragma unroll
							for (int h = 0; h < R4 / VX; h++)
								lds_vec<S, C, VX>(t + (yl + v + RY) * BX + R4 + xl + VX + h * VX,
										&xv[R4 + VX + h * VX]);
						}
						if constexpr (std::is_same_v<C, float> && VX % 2 == 0) {
							// FP32: pairs of points with the two-wide instructions
							using A2 = Arith2<EX>;
							const float2 i1 = make_float2(a.inv2_1, a.inv2_1);
							const float2 i2 = make_float2(a.inv2_2, a.inv2_2);
							const float2 i3 = make_float2(a.inv2_3, a.inv2_3);
							// the pointwise tiles of this row, one vector load each
							constexpr int NV = Cfg::P ? VX : 1;
							float pv0[NV], pv1[NV], pv2[(Cfg::MODE == MODE_GRAD) ? VX : 1];
							(void)pv0, (void)pv1, (void)pv2;
							if constexpr (Cfg::P) {
								lds_vec<S, float, VX>(pt + (yl + v) * TX + xl, pv0);
								lds_vec<SC, float, VX>(ct + (yl + v) * TX + xl, pv1);
								if constexpr (Cfg::MODE == MODE_GRAD)
									lds_vec<S, float, VX>(gt + (yl + v) * TX + xl, pv2);
							}
#pragma unroll
							for (int pp = 0; pp < VX / 2; pp++) {
								const int e = 2 * pp;
								float2 dx = make_float2(0.f, 0.f), dy = dx, dz = dx, r2;
								(void)dx, (void)dy, (void)dz;
								if constexpr (Cfg::D1) {
									// staggered first derivative, values k = -R..R-1 around the point
									if constexpr (Cfg::MODE == MODE_D1_AXIS1)
										r2 = d1_axis2_row<R, EX>([&](int kk) { return xv[R4 + e + kk]; }, i1);
									else if constexpr (Cfg::MODE == MODE_D1_AXIS2)
										r2 = d1_axis2<R, EX>([&](int kk) {
											return Q::get2(yv[v + RY + kk], e); }, i2);
									else
										r2 = d1_axis2<R, EX>([&](int kk) {
											return Q::get2(q[u + RZ + kk][v], e); }, i3);
								}
								if constexpr (Cfg::XH && !Cfg::D1)
									dx = d2_axis2_row<R, EX>([&](int kk) { return xv[R4 + e + kk]; }, i1);
								if constexpr (Cfg::YH && !Cfg::D1)
									dy = d2_axis2<R, EX>([&](int kk) {
										return Q::get2(yv[v + RY + kk], e); }, i2);
								if constexpr (Cfg::ZQ && !Cfg::D1)
									dz = d2_axis2<R, EX>([&](int kk) {
										return Q::get2(q[u + RZ + kk][v], e); }, i3);
								if constexpr (Cfg::D1) {
								} else if constexpr (Cfg::MODE == MODE_D2_AXIS1) {
									r2 = dx;
								} else if constexpr (Cfg::MODE == MODE_D2_AXIS2) {
									r2 = dy;
								} else if constexpr (Cfg::MODE == MODE_D2_AXIS3) {
									r2 = dz;
								} else if constexpr (Cfg::MODE == MODE_LAPLACIAN) {
									r2 = A2::add(A2::add(dx, dy), dz);
								} else if constexpr (Cfg::MODE == MODE_MODEL) {
									// p+ = G (2 p + C Lap p) - G^2 p-, G = (g1 g2) g3
									const float g3 = a.g3[k];
									const float2 G = make_float2(gxy[v][e] * g3, gxy[v][e + 1] * g3);
									const float2 pm = make_float2(pv0[e], pv0[e + 1]);
									const float2 cf = make_float2(pv1[e], pv1[e + 1]);
									const float2 pc = Q::get2(yv[v + RY], e);
									const float2 lap = A2::add(A2::add(dx, dy), dz);
									const float2 t = A2::mac(A2::add(pc, pc), cf, lap);
									const float2 gg = A2::mul(G, G);
									r2 = A2::mac(A2::mul(make_float2(-gg.x, -gg.y), pm), G, t);
									if (step >= 0 && k == a.src_z && Y0 + v == a.src_y) {
										// the point source: p+(src) += G amp wavelet[step]
										if (X + e == a.src_x) r2.x = fmaf(G.x * a.src_amp, a.wavelet[step], r2.x);
										if (X + e + 1 == a.src_x) r2.y = fmaf(G.y * a.src_amp, a.wavelet[step], r2.y);
									}
								} else if constexpr (Cfg::MODE == MODE_GRAD) {
									// g += k C w Lap p
									const float2 w = make_float2(pv0[e], pv0[e + 1]);
									const float2 cf = make_float2(pv1[e], pv1[e + 1]);
									const float2 g0 = make_float2(pv2[e], pv2[e + 1]);
									const float2 kw = A2::mul(A2::mul(make_float2(a.kscale, a.kscale), cf), w);
									r2 = A2::mac(g0, kw, A2::add(A2::add(dx, dy), dz));
								} else {
									float pn[2] = {pv0[e], pv0[e + 1]}, cf[2] = {pv1[e], pv1[e + 1]};
									if (a.coef_scale != 1.0f) {
										cf[0] = cf[0] * a.coef_scale;
										cf[1] = cf[1] * a.coef_scale;
									}
									r2 = leapfrog2<EX>(Q::get2(yv[v + RY], e),
											make_float2(pn[0], pn[1]), make_float2(cf[0], cf[1]),
											A2::add(A2::add(dx, dy), dz));
								}
								res[e] = r2.x;
								res[e + 1] = r2.y;
							}
						} else {
							C dx[VX], dy[VX], dz[VX];
							(void)dx, (void)dy, (void)dz;
							if constexpr (Cfg::D1) {
#pragma unroll
								for (int e = 0; e < VX; e++) {
									if constexpr (Cfg::MODE == MODE_D1_AXIS1)
										res[e] = d1_axis<C, R, EX>([&](int kk) { return xv[R4 + e + kk]; }, a.inv2_1);
									else if constexpr (Cfg::MODE == MODE_D1_AXIS2)
										res[e] = d1_axis<C, R, EX>([&](int kk) { return Q::get(yv[v + RY + kk], e); }, a.inv2_2);
									else
										res[e] = d1_axis<C, R, EX>([&](int kk) { return Q::get(q[u + RZ + kk][v], e); }, a.inv2_3);
								}
							}
							if constexpr (Cfg::XH && !Cfg::D1) {
#pragma unroll
								for (int e = 0; e < VX; e++)
									dx[e] = d2_axis<C, R, EX>([&](int kk) { return xv[R4 + e + kk]; }, a.inv2_1);
							}
							if constexpr (Cfg::YH && !Cfg::D1) {
#pragma unroll
								for (int e = 0; e < VX; e++)
									dy[e] = d2_axis<C, R, EX>([&](int kk) { return Q::get(yv[v + RY + kk], e); }, a.inv2_2);
							}
							if constexpr (Cfg::ZQ && !Cfg::D1) {
#pragma unroll
								for (int e = 0; e < VX; e++)
									dz[e] = d2_axis<C, R, EX>([&](int kk) { return Q::get(q[u + RZ + kk][v], e); }, a.inv2_3);
							}
							if constexpr (Cfg::D1) {
							} else if constexpr (Cfg::MODE == MODE_D2_AXIS1) {
#pragma unroll
								for (int e = 0; e < VX; e++) res[e] = dx[e];
							} else if constexpr (Cfg::MODE == MODE_D2_AXIS2) {
#pragma unroll
								for (int e = 0; e < VX; e++) res[e] = dy[e];
							} else if constexpr (Cfg::MODE == MODE_D2_AXIS3) {
#pragma unroll
								for (int e = 0; e < VX; e++) res[e] = dz[e];
							} else if constexpr (Cfg::MODE == MODE_LAPLACIAN) {
#pragma unroll
								for (int e = 0; e < VX; e++) res[e] = A::add(A::add(dx[e], dy[e]), dz[e]);
							} else {
								C pn[VX], cf[VX];
								lds_vec<S, C, VX>(pt + (yl + v) * TX + xl, pn);
								lds_vec<SC, C, VX>(ct + (yl + v) * TX + xl, cf);
#pragma unroll
								for (int e = 0; e < VX; e++) {
									C c = cf[e];
									if (a.coef_scale != 1.0f) c = c * (C)a.coef_scale;
									res[e] = leapfrog<C, EX>(Q::get(yv[v + RY], e), pn[e], c,
											A::add(A::add(dx[e], dy[e]), dz[e]));
								}
							}
						}
						const int Y = Y0 + v;
						if (Y <= a.e2) {
							S* dst = orow + v * a.n1;
							if (X >= a.s1 && X + VX - 1 <= a.e1) {
								using Vec = std::conditional_t<VX * sizeof(S) == 16, uint4, uint2>;
								Vec pk;
								S* ps = reinterpret_cast<S*>(&pk);
#pragma unroll
								for (int e = 0; e < VX; e++) ps[e] = Storage<S>::store(res[e]);
								*reinterpret_cast<Vec*>(dst) = pk;
							} else {
#pragma unroll
								for (int e = 0; e < VX; e++)
									if (X + e >= a.s1 && X + e <= a.e1) dst[e] = Storage<S>::store(res[e]);
							}
						}
					}
				}
				// each thread releases the slots after its own last read of them
				if constexpr (!Cfg::ZONLY) mbar_arrive(&empty_u[sc]);
				if constexpr (Cfg::P) mbar_arrive(&empty_p[rp.slot]);
				rc.advance();
				rp.advance();
				orow += a.n12;
			}
			if constexpr (Cfg::ZQ && !Cfg::ZONLY) {
				if (j < RZ || j >= J - RZ)     // planes that are never a centre plane
					mbar_arrive(&empty_u[s]);
			}
			ru.advance();
	});
		if constexpr (Cfg::ZQ && UQ > 1) {
#pragma unroll
			for (int i = 0; i < 2 * RZ; i++)
#pragma unroll
				for (int v = 0; v < VY; v++)
#pragma unroll
					for (int e = 0; e < VQ; e++) q[i][v][e] = q[i + UQ][v][e];
		} else if constexpr (Cfg::ZQ) {
#pragma unroll
			for (int i = 0; i < 2 * RZ; i++)
#pragma unroll
				for (int v = 0; v < VY; v++)
#pragma unroll
					for (int e = 0; e < VQ; e++) q[i][v][e] = q[i + 1][v][e];
		}
	}
	if (!alive && lane == 0) atomicOr(a.err, 2u);
}

template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT, Cfg::MINB) k_zmarch(
		const __grid_constant__ CUtensorMap tm_u,
		const __grid_constant__ CUtensorMap tm_prn, const __grid_constant__ CUtensorMap tm_coef,
		const ZArgs<typename Cfg::C> a)
{
	zmarch_body<Cfg, false>(&tm_u, &tm_prn, &tm_coef, &tm_coef, a, (int)blockIdx.x,
			(int)blockIdx.y, (int)blockIdx.z, 0, 0, 0, -1);
}

// One shot of a batched launch: its tensor maps (slotted grids: u, pointwise tiles 0..2), its
// arguments and its range of CTAs. Lives in device memory, 64-byte aligned.
struct alignas(64) ZShot {
	CUtensorMap tm[4];
	ZArgs<float> a;
	int cta_begin, ntx, nty, nzc;
};

// Every shot of a batch in one launch: CTA b works on the shot whose range holds b. With
// `interleave` (every shot has the same tiling) CTA b works on shot b % nshot, tile b / nshot:
// the CTAs of one tile of all shots run side by side, so that the tiles they share (the model of
// shots on one grid) come from DRAM once and from L2 for the others.
template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT, Cfg::MINB) k_zmarch_batch(const ZShot* __restrict__ shots,
		int nshot, int slot_u, int slot_p0, int slot_out, int step, int interleave)
{
	const int b = (int)blockIdx.x;
	int s = 0, local = 0;
	if (interleave) {
		s = b % nshot;
		local = b / nshot;
	} else {
		while (s + 1 < nshot && shots[s + 1].cta_begin <= b) ++s;
		local = b - shots[s].cta_begin;
	}
	const ZShot& sh = shots[s];
	const int bx = local % sh.ntx, by = (local / sh.ntx) % sh.nty, bz = local / (sh.ntx * sh.nty);
	// the shot's arguments in shared memory: read far more often than the tensor maps
	__shared__ ZArgs<float> args;
	static_assert(sizeof(ZArgs<float>) % 4 == 0, "word copy");
	for (int i = threadIdx.x; i < (int)(sizeof(ZArgs<float>) / 4); i += blockDim.x)
		reinterpret_cast<int*>(&args)[i] = reinterpret_cast<const int*>(&sh.a)[i];
	__syncthreads();
	zmarch_body<Cfg, true>(&sh.tm[0], &sh.tm[1], &sh.tm[2], &sh.tm[3], args, bx, by, bz, slot_u,
			slot_p0, slot_out, step);
}

}  // namespace

// ---- host side ------------------------------------------------------------------------------------
// Tensor map of a 3-D grid with box (bx, by, 1) (b200_stencil_zmarch.cu).
int make_map(CUtensorMap* m, const void* base, int dtype, const b200_layout* lay, int bx, int by);
// Tensor map of nslot consecutive FP32 grids of one layout (4-D, the slot outermost).
int make_map_slots(CUtensorMap* m, const void* base, const b200_layout* lay, int nslot, int bx,
		int by);

namespace {

// planes per CTA: long chunks amortise the z-halo (2R planes per chunk), as long as the grid
// still fills the GPU twice over with resident CTAs (64 planes for R <= 2, 128 beyond, at 512^3)
template <class Cfg>
int pick_nz_chunk(int ntiles, int nz, int requested)
{
	if (requested > 0) return requested < nz ? requested : nz;
	// resident CTAs per SM of this configuration, asked once per process (the call costs
	// microseconds, which a caller that synchronises after every launch would see)
	static const int per_sm_cached = [] {
		int v = 0;
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_zmarch<Cfg>, Cfg::NT, Cfg::SMEM);
		return v;
	}();
	const int per_sm = per_sm_cached < 1 ? 1 : per_sm_cached;
	const int resident = per_sm * num_sms();
	int chunk = Cfg::R <= 2 ? 64 : 128;
	while (chunk > 16 && (int64_t)ntiles * ((nz + chunk - 1) / chunk) < 2 * (int64_t)resident) chunk /= 2;
	return chunk < nz ? chunk : nz;
}

template <class Cfg>
int launch_zmarch(const ZLaunch& L)
{
	const b200_layout* lay = L.lay;
	const b200_field& in = *L.in;
	const b200_field& out = *L.out;
	const b200_field* coef = L.coef;
	const double inv2_1 = L.inv2[0], inv2_2 = L.inv2[1], inv2_3 = L.inv2[2];
	cudaStream_t s = L.s;
	using C = typename Cfg::C;
	int rc = cuda_error(cudaFuncSetAttribute(k_zmarch<Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                            Cfg::SMEM), "cudaFuncSetAttribute(k_zmarch)");
	if (rc) return rc;
	alignas(64) CUtensorMap tm_u, tm_p, tm_c;
	if ((rc = make_map(&tm_u, in.data, in.dtype, lay, Cfg::BX, Cfg::BY))) return rc;
	if (Cfg::P) {
		if ((rc = make_map(&tm_p, out.data, out.dtype, lay, Cfg::TX, Cfg::TY))) return rc;
		if ((rc = make_map(&tm_c, coef->data, coef->dtype, lay, Cfg::TX, Cfg::TY))) return rc;
	} else {
		tm_p = tm_u;
		tm_c = tm_u;
	}
	ZArgs<C> a{};
	a.out = out.data;
	a.n1 = lay->n1;
	a.n12 = lay->n1 * lay->n2;
	a.x_start = (int)(lay->s1 / Cfg::VA) * Cfg::VA;
	a.s1 = (int)lay->s1; a.e1 = (int)lay->e1;
	a.s2 = (int)lay->s2; a.e2 = (int)lay->e2;
	a.s3 = (int)lay->s3; a.e3 = (int)lay->e3;
	a.inv2_1 = (C)inv2_1;
	a.inv2_2 = (C)inv2_2;
	a.inv2_3 = (C)inv2_3;
	a.coef_scale = coef ? coef->scale : 1.0f;
	a.timeout_ns = 2000000000ull;
	a.err = L.err;
	const int ntx = (a.e1 + 1 - a.x_start + Cfg::TX - 1) / Cfg::TX;
	const int nty = (a.e2 - a.s2 + 1 + Cfg::TY - 1) / Cfg::TY;
	const int nz = a.e3 - a.s3 + 1;
	a.nz_chunk = pick_nz_chunk<Cfg>(ntx * nty, nz, L.nz_chunk);
	const int nzc = (nz + a.nz_chunk - 1) / a.nz_chunk;
	k_zmarch<Cfg><<<dim3(ntx, nty, nzc), Cfg::NT, Cfg::SMEM, s>>>(tm_u, tm_p, tm_c, a);
	return check_launch("k_zmarch");
}


// Tile shapes the kernel is instantiated with, per storage size and half width:
// (TX, TY, VY, PF); TX = 16 vectors of 16 bytes. The autotuner (b200_autotune_stencil) picks
// among them; shape 0 is the default. Consumer-thread counts are 224 (7 warps + the producer
// warp = 8 warps, two CTAs per SM) or 480 (16 warps, one CTA per SM). Two rows per thread
// (VY = 2) pay off for R <= 2 only: from R = 3 on, the longer z queue makes the registers,
// not the shared-memory traffic, the limit (measured on B200).
template <typename S, int R, int SHAPE> struct Shape;
// Shape 0 keeps FP32 R = 5..7 at two CTAs per SM (128 registers; one CTA of 8 warps at the
// 170-200 registers these would take otherwise leaves the schedulers short of warps: at 512^3 on
// B200 the pressure update takes 0.51 against 0.64 ms at O10, 0.58 against 0.66 at O12, 0.59
// against 0.62 at O14, bit-identical; at O16 the spills make it slower).
// UQP: planes per pass of the z loop for the pressure update and the fused step (0: the
// default of the mode).
template <typename S, int R> struct Shape<S, R, 0> {
	static constexpr int TX = 64 * 4 / (int)sizeof(S), TY = (R <= 2 ? 28 : 14), VY = (R <= 2 ? 2 : 1), PF = 2,
	                     MINB = (sizeof(S) == 4 && R >= 5 && R <= 7) ? 2 : 0, UQP = 0; };
// shape 0 with a deeper prefetch ring; FP32 R = 4 with eight planes per pass of the pressure
// update's z loop (half the queue shifts and loop overhead per plane; 128 registers, no spills;
// 0.349 against 0.355 ms at 512^3 on B200)
template <typename S, int R> struct Shape<S, R, 1> {
	static constexpr int TX = 64 * 4 / (int)sizeof(S), TY = (R <= 2 ? 28 : 14), VY = (R <= 2 ? 2 : 1), PF = 4, MINB = 0,
	                     UQP = (sizeof(S) == 4 && R == 4) ? 8 : 0; };
// Shape 2: 9 warps, two CTAs per SM for R <= 4; for FP32 and FP64 R = 5..6, 11 consumer warps in
// 22-row tiles at one CTA per SM (up to 168 registers, no spills) with a five-plane prefetch: at
// 512^3 on B200 the FP32 pressure update takes 0.478 against 0.523 ms at O10 and 0.488 against
// 0.566 at O12, the O12 Laplacian 0.45 against 0.51 ms; FP64 O10 0.93 against 1.13 ms, O12 0.93
// against 1.15-1.22, the O12 Laplacian 0.92 against 1.03; all bit-identical.
// R = 7..8: the 9-warp tile with a deeper prefetch (four planes for FP32 R = 7 and FP64 R = 8,
// where five would not leave the fused step's shared memory room, five otherwise) and four
// planes per pass of the pressure update's z loop; at 512^3 on B200: FP32 O16 0.571 against
// 0.635 ms (the O16 Laplacian 0.51 against 0.55), FP32 O14 0.517 against 0.553 on the two-CTA
// tile of shape 0, FP64 O14 1.12 against 1.25, FP64 O16 1.24 against 1.26 (Laplacian 1.13
// against 1.16).
template <typename S, int R> struct Shape<S, R, 2> {
	static constexpr bool WIDE = sizeof(S) >= 4 && R >= 5 && R <= 6;
	static constexpr bool DEEP = sizeof(S) >= 4 && (R == 7 || R == 8);
	static constexpr int TX = 64 * 4 / (int)sizeof(S), TY = WIDE ? 22 : 16, VY = 1,
	                     PF = WIDE ? 5 : DEEP ? ((sizeof(S) == 4) == (R == 7) ? 4 : 5) : 2,
	                     MINB = (R <= 4 && !WIDE) ? 2 : 1, UQP = DEEP ? 4 : 0; };

// Shared memory a CTA may use on sm_100 (227 KB).
constexpr int kMaxSmemPerBlock = 232448;

template <typename S, int R, int MODE, int SHAPE, bool EXACT>
int launch_shape(const ZLaunch& L)
{
	using Sh = Shape<S, R, SHAPE>;
	// The y-only operators from R = 5 on: four rows per thread in 56-row tiles, so that the
	// 2R + 4 rows a thread reads from shared memory serve four output rows (no z queue holds
	// registers there): 0.22 against 0.32 ms for FD_D2_N2 O16 FP32 at 512^3 on B200 (at O8 the
	// one-row tiles are as fast).
	constexpr bool YROWS = (MODE == MODE_D2_AXIS2 || MODE == MODE_D1_AXIS2) && R >= 5;
	using Cfg = ZCfg<S, R, MODE, Sh::TX, YROWS ? 56 : Sh::TY, YROWS ? 4 : Sh::VY, Sh::PF, EXACT,
			Sh::MINB, S, (MODE == MODE_PRESSURE || MODE == MODE_STEP) ? Sh::UQP : 0>;
	if constexpr (Cfg::SMEM > kMaxSmemPerBlock)
		return set_error(B200_ERR_UNSUPPORTED, "stencil shape %d needs %d bytes of shared memory",
				SHAPE, Cfg::SMEM);
	else
		return launch_zmarch<Cfg>(L);
}

// 16-bit wavefields (FP16 or BF16, with a per-field scale) computing in FP32 with fused
// multiply-adds; coef in the same 16-bit type or FP32. Shape 0: 16-byte thread vectors (8
// points) with the z queue kept as packed 16-bit pairs; shapes 1 and 2: 8-byte vectors (4
// points) with the z queue in FP32, each value converted once (14-row tiles and a four-plane
// prefetch, or 28-row tiles). Shape 1 at R = 4 runs eight planes per pass of the z loop (0.390
// against 0.402 ms for FP16 waves with FP32 coef at 512^3 on B200, bit-identical).
template <int MODE, int R, typename S, typename SC>
int launch_16bit_coef(const ZLaunch& L)
{
	switch (L.shape) {
	case 1: return launch_zmarch<ZCfg<S, R, MODE, 64, 14, 1, 4, false, 0, SC, (R == 4 ? 8 : 0), 8>>(L);
	case 2:
		// R = 5..6: the 22-row tiles of 11 consumer warps at one CTA per SM with a five-plane
		// prefetch, as for FP32 (FP16 O12 0.549 against 0.659 ms at 512^3 on B200, BF16 0.560
		// against 0.627, bit-identical)
		if constexpr (R >= 5 && R <= 6)
			return launch_zmarch<ZCfg<S, R, MODE, 64, 22, 1, 5, false, 1, SC, 4, 8>>(L);
		// R = 7..8: the 9-warp tile with a deeper prefetch and four planes per z pass, as for
		// FP32 (FP16 O14 0.600 against 0.629 ms, O16 0.670 against 0.701, BF16 O16 0.647
		// against 0.672)
		else if constexpr (R >= 7)
			return launch_zmarch<ZCfg<S, R, MODE, 64, 16, 1, (R == 7 ? 4 : 5), false, 1, SC, 4, 8>>(L);
		else
			return launch_zmarch<ZCfg<S, R, MODE, 64, (R <= 4 ? 28 : 16), 1, 2, false, 0, SC, 0, 8>>(L);
	default: return launch_zmarch<ZCfg<S, R, MODE, 64, (R <= 4 ? 28 : 16), 1, 2, false, 0, SC>>(L);
	}
}

template <int MODE, int R, typename S>
int launch_16bit(const ZLaunch& L)
{
	if (L.coef && L.coef->dtype == B200_F32) return launch_16bit_coef<MODE, R, S, float>(L);
	return launch_16bit_coef<MODE, R, S, S>(L);
}

// Dispatch storage type, half width, shape and arithmetic for one operator. NSHAPES and
// WITH_FMA bound the instantiations (the single-axis operators use shape 0, exact only).
template <int MODE, int NSHAPES, bool WITH_FMA>
int launch_mode(const ZLaunch& L)
{
	return dispatch_order(2 * L.R, [&](auto rt) {
		constexpr int R = decltype(rt)::value;
		auto go = [&](auto tag) -> int {
			using S = decltype(tag);
			const int shape = (L.shape >= 0 && L.shape < NSHAPES) ? L.shape : 0;
			const bool exact = L.exact || !WITH_FMA;
			if (exact) {
				if (shape == 0) return launch_shape<S, R, MODE, 0, true>(L);
				if constexpr (NSHAPES > 1) if (shape == 1) return launch_shape<S, R, MODE, 1, true>(L);
				if constexpr (NSHAPES > 2) return launch_shape<S, R, MODE, 2, true>(L);
			} else if constexpr (WITH_FMA) {
				if (shape == 0) return launch_shape<S, R, MODE, 0, false>(L);
				if constexpr (NSHAPES > 1) if (shape == 1) return launch_shape<S, R, MODE, 1, false>(L);
				if constexpr (NSHAPES > 2) return launch_shape<S, R, MODE, 2, false>(L);
			}
			return set_error(B200_ERR_ARG, "stencil shape %d", shape);
		};
		if constexpr (MODE == MODE_PRESSURE) {
			if (L.in->dtype == B200_F16) return launch_16bit<MODE, R, __half>(L);
			if (L.in->dtype == B200_BF16) return launch_16bit<MODE, R, __nv_bfloat16>(L);
		}
		if (L.in->dtype == B200_F64) return go(double{});
		return go(float{});
	});
}

}  // namespace
}  // namespace b200
