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
// Every wait on an mbarrier is bounded by a time limit: a CTA that gives up records an
// error flag (read by b200_device_status) and returns after its issued copies have landed.
#include <cuda.h>

#include <cstring>

#include "b200_stencil.cuh"

namespace b200 {

__device__ unsigned int g_device_error;

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

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* tm)
{
	asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tm)) : "memory");
}

// ---- vector shared-memory loads (16 bytes) converted to the compute type --------------------------
template <typename S, typename C, int N>
__device__ __forceinline__ void lds_vec(const S* p, C* out)
{
	static_assert(N * sizeof(S) % 16 == 0, "vector of 16-byte multiples");
#pragma unroll
	for (int b = 0; b < N * (int)sizeof(S) / 16; b++) {
		const uint4 raw = reinterpret_cast<const uint4*>(p)[b];
		const S* v = reinterpret_cast<const S*>(&raw);
#pragma unroll
		for (int i = 0; i < 16 / (int)sizeof(S); i++)
			out[b * (16 / sizeof(S)) + i] = Storage<S>::load(v[i]);
	}
}

constexpr int round_up(int v, int m) { return (v + m - 1) / m * m; }

// ---- kernel configuration -----------------------------------------------------------------------
template <typename S, int R_, int MODE_, int TX_, int TY_, int VY_, int PF_>
struct ZCfg {
	using Stor = S;
	using C = typename Storage<S>::C;
	static constexpr int R = R_;
	static constexpr int MODE = MODE_;
	static constexpr int TX = TX_, TY = TY_, VY = VY_, PF = PF_;
	static constexpr int VX = 16 / sizeof(S);
	static constexpr bool XH = (MODE == MODE_D2_AXIS1 || MODE == MODE_LAPLACIAN || MODE == MODE_PRESSURE);
	static constexpr bool YH = (MODE == MODE_D2_AXIS2 || MODE == MODE_LAPLACIAN || MODE == MODE_PRESSURE);
	static constexpr bool ZQ = (MODE == MODE_D2_AXIS3 || MODE == MODE_LAPLACIAN || MODE == MODE_PRESSURE);
	static constexpr bool P = (MODE == MODE_PRESSURE);
	static constexpr int R4 = XH ? round_up(R, VX) : 0;     // x halo, whole vectors
	static constexpr int RY = YH ? R : 0;
	static constexpr int RZ = ZQ ? R : 0;
	static constexpr int BX = TX + 2 * R4;
	static constexpr int BY = TY + 2 * RY;
	static constexpr int NSU = RZ + 1 + PF;                  // input-tile ring
	static constexpr int NSP = P ? 1 + PF : 1;               // prn/coef ring
	static constexpr int U_BYTES = BX * BY * (int)sizeof(S);
	static constexpr int U_STRIDE = round_up(U_BYTES, 128);
	static constexpr int PT_BYTES = TX * TY * (int)sizeof(S);
	static constexpr int PT_STRIDE = round_up(PT_BYTES, 128);
	static constexpr int NTX = TX / VX;
	static constexpr int NC = NTX * (TY / VY);              // consumer threads
	static constexpr int NWC = NC / 32;                      // consumer warps
	static constexpr int NT = NC + 32;                       // + one producer warp
	static constexpr int SMEM = 128 + NSU * U_STRIDE + (P ? NSP * 2 * PT_STRIDE : 0) +
	                            (2 * NSU + 2 * NSP) * 8;
	static_assert(TX % VX == 0 && TY % VY == 0 && NC % 32 == 0, "tile shape");
	static_assert(BX <= 256 && BY <= 256, "TMA box limit");
	static_assert((BX * sizeof(S)) % 16 == 0 && (TX * sizeof(S)) % 16 == 0, "TMA inner extent");
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
};


template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT) k_zmarch(const __grid_constant__ CUtensorMap tm_u,
		const __grid_constant__ CUtensorMap tm_prn, const __grid_constant__ CUtensorMap tm_coef,
		const ZArgs<typename Cfg::C> a)
{
	using S = typename Cfg::Stor;
	using C = typename Cfg::C;
	using A = Arith<true>;
	constexpr int R = Cfg::R, VX = Cfg::VX, VY = Cfg::VY, TX = Cfg::TX;
	constexpr int R4 = Cfg::R4, RY = Cfg::RY, RZ = Cfg::RZ, BX = Cfg::BX;
	constexpr int NSU = Cfg::NSU, NSP = Cfg::NSP, NC = Cfg::NC;
	constexpr int UE = Cfg::U_STRIDE / (int)sizeof(S);     // elements between input tiles
	constexpr int PE = Cfg::PT_STRIDE / (int)sizeof(S);    // elements between prn/coef tiles
	constexpr unsigned FULL = 0xffffffffu;

	extern __shared__ unsigned char smem_raw[];
	unsigned char* smem = reinterpret_cast<unsigned char*>(
			(reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
	S* su = reinterpret_cast<S*>(smem);
	S* sp = reinterpret_cast<S*>(smem + NSU * Cfg::U_STRIDE);
	uint64_t* bars = reinterpret_cast<uint64_t*>(
			smem + NSU * Cfg::U_STRIDE + (Cfg::P ? NSP * 2 * Cfg::PT_STRIDE : 0));
	uint64_t* full_u = bars;
	uint64_t* empty_u = bars + NSU;
	uint64_t* full_p = bars + 2 * NSU;
	uint64_t* empty_p = full_p + NSP;

	const int tile_x0 = a.x_start + (int)blockIdx.x * TX;
	const int tile_y0 = a.s2 + (int)blockIdx.y * Cfg::TY;
	const int z0 = a.s3 + (int)blockIdx.z * a.nz_chunk;
	const int z1 = min(z0 + a.nz_chunk, a.e3 + 1);
	const int J = (z1 - z0) + 2 * RZ;          // planes this CTA streams in

	if (threadIdx.x == 0) {
		for (int s = 0; s < NSU; s++) {
			mbar_init(&full_u[s], 1);
			mbar_init(&empty_u[s], Cfg::NWC);
		}
		for (int s = 0; s < NSP; s++) {
			mbar_init(&full_p[s], 1);
			mbar_init(&empty_p[s], Cfg::NWC);
		}
		fence_mbar_init();
	}
	__syncthreads();
	const uint64_t deadline = global_timer_ns() + a.timeout_ns;

	if (threadIdx.x >= NC) {
		// ---- producer: one thread issues every TMA copy ------------------------------------------
		if (threadIdx.x != NC) return;
		prefetch_tmap(&tm_u);
		if constexpr (Cfg::P) {
			prefetch_tmap(&tm_prn);
			prefetch_tmap(&tm_coef);
		}
		int issued_u = 0, issued_p = 0;
		bool ok = true;
		for (int j = 0; j < J; ++j) {
			const int s = j % NSU;
			if (j >= NSU && !mbar_wait(&empty_u[s], ((j / NSU) - 1) & 1, deadline)) {
				ok = false;
				break;
			}
			mbar_arrive_expect_tx(&full_u[s], Cfg::U_BYTES);
			tma_load_3d(su + s * UE, &tm_u, tile_x0 - R4, tile_y0 - RY, z0 - RZ + j, &full_u[s]);
			issued_u = j + 1;
			if constexpr (Cfg::P) {
				if (j >= 2 * RZ) {
					const int o = j - 2 * RZ, t = o % NSP;
					if (o >= NSP && !mbar_wait(&empty_p[t], ((o / NSP) - 1) & 1, deadline)) {
						ok = false;
						break;
					}
					mbar_arrive_expect_tx(&full_p[t], 2 * Cfg::PT_BYTES);
					tma_load_3d(sp + (2 * t) * PE, &tm_prn, tile_x0, tile_y0, z0 + o, &full_p[t]);
					tma_load_3d(sp + (2 * t + 1) * PE, &tm_coef, tile_x0, tile_y0, z0 + o, &full_p[t]);
					issued_p = o + 1;
				}
			}
		}
		if (!ok) atomicOr(&g_device_error, 1u);
		// every issued copy lands before the CTA may retire its shared memory
		const uint64_t drain = global_timer_ns() + a.timeout_ns;
		for (int j = max(0, issued_u - NSU); j < issued_u; ++j)
			mbar_wait(&full_u[j % NSU], (j / NSU) & 1, drain);
		for (int o = max(0, issued_p - NSP); o < issued_p; ++o)
			mbar_wait(&full_p[o % NSP], (o / NSP) & 1, drain);
		return;
	}

	// ---- consumers ---------------------------------------------------------------------------
	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const int xl = (tid % Cfg::NTX) * VX;
	const int yl = (tid / Cfg::NTX) * VY;
	C q[2 * RZ + 1][VY][VX];           // values along i3 of this thread's points
	bool ok = true;
	for (int j = 0; j < J; ++j) {
		const int s = j % NSU;
		if (!__all_sync(FULL, mbar_wait(&full_u[s], (j / NSU) & 1, deadline))) {
			ok = false;
			break;
		}
		if constexpr (Cfg::ZQ) {
#pragma unroll
			for (int i = 0; i < 2 * RZ; i++)
#pragma unroll
				for (int v = 0; v < VY; v++)
#pragma unroll
					for (int e = 0; e < VX; e++) q[i][v][e] = q[i + 1][v][e];
			const S* t = su + s * UE;
#pragma unroll
			for (int v = 0; v < VY; v++) lds_vec<S, C, VX>(t + (yl + v + RY) * BX + R4 + xl, q[2 * RZ][v]);
		}
		if (j >= 2 * RZ) {
			const int o = j - 2 * RZ;
			const int k = z0 + o;                     // output plane
			const int sc = (j - RZ) % NSU;            // slot holding plane k with its halos
			const S* t = su + sc * UE;
			const S* pt = nullptr;
			if constexpr (Cfg::P) {
				const int tp = o % NSP;
				if (!__all_sync(FULL, mbar_wait(&full_p[tp], (o / NSP) & 1, deadline))) {
					ok = false;
					break;
				}
				pt = sp + (2 * tp) * PE;
			}
			// rows of this thread's columns, plane k: (VY + 2 RY) x VX values
			C yv[VY + 2 * RY][VX];
#pragma unroll
			for (int r = 0; r < VY + 2 * RY; r++) {
				const int v = r - RY;
				if (v >= 0 && v < VY && Cfg::ZQ) {
#pragma unroll
					for (int e = 0; e < VX; e++) yv[r][e] = q[RZ][v < 0 ? 0 : (v >= VY ? VY - 1 : v)][e];
				} else {
					lds_vec<S, C, VX>(t + (yl + r) * BX + R4 + xl, yv[r]);
				}
			}
			const int Y0 = tile_y0 + yl;
			const int X = tile_x0 + xl;
#pragma unroll
			for (int v = 0; v < VY; v++) {
				C res[VX];
				C dx[VX], dy[VX], dz[VX];
				if constexpr (Cfg::XH) {
					C xv[VX + 2 * R4];
#pragma unroll
					for (int h = 0; h < R4 / VX; h++)
						lds_vec<S, C, VX>(t + (yl + v + RY) * BX + xl + h * VX, &xv[h * VX]);
#pragma unroll
					for (int e = 0; e < VX; e++) xv[R4 + e] = yv[v + RY][e];
#pragma unroll
					for (int h = 0; h < R4 / VX; h++)
						lds_vec<S, C, VX>(t + (yl + v + RY) * BX + R4 + xl + VX + h * VX,
								&xv[R4 + VX + h * VX]);
#pragma unroll
					for (int e = 0; e < VX; e++)
						dx[e] = d2_axis<C, R, true>([&](int kk) { return xv[R4 + e + kk]; }, a.inv2_1);
				}
				if constexpr (Cfg::YH) {
#pragma unroll
					for (int e = 0; e < VX; e++)
						dy[e] = d2_axis<C, R, true>([&](int kk) { return yv[v + RY + kk][e]; }, a.inv2_2);
				}
				if constexpr (Cfg::ZQ) {
#pragma unroll
					for (int e = 0; e < VX; e++)
						dz[e] = d2_axis<C, R, true>([&](int kk) { return q[RZ + kk][v][e]; }, a.inv2_3);
				}
				if constexpr (Cfg::MODE == MODE_D2_AXIS1) {
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
					lds_vec<S, C, VX>(pt + PE + (yl + v) * TX + xl, cf);
#pragma unroll
					for (int e = 0; e < VX; e++) {
						C c = cf[e];
						if (a.coef_scale != 1.0f) c = c * (C)a.coef_scale;
						res[e] = leapfrog<C, true>(yv[v + RY][e], pn[e], c,
								A::add(A::add(dx[e], dy[e]), dz[e]));
					}
				}
				const int Y = Y0 + v;
				if (Y <= a.e2) {
					S* dst = static_cast<S*>(a.out) + X + (int64_t)Y * a.n1 + (int64_t)k * a.n12;
					if (X >= a.s1 && X + VX - 1 <= a.e1) {
						uint4 pk;
						S* ps = reinterpret_cast<S*>(&pk);
#pragma unroll
						for (int e = 0; e < VX; e++) ps[e] = Storage<S>::store(res[e]);
						*reinterpret_cast<uint4*>(dst) = pk;
					} else {
#pragma unroll
						for (int e = 0; e < VX; e++)
							if (X + e >= a.s1 && X + e <= a.e1) dst[e] = Storage<S>::store(res[e]);
					}
				}
			}
			__syncwarp();
			if (lane == 0) {
				mbar_arrive(&empty_u[sc]);
				if constexpr (Cfg::P) mbar_arrive(&empty_p[o % NSP]);
			}
		}
		if constexpr (Cfg::ZQ) {
			if (j < RZ || j >= J - RZ) {   // planes that are never a centre plane
				__syncwarp();
				if (lane == 0) mbar_arrive(&empty_u[s]);
			}
		}
	}
	if (!ok && lane == 0) atomicOr(&g_device_error, 2u);
}

// ---- host side ------------------------------------------------------------------------------------
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

// planes per CTA: enough CTAs for several waves, long enough chunks to amortise the z-halo
template <class Cfg>
int pick_nz_chunk(int ntiles, int nz)
{
	int per_sm = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_zmarch<Cfg>, Cfg::NT, Cfg::SMEM);
	if (per_sm < 1) per_sm = 1;
	const int resident = per_sm * num_sms();
	int chunk = 64;
	while (chunk > 16 && (int64_t)ntiles * ((nz + chunk - 1) / chunk) < 4 * (int64_t)resident) chunk /= 2;
	return chunk < nz ? chunk : nz;
}

template <class Cfg>
int launch_zmarch(const b200_layout* lay, const b200_field& in, const b200_field& out,
		const b200_field* coef, double inv2_1, double inv2_2, double inv2_3, cudaStream_t s)
{
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
	ZArgs<C> a;
	a.out = out.data;
	a.n1 = lay->n1;
	a.n12 = lay->n1 * lay->n2;
	a.x_start = (int)(lay->s1 / Cfg::VX) * Cfg::VX;
	a.s1 = (int)lay->s1; a.e1 = (int)lay->e1;
	a.s2 = (int)lay->s2; a.e2 = (int)lay->e2;
	a.s3 = (int)lay->s3; a.e3 = (int)lay->e3;
	a.inv2_1 = (C)inv2_1;
	a.inv2_2 = (C)inv2_2;
	a.inv2_3 = (C)inv2_3;
	a.coef_scale = coef ? coef->scale : 1.0f;
	a.timeout_ns = 2000000000ull;
	const int ntx = (a.e1 + 1 - a.x_start + Cfg::TX - 1) / Cfg::TX;
	const int nty = (a.e2 - a.s2 + 1 + Cfg::TY - 1) / Cfg::TY;
	const int nz = a.e3 - a.s3 + 1;
	a.nz_chunk = pick_nz_chunk<Cfg>(ntx * nty, nz);
	const int nzc = (nz + a.nz_chunk - 1) / a.nz_chunk;
	k_zmarch<Cfg><<<dim3(ntx, nty, nzc), Cfg::NT, Cfg::SMEM, s>>>(tm_u, tm_p, tm_c, a);
	return check_launch("k_zmarch");
}

// tile shapes per storage type and half width
template <typename S, int R, int MODE>
int launch_for(const b200_layout* lay, const b200_field& in, const b200_field& out,
		const b200_field* coef, double i1, double i2, double i3, cudaStream_t s)
{
	if constexpr (sizeof(S) == 8) {
		return launch_zmarch<ZCfg<S, R, MODE, 32, 16, 1, 2>>(lay, in, out, coef, i1, i2, i3, s);
	} else {
		return launch_zmarch<ZCfg<S, R, MODE, 64, 16, 1, 2>>(lay, in, out, coef, i1, i2, i3, s);
	}
}

}  // namespace

bool zmarch_accepts(const b200_layout* lay, int dtype)
{
	if (lay->dim != 3) return false;
	if (dtype != B200_F32 && dtype != B200_F64) return false;
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
	if ((reinterpret_cast<uintptr_t>(in.data) | reinterpret_cast<uintptr_t>(out.data)) % 16) return B200_OK;
	if (coef) {
		if (coef->dtype != in.dtype) return B200_OK;
		if (reinterpret_cast<uintptr_t>(coef->data) % 16) return B200_OK;
	}
	*handled = 1;
	return dispatch_order(order, [&](auto rt) {
		constexpr int R = decltype(rt)::value;
		auto go = [&](auto tag) {
			using S = decltype(tag);
			switch (mode) {
			case MODE_D2_AXIS1: return launch_for<S, R, MODE_D2_AXIS1>(lay, in, out, coef, inv2_1, inv2_2, inv2_3, s);
			case MODE_D2_AXIS2: return launch_for<S, R, MODE_D2_AXIS2>(lay, in, out, coef, inv2_1, inv2_2, inv2_3, s);
			case MODE_D2_AXIS3: return launch_for<S, R, MODE_D2_AXIS3>(lay, in, out, coef, inv2_1, inv2_2, inv2_3, s);
			case MODE_LAPLACIAN: return launch_for<S, R, MODE_LAPLACIAN>(lay, in, out, coef, inv2_1, inv2_2, inv2_3, s);
			default: return launch_for<S, R, MODE_PRESSURE>(lay, in, out, coef, inv2_1, inv2_2, inv2_3, s);
			}
		};
		if (in.dtype == B200_F64) return go(double{});
		return go(float{});
	});
}

}  // namespace b200

extern "C" int b200_device_status(int* status, int clear)
{
	using namespace b200;
	if (!status) return set_error(B200_ERR_ARG, "status is NULL");
	unsigned int v = 0;
	int rc = cuda_error(cudaMemcpyFromSymbol(&v, g_device_error, sizeof(v)), "cudaMemcpyFromSymbol");
	if (rc) return rc;
	*status = (int)v;
	if (clear && v) {
		const unsigned int zero = 0;
		rc = cuda_error(cudaMemcpyToSymbol(g_device_error, &zero, sizeof(zero)), "cudaMemcpyToSymbol");
	}
	return rc;
}
