// Staggered first derivative of the hpcscan_b200 C ABI: Grid::FD_D1_N1/N2/N3
// (reference src/grid.cpp:3401, 3735, 4069; stencils src/fdm.h:27-275).
//
// w[i] = ((A1 (u[i] - u[i-1]) + A2 (u[i+1] - u[i-2])) + ... + AR (u[i+R-1] - u[i-R])) * inv_d,
// the derivative at i - 1/2, on the INNER points; O2 has no A1 factor. Every operation is
// separately rounded in the reference's order, so the results are bit-identical to the CPU path.
//
// The operator reads 2R points along one axis and writes one: HBM-bound at 2 accesses per point
// (one read, one write) when each input plane or row is fetched from DRAM once. 3-D grids whose
// layout meets the TMA rules (every Grid_B200 grid) take the z-marching kernel
// (b200_zmarch.cuh, MODE_D1_AXIS1..3: TMA-staged tiles, packed FP32 pairs); the kernels below
// take 1-D and 2-D grids, 16-bit storage and the other layouts:
//  * axis 1: one thread per point, a warp on 32 consecutive i1; the 2R - 1 neighbours of a
//    row segment are L1 hits of the same cache lines;
//  * axes 2 and 3: each thread marches along the axis over a chunk of points with the last 2R
//    values in registers, so every input line is loaded once per chunk (plus 2R - 1 halo
//    lines per chunk, mostly L2 hits); a warp covers 32 consecutive i1, coalesced.
#include "b200_common.cuh"
#include "b200_stencil.cuh"

namespace b200 {

namespace {

template <typename C>
struct D1Args {
	const void* u;
	void* w;
	int64_t n1, n12;
	int64_t s1, s2, s3;
	int nx, ny, nz;   // inner extents along i1, i2, i3
	int chunk;        // points per thread along the marched axis (axes 2 and 3)
	C inv;
};

constexpr int kRowThreads = 128;
constexpr int kMarchX = 32, kMarchY = 8, kMarchUnroll = 4;

// Axis 1: one thread per inner point, blocks of 128 consecutive i1 of one (i2, i3) row.
template <typename S, int R>
__global__ void __launch_bounds__(kRowThreads) k_fd_d1_axis1(D1Args<typename Storage<S>::C> a)
{
	using C = typename Storage<S>::C;
	const int x = blockIdx.x * kRowThreads + threadIdx.x;
	if (x >= a.nx) return;
	const int64_t ii = (a.s1 + x) + (a.s2 + blockIdx.y) * a.n1 + (a.s3 + blockIdx.z) * a.n12;
	const S* __restrict__ u = static_cast<const S*>(a.u) + ii;
	auto v = [&](int k) -> C { return Storage<S>::load(__ldg(u + k)); };
	static_cast<S*>(a.w)[ii] = Storage<S>::store(d1_axis<C, R, true>(v, a.inv));
}

// Axes 2 (AXIS = 2: march along i2, the other index is i3) and 3 (march along i3, the other
// index is i2). Thread (x, o) computes the points chunk * blockIdx.z + [0, chunk) of its line.
template <typename S, int R, int AXIS>
__global__ void __launch_bounds__(kMarchX * kMarchY) k_fd_d1_march(D1Args<typename Storage<S>::C> a)
{
	using C = typename Storage<S>::C;
	const int x = blockIdx.x * kMarchX + threadIdx.x;
	const int o = blockIdx.y * kMarchY + threadIdx.y;
	const int nm = AXIS == 2 ? a.ny : a.nz;
	const int no = AXIS == 2 ? a.nz : a.ny;
	if (x >= a.nx || o >= no) return;
	const int j0 = blockIdx.z * a.chunk;
	const int j1 = min(j0 + a.chunk, nm);
	const int64_t pm = AXIS == 2 ? a.n1 : a.n12;   // stride along the marched axis
	const int64_t line = (a.s1 + x) + (AXIS == 2 ? (a.s3 + o) * a.n12 + a.s2 * a.n1
	                                             : (a.s2 + o) * a.n1 + a.s3 * a.n12);
	const S* __restrict__ u = static_cast<const S*>(a.u) + line;
	S* __restrict__ w = static_cast<S*>(a.w) + line;
	auto ld = [&](int j) -> C { return Storage<S>::load(__ldg(u + j * pm)); };

	// q[m] = u[j - R + m], m = 0..2R-1, for the output point j
	C q[2 * R];
#pragma unroll
	for (int m = 0; m < 2 * R - 1; m++) q[m + 1] = ld(j0 - R + m);
	int j = j0;
	for (; j + kMarchUnroll <= j1; j += kMarchUnroll) {
		C nx[kMarchUnroll];
#pragma unroll
		for (int t = 0; t < kMarchUnroll; t++) nx[t] = ld(j + R - 1 + t);
#pragma unroll
		for (int t = 0; t < kMarchUnroll; t++) {
#pragma unroll
			for (int m = 0; m < 2 * R - 1; m++) q[m] = q[m + 1];
			q[2 * R - 1] = nx[t];
			w[(int64_t)(j + t) * pm] = Storage<S>::store(d1_axis<C, R, true>([&](int k) { return q[R + k]; }, a.inv));
		}
	}
	for (; j < j1; j++) {
#pragma unroll
		for (int m = 0; m < 2 * R - 1; m++) q[m] = q[m + 1];
		q[2 * R - 1] = ld(j + R - 1);
		w[(int64_t)j * pm] = Storage<S>::store(d1_axis<C, R, true>([&](int k) { return q[R + k]; }, a.inv));
	}
}

// Points per thread along the marched axis: long chunks amortise the 2R - 1 halo loads, but
// the grid must still fill the GPU (at least four waves of 256-thread blocks over the SMs).
int march_chunk(int nm, int64_t lines)
{
	const int64_t blocks_per_chunk = (lines + kMarchX * kMarchY - 1) / (kMarchX * kMarchY);
	const int64_t want = 4LL * 8 * num_sms();   // 8 resident 256-thread blocks per SM
	int chunk = 64;
	while (chunk > 8 && blocks_per_chunk * ((nm + chunk - 1) / chunk) < want) chunk /= 2;
	return chunk;
}

}  // namespace

int run_fd_d1(const b200_layout* lay, int axis, int order, const b200_field& u, const b200_field& w,
		double inv_1, double inv_2, double inv_3, cudaStream_t s)
{
	if (int rc = check_layout(lay)) return rc;
	if (int rc = check_order(order)) return rc;
	if (lay->halo < order / 2)
		return set_error(B200_ERR_ARG, "layout halo %d too narrow for order %d", lay->halo, order);
	if (axis < 1 || axis > lay->dim)
		return set_error(B200_ERR_ARG, "axis %d of a %d-D grid", axis, lay->dim);
	if (int rc = check_field(u, "u")) return rc;
	if (int rc = check_field(w, "w")) return rc;
	if (u.dtype != w.dtype) return set_error(B200_ERR_UNSUPPORTED, "FD_D1: grids of different storage types");
	if (u.scale != w.scale) return set_error(B200_ERR_UNSUPPORTED, "FD_D1: grids of different scales");
	if (u.data == w.data) return set_error(B200_ERR_ARG, "FD_D1: input and output are the same array");
	const int mode = axis == 1 ? MODE_D1_AXIS1 : axis == 2 ? MODE_D1_AXIS2 : MODE_D1_AXIS3;
	int handled = 0;
	if (int rc = run_zmarch(mode, lay, order, u, w, nullptr, inv_1, inv_2, inv_3, s, &handled))
		return rc;
	if (handled) return B200_OK;
	return dispatch_dtype(u.dtype, [&](auto tag) {
		using S = decltype(tag);
		using C = typename Storage<S>::C;
		D1Args<C> a;
		a.u = u.data;
		a.w = w.data;
		a.n1 = lay->n1;
		a.n12 = lay->n1 * lay->n2;
		a.s1 = lay->s1;
		a.s2 = lay->s2;
		a.s3 = lay->s3;
		a.nx = (int)(lay->e1 - lay->s1 + 1);
		a.ny = (int)(lay->e2 - lay->s2 + 1);
		a.nz = (int)(lay->e3 - lay->s3 + 1);
		a.inv = (C)(axis == 1 ? inv_1 : axis == 2 ? inv_2 : inv_3);
		if (a.ny > 65535 || a.nz > 65535)
			return set_error(B200_ERR_UNSUPPORTED, "FD_D1: inner extents %d x %d beyond the grid limits",
					a.ny, a.nz);
		return dispatch_order(order, [&](auto rt) {
			constexpr int R = decltype(rt)::value;
			if (axis == 1) {
				a.chunk = 0;
				const dim3 grd((a.nx + kRowThreads - 1) / kRowThreads, a.ny, a.nz);
				k_fd_d1_axis1<S, R><<<grd, kRowThreads, 0, s>>>(a);
				return check_launch("k_fd_d1_axis1");
			}
			const int nm = axis == 2 ? a.ny : a.nz;
			const int no = axis == 2 ? a.nz : a.ny;
			a.chunk = march_chunk(nm, (int64_t)a.nx * no);
			const dim3 blk(kMarchX, kMarchY);
			const dim3 grd((a.nx + kMarchX - 1) / kMarchX, (no + kMarchY - 1) / kMarchY,
					(nm + a.chunk - 1) / a.chunk);
			if (axis == 2) k_fd_d1_march<S, R, 2><<<grd, blk, 0, s>>>(a);
			else k_fd_d1_march<S, R, 3><<<grd, blk, 0, s>>>(a);
			return check_launch("k_fd_d1_march");
		});
	});
}

}  // namespace b200

using namespace b200;

extern "C" int b200_fd_d1(const b200_layout* lay, int axis, int order, b200_field u, b200_field w,
		double inv_1, double inv_2, double inv_3, void* stream)
{
	return run_fd_d1(lay, axis, order, u, w, inv_1, inv_2, inv_3, as_stream(stream));
}
