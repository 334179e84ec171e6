// Grid operations of the hpcscan_b200 C ABI other than the stencils: fills, the
// anti-mirror boundary condition, the split pressure update and the FP64 norms.
#include <mutex>

#include "b200_common.cuh"

namespace b200 {

namespace {

constexpr int kRowThreads = 256;

struct Box3 {
	int64_t i1s, i2s, i3s;
	int nx, ny, nz;
};

Box3 to_box3(const b200_box* b)
{
	return Box3{b->i1s, b->i2s, b->i3s, (int)(b->i1e - b->i1s + 1), (int)(b->i2e - b->i2s + 1),
			(int)(b->i3e - b->i3s + 1)};
}

// Row index -> (i2, i3) offsets of a box; 32-bit division (boxes of fewer than 2^31 rows,
// checked by box_rows_ok on the host).
__device__ __forceinline__ void row_yz(int64_t row, int ny, int& y, int& z)
{
	const unsigned r = (unsigned)row;
	z = (int)(r / (unsigned)ny);
	y = (int)(r - (unsigned)z * (unsigned)ny);
}

int box_rows_ok(const Box3& b)
{
	if ((int64_t)b.ny * b.nz >= (1LL << 31))
		return set_error(B200_ERR_UNSUPPORTED, "box of %d x %d rows (2^31 at most)", b.ny, b.nz);
	return B200_OK;
}

// Row walk: the blocks of a grid take the rows (i2, i3) of a box, kUnroll rows at a time, and
// the threads of a block stride along i1 (coalesced). A grid of at most 8 blocks per SM, each
// thread with kUnroll independent loads in flight per step.
constexpr int kRowUnroll = 4;

int row_blocks(const Box3& b, int unroll)
{
	const int64_t rows = (int64_t)b.ny * b.nz;
	const int64_t want = (rows + unroll - 1) / unroll;
	const int64_t cap = (int64_t)num_sms() * 8;
	return (int)(want < 1 ? 1 : (want < cap ? want : cap));
}

// ---- fills ------------------------------------------------------------------------------------
template <typename S>
__global__ void __launch_bounds__(kRowThreads) k_fill_const(S* __restrict__ u, int64_t n1,
		int64_t n12, Box3 b, S val)
{
	const int64_t rows = (int64_t)b.ny * b.nz;
	for (int64_t row = blockIdx.x; row < rows; row += gridDim.x) {
		int y, z;
		row_yz(row, b.ny, y, z);
		S* dst = u + b.i1s + (b.i2s + y) * n1 + (b.i3s + z) * n12;
		for (int x = threadIdx.x; x < b.nx; x += blockDim.x) dst[x] = val;
	}
}

// Whole-array operations of the Memory test case (Grid::fillArray .. addUpdateArray).
template <typename S, int OP>
__global__ void k_array_op(S* __restrict__ out, const S* __restrict__ a, const S* __restrict__ b,
		int64_t n, S val)
{
	using A = Arith<true>;
	const int64_t stride = (int64_t)gridDim.x * blockDim.x;
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
		if constexpr (OP == B200_ARRAY_FILL) {
			out[i] = val;
		} else if constexpr (OP == B200_ARRAY_COPY) {
			out[i] = a[i];
		} else if constexpr (OP == B200_ARRAY_ADD) {
			out[i] = Storage<S>::store(A::add(Storage<S>::load(a[i]), Storage<S>::load(b[i])));
		} else if constexpr (OP == B200_ARRAY_MUL) {
			out[i] = Storage<S>::store(A::mul(Storage<S>::load(a[i]), Storage<S>::load(b[i])));
		} else {
			out[i] = Storage<S>::store(A::add(Storage<S>::load(out[i]), Storage<S>::load(a[i])));
		}
	}
}

// Point gather (receivers) and point assignment (a source term).
template <typename S>
__global__ void k_gather_points(const S* __restrict__ u, const int64_t* __restrict__ idx, int64_t n,
		S* __restrict__ out, int64_t stride)
{
	const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
	if (i < n) out[i * stride] = u[idx[i]];
}

template <typename S>
__global__ void k_set_point(S* __restrict__ u, int64_t idx, S v)
{
	u[idx] = v;
}

template <typename S>
__global__ void __launch_bounds__(kRowThreads) k_fill_separable(S* __restrict__ u, int64_t n1,
		int64_t n12, Box3 b, const double* __restrict__ v1, const double* __restrict__ v2,
		const double* __restrict__ v3, double amp)
{
	const int64_t rows = (int64_t)b.ny * b.nz;
	for (int64_t row = blockIdx.x; row < rows; row += gridDim.x) {
		int y, z;
		row_yz(row, b.ny, y, z);
		const double w2 = v2[y], w3 = v3[z];
		S* dst = u + b.i1s + (b.i2s + y) * n1 + (b.i3s + z) * n12;
		// (((amp * v1) * v2) * v3), each product rounded in FP64, then one rounding to S
		for (int x = threadIdx.x; x < b.nx; x += blockDim.x)
			dst[x] = Storage<S>::store_d(__dmul_rn(__dmul_rn(__dmul_rn(amp, v1[x]), w2), w3));
	}
}

// ---- boundary condition ----------------------------------------------------------------------
struct BcArgs {
	int64_t n1, n12;
	int64_t s[3], e[3];
	int halo, dim, faces;
};

// Phase A: every halo value of the active faces, computed from the values before the
// boundary condition. A mirror point that an earlier face (in the reference's order
// I1HALO1, I1HALO2, I2HALO1, I2HALO2, I3HALO1, I3HALO2) sets to zero reads as zero.
// Reads touch inner points only and writes touch halo points only, so one launch is safe.
// Valid when every used axis has at least halo + 2 inner points (checked by the caller).
//
// Block partition (kBcThreads threads per block, every index decoded once per block):
//   [0, nbx)            x faces: L = 2 halo lanes (side, k) per row (i2, i3), kBcThreads / L
//                       rows per block (L = 2 for the boundary planes)
//   [nbx, nbx+nby)      y faces: one run of up to kBcThreads i1 values per (i3, side), all k
//   [nbx+nby, +nbz)     z faces: one run of up to kBcThreads i1 values per (i2, side), all k
constexpr int kBcThreads = 256;

struct BcPart {
	int nbx, nby, nbz;     // blocks per group
	int nchunk;            // i1 runs per row for y/z groups
	int lanes;             // x faces: lanes per row
};

BcPart bc_partition(const BcArgs& a, bool planes)
{
	const int nx = (int)(a.e[0] - a.s[0] + 1), ny = (int)(a.e[1] - a.s[1] + 1),
	          nz = (int)(a.e[2] - a.s[2] + 1);
	BcPart p;
	p.lanes = planes ? 2 : 2 * a.halo;
	p.nchunk = (nx + kBcThreads - 1) / kBcThreads;
	const int rows_per_block = kBcThreads / p.lanes;
	p.nbx = (ny * nz + rows_per_block - 1) / rows_per_block;
	p.nby = a.dim >= 2 ? p.nchunk * nz * 2 : 0;
	p.nbz = a.dim >= 3 ? p.nchunk * ny * 2 : 0;
	return p;
}

template <typename S>
__global__ void __launch_bounds__(kBcThreads) k_bc_halos(S* __restrict__ u, BcArgs a, BcPart p)
{
	constexpr int KMAX = 8;
	const int R = a.halo;
	const int ny = (int)(a.e[1] - a.s[1] + 1);
	const bool lo_x = a.faces & 1, hi_x = a.faces & 2, lo_y = a.faces & 4, hi_y = a.faces & 8;
	int b = blockIdx.x;
	if (b < p.nbx) {
		const int lane = threadIdx.x % p.lanes, rib = threadIdx.x / p.lanes;
		if (rib >= kBcThreads / p.lanes) return;
		const int side = lane / R, k = lane % R + 1;
		if (!(a.faces & (1 << side))) return;
		const int row = b * (kBcThreads / p.lanes) + rib;
		const int nrow = ny * (int)(a.e[2] - a.s[2] + 1);
		if (row >= nrow) return;
		const int64_t base = (a.s[1] + row % ny) * a.n1 + (a.s[2] + row / ny) * a.n12;
		const int64_t h = side ? a.e[0] + k : a.s[0] - k, m = side ? a.e[0] - k : a.s[0] + k;
		u[base + h] = Storage<S>::store(-Storage<S>::load(u[base + m]));
		return;
	}
	b -= p.nbx;
	const int axis = (b < p.nby) ? 1 : 2;
	if (axis == 2) b -= p.nby;
	const int chunk = b % p.nchunk;
	const int r = b / p.nchunk;
	const int side = r % 2;
	const int line = r / 2;                      // i3 (y faces) or i2 (z faces), inner offset
	const int x = chunk * kBcThreads + threadIdx.x;
	if (a.s[0] + x > a.e[0]) return;
	const int64_t i1 = a.s[0] + x;
	S mv[KMAX];
	if (axis == 1) {
		if (!(a.faces & (4 << side))) return;
		const int64_t i3 = a.s[2] + line;
		const bool zero = (lo_x && i1 == a.s[0]) || (hi_x && i1 == a.e[0]);
		const int64_t col = i1 + i3 * a.n12;
#pragma unroll
		for (int k = 1; k <= KMAX; k++)
			if (k <= R) mv[k - 1] = zero ? S(0.0f) : u[col + (side ? a.e[1] - k : a.s[1] + k) * a.n1];
#pragma unroll
		for (int k = 1; k <= KMAX; k++)
			if (k <= R)
				u[col + (side ? a.e[1] + k : a.s[1] - k) * a.n1] = Storage<S>::store(-Storage<S>::load(mv[k - 1]));
	} else {
		if (!(a.faces & (16 << side))) return;
		const int64_t i2 = a.s[1] + line;
		const bool zero = (lo_x && i1 == a.s[0]) || (hi_x && i1 == a.e[0]) ||
		                  (lo_y && i2 == a.s[1]) || (hi_y && i2 == a.e[1]);
		const int64_t col = i1 + i2 * a.n1;
#pragma unroll
		for (int k = 1; k <= KMAX; k++)
			if (k <= R) mv[k - 1] = zero ? S(0.0f) : u[col + (side ? a.e[2] - k : a.s[2] + k) * a.n12];
#pragma unroll
		for (int k = 1; k <= KMAX; k++)
			if (k <= R)
				u[col + (side ? a.e[2] + k : a.s[2] - k) * a.n12] = Storage<S>::store(-Storage<S>::load(mv[k - 1]));
	}
}

// Phase B: the boundary planes (first/last inner point of each active face) set to zero,
// same block partition with one lane per side for the x faces.
template <typename S>
__global__ void __launch_bounds__(kBcThreads) k_bc_planes(S* __restrict__ u, BcArgs a, BcPart p)
{
	const int ny = (int)(a.e[1] - a.s[1] + 1);
	int b = blockIdx.x;
	if (b < p.nbx) {
		const int side = threadIdx.x % 2;
		if (!(a.faces & (1 << side))) return;
		const int row = b * (kBcThreads / 2) + threadIdx.x / 2;
		const int nrow = ny * (int)(a.e[2] - a.s[2] + 1);
		if (row >= nrow) return;
		const int64_t base = (a.s[1] + row % ny) * a.n1 + (a.s[2] + row / ny) * a.n12;
		u[base + (side ? a.e[0] : a.s[0])] = S(0.0f);
		return;
	}
	b -= p.nbx;
	const int axis = (b < p.nby) ? 1 : 2;
	if (axis == 2) b -= p.nby;
	const int chunk = b % p.nchunk;
	int r = b / p.nchunk;
	const int side = r % 2;
	r /= 2;
	const int x = chunk * kBcThreads + threadIdx.x;
	if (a.s[0] + x > a.e[0]) return;
	const int64_t i1 = a.s[0] + x;
	if (axis == 1) {
		if (!(a.faces & (4 << side))) return;
		u[i1 + (side ? a.e[1] : a.s[1]) * a.n1 + (a.s[2] + r) * a.n12] = S(0.0f);
	} else {
		if (!(a.faces & (16 << side))) return;
		u[i1 + (a.s[1] + r) * a.n1 + (side ? a.e[2] : a.s[2]) * a.n12] = S(0.0f);
	}
}

// The whole anti-mirror condition in one launch, for a single-rank 3-D grid whose axes all have
// at least 2 halo + 2 inner points (phase A's partition). Phase A reads values from before the
// boundary planes are zeroed; here the zeroing happens in the same launch, so each point that
// is both read and zeroed is zeroed by its only reader, after the read:
//  * i1 faces (one (row, side, distance) per thread): the mirror point xm = s1 + k (e1 - k) is
//    read, its halo written; xm is zeroed by this thread when it lies on an i2 or i3 boundary
//    plane; on an i3 boundary plane within the i2 band (rows s2+1..s2+R, e2-R..e2-1) this thread
//    also writes xm's i2 halo, which would otherwise need a second reader; the k = 1 lane zeroes
//    the i1 boundary point of its row;
//  * i2 faces (column (x, z)): columns with x in the i1 band on an i3 boundary plane are left to
//    the i1 faces; the others read, write their halos, zero the i2 boundary point (outside the
//    i1 band) and, on an i3 boundary plane, the mirror points they read;
//  * i3 faces (column (x, y)): read, write the halos, and zero the i3 boundary point unless
//    x is in the i1 band or on an i1 boundary line, or y in the i2 band or on an i2 line.
// Mirror values from a boundary line an earlier face zeroes are -0 without a read, as in phase A.
//
// Launch grid (nbx + 4 nchunk, ceil(max(ny, nz) / kBcLines)), the halo width R a template
// parameter so that every index comes from constant divisions: blockIdx.y * kBcLines + l,
// l < kBcLines, are the block's lines (i3 - s3 for the i1 and i2 faces, i2 - s2 for the i3
// faces) and blockIdx.x the part:
//   [0, nbx)                      i1 faces of plane i3: 2R lanes (side, k) per i2 row,
//                                 kBcThreads / 2R rows per block
//   [nbx, nbx + 2 nchunk)         i2 faces of plane i3: one run of kBcThreads i1 per (run, side)
//   [nbx + 2 nchunk, + 2 nchunk)  i3 faces of row i2: the same runs
// A thread reads its values of every line of the block before it writes any: the lines share
// no point, so the order is free, and the reads are in flight together (one line per block
// left each thread a single dependent read and the launch latency-bound: 22.9 us at 512^3 O8).
constexpr int kBcLines = 4;

template <typename S, int R>
__global__ void __launch_bounds__(kBcThreads) k_bc_one(S* __restrict__ u, BcArgs a, int nbx, int nchunk)
{
	constexpr int L = 2 * R, RPB = kBcThreads / L;
	const int ny = (int)(a.e[1] - a.s[1] + 1), nz = (int)(a.e[2] - a.s[2] + 1);
	const int64_t s1 = a.s[0], e1 = a.e[0], s2 = a.s[1], e2 = a.e[1], s3 = a.s[2], e3 = a.e[2];
	const int64_t n1 = a.n1, n12 = a.n12;
	auto neg = [](S v) { return Storage<S>::store(-Storage<S>::load(v)); };
	auto xband = [&](int64_t x) { return (x > s1 && x <= s1 + R) || (x < e1 && x >= e1 - R); };
	auto yband = [&](int64_t y) { return (y > s2 && y <= s2 + R) || (y < e2 && y >= e2 - R); };
	const int line0 = (int)blockIdx.y * kBcLines;
	int b = (int)blockIdx.x;
	if (b < nbx) {
		const int rib = (int)threadIdx.x / L, lane = (int)threadIdx.x % L;
		const int yr = b * RPB + rib;
		if (rib >= RPB || yr >= ny) return;
		const int side = lane / R, k = lane % R + 1;
		const int64_t y = s2 + yr;
		const int64_t xm = side ? e1 - k : s1 + k;
		const bool yplane = y == s2 || y == e2;
		S v[kBcLines];
#pragma unroll
		for (int l = 0; l < kBcLines; l++)
			if (line0 + l < nz) v[l] = u[y * n1 + (s3 + line0 + l) * n12 + xm];
#pragma unroll
		for (int l = 0; l < kBcLines; l++) {
			if (line0 + l >= nz) break;
			const int64_t z = s3 + line0 + l;
			const int64_t base = y * n1 + z * n12;
			u[base + (side ? e1 + k : s1 - k)] = neg(v[l]);
			const bool zplane = z == s3 || z == e3;
			if (zplane && yband(y)) u[(y <= s2 + R ? 2 * s2 - y : 2 * e2 - y) * n1 + z * n12 + xm] = neg(v[l]);
			if (yplane || zplane) u[base + xm] = S(0.0f);
			if (k == 1) u[base + (side ? e1 : s1)] = S(0.0f);
		}
		return;
	}
	b -= nbx;
	const int axis = (b < 2 * nchunk) ? 1 : 2;
	if (axis == 2) b -= 2 * nchunk;
	const int side = b & 1, chunk = b >> 1;
	const int nline = axis == 1 ? nz : ny;
	const int x = chunk * kBcThreads + (int)threadIdx.x;
	if (s1 + x > e1) return;
	const int64_t i1 = s1 + x;
	const bool xline = i1 == s1 || i1 == e1;
	S mv[kBcLines][R];
	if (axis == 1) {
		const bool xb = xband(i1);
		const int64_t bnd = side ? e2 : s2;
#pragma unroll
		for (int l = 0; l < kBcLines; l++) {
			const int64_t i3 = s3 + line0 + l;
			if (line0 + l >= nline || ((i3 == s3 || i3 == e3) && xb)) continue;
			const int64_t col = i1 + i3 * n12;
#pragma unroll
			for (int k = 1; k <= R; k++)
				mv[l][k - 1] = xline ? S(0.0f) : u[col + (side ? bnd - k : bnd + k) * n1];
		}
#pragma unroll
		for (int l = 0; l < kBcLines; l++) {
			const int64_t i3 = s3 + line0 + l;
			const bool zplane = i3 == s3 || i3 == e3;
			if (line0 + l >= nline || (zplane && xb)) continue;
			const int64_t col = i1 + i3 * n12;
#pragma unroll
			for (int k = 1; k <= R; k++) u[col + (side ? bnd + k : bnd - k) * n1] = neg(mv[l][k - 1]);
			if (!xb) u[col + bnd * n1] = S(0.0f);
			if (zplane) {
#pragma unroll
				for (int k = 1; k <= R; k++) u[col + (side ? bnd - k : bnd + k) * n1] = S(0.0f);
			}
		}
	} else {
		const int64_t bnd = side ? e3 : s3;
#pragma unroll
		for (int l = 0; l < kBcLines; l++) {
			if (line0 + l >= nline) continue;
			const int64_t i2 = s2 + line0 + l;
			const bool yline = i2 == s2 || i2 == e2;
			const int64_t col = i1 + i2 * n1;
#pragma unroll
			for (int k = 1; k <= R; k++)
				mv[l][k - 1] = (xline || yline) ? S(0.0f) : u[col + (side ? bnd - k : bnd + k) * n12];
		}
#pragma unroll
		for (int l = 0; l < kBcLines; l++) {
			if (line0 + l >= nline) continue;
			const int64_t i2 = s2 + line0 + l;
			const bool yline = i2 == s2 || i2 == e2;
			const int64_t col = i1 + i2 * n1;
#pragma unroll
			for (int k = 1; k <= R; k++) u[col + (side ? bnd + k : bnd - k) * n12] = neg(mv[l][k - 1]);
			if (!(xline || yline || xband(i1) || yband(i2))) u[col + bnd * n12] = S(0.0f);
		}
	}
}

// k_bc_one for halo widths 1..8 (FD orders 2..16); *handled stays 0 for other widths and for
// grids beyond the launch's line limit, which take the two-launch form.
template <typename S>
int launch_bc_one(S* u, const BcArgs& a, cudaStream_t s, int* handled)
{
	*handled = 0;
	const int64_t nx = a.e[0] - a.s[0] + 1, ny = a.e[1] - a.s[1] + 1, nz = a.e[2] - a.s[2] + 1;
	if (a.halo < 1 || a.halo > 8 || ny > 65535 || nz > 65535) return B200_OK;
	*handled = 1;
	const int nchunk = (int)((nx + kBcThreads - 1) / kBcThreads);
	auto go = [&](auto rt) {
		constexpr int R = decltype(rt)::value;
		constexpr int RPB = kBcThreads / (2 * R);
		const int nbx = (int)((ny + RPB - 1) / RPB);
		const int64_t nline = ny > nz ? ny : nz;
		const dim3 grd(nbx + 4 * nchunk, (unsigned)((nline + kBcLines - 1) / kBcLines));
		k_bc_one<S, R><<<grd, kBcThreads, 0, s>>>(u, a, nbx, nchunk);
		return check_launch("k_bc_one");
	};
	switch (a.halo) {
	case 1: return go(std::integral_constant<int, 1>{});
	case 2: return go(std::integral_constant<int, 2>{});
	case 3: return go(std::integral_constant<int, 3>{});
	case 4: return go(std::integral_constant<int, 4>{});
	case 5: return go(std::integral_constant<int, 5>{});
	case 6: return go(std::integral_constant<int, 6>{});
	case 7: return go(std::integral_constant<int, 7>{});
	default: return go(std::integral_constant<int, 8>{});
	}
}

// Sequential form for tiny grids (an axis with fewer than halo + 2 inner points): one face
// per launch in the reference order, each thread owning one line normal to the face.
template <typename S>
__global__ void k_bc_face(S* __restrict__ u, BcArgs a, int face)
{
	const int axis = face / 2, side = face % 2;
	const int64_t nx = a.e[0] - a.s[0] + 1, ny = a.e[1] - a.s[1] + 1, nz = a.e[2] - a.s[2] + 1;
	const int64_t lines = (axis == 0) ? ny * nz : (axis == 1) ? nx * nz : nx * ny;
	const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
	if (t >= lines) return;
	int64_t base, st, b;
	if (axis == 0) {
		base = (a.s[1] + t % ny) * a.n1 + (a.s[2] + t / ny) * a.n12;
		st = 1;
		b = side ? a.e[0] : a.s[0];
	} else if (axis == 1) {
		base = (a.s[0] + t % nx) + (a.s[2] + t / nx) * a.n12;
		st = a.n1;
		b = side ? a.e[1] : a.s[1];
	} else {
		base = (a.s[0] + t % nx) + (a.s[1] + t / nx) * a.n1;
		st = a.n12;
		b = side ? a.e[2] : a.s[2];
	}
	u[base + b * st] = S(0.0f);
	for (int k = 1; k <= a.halo; k++) {
		const int64_t h = side ? b + k : b - k, m = side ? b - k : b + k;
		u[base + h * st] = Storage<S>::store(-Storage<S>::load(u[base + m * st]));
	}
}

// ---- split update ------------------------------------------------------------------------------
template <typename S, bool EXACT>
__global__ void __launch_bounds__(kRowThreads) k_update_pressure(S* __restrict__ prn,
		const S* __restrict__ prc, const S* __restrict__ coef, const S* __restrict__ lapla,
		int64_t n1, int64_t n12, Box3 b, float coef_scale)
{
	using C = typename Storage<S>::C;
	const int64_t rows = (int64_t)b.ny * b.nz;
	for (int64_t r0 = (int64_t)blockIdx.x * kRowUnroll; r0 < rows; r0 += (int64_t)gridDim.x * kRowUnroll) {
		for (int x = threadIdx.x; x < b.nx; x += blockDim.x) {
			int64_t ii[kRowUnroll];
			C pc[kRowUnroll], pn[kRowUnroll], cf[kRowUnroll], lp[kRowUnroll];
#pragma unroll
			for (int k = 0; k < kRowUnroll; k++) {
				int y, z;
				row_yz(r0 + k < rows ? r0 + k : rows - 1, b.ny, y, z);
				ii[k] = (b.i1s + x) + (b.i2s + y) * n1 + (b.i3s + z) * n12;
				pc[k] = Storage<S>::load(prc[ii[k]]);
				pn[k] = Storage<S>::load(prn[ii[k]]);
				cf[k] = Storage<S>::load(coef[ii[k]]);
				lp[k] = Storage<S>::load(lapla[ii[k]]);
			}
#pragma unroll
			for (int k = 0; k < kRowUnroll; k++) {
				if (r0 + k >= rows) break;
				C c = cf[k];
				if (coef_scale != 1.0f) c = c * (C)coef_scale;
				prn[ii[k]] = Storage<S>::store(leapfrog<C, EXACT>(pc[k], pn[k], c, lp[k]));
			}
		}
	}
}

// ---- reductions -------------------------------------------------------------------------------
enum RedOp { RED_SUM_ABS = 0, RED_L1 = 1, RED_MAX_ERR = 2, RED_MIN_MAX = 3, RED_L1_SEP = 4 };

constexpr int kRedThreads = 256;

struct RedArgs {
	int64_t n1, n12;
	Box3 b;
	double s1, s2;                  // field scales
	double max_err_float;
	const double* v1;               // separable reference tables (RED_L1_SEP)
	const double* v2;
	const double* v3;
	double amp;
	int ref_dtype;
};

__device__ __forceinline__ double warp_sum(double v)
{
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}
__device__ __forceinline__ double warp_max(double v)
{
	for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
	return v;
}
__device__ __forceinline__ double warp_min(double v)
{
	for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
	return v;
}

// combine two accumulators (a: first result, b: second) over the block
template <int OP>
__device__ void block_combine(double& a, double& b)
{
	__shared__ double sa[kRedThreads / 32], sb[kRedThreads / 32];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	if (OP == RED_MAX_ERR) {
		a = warp_max(a);
	} else if (OP == RED_MIN_MAX) {
		a = warp_min(a);
		b = warp_max(b);
	} else {
		a = warp_sum(a);
		b = warp_sum(b);
	}
	if (lane == 0) {
		sa[w] = a;
		sb[w] = b;
	}
	__syncthreads();
	if (w == 0) {
		a = lane < kRedThreads / 32 ? sa[lane] : (OP == RED_MAX_ERR ? -1.0e308 : (OP == RED_MIN_MAX ? 1.0e308 : 0.0));
		b = lane < kRedThreads / 32 ? sb[lane] : (OP == RED_MIN_MAX ? -1.0e308 : 0.0);
		if (OP == RED_MAX_ERR) {
			a = warp_max(a);
		} else if (OP == RED_MIN_MAX) {
			a = warp_min(a);
			b = warp_max(b);
		} else {
			a = warp_sum(a);
			b = warp_sum(b);
		}
	}
}

template <typename S>
__device__ __forceinline__ double ref_value(const RedArgs& r, int x, int y, int z)
{
	const double v = __dmul_rn(__dmul_rn(__dmul_rn(r.amp, r.v1[x]), r.v2[y]), r.v3[z]);
	switch (r.ref_dtype) {
	case B200_F32: return (double)__double2float_rn(v);
	case B200_F16: return (double)__half2float(__double2half(v));
	case B200_BF16: return (double)__bfloat162float(__double2bfloat16(v));
	default: return v;
	}
}

// Stage 1: one partial (pair) per block; the blocks walk the rows (i2, i3) of the box
// kRowUnroll at a time, threads along i1 (coalesced, kRowUnroll loads in flight per thread).
// Deterministic for a given grid size.
template <typename S, int OP>
__global__ void __launch_bounds__(kRedThreads) k_reduce(const S* __restrict__ u1,
		const S* __restrict__ u2, RedArgs r, double2* __restrict__ partial)
{
	constexpr bool TWO = (OP == RED_L1 || OP == RED_MAX_ERR);
	double a = (OP == RED_MAX_ERR) ? -(double)3.402823466e+38f : (OP == RED_MIN_MAX ? 1.0e308 : 0.0);
	double b = (OP == RED_MIN_MAX) ? -1.0e308 : 0.0;
	const int64_t rows = (int64_t)r.b.ny * r.b.nz;
	for (int64_t r0 = (int64_t)blockIdx.x * kRowUnroll; r0 < rows; r0 += (int64_t)gridDim.x * kRowUnroll) {
		int yk[kRowUnroll], zk[kRowUnroll];
		int64_t base[kRowUnroll];
#pragma unroll
		for (int k = 0; k < kRowUnroll; k++) {
			const int64_t row = r0 + k < rows ? r0 + k : rows - 1;
			row_yz(row, r.b.ny, yk[k], zk[k]);
			base[k] = r.b.i1s + (r.b.i2s + yk[k]) * r.n1 + (r.b.i3s + zk[k]) * r.n12;
		}
		for (int x = threadIdx.x; x < r.b.nx; x += blockDim.x) {
			double w1[kRowUnroll], w2[kRowUnroll];
#pragma unroll
			for (int k = 0; k < kRowUnroll; k++) {
				w1[k] = (double)Storage<S>::load(u1[base[k] + x]) * r.s1;
				if constexpr (TWO) w2[k] = (double)Storage<S>::load(u2[base[k] + x]) * r.s2;
			}
#pragma unroll
			for (int k = 0; k < kRowUnroll; k++) {
				if (r0 + k >= rows) break;
				const double v1 = w1[k];
				if constexpr (OP == RED_SUM_ABS) {
					a += fabs(v1);
				} else if constexpr (OP == RED_MIN_MAX) {
					a = fmin(a, v1);
					b = fmax(b, v1);
				} else {
					double v2;
					if constexpr (OP == RED_L1_SEP) v2 = ref_value<S>(r, x, yk[k], zk[k]);
					else v2 = w2[k];
					if constexpr (OP == RED_L1 || OP == RED_L1_SEP) {
						a += fabs(v1 - v2);
						b += fabs(v2);
					} else {   // RED_MAX_ERR (src/grid.cpp:2031-2043)
						double e;
						if (fabsf((float)v2) < (float)r.max_err_float) e = fabs(v1 - v2);
						else e = fabs(v1 - v2) / fabs(v2);
						a = fmax(a, e);
					}
				}
			}
		}
	}
	block_combine<OP>(a, b);
	if (threadIdx.x == 0) partial[blockIdx.x] = make_double2(a, b);
}

template <int OP>
__global__ void __launch_bounds__(kRedThreads) k_reduce_final(const double2* __restrict__ partial,
		int n, double2* __restrict__ out)
{
	double a = (OP == RED_MAX_ERR) ? -(double)3.402823466e+38f : (OP == RED_MIN_MAX ? 1.0e308 : 0.0);
	double b = (OP == RED_MIN_MAX) ? -1.0e308 : 0.0;
	for (int i = threadIdx.x; i < n; i += blockDim.x) {
		const double2 p = partial[i];
		if (OP == RED_MAX_ERR) {
			a = fmax(a, p.x);
		} else if (OP == RED_MIN_MAX) {
			a = fmin(a, p.x);
			b = fmax(b, p.y);
		} else {
			a += p.x;
			b += p.y;
		}
	}
	block_combine<OP>(a, b);
	if (threadIdx.x == 0) *out = make_double2(a, b);
}

template <int OP>
int run_reduce(const b200_layout* lay, const b200_field& u1, const b200_field* u2,
		const b200_box* box, RedArgs r, double* out_a, double* out_b, void* stream)
{
	if (int rc = check_layout(lay)) return rc;
	if (int rc = check_box(lay, box)) return rc;
	if (int rc = check_field(u1, "u1")) return rc;
	if (u2) {
		if (int rc = check_field(*u2, "u2")) return rc;
		if (u2->dtype != u1.dtype)
			return set_error(B200_ERR_UNSUPPORTED, "norm of two grids of different storage types");
	}
	r.n1 = lay->n1;
	r.n12 = lay->n1 * lay->n2;
	r.b = to_box3(box);
	if (int rc = box_rows_ok(r.b)) return rc;
	r.s1 = u1.scale;
	r.s2 = u2 ? u2->scale : 1.0;
	const int blocks = row_blocks(r.b, kRowUnroll);
	void* scr;
	if (int rc = scratch(sizeof(double2) * (blocks + 1), &scr)) return rc;
	double2* partial = reinterpret_cast<double2*>(scr);
	double2* result = partial + blocks;
	cudaStream_t s = as_stream(stream);
	int rc = dispatch_dtype(u1.dtype, [&](auto tag) {
		using S = decltype(tag);
		k_reduce<S, OP><<<blocks, kRedThreads, 0, s>>>(static_cast<const S*>(u1.data),
				u2 ? static_cast<const S*>(u2->data) : nullptr, r, partial);
		return check_launch("k_reduce");
	});
	if (rc) return rc;
	k_reduce_final<OP><<<1, kRedThreads, 0, s>>>(partial, blocks, result);
	if ((rc = check_launch("k_reduce_final"))) return rc;
	void* host;
	if ((rc = host_staging(sizeof(double2), &host))) return rc;
	if ((rc = cuda_error(cudaMemcpyAsync(host, result, sizeof(double2), cudaMemcpyDeviceToHost, s),
				 "cudaMemcpyAsync(norm)")))
		return rc;
	if ((rc = cuda_error(cudaStreamSynchronize(s), "cudaStreamSynchronize(norm)"))) return rc;
	const double2 v = *reinterpret_cast<double2*>(host);
	if (out_a) *out_a = v.x;
	if (out_b) *out_b = v.y;
	return B200_OK;
}

int upload_tables(const b200_box* box, const double* v1, const double* v2, const double* v3,
		cudaStream_t s, size_t offset_bytes, double** d1, double** d2, double** d3)
{
	if (!v1 || !v2 || !v3) return set_error(B200_ERR_ARG, "NULL table");
	const size_t n1 = box->i1e - box->i1s + 1, n2 = box->i2e - box->i2s + 1,
	             n3 = box->i3e - box->i3s + 1;
	void* scr;
	const size_t need = offset_bytes + (n1 + n2 + n3) * sizeof(double);
	if (int rc = scratch(need, &scr)) return rc;
	double* t = reinterpret_cast<double*>(static_cast<char*>(scr) + offset_bytes);
	*d1 = t;
	*d2 = t + n1;
	*d3 = t + n1 + n2;
	int rc = cuda_error(cudaMemcpyAsync(*d1, v1, n1 * sizeof(double), cudaMemcpyHostToDevice, s), "tables");
	if (!rc) rc = cuda_error(cudaMemcpyAsync(*d2, v2, n2 * sizeof(double), cudaMemcpyHostToDevice, s), "tables");
	if (!rc) rc = cuda_error(cudaMemcpyAsync(*d3, v3, n3 * sizeof(double), cudaMemcpyHostToDevice, s), "tables");
	return rc;
}

}  // namespace

// Host entry used by the propagator step (b200_stencil.cu).
int apply_boundary(const b200_layout* lay, const b200_field& u, int bc_type, int faces,
		cudaStream_t s)
{
	if (bc_type == B200_NO_BOUND_COND) return B200_OK;
	if (bc_type != B200_BOUND_COND_ANTI_MIRROR)
		return set_error(B200_ERR_ARG, "invalid boundary condition type %d", bc_type);
	BcArgs a;
	a.n1 = lay->n1;
	a.n12 = lay->n1 * lay->n2;
	a.s[0] = lay->s1; a.s[1] = lay->s2; a.s[2] = lay->s3;
	a.e[0] = lay->e1; a.e[1] = lay->e2; a.e[2] = lay->e3;
	a.halo = lay->halo;
	a.dim = lay->dim;
	a.faces = faces & 0x3F;
	if (a.halo == 0 || a.faces == 0) return B200_OK;
	bool small = false;
	for (int d = 0; d < lay->dim; d++) small |= (a.e[d] - a.s[d] + 1) < (a.halo + 2);
	return dispatch_dtype(u.dtype, [&](auto tag) {
		using S = decltype(tag);
		S* p = static_cast<S*>(u.data);
		if (small) {
			for (int f = 0; f < 2 * lay->dim; f++) {
				if (!(a.faces & (1 << f))) continue;
				const int axis = f / 2;
				const int64_t nx = a.e[0] - a.s[0] + 1, ny = a.e[1] - a.s[1] + 1,
				              nz = a.e[2] - a.s[2] + 1;
				const int64_t lines = (axis == 0) ? ny * nz : (axis == 1) ? nx * nz : nx * ny;
				k_bc_face<S><<<(unsigned)((lines + 127) / 128), 128, 0, s>>>(p, a, f);
				if (int rc = check_launch("k_bc_face")) return rc;
			}
			return B200_OK;
		}
		const BcPart ph = bc_partition(a, false), pp = bc_partition(a, true);
		bool one = lay->dim == 3 && a.faces == 0x3F;
		for (int d = 0; d < 3; d++) one = one && (a.e[d] - a.s[d] + 1) >= 2 * a.halo + 2;
		if (one) {
			int handled = 0;
			const int rc = launch_bc_one<S>(p, a, s, &handled);
			if (handled) return rc;
		}
		k_bc_halos<S><<<ph.nbx + ph.nby + ph.nbz, kBcThreads, 0, s>>>(p, a, ph);
		if (int rc = check_launch("k_bc_halos")) return rc;
		k_bc_planes<S><<<pp.nbx + pp.nby + pp.nbz, kBcThreads, 0, s>>>(p, a, pp);
		return check_launch("k_bc_planes");
	});
}

// The boundary planes of the anti-mirror condition alone (its phase B): after a fused
// propagator step, prc's inner boundary points become zero as applyBoundaryCondition leaves them.
int apply_boundary_planes(const b200_layout* lay, const b200_field& u, int faces, cudaStream_t s)
{
	BcArgs a;
	a.n1 = lay->n1;
	a.n12 = lay->n1 * lay->n2;
	a.s[0] = lay->s1; a.s[1] = lay->s2; a.s[2] = lay->s3;
	a.e[0] = lay->e1; a.e[1] = lay->e2; a.e[2] = lay->e3;
	a.halo = lay->halo;
	a.dim = lay->dim;
	a.faces = faces & 0x3F;
	if (a.faces == 0) return B200_OK;
	return dispatch_dtype(u.dtype, [&](auto tag) {
		using S = decltype(tag);
		const BcPart pp = bc_partition(a, true);
		k_bc_planes<S><<<pp.nbx + pp.nby + pp.nbz, kBcThreads, 0, s>>>(static_cast<S*>(u.data), a, pp);
		return check_launch("k_bc_planes");
	});
}

}  // namespace b200

using namespace b200;

extern "C" {

int b200_fill_const(const b200_layout* lay, b200_field u, const b200_box* box, double val,
		void* stream)
{
	if (int rc = check_layout(lay)) return rc;
	if (int rc = check_box(lay, box)) return rc;
	if (int rc = check_field(u, "u")) return rc;
	const Box3 b = to_box3(box);
	if (int rc = box_rows_ok(b)) return rc;
	const double v = val / (double)u.scale;
	return dispatch_dtype(u.dtype, [&](auto tag) {
		using S = decltype(tag);
		const S sv = host_store<S>(v);
		k_fill_const<S><<<row_blocks(b, 1), kRowThreads, 0, as_stream(stream)>>>(
				static_cast<S*>(u.data), lay->n1, lay->n1 * lay->n2, b, sv);
		return check_launch("k_fill_const");
	});
}

int b200_array_op(int op, int64_t n, b200_field out, b200_field in1, b200_field in2, double val,
		void* stream)
{
	if (op < B200_ARRAY_FILL || op > B200_ARRAY_ADD_UPDATE)
		return set_error(B200_ERR_ARG, "array operation %d", op);
	if (n < 0) return set_error(B200_ERR_ARG, "array size %lld", (long long)n);
	if (int rc = check_field(out, "out")) return rc;
	const bool one = op == B200_ARRAY_COPY || op == B200_ARRAY_ADD_UPDATE;
	const bool two = op == B200_ARRAY_ADD || op == B200_ARRAY_MUL;
	if (one || two) {
		if (int rc = check_field(in1, "in1")) return rc;
		if (in1.dtype != out.dtype) return set_error(B200_ERR_UNSUPPORTED, "mixed storage types");
	}
	if (two) {
		if (int rc = check_field(in2, "in2")) return rc;
		if (in2.dtype != out.dtype) return set_error(B200_ERR_UNSUPPORTED, "mixed storage types");
	}
	if (op != B200_ARRAY_FILL && (out.scale != 1.0f || in1.scale != 1.0f || (two && in2.scale != 1.0f)))
		return set_error(B200_ERR_UNSUPPORTED, "array operations on scaled fields");
	if (n == 0) return B200_OK;
	int blocks = num_sms() * 4;
	if ((int64_t)blocks * kRowThreads > n) blocks = (int)((n + kRowThreads - 1) / kRowThreads);
	cudaStream_t s = as_stream(stream);
	return dispatch_dtype(out.dtype, [&](auto tag) {
		using S = decltype(tag);
		S* o = static_cast<S*>(out.data);
		const S* a = static_cast<const S*>(in1.data);
		const S* b = static_cast<const S*>(in2.data);
		const S v = host_store<S>(val / (double)out.scale);
		switch (op) {
		case B200_ARRAY_FILL: k_array_op<S, B200_ARRAY_FILL><<<blocks, kRowThreads, 0, s>>>(o, a, b, n, v); break;
		case B200_ARRAY_COPY: k_array_op<S, B200_ARRAY_COPY><<<blocks, kRowThreads, 0, s>>>(o, a, b, n, v); break;
		case B200_ARRAY_ADD: k_array_op<S, B200_ARRAY_ADD><<<blocks, kRowThreads, 0, s>>>(o, a, b, n, v); break;
		case B200_ARRAY_MUL: k_array_op<S, B200_ARRAY_MUL><<<blocks, kRowThreads, 0, s>>>(o, a, b, n, v); break;
		default: k_array_op<S, B200_ARRAY_ADD_UPDATE><<<blocks, kRowThreads, 0, s>>>(o, a, b, n, v); break;
		}
		return check_launch("k_array_op");
	});
}

int b200_gather_points(b200_field u, const int64_t* idx, int64_t n, void* out, int64_t stride,
		void* stream)
{
	if (int rc = check_field(u, "u")) return rc;
	if (n < 0 || (n > 0 && (!idx || !out)) || stride < 1)
		return set_error(B200_ERR_ARG, "gather: n %lld, stride %lld", (long long)n, (long long)stride);
	if (n == 0) return B200_OK;
	return dispatch_dtype(u.dtype, [&](auto tag) {
		using S = decltype(tag);
		k_gather_points<S><<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream)>>>(
				static_cast<const S*>(u.data), idx, n, static_cast<S*>(out), stride);
		return check_launch("k_gather_points");
	});
}

int b200_set_point(b200_field u, int64_t idx, double value, void* stream)
{
	if (int rc = check_field(u, "u")) return rc;
	if (idx < 0) return set_error(B200_ERR_ARG, "point index %lld", (long long)idx);
	return dispatch_dtype(u.dtype, [&](auto tag) {
		using S = decltype(tag);
		k_set_point<S><<<1, 1, 0, as_stream(stream)>>>(static_cast<S*>(u.data), idx,
				host_store<S>(value / (double)u.scale));
		return check_launch("k_set_point");
	});
}

int b200_fill_separable(const b200_layout* lay, b200_field u, const b200_box* box,
		const double* v1, const double* v2, const double* v3, double amp, void* stream)
{
	if (int rc = check_layout(lay)) return rc;
	if (int rc = check_box(lay, box)) return rc;
	if (int rc = check_field(u, "u")) return rc;
	cudaStream_t s = as_stream(stream);
	double *d1, *d2, *d3;
	if (int rc = upload_tables(box, v1, v2, v3, s, 0, &d1, &d2, &d3)) return rc;
	const Box3 b = to_box3(box);
	if (int rc = box_rows_ok(b)) return rc;
	const double a = amp / (double)u.scale;
	int rc = dispatch_dtype(u.dtype, [&](auto tag) {
		using S = decltype(tag);
		k_fill_separable<S><<<row_blocks(b, 1), kRowThreads, 0, s>>>(static_cast<S*>(u.data), lay->n1,
				lay->n1 * lay->n2, b, d1, d2, d3, a);
		return check_launch("k_fill_separable");
	});
	if (rc) return rc;
	// the tables live in the shared scratch buffer: keep them until the kernel has read them
	return cuda_error(cudaStreamSynchronize(s), "cudaStreamSynchronize(fill)");
}

int b200_apply_boundary(const b200_layout* lay, b200_field u, int bc_type, int faces, void* stream)
{
	if (int rc = check_layout(lay)) return rc;
	if (int rc = check_field(u, "u")) return rc;
	return apply_boundary(lay, u, bc_type, faces, as_stream(stream));
}

int b200_update_pressure(const b200_layout* lay, b200_field prn, b200_field prc, b200_field coef,
		b200_field lapla, void* stream)
{
	if (int rc = check_layout(lay)) return rc;
	if (int rc = check_field(prn, "prn")) return rc;
	if (int rc = check_field(prc, "prc")) return rc;
	if (int rc = check_field(coef, "coef")) return rc;
	if (int rc = check_field(lapla, "lapla")) return rc;
	if (prc.dtype != prn.dtype || coef.dtype != prn.dtype || lapla.dtype != prn.dtype)
		return set_error(B200_ERR_UNSUPPORTED, "updatePressure needs one storage type");
	if (prn.scale != prc.scale || lapla.scale != prn.scale)
		return set_error(B200_ERR_UNSUPPORTED, "prn, prc and lapla must share one scale");
	const b200_box box{lay->s1, lay->e1, lay->s2, lay->e2, lay->s3, lay->e3};
	const Box3 b = to_box3(&box);
	if (int rc = box_rows_ok(b)) return rc;
	return dispatch_dtype(prn.dtype, [&](auto tag) {
		using S = decltype(tag);
		k_update_pressure<S, true><<<row_blocks(b, kRowUnroll), kRowThreads, 0, as_stream(stream)>>>(
				static_cast<S*>(prn.data), static_cast<const S*>(prc.data),
				static_cast<const S*>(coef.data), static_cast<const S*>(lapla.data), lay->n1,
				lay->n1 * lay->n2, b, coef.scale);
		return check_launch("k_update_pressure");
	});
}

int b200_sum_abs(const b200_layout* lay, b200_field u, const b200_box* box, double* out,
		void* stream)
{
	RedArgs r{};
	return run_reduce<RED_SUM_ABS>(lay, u, nullptr, box, r, out, nullptr, stream);
}

int b200_sum_abs_diff(const b200_layout* lay, b200_field u1, b200_field u2, const b200_box* box,
		double* out, void* stream)
{
	RedArgs r{};
	return run_reduce<RED_L1>(lay, u1, &u2, box, r, out, nullptr, stream);
}

int b200_l1_sums(const b200_layout* lay, b200_field u1, b200_field u2, const b200_box* box,
		double* sum_abs_diff, double* sum_abs_ref, void* stream)
{
	RedArgs r{};
	return run_reduce<RED_L1>(lay, u1, &u2, box, r, sum_abs_diff, sum_abs_ref, stream);
}

int b200_max_err(const b200_layout* lay, b200_field u1, b200_field u2, const b200_box* box,
		double max_err_float, double* out, void* stream)
{
	RedArgs r{};
	r.max_err_float = max_err_float;
	return run_reduce<RED_MAX_ERR>(lay, u1, &u2, box, r, out, nullptr, stream);
}

int b200_min_max(const b200_layout* lay, b200_field u, const b200_box* box, double* mn,
		double* mx, void* stream)
{
	RedArgs r{};
	return run_reduce<RED_MIN_MAX>(lay, u, nullptr, box, r, mn, mx, stream);
}

int b200_l1_sums_separable(const b200_layout* lay, b200_field u, const b200_box* box,
		const double* v1, const double* v2, const double* v3, double amp, int ref_dtype,
		double* sum_abs_diff, double* sum_abs_ref, void* stream)
{
	if (int rc = check_layout(lay)) return rc;
	if (int rc = check_box(lay, box)) return rc;
	if (dtype_size(ref_dtype) == 0) return set_error(B200_ERR_ARG, "ref dtype %d", ref_dtype);
	RedArgs r{};
	double *d1, *d2, *d3;
	// tables after the partial sums in the scratch buffer
	const size_t off = sizeof(double2) * (num_sms() * 8 + 1);
	if (int rc = upload_tables(box, v1, v2, v3, as_stream(stream), (off + 255) & ~(size_t)255, &d1,
				&d2, &d3))
		return rc;
	r.v1 = d1;
	r.v2 = d2;
	r.v3 = d3;
	r.amp = amp;
	r.ref_dtype = ref_dtype;
	return run_reduce<RED_L1_SEP>(lay, u, nullptr, box, r, sum_abs_diff, sum_abs_ref, stream);
}

}  // extern "C"

// ---- b200_l1_sums_separable_noalloc: the same norm on preallocated scratch ---------------------
namespace b200 {
namespace {
constexpr int kNoAllocTableMax = 16384;    // table entries: nx + ny + nz of the box
constexpr int kNoAllocPartialMax = 2048;   // stage-1 partial pairs
constexpr int kNoAllocDevices = 64;
}  // namespace

// The tables (kNoAllocTableMax doubles), then the partial pairs, then the result pair: about
// 160 KB per device, part of the library's device image, so that no call allocates.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocTableMax + 2 * kNoAllocPartialMax + 2];

namespace {
double* g_noalloc_ptr[kNoAllocDevices] = {};
std::mutex g_noalloc_mutex;

// Once per device, with that device current: the scratch's device address, and the kernels the
// entry point launches loaded, so that later calls neither load nor allocate anything.
int noalloc_scratch(double** out)
{
	int dev = 0;
	if (int rc = cuda_error(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
	if (dev < 0 || dev >= kNoAllocDevices) return set_error(B200_ERR_ARG, "device index %d", dev);
	std::lock_guard<std::mutex> lock(g_noalloc_mutex);
	if (!g_noalloc_ptr[dev]) {
		void* p = nullptr;
		if (int rc = cuda_error(cudaGetSymbolAddress(&p, g_noalloc_scratch),
					"cudaGetSymbolAddress(no-alloc scratch)"))
			return rc;
		cudaFuncAttributes fa;
		const void* kernels[] = {
				reinterpret_cast<const void*>(k_reduce<float, RED_L1_SEP>),
				reinterpret_cast<const void*>(k_reduce<double, RED_L1_SEP>),
				reinterpret_cast<const void*>(k_reduce<__half, RED_L1_SEP>),
				reinterpret_cast<const void*>(k_reduce<__nv_bfloat16, RED_L1_SEP>),
				reinterpret_cast<const void*>(k_reduce_final<RED_L1_SEP>)};
		for (const void* k : kernels)
			if (int rc = cuda_error(cudaFuncGetAttributes(&fa, k), "cudaFuncGetAttributes(no-alloc)"))
				return rc;
		num_sms();
		g_noalloc_ptr[dev] = static_cast<double*>(p);
	}
	*out = g_noalloc_ptr[dev];
	return B200_OK;
}
}  // namespace
}  // namespace b200

extern "C" {

int b200_l1_sums_separable_noalloc(const b200_layout* lay, b200_field u, const b200_box* box,
		const double* v1, const double* v2, const double* v3, double amp, int ref_dtype,
		double* sum_abs_diff, double* sum_abs_ref, void* stream)
{
	if (int rc = check_layout(lay)) return rc;
	if (int rc = check_box(lay, box)) return rc;
	if (int rc = check_field(u, "u")) return rc;
	if (dtype_size(ref_dtype) == 0) return set_error(B200_ERR_ARG, "ref dtype %d", ref_dtype);
	if (!v1 || !v2 || !v3) return set_error(B200_ERR_ARG, "NULL table");
	const Box3 b = to_box3(box);
	if (int rc = box_rows_ok(b)) return rc;
	const int64_t entries = (int64_t)b.nx + b.ny + b.nz;
	if (entries > kNoAllocTableMax)
		return set_error(B200_ERR_UNSUPPORTED,
				"b200_l1_sums_separable_noalloc: the box needs %lld table entries (nx + ny + nz), "
				"its preallocated scratch holds %d; use b200_l1_sums_separable",
				(long long)entries, kNoAllocTableMax);
	double* scr = nullptr;
	if (int rc = noalloc_scratch(&scr)) return rc;
	double* t1 = scr;
	double* t2 = t1 + b.nx;
	double* t3 = t2 + b.ny;
	double2* partial = reinterpret_cast<double2*>(scr + kNoAllocTableMax);
	double2* result = partial + kNoAllocPartialMax;
	cudaStream_t s = as_stream(stream);
	int rc = cuda_error(cudaMemcpyAsync(t1, v1, b.nx * sizeof(double), cudaMemcpyHostToDevice, s), "tables");
	if (!rc) rc = cuda_error(cudaMemcpyAsync(t2, v2, b.ny * sizeof(double), cudaMemcpyHostToDevice, s), "tables");
	if (!rc) rc = cuda_error(cudaMemcpyAsync(t3, v3, b.nz * sizeof(double), cudaMemcpyHostToDevice, s), "tables");
	if (rc) return rc;
	RedArgs r{};
	r.n1 = lay->n1;
	r.n12 = lay->n1 * lay->n2;
	r.b = b;
	r.s1 = u.scale;
	r.s2 = 1.0;
	r.v1 = t1;
	r.v2 = t2;
	r.v3 = t3;
	r.amp = amp;
	r.ref_dtype = ref_dtype;
	// the partition of the allocating entry point, so that both give the same sums
	int blocks = row_blocks(b, kRowUnroll);
	if (blocks > kNoAllocPartialMax) blocks = kNoAllocPartialMax;
	rc = dispatch_dtype(u.dtype, [&](auto tag) {
		using S = decltype(tag);
		k_reduce<S, RED_L1_SEP><<<blocks, kRedThreads, 0, s>>>(static_cast<const S*>(u.data),
				nullptr, r, partial);
		return check_launch("k_reduce(no-alloc)");
	});
	if (rc) return rc;
	k_reduce_final<RED_L1_SEP><<<1, kRedThreads, 0, s>>>(partial, blocks, result);
	if ((rc = check_launch("k_reduce_final(no-alloc)"))) return rc;
	double2 v;
	if ((rc = cuda_error(cudaMemcpyAsync(&v, result, sizeof(double2), cudaMemcpyDeviceToHost, s),
				 "cudaMemcpyAsync(no-alloc norm)")))
		return rc;
	if ((rc = cuda_error(cudaStreamSynchronize(s), "cudaStreamSynchronize(no-alloc norm)"))) return rc;
	if (sum_abs_diff) *sum_abs_diff = v.x;
	if (sum_abs_ref) *sum_abs_ref = v.y;
	return B200_OK;
}

}  // extern "C"
