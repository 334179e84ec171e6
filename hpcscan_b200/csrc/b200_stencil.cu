// Finite-difference entry points of the hpcscan_b200 C ABI: FD_D2_N1/N2/N3, FD_LAPLACIAN,
// computePressureWithFD and the fused propagator step.
//
// Two kernel families implement them:
//  * the 3-D z-marching kernel (b200_stencil_zmarch.cu): TMA-staged plane tiles in shared
//    memory, a register queue along n3; used for 3-D grids whose layout meets the TMA
//    alignment rules (always true for the Grid_B200 layout);
//  * the direct kernel below: one thread per inner point, neighbours read through L1/L2;
//    used for 1-D and 2-D grids and for 3-D layouts the z-marching kernel cannot take.
// Both evaluate the reference's expressions in the same order with separately rounded
// operations, so their results are bit-identical to each other and to the reference CPU path.
#include "b200_common.cuh"
#include "b200_stencil.cuh"

namespace b200 {

namespace {

template <typename C>
struct DirectArgs {
	const void* u;      // input grid (prc for the pressure update)
	void* w;            // output grid (prn for the pressure update)
	const void* coef;
	int64_t n1, n12;
	int64_t s1, s2, s3;
	int nx, ny, nz;
	C inv2_1, inv2_2, inv2_3;
	float coef_scale;
	int mode;
};

template <typename S, int R, int DIM>
__global__ void __launch_bounds__(256) k_stencil_direct(DirectArgs<typename Storage<S>::C> a)
{
	using C = typename Storage<S>::C;
	using A = Arith<true>;
	const int x = blockIdx.x * blockDim.x + threadIdx.x;
	const int y = blockIdx.y * blockDim.y + threadIdx.y;
	const int z = blockIdx.z * blockDim.z + threadIdx.z;
	if (x >= a.nx || y >= a.ny || z >= a.nz) return;
	const int64_t ii = (a.s1 + x) + (a.s2 + y) * a.n1 + (a.s3 + z) * a.n12;
	const S* __restrict__ u = static_cast<const S*>(a.u);
	S* __restrict__ w = static_cast<S*>(a.w);
	auto v1 = [&](int k) -> C { return Storage<S>::load(__ldg(u + ii + k)); };
	auto v2 = [&](int k) -> C { return Storage<S>::load(__ldg(u + ii + k * a.n1)); };
	auto v3 = [&](int k) -> C { return Storage<S>::load(__ldg(u + ii + k * a.n12)); };
	C r;
	if (a.mode == MODE_D2_AXIS1) {
		r = d2_axis<C, R, true>(v1, a.inv2_1);
	} else if (DIM >= 2 && a.mode == MODE_D2_AXIS2) {
		r = d2_axis<C, R, true>(v2, a.inv2_2);
	} else if (DIM >= 3 && a.mode == MODE_D2_AXIS3) {
		r = d2_axis<C, R, true>(v3, a.inv2_3);
	} else {
		C lap = d2_axis<C, R, true>(v1, a.inv2_1);
		if constexpr (DIM >= 2) lap = A::add(lap, d2_axis<C, R, true>(v2, a.inv2_2));
		if constexpr (DIM >= 3) lap = A::add(lap, d2_axis<C, R, true>(v3, a.inv2_3));
		if (a.mode == MODE_LAPLACIAN) {
			r = lap;
		} else {   // MODE_PRESSURE: w = prn
			C c = Storage<S>::load(static_cast<const S*>(a.coef)[ii]);
			if (a.coef_scale != 1.0f) c = c * (C)a.coef_scale;
			r = leapfrog<C, true>(v1(0), Storage<S>::load(w[ii]), c, lap);
		}
	}
	w[ii] = Storage<S>::store(r);
}

int run_direct(int mode, const b200_layout* lay, int order, const b200_field& in,
		const b200_field& out, const b200_field* coef, double inv2_1, double inv2_2, double inv2_3,
		cudaStream_t s)
{
	return dispatch_dtype(in.dtype, [&](auto tag) {
		using S = decltype(tag);
		using C = typename Storage<S>::C;
		DirectArgs<C> a;
		a.u = in.data;
		a.w = out.data;
		a.coef = coef ? coef->data : nullptr;
		a.n1 = lay->n1;
		a.n12 = lay->n1 * lay->n2;
		a.s1 = lay->s1;
		a.s2 = lay->s2;
		a.s3 = lay->s3;
		a.nx = (int)(lay->e1 - lay->s1 + 1);
		a.ny = (int)(lay->e2 - lay->s2 + 1);
		a.nz = (int)(lay->e3 - lay->s3 + 1);
		a.inv2_1 = (C)inv2_1;
		a.inv2_2 = (C)inv2_2;
		a.inv2_3 = (C)inv2_3;
		a.coef_scale = coef ? coef->scale : 1.0f;
		a.mode = mode;
		const dim3 blk(32, 4, 2);
		const dim3 grd((a.nx + 31) / 32, (a.ny + 3) / 4, (a.nz + 1) / 2);
		return dispatch_order(order, [&](auto rt) {
			constexpr int R = decltype(rt)::value;
			switch (lay->dim) {
			case 1: k_stencil_direct<S, R, 1><<<grd, blk, 0, s>>>(a); break;
			case 2: k_stencil_direct<S, R, 2><<<grd, blk, 0, s>>>(a); break;
			default: k_stencil_direct<S, R, 3><<<grd, blk, 0, s>>>(a); break;
			}
			return check_launch("k_stencil_direct");
		});
	});
}

int check_same_grid(const b200_field& a, const b200_field& b, const char* what)
{
	if (a.dtype != b.dtype)
		return set_error(B200_ERR_UNSUPPORTED, "%s: grids of different storage types", what);
	if (a.scale != b.scale) return set_error(B200_ERR_UNSUPPORTED, "%s: grids of different scales", what);
	if (a.data == b.data) return set_error(B200_ERR_ARG, "%s: input and output are the same array", what);
	return B200_OK;
}

}  // namespace

int run_stencil(int mode, const b200_layout* lay, int order, const b200_field& in,
		const b200_field& out, const b200_field* coef, double inv2_1, double inv2_2, double inv2_3,
		cudaStream_t s)
{
	if (int rc = check_layout(lay)) return rc;
	if (int rc = check_order(order)) return rc;
	if (lay->halo != order / 2)
		return set_error(B200_ERR_ARG, "layout halo %d does not match order %d", lay->halo, order);
	if (int rc = check_field(in, "u")) return rc;
	if (int rc = check_field(out, "w")) return rc;
	if (int rc = check_same_grid(in, out, "stencil")) return rc;
	if (coef) {
		if (int rc = check_field(*coef, "coef")) return rc;
		if (coef->dtype != in.dtype && !(in.dtype != B200_F64 && coef->dtype == B200_F32))
			return set_error(B200_ERR_UNSUPPORTED, "coef storage type %d with wavefield type %d",
					coef->dtype, in.dtype);
	}
	if ((mode == MODE_D2_AXIS2 && lay->dim < 2) || (mode == MODE_D2_AXIS3 && lay->dim < 3))
		return set_error(B200_ERR_ARG, "derivative along an axis beyond dim %d", lay->dim);
	int handled = 0;
	if (int rc = run_zmarch(mode, lay, order, in, out, coef, inv2_1, inv2_2, inv2_3, s, &handled))
		return rc;
	if (handled) return B200_OK;
	if (coef && coef->dtype != in.dtype)
		return set_error(B200_ERR_UNSUPPORTED, "mixed coef/wavefield storage needs the 3-D path");
	return run_direct(mode, lay, order, in, out, coef, inv2_1, inv2_2, inv2_3, s);
}

int apply_boundary(const b200_layout* lay, const b200_field& u, int bc_type, int faces,
		cudaStream_t s);
int apply_boundary_planes(const b200_layout* lay, const b200_field& u, int faces, cudaStream_t s);

}  // namespace b200

using namespace b200;

extern "C" {

int b200_fd_d2(const b200_layout* lay, int axis, int order, b200_field u, b200_field w,
		double inv2_1, double inv2_2, double inv2_3, void* stream)
{
	if (axis < 1 || axis > 3) return set_error(B200_ERR_ARG, "axis %d", axis);
	const int mode = axis == 1 ? MODE_D2_AXIS1 : axis == 2 ? MODE_D2_AXIS2 : MODE_D2_AXIS3;
	return run_stencil(mode, lay, order, u, w, nullptr, inv2_1, inv2_2, inv2_3, as_stream(stream));
}

int b200_laplacian(const b200_layout* lay, int order, b200_field u, b200_field w, double inv2_1,
		double inv2_2, double inv2_3, void* stream)
{
	return run_stencil(MODE_LAPLACIAN, lay, order, u, w, nullptr, inv2_1, inv2_2, inv2_3,
			as_stream(stream));
}

int b200_compute_pressure(const b200_layout* lay, int order, b200_field prn, b200_field prc,
		b200_field coef, double inv2_1, double inv2_2, double inv2_3, void* stream)
{
	return run_stencil(MODE_PRESSURE, lay, order, prc, prn, &coef, inv2_1, inv2_2, inv2_3,
			as_stream(stream));
}

int b200_stencil_route(const b200_layout* lay, int order, int dtype, int* route)
{
	if (!route) return set_error(B200_ERR_ARG, "route is NULL");
	*route = 0;
	if (int rc = check_layout(lay)) return rc;
	if (int rc = check_order(order)) return rc;
	if (dtype_size(dtype) == 0) return set_error(B200_ERR_ARG, "dtype %d", dtype);
	*route = zmarch_accepts(lay, dtype) ? 1 : 2;
	return B200_OK;
}

int b200_propagate_step(const b200_layout* lay, int order, b200_field prn, b200_field prc,
		b200_field coef, double inv2_1, double inv2_2, double inv2_3, int bc_type, void* stream)
{
	if (int rc = check_layout(lay)) return rc;
	if (int rc = check_field(prc, "prc")) return rc;
	if (bc_type == B200_BOUND_COND_ANTI_MIRROR) {
		// one kernel: the boundary condition of prc applied in the tiles of the pressure update
		if (int rc = check_order(order)) return rc;
		if (lay->halo != order / 2)
			return set_error(B200_ERR_ARG, "layout halo %d does not match order %d", lay->halo, order);
		if (int rc = check_field(prn, "prn")) return rc;
		if (int rc = check_field(coef, "coef")) return rc;
		if (int rc = check_same_grid(prc, prn, "propagate_step")) return rc;
		int handled = 0;
		if (int rc = run_zmarch(MODE_STEP, lay, order, prc, prn, &coef, inv2_1, inv2_2, inv2_3,
					as_stream(stream), &handled))
			return rc;
		if (handled) return apply_boundary_planes(lay, prc, 0x3F, as_stream(stream));
	}
	if (int rc = apply_boundary(lay, prc, bc_type, 0x3F, as_stream(stream))) return rc;
	return run_stencil(MODE_PRESSURE, lay, order, prc, prn, &coef, inv2_1, inv2_2, inv2_3,
			as_stream(stream));
}

}  // extern "C"
