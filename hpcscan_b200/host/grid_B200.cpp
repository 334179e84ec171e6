//-------------------------------------------------------------------------------------------------------
// Grid_B200: each virtual of the reference's Grid (src/grid.h:50-208) that the test cases and
// propagators call, forwarded to one entry point of the C ABI (include/hpcscan_b200.h).
//
// Conventions kept from the reference: `this` is the input of the FD operators and the output
// of updatePressure / computePressureWithFD (src/grid.cpp:3254-3255, 4587-4590, 4627-4629);
// size mismatches print an error and return RTN_CODE_KO or -1.0 (src/grid.cpp:2011-2015); errors
// are printed, never thrown. Every operator synchronises the device before it returns, so that
// the reference's per-call wall-clock timers (e.g. src/propagator_Ac2.cpp:379-389) time the work.
//-------------------------------------------------------------------------------------------------------

#include "grid_B200.h"

#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>

#include "config.h"
#include "constant.h"
#include "global.h"
#include "output_report.h"

#if defined(_STORAGE_FP16_)
#error "Grid_B200 supports the FP32 and FP64 builds of hpcscan"
#endif

namespace hpcscan {

namespace {

constexpr int kDtype = sizeof(Myfloat) == 8 ? B200_F64 : B200_F32;

void error(const string& text) { printError(text.c_str()); }

// Report a failed ABI call the reference's way; true when the call succeeded.
bool ok(int rc, const char* caller)
{
	if (rc == B200_OK) return true;
	error(string("IN ") + caller + ", " + b200_last_error());
	return false;
}

// One FP64 table of Grid::fill(pType, f1, f2, f3, p1, p2, p3, amp) (src/grid.cpp:1662-1800):
// coord = Orig + i * d in FP64, then sin / cos / coord / 1 / rand, or 1 on an axis beyond dim.
std::vector<Myfloat64> fill_table(Myint64 iStart, Myint64 iEnd, bool active, Func_type t,
		Myfloat64 orig, Myfloat64 d, Myfloat64 param)
{
	std::vector<Myfloat64> v(iEnd - iStart + 1);
	for (Myint64 i = iStart; i <= iEnd; i++) {
		const Myfloat64 coord = Myfloat64(orig + i * d);
		Myfloat64 x = 1.0;
		if (active) {
			switch (t) {
			case FUNC_SINE: x = sin(coord * param); break;
			case FUNC_COSINE: x = cos(coord * param); break;
			case FUNC_LINEAR: x = coord; break;
			case FUNC_RANDOM: x = Myfloat(rand()) / RAND_MAX; break;
			default: x = 1.0; break;
			}
		}
		v[i - iStart] = x;
	}
	return v;
}

} // namespace

//-------------------------------------------------------------------------------------------------------

Grid_B200::Grid_B200(Grid_type gridTypeIn) : Grid(gridTypeIn)
{
	gridMode = GRID_MODE_B200;
}

Grid_B200::Grid_B200(Grid_type gridTypeIn, Dim_type dimIn, Myint64 n1InnerIn, Myint64 n2InnerIn,
		Myint64 n3InnerIn)
	: Grid(gridTypeIn, dimIn, n1InnerIn, n2InnerIn, n3InnerIn)
{
	gridMode = GRID_MODE_B200;
}

Grid_B200::~Grid_B200(void)
{
	if (d_grid) b200_free(d_grid);
	d_grid = nullptr;
}

//-------------------------------------------------------------------------------------------------------

void Grid_B200::padGridn1(void)
{
	Grid::padGridn1();
	const Myint align = 32 / Myint(sizeof(Myfloat));
	const Myint nTot = i1PadEnd + 1;
	if (nTot % align) {
		if (i1PadEnd == i1Halo2End) i1PadStart = i1Halo2End + 1;
		i1PadEnd = (nTot + align - 1) / align * align - 1;
	}
}

Rtn_code Grid_B200::initializeGrid(void)
{
	printDebug(MID_DEBUG, "IN Grid_B200::initializeGrid");
	if (Grid::initializeGrid() != RTN_CODE_OK) return RTN_CODE_KO;

	// one device per MPI rank, as the reference's CUDA grids choose it (src/grid_Cuda.cu:2757-2762)
	int count = 0;
	if (!ok(b200_device_count(&count), "Grid_B200::initializeGrid")) return RTN_CODE_KO;
	if (count < 1) {
		printError("IN Grid_B200::initializeGrid, no CUDA device");
		return RTN_CODE_KO;
	}
	if (!ok(b200_init(myMpiRank % count), "Grid_B200::initializeGrid")) return RTN_CODE_KO;

	lay.n1 = n1;
	lay.n2 = n2;
	lay.n3 = n3;
	lay.s1 = i1InnerStart;
	lay.e1 = i1InnerEnd;
	lay.s2 = i2InnerStart;
	lay.e2 = i2InnerEnd;
	lay.s3 = i3InnerStart;
	lay.e3 = i3InnerEnd;
	lay.dim = dim;
	lay.halo = haloWidth;

	if (d_grid) b200_free(d_grid);
	d_grid = nullptr;
	const size_t bytes = size_t(npoint) * sizeof(Myfloat);
	if (!ok(b200_malloc(&d_grid, bytes), "Grid_B200::initializeGrid")) return RTN_CODE_KO;
	if (!ok(b200_memset(d_grid, 0, bytes, nullptr), "Grid_B200::initializeGrid")) return RTN_CODE_KO;
	printDebug(MID_DEBUG, "OUT Grid_B200::initializeGrid");
	return RTN_CODE_OK;
}

void Grid_B200::info(void)
{
	Grid::info();
	printInfo(MASTER, " B200 device grid");
	printInfo(MASTER, " n1 with B200 padding", Myint(n1));
	printInfo(MASTER, " Device memory (MB)", Myfloat(npoint * sizeof(Myfloat) / 1.e6));
}

//-------------------------------------------------------------------------------------------------------

b200_field Grid_B200::rawField(void) const
{
	b200_field f;
	f.data = d_grid;
	f.dtype = kDtype;
	f.scale = 1.0f;
	return f;
}

b200_field Grid_B200::field(void) const
{
	applyPendingBoundaryCondition();
	return rawField();
}

bool Grid_B200::applyPendingBoundaryCondition(void) const
{
	if (bc_pending == 0) return true;
	const int mask = bc_pending;
	bc_pending = 0;
	return ok(b200_apply_boundary(&lay, rawField(), B200_BOUND_COND_ANTI_MIRROR, mask, nullptr),
			"Grid_B200::applyBoundaryCondition");
}

b200_box Grid_B200::box(Point_type pointType) const
{
	Myint64 i1s, i1e, i2s, i2e, i3s, i3e;
	getGridIndex(pointType, &i1s, &i1e, &i2s, &i2e, &i3s, &i3e);
	b200_box b;
	b.i1s = i1s;
	b.i1e = i1e;
	b.i2s = i2s;
	b.i2e = i2e;
	b.i3s = i3s;
	b.i3e = i3e;
	return b;
}

const Grid_B200* Grid_B200::peer(const Grid& g, const char* caller)
{
	const Grid_B200* p = dynamic_cast<const Grid_B200*>(&g);
	if (!p) error(string("IN ") + caller + ", the other grid is not a B200 grid");
	return p;
}

// inv2_d = (ONE / d)^2 in the compute type Myfloat2, as every FD operator of the reference
// evaluates it (src/grid.cpp:3247-3253); 0 on the axes beyond dim.
Rtn_code Grid_B200::inv2(Myfloat64 out[3]) const
{
	const Myfloat64 d[3] = {d1, d2, d3};
	for (int a = 0; a < 3; a++) {
		if (a + 1 > dim) {
			out[a] = 0.0;
			continue;
		}
		const Myfloat2 inv = ONE / d[a];
		const Myfloat2 inv2 = inv * inv;
		out[a] = Myfloat64(inv2);
	}
	return RTN_CODE_OK;
}

// inv_d = ONE / d in Myfloat2, the factor of the FD_D1 operators (src/grid.cpp:3414-3416);
// 0 on the axes beyond dim.
Rtn_code Grid_B200::inv1(Myfloat64 out[3]) const
{
	const Myfloat64 d[3] = {d1, d2, d3};
	for (int a = 0; a < 3; a++) {
		const Myfloat2 inv = ONE / d[a];
		out[a] = a + 1 > dim ? 0.0 : Myfloat64(inv);
	}
	return RTN_CODE_OK;
}

Rtn_code Grid_B200::copyGridDeviceToHost(Point_type pointType) const
{
	const b200_box b = box(pointType);
	applyPendingBoundaryCondition();
	if (!ok(b200_copy_box_d2h(&lay, sizeof(Myfloat), grid_3d, d_grid, &b, nullptr),
				"Grid_B200::copyGridDeviceToHost"))
		return RTN_CODE_KO;
	return ok(b200_stream_sync(nullptr), "Grid_B200::copyGridDeviceToHost") ? RTN_CODE_OK : RTN_CODE_KO;
}

Rtn_code Grid_B200::copyGridHostToDevice(Point_type pointType)
{
	if (pointType == ALL_POINTS) host_ahead = false;
	const b200_box b = box(pointType);
	applyPendingBoundaryCondition();
	if (!ok(b200_copy_box_h2d(&lay, sizeof(Myfloat), d_grid, grid_3d, &b, nullptr),
				"Grid_B200::copyGridHostToDevice"))
		return RTN_CODE_KO;
	return ok(b200_stream_sync(nullptr), "Grid_B200::copyGridHostToDevice") ? RTN_CODE_OK : RTN_CODE_KO;
}

//-------------------------------------------------------------------------------------------------------
// I/O: the device data goes through the host array, then the reference's own file formats

Rtn_code Grid_B200::write(string fileName)
{
	if (Config::Instance()->writeGrid && !host_ahead && copyGridDeviceToHost(ALL_POINTS) != RTN_CODE_OK)
		return RTN_CODE_KO;
	return Grid::write(fileName);
}

Rtn_code Grid_B200::write(Point_type pointType, string fileName)
{
	if (Config::Instance()->writeGrid && !host_ahead && copyGridDeviceToHost(pointType) != RTN_CODE_OK)
		return RTN_CODE_KO;
	return Grid::write(pointType, fileName);
}

Rtn_code Grid_B200::writeGlobal(Point_type pointType, string fileName, Myint n_iter)
{
	if (Config::Instance()->writeGrid && pointType == INNER_POINTS && !host_ahead &&
			copyGridDeviceToHost(INNER_POINTS) != RTN_CODE_OK)
		return RTN_CODE_KO;
	return Grid::writeGlobal(pointType, fileName, n_iter);
}

Rtn_code Grid_B200::read(string fileName)
{
	if (Grid::read(fileName) != RTN_CODE_OK) return RTN_CODE_KO;
	const Rtn_code rc = copyGridHostToDevice(ALL_POINTS);
	host_ahead = true;
	return rc;
}

Rtn_code Grid_B200::read(Point_type pointType, string fileName)
{
	if (Grid::read(pointType, fileName) != RTN_CODE_OK) return RTN_CODE_KO;
	const Rtn_code rc = copyGridHostToDevice(pointType);
	host_ahead = true;
	return rc;
}

//-------------------------------------------------------------------------------------------------------
// fills and whole-array operations

void Grid_B200::fill(Point_type pointType, Myfloat val)
{
	printDebug(MID_DEBUG, "IN Grid_B200::fill");
	host_ahead = false;
	const b200_box b = box(pointType);
	if (ok(b200_fill_const(&lay, field(), &b, val, nullptr), "Grid_B200::fill"))
		ok(b200_stream_sync(nullptr), "Grid_B200::fill");
}

void Grid_B200::fill(Point_type pointType, Func_type t1, Func_type t2, Func_type t3,
		Myfloat64 param1, Myfloat64 param2, Myfloat64 param3, Myfloat64 amp)
{
	printDebug(MID_DEBUG, "IN Grid_B200::fill");
	host_ahead = false;
	const b200_box b = box(pointType);
	// the tables in the reference's order (axis 1, 2, 3), so that FUNC_RANDOM draws alike
	const std::vector<Myfloat64> v1 = fill_table(b.i1s, b.i1e, dim >= DIM1, t1, Orig1, d1, param1);
	const std::vector<Myfloat64> v2 = fill_table(b.i2s, b.i2e, dim >= DIM2, t2, Orig2, d2, param2);
	const std::vector<Myfloat64> v3 = fill_table(b.i3s, b.i3e, dim >= DIM3, t3, Orig3, d3, param3);
	if (ok(b200_fill_separable(&lay, field(), &b, v1.data(), v2.data(), v3.data(), amp, nullptr),
				"Grid_B200::fill"))
		ok(b200_stream_sync(nullptr), "Grid_B200::fill");
}

void Grid_B200::fillArray(Myfloat val)
{
	host_ahead = false;
	const b200_field none{nullptr, kDtype, 1.0f};
	if (ok(b200_array_op(B200_ARRAY_FILL, npoint, field(), none, none, val, nullptr), "Grid_B200::fillArray"))
		ok(b200_stream_sync(nullptr), "Grid_B200::fillArray");
}

void Grid_B200::copyArray(const Grid& gridIn)
{
	host_ahead = false;
	const Grid_B200* a = peer(gridIn, "Grid_B200::copyArray");
	if (!a) return;
	if (ok(b200_array_op(B200_ARRAY_COPY, npoint, field(), a->field(), a->field(), 0.0, nullptr),
				"Grid_B200::copyArray"))
		ok(b200_stream_sync(nullptr), "Grid_B200::copyArray");
}

void Grid_B200::addArray(const Grid& gridIn1, const Grid& gridIn2)
{
	host_ahead = false;
	const Grid_B200* a = peer(gridIn1, "Grid_B200::addArray");
	const Grid_B200* b = peer(gridIn2, "Grid_B200::addArray");
	if (!a || !b) return;
	if (ok(b200_array_op(B200_ARRAY_ADD, npoint, field(), a->field(), b->field(), 0.0, nullptr),
				"Grid_B200::addArray"))
		ok(b200_stream_sync(nullptr), "Grid_B200::addArray");
}

void Grid_B200::multiplyArray(const Grid& gridIn1, const Grid& gridIn2)
{
	host_ahead = false;
	const Grid_B200* a = peer(gridIn1, "Grid_B200::multiplyArray");
	const Grid_B200* b = peer(gridIn2, "Grid_B200::multiplyArray");
	if (!a || !b) return;
	if (ok(b200_array_op(B200_ARRAY_MUL, npoint, field(), a->field(), b->field(), 0.0, nullptr),
				"Grid_B200::multiplyArray"))
		ok(b200_stream_sync(nullptr), "Grid_B200::multiplyArray");
}

void Grid_B200::addUpdateArray(const Grid& gridIn)
{
	host_ahead = false;
	const Grid_B200* a = peer(gridIn, "Grid_B200::addUpdateArray");
	if (!a) return;
	if (ok(b200_array_op(B200_ARRAY_ADD_UPDATE, npoint, field(), a->field(), a->field(), 0.0, nullptr),
				"Grid_B200::addUpdateArray"))
		ok(b200_stream_sync(nullptr), "Grid_B200::addUpdateArray");
}

//-------------------------------------------------------------------------------------------------------
// norms (FP64 accumulation on the device; src/grid.cpp:2006-2336)

Myfloat Grid_B200::L1Err(Point_type pointType, const Grid& gridIn) const
{
	if (!(this->sameSize(gridIn))) {
		printError("Grid::L1Err, grids have different size");
		return -1.0;
	}
	const Grid_B200* g = peer(gridIn, "Grid_B200::L1Err");
	if (!g) return -1.0;
	const b200_box b = box(pointType);
	double sum1 = 0.0, sum2 = 0.0;
	if (!ok(b200_l1_sums(&lay, field(), g->field(), &b, &sum1, &sum2, nullptr), "Grid_B200::L1Err"))
		return -1.0;
	// prevent divide by zero (src/grid.cpp:2094-2095)
	if (sum2 < MAX_ERR_FLOAT) sum2 = 1.0 * npoint;
	const Myfloat64 err = sum1 / sum2;
	if (std::isnan(err)) printError("In Grid::L1Err, std::isnan(err)");
	return err;
}

// The local sums on the device, then the reference's reduction over the ranks and its guard
// against a zero reference (src/grid.cpp:2113-2166).
Myfloat Grid_B200::allProcL1Err(Point_type pointType, const Grid& gridIn) const
{
	if (!(this->sameSize(gridIn))) {
		printError("Grid::allProcL1Err, grids have different size");
		return -1.0;
	}
	const Grid_B200* g = peer(gridIn, "Grid_B200::allProcL1Err");
	if (!g) return -1.0;
	const b200_box b = box(pointType);
	Myfloat64 sum1Loc = 0.0, sum2Loc = 0.0, sum1 = 0.0, sum2 = 0.0;
	if (!ok(b200_l1_sums(&lay, field(), g->field(), &b, &sum1Loc, &sum2Loc, nullptr),
				"Grid_B200::allProcL1Err"))
		return -1.0;
	MPI_Reduce(&sum1Loc, &sum1, 1, MPI_MYFLOAT64, MPI_SUM, 0, MPI_COMM_WORLD);
	MPI_Reduce(&sum2Loc, &sum2, 1, MPI_MYFLOAT64, MPI_SUM, 0, MPI_COMM_WORLD);
	if (sum2 == 0.0) sum2 = 1.0 * npoint;
	const Myfloat64 err = sum1 / sum2;
	if (std::isnan(err)) printError("In Grid::allProcL1Err, std::isnan(err)");
	return err;
}

Myfloat Grid_B200::maxErr(Point_type pointType, const Grid& gridIn) const
{
	if (!(this->sameSize(gridIn))) {
		printError("Grid::maxErr, grids have different size");
		return -1.0;
	}
	const Grid_B200* g = peer(gridIn, "Grid_B200::maxErr");
	if (!g) return -1.0;
	const b200_box b = box(pointType);
	double err = 0.0;
	if (!ok(b200_max_err(&lay, field(), g->field(), &b, MAX_ERR_FLOAT, &err, nullptr), "Grid_B200::maxErr"))
		return -1.0;
	return err;
}

Myfloat Grid_B200::getMin(Point_type pointType)
{
	const b200_box b = box(pointType);
	double mn = 0.0, mx = 0.0;
	if (!ok(b200_min_max(&lay, field(), &b, &mn, &mx, nullptr), "Grid_B200::getMin")) return FLT_MAX;
	return mn;
}

Myfloat Grid_B200::getMax(Point_type pointType)
{
	const b200_box b = box(pointType);
	double mn = 0.0, mx = 0.0;
	if (!ok(b200_min_max(&lay, field(), &b, &mn, &mx, nullptr), "Grid_B200::getMax")) return -FLT_MAX;
	return mx;
}

Myfloat Grid_B200::getSumAbs(Point_type pointType) const
{
	const b200_box b = box(pointType);
	double s = 0.0;
	if (!ok(b200_sum_abs(&lay, field(), &b, &s, nullptr), "Grid_B200::getSumAbs")) return -1.0;
	return s;
}

Myfloat Grid_B200::getSumAbsDiff(Point_type pointType, const Grid& gridIn) const
{
	if (!(this->sameSize(gridIn))) {
		printError("Grid::getSumAbsDiff, grids have different size");
		return -1.0;
	}
	const Grid_B200* g = peer(gridIn, "Grid_B200::getSumAbsDiff");
	if (!g) return -1.0;
	const b200_box b = box(pointType);
	double s = 0.0;
	if (!ok(b200_sum_abs_diff(&lay, field(), g->field(), &b, &s, nullptr), "Grid_B200::getSumAbsDiff"))
		return -1.0;
	return s;
}

//-------------------------------------------------------------------------------------------------------
// halos and boundary condition

Rtn_code Grid_B200::exchangeHalo(MPI_comm_mode_type commMode, Point_type pointType)
{
	// no neighbour on this face: nothing crosses, nothing to stage
	if (getNeighbourProc(pointType) == MPI_PROC_NULL) return Grid::exchangeHalo(commMode, pointType);
	if (copyGridDeviceToHost(ALL_POINTS) != RTN_CODE_OK) return RTN_CODE_KO;
	if (Grid::exchangeHalo(commMode, pointType) != RTN_CODE_OK) return RTN_CODE_KO;
	return copyGridHostToDevice(pointType);
}

Rtn_code Grid_B200::myExchangeAll_halos()
{
	if (getNumberOfNeighbour() == 0) return RTN_CODE_OK;
	if (copyGridDeviceToHost(ALL_POINTS) != RTN_CODE_OK) return RTN_CODE_KO;
	if (Grid::myExchangeAll_halos() != RTN_CODE_OK) return RTN_CODE_KO;
	return copyGridHostToDevice(ALL_POINTS);
}

Rtn_code Grid_B200::applyBoundaryCondition(BoundCond_type boundCondType)
{
	printDebug(FULL_DEBUG, "IN Grid_B200::applyBoundaryCondition");
	if (boundCondType == NO_BOUND_COND) return RTN_CODE_OK;
	if (boundCondType != BOUND_COND_ANTI_MIRROR) {
		printError("IN Grid::applyBoundaryCondition, invalid boundCondType", boundCondType);
		return RTN_CODE_KO;
	}
	// faces with no neighbour, in the reference's face order (src/grid.cpp:3077-3226)
	const Point_type faces[6] = {I1HALO1, I1HALO2, I2HALO1, I2HALO2, I3HALO1, I3HALO2};
	int mask = 0;
	for (int f = 0; f < 6; f++)
		if (f / 2 < dim && getNeighbourProc(faces[f]) == MPI_PROC_NULL) mask |= 1 << f;
	host_ahead = false;
	if (bc_defer) {              // built by the next propagateStep, or applied before any other use
		bc_pending = mask;
		return RTN_CODE_OK;
	}
	if (!ok(b200_apply_boundary(&lay, field(), B200_BOUND_COND_ANTI_MIRROR, mask, nullptr),
				"Grid_B200::applyBoundaryCondition"))
		return RTN_CODE_KO;
	return ok(b200_stream_sync(nullptr), "Grid_B200::applyBoundaryCondition") ? RTN_CODE_OK : RTN_CODE_KO;
}

Rtn_code Grid_B200::propagateStep(Grid& prcGridIn, Grid& coefGridIn, Myint fdOrder)
{
	printDebug(FULL_DEBUG, "In Grid_B200::propagateStep");
	Grid_B200* prc = dynamic_cast<Grid_B200*>(&prcGridIn);
	const Grid_B200* coef = peer(coefGridIn, "Grid_B200::propagateStep");
	if (!prc || !coef || this->sameSize(prcGridIn) != true || this->sameSize(coefGridIn) != true ||
			prc->bc_pending != 0x3F || dim != DIM3)
		return computePressureWithFD(prcGridIn, coefGridIn, fdOrder);
	// every face of a single-rank 3-D grid: the library's step (the fused kernel where the
	// tuner measured it faster, else the boundary-condition and pressure kernels)
	prc->bc_pending = 0;
	host_ahead = false;
	prc->host_ahead = false;
	Myfloat64 i2[3];
	inv2(i2);
	if (!ok(b200_propagate_step(&lay, fdOrder, field(), prc->rawField(), coef->field(), i2[0], i2[1],
				    i2[2], B200_BOUND_COND_ANTI_MIRROR, nullptr),
				"Grid_B200::propagateStep"))
		return RTN_CODE_KO;
	return ok(b200_stream_sync(nullptr), "Grid_B200::propagateStep") ? RTN_CODE_OK : RTN_CODE_KO;
}

//-------------------------------------------------------------------------------------------------------
// FD operators and the pressure update

namespace {
Rtn_code fd_call(const Grid_B200& u, const Grid& Wgrid, Myint fdOrder, int axis, const char* name,
		const Myfloat64 inv2[3], const b200_layout& lay)
{
	if (u.sameSize(Wgrid) != true) {
		error(string("Grid::") + name + ", grids have not same size");
		return RTN_CODE_KO;
	}
	const Grid_B200* w = dynamic_cast<const Grid_B200*>(&Wgrid);
	if (!w) {
		error(string("IN Grid_B200::") + name + ", the other grid is not a B200 grid");
		return RTN_CODE_KO;
	}
	w->markDeviceWritten();
	const int rc = axis == 0
			? b200_laplacian(&lay, fdOrder, u.field(), w->field(), inv2[0], inv2[1], inv2[2], nullptr)
			: b200_fd_d2(&lay, axis, fdOrder, u.field(), w->field(), inv2[0], inv2[1], inv2[2], nullptr);
	if (!ok(rc, name)) return RTN_CODE_KO;
	return ok(b200_stream_sync(nullptr), name) ? RTN_CODE_OK : RTN_CODE_KO;
}
} // namespace

// Grid::FD_D1_N1/N2/N3 (src/grid.cpp:3401, 3735, 4069): same checks and messages.
Rtn_code Grid_B200::fd_d1(const Grid& Wgrid, Myint fdOrder, int axis, const char* name) const
{
	if (this->sameSize(Wgrid) != true) {
		error(string("Grid::") + name + ", grids have not same size");
		return RTN_CODE_KO;
	}
	const Grid_B200* w = peer(Wgrid, name);
	if (!w) return RTN_CODE_KO;
	Myfloat64 inv[3];
	inv1(inv);
	w->markDeviceWritten();
	if (!ok(b200_fd_d1(&lay, axis, fdOrder, field(), w->field(), inv[0], inv[1], inv[2], nullptr), name))
		return RTN_CODE_KO;
	return ok(b200_stream_sync(nullptr), name) ? RTN_CODE_OK : RTN_CODE_KO;
}

Rtn_code Grid_B200::FD_D1_N1(Point_type, const Grid& Wgrid, Myint fdOrder)
{
	return fd_d1(Wgrid, fdOrder, 1, "FD_D1_N1");
}

Rtn_code Grid_B200::FD_D1_N2(Point_type, const Grid& Wgrid, Myint fdOrder)
{
	return fd_d1(Wgrid, fdOrder, 2, "FD_D1_N2");
}

Rtn_code Grid_B200::FD_D1_N3(Point_type, const Grid& Wgrid, Myint fdOrder)
{
	return fd_d1(Wgrid, fdOrder, 3, "FD_D1_N3");
}

Rtn_code Grid_B200::FD_D2_N1(Point_type, const Grid& Wgrid, Myint fdOrder)
{
	Myfloat64 i2[3];
	inv2(i2);
	return fd_call(*this, Wgrid, fdOrder, 1, "FD_D2_N1", i2, lay);
}

Rtn_code Grid_B200::FD_D2_N2(Point_type, const Grid& Wgrid, Myint fdOrder)
{
	Myfloat64 i2[3];
	inv2(i2);
	return fd_call(*this, Wgrid, fdOrder, 2, "FD_D2_N2", i2, lay);
}

Rtn_code Grid_B200::FD_D2_N3(Point_type, const Grid& Wgrid, Myint fdOrder)
{
	Myfloat64 i2[3];
	inv2(i2);
	return fd_call(*this, Wgrid, fdOrder, 3, "FD_D2_N3", i2, lay);
}

Rtn_code Grid_B200::FD_LAPLACIAN(Point_type, const Grid& Wgrid, Myint fdOrder)
{
	Myfloat64 i2[3];
	inv2(i2);
	return fd_call(*this, Wgrid, fdOrder, 0, "FD_LAPLACIAN", i2, lay);
}

Rtn_code Grid_B200::updatePressure(Point_type, const Grid& prcGrid, const Grid& coefGrid,
		const Grid& laplaGrid)
{
	const Grid_B200* prc = peer(prcGrid, "Grid_B200::updatePressure");
	const Grid_B200* coef = peer(coefGrid, "Grid_B200::updatePressure");
	const Grid_B200* lapla = peer(laplaGrid, "Grid_B200::updatePressure");
	if (!prc || !coef || !lapla) return RTN_CODE_KO;
	// the library reads every grid with this grid's layout
	if (!sameSize(prcGrid) || !sameSize(coefGrid) || !sameSize(laplaGrid)) {
		printError("In Grid::updatePressure, grids have not same size");
		return RTN_CODE_KO;
	}
	host_ahead = false;
	if (!ok(b200_update_pressure(&lay, field(), prc->field(), coef->field(), lapla->field(), nullptr),
				"Grid_B200::updatePressure"))
		return RTN_CODE_KO;
	return ok(b200_stream_sync(nullptr), "Grid_B200::updatePressure") ? RTN_CODE_OK : RTN_CODE_KO;
}

Rtn_code Grid_B200::computePressureWithFD(Grid& prcGridIn, Grid& coefGridIn, Myint fdOrder)
{
	printDebug(FULL_DEBUG, "In Grid_B200::computePressureWithFD");
	if (this->sameSize(prcGridIn) != true) {
		printError("In Grid::computePressureWithFD, grids have not same size");
		return RTN_CODE_KO;
	}
	const Grid_B200* prc = peer(prcGridIn, "Grid_B200::computePressureWithFD");
	const Grid_B200* coef = peer(coefGridIn, "Grid_B200::computePressureWithFD");
	if (!prc || !coef) return RTN_CODE_KO;
	if (this->sameSize(coefGridIn) != true) {        // read with this grid's layout
		printError("In Grid::computePressureWithFD, grids have not same size");
		return RTN_CODE_KO;
	}
	host_ahead = false;
	Myfloat64 i2[3];
	inv2(i2);
	if (!ok(b200_compute_pressure(&lay, fdOrder, field(), prc->field(), coef->field(), i2[0], i2[1],
				    i2[2], nullptr),
				"Grid_B200::computePressureWithFD"))
		return RTN_CODE_KO;
	return ok(b200_stream_sync(nullptr), "Grid_B200::computePressureWithFD") ? RTN_CODE_OK : RTN_CODE_KO;
}

} // namespace hpcscan
