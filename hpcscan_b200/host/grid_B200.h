//-------------------------------------------------------------------------------------------------------
// Grid_B200: the NVIDIA B200 (sm_100a) test mode of hpcscan, -testMode B200.
//
// Derives from the reference's Grid (src/grid.h) and forwards every virtual that the
// FD_D2, Grid, Memory and Propa test cases and the acoustic propagators call to the C ABI
// of libhpcscan_b200 (include/hpcscan_b200.h). The wavefield lives in device memory; the
// base class's host array grid_3d is kept (the drivers take its address) and is refreshed
// from the device only where the reference reads it on the host: write, writeGlobal and the
// halo exchange with MPI neighbours.
//
// Registration: Grid_Factory::create(GRID_MODE_B200, ...) returns std::make_shared<Grid_B200>
// (the control block then runs ~Grid_B200, although ~Grid is not virtual), and
// Hardware_Factory::create(GRID_MODE_B200) the base Hardware. See factory_B200.cpp.
//-------------------------------------------------------------------------------------------------------

#ifndef HPCSCAN_GRID_B200_H_
#define HPCSCAN_GRID_B200_H_

#include <string>

#include "grid.h"
#include "hpcscan_b200.h"
#include "type_def.h"

namespace hpcscan {

const std::string GRID_MODE_B200 = "B200";

class Grid_B200 : public Grid
{
public:
	Grid_B200(Grid_type);
	Grid_B200(Grid_type, Dim_type, Myint64, Myint64, Myint64);
	~Grid_B200(void);

	virtual Rtn_code initializeGrid(void);
	virtual void info(void);

	virtual Rtn_code write(string);
	virtual Rtn_code write(Point_type pointType, string);
	virtual Rtn_code writeGlobal(Point_type pointType, string fileName, Myint n_iter);
	virtual Rtn_code read(string);
	virtual Rtn_code read(Point_type pointType, string);

	virtual Myfloat L1Err(Point_type pointType, const Grid& gridIn) const;
	virtual Myfloat allProcL1Err(Point_type, const Grid&) const;
	virtual Myfloat maxErr(Point_type, const Grid&) const;
	virtual Myfloat getMin(Point_type);
	virtual Myfloat getMax(Point_type);
	virtual Myfloat getSumAbs(Point_type) const;
	virtual Myfloat getSumAbsDiff(Point_type, const Grid&) const;

	virtual void fill(Point_type pointType, Myfloat val);
	virtual void fill(Point_type pType, Func_type t1, Func_type t2, Func_type t3,
			Myfloat64 param1, Myfloat64 param2, Myfloat64 param3, Myfloat64 amp);
	virtual void fillArray(Myfloat val);
	virtual void copyArray(const Grid& gridIn);
	virtual void addArray(const Grid& gridIn1, const Grid& gridIn2);
	virtual void multiplyArray(const Grid& gridIn1, const Grid& gridIn2);
	virtual void addUpdateArray(const Grid& gridIn);

	virtual Rtn_code exchangeHalo(MPI_comm_mode_type, Point_type pointType);
	virtual Rtn_code myExchangeAll_halos();
	virtual Rtn_code applyBoundaryCondition(BoundCond_type boundCondType);

	virtual Rtn_code FD_D1_N1(Point_type pType, const Grid& Wgrid, Myint fdOrder);
	virtual Rtn_code FD_D1_N2(Point_type pType, const Grid& Wgrid, Myint fdOrder);
	virtual Rtn_code FD_D1_N3(Point_type pType, const Grid& Wgrid, Myint fdOrder);
	virtual Rtn_code FD_D2_N1(Point_type pType, const Grid& Wgrid, Myint fdOrder);
	virtual Rtn_code FD_D2_N2(Point_type pType, const Grid& Wgrid, Myint fdOrder);
	virtual Rtn_code FD_D2_N3(Point_type pType, const Grid& Wgrid, Myint fdOrder);
	virtual Rtn_code FD_LAPLACIAN(Point_type pType, const Grid& Wgrid, Myint fdOrder);
	virtual Rtn_code updatePressure(Point_type pType, const Grid& prcGrid, const Grid& coefGrid,
			const Grid& laplaGrid);
	virtual Rtn_code computePressureWithFD(Grid& prcGridIn, Grid& coefGridIn, Myint fdOrder);

	// device side of the grid (applies a deferred boundary condition first)
	b200_field field(void) const;

	// Deferred boundary condition, for the fused propagator step (Propagator_Ac2Fused_B200):
	// once deferral is on, applyBoundaryCondition(BOUND_COND_ANTI_MIRROR) only records its
	// faces; the next propagateStep with this grid as prc builds the condition inside the
	// pressure kernel's tiles, and any other use of the grid's device data applies it first.
	void deferBoundaryCondition(bool on) { bc_defer = on; }
	// computePressureWithFD(prc, coef) of this grid with prc's deferred boundary condition, in
	// one library call (b200_propagate_step); without a deferred condition on prc it is
	// computePressureWithFD
	Rtn_code propagateStep(Grid& prcGridIn, Grid& coefGridIn, Myint fdOrder);
	const b200_layout& layout(void) const { return lay; }
	// copy one point type of the grid between host (grid_3d) and device
	Rtn_code copyGridDeviceToHost(Point_type) const;
	Rtn_code copyGridHostToDevice(Point_type);
	// true from read() until the device data is written again: the host array may then hold
	// values the device does not have yet (hpcscan's Modeling set-up transforms the velocity
	// read from file on the host), so write() must not overwrite it from the device
	bool hostAhead(void) const { return host_ahead; }
	void markDeviceWritten(void) const { host_ahead = false; }

protected:
	// B200 layout: the reference's padding, then n1 rounded up to 32 bytes, so that every
	// row starts on a 32-byte boundary (the TMA tiles of the z-marching kernels need 16)
	virtual void padGridn1(void);

private:
	void* d_grid = nullptr;
	b200_layout lay{};
	mutable bool host_ahead = false;
	bool bc_defer = false;
	mutable int bc_pending = 0;          // faces of a deferred boundary condition (0: none)
	b200_field rawField(void) const;     // the device field as it is
	bool applyPendingBoundaryCondition(void) const;
	b200_box box(Point_type) const;
	// the device field of another grid of this mode, or nullptr (message printed)
	static const Grid_B200* peer(const Grid& g, const char* caller);
	Rtn_code inv2(Myfloat64 out[3]) const;
	Rtn_code inv1(Myfloat64 out[3]) const;
	Rtn_code fd_d1(const Grid& Wgrid, Myint fdOrder, int axis, const char* name) const;
};

} // namespace hpcscan

#endif
