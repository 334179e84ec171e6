#include "propagator_B200.h"

#include "grid_B200.h"
#include "output_report.h"

namespace hpcscan {

namespace {
constexpr int kDtype = sizeof(Myfloat) == 8 ? B200_F64 : B200_F32;

// The kernels of the propagator's step readied before hpcscan's time loop (its first-use tuning
// or one launch on scratch grids), so that the loop's timers see neither.
Rtn_code prepare(Grid* wave, Myint fdOrder, int op)
{
	const Grid_B200* g = dynamic_cast<const Grid_B200*>(wave);
	if (!g) return RTN_CODE_OK;
	if (b200_prepare_stencil(&g->layout(), fdOrder, kDtype, op, -1) != B200_OK) {
		printError("IN Propagator_B200::initialize", b200_last_error());
		return RTN_CODE_KO;
	}
	return RTN_CODE_OK;
}

Rtn_code upload_coef(Grid* coef)
{
	Grid_B200* g = dynamic_cast<Grid_B200*>(coef);
	if (!g) {
		printError("IN Propagator_B200::initialize, the coef grid is not a B200 grid");
		return RTN_CODE_KO;
	}
	return g->hostAhead() ? g->copyGridHostToDevice(ALL_POINTS) : RTN_CODE_OK;
}
} // namespace

Rtn_code Propagator_Ac2_B200::initialize(PropaInit_type propaInitType)
{
	if (Propagator_Ac2::initialize(propaInitType) != RTN_CODE_OK) return RTN_CODE_KO;
	if (upload_coef(coefGrid.get()) != RTN_CODE_OK) return RTN_CODE_KO;
	return prepare(prnGrid.get(), fdOrder, B200_OP_PRESSURE);
}

Rtn_code Propagator_Ac2SplitComp_B200::initialize(PropaInit_type propaInitType)
{
	if (Propagator_Ac2SplitComp::initialize(propaInitType) != RTN_CODE_OK) return RTN_CODE_KO;
	if (upload_coef(coefGrid.get()) != RTN_CODE_OK) return RTN_CODE_KO;
	return prepare(prnGrid.get(), fdOrder, B200_OP_LAPLACIAN);
}

Propagator_Ac2Fused_B200::Propagator_Ac2Fused_B200(void) : Propagator_Ac2_B200()
{
	propaKernelType = "Boundary condition fused into the FD kernel (B200)";
}

Rtn_code Propagator_Ac2Fused_B200::initialize(PropaInit_type propaInitType)
{
	if (Propagator_Ac2_B200::initialize(propaInitType) != RTN_CODE_OK) return RTN_CODE_KO;
	if (prepare(prnGrid.get(), fdOrder, B200_OP_STEP) != RTN_CODE_OK) return RTN_CODE_KO;
	for (Grid* g : {prnGrid.get(), prcGrid.get()}) {
		Grid_B200* b = dynamic_cast<Grid_B200*>(g);
		if (!b) {
			printError("IN Propagator_Ac2Fused_B200::initialize, the wavefields are not B200 grids");
			return RTN_CODE_KO;
		}
		b->deferBoundaryCondition(true);
	}
	return RTN_CODE_OK;
}

Rtn_code Propagator_Ac2Fused_B200::computePressureWithFD(Grid& prnGridIn, Grid& prcGridIn)
{
	printDebug(FULL_DEBUG, "In Propagator_Ac2Fused_B200::computePressureWithFD");
	Grid_B200* prn = dynamic_cast<Grid_B200*>(&prnGridIn);
	if (!prn) return Propagator_Ac2_B200::computePressureWithFD(prnGridIn, prcGridIn);
	return prn->propagateStep(prcGridIn, *coefGrid, fdOrder);
}

} // namespace hpcscan
