#include "propagator_B200.h"

#include "grid_B200.h"
#include "output_report.h"

namespace hpcscan {

namespace {
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
	return upload_coef(coefGrid.get());
}

Rtn_code Propagator_Ac2SplitComp_B200::initialize(PropaInit_type propaInitType)
{
	if (Propagator_Ac2SplitComp::initialize(propaInitType) != RTN_CODE_OK) return RTN_CODE_KO;
	return upload_coef(coefGrid.get());
}

Propagator_Ac2Fused_B200::Propagator_Ac2Fused_B200(void) : Propagator_Ac2_B200()
{
	propaKernelType = "Boundary condition fused into the FD kernel (B200)";
}

Rtn_code Propagator_Ac2Fused_B200::initialize(PropaInit_type propaInitType)
{
	if (Propagator_Ac2_B200::initialize(propaInitType) != RTN_CODE_OK) return RTN_CODE_KO;
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
