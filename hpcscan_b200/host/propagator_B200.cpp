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

} // namespace hpcscan
