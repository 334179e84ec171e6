//-------------------------------------------------------------------------------------------------------
// The acoustic propagators of hpcscan on B200 grids. Propagator_Ac2::initialize(MODELING)
// (src/propagator_Ac2.cpp:84-303) reads the velocity into the coef grid, then turns it into
// v^2 dt^2 on the host array; these subclasses run hpcscan's own initialize and then upload
// the coef grid, so the device holds what the host computed.
//-------------------------------------------------------------------------------------------------------

#ifndef HPCSCAN_PROPAGATOR_B200_H_
#define HPCSCAN_PROPAGATOR_B200_H_

#include "propagator_Ac2.h"
#include "propagator_Ac2SplitComp.h"

namespace hpcscan {

class Propagator_Ac2_B200 : public Propagator_Ac2
{
public:
	virtual Rtn_code initialize(PropaInit_type propaInitType);
};

class Propagator_Ac2SplitComp_B200 : public Propagator_Ac2SplitComp
{
public:
	virtual Rtn_code initialize(PropaInit_type propaInitType);
};

// -propagator Ac2Fused (B200 test mode only): the standard acoustic propagator with the
// boundary condition and the pressure update in one library call per step. Its grids defer
// applyBoundaryCondition; computePressureWithFD then runs b200_propagate_step, which builds the
// anti-mirror condition inside the pressure kernel's tiles where the tuner measured that
// faster for the grid (else runs the two kernels back to back). prn and the inner points of
// prc are bit-identical to Ac2Standard. Under hpcscan's timers the boundary condition's time
// moves into the compute-pressure time. No counterpart in the reference's factory
// (src/propagator_Factory.cpp:19-40 knows Ac2Standard and Ac2SplitComp).
const string PROPA_TYPE_AC2FUSED = "Ac2Fused";

class Propagator_Ac2Fused_B200 : public Propagator_Ac2_B200
{
public:
	Propagator_Ac2Fused_B200(void);
	virtual Rtn_code initialize(PropaInit_type propaInitType);
	virtual Rtn_code computePressureWithFD(Grid& prnGridIn, Grid& prcGridIn);
};

} // namespace hpcscan

#endif
