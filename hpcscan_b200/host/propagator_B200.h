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

} // namespace hpcscan

#endif
