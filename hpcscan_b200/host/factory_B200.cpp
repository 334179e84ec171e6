//-------------------------------------------------------------------------------------------------------
// Registration of the B200 test mode in the reference's factories, without editing them.
//
// The B200 binary is linked with GNU ld's --wrap for Grid_Factory::create (both overloads,
// src/grid_Factory.cpp:38-119, 123-204), Hardware_Factory::create
// (src/hardware_Factory.cpp:33-124), DataAcquisition_Factory::create and
// Propagator_Factory::create: every call of the drivers lands in a __wrap_ function
// below, which answers the mode "B200" and hands every other mode to the reference's factory
// (__real_). This is exactly the branch a maintainer would add to those factories:
//
//     else if (gridMode.compare(GRID_MODE_B200) == 0)
//         return make_shared<Grid_B200>(gridType);          // and (gridType, dim, n1, n2, n3)
//
// make_shared keeps the derived deleter in the control block, so ~Grid_B200 frees the device
// buffer although ~Grid is not virtual (src/grid.h:47).
//-------------------------------------------------------------------------------------------------------

#include <memory>
#include <string>

#include "config.h"
#include "constant.h"
#include "data_Acquisition_B200.h"
#include "grid_B200.h"
#include "hardware.h"
#include "propagator_B200.h"

using hpcscan::Dim_type;
using hpcscan::Grid;
using hpcscan::Grid_B200;
using hpcscan::Grid_type;
using hpcscan::Hardware;
using std::shared_ptr;
using std::string;

// The mangled names are those of the reference's factory functions (namespace hpcscan,
// std::string by value under the C++11 ABI).
#define GRID_CREATE_2 _ZN7hpcscan12Grid_Factory6createENSt7__cxx1112basic_stringIcSt11char_traitsIcESaIcEEENS_9Grid_typeE
#define GRID_CREATE_6 _ZN7hpcscan12Grid_Factory6createENSt7__cxx1112basic_stringIcSt11char_traitsIcESaIcEEENS_9Grid_typeENS_8Dim_typeElll
#define HW_CREATE _ZN7hpcscan16Hardware_Factory6createENSt7__cxx1112basic_stringIcSt11char_traitsIcESaIcEEE
#define ACQ_CREATE _ZN7hpcscan23DataAcquisition_Factory6createENSt7__cxx1112basic_stringIcSt11char_traitsIcESaIcEEE
#define PROPA_CREATE _ZN7hpcscan18Propagator_Factory6createENSt7__cxx1112basic_stringIcSt11char_traitsIcESaIcEEE

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)

extern "C" {
shared_ptr<Grid> CAT(__real_, GRID_CREATE_2)(string gridMode, Grid_type gridType);
shared_ptr<Grid> CAT(__real_, GRID_CREATE_6)(string gridMode, Grid_type gridType, Dim_type dim,
		long n1, long n2, long n3);
shared_ptr<Hardware> CAT(__real_, HW_CREATE)(string gridMode);
shared_ptr<hpcscan::DataAcquisition> CAT(__real_, ACQ_CREATE)(string testMode);
shared_ptr<hpcscan::Propagator_Ac2> CAT(__real_, PROPA_CREATE)(string propagator);

shared_ptr<Grid> CAT(__wrap_, GRID_CREATE_2)(string gridMode, Grid_type gridType)
{
	if (gridMode.compare(hpcscan::GRID_MODE_B200) == 0) return std::make_shared<Grid_B200>(gridType);
	return CAT(__real_, GRID_CREATE_2)(gridMode, gridType);
}

shared_ptr<Grid> CAT(__wrap_, GRID_CREATE_6)(string gridMode, Grid_type gridType, Dim_type dim,
		long n1, long n2, long n3)
{
	if (gridMode.compare(hpcscan::GRID_MODE_B200) == 0)
		return std::make_shared<Grid_B200>(gridType, dim, n1, n2, n3);
	return CAT(__real_, GRID_CREATE_6)(gridMode, gridType, dim, n1, n2, n3);
}

// The B200 mode runs on the base Hardware (host-side counters), as Baseline does.
shared_ptr<Hardware> CAT(__wrap_, HW_CREATE)(string gridMode)
{
	if (gridMode.compare(hpcscan::GRID_MODE_B200) == 0) return std::make_shared<Hardware>(gridMode);
	return CAT(__real_, HW_CREATE)(gridMode);
}

// Modeling: sources and receivers on the device (DataAcquisition_Factory::create,
// src/data_Acquisition_Factory.cpp:21-71).
shared_ptr<hpcscan::DataAcquisition> CAT(__wrap_, ACQ_CREATE)(string testMode)
{
	if (testMode.compare(hpcscan::GRID_MODE_B200) == 0)
		return std::make_shared<hpcscan::DataAcquisition_B200>();
	return CAT(__real_, ACQ_CREATE)(testMode);
}

// Propagators whose MODELING set-up uploads the coef grid (Propagator_Factory::create,
// src/propagator_Factory.cpp:19-40), and the fused-step propagator Ac2Fused; the test mode is
// the configuration's.
shared_ptr<hpcscan::Propagator_Ac2> CAT(__wrap_, PROPA_CREATE)(string propagator)
{
	if (hpcscan::Config::Instance()->testMode.compare(hpcscan::GRID_MODE_B200) == 0) {
		if (propagator.compare(hpcscan::PROPA_TYPE_AC2STANDARD) == 0)
			return std::make_shared<hpcscan::Propagator_Ac2_B200>();
		if (propagator.compare(hpcscan::PROPA_TYPE_AC2SPLITCOMP) == 0)
			return std::make_shared<hpcscan::Propagator_Ac2SplitComp_B200>();
		if (propagator.compare(hpcscan::PROPA_TYPE_AC2FUSED) == 0)
			return std::make_shared<hpcscan::Propagator_Ac2Fused_B200>();
	}
	return CAT(__real_, PROPA_CREATE)(propagator);
}
}
