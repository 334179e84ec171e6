// z-marching instantiations for the staggered first derivatives FD_D1_N1/N2/N3 (all orders,
// FP32/FP64, default tile shape, separately rounded arithmetic).
#include "b200_zmarch.cuh"

namespace b200 {

int zmarch_launch_d1(const ZLaunch& L)
{
	switch (L.mode) {
	case MODE_D1_AXIS1: return launch_mode<MODE_D1_AXIS1, 1, false>(L);
	case MODE_D1_AXIS2: return launch_mode<MODE_D1_AXIS2, 1, false>(L);
	default: return launch_mode<MODE_D1_AXIS3, 1, false>(L);
	}
}

}  // namespace b200
