// z-marching instantiations for the pressure operator (all orders, FP32/FP64, every tile
// shape, separately rounded and FMA arithmetic).
#include "b200_zmarch.cuh"

namespace b200 {

int zmarch_launch_pressure(const ZLaunch& L) { return launch_mode<MODE_PRESSURE, kZShapes, true>(L); }

}  // namespace b200
