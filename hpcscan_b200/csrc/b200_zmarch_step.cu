// z-marching instantiations for the fused propagator step: the anti-mirror boundary
// condition of prc applied inside computePressureWithFD (all orders, FP32/FP64, every tile
// shape, separately rounded and FMA arithmetic).
#include "b200_zmarch.cuh"

namespace b200 {

int zmarch_launch_step(const ZLaunch& L) { return launch_mode<MODE_STEP, kZShapes, true>(L); }

}  // namespace b200
