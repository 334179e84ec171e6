// Internal interface between the stencil entry points and the stencil kernel families.
#pragma once

#include "b200_common.cuh"

namespace b200 {

enum StencilMode {
	MODE_D2_AXIS1 = 1,   // Grid::FD_D2_N1
	MODE_D2_AXIS2 = 2,   // Grid::FD_D2_N2
	MODE_D2_AXIS3 = 3,   // Grid::FD_D2_N3
	MODE_LAPLACIAN = 4,  // Grid::FD_LAPLACIAN
	MODE_PRESSURE = 5,   // Grid::computePressureWithFD (in = prc, out = prn)
	MODE_STEP = 6,       // applyBoundaryCondition(prc) fused with computePressureWithFD
	MODE_MODEL = 7,      // damped leapfrog of the modelling engine: p+ = G (2 p + C Lap p) - G^2 p-
	MODE_GRAD = 8,       // gradient accumulation: g += k C w Lap p
	MODE_D1_AXIS1 = 9,   // Grid::FD_D1_N1 (staggered first derivative; inv2_* carry 1/d)
	MODE_D1_AXIS2 = 10,  // Grid::FD_D1_N2
	MODE_D1_AXIS3 = 11,  // Grid::FD_D1_N3
};

// Validating front end shared by all stencil entry points.
int run_stencil(int mode, const b200_layout* lay, int order, const b200_field& in,
		const b200_field& out, const b200_field* coef, double inv2_1, double inv2_2, double inv2_3,
		cudaStream_t s);

// The 3-D z-marching kernel family. Sets *handled = 1 when it took the call; leaves it 0
// (and returns B200_OK) when the grid is not 3-D or its layout does not meet the TMA rules
// (MODE_STEP: also when an axis has fewer than halo + 2 inner points).
int run_zmarch(int mode, const b200_layout* lay, int order, const b200_field& in,
		const b200_field& out, const b200_field* coef, double inv2_1, double inv2_2, double inv2_3,
		cudaStream_t s, int* handled);

// Layout/dtype conditions of the z-marching family (pointer alignment checked per call).
bool zmarch_accepts(const b200_layout* lay, int dtype);

// One z-marching launch: operator, grid, fields, and the tuned parameters.
struct ZLaunch {
	int mode;
	const b200_layout* lay;
	int R;                        // half width = order / 2
	const b200_field* in;
	const b200_field* out;
	const b200_field* coef;       // MODE_PRESSURE only
	double inv2[3];
	cudaStream_t s;
	int shape;                    // tile shape index (Shape<S, i> in b200_zmarch.cuh)
	int nz_chunk;                 // planes per CTA, 0 = heuristic
	bool exact;                   // separately rounded operations (bit-identical to the CPU path)
	unsigned int* err;            // device error word
};
constexpr int kZShapes = 3;       // shapes of the pressure and Laplacian operators

// Per-operator instantiations (b200_zmarch_pressure.cu, b200_zmarch_laplacian.cu,
// b200_zmarch_d2.cu, b200_zmarch_d1.cu).
int zmarch_launch_pressure(const ZLaunch& L);
int zmarch_launch_step(const ZLaunch& L);
int zmarch_launch_laplacian(const ZLaunch& L);
int zmarch_launch_d2(const ZLaunch& L);
int zmarch_launch_d1(const ZLaunch& L);

// Device address of the library's error word on the current device (b200_runtime.cu).
int device_error_word(unsigned int** ptr);

}  // namespace b200
