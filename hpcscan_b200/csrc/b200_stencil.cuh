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
};

// Validating front end shared by all stencil entry points.
int run_stencil(int mode, const b200_layout* lay, int order, const b200_field& in,
		const b200_field& out, const b200_field* coef, double inv2_1, double inv2_2, double inv2_3,
		cudaStream_t s);

// The 3-D z-marching kernel family. Sets *handled = 1 when it took the call; leaves it 0
// (and returns B200_OK) when the grid is not 3-D or its layout does not meet the TMA rules.
int run_zmarch(int mode, const b200_layout* lay, int order, const b200_field& in,
		const b200_field& out, const b200_field* coef, double inv2_1, double inv2_2, double inv2_3,
		cudaStream_t s, int* handled);

// Layout/dtype conditions of the z-marching family (pointer alignment checked per call).
bool zmarch_accepts(const b200_layout* lay, int dtype);

}  // namespace b200
