// Shared device/host helpers of the hpcscan_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "hpcscan_b200.h"

namespace b200 {

// ---- error reporting (b200_runtime.cu) -------------------------------------------------------
int set_error(int code, const char* fmt, ...);
int cuda_error(cudaError_t err, const char* what);
// After a kernel launch: report a launch-configuration error without synchronising.
int check_launch(const char* what);

// ---- per-device scratch (b200_runtime.cu) ----------------------------------------------------
// A device buffer of at least `bytes`, owned by the library for the current device and reused
// by every call (calls on one device are serialised by the caller's stream discipline).
int scratch(size_t bytes, void** ptr);
// Pinned host staging of at least `bytes` for small results.
int host_staging(size_t bytes, void** ptr);
int num_sms();

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ---- argument validation -----------------------------------------------------------------------
int check_layout(const b200_layout* lay);
int check_box(const b200_layout* lay, const b200_box* box);
int check_order(int order);
int check_field(const b200_field& f, const char* name);
inline int64_t npoint(const b200_layout* lay) { return lay->n1 * lay->n2 * lay->n3; }

// ---- storage traits ----------------------------------------------------------------------------
// S = storage type, C = compute type (Myfloat / Myfloat2 of the reference builds).
template <typename S> struct Storage;
template <> struct Storage<float> {
	using C = float;
	static __device__ __forceinline__ float load(float v) { return v; }
	static __device__ __forceinline__ float store(float v) { return v; }
	static __device__ __forceinline__ float store_d(double v) { return __double2float_rn(v); }
};
template <> struct Storage<double> {
	using C = double;
	static __device__ __forceinline__ double load(double v) { return v; }
	static __device__ __forceinline__ double store(double v) { return v; }
	static __device__ __forceinline__ double store_d(double v) { return v; }
};
template <> struct Storage<__half> {
	using C = float;
	static __device__ __forceinline__ float load(__half v) { return __half2float(v); }
	static __device__ __forceinline__ __half store(float v) { return __float2half_rn(v); }
	static __device__ __forceinline__ __half store_d(double v) { return __double2half(v); }
};
template <> struct Storage<__nv_bfloat16> {
	using C = float;
	static __device__ __forceinline__ float load(__nv_bfloat16 v) { return __bfloat162float(v); }
	static __device__ __forceinline__ __nv_bfloat16 store(float v) { return __float2bfloat16_rn(v); }
	static __device__ __forceinline__ __nv_bfloat16 store_d(double v) { return __double2bfloat16(v); }
};

// A host-side double rounded once to the storage type (for kernel arguments).
template <typename S>
inline S host_store(double v)
{
	if constexpr (std::is_same_v<S, float>) return (float)v;
	else if constexpr (std::is_same_v<S, double>) return v;
	else if constexpr (std::is_same_v<S, __half>) return __double2half(v);
	else return __double2bfloat16(v);
}

// ---- arithmetic with explicit rounding ---------------------------------------------------------
// EXACT = true: every multiply and add is a separately rounded IEEE operation (no FMA
// contraction), the order of the reference's CPU expressions compiled without FP
// contraction; the results are then bit-identical to the reference CPU path.
template <bool EXACT> struct Arith;
template <> struct Arith<true> {
	static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
	static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
	static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
	static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
	static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
	static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
	// acc + c * s, two roundings
	template <typename C> static __device__ __forceinline__ C mac(C acc, C c, C s)
	{
		return add(acc, mul(c, s));
	}
};
// EXACT = false: multiply-adds are fused (one rounding). The library is compiled with
// -fmad=false, so the fusions are exactly the explicit fma calls here.
template <> struct Arith<false> {
	template <typename C> static __device__ __forceinline__ C mul(C a, C b) { return a * b; }
	template <typename C> static __device__ __forceinline__ C add(C a, C b) { return a + b; }
	template <typename C> static __device__ __forceinline__ C sub(C a, C b) { return a - b; }
	template <typename C> static __device__ __forceinline__ C mac(C acc, C c, C s)
	{
		return fma(c, s, acc);
	}
};

// ---- packed FP32 pairs (sm_100 two-wide add/sub/mul/fma) --------------------------------------
// PTX add/sub/mul/fma.rn.f32x2 round each component like the scalar .rn instruction. The
// assembler does, however, fuse a two-wide multiply into a following two-wide add (measured on
// sm_100a with explicit .rn and with --fmad=false), and it does the same to fma(a, b, -0) with a
// literal -0 (measured: it is a multiply to the assembler). The separately rounded arithmetic
// therefore forms its two-wide products as fma(a, b, z) with z = -0 read from constant memory,
// which the assembler cannot see through: a*b + (-0) is a*b exactly (and -0 + -0 = -0 keeps the
// sign of a zero product), so the one rounding gives the IEEE product, bit-identical to the
// scalar path.
static __constant__ float2 c_neg_zero2 = {-0.0f, -0.0f};
__device__ __forceinline__ float2 f2_op_add(float2 a, float2 b)
{
	float2 d;
	asm("{\n\t.reg .b64 x, y, z;\n\tmov.b64 x, {%2, %3};\n\tmov.b64 y, {%4, %5};\n\t"
	    "add.rn.f32x2 z, x, y;\n\tmov.b64 {%0, %1}, z;\n\t}"
	    : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
	return d;
}
__device__ __forceinline__ float2 f2_op_sub(float2 a, float2 b)
{
	float2 d;
	asm("{\n\t.reg .b64 x, y, z;\n\tmov.b64 x, {%2, %3};\n\tmov.b64 y, {%4, %5};\n\t"
	    "sub.rn.f32x2 z, x, y;\n\tmov.b64 {%0, %1}, z;\n\t}"
	    : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
	return d;
}
__device__ __forceinline__ float2 f2_op_mul(float2 a, float2 b)
{
	float2 d;
	asm("{\n\t.reg .b64 x, y, z;\n\tmov.b64 x, {%2, %3};\n\tmov.b64 y, {%4, %5};\n\t"
	    "mul.rn.f32x2 z, x, y;\n\tmov.b64 {%0, %1}, z;\n\t}"
	    : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
	return d;
}
// a * b + c with one rounding per component
__device__ __forceinline__ float2 f2_op_fma(float2 a, float2 b, float2 c)
{
	float2 d;
	asm("{\n\t.reg .b64 x, y, w, z;\n\tmov.b64 x, {%2, %3};\n\tmov.b64 y, {%4, %5};\n\t"
	    "mov.b64 w, {%6, %7};\n\tfma.rn.f32x2 z, x, y, w;\n\tmov.b64 {%0, %1}, z;\n\t}"
	    : "=f"(d.x), "=f"(d.y)
	    : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
	return d;
}

template <bool EXACT> struct Arith2;
template <> struct Arith2<true> {
	static __device__ __forceinline__ float2 mul(float2 a, float2 b)
	{
		return f2_op_fma(a, b, c_neg_zero2);
	}
	static __device__ __forceinline__ float2 add(float2 a, float2 b) { return f2_op_add(a, b); }
	static __device__ __forceinline__ float2 sub(float2 a, float2 b) { return f2_op_sub(a, b); }
	static __device__ __forceinline__ float2 mac(float2 acc, float2 c, float2 s)
	{
		return f2_op_add(acc, mul(c, s));
	}
};
template <> struct Arith2<false> {
	static __device__ __forceinline__ float2 mul(float2 a, float2 b) { return f2_op_mul(a, b); }
	static __device__ __forceinline__ float2 add(float2 a, float2 b) { return f2_op_add(a, b); }
	static __device__ __forceinline__ float2 sub(float2 a, float2 b) { return f2_op_sub(a, b); }
	static __device__ __forceinline__ float2 mac(float2 acc, float2 c, float2 s)
	{
		return f2_op_fma(c, s, acc);
	}
};

// ---- FD_D2 coefficients (reference src/fdm.h:277-545), exact rationals --------------------------
// Stored in FP64; the compute type rounds them exactly as the reference's `const Myfloat2`.
struct D2Table {
	double c[9][9];
};
__host__ __device__ constexpr D2Table make_d2_table()
{
	return D2Table{{
		{0, 0, 0, 0, 0, 0, 0, 0, 0},
		{-2.0, 1.0, 0, 0, 0, 0, 0, 0, 0},
		{-5. / 2., 4. / 3., -1. / 12., 0, 0, 0, 0, 0, 0},
		{-49. / 18., 3. / 2., -3. / 20., 1. / 90., 0, 0, 0, 0, 0},
		{-205. / 72., 8. / 5., -1 / 5., 8. / 315., -1 / 560., 0, 0, 0, 0},
		{-5269. / 1800., 5. / 3., -5. / 21., 5. / 126., -5. / 1008., 1. / 3150., 0, 0, 0},
		{-5369. / 1800., 12. / 7., -15. / 56., 10. / 189., -1. / 112., 2. / 1925., -1. / 16632., 0, 0},
		{-266681. / 88200., 7. / 4., -7. / 24., 7. / 108., -7. / 528., 7. / 3300., -7. / 30888.,
		 1. / 84084., 0},
		{-1077749. / 352800., 16. / 9., -14. / 45., 112. / 1485., -7. / 396., 112. / 32175.,
		 -2. / 3861., 16. / 315315., -1. / 411840.},
	}};
}

template <typename C, int R, int K>
__device__ __forceinline__ C d2c()
{
	constexpr D2Table t = make_d2_table();
	return static_cast<C>(t.c[R][K]);
}

// Second derivative from values v(k), k = -R..R, around a point, with the reference's
// association: ((A0 u + A1 (u+1 + u-1)) + A2 (u+2 + u-2)) + ... then * inv2.
// O2 is written (A0 u + u+1) + u-1 with no A1 (src/fdm.h:286-296).
template <typename C, int R, bool EXACT, typename F>
__device__ __forceinline__ C d2_axis(F v, C inv2)
{
	using A = Arith<EXACT>;
	C acc = A::mul(d2c<C, R, 0>(), v(0));
	if constexpr (R == 1) {
		return A::mul(A::add(A::add(acc, v(1)), v(-1)), inv2);
	} else {
		acc = A::mac(acc, d2c<C, R, 1>(), A::add(v(1), v(-1)));
		acc = A::mac(acc, d2c<C, R, 2>(), A::add(v(2), v(-2)));
		if constexpr (R >= 3) acc = A::mac(acc, d2c<C, R, 3>(), A::add(v(3), v(-3)));
		if constexpr (R >= 4) acc = A::mac(acc, d2c<C, R, 4>(), A::add(v(4), v(-4)));
		if constexpr (R >= 5) acc = A::mac(acc, d2c<C, R, 5>(), A::add(v(5), v(-5)));
		if constexpr (R >= 6) acc = A::mac(acc, d2c<C, R, 6>(), A::add(v(6), v(-6)));
		if constexpr (R >= 7) acc = A::mac(acc, d2c<C, R, 7>(), A::add(v(7), v(-7)));
		if constexpr (R >= 8) acc = A::mac(acc, d2c<C, R, 8>(), A::add(v(8), v(-8)));
		return A::mul(acc, inv2);
	}
}

// d2_axis for a pair of points (packed FP32), same association and rounding per component.
template <int R, bool EXACT, typename F>
__device__ __forceinline__ float2 d2_axis2(F v, float2 inv2)
{
	using A = Arith2<EXACT>;
	auto cf = [](float c) { return make_float2(c, c); };
	float2 acc = A::mul(cf(d2c<float, R, 0>()), v(0));
	if constexpr (R == 1) {
		return A::mul(A::add(A::add(acc, v(1)), v(-1)), inv2);
	} else {
		acc = A::mac(acc, cf(d2c<float, R, 1>()), A::add(v(1), v(-1)));
		acc = A::mac(acc, cf(d2c<float, R, 2>()), A::add(v(2), v(-2)));
		if constexpr (R >= 3) acc = A::mac(acc, cf(d2c<float, R, 3>()), A::add(v(3), v(-3)));
		if constexpr (R >= 4) acc = A::mac(acc, cf(d2c<float, R, 4>()), A::add(v(4), v(-4)));
		if constexpr (R >= 5) acc = A::mac(acc, cf(d2c<float, R, 5>()), A::add(v(5), v(-5)));
		if constexpr (R >= 6) acc = A::mac(acc, cf(d2c<float, R, 6>()), A::add(v(6), v(-6)));
		if constexpr (R >= 7) acc = A::mac(acc, cf(d2c<float, R, 7>()), A::add(v(7), v(-7)));
		if constexpr (R >= 8) acc = A::mac(acc, cf(d2c<float, R, 8>()), A::add(v(8), v(-8)));
		return A::mul(acc, inv2);
	}
}

// ---- FD_D1 coefficients (reference src/fdm.h:34-234), exact rationals; index 0 unused ---------
struct D1Table {
	double c[9][9];
};
__host__ __device__ constexpr D1Table make_d1_table()
{
	return D1Table{{
		{0, 0, 0, 0, 0, 0, 0, 0, 0},
		{0, 1.0, 0, 0, 0, 0, 0, 0, 0},
		{0, 9. / 8., -1. / 24., 0, 0, 0, 0, 0, 0},
		{0, 75. / 64., -25. / 384., 3. / 640., 0, 0, 0, 0, 0},
		{0, 1225. / 1024., -245. / 3072., 49. / 5120., -5. / 7168., 0, 0, 0, 0},
		{0, 19845. / 16384., -735. / 8192., 567. / 40960., -405. / 229376., 35. / 294912., 0, 0, 0},
		{0, 160083. / 131072., -12705. / 131072., 22869. / 1310720., -5445. / 1835008.,
		 847. / 2359296., -63. / 2883584., 0, 0},
		{0, 1288287. / 1048576., -429429. / 4194304., 429429. / 20971520., -61347. / 14680064.,
		 13013. / 18874368., -3549. / 46137344., 231. / 54525952., 0},
		{0, 41409225. / 33554432., -3578575. / 33554432., 3864861. / 167772160.,
		 -1254825. / 234881024., 325325. / 301989888., -61425. / 369098752., 7425. / 436207616.,
		 -143. / 167772160.},
	}};
}

template <typename C, int R, int K>
__device__ __forceinline__ C d1c()
{
	constexpr D1Table t = make_d1_table();
	return static_cast<C>(t.c[R][K]);
}

// Staggered first derivative at i - 1/2 from v(k) = u[i + k], k = -R..R-1, with the reference's
// association ((A1 (v0 - v-1) + A2 (v1 - v-2)) + ...) * inv; O2 has no A1 factor
// (src/fdm.h:37-44, 51-275).
template <typename C, int R, bool EXACT, typename F>
__device__ __forceinline__ C d1_axis(F v, C inv)
{
	using A = Arith<EXACT>;
	if constexpr (R == 1) {
		return A::mul(A::sub(v(0), v(-1)), inv);
	} else {
		C acc = A::mul(d1c<C, R, 1>(), A::sub(v(0), v(-1)));
		acc = A::mac(acc, d1c<C, R, 2>(), A::sub(v(1), v(-2)));
		if constexpr (R >= 3) acc = A::mac(acc, d1c<C, R, 3>(), A::sub(v(2), v(-3)));
		if constexpr (R >= 4) acc = A::mac(acc, d1c<C, R, 4>(), A::sub(v(3), v(-4)));
		if constexpr (R >= 5) acc = A::mac(acc, d1c<C, R, 5>(), A::sub(v(4), v(-5)));
		if constexpr (R >= 6) acc = A::mac(acc, d1c<C, R, 6>(), A::sub(v(5), v(-6)));
		if constexpr (R >= 7) acc = A::mac(acc, d1c<C, R, 7>(), A::sub(v(6), v(-7)));
		if constexpr (R >= 8) acc = A::mac(acc, d1c<C, R, 8>(), A::sub(v(7), v(-8)));
		return A::mul(acc, inv);
	}
}

// d1_axis for a pair of points (packed FP32), same association and rounding per component.
template <int R, bool EXACT, typename F>
__device__ __forceinline__ float2 d1_axis2(F v, float2 inv)
{
	using A = Arith2<EXACT>;
	auto cf = [](float c) { return make_float2(c, c); };
	if constexpr (R == 1) {
		return A::mul(A::sub(v(0), v(-1)), inv);
	} else {
		float2 acc = A::mul(cf(d1c<float, R, 1>()), A::sub(v(0), v(-1)));
		acc = A::mac(acc, cf(d1c<float, R, 2>()), A::sub(v(1), v(-2)));
		if constexpr (R >= 3) acc = A::mac(acc, cf(d1c<float, R, 3>()), A::sub(v(2), v(-3)));
		if constexpr (R >= 4) acc = A::mac(acc, cf(d1c<float, R, 4>()), A::sub(v(3), v(-4)));
		if constexpr (R >= 5) acc = A::mac(acc, cf(d1c<float, R, 5>()), A::sub(v(4), v(-5)));
		if constexpr (R >= 6) acc = A::mac(acc, cf(d1c<float, R, 6>()), A::sub(v(5), v(-6)));
		if constexpr (R >= 7) acc = A::mac(acc, cf(d1c<float, R, 7>()), A::sub(v(6), v(-7)));
		if constexpr (R >= 8) acc = A::mac(acc, cf(d1c<float, R, 8>()), A::sub(v(7), v(-8)));
		return A::mul(acc, inv);
	}
}

// d2_axis2 along i1 for the pair of points (x(0), x(1)) of a register row, x(i) the value i
// points to the right of the pair's first point, the pair's first point at an even register.
// Two-wide operands must be aligned register pairs, so the sums at odd offsets (whose operands
// straddle two pairs) are computed as two scalar additions instead of regrouping registers.
// Same association and rounding per component as d2_axis.
template <int R, bool EXACT, typename F>
__device__ __forceinline__ float2 d2_axis2_row(F x, float2 inv2)
{
	using A = Arith2<EXACT>;
	using S1 = Arith<EXACT>;
	auto cf = [](float c) { return make_float2(c, c); };
	auto sum = [&](auto kc) -> float2 {
		constexpr int k = decltype(kc)::value;
		if constexpr (k % 2 == 0)
			return A::add(make_float2(x(k), x(k + 1)), make_float2(x(-k), x(1 - k)));
		else
			return make_float2(S1::add(x(k), x(-k)), S1::add(x(k + 1), x(1 - k)));
	};
	float2 acc = A::mul(cf(d2c<float, R, 0>()), make_float2(x(0), x(1)));
	if constexpr (R == 1) {
		const float2 t = make_float2(S1::add(acc.x, x(1)), S1::add(acc.y, x(2)));
		return A::mul(make_float2(S1::add(t.x, x(-1)), S1::add(t.y, x(0))), inv2);
	} else {
		acc = A::mac(acc, cf(d2c<float, R, 1>()), sum(std::integral_constant<int, 1>{}));
		acc = A::mac(acc, cf(d2c<float, R, 2>()), sum(std::integral_constant<int, 2>{}));
		if constexpr (R >= 3) acc = A::mac(acc, cf(d2c<float, R, 3>()), sum(std::integral_constant<int, 3>{}));
		if constexpr (R >= 4) acc = A::mac(acc, cf(d2c<float, R, 4>()), sum(std::integral_constant<int, 4>{}));
		if constexpr (R >= 5) acc = A::mac(acc, cf(d2c<float, R, 5>()), sum(std::integral_constant<int, 5>{}));
		if constexpr (R >= 6) acc = A::mac(acc, cf(d2c<float, R, 6>()), sum(std::integral_constant<int, 6>{}));
		if constexpr (R >= 7) acc = A::mac(acc, cf(d2c<float, R, 7>()), sum(std::integral_constant<int, 7>{}));
		if constexpr (R >= 8) acc = A::mac(acc, cf(d2c<float, R, 8>()), sum(std::integral_constant<int, 8>{}));
		return A::mul(acc, inv2);
	}
}

// d1_axis2 along i1 for the pair of points (x(0), x(1)) of a register row (as d2_axis2_row):
// every difference has one operand at an odd offset, so the differences are scalar.
template <int R, bool EXACT, typename F>
__device__ __forceinline__ float2 d1_axis2_row(F x, float2 inv)
{
	using A = Arith2<EXACT>;
	using S1 = Arith<EXACT>;
	auto cf = [](float c) { return make_float2(c, c); };
	auto dif = [&](int k) {   // (v(k - 1) - v(-k)) for both points
		return make_float2(S1::sub(x(k - 1), x(-k)), S1::sub(x(k), x(1 - k)));
	};
	if constexpr (R == 1) {
		return A::mul(dif(1), inv);
	} else {
		float2 acc = A::mul(cf(d1c<float, R, 1>()), dif(1));
		acc = A::mac(acc, cf(d1c<float, R, 2>()), dif(2));
		if constexpr (R >= 3) acc = A::mac(acc, cf(d1c<float, R, 3>()), dif(3));
		if constexpr (R >= 4) acc = A::mac(acc, cf(d1c<float, R, 4>()), dif(4));
		if constexpr (R >= 5) acc = A::mac(acc, cf(d1c<float, R, 5>()), dif(5));
		if constexpr (R >= 6) acc = A::mac(acc, cf(d1c<float, R, 6>()), dif(6));
		if constexpr (R >= 7) acc = A::mac(acc, cf(d1c<float, R, 7>()), dif(7));
		if constexpr (R >= 8) acc = A::mac(acc, cf(d1c<float, R, 8>()), dif(8));
		return A::mul(acc, inv);
	}
}

template <bool EXACT>
__device__ __forceinline__ float2 leapfrog2(float2 prc, float2 prn, float2 coef, float2 lap)
{
	using A = Arith2<EXACT>;
	return A::mac(A::sub(A::mul(make_float2(2.0f, 2.0f), prc), prn), coef, lap);
}

// Leapfrog update of computePressureWithFD: (2 prc - prn) + coef * lap.
template <typename C, bool EXACT>
__device__ __forceinline__ C leapfrog(C prc, C prn, C coef, C lap)
{
	using A = Arith<EXACT>;
	return A::mac(A::sub(A::mul(static_cast<C>(2.0), prc), prn), coef, lap);
}

// Dispatch a runtime FD order to a compile-time half width R.
template <typename F>
int dispatch_order(int order, F&& f)
{
	switch (order) {
	case 2: return f(std::integral_constant<int, 1>{});
	case 4: return f(std::integral_constant<int, 2>{});
	case 6: return f(std::integral_constant<int, 3>{});
	case 8: return f(std::integral_constant<int, 4>{});
	case 10: return f(std::integral_constant<int, 5>{});
	case 12: return f(std::integral_constant<int, 6>{});
	case 14: return f(std::integral_constant<int, 7>{});
	case 16: return f(std::integral_constant<int, 8>{});
	default: return set_error(B200_ERR_ARG, "FD order %d not supported (2..16, even)", order);
	}
}

// Dispatch a storage dtype code to a C++ type.
template <typename F>
int dispatch_dtype(int dtype, F&& f)
{
	switch (dtype) {
	case B200_F32: return f(float{});
	case B200_F64: return f(double{});
	case B200_F16: return f(__half{});
	case B200_BF16: return f(__nv_bfloat16{});
	default: return set_error(B200_ERR_ARG, "unknown dtype %d", dtype);
	}
}

inline int dtype_size(int dtype)
{
	switch (dtype) {
	case B200_F32: return 4;
	case B200_F64: return 8;
	case B200_F16: return 2;
	case B200_BF16: return 2;
	default: return 0;
	}
}

}  // namespace b200
