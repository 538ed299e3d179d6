// Deterministic FP64 natural logarithm and exponential for the step kernels.
//
// The friction factor needs max(wh, 1e-5) ** (7.0 / 3.0) with the exponent
// rounded to F32 as Taichi rounds Python float constants
// (solver_compact.py:456,478), and Horton capacity needs
// exp(-k * t / 3600.) (solver_compact.py:545-547). Both are evaluated here in
// FP64 from IEEE basic operations only and rounded once to F32, so that the
// result does not depend on a vendor math library and is reproduced bit for
// bit by the CPU restatement used in the tests. Build with --fmad=false.
//
// Methods (published):
//  ln  : x = m * 2^e, m in [sqrt(1/2), sqrt(2)]; ln m = 2 atanh(s) with
//        s = (m - 1) / (m + 1) and the odd Taylor series of atanh to s^25;
//        e * ln2 is added through the Cody–Waite hi/lo split of ln2 (the
//        fdlibm constants).
//  exp : Cody–Waite reduction y = n ln2 + r, |r| <= ln2 / 2; Taylor series of
//        e^r to degree 13 (Horner); 2^n applied through the exponent field.
#pragma once
#include <cstdint>

namespace nhf {

__device__ __forceinline__ double ln_f64(double x)
{
    if (x != x) return x;
    if (x <= 0.0) return x == 0.0 ? -__longlong_as_double(0x7ff0000000000000LL)
                                  : __longlong_as_double(0x7ff8000000000000LL);
    if (x == __longlong_as_double(0x7ff0000000000000LL)) return x;
    uint64_t b = (uint64_t)__double_as_longlong(x);
    int e = (int)((b >> 52) & 0x7ff);
    if (e == 0) {
        x = x * 0x1p54;
        b = (uint64_t)__double_as_longlong(x);
        e = (int)((b >> 52) & 0x7ff) - 54;
    }
    e -= 1023;
    double m = __longlong_as_double((long long)((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL));
    if (m > 0x1.6a09e667f3bcdp+0) { m = m * 0.5; e += 1; }
    double s = (m - 1.0) / (m + 1.0);
    double z = s * s;
    double p = 0x1.47ae147ae147bp-5;
    p = p * z + 0x1.642c8590b2164p-5;
    p = p * z + 0x1.8618618618618p-5;
    p = p * z + 0x1.af286bca1af28p-5;
    p = p * z + 0x1.e1e1e1e1e1e1ep-5;
    p = p * z + 0x1.1111111111111p-4;
    p = p * z + 0x1.3b13b13b13b14p-4;
    p = p * z + 0x1.745d1745d1746p-4;
    p = p * z + 0x1.c71c71c71c71cp-4;
    p = p * z + 0x1.2492492492492p-3;
    p = p * z + 0x1.999999999999ap-3;
    p = p * z + 0x1.5555555555555p-2;
    p = p * z + 1.0;
    double lnm = 2.0 * s * p;
    double de = (double)e;
    return de * 0x1.62e42fee00000p-1 + (de * 0x1.a39ef35793c76p-33 + lnm);
}

__device__ __forceinline__ double exp_f64(double y)
{
    if (y != y) return y;
    if (y > 709.0) return __longlong_as_double(0x7ff0000000000000LL);
    if (y < -745.0) return 0.0;
    double n = floor(y * 0x1.71547652b82fep+0 + 0.5);
    double r = (y - n * 0x1.62e42fee00000p-1) - n * 0x1.a39ef35793c76p-33;
    double p = 0x1.6124613a86d09p-33;
    p = p * r + 0x1.1eed8eff8d898p-29;
    p = p * r + 0x1.ae64567f544e4p-26;
    p = p * r + 0x1.27e4fb7789f5cp-22;
    p = p * r + 0x1.71de3a556c734p-19;
    p = p * r + 0x1.a01a01a01a01ap-16;
    p = p * r + 0x1.a01a01a01a01ap-13;
    p = p * r + 0x1.6c16c16c16c17p-10;
    p = p * r + 0x1.1111111111111p-7;
    p = p * r + 0x1.5555555555555p-5;
    p = p * r + 0x1.5555555555555p-3;
    p = p * r + 0.5;
    p = p * r + 1.0;
    p = p * r + 1.0;
    int ni = (int)n;
    if (ni < -1000) { p = p * 0x1p-600; ni += 600; }
    if (ni > 1000) { p = p * 0x1p600; ni -= 600; }
    return p * __longlong_as_double((long long)((uint64_t)(ni + 1023) << 52));
}

// x ** y for the F32 friction base, rounded once from FP64.
__device__ __forceinline__ float pow_f32(float x, float y)
{
    if (x != x) return x;
    if (x == 0.0f) return 0.0f;
    return (float)exp_f64((double)y * ln_f64((double)x));
}

__device__ __forceinline__ float exp_f32(float a) { return (float)exp_f64((double)a); }

// The same two functions in the build's physics type: rounded once to F32,
// or in the FP64 build kept in double.
#ifdef NHF_REAL_DOUBLE
__device__ __forceinline__ double pow_real(double x, double y)
{
    if (x != x) return x;
    if (x == 0.0) return 0.0;
    return exp_f64(y * ln_f64(x));
}
__device__ __forceinline__ double exp_real(double a) { return exp_f64(a); }
#else
__device__ __forceinline__ float pow_real(float x, float y) { return pow_f32(x, y); }
__device__ __forceinline__ float exp_real(float a) { return exp_f32(a); }
#endif

}  // namespace nhf
