/*
 * ORACLE — test infrastructure only.
 *
 * FP64 natural logarithm and exponential used by the oracle's friction
 * term (solver_compact.py:456,478: max(wh, 1e-5) ** (7.0 / 3.0)) and
 * Horton capacity (solver_compact.py:545-547: exp(-k * t / 3600.)).
 * Each result is rounded once to F32. The CUDA kernels restate the same
 * methods, so CPU and GPU produce identical bits; tests compare both
 * against the platform's powf/expf.
 *
 * Methods (published):
 *  - ln: argument reduction x = m * 2^e with m in [sqrt(1/2), sqrt(2)],
 *    ln m = 2 atanh(s), s = (m-1)/(m+1), odd Taylor series of atanh to
 *    s^25; e * ln2 added with the Cody–Waite split of ln2 (the fdlibm
 *    hi/lo constants).
 *  - exp: Cody–Waite reduction y = n ln2 + r, |r| <= ln2/2, Taylor series
 *    of e^r to degree 13 in Horner form, scaled by 2^n through the
 *    exponent field.
 * Compile with -ffp-contract=off: the sequence of IEEE operations is the
 * contract.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "step_ref.h"

static const double LN2_HI = 0x1.62e42fee00000p-1;
static const double LN2_LO = 0x1.a39ef35793c76p-33;
static const double INV_LN2 = 0x1.71547652b82fep+0;
static const double SQRT2 = 0x1.6a09e667f3bcdp+0;

static double bits_to_double(uint64_t b) { double d; memcpy(&d, &b, 8); return d; }
static uint64_t double_to_bits(double d) { uint64_t b; memcpy(&b, &d, 8); return b; }

double ora_ln(double x)
{
    if (x != x) return x;
    if (x <= 0.0) return x == 0.0 ? -INFINITY : NAN;
    if (x == INFINITY) return x;
    uint64_t b = double_to_bits(x);
    int e = (int)((b >> 52) & 0x7ff);
    if (e == 0) { /* subnormal double: scale into the normal range */
        x = x * 0x1p54;
        b = double_to_bits(x);
        e = (int)((b >> 52) & 0x7ff) - 54;
    }
    e -= 1023;
    double m = bits_to_double((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
    if (m > SQRT2) { m = m * 0.5; e += 1; }
    double s = (m - 1.0) / (m + 1.0);
    double z = s * s;
    double p = 0x1.47ae147ae147bp-5;        /* 1/25 */
    p = p * z + 0x1.642c8590b2164p-5;       /* 1/23 */
    p = p * z + 0x1.8618618618618p-5;       /* 1/21 */
    p = p * z + 0x1.af286bca1af28p-5;       /* 1/19 */
    p = p * z + 0x1.e1e1e1e1e1e1ep-5;       /* 1/17 */
    p = p * z + 0x1.1111111111111p-4;       /* 1/15 */
    p = p * z + 0x1.3b13b13b13b14p-4;       /* 1/13 */
    p = p * z + 0x1.745d1745d1746p-4;       /* 1/11 */
    p = p * z + 0x1.c71c71c71c71cp-4;       /* 1/9 */
    p = p * z + 0x1.2492492492492p-3;       /* 1/7 */
    p = p * z + 0x1.999999999999ap-3;       /* 1/5 */
    p = p * z + 0x1.5555555555555p-2;       /* 1/3 */
    p = p * z + 1.0;
    double lnm = 2.0 * s * p;
    double de = (double)e;
    return de * LN2_HI + (de * LN2_LO + lnm);
}

double ora_exp(double y)
{
    if (y != y) return y;
    if (y > 709.0) return INFINITY;
    if (y < -745.0) return 0.0;
    double n = floor(y * INV_LN2 + 0.5);
    double r = (y - n * LN2_HI) - n * LN2_LO;
    double p = 0x1.6124613a86d09p-33;       /* 1/13! */
    p = p * r + 0x1.1eed8eff8d898p-29;      /* 1/12! */
    p = p * r + 0x1.ae64567f544e4p-26;      /* 1/11! */
    p = p * r + 0x1.27e4fb7789f5cp-22;      /* 1/10! */
    p = p * r + 0x1.71de3a556c734p-19;      /* 1/9! */
    p = p * r + 0x1.a01a01a01a01ap-16;      /* 1/8! */
    p = p * r + 0x1.a01a01a01a01ap-13;      /* 1/7! */
    p = p * r + 0x1.6c16c16c16c17p-10;      /* 1/6! */
    p = p * r + 0x1.1111111111111p-7;       /* 1/5! */
    p = p * r + 0x1.5555555555555p-5;       /* 1/4! */
    p = p * r + 0x1.5555555555555p-3;       /* 1/3! */
    p = p * r + 0.5;
    p = p * r + 1.0;
    p = p * r + 1.0;
    int ni = (int)n;
    if (ni < -1000) { p = p * 0x1p-600; ni += 600; }
    if (ni > 1000) { p = p * 0x1p600; ni -= 600; }
    return p * bits_to_double((uint64_t)(ni + 1023) << 52);
}

/* x ** y in F64 through the same two series (the FP64 build of the step) */
double ora_pow(double x, double y)
{
    if (x != x) return x;
    if (x == 0.0) return 0.0;
    return ora_exp(y * ora_ln(x));
}

float ora_powf(float x, float y)
{
    if (x != x) return x;
    if (x == 0.0f) return 0.0f;
    return (float)ora_exp((double)y * ora_ln((double)x));
}

float ora_expf(float a)
{
    return (float)ora_exp((double)a);
}
