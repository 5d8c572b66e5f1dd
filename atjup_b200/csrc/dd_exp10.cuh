// 10^y to (almost always) the correctly rounded double, for the NH4SH equilibrium constant
// K_p = 10^(14.82 - 4705 / T) (ChemistryJup.h:296).
//
// The equilibrium is found by bisection on the sign of (a - x)(b - x)(RT)^2 - K_p(T); its last
// steps are decided by values of that function within rounding of zero, so two evaluations of
// K_p that differ in the last bit send the bisection to different final sub-intervals. The
// reference evaluates K_p with the C library's pow, which rounds nearly always to the nearest
// double. This routine does too: it evaluates 10^y = 2^n exp(r ln 2), n the integer nearest to
// y log2(10), in double-double arithmetic (Dekker's error-free sum and product, the product by
// an explicit fused multiply-add; about 106 bits), with the Taylor series of exp to degree 18 on
// |r ln 2| <= 0.35 (truncation below 2e-26, ten orders below an ulp), and rounds once at the end. The constants are
// log2(10), ln 2 and 1/k!, each split into a double and its remainder.
//
// Its accuracy makes it agree with any evaluation that is itself correctly rounded, whatever
// the algorithm; a residual disagreement with the C library is possible only where 10^y lies
// within the library's own error of a rounding boundary. The sums must not be contracted into
// FMAs: the including file is compiled without FMA contraction.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define ATJUP_HD __host__ __device__ __forceinline__
#else
#define ATJUP_HD inline
#endif

namespace atjup {
namespace ddx {

struct dd {
    double hi, lo;
};

ATJUP_HD dd two_sum(double a, double b) {
    const double s = a + b;
    const double bb = s - a;
    const double e = (a - (s - bb)) + (b - bb);
    return {s, e};
}
ATJUP_HD dd quick_two_sum(double a, double b) {
    const double s = a + b;
    const double e = b - (s - a);
    return {s, e};
}
ATJUP_HD dd two_prod(double a, double b) {
    const double p = a * b;
    return {p, fma(a, b, -p)};
}
ATJUP_HD dd add(dd a, dd b) {
    dd s = two_sum(a.hi, b.hi);
    const dd t = two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = quick_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return quick_two_sum(s.hi, s.lo);
}
ATJUP_HD dd mul(dd a, dd b) {
    dd p = two_prod(a.hi, b.hi);
    p.lo += a.hi * b.lo + a.lo * b.hi;
    return quick_two_sum(p.hi, p.lo);
}
ATJUP_HD dd mul_d(dd a, double b) {
    dd p = two_prod(a.hi, b);
    p.lo += a.lo * b;
    return quick_two_sum(p.hi, p.lo);
}

// 1/k!, k = 0..24, as double + remainder
ATJUP_HD dd inv_fact(int k) {
    switch (k) {
    case 0: return {1.0, 0.0};
    case 1: return {1.0, 0.0};
    case 2: return {0.5, 0.0};
    case 3: return {0.16666666666666666, 9.25185853854297e-18};
    case 4: return {0.041666666666666664, 2.3129646346357427e-18};
    case 5: return {0.008333333333333333, 1.1564823173178714e-19};
    case 6: return {0.001388888888888889, -5.300543954373577e-20};
    case 7: return {0.0001984126984126984, 1.7209558293420705e-22};
    case 8: return {2.48015873015873e-05, 2.1511947866775882e-23};
    case 9: return {2.7557319223985893e-06, -1.858393274046472e-22};
    case 10: return {2.755731922398589e-07, 2.3767714622250297e-23};
    case 11: return {2.505210838544172e-08, -1.448814070935912e-24};
    case 12: return {2.08767569878681e-09, -1.20734505911326e-25};
    case 13: return {1.6059043836821613e-10, 1.2585294588752098e-26};
    case 14: return {1.1470745597729725e-11, 2.0655512752830745e-28};
    case 15: return {7.647163731819816e-13, 7.03872877733453e-30};
    case 16: return {4.779477332387385e-14, 4.399205485834081e-31};
    case 17: return {2.8114572543455206e-15, 1.6508842730861433e-31};
    case 18: return {1.5619206968586225e-16, 1.1910679660273754e-32};
    case 19: return {8.22063524662433e-18, 2.2141894119604265e-34};
    case 20: return {4.110317623312165e-19, 1.4412973378659527e-36};
    case 21: return {1.9572941063391263e-20, -1.3643503830087908e-36};
    case 22: return {8.896791392450574e-22, -7.911402614872376e-38};
    case 23: return {3.868170170630684e-23, -8.843177655482344e-40};
    default: return {1.6117375710961184e-24, -3.6846573564509766e-41};
    }
}

// 10^y for |y| <= 300 / log2(10) (normal results); NaN in, NaN out.
ATJUP_HD double exp10(double y) {
    const dd log2_10 = {3.321928094887362, 1.661617516973592e-16};
    const dd ln2 = {0.6931471805599453, 2.3190468138462996e-17};
    const dd t = mul_d(log2_10, y);
    const double n = rint(t.hi);
    const dd r = two_sum(t.hi - n, t.lo);       // t.hi - n is exact: n is t.hi's nearest integer
    const dd x = mul(r, ln2);
    dd p = inv_fact(18);
    for (int k = 17; k >= 0; k--) p = add(mul(p, x), inv_fact(k));
    return ldexp(p.hi + p.lo, (int)n);
}

}  // namespace ddx
}  // namespace atjup
