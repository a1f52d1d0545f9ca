// Deterministic elementary functions shared by the CUDA kernels and the host.
//
// The renderer needs sin/cos/tan/atan2/log/exp/pow.  CUDA's device library and
// the host C library implement these with different code, so a path traced on
// the GPU and the same path traced on a CPU would drift apart by an ulp here
// and there, and a Russian-roulette or Fresnel coin flip would eventually go
// the other way.  These versions are written from the mathematics only:
//   * Cody-Waite range reduction (argument split by a multiple of pi/2 or
//     ln 2, with the constant cut into pieces short enough that k * piece is
//     exact),
//   * Taylor series of sin, cos, exp and atan, and the atanh series of log,
//     truncated where the first dropped term is below 1e-19 relative,
// evaluated in IEEE double with a fixed operation order and then rounded to
// float.  They use only +, -, *, / and exactly rounded helpers (rint, frexp,
// ldexp), so any IEEE-conforming target computes identical bits provided the
// compiler does not contract multiply-adds (nvcc -fmad=false, gcc
// -ffp-contract=off).  Double evaluation makes the float results correctly
// rounded except in rare near-halfway cases.
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define WF_HD __host__ __device__ __forceinline__
// The double-precision series are called from many shading sites; one
// out-of-line copy per kernel keeps the instruction footprint small.
#define WF_HD_CALL static __host__ __device__ __noinline__
#else
#define WF_HD inline
#define WF_HD_CALL inline
#endif

namespace wfm {

// pi/2 = PIO2_1 + PIO2_2 + PIO2_3 (33 + 33 + 53 significant bits).
constexpr double kPio2_1 = 0x1.921fb544p+0;
constexpr double kPio2_2 = 0x1.0b4611a6p-34;
constexpr double kPio2_3 = 0x1.3198a2e037073p-69;
constexpr double kTwoOverPi = 0x1.45f306dc9c883p-1;
constexpr double kPi = 0x1.921fb54442d18p+1;
constexpr double kPio2 = 0x1.921fb54442d18p+0;
constexpr double kPio6 = 0x1.0c152382d7366p-1;
constexpr double kSqrt3 = 0x1.bb67ae8584caap+0;
constexpr double kTan15 = 0.26794919243112270;  // 2 - sqrt(3)
// ln 2 = LN2_HI (32 bits) + LN2_LO.
constexpr double kLn2Hi = 0x1.62e42ffp-1;
constexpr double kLn2Lo = -0x1.718432a1b0e26p-35;
constexpr double kLog2e = 0x1.71547652b82fep+0;
constexpr double kSqrtHalf = 0.70710678118654752440;

// x = k * pi/2 + r, |r| <= pi/4 (+ rounding); returns r, quadrant k mod 4.
// Accurate for |x| < 2^19 * pi/2, which covers every angle the renderer forms.
WF_HD double reduce_pio2(double x, int& quadrant) {
    double k = rint(x * kTwoOverPi);
    double r = x - k * kPio2_1;
    r = r - k * kPio2_2;
    r = r - k * kPio2_3;
    quadrant = int(int64_t(k) & 3);
    return r;
}

// sin(r) on |r| <= pi/4: Taylor series through r^17.
WF_HD double sin_kernel(double r) {
    double z = r * r;
    double p = 1.0 / 355687428096000.0;
    p = p * z - 1.0 / 1307674368000.0;
    p = p * z + 1.0 / 6227020800.0;
    p = p * z - 1.0 / 39916800.0;
    p = p * z + 1.0 / 362880.0;
    p = p * z - 1.0 / 5040.0;
    p = p * z + 1.0 / 120.0;
    p = p * z - 1.0 / 6.0;
    return r + r * (z * p);
}

// cos(r) on |r| <= pi/4: Taylor series through r^18.
WF_HD double cos_kernel(double r) {
    double z = r * r;
    double p = -1.0 / 6402373705728000.0;
    p = p * z + 1.0 / 20922789888000.0;
    p = p * z - 1.0 / 87178291200.0;
    p = p * z + 1.0 / 479001600.0;
    p = p * z - 1.0 / 3628800.0;
    p = p * z + 1.0 / 40320.0;
    p = p * z - 1.0 / 720.0;
    p = p * z + 1.0 / 24.0;
    p = p * z - 0.5;
    return 1.0 + z * p;
}

WF_HD_CALL double sin(double x) {
#if defined(WF_FAST_MATH) && defined(__CUDA_ARCH__)
    return ::sin(x);
#endif
    if (!(x == x) || x == INFINITY || x == -INFINITY) return x - x;
    int q;
    double r = reduce_pio2(x, q);
    switch (q) {
    case 0: return sin_kernel(r);
    case 1: return cos_kernel(r);
    case 2: return -sin_kernel(r);
    default: return -cos_kernel(r);
    }
}

WF_HD_CALL double cos(double x) {
#if defined(WF_FAST_MATH) && defined(__CUDA_ARCH__)
    return ::cos(x);
#endif
    if (!(x == x) || x == INFINITY || x == -INFINITY) return x - x;
    int q;
    double r = reduce_pio2(x, q);
    switch (q) {
    case 0: return cos_kernel(r);
    case 1: return -sin_kernel(r);
    case 2: return -cos_kernel(r);
    default: return sin_kernel(r);
    }
}

// atan(t) for 0 <= t <= 1: t > tan(15 deg) is folded by
// atan(t) = pi/6 + atan((t*sqrt3 - 1) / (t + sqrt3)); the series
// t - t^3/3 + t^5/5 - ... is summed through t^31.
WF_HD double atan_unit(double t) {
    double base = 0.0;
    if (t > kTan15) {
        t = (t * kSqrt3 - 1.0) / (t + kSqrt3);
        base = kPio6;
    }
    double z = t * t;
    double p = -1.0 / 31.0;
    p = p * z + 1.0 / 29.0;
    p = p * z - 1.0 / 27.0;
    p = p * z + 1.0 / 25.0;
    p = p * z - 1.0 / 23.0;
    p = p * z + 1.0 / 21.0;
    p = p * z - 1.0 / 19.0;
    p = p * z + 1.0 / 17.0;
    p = p * z - 1.0 / 15.0;
    p = p * z + 1.0 / 13.0;
    p = p * z - 1.0 / 11.0;
    p = p * z + 1.0 / 9.0;
    p = p * z - 1.0 / 7.0;
    p = p * z + 1.0 / 5.0;
    p = p * z - 1.0 / 3.0;
    return base + (t + t * (z * p));
}

// atan2 with the C library's signed-zero and quadrant conventions.
WF_HD_CALL double atan2(double y, double x) {
    if (!(x == x) || !(y == y)) return x + y;
    bool xneg = std::signbit(x), yneg = std::signbit(y);
    if (y == 0.0) return xneg ? (yneg ? -kPi : kPi) : y;
    if (x == 0.0) return yneg ? -kPio2 : kPio2;
    double ax = x < 0.0 ? -x : x, ay = y < 0.0 ? -y : y;
    double angle;
    if (ax == INFINITY || ay == INFINITY) {
        if (ax == INFINITY && ay == INFINITY) angle = kPio2 * 0.5;
        else angle = ay == INFINITY ? kPio2 : 0.0;
    } else if (ay <= ax) {
        angle = atan_unit(ay / ax);
    } else {
        angle = kPio2 - atan_unit(ax / ay);
    }
    if (xneg) angle = kPi - angle;
    return yneg ? -angle : angle;
}

// log(x) = e * ln2 + 2 atanh((m - 1) / (m + 1)), m in [sqrt(1/2), sqrt(2)),
// atanh series through s^21.
WF_HD_CALL double log(double x) {
    if (!(x == x) || x < 0.0) return (x - x) / (x - x);
    if (x == 0.0) return -INFINITY;
    if (x == INFINITY) return x;
    int e;
    double m = frexp(x, &e);
    if (m < kSqrtHalf) {
        m = m * 2.0;
        e = e - 1;
    }
    double s = (m - 1.0) / (m + 1.0);
    double z = s * s;
    double p = 1.0 / 21.0;
    p = p * z + 1.0 / 19.0;
    p = p * z + 1.0 / 17.0;
    p = p * z + 1.0 / 15.0;
    p = p * z + 1.0 / 13.0;
    p = p * z + 1.0 / 11.0;
    p = p * z + 1.0 / 9.0;
    p = p * z + 1.0 / 7.0;
    p = p * z + 1.0 / 5.0;
    p = p * z + 1.0 / 3.0;
    double atanh2 = 2.0 * (s + s * (z * p));
    double de = double(e);
    return de * kLn2Hi + (atanh2 + de * kLn2Lo);
}

// exp(x) = 2^k exp(r), r = x - k ln2, Taylor series of exp(r) through r^17.
WF_HD_CALL double exp(double x) {
    if (!(x == x)) return x;
    if (x > 709.78) return INFINITY;
    if (x < -745.2) return 0.0;
    double k = rint(x * kLog2e);
    double r = (x - k * kLn2Hi) - k * kLn2Lo;
    double p = 1.0 / 355687428096000.0;
    p = p * r + 1.0 / 20922789888000.0;
    p = p * r + 1.0 / 1307674368000.0;
    p = p * r + 1.0 / 87178291200.0;
    p = p * r + 1.0 / 6227020800.0;
    p = p * r + 1.0 / 479001600.0;
    p = p * r + 1.0 / 39916800.0;
    p = p * r + 1.0 / 3628800.0;
    p = p * r + 1.0 / 362880.0;
    p = p * r + 1.0 / 40320.0;
    p = p * r + 1.0 / 5040.0;
    p = p * r + 1.0 / 720.0;
    p = p * r + 1.0 / 120.0;
    p = p * r + 1.0 / 24.0;
    p = p * r + 1.0 / 6.0;
    p = p * r + 0.5;
    p = p * r + 1.0;
    p = p * r + 1.0;
    return ldexp(p, int(k));
}

WF_HD bool is_odd_integer(double y) {
    double h = y * 0.5;
    return rint(y) == y && rint(h) != h;
}

// pow with the C library's special cases for the arguments the renderer uses.
WF_HD_CALL double pow(double x, double y) {
    if (y == 0.0 || x == 1.0) return 1.0;
    if (!(x == x) || !(y == y)) return x + y;
    if (x == 0.0) {
        bool odd = is_odd_integer(y);
        if (y > 0.0) return odd ? x : 0.0;
        return odd ? (std::signbit(x) ? -INFINITY : INFINITY) : INFINITY;
    }
    if (x < 0.0) {
        if (rint(y) != y) return (x - x) / (x - x);
        double r = exp(y * log(-x));
        return is_odd_integer(y) ? -r : r;
    }
    if (x == INFINITY) return y > 0.0 ? INFINITY : 0.0;
    return exp(y * log(x));
}

#if defined(WF_FAST_MATH) && defined(__CUDA_ARCH__)
// The fast build (libwavefront_b200_fast.so, make fast): device code calls
// CUDA's own single-precision functions and contracts multiply-adds, as the
// reference's sm_100a build does.  Results then match the reference within
// an image RMSE instead of bit for bit.
WF_HD float sinf(float x) { return ::sinf(x); }
WF_HD float cosf(float x) { return ::cosf(x); }
WF_HD float tanf(float x) { return ::tanf(x); }
WF_HD float atan2f(float y, float x) { return ::atan2f(y, x); }
WF_HD float logf(float x) { return ::logf(x); }
WF_HD float expf(float x) { return ::expf(x); }
WF_HD float powf(float x, float y) { return ::powf(x, y); }
#else
WF_HD float sinf(float x) { return float(wfm::sin(double(x))); }
WF_HD float cosf(float x) { return float(wfm::cos(double(x))); }
WF_HD float tanf(float x) {
    double d = double(x);
    return float(wfm::sin(d) / wfm::cos(d));
}
WF_HD float atan2f(float y, float x) { return float(wfm::atan2(double(y), double(x))); }
WF_HD float logf(float x) { return float(wfm::log(double(x))); }
WF_HD float expf(float x) { return float(wfm::exp(double(x))); }
WF_HD float powf(float x, float y) { return float(wfm::pow(double(x), double(y))); }
#endif

}  // namespace wfm
