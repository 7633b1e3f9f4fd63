// fhd_div.h — correctly rounded FP64 division a / b when the correctly rounded
// reciprocal y = RN(1/b) of the divisor is already known.
//
// Markstein's correction step (P. Markstein, "Computation of elementary functions
// on the IBM RISC System/6000 processor", IBM J. Res. Develop. 34(1), 1990; the
// division chapter of Muller et al., "Handbook of Floating-Point Arithmetic"):
// q0 = RN(a*y) is within one ulp of a/b, so the remainder r = a - b*q0 is exactly
// representable and one FMA computes it exactly, and RN(q0 + r*y) = RN(a/b).  The
// theorem assumes no overflow or underflow anywhere, which holds when
//   2^-900 <= |a| < 2^900  and  2^-100 <= |b| < 2^100
// (then |a y| < 2^1001, |a/b| > 2^-1000 and the remainder's last bit lies above
// 2^-1010).  A zero dividend over a finite nonzero b gives the signed zero a*b
// (its sign is sign(a) xor sign(b), as for a / b); every other a (subnormal, huge,
// inf, NaN) or b takes the plain division, so the result equals a / b for all
// inputs.  Three FP64 operations
// replace the division's reciprocal refinement; the divisors here are constants of
// the run (cell widths, molar masses, reduced masses) whose reciprocals the host
// computes once, or cell values used as divisors several times.
//
// Plain C++ on the host (the CPU test runs this same code against a / b).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define FHD_DIV_HD __host__ __device__ __forceinline__
#else
#define FHD_DIV_HD inline
#endif

namespace fhd {

// exponent windows on the high word of |x| (sign cleared)
constexpr uint32_t kDivAlo = 0x07b00000u;    // 2^-900
constexpr uint32_t kDivAspan = 0x70800000u;  // up to 2^900 (exclusive)
constexpr uint32_t kDivBlo = 0x39b00000u;    // 2^-100
constexpr uint32_t kDivBspan = 0x0c800000u;  // up to 2^100 (exclusive)

FHD_DIV_HD uint32_t div_hi_word(double x) {
#if defined(__CUDA_ARCH__)
    return (uint32_t)__double2hiint(x);
#else
    uint64_t u;
    std::memcpy(&u, &x, sizeof(u));
    return (uint32_t)(u >> 32);
#endif
}

FHD_DIV_HD bool div_in_window(double x, uint32_t lo, uint32_t span) {
    return ((div_hi_word(x) & 0x7fffffffu) - lo) < span;
}

// true when b may be used as a divisor of div_rcp (host check of run constants)
inline bool div_divisor_ok(double b) { return div_in_window(b, kDivBlo, kDivBspan); }

// a / b with a short cut for a zero dividend (a*b is then the same signed zero as
// a / b for any finite nonzero b); otherwise the plain division
FHD_DIV_HD double div_zero_short(double a, double b) {
    if (a == 0.0 && div_in_window(b, kDivBlo, kDivBspan)) return a * b;
    return a / b;
}

// single precision: the same zero-dividend short cut for a normal b (exponent
// field 1..254); otherwise the plain correctly rounded division
FHD_DIV_HD uint32_t div_bits(float x) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(x);
#else
    uint32_t u;
    std::memcpy(&u, &x, sizeof(u));
    return u;
#endif
}
FHD_DIV_HD float div_zero_short(float a, float b) {
    if (a == 0.0f && ((div_bits(b) & 0x7fffffffu) - 0x00800000u) < 0x7f000000u) return a * b;
    return a / b;
}

// the inputs outside the windows, out of line (one copy per module, two arguments
// so that call sites stay light)
#if defined(__CUDA_ARCH__)
static __device__ __noinline__ double div_outside(double a, double b) { return div_zero_short(a, b); }
#else
inline double div_outside(double a, double b) { return div_zero_short(a, b); }
#endif

// a / b for a divisor b inside the b-window (checked by the caller, e.g. on the
// host for run constants) with y = RN(1/b).  (alo, aspan) is the dividend window;
// a caller narrows it, or empties it (aspan 0: always the plain division), never
// widens it.
FHD_DIV_HD double div_rcp(double a, double b, double y, uint32_t alo = kDivAlo, uint32_t aspan = kDivAspan) {
    if (div_in_window(a, alo, aspan)) {
        const double q = a * y;
        return fma(fma(-q, b, a), y, q);
    }
    return div_outside(a, b);
}

// div_rcp with the zero dividend handled inline, for call sites where zero
// dividends are common (no out-of-line call for them)
FHD_DIV_HD double div_rcp_z(double a, double b, double y, uint32_t alo = kDivAlo, uint32_t aspan = kDivAspan) {
    if (div_in_window(a, alo, aspan)) {
        const double q = a * y;
        return fma(fma(-q, b, a), y, q);
    }
    if (a == 0.0 && aspan != 0u) return a * b;  // b: a run constant inside the divisor window
    return div_outside(a, b);
}

// a / b for any b, with y = RN(1/b) from a correctly rounded division 1.0 / b
FHD_DIV_HD double div_rcp_any(double a, double b, double y, uint32_t alo = kDivAlo,
                               uint32_t aspan = kDivAspan) {
    const bool bwin = div_in_window(b, kDivBlo, kDivBspan);
    if (div_in_window(a, alo, aspan) && bwin) {
        const double q = a * y;
        return fma(fma(-q, b, a), y, q);
    }
    return div_outside(a, b);
}

}  // namespace fhd
