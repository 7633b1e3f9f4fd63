// Checks fhd::div_rcp / fhd::div_rcp_any (fhdex_b200/csrc/fhd_div.h) against the
// IEEE division a / b, bit for bit, on the host: the run constants the kernels
// divide by, divisors spread over the whole window, divisors with all-ones or
// minimal significands, dividends over every exponent (zeros, subnormals, inf,
// NaN included), exact quotients, and dividends whose quotient lies within a few
// ulps of a rounding midpoint (the hard cases of correct rounding).
// Prints "checked N mismatches M" and exits 1 when M > 0.
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <random>
#include <vector>

#include "fhd_div.h"

static uint64_t bits(double x) {
    uint64_t u;
    std::memcpy(&u, &x, 8);
    return u;
}

static double from_bits(uint64_t u) {
    double x;
    std::memcpy(&x, &u, 8);
    return x;
}

static bool same(double a, double b) { return (std::isnan(a) && std::isnan(b)) || bits(a) == bits(b); }

int main(int argc, char** argv) {
    const long n_rand = argc > 1 ? std::atol(argv[1]) : 20000000L;
    std::mt19937_64 g(12345);
    std::uniform_int_distribution<uint64_t> mant(0, (uint64_t(1) << 52) - 1);
    auto rnd = [&](int emin, int emax) {
        std::uniform_int_distribution<int> e(emin, emax);
        const uint64_t s = g() & 1;
        return from_bits((s << 63) | (uint64_t(e(g) + 1023) << 52) | mant(g));
    };

    // divisors: run constants (CGS), then the window's edges and hard significands
    const double kB = 1.38064852e-16, Runiv = 8.314462175e7;
    std::vector<double> divs = {8e-6, 1e-6, 2e-6, 1.0 / 256, 3.0, 16.0, 3.1415926535897932, 39.95, 20.18, 83.80, 4.00};
    for (double m : {39.95, 20.18, 83.80, 4.00}) {
        const double mm = m * (kB / Runiv);
        divs.push_back(mm);
        for (double m2 : {39.95, 4.00}) {
            const double mm2 = m2 * (kB / Runiv);
            divs.push_back(mm * mm2 / (mm + mm2));
            divs.push_back(mm + mm2);
        }
    }
    divs.push_back(Runiv * 1e-12);
    for (int e : {-100, -99, -1, 0, 1, 98, 99}) {
        divs.push_back(std::ldexp(1.0, e));
        divs.push_back(std::ldexp(2.0 - std::ldexp(1.0, -52), e));  // all-ones significand
        divs.push_back(std::ldexp(1.0 + std::ldexp(1.0, -52), e));
    }
    for (int r = 0; r < 2000; ++r) divs.push_back(rnd(-100, 99));

    long checked = 0, bad = 0;
    auto check = [&](double a, double b, bool any) {
        const double y = 1.0 / b;
        const double ref = a / b;
        const double q = any ? fhd::div_rcp_any(a, b, y) : fhd::div_rcp(a, b, y);
        const double qz = any ? q : fhd::div_rcp_z(a, b, y);
        ++checked;
        if (!same(q, ref) || !same(qz, ref)) {
            if (bad < 10)
                std::printf("mismatch a=%a b=%a got %a / %a want %a\n", a, b, q, qz, ref);
            ++bad;
        }
    };

    const double specials[] = {0.0, -0.0, std::numeric_limits<double>::infinity(),
                               -std::numeric_limits<double>::infinity(), std::numeric_limits<double>::quiet_NaN(),
                               std::numeric_limits<double>::denorm_min(), -std::numeric_limits<double>::denorm_min(),
                               std::numeric_limits<double>::min(), std::numeric_limits<double>::max(),
                               std::ldexp(1.0, -900), std::ldexp(1.0, 900), std::nextafter(std::ldexp(1.0, 900), 0.0),
                               std::nextafter(std::ldexp(1.0, -900), 0.0)};
    for (double b : divs)
        for (double a : specials) { check(a, b, false); check(a, b, true); }

    // random dividends over all exponents, random divisors from the list
    std::uniform_int_distribution<size_t> pick(0, divs.size() - 1);
    for (long r = 0; r < n_rand; ++r) {
        const double b = divs[pick(g)];
        check(rnd(-1022, 1023), b, false);
        check(from_bits(mant(g) | ((g() & 1) << 63)), b, false);  // subnormal dividends
    }
    // dividends whose quotient sits next to a rounding midpoint: a = RN(b * m) for m
    // the midpoint between q and its successor, nudged by a few ulps of a
    for (long r = 0; r < n_rand / 2; ++r) {
        const double b = divs[pick(g)];
        const double q = rnd(-400, 400);
        const double up = std::nextafter(q, std::copysign(INFINITY, q));
        const double a = b * q + b * (up - q) * 0.5;  // near b * (midpoint of q and up)
        for (int k = -2; k <= 2; ++k) {
            const double ak = from_bits(bits(a) + (int64_t)k);
            check(ak, b, false);
        }
        // exact quotients
        check(b * q, b, false);
    }
    // div_rcp_any with divisors anywhere (inside and outside the window)
    for (long r = 0; r < n_rand / 4; ++r) {
        const double b = rnd(-1022, 1023);
        check(rnd(-1022, 1023), b, true);
        check(rnd(-200, 200), rnd(-150, 150), true);
    }
    for (double b : {0.0, -0.0, std::numeric_limits<double>::denorm_min(), std::numeric_limits<double>::infinity(),
                     std::numeric_limits<double>::quiet_NaN()})
        for (int r = 0; r < 1000; ++r) check(rnd(-300, 300), b, true);
    // signed zero dividends over negative and positive divisors, and div_zero_short
    for (long r = 0; r < n_rand / 100; ++r) {
        const double b = rnd(-1022, 1023);
        for (double a : {0.0, -0.0}) {
            check(a, b, true);
            if (fhd::div_in_window(b, fhd::kDivBlo, fhd::kDivBspan)) check(a, b, false);
        }
    }
    auto check_z = [&](double a, double b) {
        ++checked;
        const double q = fhd::div_zero_short(a, b), ref = a / b;
        if (!same(q, ref)) {
            if (bad < 10) std::printf("mismatch (zero short cut) a=%a b=%a got %a want %a\n", a, b, q, ref);
            ++bad;
        }
    };
    for (double b : specials)
        for (double a : specials) check_z(a, b);
    for (long r = 0; r < n_rand / 10; ++r) {
        const double b = rnd(-1022, 1023);
        check_z(0.0, b);
        check_z(-0.0, b);
        check_z(rnd(-1022, 1023), b);
    }

    // single precision short cut
    std::uniform_int_distribution<uint32_t> fbits(0u, 0xffffffffu);
    auto fsame = [](float x, float y) {
        uint32_t ux, uy;
        std::memcpy(&ux, &x, 4);
        std::memcpy(&uy, &y, 4);
        return (std::isnan(x) && std::isnan(y)) || ux == uy;
    };
    for (long r = 0; r < n_rand / 10; ++r) {
        uint32_t ub = fbits(g);
        float b;
        std::memcpy(&b, &ub, 4);
        for (float a : {0.0f, -0.0f, 1.5f, -3.0e-30f}) {
            ++checked;
            const float q = fhd::div_zero_short(a, b), ref = a / b;
            if (!fsame(q, ref)) {
                if (bad < 10) std::printf("mismatch (f32 zero short cut) a=%a b=%a got %a want %a\n", a, b, q, ref);
                ++bad;
            }
        }
    }
    std::printf("checked %ld mismatches %ld\n", checked, bad);
    return bad == 0 ? 0 : 1;
}
