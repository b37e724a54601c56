/*
 * ORACLE (test infrastructure only).  CPU restatement of the scalar math the
 * docking search uses; the product never includes this file.
 *
 * Transcendentals: the fdlibm method (Sun Microsystems' k_sin.c, k_cos.c,
 * e_rem_pio2.c medium-range Cody-Waite reduction, e_acos.c, e_exp.c), with
 * the polynomial coefficients of those sources, restated as the reference's
 * portable math does it (src/lib/portable_math.h:104-268): ksin :104,
 * kcos :115 (its qx split uses z/4, not fdlibm's x/4), reduce :133,
 * sin :143, cos :162, acos :181, exp :232.  Compiled without FMA
 * contraction these are deterministic across CPU and GPU.  Pinned against
 * the reference header by tests/golden/portable_math.json.
 *
 * mt19937 + boost::uniform_real<double> + boost::uniform_int<int> follow
 * src/lib/random.cpp:28-60 with the Boost semantics the reference restates
 * at src/gpu/gpu_rng.cuh:28-92.  Pinned by the C++ standard's known answer
 * (10000th output of the default-seeded engine) and by
 * tests/golden/mt19937.json generated from the reference header.
 */
#ifndef OR_MATH_H
#define OR_MATH_H

#include <cmath>
#include <cstdint>
#include <cstring>

namespace orc {

inline int64_t dbits(double x) { int64_t b; std::memcpy(&b, &x, 8); return b; }
inline double bitsd(int64_t b) { double x; std::memcpy(&x, &b, 8); return x; }

// 2^k scaling in at most three exact multiplications
inline double pm_scale2(double x, int k) {
    if (k > 1023) { x *= bitsd((int64_t)2046 << 52); k -= 1023; }
    else if (k < -1022) {
        x *= bitsd((int64_t)(23) << 52); k += 1000;
        if (k < -1022) { x *= bitsd((int64_t)(23) << 52); k += 1000; }
    }
    return x * bitsd((int64_t)(k + 1023) << 52);
}

// round half to even via the 1.5*2^52 trick
inline double pm_rint(double x) {
    const double shifter = 6755399441055744.0;
    return x >= 0 ? (x + shifter) - shifter : -((-x + shifter) - shifter);
}

inline double pm_ksin(double x) {
    const double s1 = -1.66666666666666324348e-01, s2 = 8.33333333332248946124e-03,
                 s3 = -1.98412698298579493134e-04, s4 = 2.75573137070700676789e-06,
                 s5 = -2.50507602534068634195e-08, s6 = 1.58969099521155010221e-10;
    double z = x * x;
    double v = z * x;
    double r = s2 + z * (s3 + z * (s4 + z * (s5 + z * s6)));
    return x + v * (s1 + z * r);
}

inline double pm_kcos(double x) {
    const double c1 = 4.16666666666666019037e-02, c2 = -1.38888888888741095749e-03,
                 c3 = 2.48015872894767294178e-05, c4 = -2.75573143513906633035e-07,
                 c5 = 2.08757232129817482790e-09, c6 = -1.13596475577881948265e-11;
    double z = x * x;
    double r = z * (c1 + z * (c2 + z * (c3 + z * (c4 + z * (c5 + z * c6)))));
    double ax = std::fabs(x);
    if (ax < 0.3) return 1.0 - (0.5 * z - z * r);
    double qx = ax > 0.78125 ? 0.28125 : bitsd(dbits(z * 0.25) & ~(int64_t)0xffffffff);
    double hz = 0.5 * z - qx;
    double a = 1.0 - qx;
    return a - (hz - z * r);
}

inline double pm_reduce(double x, int& k) {
    const double two_over_pi = 6.36619772367581382433e-01;
    const double pio2_hi = 1.57079632673412561417e+00;
    const double pio2_lo = 6.07710050650619224932e-11;
    double kd = pm_rint(x * two_over_pi);
    k = (int)kd;
    return (x - kd * pio2_hi) - kd * pio2_lo;
}

inline double pm_sin(double x) {
    if (std::fabs(x) <= 7.85398163397448278999e-01) return pm_ksin(x);
    int k;
    double r = pm_reduce(x, k);
    switch (k & 3) {
        case 0: return pm_ksin(r);
        case 1: return pm_kcos(r);
        case 2: return -pm_ksin(r);
        default: return -pm_kcos(r);
    }
}

inline double pm_cos(double x) {
    if (std::fabs(x) <= 7.85398163397448278999e-01) return pm_kcos(x);
    int k;
    double r = pm_reduce(x, k);
    switch (k & 3) {
        case 0: return pm_kcos(r);
        case 1: return -pm_ksin(r);
        case 2: return -pm_kcos(r);
        default: return pm_ksin(r);
    }
}

inline double pm_acos_rational(double z) {
    const double p0 = 1.66666666666666657415e-01, p1 = -3.25565818622400915405e-01,
                 p2 = 2.01212532134862925881e-01, p3 = -4.00555345006794114027e-02,
                 p4 = 7.91534994289814532176e-04, p5 = 3.47933107596021167570e-05;
    const double q1 = -2.40339491173441421878e+00, q2 = 2.02094576023350569471e+00,
                 q3 = -6.88283971605453293030e-01, q4 = 7.70381505559019352791e-02;
    double p = z * (p0 + z * (p1 + z * (p2 + z * (p3 + z * (p4 + z * p5)))));
    double q = 1.0 + z * (q1 + z * (q2 + z * (q3 + z * q4)));
    return p / q;
}

inline double pm_acos(double x) {
    const double pi_d = 3.14159265358979311600e+00;
    const double pio2_hi = 1.57079632679489655800e+00;
    const double pio2_lo = 6.12323399573676603587e-17;
    double ax = std::fabs(x);
    if (ax >= 1) {
        if (x == 1) return 0;
        if (x == -1) return pi_d;
        return (x - x) / (x - x);
    }
    if (ax < 0.5) {
        double r = pm_acos_rational(x * x);
        return pio2_hi - (x - (pio2_lo - x * r));
    }
    if (x < 0) {
        double z = (1.0 + x) * 0.5;
        double s = std::sqrt(z);
        double r = pm_acos_rational(z);
        double w = r * s - pio2_lo;
        return pi_d - 2.0 * (s + w);
    }
    double z = (1.0 - x) * 0.5;
    double s = std::sqrt(z);
    double df = bitsd(dbits(s) & ~(int64_t)0xffffffff);
    double c = (z - df * df) / (s + df);
    double r = pm_acos_rational(z);
    double w = r * s + c;
    return 2.0 * (df + w);
}

inline double pm_exp(double x) {
    const double ln2_hi = 6.93147180369123816490e-01, ln2_lo = 1.90821492927058770002e-10;
    const double inv_ln2 = 1.44269504088896338700e+00;
    const double e1 = 1.66666666666666019037e-01, e2 = -2.77777777770155933842e-03,
                 e3 = 6.61375632143793436117e-05, e4 = -1.65339022054652515390e-06,
                 e5 = 4.13813679705723846039e-08;
    if (x != x) return x;
    if (x > 7.09782712893383973096e+02) return bitsd(0x7ff0000000000000LL);
    if (x < -7.45133219101941108420e+02) return 0;
    double hi = x, lo = 0;
    int k = 0;
    double ax = std::fabs(x);
    if (ax > 0.5 * 6.93147180559945286227e-01) {
        k = (int)(inv_ln2 * x + (x < 0 ? -0.5 : 0.5));
        hi = x - k * ln2_hi;
        lo = k * ln2_lo;
        x = hi - lo;
    } else if (ax < 3.7252902984e-09) {
        return 1.0 + x;
    }
    double t = x * x;
    double c = x - t * (e1 + t * (e2 + t * (e3 + t * (e4 + t * e5))));
    if (k == 0) return 1.0 - ((x * c) / (c - 2.0) - x);
    double y = 1.0 - ((lo - (x * c) / (2.0 - c)) - hi);
    return pm_scale2(y, k);
}

// ---- mt19937 with Boost's uniform distributions ----------------------
struct MT {
    uint32_t x[624];
    int i;
    void seed(uint32_t s) {
        x[0] = s;
        for (int k = 1; k < 624; k++) x[k] = 1812433253u * (x[k - 1] ^ (x[k - 1] >> 30)) + (uint32_t)k;
        i = 624;
    }
    void twist() {
        const uint32_t hi = 0x80000000u, lo = 0x7fffffffu, a = 0x9908b0dfu;
        for (int k = 0; k < 624; k++) {
            uint32_t y = (x[k] & hi) | (x[(k + 1) % 624] & lo);
            x[k] = x[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? a : 0u);
        }
        i = 0;
    }
    uint32_t next() {
        if (i >= 624) twist();
        uint32_t z = x[i++];
        z ^= z >> 11;
        z ^= (z << 7) & 0x9d2c5680u;
        z ^= (z << 15) & 0xefc60000u;
        z ^= z >> 18;
        return z;
    }
};

// boost::uniform_real<double>(a, b): u32 / 2^32 scaled, rejecting b
inline double random_fl(double a, double b, MT& g) {
    for (;;) {
        double num = (double)g.next();
        double den = 4294967295.0 + 1;
        double r = num / den * (b - a) + a;
        if (r < b) return r;
    }
}

// boost::uniform_int<int>(a, b): bucketed rejection
inline int random_int(int a, int b, MT& g) {
    uint32_t range = (uint32_t)b - (uint32_t)a;
    if (range == 0) return a;
    const uint32_t brange = 0xffffffffu;
    uint32_t bucket = brange / (range + 1);
    if (brange % (range + 1) == range) ++bucket;
    for (;;) {
        uint32_t r = g.next() / bucket;
        if (r <= range) return (int)(r + (uint32_t)a);
    }
}

}  // namespace orc
#endif
