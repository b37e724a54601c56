// Scalar / vector / quaternion math of the docking search, host+device.
//
// Double precision versions keep smina's operand order (common.h vec/mat,
// quaternion.cpp, tree.h, curl.h) so that, compiled without FMA contraction
// (-fmad=false), the plain path reproduces a CPU FP64 run bit for bit.
// Transcendentals for that path use the fdlibm method (Sun k_sin/k_cos,
// Cody-Waite pi/2 reduction, e_acos, e_exp) in the arrangement the
// reference's portable math uses (src/lib/portable_math.h:104-268).
#pragma once
#include <cstdint>
#include <cfloat>
#include <cmath>

#ifdef __CUDACC__
#define SG_HD __host__ __device__ __forceinline__
#else
#define SG_HD inline
#endif

namespace sg {

constexpr double kPi = 3.1415926535897931;
constexpr double kEps = DBL_EPSILON;
constexpr double kMaxFl = DBL_MAX;

SG_HD int64_t d2bits(double x) {
#ifdef __CUDA_ARCH__
    return __double_as_longlong(x);
#else
    int64_t b;
    __builtin_memcpy(&b, &x, 8);
    return b;
#endif
}
SG_HD double bits2d(int64_t b) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double(b);
#else
    double x;
    __builtin_memcpy(&x, &b, 8);
    return x;
#endif
}

// ---- fdlibm-method double transcendentals ------------------------------------
SG_HD double fd_pow2(double x, int k) {
    if (k > 1023) { x *= bits2d((int64_t)2046 << 52); k -= 1023; }
    else if (k < -1022) {
        x *= bits2d((int64_t)23 << 52); k += 1000;
        if (k < -1022) { x *= bits2d((int64_t)23 << 52); k += 1000; }
    }
    return x * bits2d((int64_t)(k + 1023) << 52);
}
SG_HD double fd_round(double x) {
    const double c = 6755399441055744.0;  // 1.5 * 2^52
    return x >= 0 ? (x + c) - c : -((-x + c) - c);
}
SG_HD double fd_sin_kernel(double x) {
    const double z = x * x, v = z * x;
    const double r = 8.33333333332248946124e-03 +
                     z * (-1.98412698298579493134e-04 +
                          z * (2.75573137070700676789e-06 + z * (-2.50507602534068634195e-08 + z * 1.58969099521155010221e-10)));
    return x + v * (-1.66666666666666324348e-01 + z * r);
}
SG_HD double fd_cos_kernel(double x) {
    const double z = x * x;
    const double r = z * (4.16666666666666019037e-02 +
                          z * (-1.38888888888741095749e-03 +
                               z * (2.48015872894767294178e-05 +
                                    z * (-2.75573143513906633035e-07 +
                                         z * (2.08757232129817482790e-09 + z * -1.13596475577881948265e-11)))));
    const double ax = fabs(x);
    if (ax < 0.3) return 1.0 - (0.5 * z - z * r);
    const double qx = ax > 0.78125 ? 0.28125 : bits2d(d2bits(z * 0.25) & ~(int64_t)0xffffffff);
    const double hz = 0.5 * z - qx;
    const double a = 1.0 - qx;
    return a - (hz - z * r);
}
SG_HD double fd_reduce(double x, int& k) {
    const double kd = fd_round(x * 6.36619772367581382433e-01);
    k = (int)kd;
    return (x - kd * 1.57079632673412561417e+00) - kd * 6.07710050650619224932e-11;
}
SG_HD double fd_sin(double x) {
    if (fabs(x) <= 7.85398163397448278999e-01) return fd_sin_kernel(x);
    int k;
    const double r = fd_reduce(x, k);
    const int q = k & 3;
    const double v = (q & 1) ? fd_cos_kernel(r) : fd_sin_kernel(r);
    return (q & 2) ? -v : v;
}
SG_HD double fd_cos(double x) {
    if (fabs(x) <= 7.85398163397448278999e-01) return fd_cos_kernel(x);
    int k;
    const double r = fd_reduce(x, k);
    const int q = k & 3;
    const double v = (q & 1) ? fd_sin_kernel(r) : fd_cos_kernel(r);
    return (q == 1 || q == 2) ? -v : v;
}
SG_HD double fd_acos_pq(double z) {
    const double p = z * (1.66666666666666657415e-01 +
                          z * (-3.25565818622400915405e-01 +
                               z * (2.01212532134862925881e-01 +
                                    z * (-4.00555345006794114027e-02 +
                                         z * (7.91534994289814532176e-04 + z * 3.47933107596021167570e-05)))));
    const double q = 1.0 + z * (-2.40339491173441421878e+00 +
                                z * (2.02094576023350569471e+00 +
                                     z * (-6.88283971605453293030e-01 + z * 7.70381505559019352791e-02)));
    return p / q;
}
SG_HD double fd_acos(double x) {
    const double pio2_lo = 6.12323399573676603587e-17;
    const double ax = fabs(x);
    if (ax >= 1) {
        if (x == 1) return 0;
        if (x == -1) return 3.14159265358979311600e+00;
        return (x - x) / (x - x);
    }
    if (ax < 0.5) {
        const double r = fd_acos_pq(x * x);
        return 1.57079632679489655800e+00 - (x - (pio2_lo - x * r));
    }
    if (x < 0) {
        const double z = (1.0 + x) * 0.5;
        const double s = sqrt(z);
        const double w = fd_acos_pq(z) * s - pio2_lo;
        return 3.14159265358979311600e+00 - 2.0 * (s + w);
    }
    const double z = (1.0 - x) * 0.5;
    const double s = sqrt(z);
    const double df = bits2d(d2bits(s) & ~(int64_t)0xffffffff);
    const double c = (z - df * df) / (s + df);
    const double w = fd_acos_pq(z) * s + c;
    return 2.0 * (df + w);
}
SG_HD double fd_exp(double x) {
    if (x != x) return x;
    if (x > 7.09782712893383973096e+02) return bits2d(0x7ff0000000000000LL);
    if (x < -7.45133219101941108420e+02) return 0;
    double hi = x, lo = 0;
    int k = 0;
    const double ax = fabs(x);
    if (ax > 0.5 * 6.93147180559945286227e-01) {
        k = (int)(1.44269504088896338700e+00 * x + (x < 0 ? -0.5 : 0.5));
        hi = x - k * 6.93147180369123816490e-01;
        lo = k * 1.90821492927058770002e-10;
        x = hi - lo;
    } else if (ax < 3.7252902984e-09) {
        return 1.0 + x;
    }
    const double t = x * x;
    const double c = x - t * (1.66666666666666019037e-01 +
                              t * (-2.77777777770155933842e-03 +
                                   t * (6.61375632143793436117e-05 +
                                        t * (-1.65339022054652515390e-06 + t * 4.13813679705723846039e-08))));
    if (k == 0) return 1.0 - ((x * c) / (c - 2.0) - x);
    const double y = 1.0 - ((lo - (x * c) / (2.0 - c)) - hi);
    return fd_pow2(y, k);
}

// ---- small vector types -------------------------------------------------------
template <typename T>
struct V3 {
    T x, y, z;
};
template <typename T> SG_HD V3<T> v3(T x, T y, T z) { return V3<T>{x, y, z}; }
template <typename T> SG_HD V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T> SG_HD V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T> SG_HD V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <typename T> SG_HD void add_to(V3<T>& a, V3<T> b) { a.x += b.x; a.y += b.y; a.z += b.z; }
template <typename T> SG_HD void sub_from(V3<T>& a, V3<T> b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
template <typename T> SG_HD T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> SG_HD T sq(T x) { return x * x; }
template <typename T> SG_HD T norm2(V3<T> a) { return sq(a.x) + sq(a.y) + sq(a.z); }
template <typename T> SG_HD T dist2(V3<T> a, V3<T> b) { return sq(a.x - b.x) + sq(a.y - b.y) + sq(a.z - b.z); }
template <typename T> SG_HD V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// column-major 3x3 (m[i + 3j])
template <typename T> SG_HD V3<T> mat_mul(const T* m, V3<T> v) {
    return {m[0] * v.x + m[3] * v.y + m[6] * v.z, m[1] * v.x + m[4] * v.y + m[7] * v.z,
            m[2] * v.x + m[5] * v.y + m[8] * v.z};
}
template <typename T>
struct Quat {
    T a, b, c, d;
};
// boost::math::quaternion product l * r
template <typename T> SG_HD Quat<T> qmul(Quat<T> l, Quat<T> r) {
    return {l.a * r.a - l.b * r.b - l.c * r.c - l.d * r.d, l.a * r.b + l.b * r.a + l.c * r.d - l.d * r.c,
            l.a * r.c - l.b * r.d + l.c * r.a + l.d * r.b, l.a * r.d + l.b * r.c - l.c * r.b + l.d * r.a};
}
template <typename T> SG_HD void quat_to_mat(Quat<T> q, T* m) {
    const T a = q.a, b = q.b, c = q.c, d = q.d;
    const T aa = a * a, ab = a * b, ac = a * c, ad = a * d, bb = b * b, bc = b * c, bd = b * d, cc = c * c, cd = c * d,
            dd = d * d;
    m[0] = (aa + bb - cc - dd);
    m[3] = 2 * (-ad + bc);
    m[6] = 2 * (ac + bd);
    m[1] = 2 * (ad + bc);
    m[4] = (aa - bb + cc - dd);
    m[7] = 2 * (-ab + cd);
    m[2] = 2 * (-ac + bd);
    m[5] = 2 * (ab + cd);
    m[8] = (aa - bb - cc + dd);
}

// ---- double precision angle / orientation algebra (common.h, quaternion.cpp) ---
SG_HD void normalize_angle(double& x) {
    for (;;) {
        if (x > 3 * kPi) { double n = (x - kPi) / (2 * kPi); x -= 2 * kPi * ceil(n); }
        else if (x < -3 * kPi) { double n = (-x - kPi) / (2 * kPi); x += 2 * kPi * ceil(n); }
        else {
            if (x > kPi) x -= 2 * kPi;
            else if (x < -kPi) x += 2 * kPi;
            return;
        }
    }
}
SG_HD double normalized_angle(double x) { normalize_angle(x); return x; }
SG_HD Quat<double> axis_angle_q(V3<double> axis, double angle) {
    normalize_angle(angle);
    const double c = fd_cos(angle / 2), s = fd_sin(angle / 2);
    return {c, s * axis.x, s * axis.y, s * axis.z};
}
SG_HD Quat<double> rotation_q(V3<double> rot) {
    const double angle = sqrt(norm2(rot));
    if (angle > kEps) return axis_angle_q((1 / angle) * rot, angle);
    return {1, 0, 0, 0};
}
SG_HD void q_normalize_approx(Quat<double>& q) {
    const double s = sq(q.a) + sq(q.b) + sq(q.c) + sq(q.d);
    if (fabs(s - 1) < 1e-6) return;
    const double inv = 1 / sqrt(s);
    q.a *= inv; q.b *= inv; q.c *= inv; q.d *= inv;
}
SG_HD void q_increment(Quat<double>& q, V3<double> rot) {
    q = qmul(rotation_q(rot), q);
    q_normalize_approx(q);
}
SG_HD V3<double> q_to_angle(Quat<double> q) {
    const double c = q.a;
    if (c > -1 && c < 1) {
        double angle = 2 * fd_acos(c);
        if (angle > kPi) angle -= 2 * kPi;
        const double s = fd_sin(angle / 2);
        if (fabs(s) < kEps) return {0, 0, 0};
        const double k = angle / s;
        return {q.b * k, q.c * k, q.d * k};
    }
    return {0, 0, 0};
}
// soft curl (curl.h:30-43); v is always far below max double here
template <typename T> SG_HD void curl_e(T& e, T v) {
    if (e > 0) {
        const T t = (v < (T)kEps) ? T(0) : (v / (v + e));
        e *= t;
    }
}
template <typename T> SG_HD void curl_ed(T& e, V3<T>& d, T v) {
    if (e > 0) {
        const T t = (v < (T)kEps) ? T(0) : (v / (v + e));
        e *= t;
        const T t2 = t * t;
        d.x *= t2; d.y *= t2; d.z *= t2;
    }
}

}  // namespace sg
