/*
 * ORACLE pinning probe (test infrastructure only).  Compiled by the oracle
 * Makefile's `ref` target against the reference's own headers
 * (src/lib/portable_math.h, src/gpu/gpu_rng.cuh, src/gpu/gpu_math.cuh) into
 * oracle/_ref/, and used
 * only by tests/golden/make_golden.py to write the golden vectors that pin
 * the oracle's math restatement.  Not part of the product.
 */
#include <cstdint>
#include "portable_math.h"
#include "gpu_rng.cuh"
#include "gpu_math.cuh"

extern "C" {

void ref_pm_eval(int fn, const double* x, double* y, int n) {
    for (int i = 0; i < n; i++) {
        switch (fn) {
            case 0: y[i] = portable_math::sin(x[i]); break;
            case 1: y[i] = portable_math::cos(x[i]); break;
            case 2: y[i] = portable_math::acos(x[i]); break;
            default: y[i] = portable_math::exp(x[i]); break;
        }
    }
}

/* Seeds the reference's mt19937 restatement the way boost::mt19937(seed)
 * does (x[0] = seed, x[k] = 1812433253 (x[k-1] ^ x[k-1] >> 30) + k, index n),
 * then draws like or_mt_probe. */
void ref_mt_probe(uint32_t seed, int n, uint32_t* raw, double a, double b, double* fl, int lo, int hi, int* in) {
    gpusmina::MTState s;
    s.x[0] = seed;
    for (int k = 1; k < gpusmina::MT_N; k++) s.x[k] = 1812433253u * (s.x[k - 1] ^ (s.x[k - 1] >> 30)) + (unsigned)k;
    s.i = gpusmina::MT_N;
    for (int i = 0; i < n; i++) raw[i] = gpusmina::mt_next(s);
    for (int i = 0; i < n; i++) fl[i] = gpusmina::random_fl(a, b, s);
    for (int i = 0; i < n; i++) in[i] = gpusmina::random_int(lo, hi, s);
}

/* Quaternion and angle math of the reference's FP64 device code (its
 * restatement of common.h / quaternion.cpp, host-compiled here): per input
 * row in[7] = (axis xyz, angle, rotation xyz) with q0[4], writes out[22] =
 * normalized_angle(angle), angle_to_quaternion(axis, angle) [4],
 * angle_to_quaternion(rotation) [4], quaternion_increment(q0, rotation) [4],
 * quaternion_to_r3(q0) [9, column-major]. */
void ref_quat_probe(const double* in, const double* q0, double* out, int n) {
    using namespace gpusmina;
    for (int k = 0; k < n; k++) {
        const double* x = in + 7 * k;
        double* o = out + 22 * k;
        const vec3<double> axis = mk(x[0], x[1], x[2]), rot = mk(x[4], x[5], x[6]);
        o[0] = normalized_angle(x[3]);
        const quat<double> a = angle_to_quaternion(axis, x[3]);
        const quat<double> b = angle_to_quaternion(rot);
        quat<double> c = mkq(q0[4 * k], q0[4 * k + 1], q0[4 * k + 2], q0[4 * k + 3]);
        const mat3<double> m = quaternion_to_r3(c);
        quaternion_increment(c, rot);
        const quat<double> qs[3] = {a, b, c};
        for (int j = 0; j < 3; j++) {
            o[1 + 4 * j] = qs[j].a; o[2 + 4 * j] = qs[j].b; o[3 + 4 * j] = qs[j].c; o[4 + 4 * j] = qs[j].d;
        }
        for (int j = 0; j < 9; j++) o[13 + j] = m.d[j];
    }
}

}
