/*
 * ORACLE pinning probe (test infrastructure only).  Compiled by the oracle
 * Makefile's `ref` target against the reference's own headers
 * (src/lib/portable_math.h, src/gpu/gpu_rng.cuh) into oracle/_ref/, and used
 * only by tests/golden/make_golden.py to write the golden vectors that pin
 * the oracle's math restatement.  Not part of the product.
 */
#include <cstdint>
#include "portable_math.h"
#include "gpu_rng.cuh"

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

}
