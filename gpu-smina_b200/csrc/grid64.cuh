// grid::evaluate_aux (grid.cpp:111-236) in FP64: clamp each axis to the
// grid (region -1 / 0 / 1, out-of-grid distance into the penalty), 8-corner
// trilinear value, curl; the derivative form also gives the gradient with the
// penalty's slope outside the grid.  Operand order follows the CPU code, and
// every file that includes this is compiled without FMA contraction, so the
// results round as the CPU's do.
#pragma once
#include "sg_dev.cuh"

namespace sg {

struct Trilin64 {
    double f000, f100, f010, f110, f001, f101, f011, f111;
    double x, y, z, penalty;
    int region[3];
};

__device__ __forceinline__ Trilin64 trilin64(const DGeom& G, const double* D, V3<double> loc, double slope) {
    Trilin64 t;
    double s[3] = {(loc.x - G.init[0]) * G.factor[0], (loc.y - G.init[1]) * G.factor[1],
                   (loc.z - G.init[2]) * G.factor[2]};
    double miss[3] = {0, 0, 0};
    int a[3];
    for (int i = 0; i < 3; i++) {
        if (s[i] < 0) {
            miss[i] = -s[i]; t.region[i] = -1; a[i] = 0; s[i] = 0;
        } else if (s[i] >= G.dim_fl_minus_1[i]) {
            miss[i] = s[i] - G.dim_fl_minus_1[i]; t.region[i] = 1; a[i] = G.dim[i] - 2; s[i] = 1;
        } else {
            t.region[i] = 0; a[i] = (int)(unsigned long long)s[i]; s[i] -= (double)a[i];
        }
    }
    t.penalty = slope * (miss[0] * G.factor_inv[0] + miss[1] * G.factor_inv[1] + miss[2] * G.factor_inv[2]);
    const size_t d0 = G.dim[0], d01 = (size_t)G.dim[0] * G.dim[1];
    const double* b = D + a[0] + d0 * a[1] + d01 * a[2];
    t.f000 = b[0]; t.f100 = b[1]; t.f010 = b[d0]; t.f110 = b[d0 + 1];
    t.f001 = b[d01]; t.f101 = b[d01 + 1]; t.f011 = b[d01 + d0]; t.f111 = b[d01 + d0 + 1];
    t.x = s[0]; t.y = s[1]; t.z = s[2];
    return t;
}

__device__ __forceinline__ double trilin64_value(const Trilin64& t) {
    const double x = t.x, y = t.y, z = t.z;
    const double mx = 1 - x, my = 1 - y, mz = 1 - z;
    return t.f000 * mx * my * mz + t.f100 * x * my * mz + t.f010 * mx * y * mz + t.f110 * x * y * mz +
           t.f001 * mx * my * z + t.f101 * x * my * z + t.f011 * mx * y * z + t.f111 * x * y * z;
}

// value with derivative (grid::evaluate_aux with deriv)
static __device__ double grid_aux64(const DGeom& G, const double* D, V3<double> loc, double slope, double v,
                             V3<double>& deriv) {
    const Trilin64 t = trilin64(G, D, loc, slope);
    double f = trilin64_value(t);
    const double x = t.x, y = t.y, z = t.z;
    const double mx = 1 - x, my = 1 - y, mz = 1 - z;
    const double xg = -(t.f000 * my * mz) + t.f100 * my * mz + -(t.f010 * y * mz) + t.f110 * y * mz +
                      -(t.f001 * my * z) + t.f101 * my * z + -(t.f011 * y * z) + t.f111 * y * z;
    const double yg = -(t.f000 * mx * mz) + -(t.f100 * x * mz) + t.f010 * mx * mz + t.f110 * x * mz +
                      -(t.f001 * mx * z) + -(t.f101 * x * z) + t.f011 * mx * z + t.f111 * x * z;
    const double zg = -(t.f000 * mx * my) + -(t.f100 * x * my) + -(t.f010 * mx * y) + -(t.f110 * x * y) +
                      t.f001 * mx * my + t.f101 * x * my + t.f011 * mx * y + t.f111 * x * y;
    V3<double> grad{xg, yg, zg};
    curl_ed(f, grad, v);
    deriv.x = G.factor[0] * (t.region[0] == 0 ? grad.x : 0.0) + slope * t.region[0];
    deriv.y = G.factor[1] * (t.region[1] == 0 ? grad.y : 0.0) + slope * t.region[1];
    deriv.z = G.factor[2] * (t.region[2] == 0 ? grad.z : 0.0) + slope * t.region[2];
    return f + t.penalty;
}

// value only (grid::evaluate_aux without deriv)
static __device__ double grid_value64(const DGeom& G, const double* D, V3<double> loc, double slope, double v) {
    const Trilin64 t = trilin64(G, D, loc, slope);
    double f = trilin64_value(t);
    curl_e(f, v);
    return f + t.penalty;
}

}  // namespace sg
