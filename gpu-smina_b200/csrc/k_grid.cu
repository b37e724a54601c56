// Grid-map construction (cache::populate, cache.cpp:116-206).
//
// 1. Receptor cell lists (szv_grid.h:55-221): for every 3 A cell, the heavy
//    typed receptor atoms within the cutoff of both the search box and the
//    cell's brick, in receptor order.  cache::populate builds each cell's
//    list for the brick of the first grid point that queries the cell (a
//    point on a cell face gives a flat brick); k_cell_lists takes that brick
//    per axis from the host (first query in x, y, z loop order).  The
//    direct-sum path uses full 3 A bricks.  One warp per cell, ordered
//    compaction with ballots.
// 2. k_grid_map64: one thread per grid point, FP64 sums over the point's
//    cell list in receptor order for a chunk of ligand types; identical
//    rounding to the CPU's loop (each type's sum is independent).
//    A user grid (--user_grid) is added to every map at the point's index
//    coordinates (x, y, z), with the cache's slope, as cache::populate does
//    (cache.cpp:204-205).
// 3. k_grid_pack: packed-corner FP32 / FP16 copies for the mixed-precision path.
// Built without FMA contraction, like the CPU code it reproduces.
#include "grid64.cuh"

namespace sg {

__device__ __forceinline__ double closest_between(double b, double e, double x) {
    if (x <= b) return b;
    if (x >= e) return e;
    return x;
}
__device__ __forceinline__ double brick_d2(double b0, double b1, double b2, double e0, double e1, double e2, double x,
                                           double y, double z) {
    const double c0 = closest_between(b0, e0, x), c1 = closest_between(b1, e1, y), c2 = closest_between(b2, e2, z);
    return sq(c0 - x) + sq(c1 - y) + sq(c2 - z);
}

// pass 0: count; pass 1: fill (start[] already scanned)
__global__ void k_cell_lists(int natoms, const double* xyz, const int* type, DGeom g, double cutoff_sqr,
                             const double* lo, const double* hi, int* count, const int* start, int* atoms, int pass) {
    const int cell = blockIdx.x;
    const int ncells = g.cell_dim[0] * g.cell_dim[1] * g.cell_dim[2];
    if (cell >= ncells) return;
    const int cx = cell % g.cell_dim[0], cy = (cell / g.cell_dim[0]) % g.cell_dim[1],
              cz = cell / (g.cell_dim[0] * g.cell_dim[1]);
    const double l0 = lo[cx], l1 = lo[g.cell_dim[0] + cy], l2 = lo[g.cell_dim[0] + g.cell_dim[1] + cz];
    const double h0 = hi[cx], h1 = hi[g.cell_dim[0] + cy], h2 = hi[g.cell_dim[0] + g.cell_dim[1] + cz];
    const int lane = threadIdx.x;
    int running = 0;
    const bool empty = !(l0 == l0 && l1 == l1 && l2 == l2);  // NaN brick: no grid point in this cell
    for (int base = 0; base < natoms; base += 32) {
        const int i = base + lane;
        bool pass_ok = false;
        if (!empty && i < natoms) {
            const int t = type[i];
            if (t < kNumTypes && !is_h(t)) {
                const double x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
                pass_ok = brick_d2(g.gd_begin[0], g.gd_begin[1], g.gd_begin[2], g.gd_end[0], g.gd_end[1], g.gd_end[2], x,
                                   y, z) < cutoff_sqr &&
                          brick_d2(l0, l1, l2, h0, h1, h2, x, y, z) < cutoff_sqr;
            }
        }
        const unsigned mask = __ballot_sync(0xffffffffu, pass_ok);
        if (pass == 1 && pass_ok) atoms[start[cell] + running + __popc(mask & ((1u << lane) - 1))] = i;
        running += __popc(mask);
    }
    if (pass == 0 && lane == 0) count[cell] = running;
}

// one thread per grid point; threads of a warp cover a compact 8x4 tile
__global__ void __launch_bounds__(256) k_grid_map64(DGeom g, int natoms, const double* xyz, const int* rtype,
                                                    const double* rcharge, const int* cstart, const int* catoms,
                                                    const double* fast, int nc, int n, double factor, double cutoff_sqr,
                                                    const int* types, int ntypes, double** maps, double** cmaps,
                                                    const double* ugrid, DGeom ug, double ug_slope) {
    const int x = blockIdx.x * 8 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z * 4 + threadIdx.z;
    if (x >= g.dim[0] || y >= g.dim[1] || z >= g.dim[2]) return;
    const double px = g.init[0] + g.factor_inv[0] * x, py = g.init[1] + g.factor_inv[1] * y,
                 pz = g.init[2] + g.factor_inv[2] * z;
    const int cx = (int)floor(px / 3.0) - g.cell_off[0], cy = (int)floor(py / 3.0) - g.cell_off[1],
              cz = (int)floor(pz / 3.0) - g.cell_off[2];
    const bool cell_ok = cx >= 0 && cy >= 0 && cz >= 0 && cx < g.cell_dim[0] && cy < g.cell_dim[1] && cz < g.cell_dim[2];
    const int cell = cell_ok ? cx + g.cell_dim[0] * (cy + g.cell_dim[1] * cz) : 0;
    const int b = cell_ok ? cstart[cell] : 0, e = cell_ok ? cstart[cell + 1] : 0;
    const size_t idx = (size_t)x + (size_t)g.dim[0] * ((size_t)y + (size_t)g.dim[1] * z);
    const double u = ugrid ? grid_value64(ug, ugrid, V3<double>{(double)x, (double)y, (double)z}, ug_slope, 1000.0)
                           : 0.0;
    constexpr int CH = 8;
    for (int t0 = 0; t0 < ntypes; t0 += CH) {
        double aff[CH], chg[CH];
        int pidx[CH];
        bool swp[CH];
#pragma unroll
        for (int j = 0; j < CH; j++) { aff[j] = 0; chg[j] = 0; pidx[j] = 0; swp[j] = false; }
        const int nt = min(CH, ntypes - t0);
        for (int k = b; k < e; k++) {
            const int a = catoms[k];
            const double r2 = sq(xyz[3 * a] - px) + sq(xyz[3 * a + 1] - py) + sq(xyz[3 * a + 2] - pz);
            if (r2 <= cutoff_sqr) {
                const int t1 = rtype[a];
                const size_t i = (size_t)(factor * r2);
                const double q = rcharge[a];
#pragma unroll
                for (int j = 0; j < CH; j++) {
                    if (j >= nt) break;
                    const int t2 = types[t0 + j];
                    const bool sw = t1 > t2;
                    const int p = sw ? tri_index(t2, t1) : tri_index(t1, t2);
                    const double* f = fast + ((size_t)p * n + i) * nc;
                    if (nc > 1) {
                        const double c1 = sw ? f[2] : f[1], c2 = sw ? f[1] : f[2];
                        aff[j] += f[0] + c1 * fabs(q);
                        chg[j] += c2 + f[3] * q;
                    } else {
                        aff[j] += f[0];
                    }
                }
            }
        }
        for (int j = 0; j < nt; j++) {
            maps[t0 + j][idx] = ugrid ? aff[j] + u : aff[j];
            if (nc > 1) cmaps[t0 + j][idx] = chg[j];
        }
    }
}

// Packed-corner copies for the mixed-precision path: cell (x, y, z) of the
// (dim-1)^3 cells stores its 8 corners contiguously, so one trilinear lookup
// is one 32 B (FP32) or 16 B (FP16) load instead of four row segments.
__global__ void k_grid_pack(DGeom g, const double* src, float4* dst32, uint4* dst16) {
    const int cx = g.dim[0] - 1, cy = g.dim[1] - 1, cz = g.dim[2] - 1;
    const size_t ncells = (size_t)cx * cy * cz;
    const size_t d0 = g.dim[0], d01 = (size_t)g.dim[0] * g.dim[1];
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < ncells; c += (size_t)gridDim.x * blockDim.x) {
        const size_t x = c % cx, y = (c / cx) % cy, z = c / ((size_t)cx * cy);
        const double* b = src + x + d0 * y + d01 * z;
        const double v[8] = {b[0], b[1], b[d0], b[d0 + 1], b[d01], b[d01 + 1], b[d01 + d0], b[d01 + d0 + 1]};
        if (dst32) {
            dst32[2 * c] = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
            dst32[2 * c + 1] = make_float4((float)v[4], (float)v[5], (float)v[6], (float)v[7]);
        }
        if (dst16) {
            uint32_t w[4];
            for (int k = 0; k < 4; k++)
                w[k] = (uint32_t)__half_as_ushort(__double2half(v[2 * k])) |
                       ((uint32_t)__half_as_ushort(__double2half(v[2 * k + 1])) << 16);
            dst16[c] = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

cudaError_t launch_cell_lists(int natoms, const double* xyz, const int* type, const DGeom& g, double cutoff_sqr,
                              const double* lo, const double* hi, int* count, const int* start, int* atoms, int pass,
                              cudaStream_t s) {
    const int ncells = g.cell_dim[0] * g.cell_dim[1] * g.cell_dim[2];
    k_cell_lists<<<ncells, 32, 0, s>>>(natoms, xyz, type, g, cutoff_sqr, lo, hi, count, start, atoms, pass);
    return cudaGetLastError();
}

cudaError_t launch_grid_map64(const DGeom& g, int natoms, const double* xyz, const int* rtype, const double* rcharge,
                              const int* cstart, const int* catoms, const DTables& T, const int* types, int ntypes,
                              double** maps, double** cmaps, const double* ugrid, const DGeom& ug, double ug_slope,
                              cudaStream_t s) {
    dim3 block(8, 8, 4);
    dim3 grid((g.dim[0] + 7) / 8, (g.dim[1] + 7) / 8, (g.dim[2] + 3) / 4);
    k_grid_map64<<<grid, block, 0, s>>>(g, natoms, xyz, rtype, rcharge, cstart, catoms, T.fast, T.nc, T.n, T.factor,
                                        T.cutoff_sqr, types, ntypes, maps, cmaps, ugrid, ug, ug_slope);
    return cudaGetLastError();
}

cudaError_t launch_grid_pack(const DGeom& g, const double* src, float4* d32, uint4* d16, cudaStream_t s) {
    k_grid_pack<<<148 * 8, 256, 0, s>>>(g, src, d32, d16);
    return cudaGetLastError();
}

}  // namespace sg
