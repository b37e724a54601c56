// Plain (FP64) path, part 2: BFGS with its line searches, mutation,
// Metropolis acceptance and the output container, one warp per chain.
// Control flow is warp-uniform; scalars that need an order-sensitive
// reduction are reduced by lane 0 in the reference's order and broadcast.
// Reference: bfgs.h:30-282; conf.h:98-404; mutate.cpp:35-63;
// monte_carlo.cpp:44-48,95-130; coords.cpp:25-58; random.cpp:28-80;
// quaternion.cpp:42-139.
#pragma once
#include "dock64_eval.cuh"

namespace sg {

// ---- mt19937 on lane 0, Boost's uniform_real / uniform_int ------------------------
__device__ uint32_t mt_next(uint32_t* st) {
    int i = (int)st[624];
    if (i >= 624) {
        for (int k = 0; k < 624; k++) {
            const uint32_t y = (st[k] & 0x80000000u) | (st[k + 1 < 624 ? k + 1 : 0] & 0x7fffffffu);
            st[k] = st[k + 397 < 624 ? k + 397 : k + 397 - 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        i = 0;
    }
    uint32_t z = st[i];
    st[624] = (uint32_t)(i + 1);
    z ^= z >> 11;
    z ^= (z << 7) & 0x9d2c5680u;
    z ^= (z << 15) & 0xefc60000u;
    z ^= z >> 18;
    return z;
}
__device__ double rand_fl(W64& w, double a, double b) {
    double r = 0;
    if (w.lane == 0) {
        for (;;) {
            r = (double)mt_next(w.mt) / (4294967295.0 + 1) * (b - a) + a;
            if (r < b) break;
        }
    }
    return __shfl_sync(kFull, r, 0);
}
__device__ int rand_int(W64& w, int a, int b) {
    int out = a;
    if (w.lane == 0) {
        const uint32_t range = (uint32_t)b - (uint32_t)a;
        if (range != 0) {
            uint32_t bucket = 0xffffffffu / (range + 1);
            if (0xffffffffu % (range + 1) == range) ++bucket;
            for (;;) {
                const uint32_t r = mt_next(w.mt) / bucket;
                if (r <= range) { out = (int)(r + (uint32_t)a); break; }
            }
        }
    }
    return __shfl_sync(kFull, out, 0);
}
__device__ V3<double> rand_in_sphere(W64& w) {
    for (;;) {
        const double r1 = rand_fl(w, -1, 1), r2 = rand_fl(w, -1, 1), r3 = rand_fl(w, -1, 1);
        const V3<double> t{r1, r2, r3};
        if (norm2(t) < 1) return t;
    }
}

// ---- ordered scalar product (lane 0), broadcast -------------------------------------
__device__ double sprod64(W64& w, const double* a, const double* b, int n) {
    double t = 0;
    if (w.lane == 0)
        for (int i = 0; i < n; i++) t += a[i] * b[i];
    return __shfl_sync(kFull, t, 0);
}
__device__ void vcopy(W64& w, double* d, const double* s, int n) {
    for (int i = w.lane; i < n; i += 32) d[i] = s[i];
    __syncwarp();
}

// conf::increment (torsions normalized, orientation not re-normalized beyond approx)
__device__ void conf_increment64(W64& w, double* x, const double* p, double alpha) {
    const DModel& m = *w.m;
    for (int l = w.lane; l < m.nlig; l += 32) {
        const int f = m.lig_root[l];
        double* c = x + m.fconf[f];
        const double* d = p + m.fdof[f];
        const V3<double> dp = alpha * V3<double>{d[0], d[1], d[2]};
        c[0] += dp.x; c[1] += dp.y; c[2] += dp.z;
        Quat<double> q{c[3], c[4], c[5], c[6]};
        q_increment(q, alpha * V3<double>{d[3], d[4], d[5]});
        c[3] = q.a; c[4] = q.b; c[5] = q.c; c[6] = q.d;
    }
    for (int k = w.lane; k < m.ntors; k += 32) {
        double& t = x[m.tor_conf[k]];
        t += normalized_angle(alpha * p[m.tor_dof[k]]);
        normalize_angle(t);
    }
    __syncwarp();
}

// conf::operator()(index): the value of change coordinate i
__device__ double conf_value64(const DModel& m, const double* x, int i) {
    for (int l = 0; l < m.nlig; l++) {
        const int f = m.lig_root[l];
        const int d0 = m.fdof[f];
        if (i >= d0 && i < d0 + 3) return x[m.fconf[f] + (i - d0)];
        if (i >= d0 + 3 && i < d0 + 6) {
            const double* c = x + m.fconf[f];
            const V3<double> a = q_to_angle(Quat<double>{c[3], c[4], c[5], c[6]});
            const int j = i - d0 - 3;
            return j == 0 ? a.x : j == 1 ? a.y : a.z;
        }
    }
    for (int k = 0; k < m.ntors; k++)
        if (m.tor_dof[k] == i) return x[m.tor_conf[k]];
    return 0;
}

struct EvalMode {
    double v[3];
    double slope;
    bool direct;
};

__device__ double feval(W64& w, const double* x, double* g, const EvalMode& em) {
    return eval_deriv64(w, x, em.v, em.slope, em.direct, g);
}

// ---- line searches ----------------------------------------------------------------------
__device__ double fast_line_search64(W64& w, const double* x, const double* g, double f0, const double* p,
                                     double* x_new, double* g_new, double& f1, const EvalMode& em) {
    const DModel& m = *w.m;
    const int n = m.dof;
    double alpha = 1;
    const double pg = sprod64(w, p, g, n);
    for (unsigned trial = 0; trial < 10; trial++) {
        vcopy(w, x_new, x, m.conf_size);
        conf_increment64(w, x_new, p, alpha);
        f1 = feval(w, x_new, g_new, em);
        if (f1 - f0 < 0.0001 * alpha * pg) break;
        alpha *= 0.5;
    }
    return alpha;
}

__device__ double accurate_line_search64(W64& w, const double* x, const double* g, double f0, const double* p,
                                         double* x_new, double* g_new, double& f1, const EvalMode& em) {
    const DModel& m = *w.m;
    const int n = m.dof;
    double a, alpha, alpha2 = 0, alamin, b, disc, f2 = 0, rhs1, rhs2, tmplam = 0;
    const double ALF = 1.0e-4, FIRST = 1.0;
    const double slope = sprod64(w, g, p, n);
    if (slope >= 0) {
        vcopy(w, x_new, x, m.conf_size);
        for (int i = w.lane; i < n; i += 32) g_new[i] = 0;
        __syncwarp();
        return 0;
    }
    double test = 0;
    for (int i = w.lane; i < n; i += 32) {
        const double temp = fabs(p[i]) / fmax(fabs(conf_value64(m, x, i)), 1.0);
        if (temp > test) test = temp;
    }
    for (int o = 16; o > 0; o >>= 1) test = fmax(test, __shfl_xor_sync(kFull, test, o));
    alamin = kEps / test;
    alpha = FIRST;
    for (;;) {
        vcopy(w, x_new, x, m.conf_size);
        conf_increment64(w, x_new, p, alpha);
        f1 = feval(w, x_new, g_new, em);
        if (alpha < alamin) {
            vcopy(w, x_new, x, m.conf_size);
            for (int i = w.lane; i < n; i += 32) g_new[i] = 0;
            __syncwarp();
            return 0;
        } else if (f1 <= f0 + ALF * alpha * slope) {
            return alpha;
        } else {
            if (alpha == FIRST) {
                tmplam = -slope / (2.0 * (f1 - f0 - slope));
            } else {
                rhs1 = f1 - f0 - alpha * slope;
                rhs2 = f2 - f0 - alpha2 * slope;
                a = (rhs1 / (alpha * alpha) - rhs2 / (alpha2 * alpha2)) / (alpha - alpha2);
                b = (-alpha2 * rhs1 / (alpha * alpha) + alpha * rhs2 / (alpha2 * alpha2)) / (alpha - alpha2);
                if (a == 0.0) tmplam = -slope / (2.0 * b);
                else {
                    disc = b * b - 3.0 * a * slope;
                    if (disc < 0) tmplam = 0.5 * alpha;
                    else if (b <= 0) tmplam = (-b + sqrt(disc)) / (3.0 * a);
                    else tmplam = -slope / (b + sqrt(disc));
                }
                if (tmplam > .5 * alpha) tmplam = .5 * alpha;
            }
        }
        alpha2 = alpha;
        f2 = f1;
        alpha = fmax(tmplam, 0.1 * alpha);
    }
}

// ---- BFGS on the triangular inverse Hessian -------------------------------------------
__device__ __forceinline__ int tri(int i, int j) { return i < j ? i + j * (j + 1) / 2 : j + i * (i + 1) / 2; }

__device__ void minus_mat_vec64(W64& w, const double* h, const double* in, double* out, int n) {
    for (int i = w.lane; i < n; i += 32) {
        double sum = 0;
        for (int j = 0; j < n; j++) sum += h[tri(i, j)] * in[j];
        out[i] = -sum;
    }
    __syncwarp();
}

__device__ void bfgs_update64(W64& w, double* h, const double* p, const double* y, double alpha, int n) {
    const double yp = sprod64(w, y, p, n);
    if (alpha * yp < kEps) return;
    double* mhy = w.s + w.L.mhy;
    minus_mat_vec64(w, h, y, mhy, n);
    const double yhy = -sprod64(w, y, mhy, n);
    const double r = 1 / (alpha * yp);
    for (int j = 0; j < n; j++)
        for (int i = w.lane; i <= j; i += 32)
            h[i + j * (j + 1) / 2] += alpha * r * (mhy[i] * p[j] + mhy[j] * p[i]) + +alpha * alpha * (r * r * yhy + r) * p[i] * p[j];
    __syncwarp();
}

// ---- QuickVina 2 history (not smina's search) ----------------------------------------------
// QuickVina 2 (Alhossary, Handoko, Mu and Kwoh, Bioinformatics 31:2214, 2015)
// skips a local optimisation whose start the chain's recent history already
// accounts for.  The history holds the last 5n points (n = dof) that local
// optimisations visited, with their energies and gradient signs.  A stored
// point e is consistent with a start (x, f, g) when, in every coordinate in
// which both gradients have the same nonzero sign, "gradient positive" equals
// "x_i > e_i" xor "f > f_e".  A start is worth optimising when a consistent
// point is among its 4n nearest (squared distance in change coordinates,
// ties to the lower slot); until 5n points are stored, every start is.  The
// decisions are those of the reference's gpu_mc.cuh:144-264, which the
// checker restates and this path matches bit for bit.
//
// The device layout and the check are this file's own:
//  - coordinates are stored coordinate-major, so for one coordinate the
//    lanes read consecutive slots;
//  - lane l owns slots l, l + 32, ...; their squared distances and "start
//    above the point" bits build up in registers while the coordinates
//    stream past (the start's coordinate comes by shuffle), so nothing is
//    written back but the new point;
//  - the sign test is mask algebra on 64-bit words: it applies where
//    nz_e & nz_x & ~(pos_e ^ pos_x), and a point fails when any of those
//    coordinates has pos_x ^ above ^ uphill set.
constexpr int kHistSlotsPerLane = (5 * kHistMaxN + 31) / 32;

__device__ __forceinline__ Hist64 hist64_view(double* d, unsigned long long* u, int n) {
    const size_t cap = (size_t)5 * n;
    return Hist64{d, d + (size_t)n * cap, u, u + 2 * cap};
}

// (nonzero, positive) masks of the gradient's n coordinates, on every lane
__device__ __forceinline__ ulonglong2 grad_signs64(const W64& w, const double* g, int n) {
    unsigned nz[2], pos[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int i = 32 * h + w.lane;
        const double v = i < n ? g[i] : 0.0;
        nz[h] = __ballot_sync(kFull, !(v == 0));
        pos[h] = __ballot_sync(kFull, v > 0);
    }
    return make_ulonglong2(nz[0] | (unsigned long long)nz[1] << 32, pos[0] | (unsigned long long)pos[1] << 32);
}

// stores (x, f, sign(g)) in the next slot (the oldest point once the ring is full)
__device__ void hist64_add(W64& w, const Hist64& H, const double* x, double f, const double* g) {
    const DModel& m = *w.m;
    const int n = m.dof, cap = 5 * n;
    const unsigned long long adds = __shfl_sync(kFull, w.lane == 0 ? *H.adds : 0ull, 0);
    const int slot = (int)(adds % (unsigned long long)cap);
    const ulonglong2 sg = grad_signs64(w, g, n);
    for (int i = w.lane; i < n; i += 32) H.x[(size_t)i * cap + slot] = conf_value64(m, x, i);
    if (w.lane == 0) {
        H.f[slot] = f;
        H.mask[2 * slot] = sg.x;
        H.mask[2 * slot + 1] = sg.y;
        *H.adds = adds + 1;
    }
    __syncwarp();
}

// true when a local optimisation from (x, f, g) should run
__device__ bool hist64_interesting(W64& w, const Hist64& H, const double* x, double f, const double* g) {
    const DModel& m = *w.m;
    const int n = m.dof, cap = 5 * n;
    const unsigned long long adds = __shfl_sync(kFull, w.lane == 0 ? *H.adds : 0ull, 0);
    if (adds < (unsigned long long)cap) return true;
    const double x_lo = w.lane < n ? conf_value64(m, x, w.lane) : 0.0;
    const double x_hi = w.lane + 32 < n ? conf_value64(m, x, w.lane + 32) : 0.0;
    const ulonglong2 sx = grad_signs64(w, g, n);
    double d2[kHistSlotsPerLane];
    unsigned long long above[kHistSlotsPerLane];
#pragma unroll
    for (int k = 0; k < kHistSlotsPerLane; k++) { d2[k] = 0; above[k] = 0; }
    for (int i = 0; i < n; i++) {
        const double xi = __shfl_sync(kFull, i < 32 ? x_lo : x_hi, i & 31);
        const double* row = H.x + (size_t)i * cap;
#pragma unroll
        for (int k = 0; k < kHistSlotsPerLane; k++) {
            const int e = w.lane + 32 * k;
            if (e < cap) {
                const double dx = row[e] - xi;  // summed in coordinate order
                d2[k] += dx * dx;
                if (dx < 0) above[k] |= 1ull << i;
            }
        }
    }
    // nearest consistent point, in (distance, slot) order
    double best = kMaxFl;
    int besti = cap;
#pragma unroll
    for (int k = 0; k < kHistSlotsPerLane; k++) {
        const int e = w.lane + 32 * k;
        if (e < cap) {
            const unsigned long long nz = H.mask[2 * e], pos = H.mask[2 * e + 1];
            const unsigned long long uphill = f - H.f[e] > 0 ? ~0ull : 0ull;
            const unsigned long long applies = nz & sx.x & ~(pos ^ sx.y);
            if ((applies & (sx.y ^ above[k] ^ uphill)) == 0 && d2[k] < best) { best = d2[k]; besti = e; }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(kFull, best, o);
        const int oi = __shfl_xor_sync(kFull, besti, o);
        if (ob < best || (ob == best && oi < besti)) { best = ob; besti = oi; }
    }
    if (besti >= cap) return false;
    // its rank: the points strictly before it in (distance, slot) order
    int ahead = 0;
#pragma unroll
    for (int k = 0; k < kHistSlotsPerLane; k++) {
        const int e = w.lane + 32 * k;
        if (e < cap) ahead += d2[k] < best || (d2[k] == best && e < besti);
    }
    for (int o = 16; o > 0; o >>= 1) ahead += __shfl_xor_sync(kFull, ahead, o);
    return ahead < 4 * n;
}

__device__ double bfgs64(W64& w, double* x, int maxiters, int accurate, int early, const EvalMode& em,
                         const Hist64* vis = nullptr) {
    const DModel& m = *w.m;
    const int n = m.dof;
    double* S = w.s;
    double* h = S + w.L.h;
    double *g = S + w.L.g, *g_new = S + w.L.g_new, *g_orig = S + w.L.g_orig, *p = S + w.L.p, *y = S + w.L.y;
    double *x_new = S + w.L.x_new, *x_orig = S + w.L.x_orig;
    for (int t = w.lane; t < n * (n + 1) / 2; t += 32) h[t] = 0;
    __syncwarp();
    for (int i = w.lane; i < n; i += 32) h[i + i * (i + 1) / 2] = 1;
    __syncwarp();
    double f0 = feval(w, x, g, em);
    if (vis) {
        if (!hist64_interesting(w, *vis, x, f0, g)) return f0;
        hist64_add(w, *vis, x, f0, g);
    }
    const double f_orig = f0;
    vcopy(w, g_orig, g, n);
    vcopy(w, x_orig, x, m.conf_size);
    for (int step = 0; step < maxiters; step++) {
        minus_mat_vec64(w, h, g, p, n);
        double f1 = 0;
        const double alpha = accurate ? accurate_line_search64(w, x, g, f0, p, x_new, g_new, f1, em)
                                      : fast_line_search64(w, x, g, f0, p, x_new, g_new, f1, em);
        if (alpha == 0) break;
        for (int i = w.lane; i < n; i += 32) { double t = g_new[i]; t -= g[i]; y[i] = t; }
        __syncwarp();
        const double prevf0 = f0;
        f0 = f1;
        vcopy(w, x, x_new, m.conf_size);
        if (early && fabs(prevf0 - f0) < 1e-5) break;
        vcopy(w, g, g_new, n);
        const double gn = sprod64(w, g, g, n);
        if (!(gn >= 1e-4)) break;
        if (step == 0) {
            const double yy = sprod64(w, y, y, n);
            if (fabs(yy) > kEps) {
                const double d = alpha * sprod64(w, y, p, n) / yy;
                for (int i = w.lane; i < n; i += 32) h[i + i * (i + 1) / 2] = d;
                __syncwarp();
            }
        }
        bfgs_update64(w, h, p, y, alpha, n);
        if (vis) hist64_add(w, *vis, x, f0, g);
    }
    if (!(f0 <= f_orig)) {
        f0 = f_orig;
        vcopy(w, x, x_orig, m.conf_size);
        vcopy(w, g, g_orig, n);
    }
    return f0;
}

// ---- Monte Carlo pieces ----------------------------------------------------------------
__device__ double gyration64(W64& w, int l) {
    const DModel& m = *w.m;
    double r = 0;
    if (w.lane == 0) {
        double acc = 0;
        unsigned counter = 0;
        const V3<double> o = ld3(w.s + w.L.origin + 3 * m.lig_root[l]);
        for (int i = m.lig_begin[l]; i < m.lig_end[l]; i++)
            if (!is_h(m.type[i])) { acc += dist2(ld3(w.s + w.L.coords + 3 * i), o); ++counter; }
        r = counter > 0 ? sqrt(acc / counter) : 0;
    }
    return __shfl_sync(kFull, r, 0);
}

__device__ void mutate64(W64& w, double* x, double amplitude) {
    const DModel& m = *w.m;
    int num = 0;
    for (int b = 0; b < m.nblocks; b++) num += (m.blk_rigid[b] ? 2 : 0) + m.blk_ntors[b];
    if (num == 0) return;
    int which = rand_int(w, 0, num - 1);
    int lig = 0;
    for (int b = 0; b < m.nblocks; b++) {
        double* c = x + m.blk_conf[b];
        if (m.blk_rigid[b]) {
            if (which == 0) {
                const V3<double> d = amplitude * rand_in_sphere(w);
                if (w.lane == 0) { c[0] += d.x; c[1] += d.y; c[2] += d.z; }
                __syncwarp();
                return;
            }
            --which;
            if (which == 0) {
                const double gr = gyration64(w, lig);
                if (gr > kEps) {
                    const V3<double> rot = amplitude / gr * rand_in_sphere(w);
                    if (w.lane == 0) {
                        Quat<double> q{c[3], c[4], c[5], c[6]};
                        q_increment(q, rot);
                        c[3] = q.a; c[4] = q.b; c[5] = q.c; c[6] = q.d;
                    }
                    __syncwarp();
                }
                return;
            }
            --which;
            c += 7;
            lig++;
        }
        if (which < m.blk_ntors[b]) {
            const double t = rand_fl(w, -kPi, kPi);
            if (w.lane == 0) c[which] = t;
            __syncwarp();
            return;
        }
        which -= m.blk_ntors[b];
    }
}

__device__ bool metropolis64(W64& w, double old_f, double new_f, double temperature) {
    if (new_f < old_f) return true;
    const double p = fd_exp((old_f - new_f) / temperature);
    return rand_fl(w, 0, 1) < p;
}

// add_to_output_container with the container in global memory (slots + sorted order)
__device__ void add_to_output64(W64& w, const Chain64& ch, const double* x, double e, double min_rmsd, int max_size) {
    const DModel& m = *w.m;
    const int H = m.nheavy, cs = m.conf_size;
    int count = *ch.out_count;
    double* rm = w.s + w.L.rmsd;
    for (int j = w.lane; j < count; j += 32) {
        const double* oc = ch.out_coords + (size_t)ch.out_order[j] * H * 3;
        double acc = 0;
        for (int a = 0; a < H; a++) acc += dist2(ld3(w.s + w.L.coords + 3 * m.heavy[a]), ld3(oc + 3 * a));
        rm[j] = H > 0 ? sqrt(acc / H) : 0;
    }
    __syncwarp();
    int target = -1;  // slot to overwrite / fill
    if (w.lane == 0) {
        int bj = count;
        double best = kMaxFl;
        for (int j = 0; j < count; j++)
            if (j == 0 || rm[j] < best) { bj = j; best = rm[j]; }
        if (bj < count && best < min_rmsd) {
            if (e < ch.out_e[ch.out_order[bj]]) target = ch.out_order[bj];
        } else if (count < max_size) {
            target = count;
            ch.out_order[count] = count;
            count++;
        } else if (count > 0 && e < ch.out_e[ch.out_order[count - 1]]) {
            target = ch.out_order[count - 1];
        }
    }
    target = __shfl_sync(kFull, target, 0);
    count = __shfl_sync(kFull, count, 0);
    if (target >= 0) {
        for (int i = w.lane; i < cs; i += 32) ch.out_conf[(size_t)target * cs + i] = x[i];
        for (int a = w.lane; a < H; a += 32) st3(ch.out_coords + ((size_t)target * H + a) * 3, ld3(w.s + w.L.coords + 3 * m.heavy[a]));
        if (w.lane == 0) ch.out_e[target] = e;
    }
    __syncwarp();
    if (w.lane == 0) {
        *ch.out_count = count;
        for (int i = 1; i < count; i++) {  // stable insertion sort by energy
            const int key = ch.out_order[i];
            const double ek = ch.out_e[key];
            int j = i - 1;
            while (j >= 0 && ch.out_e[ch.out_order[j]] > ek) { ch.out_order[j + 1] = ch.out_order[j]; j--; }
            ch.out_order[j + 1] = key;
        }
    }
    __syncwarp();
}

}  // namespace sg
