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
// Follows the reference's restatement of QuickVina 2 (gpu_mc.cuh:144-264;
// Alhossary et al., Bioinformatics 2015): each chain keeps the last 5n points
// its local optimisations visited.  A local optimisation runs only if one of
// the 4n history points nearest its start passes the first-order consistency
// check; until the history is full every start passes.
__device__ inline Vis64 vis64_view(double* d, uint32_t* u, int n) {
    Vis64 v;
    v.x = d;
    v.f = v.x + (size_t)5 * n * n;
    v.now = v.f + 5 * n;
    v.dist = v.now + n;
    v.bits = u;
    v.state = reinterpret_cast<int*>(u + 20 * n);
    return v;
}
__device__ inline bool vis_bit(const uint32_t* b, int i) { return ((i < 32 ? b[0] >> i : b[1] >> (i - 32)) & 1u) != 0; }

// visited::add (gpu_mc.cuh:163-205)
__device__ void vis64_add(W64& w, const Vis64& V, const double* x, double f, const double* g) {
    const DModel& m = *w.m;
    const int n = m.dof, cap = 5 * n;
    int slot = 0;
    if (w.lane == 0) {
        int* st = V.state;  // size, next slot, full
        if (!st[2]) {
            slot = st[0]++;
            if (st[0] >= cap) { st[2] = 1; st[1] = 0; }
        } else {
            slot = st[1];
            st[1] = (st[1] + 1) % cap;
        }
        V.f[slot] = f;
        uint32_t zero[2] = {0, 0}, pos[2] = {0, 0};
        for (int i = 0; i < n; i++)
            if (g[i] == 0) zero[i >> 5] |= 1u << (i & 31);
            else if (g[i] > 0) pos[i >> 5] |= 1u << (i & 31);
        uint32_t* b = V.bits + 4 * slot;
        b[0] = zero[0]; b[1] = zero[1]; b[2] = pos[0]; b[3] = pos[1];
    }
    slot = __shfl_sync(kFull, slot, 0);
    for (int i = w.lane; i < n; i += 32) V.x[(size_t)slot * n + i] = conf_value64(m, x, i);
    __syncwarp();
}

// visited::interesting (gpu_mc.cuh:207-264): the nearest history point that
// passes the check (lowest index on ties) must rank below 4n by distance
__device__ bool vis64_interesting(W64& w, const Vis64& V, const double* x, double f, const double* g) {
    const DModel& m = *w.m;
    const int n = m.dof, cap = 5 * n;
    const int full = __shfl_sync(kFull, w.lane == 0 ? V.state[2] : 0, 0);
    if (!full) return true;
    for (int i = w.lane; i < n; i += 32) V.now[i] = conf_value64(m, x, i);
    __syncwarp();
    double best = kMaxFl;
    int besti = cap;
    for (int e = w.lane; e < cap; e += 32) {
        const double* xe = V.x + (size_t)e * n;
        const uint32_t* b = V.bits + 4 * e;
        const bool newY = f - V.f[e] > 0;
        double d2 = 0;
        bool pass = true;
        for (int i = 0; i < n; i++) {
            const double dx = xe[i] - V.now[i];
            d2 += dx * dx;
            if (vis_bit(b, i) || g[i] == 0) continue;
            const bool nowPos = g[i] > 0;
            if (nowPos != vis_bit(b + 2, i)) continue;
            const bool newX = V.now[i] - xe[i] > 0;
            if (nowPos ^ newX ^ newY) pass = false;
        }
        V.dist[e] = d2;
        if (pass && d2 < best) { best = d2; besti = e; }
    }
    for (int o = 16; o > 0; o >>= 1) {  // argmin of (best, index)
        const double ob = __shfl_xor_sync(kFull, best, o);
        const int oi = __shfl_xor_sync(kFull, besti, o);
        if (ob < best || (ob == best && oi < besti)) { best = ob; besti = oi; }
    }
    if (besti >= cap) return false;
    __syncwarp();
    int ahead = 0;
    for (int e = w.lane; e < cap; e += 32) ahead += (V.dist[e] < best || (V.dist[e] == best && e < besti));
    for (int o = 16; o > 0; o >>= 1) ahead += __shfl_xor_sync(kFull, ahead, o);
    return ahead < 4 * n;
}

__device__ double bfgs64(W64& w, double* x, int maxiters, int accurate, int early, const EvalMode& em,
                         const Vis64* vis = nullptr) {
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
        if (!vis64_interesting(w, *vis, x, f0, g)) return f0;
        vis64_add(w, *vis, x, f0, g);
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
        if (vis) vis64_add(w, *vis, x, f0, g);
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
