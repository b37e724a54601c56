// Mixed-precision path, part 2: the batched Monte Carlo search.
//
// A persistent kernel: every warp takes chains from a global queue (ordered
// longest first on the host) until the queue is empty, so ligands of very
// different sizes and step counts share the GPU without a tail.  One warp
// (or a team of 2 or 4, whose other warps take shares of every evaluation)
// runs one chain: mutate, BFGS on the hunt-capped energy, Metropolis test,
// BFGS on the authentic energy for accepted poses, and the chain's output
// container in global memory.  Confs, the inverse Hessian, the Armijo test
// and the orientation increment stay in FP64; energies and gradients come
// from the FP32 evaluation.  Random numbers: Philox4x32-10 keyed by the
// request seed, counter (draw, ligand key, chain) -- independent of the
// batch composition and of the launch shape (for a given team size).
// Reference semantics: monte_carlo.cpp:95-130; mutate.cpp:35-63;
// bfgs.h:30-282; conf.h:98-404; coords.cpp:25-58 (add_to_output_container).
#include "dock32_eval.cuh"

namespace sg {

__device__ __forceinline__ double warp_sum_d(double v) {
    // butterfly: every lane ends with the same bits (each step adds the
    // same two operands on both partners)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull32, v, o);
    return v;
}
// three butterfly sums at once (one latency chain)
__device__ __forceinline__ void warp_sum3_d(double& a, double& b, double& c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(kFull32, a, o);
        b += __shfl_xor_sync(kFull32, b, o);
        c += __shfl_xor_sync(kFull32, c, o);
    }
}
__device__ __forceinline__ double dotd(const W32& w, const double* a, const double* b, int n) {
    double t = 0;
    for (int i = w.lane; i < n; i += 32) t += a[i] * b[i];
    return warp_sum_d(t);
}
__device__ __forceinline__ void copyd(const W32& w, double* d, const double* s, int n) {
    for (int i = w.lane; i < n; i += 32) d[i] = s[i];
    __syncwarp();
}

// normalize_angle for the mixed-precision path: the nearest multiple of
// 2 pi is subtracted in one step (same interval as common.h's loop, not
// its rounding)
__device__ __forceinline__ double wrap_pi(double x) {
    return x - (2 * kPi) * rint(x * (1.0 / (2 * kPi)));
}

// quaternion_increment (quaternion.cpp:118-126) with an FP32 sine/cosine of
// the half angle, composed and re-normalised in FP64
__device__ __forceinline__ void q_increment32(double* c, double rx, double ry, double rz) {
    const double a2 = rx * rx + ry * ry + rz * rz;
    double s = 0, co = 1;
    if (a2 > kEps * kEps) {  // angle > epsilon
        const double inv = rsqrt(a2);
        float sf, cf;
        __sincosf((float)(0.5 * wrap_pi(a2 * inv)), &sf, &cf);
        s = (double)sf * inv;
        co = (double)cf;
    }
    Quat<double> q{c[0], c[1], c[2], c[3]};
    q = qmul(Quat<double>{co, s * rx, s * ry, s * rz}, q);
    const double n2 = q.a * q.a + q.b * q.b + q.c * q.c + q.d * q.d;
    if (fabs(n2 - 1) >= 1e-6) {  // quaternion_normalize_approx
        const double inv = rsqrt(n2);
        q.a *= inv; q.b *= inv; q.c *= inv; q.d *= inv;
    }
    c[0] = q.a; c[1] = q.b; c[2] = q.c; c[3] = q.d;
}

// conf::increment
__device__ __forceinline__ void increment32(const W32& w, double* x, const double* p, double alpha) {
    const SModel& m = smodel();
    const int* lig_root = sp<const int>(m.lig_root);
    const int* fconf = sp<const int>(m.fconf);
    const int* fdof = sp<const int>(m.fdof);
    const int* tor_conf = sp<const int>(m.tor_conf);
    const int* tor_dof = sp<const int>(m.tor_dof);
    for (int l = w.lane; l < m.nlig; l += 32) {
        const int f = lig_root[l];
        double* c = x + fconf[f];
        const double* d = p + fdof[f];
        c[0] += alpha * d[0]; c[1] += alpha * d[1]; c[2] += alpha * d[2];
        q_increment32(c + 3, alpha * d[3], alpha * d[4], alpha * d[5]);
    }
    for (int k = w.lane; k < m.ntors; k += 32) {
        double& t = x[tor_conf[k]];
        t = wrap_pi(t + wrap_pi(alpha * p[tor_dof[k]]));
    }
    __syncwarp();
}

// conf::operator()(index): value of change coordinate i (accurate line search)
__device__ double conf_value32(const double* x, int i) {
    const SModel& m = smodel();
    const int* lig_root = sp<const int>(m.lig_root);
    const int* fconf = sp<const int>(m.fconf);
    const int* fdof = sp<const int>(m.fdof);
    const int* tor_conf = sp<const int>(m.tor_conf);
    const int* tor_dof = sp<const int>(m.tor_dof);
    for (int l = 0; l < m.nlig; l++) {
        const int f = lig_root[l];
        const int d0 = fdof[f];
        if (i >= d0 && i < d0 + 3) return x[fconf[f] + (i - d0)];
        if (i >= d0 + 3 && i < d0 + 6) {
            const double* c = x + fconf[f];
            const V3<double> a = q_to_angle(Quat<double>{c[3], c[4], c[5], c[6]});
            const int j = i - d0 - 3;
            return j == 0 ? a.x : j == 1 ? a.y : a.z;
        }
    }
    for (int k = 0; k < m.ntors; k++)
        if (tor_dof[k] == i) return x[tor_conf[k]];
    return 0;
}

struct Mode32 {
    float3 v;
    float slope;
};

// energy and gradient of the conf at smem32 offset x_at (gradient to g_at),
// on the chain's team of G warps
template <int G>
__device__ __forceinline__ double feval32(int x_at, int g_at, const Mode32& em) {
    return (double)eval_deriv32<G>(x_at, em.v, em.slope, g_at);
}

// ---- line searches (bfgs.h:30-200) ------------------------------------------------------
// x, g, p, x_new, g_new: offsets of this warp's workspace arrays in smem32
// pg: p . g, computed by the caller with p
template <int G>
__device__ __forceinline__ double line_fast32(const W32& w, int x_at, double pg, double f0, int p_at, int xn_at,
                                              int gn_at, double& f1, const Mode32& em) {
    const SModel& m = smodel();
    const double* x = sp<const double>(x_at);
    const double* p = sp<const double>(p_at);
    double* x_new = sp<double>(xn_at);
    double alpha = 1;
    for (unsigned trial = 0; trial < 10; trial++) {
        SG_T0(t_ls);
        copyd(w, x_new, x, m.conf_size);
        increment32(w, x_new, p, alpha);
        SG_T1(t_ls, 4);
        f1 = feval32<G>(xn_at, gn_at, em);
        if (f1 - f0 < 0.0001 * alpha * pg) break;
        alpha *= 0.5;
    }
    return alpha;
}

// Out of line; arguments by value and (alpha, f1) returned by value, so that
// no variable of the caller has its address taken.
template <int G>
__device__ __noinline__ double2 line_accurate32(W32 w, int x_at, double pg, double f0, int p_at, int xn_at, int gn_at,
                                                 Mode32 em) {
    const SModel& m = smodel();
    const int n = m.dof;
    const double* x = sp<const double>(x_at);
    const double* p = sp<const double>(p_at);
    double* x_new = sp<double>(xn_at);
    double* g_new = sp<double>(gn_at);
    double a, alpha, alpha2 = 0, alamin, b, disc, f1 = 0, f2 = 0, rhs1, rhs2, tmplam = 0;
    const double ALF = 1.0e-4, FIRST = 1.0;
    const double slope = pg;
    auto give_up = [&]() {
        copyd(w, x_new, x, m.conf_size);
        for (int i = w.lane; i < n; i += 32) g_new[i] = 0;
        __syncwarp();
        return make_double2(0.0, f1);
    };
    if (slope >= 0) return give_up();
    double test = 0;
    for (int i = w.lane; i < n; i += 32) test = fmax(test, fabs(p[i]) / fmax(fabs(conf_value32(x, i)), 1.0));
    for (int o = 16; o > 0; o >>= 1) test = fmax(test, __shfl_xor_sync(kFull32, test, o));
    alamin = kEps / test;
    alpha = FIRST;
    // alpha at least halves every round, so 128 rounds reach any alamin > 0
    for (int it = 0; it < 128; it++) {
        copyd(w, x_new, x, m.conf_size);
        increment32(w, x_new, p, alpha);
        f1 = feval32<G>(xn_at, gn_at, em);
        if (alpha < alamin) return give_up();
        if (f1 <= f0 + ALF * alpha * slope) return make_double2(alpha, f1);
        if (alpha == FIRST) {
            tmplam = -slope / (2.0 * (f1 - f0 - slope));
        } else {
            rhs1 = f1 - f0 - alpha * slope;
            rhs2 = f2 - f0 - alpha2 * slope;
            a = (rhs1 / (alpha * alpha) - rhs2 / (alpha2 * alpha2)) / (alpha - alpha2);
            b = (-alpha2 * rhs1 / (alpha * alpha) + alpha * rhs2 / (alpha2 * alpha2)) / (alpha - alpha2);
            if (a == 0.0) {
                tmplam = -slope / (2.0 * b);
            } else {
                disc = b * b - 3.0 * a * slope;
                if (disc < 0) tmplam = 0.5 * alpha;
                else if (b <= 0) tmplam = (-b + sqrt(disc)) / (3.0 * a);
                else tmplam = -slope / (b + sqrt(disc));
            }
            if (tmplam > .5 * alpha) tmplam = .5 * alpha;
        }
        alpha2 = alpha;
        f2 = f1;
        alpha = fmax(tmplam, 0.1 * alpha);
    }
    return give_up();
}

// ---- BFGS (bfgs.h:202-282) on a full symmetric n x n inverse Hessian ------------------------
// Lane i owns row i, stored as column i of h (h[j * n + i]) so the lanes of
// a row sweep read consecutive words.  Every entry (i, j) is computed from
// (min(i, j), max(i, j)) operands in one fixed order, so h stays exactly
// symmetric.  x_at: smem32 offset of the conf, optimised in place.
template <int G>
__device__ __noinline__ double bfgs32(int x_at, int maxiters, int accurate, int early, Mode32 em) {
    const W32 w = here();
    const SModel& m = smodel();
    const Ws32& L = m.L;
    const int n = m.dof, cs = m.conf_size;
    const int g_at = w.at(L.g), gn_at = w.at(L.g_new), p_at = w.at(L.p), xn_at = w.at(L.x_new);
    double* x = sp<double>(x_at);
    double* h = w.d(L.h);
    double *g = sp<double>(g_at), *g_new = sp<double>(gn_at), *g_orig = w.d(L.g_orig), *p = sp<double>(p_at);
    double *y = w.d(L.y), *x_new = sp<double>(xn_at), *x_orig = w.d(L.x_orig), *mhy = w.d(L.mhy);
    for (int i = w.lane; i < n; i += 32)
        for (int j = 0; j < n; j++) h[j * n + i] = (i == j) ? 1.0 : 0.0;
    __syncwarp();
    double f0 = feval32<G>(x_at, g_at, em);
    const double f_orig = f0;
    copyd(w, g_orig, g, n);
    copyd(w, x_orig, x, cs);
    for (int step = 0; step < maxiters; step++) {
        SG_T0(t_alg);
        double pg = 0;  // p . g, for the line search
        for (int i = w.lane; i < n; i += 32) {
            double sum = 0;
            SG_ROLLED
            for (int j = 0; j < n; j++) sum += h[j * n + i] * g[j];
            p[i] = -sum;
            pg += -sum * g[i];
        }
        pg = warp_sum_d(pg);
        __syncwarp();
        SG_T1(t_alg, 5);
        double f1 = 0, alpha;
        if (accurate) {
            const double2 r = line_accurate32<G>(w, x_at, pg, f0, p_at, xn_at, gn_at, em);
            alpha = r.x;
            f1 = r.y;
        } else {
            alpha = line_fast32<G>(w, x_at, pg, f0, p_at, xn_at, gn_at, f1, em);
        }
        if (alpha == 0) break;
        SG_T0(t_alg2);
        // y = g_new - g, g = g_new, and the three dot products the update needs
        double gg = 0, yy = 0, yp = 0;
        for (int i = w.lane; i < n; i += 32) {
            const double gi = g_new[i], yi = gi - g[i];
            y[i] = yi;
            g[i] = gi;
            gg += gi * gi;
            yy += yi * yi;
            yp += yi * p[i];
        }
        warp_sum3_d(gg, yy, yp);
        __syncwarp();
        const double prevf0 = f0;
        f0 = f1;
        copyd(w, x, x_new, cs);
        if (early && fabs(prevf0 - f0) < 1e-5) break;
        if (!(gg >= 1e-4)) break;
        if (step == 0 && fabs(yy) > kEps) {
            const double dg = alpha * yp / yy;
            for (int i = w.lane; i < n; i += 32) h[i * n + i] = dg;
            __syncwarp();
        }
        // bfgs_update
        if (alpha * yp >= kEps) {
            double yhy = 0;
            for (int i = w.lane; i < n; i += 32) {
                double sum = 0;
                SG_ROLLED
                for (int j = 0; j < n; j++) sum += h[j * n + i] * y[j];
                mhy[i] = -sum;
                yhy += y[i] * -sum;
            }
            yhy = -warp_sum_d(yhy);
            __syncwarp();
            const double r = 1 / (alpha * yp);
            const double c1 = alpha * r, c2 = alpha * alpha * (r * r * yhy + r);
            for (int i = w.lane; i < n; i += 32) {
                const double mi = mhy[i], pi = p[i];
                SG_ROLLED
                for (int j = 0; j < n; j++) {
                    // operands ordered (lower index, higher index) so h stays symmetric
                    const double mj = mhy[j], pj = p[j];
                    const bool own_lo = i <= j;
                    const double ml = own_lo ? mi : mj, mh = own_lo ? mj : mi;
                    const double pl = own_lo ? pi : pj, ph = own_lo ? pj : pi;
                    h[j * n + i] += c1 * (ml * ph + mh * pl) + c2 * pl * ph;
                }
            }
            __syncwarp();
        }
        SG_T1(t_alg2, 5);
    }
    if (!(f0 <= f_orig)) {
        f0 = f_orig;
        copyd(w, x, x_orig, cs);
        copyd(w, g, g_orig, n);
    }
    return f0;
}

// ---- Monte Carlo pieces -------------------------------------------------------------------
__device__ __forceinline__ V3<double> sphere32(Philox& rng) {  // random_inside_sphere, bounded rejection
    for (int k = 0; k < 64; k++) {
        const double a = ph_range(rng, -1, 1), b = ph_range(rng, -1, 1), c = ph_range(rng, -1, 1);
        if (a * a + b * b + c * c < 1) return V3<double>{a, b, c};
    }
    return V3<double>{0, 0, 0};
}

// gyration radius of ligand l's heavy atoms about its root origin (current coords)
__device__ __forceinline__ double gyration32(const W32& w, int l) {
    const SModel& m = smodel();
    const int* type = sp<const int>(m.type);
    const float3 o = f3(w.origin()[sp<const int>(m.lig_root)[l]]);
    float acc = 0;
    int cnt = 0;
    const int end = sp<const int>(m.lig_end)[l];
    for (int i = sp<const int>(m.lig_begin)[l] + w.lane; i < end; i += 32)
        if (!is_h(type[i])) {
            const float3 d = f3(w.coords()[i]) - o;
            acc += dot3(d, d);
            cnt++;
        }
    acc = warp_sum(acc);
    for (int s = 16; s > 0; s >>= 1) cnt += __shfl_xor_sync(kFull32, cnt, s);
    return cnt > 0 ? sqrt((double)acc / cnt) : 0.0;
}

__device__ __forceinline__ void mutate32(const W32& w, Philox& rng, double* x, double amplitude) {
    const SModel& m = smodel();
    const int* blk_rigid = sp<const int>(m.blk_rigid);
    const int* blk_ntors = sp<const int>(m.blk_ntors);
    const int* blk_conf = sp<const int>(m.blk_conf);
    int num = 0;
    for (int b = 0; b < m.nblocks; b++) num += (blk_rigid[b] ? 2 : 0) + blk_ntors[b];
    if (num == 0) return;
    int which = ph_int(rng, num);
    int lig = 0;
    for (int b = 0; b < m.nblocks; b++) {
        double* c = x + blk_conf[b];
        if (blk_rigid[b]) {
            if (which == 0) {
                const V3<double> d = amplitude * sphere32(rng);
                if (w.lane == 0) { c[0] += d.x; c[1] += d.y; c[2] += d.z; }
                __syncwarp();
                return;
            }
            --which;
            if (which == 0) {
                const double gr = gyration32(w, lig);
                if (gr > kEps) {
                    const V3<double> rot = (amplitude / gr) * sphere32(rng);
                    if (w.lane == 0) q_increment32(c + 3, rot.x, rot.y, rot.z);
                    __syncwarp();
                }
                return;
            }
            --which;
            c += 7;
            lig++;
        }
        const int nt = blk_ntors[b];
        if (which < nt) {
            const double t = ph_range(rng, -kPi, kPi);
            if (w.lane == 0) c[which] = t;
            __syncwarp();
            return;
        }
        which -= nt;
    }
}

// conf::randomize: position uniform in the box, orientation from four
// normal deviates, torsions uniform in [-pi, pi)
// box: 6 doubles (lo xyz, hi xyz) of the search box
__device__ __forceinline__ void randomize32(const W32& w, Philox& rng, double* x, const double* box) {
    const SModel& m = smodel();
    const int* blk_rigid = sp<const int>(m.blk_rigid);
    const int* blk_ntors = sp<const int>(m.blk_ntors);
    const int* blk_conf = sp<const int>(m.blk_conf);
    for (int b = 0; b < m.nblocks; b++) {
        double* c = x + blk_conf[b];
        if (blk_rigid[b]) {
            double v[7];
            for (int k = 0; k < 3; k++) v[k] = ph_range(rng, __ldcg(box + k), __ldcg(box + 3 + k));
            double q[4], nq = 0;
            for (int k = 0; k < 4; k++) { q[k] = ph_normal(rng); nq += q[k] * q[k]; }
            nq = sqrt(nq);
            if (nq > kEps) for (int k = 0; k < 4; k++) v[3 + k] = q[k] / nq;
            else { v[3] = 1; v[4] = v[5] = v[6] = 0; }
            if (w.lane == 0) for (int k = 0; k < 7; k++) c[k] = v[k];
            c += 7;
        }
        const int nt = blk_ntors[b];
        for (int t = 0; t < nt; t++) {
            const double a = ph_range(rng, -kPi, kPi);
            if (w.lane == 0) c[t] = a;
        }
    }
    __syncwarp();
}

// add_to_output_container with the chain's container in global memory;
// returns the new size
__device__ __forceinline__ int add_output32(const W32& w, const Chain32& ch, const double* x, double e,
                                            double min_rmsd, int max_size, int count) {
    const SModel& m = smodel();
    const int H = m.nheavy, cs = m.conf_size;
    const int* heavy = sp<const int>(m.heavy);
    const float4* X = w.coords();
    // RMSD to every saved pose: lanes over atoms, one pose at a time
    float best = 3.4e38f;
    int bj = count;
    for (int j = 0; j < count; j++) {
        const float* oc = ch.out_coords + (size_t)ch.out_order[j] * H * 3;
        float acc = 0;
        for (int a = w.lane; a < H; a += 32) {
            const float3 c = f3(X[heavy[a]]);
            const float dx = c.x - oc[3 * a], dy = c.y - oc[3 * a + 1], dz = c.z - oc[3 * a + 2];
            acc += dx * dx + dy * dy + dz * dz;
        }
        acc = warp_sum(acc);
        const float r = H > 0 ? sqrtf(acc / H) : 0.f;
        if (j == 0 || r < best) { bj = j; best = r; }
    }
    int target = -1;
    if (bj < count && best < min_rmsd) {
        if (e < ch.out_e[ch.out_order[bj]]) target = ch.out_order[bj];
    } else if (count < max_size) {
        target = count;
        if (w.lane == 0) ch.out_order[count] = count;
        count++;
    } else if (count > 0 && e < ch.out_e[ch.out_order[count - 1]]) {
        target = ch.out_order[count - 1];
    }
    __syncwarp();
    if (target >= 0) {
        for (int i = w.lane; i < cs; i += 32) ch.out_conf[(size_t)target * cs + i] = x[i];
        for (int a = w.lane; a < H; a += 32) {
            const float3 c = f3(X[heavy[a]]);
            float* o = ch.out_coords + ((size_t)target * H + a) * 3;
            o[0] = c.x; o[1] = c.y; o[2] = c.z;
        }
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
    return count;
}

// monte_carlo::operator() for one chain, run by the leader of its team of G
// warps
template <int G>
__device__ __noinline__ void run_chain32(const Chain32& ch, const MCParams32& P) {
    SG_T0(t_chain);
    const W32 w = here();
    if (ch.span && w.lane == 0) ch.span[0] = global_ns();
    const SModel& m = smodel();
    const Ws32& L = m.L;
    unsigned* C = w.counters();
    for (int i = w.lane; i < 65; i += 32) C[i] = 0;
    const int cs = m.conf_size;
    // model state as read (mutation may read it before the first set)
    const unsigned first = ch.begin, last = ch.end ? ch.end : ch.steps;
    const bool resumed = ch.resume && first > 0;
    const int tmp_at = w.at(L.x_tmp), cand_at = w.at(L.x_cand);
    double* tmp = sp<double>(tmp_at);
    double* cand = sp<double>(cand_at);
    Philox rng{ch.key0, ch.key1, ch.lig, ch.chain, 0u};
    double tmp_e = 0, best_e = kMaxFl;
    int count = 0;
    const float4* saved_xyz = ch.resume ? reinterpret_cast<const float4*>(ch.resume + resume32_coords_at(cs)) : nullptr;
    if (resumed) {  // a later phase: the state the previous one saved
        for (int i = w.lane; i < cs; i += 32) tmp[i] = ch.resume[i];
        for (int i = w.lane; i < m.natoms; i += 32) w.coords()[i] = saved_xyz[i];
        for (int f = w.lane; f < m.nframes; f += 32) w.origin()[f] = saved_xyz[m.natoms + f];
        tmp_e = ch.resume[cs];
        best_e = ch.resume[cs + 1];
        rng.n = (uint32_t)ch.resume[cs + 2];
        count = *ch.out_count;
        __syncwarp();
    } else {
        // (L2-only loads: a serving grid may read a ligand placed where an
        // earlier one was, and this SM's L1 may still hold the earlier one's lines)
        for (int i = w.lane; i < m.natoms; i += 32) w.coords()[i] = __ldcg(m.lab32 + i);
        for (int f = w.lane; f < m.nframes; f += 32) w.origin()[f] = __ldcg(m.finit32 + f);
        __syncwarp();
        randomize32(w, rng, tmp, ch.box ? ch.box : P.box);
        if (w.lane == 0) *ch.out_count = 0;
    }
    const Mode32 hunt{make_float3(P.hunt[0], P.hunt[1], P.hunt[2]), P.slope};
    const Mode32 auth{make_float3(P.auth[0], P.auth[1], P.auth[2]), P.slope};
    for (unsigned step = first; step < last; step++) {
        SG_T0(t_mut);
        copyd(w, cand, tmp, cs);
        mutate32(w, rng, cand, P.amplitude);
        SG_T1(t_mut, 6);
        const double cand_e = bfgs32<G>(cand_at, ch.maxiters, P.accurate_line, P.early_term, hunt);
        bool accept = step == 0 || cand_e < tmp_e;
        if (!accept) accept = ph_u01(rng) < exp((tmp_e - cand_e) / P.temperature);
        if (accept) {
            copyd(w, tmp, cand, cs);
            tmp_e = cand_e;
            set_conf32(tmp_at);
            if (tmp_e < best_e || count < P.num_saved) {
                tmp_e = bfgs32<G>(tmp_at, ch.maxiters, P.accurate_line, P.early_term, auth);
                set_conf32(tmp_at);
                count = add_output32(w, ch, tmp, tmp_e, P.min_rmsd, P.num_saved, count);
                if (tmp_e < best_e) best_e = tmp_e;
            }
        }
    }
    __syncwarp();
    if (ch.resume) {  // the state a later phase resumes from (and the best energy, for the stopping rule)
        float4* sx = reinterpret_cast<float4*>(ch.resume + resume32_coords_at(cs));
        for (int i = w.lane; i < cs; i += 32) ch.resume[i] = tmp[i];
        for (int i = w.lane; i < m.natoms; i += 32) sx[i] = w.coords()[i];
        for (int f = w.lane; f < m.nframes; f += 32) sx[m.natoms + f] = w.origin()[f];
        if (w.lane == 0) {
            ch.resume[cs] = tmp_e;
            ch.resume[cs + 1] = best_e;
            ch.resume[cs + 2] = (double)rng.n;
        }
    }
    unsigned long long gh = C[w.lane], ph = C[32 + w.lane];
    for (int o = 16; o > 0; o >>= 1) {
        gh += __shfl_xor_sync(kFull32, gh, o);
        ph += __shfl_xor_sync(kFull32, ph, o);
    }
    if (w.lane == 0) {
        *ch.evals = (resumed ? *ch.evals : 0ull) + C[64];
        ch.hits[0] = (resumed ? ch.hits[0] : 0ull) + gh;
        ch.hits[1] = (resumed ? ch.hits[1] : 0ull) + ph;
        if (ch.span) ch.span[1] = global_ns();
        if (ch.done_count) {
            __threadfence();  // this chain's results, before its count
            if (atomicAdd(ch.done_count, 1u) + 1 == (unsigned)ch.lig_chains) {
                __threadfence_system();
                *reinterpret_cast<volatile unsigned*>(ch.host_flag) = 1u;
                __threadfence_system();
            }
        }
    }
    __syncwarp();
    SG_T1(t_chain, 7);
}

// Copies a model's counts and the arrays the search reads into smem32 at
// offset 0 (an SModel, then the arrays); every thread of the block takes
// part.  Ends with a block barrier.
// Loads go through L2 only (ld.global.cg): a serving grid stages ligands
// that the host placed, while it runs, where earlier ones were.
template <typename T>
__device__ __forceinline__ int stage_arr(const T* src, int n, int& o, int tid, int nthr) {
    const int at = o;
    T* d = sp<T>(at);
    o += (n * (int)sizeof(T) + 15) & ~15;
    for (int i = tid; i < n; i += nthr) d[i] = __ldcg(src + i);
    return at;
}

__shared__ __align__(16) DModel s_dmodel;  // the staged model's descriptor (its pointers)

__device__ void stage_model(const DModel* gm, int tid, int nthr) {
    static_assert(sizeof(DModel) % 16 == 0, "DModel is read in 16-byte pieces");
    for (int k = tid; k < (int)(sizeof(DModel) / 16); k += nthr)
        reinterpret_cast<int4*>(&s_dmodel)[k] = __ldcg(reinterpret_cast<const int4*>(gm) + k);
    __syncthreads();
    const DModel& g = s_dmodel;
    int o = ((int)sizeof(SModel) + 15) & ~15;
    SModel s;
    s.natoms = g.natoms; s.nmov = g.nmov; s.nframes = g.nframes; s.nlig = g.nlig; s.conf_size = g.conf_size;
    s.dof = g.dof; s.nheavy = g.nheavy; s.nlevels = g.nlevels; s.nblocks = g.nblocks; s.ntors = g.ntors;
    s.npchunks = g.npchunks;
    s.local32 = stage_arr(g.local32, g.natoms, o, tid, nthr);
    s.type = stage_arr(g.type, g.natoms, o, tid, nthr);
    s.atom_frame = stage_arr(g.atom_frame, g.natoms, o, tid, nthr);
    s.forigin32 = stage_arr(g.forigin32, g.nframes, o, tid, nthr);
    s.faxis32 = stage_arr(g.faxis32, g.nframes, o, tid, nthr);
    s.fkind = stage_arr(g.fkind, g.nframes, o, tid, nthr);
    s.fparent = stage_arr(g.fparent, g.nframes, o, tid, nthr);
    s.fbegin = stage_arr(g.fbegin, g.nframes, o, tid, nthr);
    s.fsub_end = stage_arr(g.fsub_end, g.nframes, o, tid, nthr);
    s.fconf = stage_arr(g.fconf, g.nframes, o, tid, nthr);
    s.fdof = stage_arr(g.fdof, g.nframes, o, tid, nthr);
    s.heavy = stage_arr(g.heavy, g.nheavy, o, tid, nthr);
    s.pslot = stage_arr(g.pslot, 32 * g.npchunks, o, tid, nthr);
    s.lig_root = stage_arr(g.lig_root, g.nlig, o, tid, nthr);
    s.lig_begin = stage_arr(g.lig_begin, g.nlig, o, tid, nthr);
    s.lig_end = stage_arr(g.lig_end, g.nlig, o, tid, nthr);
    s.blk_rigid = stage_arr(g.blk_rigid, g.nblocks, o, tid, nthr);
    s.blk_conf = stage_arr(g.blk_conf, g.nblocks, o, tid, nthr);
    s.blk_ntors = stage_arr(g.blk_ntors, g.nblocks, o, tid, nthr);
    s.tor_conf = stage_arr(g.tor_conf, g.ntors, o, tid, nthr);
    s.tor_dof = stage_arr(g.tor_dof, g.ntors, o, tid, nthr);
    s.lab32 = g.lab32;
    s.finit32 = g.finit32;
    s.level_start = g.level_start;
    s.level_frames = g.level_frames;
    s.L = ws32_layout(g.natoms, g.nframes, g.conf_size, g.dof);
    if (tid == 0) *sp<SModel>(0) = s;
    __syncthreads();
}

// A chain on its team of G warps: the leader runs it and then releases the
// helpers, which serve its evaluations until then.
template <int G>
__device__ __forceinline__ void run_team32(const Chain32& ch, const MCParams32& P) {
    if constexpr (G == 1) {
        run_chain32<1>(ch, P);
    } else {
        if ((threadIdx.x >> 5) % G == 0) {
            run_chain32<G>(ch, P);
            team_publish<G>(here(), make_float3(0, 0, 0), 0.f, kTeamExit);
        } else {
            team_help32<G>();
        }
    }
}

// Persistent search kernel.  A block takes work items (a group of chains
// of one ligand, longest first) from *queue, stages the ligand's model in
// shared memory once for all its warps, and runs one chain per team of G
// warps (every warp has a workspace; a helper's holds its force share).
// SG_MC32_MINB resident 256-thread blocks per SM bound the registers
// (2: 128 per thread).
#ifndef SG_MC32_MINB
#define SG_MC32_MINB 2
#endif
#ifndef SG_MC32_THREADS
#define SG_MC32_THREADS 256
#endif
// maps_tab: one DMaps32 per receptor (items name theirs), or null when the
// whole launch uses G.
template <int TEAM>
__global__ void __launch_bounds__(SG_MC32_THREADS, SG_MC32_MINB) k_mc32(const DModel* models, DTables32 T, DMaps32 G,
                                                            const DMaps32* maps_tab, const Chain32* chains,
                                                            const Item32* items, int nitems,
                                                            const __grid_constant__ MCParams32 P, unsigned* queue,
                                                            int stage_stride, int ws_stride) {
    __shared__ int s_item;
    const int tid = threadIdx.x, nthr = blockDim.x, warp = tid >> 5;
    if (tid == 0) { sT32 = T; sG32 = G; sWs0 = stage_stride; sWsStride = ws_stride; }
    for (;;) {
        if (tid == 0) s_item = (int)atomicAdd(queue, 1u);
        __syncthreads();
        const int it = s_item;
        if (it >= nitems) break;
        const Item32 item = items[it];
        if (maps_tab && tid == 0) sG32 = maps_tab[item.rec];  // read after stage_model's barrier
        stage_model(models + item.model, tid, nthr);
        if (warp / TEAM < item.count) run_team32<TEAM>(chains[item.first + warp / TEAM], P);
        SG_T0(t_bar);
        __syncthreads();  // the staged model is in use until every warp is done
        SG_T1(t_bar, 8);
    }
}

// ---- serving grid ----------------------------------------------------------------------------
// Claims the next item of the ring for this block (thread 0): the item's
// sequence number, or -1 once no item has come for idle_ns nanoseconds or
// the host has set stop.  Every wait is bounded: a block that finds no work
// sleeps in short steps and leaves after idle_ns.
__device__ long long feed_claim(FeedCtrl32* c, long long idle_ns) {
    volatile unsigned* vc = reinterpret_cast<volatile unsigned*>(c);
    long long t0 = 0;
    bool waiting = false;
    long long got = -1;
    for (;;) {
        const unsigned h = vc[0], t = vc[1];  // head, tail
        if ((int)(t - h) > 0) {
            if (atomicCAS(&c->head, h, h + 1u) == h) { got = (long long)h; break; }
            continue;
        }
        if (vc[5]) break;  // stop
        const long long now = (long long)global_ns();
        if (!waiting) {
            waiting = true;
            t0 = now;
            atomicAdd(&c->waiting, 1u);
        } else if (now - t0 > idle_ns) {
            break;
        }
        __nanosleep(8000);
    }
    if (waiting) atomicSub(&c->waiting, 1u);
    return got;
}

__shared__ __align__(16) MCParams32 s_params;  // the running item's search parameters (serving grid)
static_assert(sizeof(FeedItem32) % 16 == 0 && sizeof(DMaps32) % 16 == 0 && sizeof(MCParams32) % 16 == 0 &&
                  sizeof(Chain32) % 16 == 0,
              "serving-grid records are copied in 16-byte pieces");

// The serving grid: persistent blocks that take items from a ring the host
// keeps filling while the grid runs, so that a ligand's chains start as
// soon as a block is free, whatever launch it came with.  An item's block
// stages its ligand's model and runs one chain per team of warps (the
// item's team size); its chains signal completion as in k_mc32.  Everything an item points to is read through
// L2 only (the host reuses device memory while the grid runs).  A block
// leaves after idle_ns without work; the host starts more blocks when
// items wait and none is free.
__global__ void __launch_bounds__(SG_MC32_THREADS, SG_MC32_MINB) k_mc32_feed(DTables32 T, const FeedItem32* ring,
                                                                 unsigned cap, FeedCtrl32* ctrl, long long idle_ns) {
    __shared__ long long s_seq;
    __shared__ FeedItem32 s_fi;
    const int tid = threadIdx.x, nthr = blockDim.x, warp = tid >> 5;
    if (tid == 0) {
        sT32 = T;
        atomicAdd(&ctrl->started, 1u);
    }
    for (;;) {
        if (tid == 0) {
            s_seq = feed_claim(ctrl, idle_ns);
            if (s_seq >= 0) {
                const int4* src = reinterpret_cast<const int4*>(ring + (size_t)(s_seq % cap));
                int4* dst = reinterpret_cast<int4*>(&s_fi);
                for (int k = 0; k < (int)(sizeof(FeedItem32) / 16); k++) dst[k] = __ldcg(src + k);
                const int4* gs = reinterpret_cast<const int4*>(s_fi.maps);
                int4* gd = reinterpret_cast<int4*>(&sG32);
                for (int k = 0; k < (int)(sizeof(DMaps32) / 16); k++) gd[k] = __ldcg(gs + k);
                const int4* ps = reinterpret_cast<const int4*>(s_fi.params);
                int4* pd = reinterpret_cast<int4*>(&s_params);
                for (int k = 0; k < (int)(sizeof(MCParams32) / 16); k++) pd[k] = __ldcg(ps + k);
                sWs0 = s_fi.stage_stride;
                sWsStride = s_fi.ws_stride;
            }
        }
        __syncthreads();
        if (s_seq < 0) break;
        stage_model(s_fi.model, tid, nthr);
        const int team = s_fi.team == 4 ? 4 : s_fi.team == 2 ? 2 : 1;
        if (warp / team < s_fi.count) {
            Chain32 ch;
            const int4* cs = reinterpret_cast<const int4*>(s_fi.chains + warp / team);
            int4* cd = reinterpret_cast<int4*>(&ch);
            for (int k = 0; k < (int)(sizeof(Chain32) / 16); k++) cd[k] = __ldcg(cs + k);
            if (team == 4) run_team32<4>(ch, s_params);
            else if (team == 2) run_team32<2>(ch, s_params);
            else run_team32<1>(ch, s_params);
        }
        __syncthreads();  // the staged model is in use until every warp is done
    }
    if (tid == 0) atomicAdd(&ctrl->exited, 1u);
}

// model::eval_deriv in FP32 for a batch of confs of one model (one team of
// TEAM warps per conf); the model is staged like the search kernel's, the
// warps' workspaces follow it at ws_at, ws_stride apart
template <int TEAM>
__global__ void __launch_bounds__(32 * TEAM) k_eval32(const DModel* model, DTables32 T, DMaps32 G, int n,
                                                      const double* confs, float v0, float v1, float v2, float slope,
                                                      double* out_e, double* out_g, double* out_coords, int ws_at,
                                                      int ws_stride) {
    const int k = blockIdx.x;
    if (k >= n) return;
    if (threadIdx.x == 0) { sT32 = T; sG32 = G; sWs0 = ws_at; sWsStride = ws_stride; }
    stage_model(model, threadIdx.x, 32 * TEAM);
    if constexpr (TEAM > 1) {
        if (threadIdx.x >= 32) {
            team_help32<TEAM>();
            return;
        }
    }
    const W32 w = here();
    const SModel& m = smodel();
    const Ws32& L = m.L;
    unsigned* C = w.counters();
    for (int i = w.lane; i < 65; i += 32) C[i] = 0;
    for (int i = w.lane; i < m.natoms; i += 32) w.coords()[i] = __ldg(m.lab32 + i);  // inflex atoms stay here
    copyd(w, w.d(L.x_tmp), confs + (size_t)k * m.conf_size, m.conf_size);
    const float e = eval_deriv32<TEAM>(w.at(L.x_tmp), make_float3(v0, v1, v2), slope, w.at(L.g));
    if constexpr (TEAM > 1) team_publish<TEAM>(w, make_float3(0, 0, 0), 0.f, kTeamExit);
    const double* g = w.d(L.g);
    if (w.lane == 0) out_e[k] = e;
    for (int i = w.lane; i < m.dof; i += 32) out_g[(size_t)k * m.dof + i] = g[i];
    if (out_coords)
        for (int i = w.lane; i < m.nmov; i += 32) {
            const float4 c = w.coords()[i];
            double* o = out_coords + ((size_t)k * m.nmov + i) * 3;
            o[0] = c.x; o[1] = c.y; o[2] = c.z;
        }
}

// quasi_newton for a batch of confs of one model with the search's own
// mixed-precision BFGS (one team of TEAM warps per conf); confs are
// optimised in place
template <int TEAM>
__global__ void __launch_bounds__(32 * TEAM) k_bfgs32(const DModel* model, DTables32 T, DMaps32 G, int n,
                                                      double* confs, float v0, float v1, float v2, float slope,
                                                      int maxiters, int accurate, int early, double* out_e, int ws_at,
                                                      int ws_stride) {
    const int k = blockIdx.x;
    if (k >= n) return;
    if (threadIdx.x == 0) { sT32 = T; sG32 = G; sWs0 = ws_at; sWsStride = ws_stride; }
    stage_model(model, threadIdx.x, 32 * TEAM);
    if constexpr (TEAM > 1) {
        if (threadIdx.x >= 32) {
            team_help32<TEAM>();
            return;
        }
    }
    const W32 w = here();
    const SModel& m = smodel();
    const Ws32& L = m.L;
    unsigned* C = w.counters();
    for (int i = w.lane; i < 65; i += 32) C[i] = 0;
    for (int i = w.lane; i < m.natoms; i += 32) w.coords()[i] = __ldg(m.lab32 + i);  // inflex atoms stay here
    for (int f = w.lane; f < m.nframes; f += 32) w.origin()[f] = __ldg(m.finit32 + f);
    double* c = confs + (size_t)k * m.conf_size;
    copyd(w, w.d(L.x_tmp), c, m.conf_size);
    const double e = bfgs32<TEAM>(w.at(L.x_tmp), maxiters, accurate, early, Mode32{make_float3(v0, v1, v2), slope});
    if constexpr (TEAM > 1) team_publish<TEAM>(w, make_float3(0, 0, 0), 0.f, kTeamExit);
    const double* x = w.d(L.x_tmp);
    for (int i = w.lane; i < m.conf_size; i += 32) c[i] = x[i];
    if (w.lane == 0) out_e[k] = e;
}

// ---- host launchers -----------------------------------------------------------------------
size_t ws32_bytes(const DModel& hm) {
    return (size_t)ws32_layout(hm.natoms, hm.nframes, hm.conf_size, hm.dof).total;
}

// Raises the kernel's dynamic shared memory limit to `smem` (never lowers it,
// so launches sized against an earlier, larger limit stay valid).
static cudaError_t prep32(const void* fn, size_t smem) {
    cudaFuncAttributes fa{};
    cudaError_t rc = cudaFuncGetAttributes(&fa, fn);
    if (rc != cudaSuccess) return rc;
    if ((size_t)fa.maxDynamicSharedSizeBytes >= smem) return cudaSuccess;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

static const void* k_mc32_for(int team) {
    return team == 4 ? (const void*)k_mc32<4> : team == 2 ? (const void*)k_mc32<2> : (const void*)k_mc32<1>;
}

// resident blocks per SM of k_mc32 with `wpb` warps per block in teams of
// `team`; 0 when the shape does not fit (the failed call's error is
// cleared, so the next launch's check does not see it)
int mc32_occupancy(int team, int wpb, size_t smem) {
    int blocks = 0;
    const void* fn = k_mc32_for(team);
    if (prep32(fn, smem) != cudaSuccess || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, 32 * wpb, smem) !=
                                               cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return blocks;
}

cudaError_t launch_mc32(const DModel* dms, const DTables32& T, const DMaps32& G, const DMaps32* maps_tab,
                        const Chain32* chains, const Item32* items, int nitems, const MCParams32& P, unsigned* queue,
                        int blocks, int wpb, size_t stage_stride, size_t ws_stride, int team, cudaStream_t s) {
    if (!(team == 1 || team == 2 || team == 4) || wpb % team) return cudaErrorInvalidValue;
    const size_t smem = stage_stride + (size_t)wpb * ws_stride;
    cudaError_t rc = prep32(k_mc32_for(team), smem);
    if (rc != cudaSuccess) return rc;
    if (team == 4)
        k_mc32<4><<<blocks, 32 * wpb, smem, s>>>(dms, T, G, maps_tab, chains, items, nitems, P, queue,
                                                 (int)stage_stride, (int)ws_stride);
    else if (team == 2)
        k_mc32<2><<<blocks, 32 * wpb, smem, s>>>(dms, T, G, maps_tab, chains, items, nitems, P, queue,
                                                 (int)stage_stride, (int)ws_stride);
    else
        k_mc32<1><<<blocks, 32 * wpb, smem, s>>>(dms, T, G, maps_tab, chains, items, nitems, P, queue,
                                                 (int)stage_stride, (int)ws_stride);
    return cudaGetLastError();
}

// Raises k_mc32's dynamic shared-memory limit ahead of time, so that later
// launches (serving's many concurrent ones, the no-allocation entry point's)
// set no function attribute while other launches of the kernel run.  The
// first use also loads the kernel's module.
cudaError_t mc32_reserve_smem(size_t smem) { return prep32((const void*)k_mc32<1>, smem); }

// the largest dynamic shared memory a k_mc32 block can take: the device's
// opt-in limit less the kernel's static shared memory
cudaError_t mc32_max_dynamic_smem(size_t optin, size_t* out) {
    cudaFuncAttributes fa{};
    cudaError_t rc = cudaFuncGetAttributes(&fa, (const void*)k_mc32<1>);
    if (rc != cudaSuccess) return rc;
    *out = optin > fa.sharedSizeBytes ? optin - fa.sharedSizeBytes : 0;
    return cudaSuccess;
}

cudaError_t launch_mc32_fixed(const DModel* dms, const DTables32& T, const DMaps32& G, const DMaps32* maps_tab,
                              const Chain32* chains, const Item32* items, int nitems, const MCParams32& P,
                              unsigned* queue, int blocks, int wpb, size_t stage_stride, size_t ws_stride,
                              size_t smem_fixed, cudaStream_t s) {
    if (stage_stride + (size_t)wpb * ws_stride > smem_fixed) return cudaErrorInvalidValue;
    k_mc32<1><<<blocks, 32 * wpb, smem_fixed, s>>>(dms, T, G, maps_tab, chains, items, nitems, P, queue,
                                                   (int)stage_stride, (int)ws_stride);
    return cudaGetLastError();
}

// ws: one warp's workspace bytes (a multiple of 16); a team's block holds
// `team` of them
cudaError_t launch_eval32(const DModel* dm, size_t stage, size_t ws, const DTables32& T, const DMaps32& G, int n,
                          const double* confs, const double v[3], double slope, double* e, double* g, double* coords,
                          int team, cudaStream_t s) {
    if (!(team == 1 || team == 2 || team == 4)) return cudaErrorInvalidValue;
    const size_t smem = stage + (size_t)team * ws;
    const void* fn = team == 4 ? (const void*)k_eval32<4> : team == 2 ? (const void*)k_eval32<2> : (const void*)k_eval32<1>;
    cudaError_t rc = prep32(fn, smem);
    if (rc != cudaSuccess) return rc;
    const float v0 = (float)v[0], v1 = (float)v[1], v2 = (float)v[2], sl = (float)slope;
    if (team == 4) k_eval32<4><<<n, 128, smem, s>>>(dm, T, G, n, confs, v0, v1, v2, sl, e, g, coords, (int)stage, (int)ws);
    else if (team == 2) k_eval32<2><<<n, 64, smem, s>>>(dm, T, G, n, confs, v0, v1, v2, sl, e, g, coords, (int)stage, (int)ws);
    else k_eval32<1><<<n, 32, smem, s>>>(dm, T, G, n, confs, v0, v1, v2, sl, e, g, coords, (int)stage, (int)ws);
    return cudaGetLastError();
}

cudaError_t launch_bfgs32(const DModel* dm, size_t stage, size_t ws, const DTables32& T, const DMaps32& G, int n,
                          double* confs, const double v[3], double slope, int maxiters, int accurate, int early,
                          double* e, int team, cudaStream_t s) {
    if (!(team == 1 || team == 2 || team == 4)) return cudaErrorInvalidValue;
    const size_t smem = stage + (size_t)team * ws;
    const void* fn = team == 4 ? (const void*)k_bfgs32<4> : team == 2 ? (const void*)k_bfgs32<2> : (const void*)k_bfgs32<1>;
    cudaError_t rc = prep32(fn, smem);
    if (rc != cudaSuccess) return rc;
    const float v0 = (float)v[0], v1 = (float)v[1], v2 = (float)v[2], sl = (float)slope;
    if (team == 4)
        k_bfgs32<4><<<n, 128, smem, s>>>(dm, T, G, n, confs, v0, v1, v2, sl, maxiters, accurate, early, e, (int)stage, (int)ws);
    else if (team == 2)
        k_bfgs32<2><<<n, 64, smem, s>>>(dm, T, G, n, confs, v0, v1, v2, sl, maxiters, accurate, early, e, (int)stage, (int)ws);
    else
        k_bfgs32<1><<<n, 32, smem, s>>>(dm, T, G, n, confs, v0, v1, v2, sl, maxiters, accurate, early, e, (int)stage, (int)ws);
    return cudaGetLastError();
}

// A serving grid of `blocks` blocks of 32 * wpb threads with `smem` bytes
// of dynamic shared memory (raised beforehand with mc32_reserve_smem).
cudaError_t launch_mc32_feed(const DTables32& T, const FeedItem32* ring, unsigned cap, FeedCtrl32* ctrl,
                             long long idle_ns, int blocks, int wpb, size_t smem, cudaStream_t s) {
    k_mc32_feed<<<blocks, 32 * wpb, smem, s>>>(T, ring, cap, ctrl, idle_ns);
    return cudaGetLastError();
}

// raises k_mc32_feed's dynamic shared-memory limit ahead of its launches
cudaError_t mc32_feed_reserve_smem(size_t smem) { return prep32((const void*)k_mc32_feed, smem); }

// the largest dynamic shared memory a k_mc32_feed block can take within
// `optin` bytes: less the kernel's static shared memory
cudaError_t mc32_feed_max_dynamic_smem(size_t optin, size_t* out) {
    cudaFuncAttributes fa{};
    cudaError_t rc = cudaFuncGetAttributes(&fa, (const void*)k_mc32_feed);
    if (rc != cudaSuccess) return rc;
    *out = optin > fa.sharedSizeBytes ? optin - fa.sharedSizeBytes : 0;
    return cudaSuccess;
}

// resident k_mc32_feed blocks per SM with `wpb` warps and `smem` bytes
cudaError_t mc32_feed_occupancy(int wpb, size_t smem, int* blocks) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, k_mc32_feed, 32 * wpb, smem);
}

#ifdef SG_PROFILE
cudaError_t profile_read32(unsigned long long* out16, bool clear) {
    cudaError_t rc = cudaMemcpyFromSymbol(out16, g_prof, sizeof(unsigned long long) * 16);
    if (rc == cudaSuccess && clear) {
        static const unsigned long long zero[16] = {};
        rc = cudaMemcpyToSymbol(g_prof, zero, sizeof(zero));
    }
    return rc;
}
#endif

}  // namespace sg
