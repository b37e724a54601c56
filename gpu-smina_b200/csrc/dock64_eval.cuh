// Plain (FP64) path, part 1: one warp evaluates model::eval_deriv.
//
// Bit-exact with a CPU FP64 run when compiled with -fmad=false: every
// reduction whose order matters is done in the reference's order
// (per-atom force accumulation over an ordered pair list, sequential energy
// sums, per-frame force/torque sums in atom order, children added in order).
// Reference: model.cpp:837-841,904-928,969-985; grid.cpp:27-46,111-236;
// cache.cpp:69-90; non_cache.cpp:109-191; tree.h:108-243;
// precalculate.h:111-151,245-293.
#pragma once
#include "grid64.cuh"

namespace sg {

constexpr unsigned kFull = 0xffffffffu;

struct W64 {
    double* s;       // this warp's workspace
    uint8_t* pin;    // pair-in-cutoff flags
    uint32_t* mt;    // mt19937 state (625 words)
    Ws64 L;
    const DModel* m;
    const DTables* T;
    const DReceptor* R;
    int lane;
    int* err;
    unsigned long long evals;
    const double* box;  // this item's own box (lo xyz, hi xyz) for the direct sum; null: the receptor's
};

__device__ __forceinline__ V3<double> ld3(const double* p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ void st3(double* p, V3<double> v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

// model::set: frames level by level, then atoms
__device__ void set_conf64(W64& w, const double* conf) {
    const DModel& m = *w.m;
    double* S = w.s;
    for (int lv = 0; lv < m.nlevels; lv++) {
        for (int idx = m.level_start[lv] + w.lane; idx < m.level_start[lv + 1]; idx += 32) {
            const int f = m.level_frames[idx];
            const int kind = m.fkind[f];
            Quat<double> q;
            if (kind == SG_FRAME_RIGID) {
                const double* c = conf + m.fconf[f];
                st3(S + w.L.origin + 3 * f, V3<double>{c[0], c[1], c[2]});
                q = Quat<double>{c[3], c[4], c[5], c[6]};
            } else if (kind == SG_FRAME_SEGMENT) {
                const int p = m.fparent[f];
                const double* prot = S + w.L.rot + 9 * p;
                V3<double> o = ld3(S + w.L.origin + 3 * p) + mat_mul(prot, ld3(m.forigin + 3 * f));
                V3<double> ax = mat_mul(prot, ld3(m.faxis + 3 * f));
                st3(S + w.L.origin + 3 * f, o);
                st3(S + w.L.axis + 3 * f, ax);
                const double* pq = S + w.L.q + 4 * p;
                q = qmul(axis_angle_q(ax, conf[m.fconf[f]]), Quat<double>{pq[0], pq[1], pq[2], pq[3]});
                q_normalize_approx(q);
            } else {
                V3<double> ax = ld3(m.faxis + 3 * f);
                st3(S + w.L.origin + 3 * f, ld3(m.forigin + 3 * f));
                st3(S + w.L.axis + 3 * f, ax);
                q = axis_angle_q(ax, conf[m.fconf[f]]);
            }
            double* qd = S + w.L.q + 4 * f;
            qd[0] = q.a; qd[1] = q.b; qd[2] = q.c; qd[3] = q.d;
            quat_to_mat(q, S + w.L.rot + 9 * f);
        }
        __syncwarp();
    }
    for (int i = w.lane; i < m.nmov; i += 32) {
        const int f = m.atom_frame[i];
        V3<double> c = ld3(S + w.L.origin + 3 * f) + mat_mul(S + w.L.rot + 9 * f, ld3(m.local + 3 * i));
        st3(S + w.L.coords + 3 * i, c);
    }
    __syncwarp();
}

// precalculate_linear::eval_deriv (type-ordered lookup, charge-weighted components)
__device__ __forceinline__ double comp_eval(const double* c, double qa, double qb) {
    return c[0] + fabs(qa) * c[2] + fabs(qb) * c[4] + qa * qb * c[6];
}
__device__ void table_deriv64(const DTables& T, int ta, double qa, int tb, double qb, double r2, double& e,
                              double& dor) {
    if (ta > tb) {
        int t = ta; ta = tb; tb = t;
        double q = qa; qa = qb; qb = q;
    }
    const int p = tri_index(ta, tb);
    const double rf = T.factor * r2;
    const size_t i1 = (size_t)rf;
    const double rem = rf - (double)i1;
    const int nc = T.nc;
    const double* s1 = T.smooth + ((size_t)p * T.n + i1) * nc * 2;
    const double* s2 = s1 + nc * 2;
    double e1, e2, d1, d2;
    if (nc == 1) {
        e1 = s1[0]; d1 = s1[1]; e2 = s2[0]; d2 = s2[1];
    } else {
        e1 = comp_eval(s1, qa, qb);
        e2 = comp_eval(s2, qa, qb);
        d1 = comp_eval(s1 + 1, qa, qb);
        d2 = comp_eval(s2 + 1, qa, qb);
    }
    e = e1 + rem * (e2 - e1);
    dor = d1 + rem * (d2 - d1);
}

// cache::eval_deriv: per movable atom grid energy and derivative
__device__ void grid_atoms64(W64& w, double v, double slope) {
    const DModel& m = *w.m;
    double* S = w.s;
    for (int i = w.lane; i < m.nmov; i += 32) {
        const int t = m.type[i];
        double* mf = S + w.L.mf + 3 * i;
        if (t >= kNumTypes || is_h(t)) {
            mf[0] = mf[1] = mf[2] = 0;
            S[w.L.eatom + i] = 0;
            continue;
        }
        const V3<double> loc = ld3(S + w.L.coords + 3 * i);
        V3<double> d;
        double ret = grid_aux64(w.R->g, w.R->map[t], loc, slope, v, d);
        const double q = m.charge[i];
        if (q != 0 && w.R->cmap[t]) {
            V3<double> cd{0, 0, 0};
            ret += q * grid_aux64(w.R->g, w.R->cmap[t], loc, slope, v, cd);
            add_to(d, q * cd);
        }
        S[w.L.eatom + i] = ret;
        st3(mf, d);
    }
}

// non_cache::eval_deriv: direct sum over the 3 A cell list of the clamped atom
__device__ void direct_atoms64(W64& w, double v, double slope) {
    const DModel& m = *w.m;
    const DReceptor& R = *w.R;
    const DGeom& G = R.g;
    double* S = w.s;
    for (int i = w.lane; i < m.nmov; i += 32) {
        const int t = m.type[i];
        double* mf = S + w.L.mf + 3 * i;
        if (t >= kNumTypes || is_h(t)) {
            mf[0] = mf[1] = mf[2] = 0;
            S[w.L.eatom + i] = 0;
            continue;
        }
        const double a[3] = {S[w.L.coords + 3 * i], S[w.L.coords + 3 * i + 1], S[w.L.coords + 3 * i + 2]};
        double adj[3] = {a[0], a[1], a[2]}, oobd[3] = {0, 0, 0}, oob = 0;
        for (int j = 0; j < 3; j++) {
            const double lo = w.box ? w.box[j] : G.gd_begin[j], hi = w.box ? w.box[3 + j] : G.gd_end[j];
            if (w.box || G.gd_n[j] > 0) {
                if (a[j] < lo) { adj[j] = lo; oobd[j] = -1; oob += fabs(a[j] - lo); }
                else if (a[j] > hi) { adj[j] = hi; oobd[j] = 1; oob += fabs(a[j] - hi); }
            }
        }
        oob *= slope;
        oobd[0] *= slope; oobd[1] *= slope; oobd[2] *= slope;
        int ci[3];
        for (int j = 0; j < 3; j++) ci[j] = (int)floor(adj[j] / 3.0) - G.cell_off[j];
        double this_e = 0;
        V3<double> deriv{0, 0, 0};
        const bool inside = ci[0] >= 0 && ci[1] >= 0 && ci[2] >= 0 && ci[0] < G.cell_dim[0] && ci[1] < G.cell_dim[1] &&
                            ci[2] < G.cell_dim[2];
        if (inside) {
            const int cell = ci[0] + G.cell_dim[0] * (ci[1] + G.cell_dim[1] * ci[2]);
            const double qi = m.charge[i];
            for (int k = R.full_start[cell]; k < R.full_start[cell + 1]; k++) {
                const int j = R.full_atoms[k];
                const V3<double> rba{adj[0] - R.xyz[3 * j], adj[1] - R.xyz[3 * j + 1], adj[2] - R.xyz[3 * j + 2]};
                const double r2 = norm2(rba);
                if (r2 < w.T->cutoff_sqr) {
                    if (r2 < kEps) atomicExch(w.err, kDevOverlap);
                    double pe, dor;
                    table_deriv64(*w.T, t, qi, R.type[j], R.charge[j], r2, pe, dor);
                    this_e += pe;
                    add_to(deriv, dor * rba);
                }
            }
        } else {
            atomicExch(w.err, kDevBadModel);
        }
        if (R.ugrid) {  // the user grid at the atom's own coordinates (non_cache.cpp:180-184)
            V3<double> ugd;
            this_e += grid_aux64(R.ug, R.ugrid, V3<double>{a[0], a[1], a[2]}, slope, 1000.0, ugd);
            add_to(deriv, ugd);
        }
        curl_ed(this_e, deriv, v);
        mf[0] = deriv.x + oobd[0];
        mf[1] = deriv.y + oobd[1];
        mf[2] = deriv.z + oobd[2];
        S[w.L.eatom + i] = this_e + oob;
    }
}

// intramolecular / other pairs: force and energy per pair, into the workspace
__device__ void pairs64(W64& w, const double v[3]) {
    const DModel& m = *w.m;
    double* S = w.s;
    for (int k = w.lane; k < m.npairs; k += 32) {
        const int a = m.pairs[2 * k], b = m.pairs[2 * k + 1];
        const V3<double> r = ld3(S + w.L.coords + 3 * b) - ld3(S + w.L.coords + 3 * a);
        const double r2 = norm2(r);
        uint8_t in = 0;
        if (r2 < w.T->cutoff_sqr) {
            double pe, dor;
            table_deriv64(*w.T, m.type[a], m.charge[a], m.type[b], m.charge[b], r2, pe, dor);
            V3<double> force = dor * r;
            curl_ed(pe, force, m.pair_group[k] == 0 ? v[2] : v[0]);
            S[w.L.pe + k] = pe;
            st3(S + w.L.pf + 3 * k, force);
            in = 1;
        }
        w.pin[k] = in;
    }
    __syncwarp();
}

// minus_forces: grid derivative, then every pair contribution in pair order
__device__ void gather_forces64(W64& w) {
    const DModel& m = *w.m;
    double* S = w.s;
    for (int i = w.lane; i < m.nmov; i += 32) {
        V3<double> f = ld3(S + w.L.mf + 3 * i);
        for (int c = m.csr_start[i]; c < m.csr_start[i + 1]; c++) {
            const int e = m.csr[c];
            const int k = e >> 1;
            if (!w.pin[k]) continue;
            const V3<double> pf = ld3(S + w.L.pf + 3 * k);
            if (e & 1) add_to(f, pf);
            else sub_from(f, pf);
        }
        st3(S + w.L.mf + 3 * i, f);
    }
}

// total energy in the reference's order: grid atoms, other pairs, each ligand
__device__ double energy64(W64& w) {
    const DModel& m = *w.m;
    const double* S = w.s;
    double part = 0;
    if (w.lane == 0) {
        for (int i = 0; i < m.nmov; i++) {
            const int t = m.type[i];
            if (t < kNumTypes && !is_h(t)) part += S[w.L.eatom + i];
        }
    } else if (w.lane == 1) {
        for (int k = 0; k < m.nother; k++)
            if (w.pin[k]) part += S[w.L.pe + k];
    } else if (w.lane - 2 < m.nlig) {
        const int l = w.lane - 2;
        const int b = l == 0 ? m.nother : m.lig_pair_end[l - 1];
        for (int k = b; k < m.lig_pair_end[l]; k++)
            if (w.pin[k]) part += S[w.L.pe + k];
    }
    double e = __shfl_sync(kFull, part, 0);
    e += __shfl_sync(kFull, part, 1);
    for (int l = 0; l < m.nlig && l < 30; l++) e += __shfl_sync(kFull, part, 2 + l);
    return e;
}

// ---- energy-only scoring (final rescoring of docked poses) ---------------------------------
// precalculate_linear::eval (precalculate.h:75-83,103-108,191-203): the fast
// table's components at sz(factor r2), weighted by a's and b's charges
// (result_components::eval, result_components.h:75-81); for t_a > t_b the
// (t_b, t_a) entry with its A and B components swapped (swapOrder).
__device__ __forceinline__ double table_fast64(const DTables& T, int ta, double qa, int tb, double qb, double r2) {
    const bool sw = ta > tb;
    const int p = sw ? tri_index(tb, ta) : tri_index(ta, tb);
    const double* c = T.fast + ((size_t)p * T.n + (size_t)(T.factor * r2)) * T.nc;
    double ca = 0, cb = 0, cab = 0;
    if (T.nc > 1) { ca = sw ? c[2] : c[1]; cb = sw ? c[1] : c[2]; cab = c[3]; }
    return c[0] + fabs(qa) * ca + fabs(qb) * cb + qa * qb * cab;
}

// non_cache::eval (non_cache.cpp:34-91): per movable heavy atom, the direct
// sum over its clamped position's cell list, curled, plus the out-of-box
// penalty; into eatom (summed in atom order by energy64)
__device__ void direct_energy64(W64& w, double v, double slope) {
    const DModel& m = *w.m;
    const DReceptor& R = *w.R;
    const DGeom& G = R.g;
    double* S = w.s;
    for (int i = w.lane; i < m.nmov; i += 32) {
        const int t = m.type[i];
        if (t >= kNumTypes || is_h(t)) { S[w.L.eatom + i] = 0; continue; }
        const double a[3] = {S[w.L.coords + 3 * i], S[w.L.coords + 3 * i + 1], S[w.L.coords + 3 * i + 2]};
        double adj[3] = {a[0], a[1], a[2]}, oob = 0;
        for (int j = 0; j < 3; j++) {
            if (G.gd_n[j] > 0) {
                if (a[j] < G.gd_begin[j]) { adj[j] = G.gd_begin[j]; oob += fabs(a[j] - G.gd_begin[j]); }
                else if (a[j] > G.gd_end[j]) { adj[j] = G.gd_end[j]; oob += fabs(a[j] - G.gd_end[j]); }
            }
        }
        oob *= slope;
        int ci[3];
        for (int j = 0; j < 3; j++) ci[j] = (int)floor(adj[j] / 3.0) - G.cell_off[j];
        double this_e = 0;
        if (ci[0] >= 0 && ci[1] >= 0 && ci[2] >= 0 && ci[0] < G.cell_dim[0] && ci[1] < G.cell_dim[1] &&
            ci[2] < G.cell_dim[2]) {
            const int cell = ci[0] + G.cell_dim[0] * (ci[1] + G.cell_dim[1] * ci[2]);
            for (int k = R.full_start[cell]; k < R.full_start[cell + 1]; k++) {
                const int j = R.full_atoms[k];
                const V3<double> rba{adj[0] - R.xyz[3 * j], adj[1] - R.xyz[3 * j + 1], adj[2] - R.xyz[3 * j + 2]};
                const double r2 = norm2(rba);
                if (r2 < w.T->cutoff_sqr) this_e += table_fast64(*w.T, t, m.charge[i], R.type[j], R.charge[j], r2);
            }
        } else {
            atomicExch(w.err, kDevBadModel);
        }
        curl_e(this_e, v);
        S[w.L.eatom + i] = this_e + oob;
    }
}

// model::eval_interacting_pairs (model.cpp:885-902) for every pair: curled
// energy into pe, in-cutoff flag into pin
__device__ void pairs_energy64(W64& w, const double v[3]) {
    const DModel& m = *w.m;
    double* S = w.s;
    for (int k = w.lane; k < m.npairs; k += 32) {
        const int a = m.pairs[2 * k], b = m.pairs[2 * k + 1];
        const double r2 = norm2(ld3(S + w.L.coords + 3 * a) - ld3(S + w.L.coords + 3 * b));
        uint8_t in = 0;
        if (r2 < w.T->cutoff_sqr) {
            double pe = table_fast64(*w.T, m.type[a], m.charge[a], m.type[b], m.charge[b], r2);
            curl_e(pe, m.pair_group[k] == 0 ? v[2] : v[0]);
            S[w.L.pe + k] = pe;
            in = 1;
        }
        w.pin[k] = in;
    }
    __syncwarp();
}

// model::eval_intramolecular (model.cpp:1027-1079) after pairs_energy64 on the
// same coords: each ligand's pairs, then every flexible movable atom against
// every receptor atom (curled per pair), then flex-flex other pairs.  One
// running sum in the reference's order; the flex-rigid energies of 32
// receptor atoms are computed at once and added by lane 0 in atom order.
__device__ double intramolecular64(W64& w, const double v[3]) {
    const DModel& m = *w.m;
    const DReceptor& R = *w.R;
    const double* S = w.s;
    auto in_ligand = [&](int i) {
        for (int l = 0; l < m.nlig; l++)
            if (i >= m.lig_begin[l] && i < m.lig_end[l]) return true;
        return false;
    };
    double e = 0;
    if (w.lane == 0) {
        int start = m.nother;
        for (int l = 0; l < m.nlig; l++) {
            double el = 0;
            for (int k = start; k < m.lig_pair_end[l]; k++)
                if (w.pin[k]) el += S[w.L.pe + k];
            e += el;
            start = m.lig_pair_end[l];
        }
    }
    for (int i = 0; i < m.nmov; i++) {  // warp-uniform
        if (in_ligand(i) || m.type[i] >= kNumTypes) continue;
        const V3<double> a = ld3(S + w.L.coords + 3 * i);
        for (int j0 = 0; j0 < R.natoms; j0 += 32) {
            const int j = j0 + w.lane;
            double this_e = 0;
            bool add = false;
            if (j < R.natoms && R.type[j] < kNumTypes) {
                const double r2 = norm2(a - V3<double>{R.xyz[3 * j], R.xyz[3 * j + 1], R.xyz[3 * j + 2]});
                if (r2 < w.T->cutoff_sqr) {
                    this_e = table_fast64(*w.T, m.type[i], m.charge[i], R.type[j], R.charge[j], r2);
                    curl_e(this_e, v[1]);
                    add = true;
                }
            }
            for (int l = 0; l < 32; l++) {
                const double x = __shfl_sync(kFull, this_e, l);
                const int ok = __shfl_sync(kFull, (int)add, l);
                if (w.lane == 0 && ok) e += x;
            }
        }
    }
    if (w.lane == 0)
        for (int k = 0; k < m.nother; k++) {
            const int a = m.pairs[2 * k], b = m.pairs[2 * k + 1];
            if (w.pin[k] && !in_ligand(a) && !in_ligand(b)) e += S[w.L.pe + k];
        }
    return __shfl_sync(kFull, e, 0);
}

// tree derivative: per-frame sums, children bottom-up, then the change vector
__device__ void derivative64(W64& w, double* g) {
    const DModel& m = *w.m;
    double* S = w.s;
    for (int f = w.lane; f < m.nframes; f += 32) {
        V3<double> F{0, 0, 0}, T{0, 0, 0};
        const V3<double> o = ld3(S + w.L.origin + 3 * f);
        for (int i = m.fbegin[f]; i < m.fend[f]; i++) {
            const V3<double> fi = ld3(S + w.L.mf + 3 * i);
            add_to(F, fi);
            add_to(T, cross(ld3(S + w.L.coords + 3 * i) - o, fi));
        }
        st3(S + w.L.fF + 3 * f, F);
        st3(S + w.L.fT + 3 * f, T);
    }
    __syncwarp();
    for (int lv = m.nlevels - 2; lv >= 0; lv--) {
        for (int idx = m.level_start[lv] + w.lane; idx < m.level_start[lv + 1]; idx += 32) {
            const int f = m.level_frames[idx];
            if (m.child_start[f] == m.child_start[f + 1]) continue;
            V3<double> F = ld3(S + w.L.fF + 3 * f), T = ld3(S + w.L.fT + 3 * f);
            const V3<double> o = ld3(S + w.L.origin + 3 * f);
            for (int c = m.child_start[f]; c < m.child_start[f + 1]; c++) {
                const int ch = m.child_list[c];
                const V3<double> cF = ld3(S + w.L.fF + 3 * ch);
                add_to(F, cF);
                const V3<double> r = ld3(S + w.L.origin + 3 * ch) - o;
                add_to(T, cross(r, cF) + ld3(S + w.L.fT + 3 * ch));
            }
            st3(S + w.L.fF + 3 * f, F);
            st3(S + w.L.fT + 3 * f, T);
        }
        __syncwarp();
    }
    for (int f = w.lane; f < m.nframes; f += 32) {
        const V3<double> F = ld3(S + w.L.fF + 3 * f), T = ld3(S + w.L.fT + 3 * f);
        if (m.fkind[f] == SG_FRAME_RIGID) {
            double* d = g + m.fdof[f];
            d[0] = F.x; d[1] = F.y; d[2] = F.z; d[3] = T.x; d[4] = T.y; d[5] = T.z;
        } else {
            g[m.fdof[f]] = dot(T, ld3(S + w.L.axis + 3 * f));
        }
    }
    __syncwarp();
}

// model::eval_deriv; `direct` selects non_cache instead of the grid maps
__device__ double eval_deriv64(W64& w, const double* conf, const double v[3], double slope, bool direct, double* g) {
    set_conf64(w, conf);
    if (direct) direct_atoms64(w, v[1], slope);
    else grid_atoms64(w, v[1], slope);
    pairs64(w, v);
    gather_forces64(w);
    __syncwarp();
    const double e = energy64(w);
    derivative64(w, g);
    w.evals++;
    return e;
}

}  // namespace sg
