/*
 * ORACLE (test infrastructure only): CPU FP64 restatement of smina's search
 * path.  See or_core.h.  Reference paths are relative to the reference
 * project root.
 */
#include "or_core.h"
#include <algorithm>
#include <cmath>
#include <memory>
#include <stdexcept>

namespace orc {

// common.h:262-281
void normalize_angle(double& x) {
    if (x > 3 * PI) {
        double n = (x - PI) / (2 * PI);
        x -= 2 * PI * std::ceil(n);
        normalize_angle(x);
    } else if (x < -3 * PI) {
        double n = (-x - PI) / (2 * PI);
        x += 2 * PI * std::ceil(n);
        normalize_angle(x);
    } else if (x > PI) {
        x -= 2 * PI;
    } else if (x < -PI) {
        x += 2 * PI;
    }
}
static double normalized_angle(double x) { normalize_angle(x); return x; }

// quaternion.cpp:42-49
Q angle_to_quaternion(const V3& axis, double angle) {
    normalize_angle(angle);
    double c = pm_cos(angle / 2);
    double s = pm_sin(angle / 2);
    return Q{c, s * axis[0], s * axis[1], s * axis[2]};
}
// quaternion.cpp:51-61
Q angle_to_quaternion(const V3& rotation) {
    double angle = std::sqrt(sqrv(rotation));
    if (angle > EPS) {
        V3 axis = (1 / angle) * rotation;
        return angle_to_quaternion(axis, angle);
    }
    return Q{1, 0, 0, 0};
}
// quaternion.cpp:63-81
V3 quaternion_to_angle(const Q& q) {
    double c = q.a;
    if (c > -1 && c < 1) {
        double angle = 2 * pm_acos(c);
        if (angle > PI) angle -= 2 * PI;
        V3 axis(q.b, q.c, q.d);
        double s = pm_sin(angle / 2);
        if (std::fabs(s) < EPS) return V3(0, 0, 0);
        double k = angle / s;
        axis[0] *= k; axis[1] *= k; axis[2] *= k;
        return axis;
    }
    return V3(0, 0, 0);
}
// quaternion.cpp:83-118
M3 quaternion_to_r3(const Q& q) {
    double a = q.a, b = q.b, c = q.c, d = q.d;
    double aa = a * a, ab = a * b, ac = a * c, ad = a * d, bb = b * b, bc = b * c, bd = b * d,
           cc = c * c, cd = c * d, dd = d * d;
    M3 m;
    m.d[0] = (aa + bb - cc - dd);
    m.d[3] = 2 * (-ad + bc);
    m.d[6] = 2 * (ac + bd);
    m.d[1] = 2 * (ad + bc);
    m.d[4] = (aa - bb + cc - dd);
    m.d[7] = 2 * (-ab + cd);
    m.d[2] = 2 * (-ac + bd);
    m.d[5] = 2 * (ab + cd);
    m.d[8] = (aa - bb - cc + dd);
    return m;
}
// quaternion.h:86-97
void quaternion_normalize_approx(Q& q) {
    double s = sqr(q.a) + sqr(q.b) + sqr(q.c) + sqr(q.d);
    if (std::fabs(s - 1) < 1e-6) return;
    double a = std::sqrt(s);
    double inv = 1 / a;
    q.a *= inv; q.b *= inv; q.c *= inv; q.d *= inv;
}
// quaternion.cpp:135-139
void quaternion_increment(Q& q, const V3& rotation) {
    q = qmul(angle_to_quaternion(rotation), q);
    quaternion_normalize_approx(q);
}
// curl.h:30-43 (soft curl)
template <> void curl<V3>(double& e, V3& deriv, double v) {
    if (e > 0 && v < 0.1 * MAXF) {
        double tmp = (v < EPS) ? 0 : (v / (v + e));
        e *= tmp;
        double t2 = sqr(tmp);
        deriv[0] *= t2; deriv[1] *= t2; deriv[2] *= t2;
    }
}
void curl(double& e, double v) {
    if (e > 0 && v < 0.1 * MAXF) {
        double tmp = (v < EPS) ? 0 : (v / (v + e));
        e *= tmp;
    }
}

static inline bool is_h(int t) { return t == 0 || t == 1; }

// ---- loading ------------------------------------------------------------
void Model::load(const sg_model_desc& m) {
    num_atoms = m.num_atoms; num_movable = m.num_movable; num_frames = m.num_frames;
    num_ligands = m.num_ligands; num_flex = m.num_flex; conf_size = m.conf_size; dof = m.dof;
    num_pairs = m.num_pairs; num_other_pairs = m.num_other_pairs;
    lig_pair_end.assign(m.lig_pair_end, m.lig_pair_end + num_ligands);
    lig_begin.assign(m.ligand_atom_begin, m.ligand_atom_begin + num_ligands);
    lig_end.assign(m.ligand_atom_end, m.ligand_atom_end + num_ligands);
    lig_root.assign(m.ligand_root, m.ligand_root + num_ligands);
    type.assign(m.atom_type, m.atom_type + num_atoms);
    charge.assign(m.atom_charge, m.atom_charge + num_atoms);
    local.resize(num_atoms);
    lab.resize(num_atoms);
    for (int i = 0; i < num_atoms; i++) {
        local[i] = V3(m.atom_local[3 * i], m.atom_local[3 * i + 1], m.atom_local[3 * i + 2]);
        lab[i] = V3(m.atom_lab[3 * i], m.atom_lab[3 * i + 1], m.atom_lab[3 * i + 2]);
    }
    fkind.assign(m.frame_kind, m.frame_kind + num_frames);
    fparent.assign(m.frame_parent, m.frame_parent + num_frames);
    fbegin.assign(m.frame_begin, m.frame_begin + num_frames);
    fend.assign(m.frame_end, m.frame_end + num_frames);
    fconf.assign(m.frame_conf, m.frame_conf + num_frames);
    fdof.assign(m.frame_dof, m.frame_dof + num_frames);
    forigin.resize(num_frames); faxis.resize(num_frames); finit.resize(num_frames);
    children.assign(num_frames, {});
    for (int f = 0; f < num_frames; f++) {
        forigin[f] = V3(m.frame_origin[3 * f], m.frame_origin[3 * f + 1], m.frame_origin[3 * f + 2]);
        faxis[f] = V3(m.frame_axis[3 * f], m.frame_axis[3 * f + 1], m.frame_axis[3 * f + 2]);
        finit[f] = V3(m.frame_init_origin[3 * f], m.frame_init_origin[3 * f + 1], m.frame_init_origin[3 * f + 2]);
        if (fparent[f] >= 0) children[fparent[f]].push_back(f);
    }
    pairs.resize(num_pairs);
    for (int k = 0; k < num_pairs; k++) pairs[k] = {m.pairs[2 * k], m.pairs[2 * k + 1]};
    heavy.clear();
    for (int i = 0; i < num_movable; i++)
        if (!is_h(type[i])) heavy.push_back(i);
    // conf blocks: ligands then flex residues (conf.h: conf::increment)
    blocks.clear();
    for (int f = 0; f < num_frames; f++) {
        if (fkind[f] == SG_FRAME_RIGID || fkind[f] == SG_FRAME_FIRST_SEGMENT) {
            Block b;
            b.rigid = fkind[f] == SG_FRAME_RIGID;
            b.conf_off = fconf[f];
            b.dof_off = fdof[f];
            b.ntors = 0;
            blocks.push_back(b);
        }
        if (fkind[f] != SG_FRAME_RIGID) blocks.back().ntors++;
    }
}

void Tables::load(const sg_tables_desc& t) {
    nt = t.num_types; nc = t.num_components; n = t.n; factor = t.factor; cutoff_sqr = t.cutoff_sqr;
    size_t np = (size_t)nt * (nt + 1) / 2;
    smooth.assign(t.smooth, t.smooth + np * n * nc * 2);
    fast.assign(t.fast, t.fast + np * n * nc);
}

void GridGeom::init_from(const sg_grid_dims& g) {  // grid.cpp:57-75
    gd = g;
    for (int i = 0; i < 3; i++) {
        dim[i] = g.n[i] + 1;
        init[i] = g.begin[i];
        double range = g.end[i] - g.begin[i];
        dim_fl_minus_1[i] = dim[i] - 1.0;
        factor[i] = dim_fl_minus_1[i] / range;
        factor_inv[i] = 1 / factor[i];
    }
}
V3 GridGeom::index_to_argument(int x, int y, int z) const {  // grid.h:75-80
    return V3(init[0] + factor_inv[0] * x, init[1] + factor_inv[1] * y, init[2] + factor_inv[2] * z);
}

// brick.h:20-38
static double closest_between(double b, double e, double x) {
    if (x <= b) return b;
    if (x >= e) return e;
    return x;
}
static double brick_distance_sqr(const V3& b, const V3& e, const V3& v) {
    V3 c(closest_between(b[0], e[0], v[0]), closest_between(b[1], e[1], v[1]), closest_between(b[2], e[2], v[2]));
    return dist2(c, v);
}

// szv_grid.h:97-160
void CellLists::init(const Receptor& rec, double cut2, const sg_grid_dims& gd) {
    r = &rec;
    cutoff_sqr = cut2;
    relevant.clear();
    cache.clear();
    V3 s(gd.begin[0], gd.begin[1], gd.begin[2]), e(gd.end[0], gd.end[1], gd.end[2]);
    for (size_t i = 0; i < rec.xyz.size(); i++) {
        int t = rec.type[i];
        if (t < SG_NUM_TYPES && !is_h(t) && brick_distance_sqr(s, e, rec.xyz[i]) < cutoff_sqr)
            relevant.push_back((int)i);
    }
}
const std::vector<int>& CellLists::get(const V3& coord) {
    const double gran = 3.0;
    std::array<int, 3> key;
    for (int i = 0; i < 3; i++) key[i] = (int)std::floor(coord[i] / gran);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    V3 lo, hi;
    for (int i = 0; i < 3; i++) {
        lo[i] = std::floor(coord[i] / gran) * gran;
        hi[i] = full_cells ? lo[i] + gran : std::ceil(coord[i] / gran) * gran;
    }
    std::vector<int> atoms;
    for (int i : relevant)
        if (brick_distance_sqr(lo, hi, r->xyz[i]) < cutoff_sqr) atoms.push_back(i);
    return cache.emplace(key, std::move(atoms)).first->second;
}

// ---- tables ---------------------------------------------------------------
// result_components::eval (result_components.h:73-79)
static inline double comp_eval(const double* c, double qa, double qb) {
    return c[0] + std::fabs(qa) * c[1] + std::fabs(qb) * c[2] + qa * qb * c[3];
}
// precalculate_linear::eval_deriv + element eval_deriv (precalculate.h:111-151, 245-293)
static void table_eval_deriv(const Tables& T, int ta, double qa, int tb, double qb, double r2, double& e, double& dor) {
    if (ta > tb) { std::swap(ta, tb); std::swap(qa, qb); }
    int p = ta + tb * (tb + 1) / 2;
    double rf = T.factor * r2;
    size_t i1 = (size_t)rf;
    size_t i2 = i1 + 1;
    double rem = rf - i1;
    const int nc = T.nc;
    const double* s1 = &T.smooth[(((size_t)p * T.n + i1) * nc) * 2];
    const double* s2 = &T.smooth[(((size_t)p * T.n + i2) * nc) * 2];
    double e1, e2, d1, d2;
    if (nc == 1) {
        e1 = s1[0]; d1 = s1[1]; e2 = s2[0]; d2 = s2[1];
    } else {
        double c[4];
        for (int k = 0; k < 4; k++) c[k] = s1[2 * k];
        e1 = comp_eval(c, qa, qb);
        for (int k = 0; k < 4; k++) c[k] = s2[2 * k];
        e2 = comp_eval(c, qa, qb);
        for (int k = 0; k < 4; k++) c[k] = s1[2 * k + 1];
        d1 = comp_eval(c, qa, qb);
        for (int k = 0; k < 4; k++) c[k] = s2[2 * k + 1];
        d2 = comp_eval(c, qa, qb);
    }
    e = e1 + rem * (e2 - e1);
    dor = d1 + rem * (d2 - d1);
}

// precalculate_linear::eval_fast (precalculate.h:190-203, 239-243)
static void table_eval_fast(const Tables& T, int t1, int t2, double r2, double* out) {
    bool swapped = t1 > t2;
    int p = swapped ? t2 + t1 * (t1 + 1) / 2 : t1 + t2 * (t2 + 1) / 2;
    size_t i = (size_t)(T.factor * r2);
    const double* f = &T.fast[((size_t)p * T.n + i) * T.nc];
    for (int c = 0; c < T.nc; c++) out[c] = f[c];
    if (swapped && T.nc > 1) std::swap(out[1], out[2]);
}

// ---- cache::populate (cache.cpp:116-206) ----------------------------------
static double evaluate_aux(const GridGeom& G, const std::vector<double>& D, const V3& loc, double slope, double v,
                           V3* deriv);

void populate(Ctx& c, const int* types, int ntypes) {
    std::vector<int> needed;
    for (int k = 0; k < ntypes; k++) {
        int t = types[k];
        if (t < 0 || t >= SG_NUM_TYPES) continue;
        if (!c.built[t] && std::find(needed.begin(), needed.end(), t) == needed.end()) needed.push_back(t);
    }
    if (needed.empty()) return;
    const GridGeom& g = c.geom;
    const bool charged = c.tab.nc > 1;
    size_t npts = (size_t)g.dim[0] * g.dim[1] * g.dim[2];
    for (int t : needed) {
        c.grids[t].data.assign(npts, 0);
        if (charged) c.grids[t].chargedata.assign(npts, 0);
    }
    CellLists cl;
    cl.init(c.rec, c.tab.cutoff_sqr, g.gd);
    std::vector<double> aff(needed.size()), chg(needed.size());
    double val[4];
    for (int x = 0; x < g.dim[0]; x++)
        for (int y = 0; y < g.dim[1]; y++)
            for (int z = 0; z < g.dim[2]; z++) {
                std::fill(aff.begin(), aff.end(), 0.0);
                std::fill(chg.begin(), chg.end(), 0.0);
                V3 probe = g.index_to_argument(x, y, z);
                const std::vector<int>& poss = cl.get(probe);
                for (int i : poss) {
                    int t1 = c.rec.type[i];
                    double r2 = dist2(c.rec.xyz[i], probe);
                    if (r2 <= c.tab.cutoff_sqr) {
                        for (size_t j = 0; j < needed.size(); j++) {
                            table_eval_fast(c.tab, t1, needed[j], r2, val);
                            if (charged) {
                                aff[j] += val[0] + val[1] * std::fabs(c.rec.charge[i]);
                                chg[j] += val[2] + val[3] * c.rec.charge[i];
                            } else {
                                aff[j] += val[0];
                            }
                        }
                    }
                }
                size_t idx = (size_t)x + (size_t)g.dim[0] * ((size_t)y + (size_t)g.dim[1] * z);
                // the user grid is evaluated at the point's index coordinates, as
                // cache::populate does (cache.cpp:204-205)
                const double u = c.ug.init ? evaluate_aux(c.ug.geom, c.ug.data, V3(x, y, z), c.ug.slope, 1000, nullptr)
                                           : 0.0;
                for (size_t j = 0; j < needed.size(); j++) {
                    c.grids[needed[j]].data[idx] = aff[j];
                    if (c.ug.init) c.grids[needed[j]].data[idx] += u;
                    if (charged) c.grids[needed[j]].chargedata[idx] = chg[j];
                }
            }
    for (int t : needed) c.built[t] = true;
}

// ---- grid::evaluate_aux (grid.cpp:111-236) -----------------------------------
static double evaluate_aux(const GridGeom& G, const std::vector<double>& D, const V3& loc, double slope, double v,
                           V3* deriv) {
    V3 s(0, 0, 0);
    for (int i = 0; i < 3; i++) s[i] = (loc[i] - G.init[i]) * G.factor[i];
    V3 miss(0, 0, 0);
    int region[3];
    size_t a[3];
    for (int i = 0; i < 3; i++) {
        if (s[i] < 0) {
            miss[i] = -s[i]; region[i] = -1; a[i] = 0; s[i] = 0;
        } else if (s[i] >= G.dim_fl_minus_1[i]) {
            miss[i] = s[i] - G.dim_fl_minus_1[i]; region[i] = 1; a[i] = G.dim[i] - 2; s[i] = 1;
        } else {
            region[i] = 0; a[i] = (size_t)s[i]; s[i] -= a[i];
        }
    }
    const double penalty = slope * dot(miss, G.factor_inv);
    const size_t d0 = G.dim[0], d1 = G.dim[1];
    auto at = [&](size_t x, size_t y, size_t z) { return D[x + d0 * (y + d1 * z)]; };
    const size_t x0 = a[0], y0 = a[1], z0 = a[2], x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
    const double f000 = at(x0, y0, z0), f100 = at(x1, y0, z0), f010 = at(x0, y1, z0), f110 = at(x1, y1, z0),
                 f001 = at(x0, y0, z1), f101 = at(x1, y0, z1), f011 = at(x0, y1, z1), f111 = at(x1, y1, z1);
    const double x = s[0], y = s[1], z = s[2];
    const double mx = 1 - x, my = 1 - y, mz = 1 - z;
    double f = f000 * mx * my * mz + f100 * x * my * mz + f010 * mx * y * mz + f110 * x * y * mz +
               f001 * mx * my * z + f101 * x * my * z + f011 * mx * y * z + f111 * x * y * z;
    if (deriv) {
        const double x_g = f000 * (-1) * my * mz + f100 * 1 * my * mz + f010 * (-1) * y * mz + f110 * 1 * y * mz +
                           f001 * (-1) * my * z + f101 * 1 * my * z + f011 * (-1) * y * z + f111 * 1 * y * z;
        const double y_g = f000 * mx * (-1) * mz + f100 * x * (-1) * mz + f010 * mx * 1 * mz + f110 * x * 1 * mz +
                           f001 * mx * (-1) * z + f101 * x * (-1) * z + f011 * mx * 1 * z + f111 * x * 1 * z;
        const double z_g = f000 * mx * my * (-1) + f100 * x * my * (-1) + f010 * mx * y * (-1) + f110 * x * y * (-1) +
                           f001 * mx * my * 1 + f101 * x * my * 1 + f011 * mx * y * 1 + f111 * x * y * 1;
        V3 grad(x_g, y_g, z_g);
        curl(f, grad, v);
        for (int i = 0; i < 3; i++) {
            double ge = region[i] == 0 ? grad[i] : 0;
            (*deriv)[i] = G.factor[i] * ge + slope * region[i];
        }
        return f + penalty;
    }
    curl(f, v);
    return f + penalty;
}

// ---- model::set (model.cpp:837-841 -> tree.h set_conf) ---------------------
void model_set(const Model& m, const double* conf, State& s) {
    for (int f = 0; f < m.num_frames; f++) {
        const int k = m.fkind[f];
        if (k == SG_FRAME_RIGID) {  // rigid_body::set_conf (tree.h:108-113)
            const double* c = conf + m.fconf[f];
            s.origin[f] = V3(c[0], c[1], c[2]);
            s.q[f] = Q{c[3], c[4], c[5], c[6]};
        } else if (k == SG_FRAME_SEGMENT) {  // segment::set_conf (tree.h:159-170)
            const int p = m.fparent[f];
            const double torsion = conf[m.fconf[f]];
            s.origin[f] = s.origin[p] + mul(s.rot[p], m.forigin[f]);
            s.axis[f] = mul(s.rot[p], m.faxis[f]);
            Q t = qmul(angle_to_quaternion(s.axis[f], torsion), s.q[p]);
            quaternion_normalize_approx(t);
            s.q[f] = t;
        } else {  // first_segment::set_conf (tree.h:192-195)
            const double torsion = conf[m.fconf[f]];
            s.origin[f] = m.forigin[f];
            s.axis[f] = m.faxis[f];
            s.q[f] = angle_to_quaternion(s.axis[f], torsion);
        }
        s.rot[f] = quaternion_to_r3(s.q[f]);
        for (int i = m.fbegin[f]; i < m.fend[f]; i++) s.coords[i] = s.origin[f] + mul(s.rot[f], m.local[i]);
    }
}

static void state_init(const Model& m, State& s) {
    s.coords = m.lab;
    s.minus_forces.assign(m.num_atoms, V3(0, 0, 0));
    s.origin = m.finit;
    s.axis.assign(m.num_frames, V3(0, 0, 0));
    for (int f = 0; f < m.num_frames; f++)
        if (m.fkind[f] == SG_FRAME_FIRST_SEGMENT) s.axis[f] = m.faxis[f];
    s.q.assign(m.num_frames, Q{1, 0, 0, 0});
    s.rot.assign(m.num_frames, quaternion_to_r3(Q{1, 0, 0, 0}));
}

// model::eval_interacting_pairs_deriv (model.cpp:904-928)
static double pairs_deriv(const Tables& T, const Model& m, int begin, int end, double v, State& s) {
    double e = 0;
    for (int k = begin; k < end; k++) {
        const int a = m.pairs[k][0], b = m.pairs[k][1];
        V3 r = s.coords[b] - s.coords[a];
        double r2 = sqrv(r);
        if (r2 < T.cutoff_sqr) {
            double pe, dor;
            table_eval_deriv(T, m.type[a], m.charge[a], m.type[b], m.charge[b], r2, pe, dor);
            V3 force = dor * r;
            curl(pe, force, v);
            e += pe;
            subfrom(s.minus_forces[a], force);
            addto(s.minus_forces[b], force);
        }
    }
    return e;
}

// tree.h:214-243 + heterotree::derivative, frames visited children-first
static void derivative(const Model& m, State& s, double* g) {
    std::vector<V3> F(m.num_frames), T(m.num_frames);
    for (int f = m.num_frames - 1; f >= 0; f--) {
        V3 force(0, 0, 0), torque(0, 0, 0);
        for (int i = m.fbegin[f]; i < m.fend[f]; i++) {  // atom_frame::sum_force_and_torque
            addto(force, s.minus_forces[i]);
            addto(torque, cross(s.coords[i] - s.origin[f], s.minus_forces[i]));
        }
        for (int c : m.children[f]) {  // branches_derivative
            addto(force, F[c]);
            V3 r = s.origin[c] - s.origin[f];
            addto(torque, cross(r, F[c]) + T[c]);
        }
        F[f] = force;
        T[f] = torque;
        if (m.fkind[f] == SG_FRAME_RIGID) {
            double* d = g + m.fdof[f];
            d[0] = force[0]; d[1] = force[1]; d[2] = force[2];
            d[3] = torque[0]; d[4] = torque[1]; d[5] = torque[2];
        } else {
            g[m.fdof[f]] = dot(torque, s.axis[f]);
        }
    }
}

// grid::evaluate (grid.cpp:27-46) + cache::eval_deriv (cache.cpp:69-90)
double eval_deriv(const Ctx& c, const Model& m, const double* conf, const double v[3], double slope, State& s,
                  double* g, uint64_t* evals) {
    if (evals) ++*evals;
    model_set(m, conf, s);
    double e = 0;
    for (int i = 0; i < m.num_movable; i++) {
        const int t = m.type[i];
        if (t >= SG_NUM_TYPES || is_h(t)) { s.minus_forces[i] = V3(0, 0, 0); continue; }
        const Grid& gr = c.grids[t];
        if (!c.built[t]) throw std::runtime_error("grid map missing for a ligand atom type");
        V3 deriv;
        double ret = evaluate_aux(c.geom, gr.data, s.coords[i], slope, v[1], &deriv);
        if (m.charge[i] != 0 && !gr.chargedata.empty()) {
            V3 cd(0, 0, 0);
            ret += m.charge[i] * evaluate_aux(c.geom, gr.chargedata, s.coords[i], slope, v[1], &cd);
            addto(deriv, m.charge[i] * cd);
        }
        e += ret;
        s.minus_forces[i] = deriv;
    }
    e += pairs_deriv(c.tab, m, 0, m.num_other_pairs, v[2], s);
    int start = m.num_other_pairs;
    for (int l = 0; l < m.num_ligands; l++) {
        e += pairs_deriv(c.tab, m, start, m.lig_pair_end[l], v[0], s);
        start = m.lig_pair_end[l];
    }
    derivative(m, s, g);
    return e;
}

// non_cache::eval_deriv (non_cache.cpp:109-191) + the rest of model::eval_deriv
// box: the job's own box (minimize_batch, gpu_docking.h:96-107); null: the receptor's
double eval_direct_deriv(Ctx& c, CellLists& cl, const Model& m, const double* conf, const double v[3], double slope,
                         State& s, double* g, bool* overlap, const sg_grid_dims* box) {
    model_set(m, conf, s);
    const sg_grid_dims& gd = box ? *box : c.geom.gd;
    double e = 0;
    for (int i = 0; i < m.num_movable; i++) {
        double this_e = 0, oob = 0;
        V3 deriv(0, 0, 0), oobd(0, 0, 0);
        const int t = m.type[i];
        if (t >= SG_NUM_TYPES || is_h(t)) { s.minus_forces[i] = V3(0, 0, 0); continue; }
        const V3 a = s.coords[i];
        V3 adj = a;
        for (int j = 0; j < 3; j++) {
            if (gd.n[j] > 0) {
                if (a[j] < gd.begin[j]) { adj[j] = gd.begin[j]; oobd[j] = -1; oob += std::fabs(a[j] - gd.begin[j]); }
                else if (a[j] > gd.end[j]) { adj[j] = gd.end[j]; oobd[j] = 1; oob += std::fabs(a[j] - gd.end[j]); }
            }
        }
        oob *= slope;
        oobd[0] *= slope; oobd[1] *= slope; oobd[2] *= slope;
        const std::vector<int>& poss = cl.get(adj);
        for (int j : poss) {
            V3 rba = adj - c.rec.xyz[j];
            double r2 = sqrv(rba);
            if (r2 < c.tab.cutoff_sqr) {
                if (r2 < EPS) { if (overlap) *overlap = true; throw std::runtime_error("Ligand atom exactly overlaps receptor atom."); }
                double pe, dor;
                table_eval_deriv(c.tab, t, m.charge[i], c.rec.type[j], c.rec.charge[j], r2, pe, dor);
                this_e += pe;
                addto(deriv, dor * rba);
            }
        }
        if (c.ug.init) {  // non_cache.cpp:180-184: at the atom's own coordinates
            V3 ugd(0, 0, 0);
            this_e += evaluate_aux(c.ug.geom, c.ug.data, a, slope, 1000, &ugd);
            deriv = deriv + ugd;
        }
        curl(this_e, deriv, v[1]);
        s.minus_forces[i] = deriv + oobd;
        e += this_e + oob;
    }
    e += pairs_deriv(c.tab, m, 0, m.num_other_pairs, v[2], s);
    int start = m.num_other_pairs;
    for (int l = 0; l < m.num_ligands; l++) {
        e += pairs_deriv(c.tab, m, start, m.lig_pair_end[l], v[0], s);
        start = m.lig_pair_end[l];
    }
    derivative(m, s, g);
    return e;
}

// non_cache::within (non_cache.cpp:93-107)
static bool within(const Ctx& c, const Model& m, const State& s, const sg_grid_dims* box = nullptr,
                   double margin = 0.0001) {
    const sg_grid_dims& gd = box ? *box : c.geom.gd;
    for (int i = 0; i < m.num_movable; i++) {
        if (is_h(m.type[i])) continue;
        for (int j = 0; j < 3; j++)
            if (gd.n[j] > 0)
                if (s.coords[i][j] < gd.begin[j] - margin || s.coords[i][j] > gd.end[j] + margin) return false;
    }
    return true;
}

// ---- conf algebra (conf.h) --------------------------------------------------
// conf::increment (conf.h:316-320 -> rigid_conf::increment :98-103, torsions_increment :44-49)
static void conf_increment(const Model& m, double* x, const double* p, double alpha) {
    for (const Block& b : m.blocks) {
        double* c = x + b.conf_off;
        const double* d = p + b.dof_off;
        int nt0 = 0;
        if (b.rigid) {
            V3 dp = alpha * V3(d[0], d[1], d[2]);
            c[0] += dp[0]; c[1] += dp[1]; c[2] += dp[2];
            V3 rot = alpha * V3(d[3], d[4], d[5]);
            Q q{c[3], c[4], c[5], c[6]};
            quaternion_increment(q, rot);
            c[3] = q.a; c[4] = q.b; c[5] = q.c; c[6] = q.d;
            c += 7; d += 6;
        }
        (void)nt0;
        for (int k = 0; k < b.ntors; k++) {
            c[k] += normalized_angle(alpha * d[k]);
            normalize_angle(c[k]);
        }
    }
}
// conf::operator()(index) (conf.h:380-404)
static double conf_value(const Model& m, const double* x, int index) {
    for (const Block& b : m.blocks) {
        const double* c = x + b.conf_off;
        if (b.rigid) {
            if (index < 3) return c[index];
            index -= 3;
            if (index < 3) return quaternion_to_angle(Q{c[3], c[4], c[5], c[6]})[index];
            index -= 3;
            c += 7;
        }
        if (index < b.ntors) return c[index];
        index -= b.ntors;
    }
    return 0;
}

// ---- BFGS (bfgs.h:30-282) ---------------------------------------------------
struct Tri {  // triangular_matrix<fl>
    int n;
    std::vector<double> d;
    Tri(int n_) : n(n_), d((size_t)n_ * (n_ + 1) / 2, 0) {}
    double& at(int i, int j) { return d[i + j * (j + 1) / 2]; }
    double perm(int i, int j) const { return i < j ? d[i + j * (j + 1) / 2] : d[j + i * (i + 1) / 2]; }
};
static void minus_mat_vec(const Tri& h, const double* in, double* out) {
    for (int i = 0; i < h.n; i++) {
        double sum = 0;
        for (int j = 0; j < h.n; j++) sum += h.perm(i, j) * in[j];
        out[i] = -sum;
    }
}
static double sprod(const double* a, const double* b, int n) {
    double t = 0;
    for (int i = 0; i < n; i++) t += a[i] * b[i];
    return t;
}
static bool bfgs_update(Tri& h, const double* p, const double* y, double alpha) {
    const int n = h.n;
    const double yp = sprod(y, p, n);
    if (alpha * yp < EPS) return false;
    std::vector<double> mhy(n);
    minus_mat_vec(h, y, mhy.data());
    const double yhy = -sprod(y, mhy.data(), n);
    const double r = 1 / (alpha * yp);
    for (int i = 0; i < n; i++)
        for (int j = i; j < n; j++)
            h.at(i, j) += alpha * r * (mhy[i] * p[j] + mhy[j] * p[i]) + +alpha * alpha * (r * r * yhy + r) * p[i] * p[j];
    return true;
}

template <typename F>
static double fast_line_search(F& f, int n, const Model& m, const std::vector<double>& x, const std::vector<double>& g,
                               double f0, const std::vector<double>& p, std::vector<double>& x_new,
                               std::vector<double>& g_new, double& f1) {
    const double c0 = 0.0001;
    const double mult = 0.5;
    double alpha = 1;
    const double pg = sprod(p.data(), g.data(), n);
    for (unsigned trial = 0; trial < 10; trial++) {
        x_new = x;
        conf_increment(m, x_new.data(), p.data(), alpha);
        f1 = f(x_new.data(), g_new.data());
        if (f1 - f0 < c0 * alpha * pg) break;
        alpha *= mult;
    }
    return alpha;
}

template <typename F>
static double accurate_line_search(F& f, int n, const Model& m, const std::vector<double>& x,
                                   const std::vector<double>& g, double f0, const std::vector<double>& p,
                                   std::vector<double>& x_new, std::vector<double>& g_new, double& f1) {
    double a, alpha, alpha2 = 0, alamin, b, disc, f2 = 0;
    double rhs1, rhs2, slope = 0, temp, test, tmplam = 0;
    const double ALF = 1.0e-4, FIRST = 1.0;
    slope = sprod(g.data(), p.data(), n);
    if (slope >= 0) {
        x_new = x;
        std::fill(g_new.begin(), g_new.end(), 0.0);
        return 0;
    }
    test = 0;
    for (int i = 0; i < n; i++) {
        temp = std::fabs(p[i]) / std::max(std::fabs(conf_value(m, x.data(), i)), 1.0);
        if (temp > test) test = temp;
    }
    alamin = EPS / test;
    alpha = FIRST;
    for (;;) {
        x_new = x;
        conf_increment(m, x_new.data(), p.data(), alpha);
        f1 = f(x_new.data(), g_new.data());
        if (alpha < alamin) {
            x_new = x;
            std::fill(g_new.begin(), g_new.end(), 0.0);
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
                if (a == 0.0) {
                    tmplam = -slope / (2.0 * b);
                } else {
                    disc = b * b - 3.0 * a * slope;
                    if (disc < 0) tmplam = 0.5 * alpha;
                    else if (b <= 0) tmplam = (-b + std::sqrt(disc)) / (3.0 * a);
                    else tmplam = -slope / (b + std::sqrt(disc));
                }
                if (tmplam > .5 * alpha) tmplam = .5 * alpha;
            }
        }
        alpha2 = alpha;
        f2 = f1;
        alpha = std::max(tmplam, 0.1 * alpha);
    }
}

// ---- QuickVina 2 history (the reference's gpu_mc.cuh:144-264; not smina's search) ----
// A chain's last 5n visited points (n = dof) in change coordinates, their
// energies and the zero / positive signs of their gradients.
struct Visited {
    int n = 0, size = 0, next = 0;
    bool full = false;
    std::vector<double> x, f;
    std::vector<uint8_t> zero, pos;  // [5n][n]
    explicit Visited(int n_) : n(n_), x(5 * (size_t)n_ * n_), f(5 * n_), zero(5 * (size_t)n_ * n_), pos(5 * (size_t)n_ * n_) {}
};
// visited::add (gpu_mc.cuh:163-205)
static void visited_add(Visited& V, const Model& m, const double* x, double f, const double* g) {
    const int n = V.n, cap = 5 * n;
    int slot;
    if (!V.full) {
        slot = V.size++;
        if (V.size >= cap) { V.full = true; V.next = 0; }
    } else {
        slot = V.next;
        V.next = (V.next + 1) % cap;
    }
    V.f[slot] = f;
    for (int i = 0; i < n; i++) {
        V.zero[(size_t)slot * n + i] = g[i] == 0;
        V.pos[(size_t)slot * n + i] = g[i] > 0;
        V.x[(size_t)slot * n + i] = conf_value(m, x, i);
    }
}
// visited::interesting (gpu_mc.cuh:207-264): until the history is full every
// start is interesting; otherwise the nearest point passing the first-order
// check (lowest index on ties) must rank below 4n by distance
static bool visited_interesting(const Visited& V, const Model& m, const double* x, double f, const double* g) {
    const int n = V.n, cap = 5 * n;
    if (!V.full) return true;
    std::vector<double> now(n), dist(cap);
    for (int i = 0; i < n; i++) now[i] = conf_value(m, x, i);
    double best = MAXF;
    int besti = cap;
    for (int e = 0; e < cap; e++) {
        const double* xe = &V.x[(size_t)e * n];
        const bool newY = f - V.f[e] > 0;
        double d2 = 0;
        bool pass = true;
        for (int i = 0; i < n; i++) {
            const double dx = xe[i] - now[i];
            d2 += dx * dx;
            if (V.zero[(size_t)e * n + i] || g[i] == 0) continue;
            const bool nowPos = g[i] > 0;
            if (nowPos != (V.pos[(size_t)e * n + i] != 0)) continue;
            const bool newX = now[i] - xe[i] > 0;
            if (nowPos ^ newX ^ newY) pass = false;
        }
        dist[e] = d2;
        if (pass && d2 < best) { best = d2; besti = e; }
    }
    if (besti >= cap) return false;
    int ahead = 0;
    for (int e = 0; e < cap; e++) ahead += (dist[e] < best || (dist[e] == best && e < besti));
    return ahead < 4 * n;
}

template <typename F>
double bfgs(F& f, const Model& m, std::vector<double>& x, std::vector<double>& g, const MinParams& mp,
            Visited* vis = nullptr) {
    const int n = m.dof;
    Tri h(n);
    for (int i = 0; i < n; i++) h.at(i, i) = 1;
    std::vector<double> g_new(g), x_new(x);
    double f0 = f(x.data(), g.data());
    if (vis) {  // the reference's bfgs() with a history (gpu_mc.cuh:459-465)
        if (!visited_interesting(*vis, m, x.data(), f0, g.data())) return f0;
        visited_add(*vis, m, x.data(), f0, g.data());
    }
    const double f_orig = f0;
    std::vector<double> g_orig(g), x_orig(x), p(g), y(n);
    for (unsigned step = 0; step < (unsigned)mp.maxiters; step++) {
        minus_mat_vec(h, g.data(), p.data());
        double f1 = 0, alpha;
        if (mp.accurate_line)
            alpha = accurate_line_search(f, n, m, x, g, f0, p, x_new, g_new, f1);
        else
            alpha = fast_line_search(f, n, m, x, g, f0, p, x_new, g_new, f1);
        if (alpha == 0) break;
        for (int i = 0; i < n; i++) y[i] = g_new[i];
        for (int i = 0; i < n; i++) y[i] -= g[i];
        double prevf0 = f0;
        f0 = f1;
        x = x_new;
        if (mp.early_term) {
            double diff = prevf0 - f0;
            if (std::fabs(diff) < 1e-5) break;
        }
        g = g_new;
        double gn = sprod(g.data(), g.data(), n);
        if (!(gn >= 1e-4)) break;
        if (step == 0) {
            const double yy = sprod(y.data(), y.data(), n);
            if (std::fabs(yy) > EPS) {
                double d = alpha * sprod(y.data(), p.data(), n) / yy;
                for (int i = 0; i < n; i++) h.at(i, i) = d;
            }
        }
        bfgs_update(h, p.data(), y.data(), alpha);
        if (vis) visited_add(*vis, m, x.data(), f0, g.data());
    }
    if (!(f0 <= f_orig)) {
        f0 = f_orig;
        x = x_orig;
        g = g_orig;
    }
    return f0;
}

// ---- Monte Carlo (monte_carlo.cpp:95-130, mutate.cpp:35-63) ----------------
// random.cpp:63-74
static V3 random_inside_sphere(MT& g) {
    for (;;) {
        double r1 = random_fl(-1, 1, g), r2 = random_fl(-1, 1, g), r3 = random_fl(-1, 1, g);
        V3 t(r1, r2, r3);
        if (sqrv(t) < 1) return t;
    }
}
// model.cpp:868-883
static double gyration_radius(const Model& m, const State& s, int l) {
    double acc = 0;
    unsigned counter = 0;
    const int root = m.lig_root[l];
    for (int i = m.lig_begin[l]; i < m.lig_end[l]; i++)
        if (!is_h(m.type[i])) {
            acc += dist2(s.coords[i], s.origin[root]);
            ++counter;
        }
    return counter > 0 ? std::sqrt(acc / counter) : 0;
}
static void mutate_conf(const Model& m, const State& s, double* c, double amplitude, MT& g) {
    int num = 0;
    for (const Block& b : m.blocks) num += (b.rigid ? 2 : 0) + b.ntors;
    if (num == 0) return;
    int which = random_int(0, num - 1, g);
    int lig = 0;
    for (const Block& b : m.blocks) {
        double* x = c + b.conf_off;
        if (b.rigid) {
            if (which == 0) {
                V3 d = amplitude * random_inside_sphere(g);
                x[0] += d[0]; x[1] += d[1]; x[2] += d[2];
                return;
            }
            --which;
            if (which == 0) {
                double gr = gyration_radius(m, s, lig);
                if (gr > EPS) {
                    V3 rot = amplitude / gr * random_inside_sphere(g);
                    Q q{x[3], x[4], x[5], x[6]};
                    quaternion_increment(q, rot);
                    x[3] = q.a; x[4] = q.b; x[5] = q.c; x[6] = q.d;
                }
                return;
            }
            --which;
            x += 7;
            lig++;
        }
        if (which < b.ntors) { x[which] = random_fl(-PI, PI, g); return; }
        which -= b.ntors;
    }
}
static bool metropolis_accept(double old_f, double new_f, double temperature, MT& g) {
    if (new_f < old_f) return true;
    const double p = pm_exp((old_f - new_f) / temperature);
    return random_fl(0, 1, g) < p;
}

// coords.cpp:25-58
static double rmsd_upper_bound(const std::vector<V3>& a, const std::vector<V3>& b) {
    double acc = 0;
    for (size_t i = 0; i < a.size(); i++) acc += dist2(a[i], b[i]);
    return a.size() > 0 ? std::sqrt(acc / a.size()) : 0;
}
static void sort_container(Container& out) {  // ptr_vector::sort by e (stable)
    std::stable_sort(out.v.begin(), out.v.end(), [](const Out& a, const Out& b) { return a.e < b.e; });
}
void add_to_output_container(Container& out, const Out& t, double min_rmsd, int max_size) {
    size_t ci = out.v.size();
    double cr = MAXF;
    for (size_t i = 0; i < out.v.size(); i++) {
        double res = rmsd_upper_bound(t.coords, out.v[i].coords);
        if (i == 0 || res < cr) { ci = i; cr = res; }
    }
    if (ci < out.v.size() && cr < min_rmsd) {
        if (t.e < out.v[ci].e) out.v[ci] = t;
    } else {
        if ((int)out.v.size() < max_size) out.v.push_back(t);
        else if (!out.v.empty() && t.e < out.v.back().e) out.v.back() = t;
    }
    sort_container(out);
}

static std::vector<V3> heavy_coords(const Model& m, const State& s) {
    std::vector<V3> h;
    h.reserve(m.heavy.size());
    for (int i : m.heavy) h.push_back(s.coords[i]);
    return h;
}

struct CacheFn {  // quasi_newton_aux (quasi_newton.cpp:25-35) over the cache
    const Ctx* c; const Model* m; State* s; double v[3]; double slope; uint64_t* evals;
    double operator()(const double* x, double* g) { return eval_deriv(*c, *m, x, v, slope, *s, g, evals); }
};

void mc_chain(const Ctx& c, const Model& m, const sg_mc_params& P, const double* conf0, MT& gen, unsigned steps,
              Container& out, uint64_t* evals) {
    State s;
    state_init(m, s);
    MinParams mp{P.maxiters, P.accurate_line, P.early_term};
    CacheFn hunt{&c, &m, &s, {P.hunt_cap[0], P.hunt_cap[1], P.hunt_cap[2]}, P.cache_slope, evals};
    CacheFn auth{&c, &m, &s, {P.authentic_v[0], P.authentic_v[1], P.authentic_v[2]}, P.cache_slope, evals};
    Out tmp;
    tmp.c.assign(conf0, conf0 + m.conf_size);
    tmp.e = 0;
    std::vector<double> g(m.dof, 0.0);
    double best_e = MAXF;
    std::unique_ptr<Visited> vis;  // MCParams::visited: QuickVina 2's history (dof <= 64)
    if (P.visited && m.dof <= 64) vis.reset(new Visited(m.dof));
    for (unsigned step = 0; step < steps; step++) {
        Out cand = tmp;
        mutate_conf(m, s, cand.c.data(), P.mutation_amplitude, gen);
        cand.e = bfgs(hunt, m, cand.c, g, mp, vis.get());
        if (step == 0 || metropolis_accept(tmp.e, cand.e, P.temperature, gen)) {
            tmp = cand;
            model_set(m, tmp.c.data(), s);
            if (tmp.e < best_e || (int)out.v.size() < P.num_saved_mins) {
                tmp.e = bfgs(auth, m, tmp.c, g, mp, vis.get());
                model_set(m, tmp.c.data(), s);
                tmp.coords = heavy_coords(m, s);
                add_to_output_container(out, tmp, P.min_rmsd, P.num_saved_mins);
                if (tmp.e < best_e) best_e = tmp.e;
            }
        }
    }
}

struct DirectFn {
    Ctx* c; CellLists* cl; const Model* m; State* s; double v[3]; double slope; const sg_grid_dims* box;
    double operator()(const double* x, double* g) {
        return eval_direct_deriv(*c, *cl, *m, x, v, slope, *s, g, nullptr, box);
    }
};

// refine_structure (main.cpp:165-190)
void refine(Ctx& c, const Model& m, double* conf, const double cap[3], const MinParams& mp, double& e_out,
            std::vector<V3>& coords_out, const sg_grid_dims* box) {
    CellLists cl;
    cl.full_cells = c.full_cells;
    cl.init(c.rec, c.tab.cutoff_sqr, c.geom.gd);
    State s;
    state_init(m, s);
    std::vector<double> x(conf, conf + m.conf_size), g(m.dof, 0.0);
    double slope = 10;
    double e = 0;
    for (int p = 0; p < 5; p++) {
        DirectFn fn{&c, &cl, &m, &s, {cap[0], cap[1], cap[2]}, slope, box};
        e = bfgs(fn, m, x, g, mp);
        model_set(m, x.data(), s);
        if (within(c, m, s, box)) break;
        slope *= 10;
    }
    coords_out = heavy_coords(m, s);
    if (!within(c, m, s, box)) e = MAXF;
    e_out = e;
    std::copy(x.begin(), x.end(), conf);
}

double bfgs_cache(const Ctx& c, const Model& m, std::vector<double>& x, const double v[3], double slope,
                  const MinParams& mp, uint64_t* evals) {
    State s;
    state_init(m, s);
    CacheFn fn{&c, &m, &s, {v[0], v[1], v[2]}, slope, evals};
    std::vector<double> g(m.dof, 0.0);
    return bfgs(fn, m, x, g, mp);
}

void state_for_eval(const Model& m, State& s) { state_init(m, s); }


// ---- final rescoring energies (finish_docking, main.cpp:257-282) -----------------------------
// precalculate_linear::eval (precalculate.h:75-83,103-108,191-203) with
// result_components::eval (result_components.h:75-81): the fast table at
// sz(factor r2); for t1 > t2 the (t2, t1) components with A and B swapped
static double table_eval_fast(const Tables& T, int t1, double qa, int t2, double qb, double r2) {
    const double* c = &T.fast[((size_t)T.pair_index(t1, t2) * T.n + (size_t)(T.factor * r2)) * T.nc];
    double comp[4] = {c[0], 0, 0, 0};
    if (T.nc > 1) { comp[1] = c[1]; comp[2] = c[2]; comp[3] = c[3]; }
    if (t1 > t2) std::swap(comp[1], comp[2]);  // result_components::swapOrder
    return comp[0] + std::fabs(qa) * comp[1] + std::fabs(qb) * comp[2] + qa * qb * comp[3];
}

// model::eval_interacting_pairs (model.cpp:885-902)
static double pairs_energy(const Tables& T, const Model& m, int begin, int end, double v, const State& s) {
    double e = 0;
    for (int k = begin; k < end; k++) {
        const int a = m.pairs[k][0], b = m.pairs[k][1];
        const double r2 = sqrv(s.coords[a] - s.coords[b]);
        if (r2 < T.cutoff_sqr) {
            double tmp = table_eval_fast(T, m.type[a], m.charge[a], m.type[b], m.charge[b], r2);
            curl(tmp, v);
            e += tmp;
        }
    }
    return e;
}

static bool in_ligand(const Model& m, int i) {  // model::find_ligand(i) < ligands.size()
    for (int l = 0; l < m.num_ligands; l++)
        if (i >= m.lig_begin[l] && i < m.lig_end[l]) return true;
    return false;
}

// model::eval (model.cpp:945-967) with non_cache::eval (non_cache.cpp:34-91),
// and model::eval_intramolecular (model.cpp:1027-1079), at one conf
void score_pose(Ctx& c, const Model& m, const double* conf, const double v[3], double slope, double& e_out,
                double& intra_out, std::vector<V3>& coords_out) {
    CellLists cl;
    cl.full_cells = c.full_cells;
    cl.init(c.rec, c.tab.cutoff_sqr, c.geom.gd);
    State s;
    state_init(m, s);
    model_set(m, conf, s);
    const sg_grid_dims& gd = c.geom.gd;
    // non_cache::eval
    double e = 0;
    for (int i = 0; i < m.num_movable; i++) {
        const int t = m.type[i];
        if (t >= SG_NUM_TYPES || is_h(t)) continue;
        double this_e = 0, oob = 0;
        const V3 a = s.coords[i];
        V3 adj = a;
        for (int j = 0; j < 3; j++) {
            if (gd.n[j] > 0) {
                if (a[j] < gd.begin[j]) { adj[j] = gd.begin[j]; oob += std::fabs(a[j] - gd.begin[j]); }
                else if (a[j] > gd.end[j]) { adj[j] = gd.end[j]; oob += std::fabs(a[j] - gd.end[j]); }
            }
        }
        oob *= slope;
        for (int j : cl.get(adj)) {
            const double r2 = sqrv(adj - c.rec.xyz[j]);
            if (r2 < c.tab.cutoff_sqr) this_e += table_eval_fast(c.tab, t, m.charge[i], c.rec.type[j], c.rec.charge[j], r2);
        }
        curl(this_e, v[1]);
        e += this_e + oob;
    }
    // model::evale: + other pairs; model::eval: + each ligand's pairs
    e += pairs_energy(c.tab, m, 0, m.num_other_pairs, v[2], s);
    int start = m.num_other_pairs;
    for (int l = 0; l < m.num_ligands; l++) {
        e += pairs_energy(c.tab, m, start, m.lig_pair_end[l], v[0], s);
        start = m.lig_pair_end[l];
    }
    // model::eval_intramolecular
    double intra = 0;
    start = m.num_other_pairs;
    for (int l = 0; l < m.num_ligands; l++) {
        intra += pairs_energy(c.tab, m, start, m.lig_pair_end[l], v[0], s);
        start = m.lig_pair_end[l];
    }
    for (int i = 0; i < m.num_movable; i++) {  // flex-rigid
        if (in_ligand(m, i)) continue;
        const int t1 = m.type[i];
        if (t1 >= SG_NUM_TYPES) continue;
        for (size_t j = 0; j < c.rec.xyz.size(); j++) {
            const int t2 = c.rec.type[j];
            if (t2 >= SG_NUM_TYPES) continue;
            const double r2 = sqrv(s.coords[i] - c.rec.xyz[j]);
            if (r2 < c.tab.cutoff_sqr) {
                double this_e = table_eval_fast(c.tab, t1, m.charge[i], t2, c.rec.charge[j], r2);
                curl(this_e, v[1]);
                intra += this_e;
            }
        }
    }
    for (int k = 0; k < m.num_other_pairs; k++) {  // flex-flex
        const int a = m.pairs[k][0], b = m.pairs[k][1];
        if (in_ligand(m, a) || in_ligand(m, b)) continue;
        const double r2 = sqrv(s.coords[a] - s.coords[b]);
        if (r2 < c.tab.cutoff_sqr) {
            double this_e = table_eval_fast(c.tab, m.type[a], m.charge[a], m.type[b], m.charge[b], r2);
            curl(this_e, v[2]);
            intra += this_e;
        }
    }
    e_out = e;
    intra_out = intra;
    coords_out = heavy_coords(m, s);
}

}  // namespace orc
