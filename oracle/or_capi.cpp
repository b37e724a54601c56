/*
 * ORACLE (test infrastructure only): C entry points of the CPU restatement,
 * loaded by tests/ and by bench.py's CPU baseline through ctypes.  The
 * product never calls these.
 */
#include "or_core.h"
#include <atomic>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>

namespace orc {
void mc_chain(const Ctx& c, const Model& m, const sg_mc_params& P, const double* conf0, MT& gen, unsigned steps,
              Container& out, uint64_t* evals);
void refine(Ctx& c, const Model& m, double* conf, const double cap[3], const MinParams& mp, double& e_out,
            std::vector<V3>& coords_out, const sg_grid_dims* box = nullptr);
double bfgs_cache(const Ctx& c, const Model& m, std::vector<double>& x, const double v[3], double slope,
                  const MinParams& mp, uint64_t* evals);
void state_for_eval(const Model& m, State& s);
}  // namespace orc

using namespace orc;

struct or_ctx {
    Ctx c;
    std::string err;
};

static thread_local std::string g_err;

extern "C" {

or_ctx* or_create(void) {
    or_ctx* o = new or_ctx();
    o->c.grids.resize(SG_NUM_TYPES);
    o->c.built.assign(SG_NUM_TYPES, false);
    return o;
}
void or_destroy(or_ctx* o) { delete o; }
const char* or_last_error(or_ctx* o) { return o ? o->err.c_str() : g_err.c_str(); }

int or_set_tables(or_ctx* o, const sg_tables_desc* t) {
    o->c.tab.load(*t);
    return 0;
}

int or_set_receptor(or_ctx* o, const sg_receptor_desc* r, const sg_grid_dims* gd, int full_cells) {
    Receptor& R = o->c.rec;
    R.xyz.resize(r->num_atoms);
    R.type.assign(r->type, r->type + r->num_atoms);
    R.charge.assign(r->charge, r->charge + r->num_atoms);
    for (int i = 0; i < r->num_atoms; i++) R.xyz[i] = V3(r->coords[3 * i], r->coords[3 * i + 1], r->coords[3 * i + 2]);
    o->c.geom.init_from(*gd);
    o->c.built.assign(SG_NUM_TYPES, false);
    for (auto& g : o->c.grids) { g.data.clear(); g.chargedata.clear(); }
    o->c.has_receptor = true;
    o->c.full_cells = full_cells != 0;
    return 0;
}

/* A user grid (--user_grid) on the same footing as the receptor: added to
 * every map at the map point's index coordinates (cache.cpp:204-205, with
 * the cache's slope) and to the direct sum at each atom (non_cache.cpp:
 * 180-184).  data [(n0+1)(n1+1)(n2+1)], x fastest; NULL clears it.  Maps
 * built before are dropped. */
int or_set_user_grid(or_ctx* o, const sg_grid_dims* gd, const double* data, double cache_slope) {
    o->c.ug = UserGrid();
    if (gd && data) {
        o->c.ug.init = true;
        o->c.ug.geom.init_from(*gd);
        const size_t n = (size_t)(gd->n[0] + 1) * (gd->n[1] + 1) * (gd->n[2] + 1);
        o->c.ug.data.assign(data, data + n);
        o->c.ug.slope = cache_slope;
    }
    std::fill(o->c.built.begin(), o->c.built.end(), false);
    return 0;
}

int or_build_grids(or_ctx* o, const int* types, int n) {
    try {
        populate(o->c, types, n);
    } catch (std::exception& e) { o->err = e.what(); return 1; }
    return 0;
}

int or_get_grid(or_ctx* o, int type, double* data, double* chargedata) {
    if (type < 0 || type >= SG_NUM_TYPES || !o->c.built[type]) { o->err = "grid not built"; return 1; }
    const Grid& g = o->c.grids[type];
    std::memcpy(data, g.data.data(), g.data.size() * 8);
    if (chargedata && !g.chargedata.empty()) std::memcpy(chargedata, g.chargedata.data(), g.chargedata.size() * 8);
    return 0;
}

int or_eval(or_ctx* o, const sg_model_desc* md, int nconfs, const double* confs, const double v[3], double slope,
            double* out_e, double* out_g, double* out_coords) {
    try {
        Model m;
        m.load(*md);
        State s;
        state_for_eval(m, s);
        std::vector<double> g(m.dof);
        for (int k = 0; k < nconfs; k++) {
            double e = eval_deriv(o->c, m, confs + (size_t)k * m.conf_size, v, slope, s, g.data(), nullptr);
            out_e[k] = e;
            if (out_g) std::memcpy(out_g + (size_t)k * m.dof, g.data(), m.dof * 8);
            if (out_coords)
                for (int i = 0; i < m.num_movable; i++)
                    for (int j = 0; j < 3; j++) out_coords[((size_t)k * m.num_movable + i) * 3 + j] = s.coords[i][j];
        }
    } catch (std::exception& e) { o->err = e.what(); return 1; }
    return 0;
}

int or_eval_direct(or_ctx* o, const sg_model_desc* md, int nconfs, const double* confs, const double v[3],
                   double slope, double* out_e, double* out_g) {
    Model m;
    m.load(*md);
    State s;
    state_for_eval(m, s);
    CellLists cl;
    cl.full_cells = o->c.full_cells;
    cl.init(o->c.rec, o->c.tab.cutoff_sqr, o->c.geom.gd);
    std::vector<double> g(m.dof);
    for (int k = 0; k < nconfs; k++) {
        bool overlap = false;
        try {
            out_e[k] = eval_direct_deriv(o->c, cl, m, confs + (size_t)k * m.conf_size, v, slope, s, g.data(), &overlap);
        } catch (std::exception& e) {
            o->err = e.what();
            return overlap ? SG_ERR_OVERLAP : 1;
        }
        if (out_g) std::memcpy(out_g + (size_t)k * m.dof, g.data(), m.dof * 8);
    }
    return 0;
}

/* One BFGS (quasi_newton) per conf against the maps; confs updated in place. */
int or_bfgs(or_ctx* o, const sg_model_desc* md, int nconfs, double* confs, const double v[3], double slope,
            int maxiters, int accurate_line, int early_term, double* out_e) {
    try {
        Model m;
        m.load(*md);
        MinParams mp{maxiters, accurate_line, early_term};
        for (int k = 0; k < nconfs; k++) {
            std::vector<double> x(confs + (size_t)k * m.conf_size, confs + (size_t)(k + 1) * m.conf_size);
            out_e[k] = bfgs_cache(o->c, m, x, v, slope, mp, nullptr);
            std::memcpy(confs + (size_t)k * m.conf_size, x.data(), m.conf_size * 8);
        }
    } catch (std::exception& e) { o->err = e.what(); return 1; }
    return 0;
}

/* monte_carlo::operator() for each chain on `nthreads` host threads. */
int or_dock(or_ctx* o, const sg_model_desc* models, int nmodels, const sg_chain_input* chains, int nchains,
            const sg_mc_params* p, sg_chain_result* out, int nthreads) {
    std::vector<Model> ms(nmodels);
    for (int i = 0; i < nmodels; i++) ms[i].load(models[i]);
    std::atomic<int> next(0);
    std::atomic<int> failed(0);
    std::string errmsg;
    auto worker = [&]() {
        for (;;) {
            int k = next.fetch_add(1);
            if (k >= nchains) return;
            const sg_chain_input& ci = chains[k];
            const Model& m = ms[ci.model];
            MT gen;
            std::memcpy(gen.x, ci.mt, 624 * 4);
            gen.i = (int)ci.mt[624];
            Container c;
            uint64_t evals = 0;
            try {
                sg_mc_params pc = *p;  // a chain's own BFGS iteration count, if it has one
                if (ci.maxiters > 0) pc.maxiters = ci.maxiters;
                mc_chain(o->c, m, pc, ci.conf, gen, ci.num_steps, c, &evals);
            } catch (std::exception& e) {
                failed = 1;
                errmsg = e.what();
                return;
            }
            sg_chain_result& r = out[k];
            r.count = (int)c.v.size();
            r.evals = evals;
            const int H = (int)m.heavy.size();
            for (int j = 0; j < r.count; j++) {
                r.e[j] = c.v[j].e;
                std::memcpy(r.conf + (size_t)j * m.conf_size, c.v[j].c.data(), m.conf_size * 8);
                for (int a = 0; a < H; a++)
                    for (int d = 0; d < 3; d++) r.coords[((size_t)j * H + a) * 3 + d] = c.v[j].coords[a][d];
            }
        }
    };
    if (nthreads < 1) nthreads = 1;
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; t++) th.emplace_back(worker);
    for (auto& t : th) t.join();
    if (failed) { o->err = errmsg; return 1; }
    return 0;
}

/* merge_output_containers (parallel_mc.cpp:71-78): fold each chain's
 * container into one with min_rmsd, keeping max_size entries. Returns count. */
int or_merge(const sg_chain_result* chains, int nchains, int conf_size, int nheavy, double min_rmsd, int max_size,
             double* out_e, double* out_conf, double* out_coords) {
    Container merged;
    for (int k = 0; k < nchains; k++) {
        for (int j = 0; j < chains[k].count; j++) {
            Out t;
            t.e = chains[k].e[j];
            t.c.assign(chains[k].conf + (size_t)j * conf_size, chains[k].conf + (size_t)(j + 1) * conf_size);
            t.coords.resize(nheavy);
            for (int a = 0; a < nheavy; a++)
                t.coords[a] = V3(chains[k].coords[((size_t)j * nheavy + a) * 3], chains[k].coords[((size_t)j * nheavy + a) * 3 + 1],
                                 chains[k].coords[((size_t)j * nheavy + a) * 3 + 2]);
            add_to_output_container(merged, t, min_rmsd, max_size);
        }
    }
    for (size_t j = 0; j < merged.v.size(); j++) {
        out_e[j] = merged.v[j].e;
        std::memcpy(out_conf + j * conf_size, merged.v[j].c.data(), conf_size * 8);
        for (int a = 0; a < nheavy; a++)
            for (int d = 0; d < 3; d++) out_coords[(j * nheavy + a) * 3 + d] = merged.v[j].coords[a][d];
    }
    return (int)merged.v.size();
}

/* refine_structure for each pose (confs in/out). */
int or_refine(or_ctx* o, const sg_model_desc* models, const int* pose_model, int nposes, double* confs,
              const double cap[3], int maxiters, int accurate_line, int early_term, double* out_e,
              double* out_coords) {
    Model m;
    try {
        for (int k = 0; k < nposes; k++) {
            const sg_model_desc& md = models[pose_model[k]];
            m.load(md);
            std::vector<V3> hc;
            MinParams mp{maxiters, accurate_line, early_term};
            refine(o->c, m, confs + (size_t)k * m.conf_size, cap, mp, out_e[k], hc);
            if (out_coords)
                for (size_t a = 0; a < hc.size(); a++)
                    for (int d = 0; d < 3; d++) out_coords[((size_t)k * hc.size() + a) * 3 + d] = hc[a][d];
        }
    } catch (std::exception& e) {
        o->err = e.what();
        return std::string(e.what()).find("overlaps") != std::string::npos ? SG_ERR_OVERLAP : 1;
    }
    return 0;
}

/* minimize_batch (gpu_docking.h:96-107): refine_structure of each pose in
 * its own box (boxes: [n][6] lo xyz, hi xyz, or null for the receptor's)
 * with its own BFGS iteration count. */
int or_minimize(or_ctx* o, const sg_model_desc* models, const int* pose_model, int nposes, double* confs,
                int conf_stride, const double* boxes, const double cap[3], const int* maxiters, int accurate_line,
                int early_term, double* out_e, double* out_coords, int coord_stride) {
    Model m;
    try {
        for (int k = 0; k < nposes; k++) {
            m.load(models[pose_model[k]]);
            std::vector<V3> hc;
            MinParams mp{maxiters[k], accurate_line, early_term};
            sg_grid_dims gd = o->c.geom.gd;
            if (boxes)
                for (int d = 0; d < 3; d++) {
                    gd.begin[d] = boxes[6 * k + d];
                    gd.end[d] = boxes[6 * k + 3 + d];
                    gd.n[d] = 1;
                }
            refine(o->c, m, confs + (size_t)k * conf_stride, cap, mp, out_e[k], hc, boxes ? &gd : nullptr);
            if (out_coords)
                for (size_t a = 0; a < hc.size(); a++)
                    for (int d = 0; d < 3; d++) out_coords[((size_t)k * coord_stride + a) * 3 + d] = hc[a][d];
        }
    } catch (std::exception& e) {
        o->err = e.what();
        return std::string(e.what()).find("overlaps") != std::string::npos ? SG_ERR_OVERLAP : 1;
    }
    return 0;
}

/* finish_docking's rescoring energies per pose (model::eval on the direct
 * sum, model::eval_intramolecular), heavy-atom coords */
int or_score(or_ctx* o, const sg_model_desc* models, const int* pose_model, int nposes, const double* confs,
             int conf_stride, const double v[3], double slope, double* out_e, double* out_intra, double* out_coords,
             int coord_stride) {
    Model m;
    try {
        for (int k = 0; k < nposes; k++) {
            m.load(models[pose_model[k]]);
            std::vector<V3> hc;
            score_pose(o->c, m, confs + (size_t)k * conf_stride, v, slope, out_e[k], out_intra[k], hc);
            if (out_coords)
                for (size_t a = 0; a < hc.size(); a++)
                    for (int d = 0; d < 3; d++) out_coords[((size_t)k * coord_stride + a) * 3 + d] = hc[a][d];
        }
    } catch (std::exception& e) {
        o->err = e.what();
        return 1;
    }
    return 0;
}

/* quaternion and angle math (common.h:262-281, quaternion.cpp:42-139) on
 * the rows of in[7] / q0[4]; the layout of out[22] is the reference probe's
 * (oracle/ref_probe.cpp) */
void or_quat_probe(const double* in, const double* q0, double* out, int n) {
    for (int k = 0; k < n; k++) {
        const double* x = in + 7 * k;
        double* o = out + 22 * k;
        const V3 axis(x[0], x[1], x[2]), rot(x[4], x[5], x[6]);
        double ang = x[3];
        normalize_angle(ang);
        o[0] = ang;
        const Q a = angle_to_quaternion(axis, x[3]);
        const Q b = angle_to_quaternion(rot);
        Q c{q0[4 * k], q0[4 * k + 1], q0[4 * k + 2], q0[4 * k + 3]};
        const M3 m = quaternion_to_r3(c);
        quaternion_increment(c, rot);
        const Q qs[3] = {a, b, c};
        for (int j = 0; j < 3; j++) {
            o[1 + 4 * j] = qs[j].a; o[2 + 4 * j] = qs[j].b; o[3 + 4 * j] = qs[j].c; o[4 + 4 * j] = qs[j].d;
        }
        for (int j = 0; j < 9; j++) o[13 + j] = m.d[j];
    }
}

/* scalar math probes: fn 0 sin, 1 cos, 2 acos, 3 exp */
void or_pm_eval(int fn, const double* x, double* y, int n) {
    for (int i = 0; i < n; i++) {
        switch (fn) {
            case 0: y[i] = pm_sin(x[i]); break;
            case 1: y[i] = pm_cos(x[i]); break;
            case 2: y[i] = pm_acos(x[i]); break;
            default: y[i] = pm_exp(x[i]); break;
        }
    }
}

/* mt19937 probe: n raw outputs after seeding; then n uniform_real(a,b)
 * and n uniform_int(lo,hi) draws continuing the same stream */
void or_mt_probe(uint32_t seed, int n, uint32_t* raw, double a, double b, double* fl, int lo, int hi, int* in) {
    MT g;
    g.seed(seed);
    for (int i = 0; i < n; i++) raw[i] = g.next();
    for (int i = 0; i < n; i++) fl[i] = random_fl(a, b, g);
    for (int i = 0; i < n; i++) in[i] = random_int(lo, hi, g);
}

}  // extern "C"
