/*
 * ORACLE pinning harness (test infrastructure only; not part of the product).
 *
 * Built by the oracle Makefile's `ref` target into oracle/_ref/, from
 * this file plus the reference's own FP64 device library
 * (src/gpu/gpu_device.cu and src/gpu/gpu_kernels_f64.cu, compiled from the
 * reference tree with the reference's own flags: --fmad=false,
 * --expt-relaxed-constexpr, --default-stream per-thread).  Run on a GPU by
 * tests/golden/make_ref_golden.py, it records the reference's FP64 outputs
 * (grid maps, eval, direct eval, BFGS, Monte Carlo chains, refinement) on
 * synthetic inputs; CPU tests check the oracle against those records.
 *
 * The reference's GPU FP64 path is its validation path: it is built to
 * reproduce the CPU smina trajectories bit for bit (src/gpu/CMakeLists.txt:
 * smina_portable vs smina_portable --gpu --gpu_fp64), and its own tests hold
 * it to the CPU build (src/gpu/tests/gpu_eval_test.cpp,
 * src/gpu/tests/gpu_mc_test.cpp).
 *
 * The conversion from this project's descriptors to the reference's flat
 * structures, with its host-side index checks, is baseline/ref_gpu/flatten.h
 * (a restatement of the reference's src/gpu/gpu_flatten.cpp); nothing is
 * uploaded before those checks pass.
 */
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "gpu_kernels.h"
#include "gpu_flatten_data.h"
#include "../include/smina_b200.h"
#include "../baseline/ref_gpu/flatten.h"

using namespace gpusmina;

namespace {
std::string g_err;
}  // namespace

using namespace refflat;

struct refg_ctx {
    FlatTables ft;
    FlatGridGeometry geo;
    FlatReceptor rec_grid, rec_full;
    FlatUserGrid ug;
    double slope = 1e6;
    DeviceTables<double> tables;
    DeviceGrids<double> grids;
    DeviceReceptor<double> receptor;
    DeviceUserGrid<double> dug;
    InterContext<double> context(bool use_cache, double s) const {
        InterContext<double> ic = InterContext<double>();  // zeroed: no stale map pointers without the cache
        ic.use_cache = use_cache;
        if (use_cache) ic.grids = grids.dev;
        ic.rec = receptor.dev;
        ic.box = make_box<double>(geo);
        ic.ug = dug.dev;
        ic.slope = s;
        return ic;
    }
};

namespace {
std::vector<FlatModel> flatten_all(const sg_model_desc* models, int n) {
    need(models && n > 0, "models: none");
    std::vector<FlatModel> out;
    for (int i = 0; i < n; i++) {
        out.push_back(flatten(models[i]));
        check_model(out.back());
    }
    return out;
}

void upload_models(const std::vector<FlatModel>& fms, DeviceModels<double>& dm) {
    std::vector<const FlatModel*> ptrs;
    for (const FlatModel& f : fms) ptrs.push_back(&f);
    dm.upload(ptrs);
}
}  // namespace

extern "C" {

const char* refg_last_error(void) { return g_err.c_str(); }

/* Builds and checks the flat model on the host only (no device work). */
int refg_check_model(const sg_model_desc* m, int* out_counts) {
    try {
        FlatModel f = flatten(*m);
        check_model(f);
        if (out_counts) {
            out_counts[0] = int(f.frames.size());
            out_counts[1] = int(f.blocks.size());
            out_counts[2] = int(f.nbr.size());
            out_counts[3] = int(f.level_start.size()) - 1;
        }
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
    return 0;
}

/* Builds and checks both receptor cell lists on the host only; counts:
 * grid receptor atoms, grid cell entries, full receptor atoms, full cell
 * entries. */
int refg_check_receptor(const sg_tables_desc* t, const sg_receptor_desc* r, const sg_grid_dims* gd,
                        long long* out_counts) {
    try {
        const FlatGridGeometry geo = geometry(*gd);
        const FlatReceptor a = receptor_for_grid(*r, *gd, geo, t->cutoff_sqr);
        const FlatReceptor b = receptor_full(*r, t->cutoff_sqr);
        check_receptor(a);
        check_receptor(b);
        if (out_counts) {
            out_counts[0] = (long long)a.type.size();
            out_counts[1] = (long long)a.cell_atoms.size();
            out_counts[2] = (long long)b.type.size();
            out_counts[3] = (long long)b.cell_atoms.size();
        }
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
    return 0;
}

/* Uploads tables and receptor and builds the reference's FP64 grid maps
 * for `types` (DeviceGrids::build, cache::populate).  ug_dims / ug_data
 * (both NULL for none): a user grid over ug_dims, values x fastest, as
 * smina holds it after reading (FlatUserGrid, gpu_flatten.cpp:506-531). */
int refg_create(const sg_tables_desc* t, const sg_receptor_desc* r, const sg_grid_dims* gd, const int* types,
                int ntypes, double slope, const sg_grid_dims* ug_dims, const double* ug_data, refg_ctx** out) {
    refg_ctx* c = nullptr;
    try {
        need(t && r && gd && out && (ntypes == 0 || types), "create: null argument");
        need((ug_dims == nullptr) == (ug_data == nullptr), "create: user grid needs both dims and data");
        c = new refg_ctx;
        c->ft = tables(*t);
        c->geo = geometry(*gd);
        if (ug_dims) {
            const FlatGridGeometry g = geometry(*ug_dims);
            c->ug.initialized = true;
            c->ug.geom = g;
            for (int i = 0; i < 3; i++) {
                c->ug.geom.gd_begin[i] = c->ug.geom.gd_end[i] = 0;
                c->ug.geom.gd_enabled[i] = 0;
            }
            c->ug.data.assign(ug_data, ug_data + size_t(g.dim[0]) * g.dim[1] * g.dim[2]);
        }
        c->rec_grid = receptor_for_grid(*r, *gd, c->geo, t->cutoff_sqr);
        c->rec_full = receptor_full(*r, t->cutoff_sqr);
        check_receptor(c->rec_grid);
        check_receptor(c->rec_full);
        std::vector<int> tl;
        for (int i = 0; i < ntypes; i++) {
            need(usable(types[i]), "create: grid type out of range");
            tl.push_back(types[i]);
        }
        c->slope = slope;
        if (c->ug.initialized) c->dug.upload(c->ug);
        c->tables.upload(c->ft);
        c->receptor.upload(c->rec_full);
        c->grids.build(c->rec_grid, c->geo, c->ft, tl, c->ug, slope);
        *out = c;
    } catch (std::exception& e) {
        g_err = e.what();
        delete c;
        return 1;
    }
    return 0;
}

void refg_destroy(refg_ctx* c) { delete c; }

/* One grid map (npts = product of n + 1, x fastest); chargedata only with
 * charge-dependent tables. */
int refg_get_grid(refg_ctx* c, int type, double* data, double* chargedata) {
    try {
        need(type >= 0 && type < NUM_TYPES && c->grids.has(type), "grid: type not built");
        std::vector<double> d, cd;
        c->grids.download(type, d, cd);
        std::memcpy(data, d.data(), d.size() * sizeof(double));
        if (chargedata && !cd.empty()) std::memcpy(chargedata, cd.data(), cd.size() * sizeof(double));
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
    return 0;
}

/* model::eval_deriv of nconfs confs (eval_confs): use_cache 1 against the
 * grid maps with the cache slope, 0 against the receptor atoms (non_cache)
 * with `slope`.  coords: movable atoms [nconfs][num_movable][3] (may be
 * null).  Returns 2 when a ligand atom sat on a receptor atom. */
int refg_eval(refg_ctx* c, const sg_model_desc* m, int nconfs, const double* confs, const double v[3],
              int use_cache, double slope, double* out_e, double* out_g, double* out_coords) {
    try {
        std::vector<FlatModel> fms = flatten_all(m, 1);
        DeviceModels<double> dm;
        upload_models(fms, dm);
        std::vector<double> cv(confs, confs + size_t(nconfs) * m->conf_size), e, g, xyz;
        const bool ok = eval_confs<double>(dm, 0, c->tables, c->context(use_cache != 0, use_cache ? c->slope : slope),
                                           v, cv, e, g, out_coords ? &xyz : nullptr, 32);
        std::memcpy(out_e, e.data(), e.size() * sizeof(double));
        if (out_g) std::memcpy(out_g, g.data(), g.size() * sizeof(double));
        if (out_coords) std::memcpy(out_coords, xyz.data(), xyz.size() * sizeof(double));
        return ok ? 0 : 2;
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

/* quasi_newton on the grid maps (run_bfgs), confs updated in place. */
int refg_bfgs(refg_ctx* c, const sg_model_desc* m, int nconfs, double* confs, const double v[3], int maxiters,
              int accurate_line, int early_term, double* out_e) {
    try {
        std::vector<FlatModel> fms = flatten_all(m, 1);
        DeviceModels<double> dm;
        upload_models(fms, dm);
        std::vector<std::vector<double> > cv(nconfs);
        for (int k = 0; k < nconfs; k++)
            cv[k].assign(confs + size_t(k) * m->conf_size, confs + size_t(k + 1) * m->conf_size);
        std::vector<double> e;
        MinParams mp{unsigned(maxiters), accurate_line, early_term};
        const std::vector<int> model_of(nconfs, 0);
        const bool ok = run_bfgs<double>(dm, c->tables, c->context(true, c->slope), mp, v, model_of, cv, e, 32);
        for (int k = 0; k < nconfs; k++) {
            std::memcpy(confs + size_t(k) * m->conf_size, cv[k].data(), m->conf_size * sizeof(double));
            out_e[k] = e[k];
        }
        return ok ? 0 : 2;
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

/* monte_carlo::operator() per chain (run_monte_carlo, 32 threads per
 * chain), results written like sg_dock's: [count] energies, confs and heavy
 * atom coordinates of the chain's sorted output container. */
int refg_dock(refg_ctx* c, const sg_model_desc* models, int nmodels, const sg_chain_input* chains, int nchains,
              const sg_mc_params* p, sg_chain_result* out) {
    try {
        need(!p->visited, "dock: the history check is not pinned here");
        std::vector<FlatModel> fms = flatten_all(models, nmodels);
        DeviceModels<double> dm;
        upload_models(fms, dm);
        MCParams mp;
        mp.num_steps = p->num_steps;
        mp.temperature = p->temperature;
        mp.mutation_amplitude = p->mutation_amplitude;
        mp.min_rmsd = p->min_rmsd;
        mp.num_saved_mins = p->num_saved_mins;
        for (int k = 0; k < 3; k++) {
            mp.hunt_cap[k] = p->hunt_cap[k];
            mp.authentic_v[k] = p->authentic_v[k];
        }
        mp.min.maxiters = unsigned(p->maxiters);
        mp.min.accurate_line = p->accurate_line;
        mp.min.early_term = p->early_term;
        mp.visited = 0;
        std::vector<ChainInput> in(nchains);
        for (int k = 0; k < nchains; k++) {
            const sg_chain_input& ci = chains[k];
            need(ci.model >= 0 && ci.model < nmodels && ci.conf && ci.mt, "dock: bad chain input");
            need(ci.mt[624] <= 624, "dock: bad generator index");
            in[k].model = ci.model;
            in[k].conf.assign(ci.conf, ci.conf + models[ci.model].conf_size);
            std::memcpy(in[k].rng.x, ci.mt, sizeof(in[k].rng.x));
            in[k].rng.i = int(ci.mt[624]);
            in[k].num_steps = ci.num_steps;
            in[k].maxiters = ci.maxiters > 0 ? unsigned(ci.maxiters) : 0u;
            in[k].unit = 0;
        }
        std::vector<ChainResult> res;
        run_monte_carlo<double>(dm, c->tables, c->context(true, p->cache_slope), mp, in, res, nullptr, 32, nullptr,
                                nullptr);
        for (int k = 0; k < nchains; k++) {
            const FlatModel& fm = fms[chains[k].model];
            const ChainResult& r = res[k];
            const int cnt = int(r.e.size());
            need(cnt <= p->num_saved_mins, "dock: container larger than num_saved_mins");
            out[k].count = cnt;
            out[k].evals = 0;
            const size_t H = fm.heavy.size();
            for (int j = 0; j < cnt; j++) {
                out[k].e[j] = r.e[j];
                std::memcpy(out[k].conf + size_t(j) * fm.conf_size, r.conf[j].data(), fm.conf_size * sizeof(double));
                std::memcpy(out[k].coords + size_t(j) * 3 * H, r.coords[j].data(), 3 * H * sizeof(double));
            }
        }
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
    return 0;
}

/* refine_structure of each pose against the receptor atoms (run_refine,
 * non_cache with the slope schedule), confs updated in place; coords:
 * heavy atoms of each pose, packed with its model's heavy atom count. */
int refg_refine(refg_ctx* c, const sg_model_desc* models, int nmodels, const int* pose_model, int nposes,
                double* confs, const double cap[3], int maxiters, int accurate_line, int early_term, double* out_e,
                double* out_coords) {
    try {
        std::vector<FlatModel> fms = flatten_all(models, nmodels);
        DeviceModels<double> dm;
        upload_models(fms, dm);
        std::vector<int> model_of(pose_model, pose_model + nposes);
        std::vector<std::vector<double> > cv(nposes), xyz;
        size_t at = 0;
        for (int k = 0; k < nposes; k++) {
            need(model_of[k] >= 0 && model_of[k] < nmodels, "refine: bad pose model");
            const int cs = models[model_of[k]].conf_size;
            cv[k].assign(confs + at, confs + at + cs);
            at += cs;
        }
        std::vector<double> e;
        MinParams mp{unsigned(maxiters), accurate_line, early_term};
        const bool ok = run_refine<double>(dm, c->tables, c->context(false, 0.0), mp, cap, model_of, cv, e, xyz, 32);
        at = 0;
        size_t xat = 0;
        for (int k = 0; k < nposes; k++) {
            std::memcpy(confs + at, cv[k].data(), cv[k].size() * sizeof(double));
            at += cv[k].size();
            out_e[k] = e[k];
            if (out_coords) {
                std::memcpy(out_coords + xat, xyz[k].data(), xyz[k].size() * sizeof(double));
                xat += xyz[k].size();
            }
        }
        return ok ? 0 : 2;
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

}  // extern "C"
