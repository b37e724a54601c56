/*
 * The reference's own GPU search as a baseline on B200 (not part of the
 * product, and not a checker).
 *
 * Built by this directory's Makefile into baseline/_ref/, from this file
 * plus the reference's device library compiled from its own sources with its
 * own flags: src/gpu/gpu_device.cu (--fmad=false) and
 * src/gpu/gpu_kernels_f32.cu, i.e. the FP32 kernels its --gpu search runs.
 * bench.py --ref-gpu feeds it the same synthetic screen as this engine and
 * times the reference's run_monte_carlo (src/gpu/gpu_kernels.h:90-101,
 * gpu_kernels_impl.cuh:659-887) over every chain of every ligand at 32
 * threads per chain, the reference's throughput configuration for screens.
 * Its grid maps are built by the reference's DeviceGrids<float>::build.
 *
 * Inputs pass through baseline/ref_gpu/flatten.h, which converts them to the
 * reference's flat structures and checks every index the kernels read
 * before anything is uploaded.
 */
#include <chrono>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "gpu_kernels.h"
#include "flatten.h"

using namespace gpusmina;
using namespace refflat;

namespace {
std::string g_err;
}

struct refs_ctx {
    FlatTables ft;
    FlatGridGeometry geo;
    FlatReceptor rec_grid;
    FlatUserGrid ug;
    DeviceTables<float> tables;
    DeviceGrids<float> grids;
    DeviceUserGrid<float> dug;
    DeviceReceptor<float> receptor;  // empty: the search reads the maps only
};

extern "C" {

const char* refs_last_error(void) { return g_err.c_str(); }

/* Tables and the FP32 grid maps of `types` (cache::populate on the device,
 * sums in double, stored as float). */
int refs_create(const sg_tables_desc* t, const sg_receptor_desc* r, const sg_grid_dims* gd, const int* types,
                int ntypes, double slope, refs_ctx** out) {
    refs_ctx* c = nullptr;
    try {
        need(t && r && gd && out && ntypes > 0 && types, "create: bad arguments");
        c = new refs_ctx;
        c->ft = tables(*t);
        c->geo = geometry(*gd);
        c->rec_grid = receptor_for_grid(*r, *gd, c->geo, t->cutoff_sqr);
        check_receptor(c->rec_grid);
        std::vector<int> tl;
        for (int i = 0; i < ntypes; i++) {
            need(usable(types[i]), "create: grid type out of range");
            tl.push_back(types[i]);
        }
        c->tables.upload(c->ft);
        c->grids.build(c->rec_grid, c->geo, c->ft, tl, c->ug, slope);
        *out = c;
    } catch (std::exception& e) {
        g_err = e.what();
        delete c;
        return 1;
    }
    return 0;
}

void refs_destroy(refs_ctx* c) { delete c; }

/* run_monte_carlo<float> over every chain (results written like sg_dock's);
 * *seconds gets the wall time of that call (it returns when the search is
 * done and its results are on the host). */
int refs_dock(refs_ctx* c, const sg_model_desc* models, int nmodels, const sg_chain_input* chains, int nchains,
              const sg_mc_params* p, sg_chain_result* out, double* seconds) {
    try {
        need(models && nmodels > 0 && chains && nchains > 0 && p && out && seconds, "dock: bad arguments");
        need(!p->visited, "dock: smina's search only");
        std::vector<FlatModel> fms;
        for (int i = 0; i < nmodels; i++) {
            fms.push_back(flatten(models[i]));
            check_model(fms.back());
        }
        std::vector<const FlatModel*> ptrs;
        for (const FlatModel& f : fms) ptrs.push_back(&f);
        DeviceModels<float> dm;
        dm.upload(ptrs);
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
            need(ci.model >= 0 && ci.model < nmodels && ci.conf && ci.mt && ci.mt[624] <= 624, "dock: bad chain input");
            in[k].model = ci.model;
            in[k].conf.assign(ci.conf, ci.conf + models[ci.model].conf_size);
            std::memcpy(in[k].rng.x, ci.mt, sizeof(in[k].rng.x));
            in[k].rng.i = int(ci.mt[624]);
            in[k].num_steps = ci.num_steps;
            in[k].maxiters = ci.maxiters > 0 ? unsigned(ci.maxiters) : 0u;
            in[k].unit = 0;
        }
        InterContext<float> ic = InterContext<float>();
        ic.use_cache = 1;
        ic.grids = c->grids.dev;
        ic.rec = c->receptor.dev;
        ic.box = make_box<float>(c->geo);
        ic.ug = c->dug.dev;
        ic.slope = float(p->cache_slope);
        std::vector<ChainResult> res;
        const auto t0 = std::chrono::steady_clock::now();
        run_monte_carlo<float>(dm, c->tables, ic, mp, in, res, nullptr, 32, nullptr, nullptr);
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
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

}  // extern "C"
