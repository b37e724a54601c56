// sg_dock_batch32_noalloc: the batched mixed-precision search without any
// device allocation inside the call.
//
// Some callers cannot have a library allocate device memory while they
// run.  A serving loop may already have promised the rest of the GPU's
// memory to requests in flight, or handed it to a caching allocator such as
// PyTorch's; a cudaMalloc in the middle of a request could then fail or
// fragment that memory.  And cudaFree waits until the whole device is idle,
// which stalls every other stream the caller keeps busy.  For them this
// entry point runs the same search kernel as sg_dock_batch32 (k_mc32),
// with everything the kernel writes besides shared memory -- its copy of
// the models, the chain and work tables, the work-queue counter and the
// chains' result slots -- placed in one fixed array that is part of the
// library's device image, so nothing is allocated or freed per call.
//
// The price is a hard size limit (kScratchBytes per device) and one shared
// array: two calls that run on the same GPU at the same time, from two
// engines or two host threads, write over each other's data.  Callers must
// keep calls on one device from overlapping.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include "engine.h"

namespace sg {

// The fixed array.  8 MiB holds, for example, 16 ligands of 50 heavy atoms
// and 12 torsions at 8 chains each, with 20 result slots per chain.
constexpr size_t kScratchBytes = size_t(8) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of the fixed array, looked up once per device with that
// device current.  The lookup also loads this file's module, and with it the
// array: under lazy module loading that is the moment the 8 MiB is taken from
// the device, so engine creation does it (noalloc_claim), not a call.
static std::mutex g_scratch_mu;
static unsigned char* g_scratch_ptr[64] = {};

static unsigned char* scratch_on(int device) {
    require(device >= 0 && device < 64, "device index out of range for the fixed scratch table");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "address of the fixed scratch array");
        g_scratch_ptr[device] = static_cast<unsigned char*>(p);
    }
    return g_scratch_ptr[device];
}

// At engine creation (mixed-precision engines): claim the fixed array and
// load the search kernel with its shared-memory limit raised to the device's
// maximum, so that a later call neither loads a module nor sets a kernel
// attribute.
void noalloc_claim(sg_engine* e) {
    scratch_on(e->device);
    size_t dyn = 0;
    cuda_check(mc32_max_dynamic_smem((size_t)e->max_smem, &dyn), "search kernel attributes");
    cuda_check(mc32_reserve_smem(dyn), "search kernel shared-memory limit");
}

// bump placement inside the fixed array
struct Placer {
    size_t used = 0;
    size_t take(size_t bytes) {
        const size_t at = (used + 255) & ~(size_t)255;
        used = at + bytes;
        return at;
    }
};

// add_to_output_container (coords.cpp:25-58), as the batched entry point merges
struct NaPose {
    double e;
    std::vector<double> conf, xyz;
};
static void na_add_pose(std::vector<NaPose>& out, NaPose&& t, double min_rmsd, int max_size) {
    size_t ci = out.size();
    double cr = DBL_MAX;
    const size_t H3 = t.xyz.size();
    for (size_t i = 0; i < out.size(); i++) {
        double acc = 0;
        for (size_t a = 0; a < H3; a++) {
            const double d = t.xyz[a] - out[i].xyz[a];
            acc += d * d;
        }
        const double r = H3 ? std::sqrt(acc / (double)(H3 / 3)) : 0.0;
        if (i == 0 || r < cr) { ci = i; cr = r; }
    }
    if (ci < out.size() && cr < min_rmsd) {
        if (t.e < out[ci].e) out[ci] = std::move(t);
    } else if ((int)out.size() < max_size) {
        out.push_back(std::move(t));
    } else if (!out.empty() && t.e < out.back().e) {
        out.back() = std::move(t);
    }
    std::stable_sort(out.begin(), out.end(), [](const NaPose& a, const NaPose& b) { return a.e < b.e; });
}

}  // namespace sg

using namespace sg;

extern "C" {

int sg_dock_batch32_noalloc(sg_engine* e, int rid, const sg_model_desc* models, int nmodels, const sg_ligand_job* jobs,
                            int njobs, const sg_mc_params* p, sg_ligand_result* out) {
    return guarded(e, [&] {
        require(jobs && p && out && njobs > 0 && njobs <= (1 << 22), "dock_batch32_noalloc: bad arguments");
        require(e->precision != SG_PREC_FP64,
                "dock_batch32_noalloc needs an engine created with SG_PREC_FP32 or SG_PREC_FP32_H16");
        require(p->num_saved_mins >= 1 && p->num_saved_mins <= 1024 && p->maxiters >= 0 && p->temperature > 0,
                "dock_batch32_noalloc: bad search parameters");
        require(!p->visited, "the QuickVina 2 history (visited) runs on the plain path only");
        require(e->has_tables, "no tables set");
        RecState& r = receptor_for(e, rid);
        unsigned char* base = scratch_on(e->device);
        Placer at;
        // models first: their descriptors point into the array
        ModelImage img;
        pack_models_image(models, nmodels, reinterpret_cast<char*>(base), img);
        const size_t models_at = at.take(img.bytes.size());
        require(models_at == 0, "fixed scratch: models must start the array");
        // the maps must already be resident: building them would allocate
        for (int k = 0; k < nmodels; k++) {
            require(img.host[k].npchunks >= 0, "mixed-precision path: at most 255 atoms per model");
            for (int i = 0; i < models[k].num_movable; i++) {
                const int t = models[k].atom_type[i];
                if (t >= kNumTypes || is_h(t)) continue;
                require(r.built[t] && r.map32[t].p && (e->precision != SG_PREC_FP32_H16 || r.map16[t].p) &&
                            (e->tables.nc == 1 || r.cmap32[t].p),
                        "dock_batch32_noalloc: the receptor's maps for this ligand's atom types are not built "
                        "(call sg_build_grids first; building them allocates)");
            }
        }
        size_t ws_stride = 0, stage_stride = 0;
        for (const DModel& h : img.host) {
            ws_stride = std::max(ws_stride, ws32_bytes(h));
            stage_stride = std::max(stage_stride, (size_t)stage32_bytes(h.natoms, h.nframes, h.nheavy, h.npchunks,
                                                                        h.nlig, h.nblocks, h.ntors));
        }
        ws_stride = (ws_stride + 15) & ~(size_t)15;
        const int S = p->num_saved_mins;
        // first pass: check the jobs and count what the batch needs, so that
        // a batch too large for the array is refused before any per-chain
        // host table is built
        size_t nchains = 0, nconf_res = 0, nxyz_res = 0;
        int max_chains = 1;
        for (int j = 0; j < njobs; j++) {
            const sg_ligand_job& J = jobs[j];
            require(J.model >= 0 && J.model < nmodels && J.num_chains >= 1 && J.num_chains <= (1 << 16) &&
                        J.maxiters >= 0,
                    "dock_batch32_noalloc: bad ligand job");
            require(out[j].e && out[j].conf && out[j].coords, "dock_batch32_noalloc: null result arrays");
            max_chains = std::max(max_chains, J.num_chains);
            const DModel& h = img.host[J.model];
            nchains += (size_t)J.num_chains;
            nconf_res += (size_t)J.num_chains * S * h.conf_size;
            nxyz_res += (size_t)J.num_chains * S * h.nheavy * 3;
        }
        require(nchains <= (size_t(1) << 24), "dock_batch32_noalloc: at most 2^24 chains per call");
        // launch shape as sg_dock_batch32 picks it (a shape set by
        // sg_set_chains_per_block or sg_autotune32 included)
        int wpb = 1, occ = 1;
        choose_launch(e, stage_stride, ws_stride, max_chains, wpb, occ);
        size_t nitems_sz = 0;
        for (int j = 0; j < njobs; j++) nitems_sz += (size_t)(jobs[j].num_chains + wpb - 1) / wpb;
        const size_t chains_at = at.take(nchains * sizeof(Chain32));
        const size_t items_at = at.take(nitems_sz * sizeof(Item32));
        const size_t queue_at = at.take(sizeof(unsigned));
        const size_t e_at = at.take(nchains * S * sizeof(double));
        const size_t conf_at = at.take(nconf_res * sizeof(double));
        const size_t xyz_at = at.take(nxyz_res * sizeof(float));
        const size_t order_at = at.take(nchains * S * sizeof(int));
        const size_t count_at = at.take(nchains * sizeof(int));
        const size_t evals_at = at.take(nchains * sizeof(unsigned long long));
        const size_t hits_at = at.take(nchains * 2 * sizeof(unsigned long long));
        if (at.used > kScratchBytes)
            throw EngineError(SG_ERR_ARG, "dock_batch32_noalloc: this batch needs " + std::to_string(at.used) +
                                              " bytes of scratch but the fixed array holds " +
                                              std::to_string(kScratchBytes) + "; dock fewer ligands per call");
        // second pass: the chains and their result slots
        std::vector<Chain32> hc;
        std::vector<int> chain_job;
        std::vector<size_t> cres_off, xres_off;
        hc.reserve(nchains);
        chain_job.reserve(nchains);
        cres_off.reserve(nchains);
        xres_off.reserve(nchains);
        size_t conf_cur = 0, xyz_cur = 0;
        for (int j = 0; j < njobs; j++) {
            const sg_ligand_job& J = jobs[j];
            const DModel& h = img.host[J.model];
            for (int c = 0; c < J.num_chains; c++) {
                Chain32 ch{};
                ch.model = J.model;
                ch.steps = J.num_steps;
                ch.maxiters = J.maxiters > 0 ? J.maxiters : p->maxiters;
                ch.key0 = (uint32_t)J.seed;
                ch.key1 = (uint32_t)(J.seed >> 32) ^ (uint32_t)(J.ligand_key >> 32);
                ch.lig = (uint32_t)J.ligand_key;
                ch.chain = (uint32_t)c;
                hc.push_back(ch);
                chain_job.push_back(j);
                cres_off.push_back(conf_cur);
                xres_off.push_back(xyz_cur);
                conf_cur += (size_t)S * h.conf_size;
                xyz_cur += (size_t)S * h.nheavy * 3;
            }
        }
        std::vector<Item32> items;
        std::vector<double> item_cost;
        for (size_t k = 0; k < nchains;) {
            const int j = chain_job[k];
            int n = 0;
            while (k + n < nchains && chain_job[k + n] == j && n < wpb) n++;
            items.push_back(Item32{hc[k].model, (int)k, n, 0});
            item_cost.push_back((double)hc[k].steps * img.host[hc[k].model].cost * std::max(1, hc[k].maxiters));
            k += n;
        }
        require(items.size() == nitems_sz, "dock_batch32_noalloc: work item count");
        std::vector<int> order(items.size());
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return item_cost[a] > item_cost[b]; });
        std::vector<Item32> queue(items.size());
        for (size_t k = 0; k < items.size(); k++) queue[k] = items[order[k]];
        for (size_t k = 0; k < nchains; k++) {
            Chain32& ch = hc[k];
            ch.out_e = reinterpret_cast<double*>(base + e_at) + k * S;
            ch.out_conf = reinterpret_cast<double*>(base + conf_at) + cres_off[k];
            ch.out_coords = reinterpret_cast<float*>(base + xyz_at) + xres_off[k];
            ch.out_order = reinterpret_cast<int*>(base + order_at) + k * S;
            ch.out_count = reinterpret_cast<int*>(base + count_at) + k;
            ch.evals = reinterpret_cast<unsigned long long*>(base + evals_at) + k;
            ch.hits = reinterpret_cast<unsigned long long*>(base + hits_at) + 2 * k;
        }
        cudaStream_t s = e->stream;
        cuda_check(cudaMemcpyAsync(base + models_at, img.bytes.data(), img.bytes.size(), cudaMemcpyHostToDevice, s),
                   "models to scratch");
        cuda_check(cudaMemcpyAsync(base + chains_at, hc.data(), nchains * sizeof(Chain32), cudaMemcpyHostToDevice, s),
                   "chains to scratch");
        cuda_check(cudaMemcpyAsync(base + items_at, queue.data(), queue.size() * sizeof(Item32),
                                   cudaMemcpyHostToDevice, s),
                   "work items to scratch");
        // the array keeps the previous call's contents: the queue counter
        // must start at zero (the kernel resets each chain's slot count)
        cuda_check(cudaMemsetAsync(base + queue_at, 0, sizeof(unsigned), s), "queue reset");
        MCParams32 P{};
        for (int i = 0; i < 3; i++) {
            P.hunt[i] = (float)p->hunt_cap[i];
            P.auth[i] = (float)p->authentic_v[i];
            P.box[i] = r.gd.begin[i];
            P.box[3 + i] = r.gd.end[i];
        }
        P.slope = (float)p->cache_slope;
        P.temperature = p->temperature;
        P.amplitude = p->mutation_amplitude;
        P.min_rmsd = p->min_rmsd;
        P.num_saved = S;
        P.maxiters = p->maxiters;
        P.accurate_line = p->accurate_line;
        P.early_term = p->early_term;
        const int nitems = (int)queue.size();
        const int blocks = (int)std::min<long long>((long long)occ * e->num_sms, nitems);
        // the kernel's shared-memory limit was raised at engine creation, so
        // this launch sets no kernel attribute (a serving loop's launches may
        // be running on other streams)
        cuda_check(launch_mc32_fixed(reinterpret_cast<const DModel*>(base + models_at + img.dmodel_off), tables32(e),
                                     maps32(e, r), nullptr, reinterpret_cast<const Chain32*>(base + chains_at),
                                     reinterpret_cast<const Item32*>(base + items_at), nitems, P,
                                     reinterpret_cast<unsigned*>(base + queue_at), blocks, wpb, stage_stride,
                                     ws_stride, stage_stride + (size_t)wpb * ws_stride, s),
                   "search launch");
        std::vector<double> he(nchains * S), hconf(nconf_res);
        std::vector<float> hxyz(nxyz_res);
        std::vector<int> horder(nchains * S), hcount(nchains);
        std::vector<unsigned long long> hev(nchains);
        auto fetch = [&](void* dst, size_t from, size_t bytes) {
            if (bytes) cuda_check(cudaMemcpyAsync(dst, base + from, bytes, cudaMemcpyDeviceToHost, s), "fetch results");
        };
        fetch(he.data(), e_at, he.size() * sizeof(double));
        fetch(hconf.data(), conf_at, hconf.size() * sizeof(double));
        fetch(hxyz.data(), xyz_at, hxyz.size() * sizeof(float));
        fetch(horder.data(), order_at, horder.size() * sizeof(int));
        fetch(hcount.data(), count_at, hcount.size() * sizeof(int));
        fetch(hev.data(), evals_at, hev.size() * sizeof(unsigned long long));
        cuda_check(cudaStreamSynchronize(s), "search");
        // merge_output_containers per ligand, chains in job order
        std::vector<std::vector<NaPose>> merged(njobs);
        std::vector<uint64_t> job_evals(njobs, 0);
        for (size_t k = 0; k < nchains; k++) {
            const int j = chain_job[k];
            const DModel& h = img.host[hc[k].model];
            job_evals[j] += hev[k];
            const int cnt = std::min(std::max(hcount[k], 0), S);
            for (int i = 0; i < cnt; i++) {
                const int slot = horder[k * S + i];
                require(slot >= 0 && slot < S, "dock_batch32_noalloc: corrupt result order");
                NaPose t;
                t.e = he[k * S + slot];
                const double* c = &hconf[cres_off[k] + (size_t)slot * h.conf_size];
                t.conf.assign(c, c + h.conf_size);
                const float* x = &hxyz[xres_off[k] + (size_t)slot * h.nheavy * 3];
                t.xyz.assign(x, x + (size_t)h.nheavy * 3);
                na_add_pose(merged[j], std::move(t), 2.0, S);
            }
        }
        for (int j = 0; j < njobs; j++) {
            const DModel& h = img.host[jobs[j].model];
            out[j].count = (int)merged[j].size();
            out[j].evals = job_evals[j];
            for (size_t i = 0; i < merged[j].size(); i++) {
                out[j].e[i] = merged[j][i].e;
                std::memcpy(out[j].conf + i * h.conf_size, merged[j][i].conf.data(), h.conf_size * sizeof(double));
                std::memcpy(out[j].coords + i * h.nheavy * 3, merged[j][i].xyz.data(),
                            (size_t)h.nheavy * 3 * sizeof(double));
            }
        }
    });
}

}  // extern "C"
