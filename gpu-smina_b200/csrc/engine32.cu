// Batched mixed-precision docking behind the C ABI (sg_dock_batch32):
// every ligand job's chains run in one persistent search launch (k_mc32),
// the chains of a ligand are merged like merge_output_containers with
// min_rmsd 2, and every merged pose is refined in FP64 on the direct
// receptor sum (k_refine64).  Reference: gpu_docking.cpp:560-625
// (GpuDocking::dock_batch), parallel_mc.cpp:64-98, main.cpp:165-200.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <numeric>
#include "engine.h"

namespace sg {

DTables32 tables32(const sg_engine* e) {
    DTables32 T{};
    T.nc = e->tables.nc;
    T.n = e->tables.n;
    T.factor = (float)e->tables.factor;
    T.cutoff_sqr = (float)e->tables.cutoff_sqr;
    T.tab = e->tab32.as<float4>();
    return T;
}

DMaps32 maps32(const sg_engine* e, const RecState& r) {
    DMaps32 G{};
    for (int i = 0; i < 3; i++) {
        require(r.geom.dim[i] >= 2, "mixed-precision path: the box needs at least one grid cell per axis");
        G.cdim[i] = r.geom.dim[i] - 1;
        G.init[i] = (float)r.geom.init[i];
        G.factor[i] = (float)r.geom.factor[i];
        G.factor_inv[i] = (float)r.geom.factor_inv[i];
        G.dim_fl_minus_1[i] = (float)r.geom.dim_fl_minus_1[i];
    }
    for (int t = 0; t < kNumTypes; t++) {
        G.m32[t] = r.map32[t].as<float4>();
        G.c32[t] = r.cmap32[t].as<float4>();
        G.m16[t] = r.map16[t].as<uint4>();
    }
    G.half = e->precision == SG_PREC_FP32_H16;
    return G;
}

// every grid type the models look up has its packed maps
static void check_packed(const sg_engine* e, const RecState& r, const sg_model_desc* models, int nmodels) {
    for (int k = 0; k < nmodels; k++)
        for (int i = 0; i < models[k].num_movable; i++) {
            const int t = models[k].atom_type[i];
            if (t >= kNumTypes || is_h(t)) continue;
            require(r.map32[t].p && (e->precision != SG_PREC_FP32_H16 || r.map16[t].p) &&
                        (e->tables.nc == 1 || r.cmap32[t].p),
                    "mixed-precision maps missing for a ligand type");
        }
}

// add_to_output_container (coords.cpp:25-58) on the host, for the merge
struct HostPose {
    double e;
    std::vector<double> conf, xyz;
};
static void add_pose(std::vector<HostPose>& out, HostPose&& t, double min_rmsd, int max_size) {
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
    std::stable_sort(out.begin(), out.end(), [](const HostPose& a, const HostPose& b) { return a.e < b.e; });
}

// Launch shape for chains on teams of `team` warps: chains per block (wpb)
// with the most resident chains per SM (ties: more chains per block, so
// fewer model copies).  A batch of at most one chain per SM (nchains) runs
// one chain per block, so that every chain has an SM to itself.  False
// when no shape fits the shared memory.
bool try_launch(sg_engine* e, size_t stage_stride, size_t ws_stride, int max_chains, int team, long long nchains,
                int& wpb, int& occ) {
    const int cands[4] = {8, 4, 2, 1};
    int best_w = 0, best_occ = 0, best_res = 0;
    const bool spread = !e->force_wpb && nchains <= e->num_sms;
    for (int c : cands) {
        if (c * team > 8) continue;
        if (e->force_wpb && c != e->force_wpb) continue;
        if (!e->force_wpb && c > 1 && c / 2 >= max_chains) continue;  // half the chains' warps would idle
        if (spread && c > 1) continue;
        const size_t smem = stage_stride + (size_t)c * team * ws_stride;
        if (smem > (size_t)e->max_smem) continue;
        const int o = mc32_occupancy(team, c * team, smem);
        if (o * c > best_res) { best_res = o * c; best_w = c; best_occ = o; }
    }
    wpb = best_w;
    occ = best_occ;
    return best_res > 0;
}

void choose_launch(sg_engine* e, size_t stage_stride, size_t ws_stride, int max_chains, int& wpb, int& occ) {
    require(try_launch(e, stage_stride, ws_stride, max_chains, 1, 1ll << 40, wpb, occ),
            "model too large for the mixed-precision path's shared memory");
}

#ifdef SG_PROFILE
cudaError_t profile_read32(unsigned long long* out16, bool clear);
#endif

}  // namespace sg

using namespace sg;

extern "C" {

int sg_dock_batch32(sg_engine* e, int rid, const sg_model_desc* models, int nmodels, const sg_ligand_job* jobs, int njobs,
                    const sg_mc_params* p, int refine, sg_ligand_result* out) {
    return guarded(e, [&] {
        require(jobs && p && out && njobs > 0 && njobs <= (1 << 22), "dock_batch32: bad arguments");
        require(e->precision != SG_PREC_FP64, "dock_batch32 needs an engine created with SG_PREC_FP32 or SG_PREC_FP32_H16");
        require(p->num_saved_mins >= 1 && p->num_saved_mins <= 1024 && p->maxiters >= 0 && p->temperature > 0,
                "dock_batch32: bad search parameters");
        require(!p->visited, "the QuickVina 2 history (visited) runs on the plain path only");
        require(e->has_tables, "no tables set");
        RecState& r = receptor_for(e, rid);
        PackedModels pm;
        pack_models(e, models, nmodels, pm);
        ensure_model_maps(e, r, pm, models, nmodels);
        check_packed(e, r, models, nmodels);
        uint64_t h2d = pm.ints.bytes + pm.flts.bytes + pm.dbls.bytes + pm.dmodels.bytes, d2h = 0;
        size_t ws_stride = 0, stage_stride = 0;
        for (const DModel& h : pm.host) {
            require(h.npchunks >= 0, "mixed-precision path: at most 255 atoms per model");
            ws_stride = std::max(ws_stride, ws32_bytes(h));
            stage_stride = std::max(stage_stride, (size_t)stage32_bytes(h.natoms, h.nframes, h.nheavy, h.npchunks,
                                                                        h.nlig, h.nblocks, h.ntors));
        }
        ws_stride = (ws_stride + 15) & ~(size_t)15;
        const int S = p->num_saved_mins;
        // chains of every job, with their result slots
        std::vector<Chain32> hc;
        std::vector<int> chain_job;
        std::vector<size_t> cres_off, xres_off;
        size_t nconf_res = 0, nxyz_res = 0;
        for (int j = 0; j < njobs; j++) {
            const sg_ligand_job& J = jobs[j];
            require(J.model >= 0 && J.model < nmodels && J.num_chains >= 1 && J.num_chains <= (1 << 16) && J.maxiters >= 0,
                    "dock_batch32: bad ligand job");
            require(out[j].e && out[j].conf && out[j].coords, "dock_batch32: null result arrays");
            const DModel& h = pm.host[J.model];
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
                cres_off.push_back(nconf_res);
                xres_off.push_back(nxyz_res);
                nconf_res += (size_t)S * h.conf_size;
                nxyz_res += (size_t)S * h.nheavy * 3;
            }
        }
        const int nchains = (int)hc.size();
        require(nchains <= (1 << 24), "dock_batch32: too many chains");
        DevBuf d_e, d_conf, d_xyz, d_order, d_count, d_evals, d_hits, d_queue;
        d_e.alloc((size_t)nchains * S * sizeof(double));
        d_conf.alloc(std::max<size_t>(1, nconf_res) * sizeof(double));
        d_xyz.alloc(std::max<size_t>(1, nxyz_res) * sizeof(float));
        d_order.alloc((size_t)nchains * S * sizeof(int));
        d_count.alloc((size_t)nchains * sizeof(int));
        d_evals.alloc((size_t)nchains * sizeof(unsigned long long));
        d_hits.alloc((size_t)nchains * 2 * sizeof(unsigned long long));
        d_queue.alloc(sizeof(unsigned));
        for (int k = 0; k < nchains; k++) {
            Chain32& ch = hc[k];
            ch.out_e = d_e.as<double>() + (size_t)k * S;
            ch.out_conf = d_conf.as<double>() + cres_off[k];
            ch.out_coords = d_xyz.as<float>() + xres_off[k];
            ch.out_order = d_order.as<int>() + (size_t)k * S;
            ch.out_count = d_count.as<int>() + k;
            ch.evals = d_evals.as<unsigned long long>() + k;
            ch.hits = d_hits.as<unsigned long long>() + 2 * k;
        }
        // work items: up to wpb chains of one job; longest first, so the
        // persistent kernel's queue ends evenly
        int max_chains = 1;
        for (int j = 0; j < njobs; j++) max_chains = std::max(max_chains, jobs[j].num_chains);
        // Threads per chain: as set, or (0) the most warps per chain whose
        // resident chains still hold the whole batch (the reference's
        // threads_per_chain, gpu_kernels_impl.cuh:572-605).
        int wpb = 1, occ = 1, team = std::max(1, e->tpc / 32);
        if (e->tpc == 0) {
            team = 1;
            for (int g : {4, 2}) {
                int w = 0, o = 0;
                if (try_launch(e, stage_stride, ws_stride, max_chains, g, nchains, w, o) &&
                    (long long)nchains <= (long long)o * w * e->num_sms) {
                    team = g;
                    break;
                }
            }
        }
        require(!e->force_wpb || e->force_wpb * team <= 8,
                "chains per block (sg_set_chains_per_block) times warps per chain is above 8 warps per block");
        require(try_launch(e, stage_stride, ws_stride, max_chains, team, nchains, wpb, occ),
                "model too large for the mixed-precision path's shared memory at this many threads per chain");
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
        // Early stop (--fast): phases ending at (first + k) / checkpoints of
        // every chain's steps, each resuming from the state the previous one
        // saved; the stopping rule between phases.  Without it, one phase.
        const bool phased = e->es_on;
        int es_n = 1, es_first = 1;
        if (phased) {
            es_n = std::max(1, e->es.checkpoints);
            es_first = std::min(es_n, std::max(1, e->es.first));
        }
        const int nphases = es_n - es_first + 1;
        std::vector<size_t> res_off(nchains, 0);
        DevBuf d_resume;
        if (phased) {
            size_t nres = 0;
            for (int k = 0; k < nchains; k++) {
                const DModel& h = pm.host[hc[k].model];
                res_off[k] = nres;
                nres += (resume32_doubles(h.conf_size, h.natoms, h.nframes) + 1) & ~(size_t)1;  // 16-byte pieces
            }
            d_resume.alloc(std::max<size_t>(1, nres) * sizeof(double));
            for (int k = 0; k < nchains; k++) hc[k].resume = d_resume.as<double>() + res_off[k];
        }
        std::vector<unsigned> done(nchains, 0);
        std::vector<char> stopped(njobs, 0);
        std::vector<double> hres;
        DevBuf d_chains, d_items;
        float mc_ms = 0;
        int first_blocks = 0;
        cudaEvent_t ev[4];
        for (auto& x : ev) cuda_check(cudaEventCreate(&x), "event");
        struct EvGuard {
            cudaEvent_t* v;
            ~EvGuard() { for (int i = 0; i < 4; i++) cudaEventDestroy(v[i]); }
        } evg{ev};
        for (int ph = 0; ph < nphases; ph++) {
            std::vector<int> active;
            for (int k = 0; k < nchains; k++) {
                if (stopped[chain_job[k]]) continue;
                const unsigned steps = hc[k].steps;
                const unsigned end = ph + 1 < nphases
                                         ? (unsigned)(((unsigned long long)steps * (es_first + ph) + es_n - 1) / es_n)
                                         : steps;
                if (end <= done[k]) continue;
                hc[k].begin = done[k];
                hc[k].end = end;
                done[k] = end;
                active.push_back(k);
            }
            if (active.empty()) continue;
            std::vector<Item32> items;
            std::vector<double> item_cost;
            for (size_t a = 0; a < active.size();) {
                const int k = active[a], j = chain_job[k];
                int n = 0;
                while (a + n < active.size() && chain_job[active[a + n]] == j && n < wpb &&
                       active[a + n] == k + n)
                    n++;
                items.push_back(Item32{hc[k].model, k, n, 0});
                item_cost.push_back((double)(hc[k].end - hc[k].begin) * pm.host[hc[k].model].cost *
                                    std::max(1, hc[k].maxiters));
                a += n;
            }
            std::vector<int> order(items.size());
            std::iota(order.begin(), order.end(), 0);
            std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return item_cost[x] > item_cost[y]; });
            std::vector<Item32> queue(items.size());
            for (size_t k = 0; k < items.size(); k++) queue[k] = items[order[k]];
            const int nitems = (int)queue.size();
            const int blocks = (int)std::min<long long>((long long)occ * e->num_sms, nitems);
            if (ph == 0) first_blocks = blocks;
            d_chains.upload(hc.data(), hc.size() * sizeof(Chain32), e->stream);
            d_items.upload(queue.data(), queue.size() * sizeof(Item32), e->stream);
            h2d += d_chains.bytes + d_items.bytes;
            cuda_check(cudaMemsetAsync(d_queue.p, 0, sizeof(unsigned), e->stream), "queue reset");
            cuda_check(cudaEventRecord(ev[0], e->stream), "event");
            cuda_check(launch_mc32(pm.dmodels.as<DModel>(), tables32(e), maps32(e, r), nullptr, d_chains.as<Chain32>(),
                                   d_items.as<Item32>(), nitems, P, d_queue.as<unsigned>(), blocks, wpb * team,
                                   stage_stride, ws_stride, team, e->stream),
                       "search launch");
            cuda_check(cudaEventRecord(ev[1], e->stream), "event");
            if (phased && ph + 1 < nphases) {  // the stopping rule on the best energies the chains saved
                hres.resize(d_resume.bytes / sizeof(double));
                cuda_check(cudaMemcpyAsync(hres.data(), d_resume.p, d_resume.bytes, cudaMemcpyDeviceToHost, e->stream),
                           "best energies");
                d2h += d_resume.bytes;
            }
            cuda_check(cudaStreamSynchronize(e->stream), "search");
            float ms = 0;
            cuda_check(cudaEventElapsedTime(&ms, ev[0], ev[1]), "event time");
            mc_ms += ms;
            if (phased && ph + 1 < nphases) {
                const int cpu = e->es.chains_per_unit;
                for (int k0 = 0; k0 < nchains;) {  // per job: its units' best energies
                    const int j = chain_job[k0];
                    int k1 = k0;
                    while (k1 < nchains && chain_job[k1] == j) k1++;
                    if (!stopped[j]) {
                        std::vector<double> ub;
                        for (int k = k0; k < k1; k++) {
                            const size_t u = (size_t)((k - k0) / cpu);
                            if (ub.size() <= u) ub.resize(u + 1, DBL_MAX);
                            const int cs = pm.host[hc[k].model].conf_size;
                            ub[u] = std::min(ub[u], hres[res_off[k] + cs + 1]);
                        }
                        if (ub.size() >= 2) {
                            const double best = *std::min_element(ub.begin(), ub.end());
                            int agree = 0;
                            for (double v : ub) agree += (v - best <= e->es.eps);
                            const int need = std::max(2, (int)std::ceil(e->es.fraction * ub.size() - 1e-9));
                            if (agree >= need) stopped[j] = 1;
                        }
                    }
                    k0 = k1;
                }
            }
        }
        const int blocks = first_blocks;
        std::vector<double> he((size_t)nchains * S), hconf(nconf_res);
        std::vector<float> hxyz(nxyz_res);
        std::vector<int> horder((size_t)nchains * S), hcount(nchains);
        std::vector<unsigned long long> hev(nchains), hhits(2 * (size_t)nchains);
        auto fetch = [&](void* dst, const DevBuf& src, size_t bytes) {
            if (!bytes) return;
            cuda_check(cudaMemcpyAsync(dst, src.p, bytes, cudaMemcpyDeviceToHost, e->stream), "fetch results");
            d2h += bytes;
        };
        fetch(he.data(), d_e, he.size() * sizeof(double));
        fetch(hconf.data(), d_conf, hconf.size() * sizeof(double));
        fetch(hxyz.data(), d_xyz, hxyz.size() * sizeof(float));
        fetch(horder.data(), d_order, horder.size() * sizeof(int));
        fetch(hcount.data(), d_count, hcount.size() * sizeof(int));
        fetch(hev.data(), d_evals, hev.size() * sizeof(unsigned long long));
        fetch(hhits.data(), d_hits, hhits.size() * sizeof(unsigned long long));
        cuda_check(cudaStreamSynchronize(e->stream), "search");
        // merge_output_containers per ligand (chains in job order)
        std::vector<std::vector<HostPose>> merged(njobs);
        std::vector<uint64_t> job_evals(njobs, 0);
        uint64_t tot_evals = 0, tot_grid = 0, tot_pair = 0;
        for (int k = 0; k < nchains; k++) {
            const int j = chain_job[k];
            const DModel& h = pm.host[hc[k].model];
            job_evals[j] += hev[k];
            tot_evals += hev[k];
            tot_grid += hhits[2 * k];
            tot_pair += hhits[2 * k + 1];
            const int cnt = std::min(std::max(hcount[k], 0), S);
            for (int i = 0; i < cnt; i++) {
                const int slot = horder[(size_t)k * S + i];
                require(slot >= 0 && slot < S, "dock_batch32: corrupt result order");
                HostPose t;
                t.e = he[(size_t)k * S + slot];
                const double* c = &hconf[cres_off[k] + (size_t)slot * h.conf_size];
                t.conf.assign(c, c + h.conf_size);
                const float* x = &hxyz[xres_off[k] + (size_t)slot * h.nheavy * 3];
                t.xyz.assign(x, x + (size_t)h.nheavy * 3);
                add_pose(merged[j], std::move(t), 2.0, S);
            }
        }
        // refine_structure of every merged pose, FP64 on the direct sum
        float ref_ms = 0;
        if (refine) {
            int nposes = 0;
            for (auto& v : merged) nposes += (int)v.size();
            if (nposes > 0) {
                require(pm.max_ws64 <= (size_t)e->max_smem, "model too large for the plain path's shared memory");
                const int cs = pm.max_conf, hs = std::max(1, pm.max_heavy);
                std::vector<double> confs((size_t)nposes * cs, 0.0);
                std::vector<int> pmodel(nposes), pmaxit(nposes);
                int q = 0;
                for (int j = 0; j < njobs; j++)
                    for (auto& t : merged[j]) {
                        std::memcpy(&confs[(size_t)q * cs], t.conf.data(), t.conf.size() * sizeof(double));
                        pmodel[q] = jobs[j].model;
                        pmaxit[q] = jobs[j].maxiters > 0 ? jobs[j].maxiters : p->maxiters;
                        q++;
                    }
                DevBuf dc, de, dx, dpm, dmi;
                dc.upload(confs.data(), confs.size() * sizeof(double), e->stream);
                dpm.upload(pmodel.data(), pmodel.size() * sizeof(int), e->stream);
                dmi.upload(pmaxit.data(), pmaxit.size() * sizeof(int), e->stream);
                h2d += dc.bytes + dpm.bytes + dmi.bytes;
                de.alloc((size_t)nposes * sizeof(double));
                dx.alloc((size_t)nposes * hs * 3 * sizeof(double));
                cuda_check(cudaEventRecord(ev[2], e->stream), "event");
                cuda_check(launch_refine64(pm.dmodels.as<DModel>(), pm.max_ws64, e->tables, r.dhdr.as<DReceptor>(),
                                           dpm.as<int>(), nposes, dc.as<double>(), cs, p->authentic_v, p->maxiters,
                                           dmi.as<int>(), nullptr, p->accurate_line, p->early_term, de.as<double>(),
                                           dx.as<double>(), hs, e->d_err.as<int>(), e->stream),
                           "refine launch");
                cuda_check(cudaEventRecord(ev[3], e->stream), "event");
                std::vector<double> re(nposes), rx((size_t)nposes * hs * 3);
                fetch(confs.data(), dc, confs.size() * sizeof(double));
                fetch(re.data(), de, re.size() * sizeof(double));
                fetch(rx.data(), dx, rx.size() * sizeof(double));
                e->check_device_errors();
                cuda_check(cudaEventElapsedTime(&ref_ms, ev[2], ev[3]), "event time");
                q = 0;
                for (int j = 0; j < njobs; j++) {
                    const DModel& h = pm.host[jobs[j].model];
                    for (auto& t : merged[j]) {
                        std::memcpy(t.conf.data(), &confs[(size_t)q * cs], t.conf.size() * sizeof(double));
                        t.e = re[q];
                        t.xyz.assign(&rx[(size_t)q * hs * 3], &rx[(size_t)q * hs * 3] + (size_t)h.nheavy * 3);
                        q++;
                    }
                    std::stable_sort(merged[j].begin(), merged[j].end(),
                                     [](const HostPose& a, const HostPose& b) { return a.e < b.e; });
                }
            }
        }
        for (int j = 0; j < njobs; j++) {
            const DModel& h = pm.host[jobs[j].model];
            out[j].count = (int)merged[j].size();
            out[j].evals = job_evals[j];
            for (size_t i = 0; i < merged[j].size(); i++) {
                out[j].e[i] = merged[j][i].e;
                std::memcpy(out[j].conf + i * h.conf_size, merged[j][i].conf.data(), h.conf_size * sizeof(double));
                std::memcpy(out[j].coords + i * h.nheavy * 3, merged[j][i].xyz.data(), (size_t)h.nheavy * 3 * sizeof(double));
            }
        }
        e->last_wpb = wpb;
        e->last_team = team;
        e->last_blocks = blocks;
        e->last_mc_ms = mc_ms;
        e->last_refine_ms = ref_ms;
        e->last_evals = tot_evals;
        e->last_grid_hits = tot_grid;
        e->last_pair_hits = tot_pair;
        e->last_h2d = h2d;
        e->last_d2h = d2h;
    });
}

int sg_batch_stats(const sg_engine* e, double* mc_ms, double* refine_ms, int* chains_per_block, int* blocks) {
    if (!e) return SG_ERR_ARG;
    if (mc_ms) *mc_ms = e->last_mc_ms;
    if (refine_ms) *refine_ms = e->last_refine_ms;
    if (chains_per_block) *chains_per_block = e->last_wpb;
    if (blocks) *blocks = e->last_blocks;
    return SG_OK;
}

int sg_batch_counters(const sg_engine* e, uint64_t* evals, uint64_t* grid_lookups, uint64_t* pair_lookups,
                      uint64_t* h2d_bytes, uint64_t* d2h_bytes) {
    if (!e) return SG_ERR_ARG;
    if (evals) *evals = e->last_evals;
    if (grid_lookups) *grid_lookups = e->last_grid_hits;
    if (pair_lookups) *pair_lookups = e->last_pair_hits;
    if (h2d_bytes) *h2d_bytes = e->last_h2d;
    if (d2h_bytes) *d2h_bytes = e->last_d2h;
    return SG_OK;
}

#ifdef SG_PROFILE
// profiling builds only: clock64() cycles per section summed over warps
int sg_profile_read(unsigned long long* out16, int clear) {
    return profile_read32(out16, clear != 0) == cudaSuccess ? SG_OK : SG_ERR_CUDA;
}
#endif

int sg_set_early_stop(sg_engine* e, const sg_early_stop* es) {
    if (!e) return SG_ERR_ARG;
    if (!es) {
        e->es_on = false;
        return SG_OK;
    }
    if (e->precision == SG_PREC_FP64 || es->checkpoints < 1 || es->checkpoints > 1000 || es->first < 1 ||
        !(es->fraction >= 0 && es->fraction <= 1) || !(es->eps == es->eps) || es->chains_per_unit < 1)
        return SG_ERR_ARG;
    e->es = *es;
    e->es_on = true;
    return SG_OK;
}

int sg_set_threads_per_chain(sg_engine* e, int threads) {
    if (!e || !(threads == 0 || threads == 32 || threads == 64 || threads == 128)) return SG_ERR_ARG;
    e->tpc = threads;
    return SG_OK;
}

int sg_threads_per_chain(const sg_engine* e, int* configured, int* last_batch) {
    if (!e) return SG_ERR_ARG;
    if (configured) *configured = e->tpc;
    if (last_batch) *last_batch = 32 * e->last_team;
    return SG_OK;
}

int sg_set_chains_per_block(sg_engine* e, int n) {
    if (!e || !(n == 0 || n == 1 || n == 2 || n == 4 || n == 8)) return SG_ERR_ARG;
    e->force_wpb = n;
    return SG_OK;
}

int sg_autotune32(sg_engine* e, int rid, const sg_model_desc* models, int nmodels, const sg_ligand_job* jobs, int njobs,
                  const sg_mc_params* p, double step_fraction, double* evals_per_s, int* chosen) {
    if (!e || !jobs || !p || njobs <= 0 || !(step_fraction > 0 && step_fraction <= 1)) return SG_ERR_ARG;
    const int cands[4] = {8, 4, 2, 1};
    const int keep = e->force_wpb;
    // the sample: every job with its step count scaled (at least one step)
    std::vector<sg_ligand_job> sample(jobs, jobs + njobs);
    for (auto& j : sample) j.num_steps = std::max(1, (int)(j.num_steps * step_fraction));
    const int S = p->num_saved_mins;
    int max_conf = 1, max_heavy = 1;
    for (int k = 0; k < nmodels && models; k++) {
        max_conf = std::max(max_conf, models[k].conf_size);
        max_heavy = std::max(max_heavy, models[k].num_movable);  // bounds the heavy atoms
    }
    std::vector<double> se((size_t)njobs * std::max(S, 1)), sc((size_t)njobs * std::max(S, 1) * max_conf),
        sx((size_t)njobs * std::max(S, 1) * max_heavy * 3);
    std::vector<sg_ligand_result> res(njobs);
    for (int j = 0; j < njobs; j++)
        res[j] = {0, &se[(size_t)j * S], &sc[(size_t)j * S * max_conf], &sx[(size_t)j * S * max_heavy * 3], 0};
    double best = -1;
    int best_c = 0;
    for (int i = 0; i < 4; i++) {
        if (evals_per_s) evals_per_s[i] = 0;
        e->force_wpb = cands[i];
        const int rc = sg_dock_batch32(e, rid, models, nmodels, sample.data(), njobs, p, 0, res.data());
        if (rc != SG_OK && rc != SG_ERR_ARG) {  // a device error ends the search; the shape stays as it was
            e->force_wpb = keep;
            return rc;
        }
        if (rc != SG_OK || e->last_wpb != cands[i] || e->last_mc_ms <= 0) continue;  // shape not possible here
        const double v = (double)e->last_evals / (e->last_mc_ms * 1e-3);
        if (evals_per_s) evals_per_s[i] = v;
        if (v > best) { best = v; best_c = cands[i]; }
    }
    e->force_wpb = best_c ? best_c : keep;
    if (chosen) *chosen = best_c;
    if (!best_c) {
        e->err = "autotune: no launch shape ran (" + e->err + ")";
        return SG_ERR_ARG;
    }
    return SG_OK;
}

}  // extern "C"
