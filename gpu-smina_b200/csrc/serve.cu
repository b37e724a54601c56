// Serving: a request loop with continuous batching over resident receptors.
//
// Requests (one ligand against one resident receptor each) are queued by
// sg_serve_submit.  A worker thread uploads them in small batches (a batch
// goes out as soon as the device can take it, or, under light load, once
// the oldest request has waited max_wait_ms for others to share it) if the
// device memory the server holds for requests in flight stays under its
// budget.  A batch's work items (a group of chains of one ligand each) go
// into a ring in device memory that a resident serving grid takes items
// from while it runs: a ligand's chains start as soon as a block is free,
// whatever batch it came with, so the device keeps a mix of requests in
// flight rather than a queue of whole launches.  Ligands of different
// receptors share a batch (every item names its receptor's map set).
// The last chain of a ligand to finish raises a flag in host-mapped memory;
// the worker then copies that ligand's chain results back, merges them
// (min_rmsd 2) and refines the merged poses in FP64 on a separate stream,
// and the result becomes available to sg_serve_poll / sg_serve_fetch.
// Results are the same as sg_dock_batch32's for the same (seed, ligand key)
// whatever else is in flight.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <thread>
#include "engine.h"

namespace sg {

using Clock = std::chrono::steady_clock;

// an owned copy of a caller's model description (the caller may free its
// arrays once sg_serve_submit returns)
struct ModelCopy {
    sg_model_desc d{};
    std::vector<int> lig_pair_end, lig_begin, lig_end, lig_root, type, fkind, fparent, fbegin, fend, fconf, fdof, pairs;
    std::vector<double> charge, local, lab, forigin, faxis, finit;
    explicit ModelCopy(const sg_model_desc& s) : d(s) {
        auto ci = [](std::vector<int>& v, const int* p, size_t n) { if (p) v.assign(p, p + n); };
        auto cd = [](std::vector<double>& v, const double* p, size_t n) { if (p) v.assign(p, p + n); };
        const size_t L = s.num_ligands, N = s.num_atoms, F = s.num_frames, P = s.num_pairs;
        ci(lig_pair_end, s.lig_pair_end, L); ci(lig_begin, s.ligand_atom_begin, L); ci(lig_end, s.ligand_atom_end, L);
        ci(lig_root, s.ligand_root, L); ci(type, s.atom_type, N); ci(fkind, s.frame_kind, F);
        ci(fparent, s.frame_parent, F); ci(fbegin, s.frame_begin, F); ci(fend, s.frame_end, F);
        ci(fconf, s.frame_conf, F); ci(fdof, s.frame_dof, F); ci(pairs, s.pairs, 2 * P);
        cd(charge, s.atom_charge, N); cd(local, s.atom_local, 3 * N); cd(lab, s.atom_lab, 3 * N);
        cd(forigin, s.frame_origin, 3 * F); cd(faxis, s.frame_axis, 3 * F); cd(finit, s.frame_init_origin, 3 * F);
        auto pi = [](const std::vector<int>& v) { return v.empty() ? nullptr : v.data(); };
        auto pd = [](const std::vector<double>& v) { return v.empty() ? nullptr : v.data(); };
        d.lig_pair_end = pi(lig_pair_end); d.ligand_atom_begin = pi(lig_begin); d.ligand_atom_end = pi(lig_end);
        d.ligand_root = pi(lig_root); d.atom_type = pi(type); d.frame_kind = pi(fkind); d.frame_parent = pi(fparent);
        d.frame_begin = pi(fbegin); d.frame_end = pi(fend); d.frame_conf = pi(fconf); d.frame_dof = pi(fdof);
        d.pairs = pi(pairs); d.atom_charge = pd(charge); d.atom_local = pd(local); d.atom_lab = pd(lab);
        d.frame_origin = pd(forigin); d.frame_axis = pd(faxis); d.frame_init_origin = pd(finit);
    }
};

struct ServeReq {
    uint64_t ticket = 0;
    int rid = 0;
    sg_ligand_job job{};
    sg_mc_params p{};
    std::shared_ptr<ModelCopy> m;
    Clock::time_point t_submit;
    size_t bytes = 0;  // device memory its share of a batch needs
    size_t stage = 0, ws = 0;  // its staged-model and per-chain workspace bytes in shared memory
};

struct ServeDone {
    sg_serve_done info{};
    std::vector<double> e, conf, coords;
};

// add_to_output_container (coords.cpp:25-58) for the per-ligand merge
struct SvPose {
    double e;
    std::vector<double> conf, xyz;
};
static void sv_add_pose(std::vector<SvPose>& out, SvPose&& t, double min_rmsd, int max_size) {
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
    std::stable_sort(out.begin(), out.end(), [](const SvPose& a, const SvPose& b) { return a.e < b.e; });
}

// One ligand inside a launched batch and its post-processing state.
struct SvLig {
    ServeReq req;
    int model = 0, first = 0, nchains = 0, flag = -1;
    int blocks = 0;  // its work items (a block's worth of its chains each)
    int team = 1;    // warps per chain of its search
    int state = 0;  // 0 searching, 1 refining, 2 published
    uint64_t evals = 0;
    uint64_t dev_start = 0, dev_end = 0;  // device clock (ns): first chain's start, last chain's end
    uint64_t launch = 0;                  // its batch's launch number
    Clock::time_point t_launch;           // when its batch was launched
    Clock::time_point t_flag;             // when the worker saw its chains done
    std::vector<SvPose> poses;
    size_t conf_off = 0, xyz_off = 0;
    struct SvBatch* batch = nullptr;
};

struct SvBatch {
    cudaStream_t stream = nullptr;
    char* dmem = nullptr;
    size_t bytes = 0;
    ModelImage img;
    std::vector<SvLig> ligs;
    std::vector<Chain32> hc;
    size_t e_at = 0, conf_at = 0, xyz_at = 0, order_at = 0, count_at = 0, evals_at = 0, span_at = 0;
    int S = 20;
    uint64_t seq = 0;  // launch number (1, 2, ... per server)
    char* pin = nullptr;           // pinned staging of its ring items and tail word
    size_t pin_cap = 0;
    int flagged = 0;               // ligands whose completion flag has been seen
    int published = 0;
};

struct Server {
    sg_engine* e = nullptr;
    sg_serve_opts o{};
    std::thread th;
    std::mutex mu;
    std::condition_variable cv_done;
    std::deque<ServeReq> queue;
    std::map<uint64_t, ServeDone> done;
    std::deque<uint64_t> done_order;  // not yet reported by poll
    std::vector<std::unique_ptr<SvBatch>> inflight;
    size_t inflight_bytes = 0;
    uint64_t launches = 0;
    uint64_t next_ticket = 1;
    bool stopping = false;
    int error = SG_OK;
    std::string error_text;
    // serving grids: items wait in a ring in device memory that resident
    // blocks take from; the worker starts blocks when items wait and no block
    // is free (blocks leave after an idle time)
    static constexpr unsigned kRing = 1u << 16;
    FeedItem32* d_ring = nullptr;
    FeedCtrl32* d_ctrl = nullptr;
    FeedCtrl32* h_ctrl = nullptr;        // pinned snapshot of the control words
    FeedCtrl32 seen{};                    // the last snapshot that landed
    cudaEvent_t ctrl_ev = nullptr;
    bool ctrl_pending = false;
    uint64_t snap_req = 0, snap_seen = 0, launch_req = 0;  // snapshot requests, and the one a launch waits past
    unsigned tail = 0;                    // items published
    unsigned blocks_launched = 0;         // blocks of every grid started so far
    int target_blocks = 0;                // serving blocks the device holds at once
    long long idle_ns = 500000000;        // a block leaves after this long without work
    cudaStream_t feed_stream = nullptr, ctrl_stream = nullptr;
    std::vector<cudaStream_t> grid_streams;  // a grid per stream; grids end on their own
    int inflight_ligs = 0;
    long long inflight_blocks = 0;  // work items of ligands whose chains are not yet seen done
    cudaStream_t refine_stream = nullptr, copy_stream = nullptr;
    // completion flags in host-mapped memory
    volatile unsigned* flags = nullptr;
    unsigned* dflags = nullptr;
    std::vector<int> free_flags;
    int* d_err = nullptr;            // device error word (refinement overlap)
    volatile int* h_err = nullptr;   // pinned copy, refreshed after every refinement launch
    Clock::time_point last_err_check;
    std::vector<std::unique_ptr<struct RefineGroup>> refining;
    // pinned staging buffers for refinements (copies into pageable memory
    // would make the worker wait for the refinement kernel)
    std::vector<std::pair<size_t, char*>> pin_free;
    std::vector<char*> pin_all;
    size_t smem_block = 0;  // dynamic shared memory of every search launch (same for all, set at start)
    static constexpr int kFlags = 1 << 16;
};

static size_t req_bytes(const sg_model_desc& m, const sg_ligand_job& j, int S) {
    const size_t conf = m.conf_size, heavy = m.num_movable;  // heavy <= movable: an upper bound
    const size_t per_chain = sizeof(Chain32) + S * (8 + 8 * conf + 12 * heavy + 4) + 4 + 8 + 16;
    const size_t model = 64 * (size_t)m.num_atoms + 96 * (size_t)m.num_frames + 24 * (size_t)m.num_pairs + 4096;
    return model + j.num_chains * per_chain + S * (8 * conf + 24 * heavy + 8) + 4096;
}

static bool same_params(const sg_mc_params& a, const sg_mc_params& b) {
    return a.temperature == b.temperature && a.mutation_amplitude == b.mutation_amplitude && a.min_rmsd == b.min_rmsd &&
           a.num_saved_mins == b.num_saved_mins && a.accurate_line == b.accurate_line && a.early_term == b.early_term &&
           a.cache_slope == b.cache_slope && std::equal(a.hunt_cap, a.hunt_cap + 3, b.hunt_cap) &&
           std::equal(a.authentic_v, a.authentic_v + 3, b.authentic_v);
}

// Chains per block a launch can run with the server's fixed shared memory,
// given its largest staged model and workspace (0: none fits).
static int serve_shape(const Server& s, size_t stage, size_t ws, int max_chains) {
    for (int c : {8, 4, 2, 1}) {
        if (s.e->force_wpb && c != s.e->force_wpb) continue;
        if (!s.e->force_wpb && c > 1 && c / 2 >= max_chains) continue;
        if (stage + (size_t)c * ws <= s.smem_block) return c;
    }
    return 0;
}

static char* pin_get(Server& s, size_t bytes, size_t& cap);

// Uploads one batch and publishes its items to the serving grid's ring;
// called by the worker with mu held.
static void launch_batch(Server& s, std::vector<ServeReq>&& reqs) {
    sg_engine* e = s.e;
    auto b = std::make_unique<SvBatch>();
    const sg_mc_params& p = reqs[0].p;
    const int S = p.num_saved_mins;
    b->S = S;
    std::vector<sg_model_desc> descs;
    for (auto& r : reqs) descs.push_back(r.m->d);
    size_t need = 0;
    for (auto& r : reqs) need += r.bytes;
    // layout: models image, then tables and results; the image is packed
    // once to size the allocation (against a placeholder base, never
    // dereferenced) and again against the allocation
    ModelImage probe;
    pack_models_image(descs.data(), (int)descs.size(), reinterpret_cast<char*>(uintptr_t(1) << 20), probe);
    auto r16 = [](size_t x) { return (x + 255) & ~(size_t)255; };
    size_t nchains = 0, nconf = 0, nxyz = 0;
    for (size_t k = 0; k < reqs.size(); k++) {
        const DModel& h = probe.host[k];
        nchains += reqs[k].job.num_chains;
        nconf += (size_t)reqs[k].job.num_chains * S * h.conf_size;
        nxyz += (size_t)reqs[k].job.num_chains * S * h.nheavy * 3;
    }
    size_t at = r16(probe.bytes.size());
    const size_t maps_at = at; at = r16(at + SG_MAX_RECEPTORS * sizeof(DMaps32));
    const size_t boxes_at = at; at = r16(at + SG_MAX_RECEPTORS * 6 * sizeof(double));
    const size_t chains_at = at; at = r16(at + nchains * sizeof(Chain32));
    const size_t cnt_at = at; at = r16(at + reqs.size() * sizeof(unsigned));
    b->e_at = at; at = r16(at + nchains * S * sizeof(double));
    b->conf_at = at; at = r16(at + nconf * sizeof(double));
    b->xyz_at = at; at = r16(at + nxyz * sizeof(float));
    b->order_at = at; at = r16(at + nchains * S * sizeof(int));
    b->count_at = at; at = r16(at + nchains * sizeof(int));
    b->evals_at = at; at = r16(at + nchains * 2 * sizeof(unsigned long long));
    const size_t hits_at = at; at = r16(at + nchains * 2 * sizeof(unsigned long long));
    b->span_at = at; at = r16(at + nchains * 2 * sizeof(unsigned long long));
    const size_t params_at = at; at = r16(at + sizeof(MCParams32));
    b->bytes = std::max(at, need);
    b->seq = ++s.launches;
    cuda_check(cudaMallocAsync((void**)&b->dmem, b->bytes, s.feed_stream), "serve: batch memory");
    pack_models_image(descs.data(), (int)descs.size(), b->dmem, b->img);
    // map sets and search boxes of every receptor
    std::vector<DMaps32> tab(SG_MAX_RECEPTORS);
    std::vector<double> boxes(SG_MAX_RECEPTORS * 6, 0.0);
    for (int rid = 0; rid < SG_MAX_RECEPTORS; rid++) {
        const RecState& r = e->rec[rid];
        bool any = false;
        for (int t = 0; t < kNumTypes; t++) any = any || r.map32[t].p != nullptr;
        if (!r.set || !any) continue;
        tab[rid] = maps32(e, r);
        for (int i = 0; i < 3; i++) {
            boxes[rid * 6 + i] = r.gd.begin[i];
            boxes[rid * 6 + 3 + i] = r.gd.end[i];
        }
    }
    // chains, items (longest first) and the ligands' slots
    size_t ws_stride = 0, stage_stride = 0;
    int max_chains = 1;
    for (const DModel& h : b->img.host) {
        ws_stride = std::max(ws_stride, ws32_bytes(h));
        stage_stride = std::max(stage_stride, (size_t)stage32_bytes(h.natoms, h.nframes, h.nheavy, h.npchunks, h.nlig,
                                                                    h.nblocks, h.ntors));
    }
    ws_stride = (ws_stride + 15) & ~(size_t)15;
    for (auto& r : reqs) max_chains = std::max(max_chains, r.job.num_chains);
    // the most chains per block (8-warp blocks, chains on teams of g warps)
    // that fit the server's fixed shared memory per block
    auto chains_per_block = [&](int g) {
        for (int c : {8, 4, 2, 1}) {
            if (c * g > 8) continue;
            if (e->force_wpb && c != e->force_wpb) continue;
            if (!e->force_wpb && c > 1 && c / 2 >= max_chains) continue;
            if (stage_stride + (size_t)c * g * ws_stride <= s.smem_block) return c;
        }
        return 0;
    };
    // Threads per chain: the engine's setting, or (0) the most warps per
    // chain (128, 64) at which the items in flight and this batch's all
    // have a block at once, so that a lone ligand's chains run shorter.
    int team = std::max(1, e->tpc / 32);
    if (e->tpc == 0) {
        team = 1;
        for (int g : {4, 2}) {
            const int c = chains_per_block(g);
            if (!c) continue;
            long long nb = 0;
            for (auto& r : reqs) nb += (r.job.num_chains + c - 1) / c;
            if (s.inflight_blocks + nb <= s.target_blocks) {
                team = g;
                break;
            }
        }
    }
    require(!e->force_wpb || e->force_wpb * team <= 8,
            "serve: chains per block (sg_set_chains_per_block) times warps per chain is above 8 warps per block");
    const int wpb = chains_per_block(team);
    require(wpb > 0, "serve: model too large for the mixed-precision path's shared memory at this many threads per chain");
    std::vector<Item32> items;
    std::vector<double> cost;
    size_t conf_off = 0, xyz_off = 0;
    for (size_t k = 0; k < reqs.size(); k++) {
        const DModel& h = b->img.host[k];
        SvLig L;
        L.req = std::move(reqs[k]);
        L.model = (int)k;
        L.first = (int)b->hc.size();
        L.nchains = L.req.job.num_chains;
        require(!s.free_flags.empty(), "serve: too many ligands in flight");
        L.flag = s.free_flags.back();
        s.free_flags.pop_back();
        s.flags[L.flag] = 0u;
        L.conf_off = conf_off;
        L.xyz_off = xyz_off;
        L.batch = b.get();
        L.launch = b->seq;
        L.team = team;
        L.t_launch = Clock::now();
        const sg_ligand_job& J = L.req.job;
        for (int c = 0; c < J.num_chains; c++) {
            Chain32 ch{};
            ch.model = (int)k;
            ch.steps = J.num_steps;
            ch.maxiters = J.maxiters > 0 ? J.maxiters : L.req.p.maxiters;
            ch.key0 = (uint32_t)J.seed;
            ch.key1 = (uint32_t)(J.seed >> 32) ^ (uint32_t)(J.ligand_key >> 32);
            ch.lig = (uint32_t)J.ligand_key;
            ch.chain = (uint32_t)c;
            const size_t kc = b->hc.size();
            ch.out_e = reinterpret_cast<double*>(b->dmem + b->e_at) + kc * S;
            ch.out_conf = reinterpret_cast<double*>(b->dmem + b->conf_at) + conf_off;
            ch.out_coords = reinterpret_cast<float*>(b->dmem + b->xyz_at) + xyz_off;
            ch.out_order = reinterpret_cast<int*>(b->dmem + b->order_at) + kc * S;
            ch.out_count = reinterpret_cast<int*>(b->dmem + b->count_at) + kc;
            ch.evals = reinterpret_cast<unsigned long long*>(b->dmem + b->evals_at) + kc;
            ch.hits = reinterpret_cast<unsigned long long*>(b->dmem + hits_at) + 2 * kc;
            ch.done_count = reinterpret_cast<unsigned*>(b->dmem + cnt_at) + k;
            ch.host_flag = s.dflags + L.flag;
            ch.lig_chains = J.num_chains;
            ch.box = reinterpret_cast<const double*>(b->dmem + boxes_at) + 6 * L.req.rid;
            ch.span = reinterpret_cast<unsigned long long*>(b->dmem + b->span_at) + 2 * kc;
            b->hc.push_back(ch);
            conf_off += (size_t)S * h.conf_size;
            xyz_off += (size_t)S * h.nheavy * 3;
        }
        for (int c0 = 0; c0 < J.num_chains; c0 += wpb) {
            items.push_back(Item32{(int)k, L.first + c0, std::min(wpb, J.num_chains - c0), L.req.rid});
            cost.push_back((double)J.num_steps * h.cost * std::max(1, b->hc[L.first].maxiters));
            L.blocks++;
        }
        s.inflight_blocks += L.blocks;
        b->ligs.push_back(std::move(L));
    }
    std::vector<int> order(items.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return cost[a] > cost[c]; });
    std::vector<Item32> q(items.size());
    for (size_t k = 0; k < items.size(); k++) q[k] = items[order[k]];
    cudaStream_t st = s.feed_stream;
    cuda_check(cudaMemcpyAsync(b->dmem, b->img.bytes.data(), b->img.bytes.size(), cudaMemcpyHostToDevice, st), "serve");
    cuda_check(cudaMemcpyAsync(b->dmem + maps_at, tab.data(), tab.size() * sizeof(DMaps32), cudaMemcpyHostToDevice, st),
               "serve");
    cuda_check(cudaMemcpyAsync(b->dmem + boxes_at, boxes.data(), boxes.size() * sizeof(double), cudaMemcpyHostToDevice,
                               st),
               "serve");
    cuda_check(cudaMemcpyAsync(b->dmem + chains_at, b->hc.data(), b->hc.size() * sizeof(Chain32),
                               cudaMemcpyHostToDevice, st),
               "serve");
    cuda_check(cudaMemsetAsync(b->dmem + cnt_at, 0, reqs.size() * sizeof(unsigned) + 16, st), "serve");
    MCParams32 P{};
    for (int i = 0; i < 3; i++) {
        P.hunt[i] = (float)p.hunt_cap[i];
        P.auth[i] = (float)p.authentic_v[i];
        P.box[i] = 0;
        P.box[3 + i] = 0;
    }
    P.slope = (float)p.cache_slope;
    P.temperature = p.temperature;
    P.amplitude = p.mutation_amplitude;
    P.min_rmsd = p.min_rmsd;
    P.num_saved = S;
    P.maxiters = p.maxiters;
    P.accurate_line = p.accurate_line;
    P.early_term = p.early_term;
    // the batch's items, in cost order, into the ring; then the tail word.
    // Everything goes through the one feed stream, so the grid sees a tail
    // only after the data it covers has landed.
    const unsigned n = (unsigned)q.size();
    require(s.tail + n - s.seen.head <= Server::kRing, "serve: work ring full");
    const size_t pin_bytes = r16(sizeof(MCParams32)) + n * sizeof(FeedItem32) + 16;
    b->pin = pin_get(s, pin_bytes, b->pin_cap);
    std::memcpy(b->pin, &P, sizeof(MCParams32));
    FeedItem32* fi = reinterpret_cast<FeedItem32*>(b->pin + r16(sizeof(MCParams32)));
    const DModel* dms = reinterpret_cast<const DModel*>(b->dmem + b->img.dmodel_off);
    const Chain32* dch = reinterpret_cast<const Chain32*>(b->dmem + chains_at);
    const DMaps32* dmaps = reinterpret_cast<const DMaps32*>(b->dmem + maps_at);
    for (unsigned k = 0; k < n; k++) {
        fi[k] = FeedItem32{dms + q[k].model, dch + q[k].first, dmaps + q[k].rec,
                           reinterpret_cast<const MCParams32*>(b->dmem + params_at), q[k].count, (int)stage_stride,
                           (int)ws_stride, team};
    }
    unsigned* tail_word = reinterpret_cast<unsigned*>(b->pin + r16(sizeof(MCParams32)) + n * sizeof(FeedItem32));
    *tail_word = s.tail + n;
    cuda_check(cudaMemcpyAsync(b->dmem + params_at, b->pin, sizeof(MCParams32), cudaMemcpyHostToDevice, st), "serve");
    const unsigned at0 = s.tail % Server::kRing, first_part = std::min(n, Server::kRing - at0);
    cuda_check(cudaMemcpyAsync(s.d_ring + at0, fi, first_part * sizeof(FeedItem32), cudaMemcpyHostToDevice, st), "serve");
    if (first_part < n)
        cuda_check(cudaMemcpyAsync(s.d_ring, fi + first_part, (n - first_part) * sizeof(FeedItem32),
                                   cudaMemcpyHostToDevice, st),
                   "serve");
    cuda_check(cudaMemcpyAsync(&s.d_ctrl->tail, tail_word, sizeof(unsigned), cudaMemcpyHostToDevice, st), "serve");
    s.tail += n;
    s.inflight_bytes += b->bytes;
    s.inflight_ligs += (int)b->ligs.size();
    s.inflight.push_back(std::move(b));
}

static char* pin_get(Server& s, size_t bytes, size_t& cap) {
    for (size_t i = 0; i < s.pin_free.size(); i++)
        if (s.pin_free[i].first >= bytes) {
            char* p = s.pin_free[i].second;
            cap = s.pin_free[i].first;
            s.pin_free.erase(s.pin_free.begin() + i);
            return p;
        }
    cap = std::max<size_t>(bytes, 1 << 20);
    char* p = nullptr;
    cuda_check(cudaHostAlloc((void**)&p, cap, cudaHostAllocDefault), "serve: pinned staging");
    s.pin_all.push_back(p);
    return p;
}
static void pin_put(Server& s, char* p, size_t cap) {
    if (p) s.pin_free.emplace_back(cap, p);
}

// A ligand's chains are done: copy their containers back and merge them.
static void fetch_merge(Server& s, SvBatch& b, SvLig& L) {
    L.t_flag = Clock::now();
    s.inflight_blocks -= L.blocks;
    const DModel& h = b.img.host[L.model];
    const int S = b.S, cs = h.conf_size, H = h.nheavy;
    const size_t nc = L.nchains;
    // one pinned staging buffer for the ligand's chain results
    auto r16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    const size_t eb = nc * S * sizeof(double), cb = (size_t)nc * S * cs * sizeof(double),
                 xb = (size_t)nc * S * H * 3 * sizeof(float), ob = nc * S * sizeof(int), nb = nc * sizeof(int),
                 vb = nc * sizeof(unsigned long long), sb = 2 * vb;
    const size_t c_at = r16(eb), x_at = c_at + r16(cb), o_at = x_at + r16(xb), n_at = o_at + r16(ob),
                 v_at = n_at + r16(nb), s_at = v_at + r16(vb), total = s_at + r16(sb);
    size_t cap = 0;
    char* hb = pin_get(s, total, cap);
    const double* he = reinterpret_cast<const double*>(hb);
    const double* hconf = reinterpret_cast<const double*>(hb + c_at);
    const float* hxyz = reinterpret_cast<const float*>(hb + x_at);
    const int* horder = reinterpret_cast<const int*>(hb + o_at);
    const int* hcount = reinterpret_cast<const int*>(hb + n_at);
    const unsigned long long* hev = reinterpret_cast<const unsigned long long*>(hb + v_at);
    const unsigned long long* hspan = reinterpret_cast<const unsigned long long*>(hb + s_at);
    cudaStream_t cp = s.copy_stream;
    auto get = [&](size_t to, size_t from, size_t bytes) {
        if (bytes)
            cuda_check(cudaMemcpyAsync(hb + to, b.dmem + from, bytes, cudaMemcpyDeviceToHost, cp), "serve: fetch");
    };
    get(0, b.e_at + (size_t)L.first * S * sizeof(double), eb);
    get(c_at, b.conf_at + L.conf_off * sizeof(double), cb);
    get(x_at, b.xyz_at + L.xyz_off * sizeof(float), xb);
    get(o_at, b.order_at + (size_t)L.first * S * sizeof(int), ob);
    get(n_at, b.count_at + (size_t)L.first * sizeof(int), nb);
    get(v_at, b.evals_at + (size_t)L.first * sizeof(unsigned long long), vb);
    get(s_at, b.span_at + (size_t)L.first * 2 * sizeof(unsigned long long), sb);
    const cudaError_t rc = cudaStreamSynchronize(cp);
    if (rc != cudaSuccess) pin_put(s, hb, cap);
    cuda_check(rc, "serve: fetch");
    for (size_t k = 0; k < nc; k++) {
        L.evals += hev[k];
        L.dev_start = k == 0 ? hspan[0] : std::min<uint64_t>(L.dev_start, hspan[2 * k]);
        L.dev_end = std::max<uint64_t>(L.dev_end, hspan[2 * k + 1]);
        const int cnt = std::min(std::max(hcount[k], 0), S);
        for (int i = 0; i < cnt; i++) {
            const int slot = horder[k * S + i];
            if (slot < 0 || slot >= S) continue;
            SvPose t;
            t.e = he[k * S + slot];
            const double* c = &hconf[(k * S + slot) * cs];
            t.conf.assign(c, c + cs);
            const float* x = &hxyz[(k * S + slot) * H * 3];
            t.xyz.assign(x, x + (size_t)H * 3);
            sv_add_pose(L.poses, std::move(t), 2.0, S);
        }
    }
    pin_put(s, hb, cap);
}

// One FP64 refinement launch for the merged poses of every ligand that
// finished since the last one (ligands of any batch and receptor).
struct RefineGroup {
    std::vector<SvLig*> ligs;
    std::vector<int> first;  // first pose of each ligand
    std::vector<double> conf;  // the merged poses' confs, built on the host
    int cs = 0, hs = 1;
    void* dbuf = nullptr;
    cudaEvent_t ev = nullptr;
    char* pin = nullptr;  // pinned copy of the device buffer's layout
    size_t pin_cap = 0;
    const double *out_conf = nullptr, *out_e = nullptr, *out_xyz = nullptr;  // results, in pin
};

static void launch_refines(Server& s, std::vector<std::pair<SvBatch*, SvLig*>>& fin) {
    sg_engine* e = s.e;
    auto g = std::make_unique<RefineGroup>();
    std::vector<DModel> dms;
    std::vector<int> pose_model, pose_maxit;
    std::vector<DReceptor*> recs;
    size_t ws = 0;
    int np = 0;
    for (auto& [b, L] : fin) {
        const DModel& h = b->img.host[L->model];
        g->cs = std::max(g->cs, h.conf_size);
        g->hs = std::max(g->hs, h.nheavy);
        ws = std::max(ws, ws64_bytes(h));
    }
    require(ws <= (size_t)e->max_smem, "serve: model too large for the plain path's shared memory");
    // refine_structure needs the pose's receptor: one launch per receptor in the group
    std::map<int, std::vector<std::pair<SvBatch*, SvLig*>>> by_rec;
    for (auto& f : fin) by_rec[f.second->req.rid].push_back(f);
    for (auto& [rid, members] : by_rec) {
        for (auto& [b, L] : members) {
            const int m = (int)dms.size();
            dms.push_back(b->img.host[L->model]);
            g->ligs.push_back(L);
            g->first.push_back(np);
            const int mi = L->req.job.maxiters > 0 ? L->req.job.maxiters : L->req.p.maxiters;
            for (const SvPose& t : L->poses) {
                g->conf.insert(g->conf.end(), t.conf.begin(), t.conf.end());
                g->conf.resize((size_t)(np + 1) * g->cs, 0.0);
                pose_model.push_back(m);
                pose_maxit.push_back(mi);
                np++;
            }
            L->state = 1;
        }
    }
    g->first.push_back(np);
    if (np == 0) {
        for (SvLig* L : g->ligs) L->state = 3;  // nothing to refine: publish as is
        s.refining.push_back(std::move(g));
        return;
    }
    const size_t cb = g->conf.size() * sizeof(double), eb = (size_t)np * sizeof(double),
                 xb = (size_t)np * g->hs * 3 * sizeof(double), ib = (size_t)np * sizeof(int),
                 mb = dms.size() * sizeof(DModel);
    cudaStream_t rs = s.refine_stream;
    const size_t total = cb + eb + xb + 2 * ib + mb + 256;
    cuda_check(cudaMallocAsync(&g->dbuf, total, rs), "serve: refine memory");
    // the same layout in a pinned buffer: one copy in, one copy of the results out
    const size_t c_at = (mb + 15) & ~(size_t)15, pm_at = c_at + cb + eb + xb;
    g->pin = pin_get(s, total, g->pin_cap);
    std::memcpy(g->pin, dms.data(), mb);
    std::memcpy(g->pin + c_at, g->conf.data(), cb);
    std::memcpy(g->pin + pm_at, pose_model.data(), ib);
    std::memcpy(g->pin + pm_at + ib, pose_maxit.data(), ib);
    char* base = static_cast<char*>(g->dbuf);
    DModel* d_models = reinterpret_cast<DModel*>(base);
    double* dc = reinterpret_cast<double*>(base + c_at);
    double* de = dc + g->conf.size();
    double* dx = de + np;
    int* dpm = reinterpret_cast<int*>(base + pm_at);
    int* dmi = dpm + np;
    cuda_check(cudaMemcpyAsync(base, g->pin, pm_at + 2 * ib, cudaMemcpyHostToDevice, rs), "serve");
    int p0 = 0;
    for (auto& [rid, members] : by_rec) {
        int n = 0;
        for (auto& [b, L] : members) n += (int)L->poses.size();
        if (n > 0) {
            const sg_mc_params& P = members[0].second->req.p;
            cuda_check(launch_refine64(d_models, ws, e->tables, e->rec[rid].dhdr.as<DReceptor>(), dpm + p0, n,
                                       dc + (size_t)p0 * g->cs, g->cs, P.authentic_v, P.maxiters, dmi + p0, nullptr,
                                       P.accurate_line, P.early_term, de + p0, dx + (size_t)p0 * g->hs * 3, g->hs,
                                       s.d_err, rs),
                       "serve: refine launch");
        }
        p0 += n;
    }
    cuda_check(cudaMemcpyAsync(g->pin + c_at, dc, cb + eb + xb, cudaMemcpyDeviceToHost, rs), "serve");
    g->out_conf = reinterpret_cast<const double*>(g->pin + c_at);
    g->out_e = g->out_conf + g->conf.size();
    g->out_xyz = g->out_e + np;
    cuda_check(cudaMemcpyAsync((void*)s.h_err, s.d_err, sizeof(int), cudaMemcpyDeviceToHost, rs), "serve");
    cuda_check(cudaFreeAsync(g->dbuf, rs), "serve");
    g->dbuf = nullptr;
    cuda_check(cudaEventCreateWithFlags(&g->ev, cudaEventDisableTiming), "serve");
    cuda_check(cudaEventRecord(g->ev, rs), "serve");
    s.refining.push_back(std::move(g));
}

// The refinement is done: publish the result.  mu held.
static void publish(Server& s, const RefineGroup& g, size_t k) {
    SvLig& L = *g.ligs[k];
    const int np = (int)L.poses.size();
    const int cs = L.poses.empty() ? 0 : (int)L.poses[0].conf.size();
    const int H = L.poses.empty() ? 0 : (int)L.poses[0].xyz.size() / 3;
    ServeDone d;
    d.info.ticket = L.req.ticket;
    d.info.status = SG_OK;
    d.info.conf_size = L.req.m->d.conf_size;
    d.info.num_heavy = H;
    d.info.evals = L.evals;
    d.info.launch = L.launch;
    d.info.queue_ms = std::chrono::duration<double, std::milli>(L.t_launch - L.req.t_submit).count();
    d.info.searched_ms = std::chrono::duration<double, std::milli>(L.t_flag - L.req.t_submit).count();
    d.info.threads_per_chain = 32 * L.team;
    d.info.device_start_ns = L.dev_start;
    d.info.device_end_ns = L.dev_end;
    for (int i = 0; i < np; i++) {
        const size_t q = (size_t)g.first[k] + i;
        L.poses[i].e = g.out_e[q];
        std::memcpy(L.poses[i].conf.data(), &g.out_conf[q * g.cs], cs * sizeof(double));
        L.poses[i].xyz.assign(&g.out_xyz[q * g.hs * 3], &g.out_xyz[q * g.hs * 3] + (size_t)H * 3);
    }
    std::stable_sort(L.poses.begin(), L.poses.end(), [](const SvPose& a, const SvPose& c) { return a.e < c.e; });
    d.info.count = np;
    for (const SvPose& t : L.poses) {
        d.e.push_back(t.e);
        d.conf.insert(d.conf.end(), t.conf.begin(), t.conf.end());
        d.coords.insert(d.coords.end(), t.xyz.begin(), t.xyz.end());
    }
    d.info.latency_ms = std::chrono::duration<double, std::milli>(Clock::now() - L.req.t_submit).count();
    s.done[L.req.ticket] = std::move(d);
    s.done_order.push_back(L.req.ticket);
    L.state = 2;
    s.free_flags.push_back(L.flag);
    s.inflight_ligs--;
}

static void fail_all(Server& s, int code, const std::string& why) {
    s.error = code;
    s.error_text = why;
    auto fail = [&](uint64_t ticket, Clock::time_point t0) {
        ServeDone d;
        d.info.ticket = ticket;
        d.info.status = code;
        d.info.latency_ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
        s.done[ticket] = std::move(d);
        s.done_order.push_back(ticket);
    };
    for (auto& b : s.inflight)
        for (auto& L : b->ligs)
            if (L.state != 2) fail(L.req.ticket, L.req.t_submit);
    for (auto& r : s.queue) fail(r.ticket, r.t_submit);
    s.queue.clear();
    s.inflight.clear();
    s.refining.clear();
    s.inflight_bytes = 0;
    s.inflight_blocks = 0;
    s.cv_done.notify_all();
}

// true once the event has completed; throws on a device error
static bool event_done(cudaEvent_t ev) {
    const cudaError_t q = cudaEventQuery(ev);
    if (q == cudaErrorNotReady) return false;
    cuda_check(q, "serve: event");
    return true;
}

static void worker(Server* sp) {
    Server& s = *sp;
    cudaSetDevice(s.e->device);
    std::unique_lock<std::mutex> lk(s.mu);
    for (;;) {
        bool busy = false;
        try {
            // 0. serving grids: a snapshot of the ring's control words (an
            // async copy, read once it has landed); blocks are started when
            // items wait and no block is free, counting blocks launched but
            // not yet seen to start, and only on a snapshot taken after the
            // last start
            if (!s.ctrl_pending) {
                cuda_check(cudaMemcpyAsync(s.h_ctrl, s.d_ctrl, sizeof(FeedCtrl32), cudaMemcpyDeviceToHost,
                                           s.ctrl_stream),
                           "serve: control words");
                cuda_check(cudaEventRecord(s.ctrl_ev, s.ctrl_stream), "serve: control words");
                s.ctrl_pending = true;
                s.snap_req++;
            } else if (event_done(s.ctrl_ev)) {
                s.ctrl_pending = false;
                s.seen = *s.h_ctrl;
                s.snap_seen = s.snap_req;
            }
            if (s.tail != s.seen.head && s.seen.waiting == 0 && s.snap_seen > s.launch_req) {
                const int live = (int)(s.blocks_launched - s.seen.exited);
                const int more = s.target_blocks - live;
                if (more > 0) {
                    cudaStream_t gs = nullptr;
                    for (cudaStream_t c : s.grid_streams)
                        if (cudaStreamQuery(c) == cudaSuccess) { gs = c; break; }
                    if (!gs && s.grid_streams.size() < 32) {
                        cuda_check(cudaStreamCreateWithFlags(&gs, cudaStreamNonBlocking), "serve: stream");
                        s.grid_streams.push_back(gs);
                    }
                    if (gs) {
                        cuda_check(launch_mc32_feed(tables32(s.e), s.d_ring, Server::kRing, s.d_ctrl, s.idle_ns, more, 8,
                                                    s.smem_block, gs),
                                   "serve: search grid");
                        s.blocks_launched += (unsigned)more;
                        s.launch_req = s.snap_req;
                        busy = true;
                    }
                }
            }
            // 1. upload.  At most max_inflight_ligands ligands are on the device;
            // the rest wait here.  While more requests wait than the device can
            // take, a batch goes out as soon as any fits; when everything
            // queued fits, it goes once a full batch has queued or the oldest
            // request has waited max_wait_ms for others to share it.  Same
            // search parameters per batch; device memory held for requests in
            // flight stays under the budget.
            if (!s.queue.empty()) {
                const double waited =
                    std::chrono::duration<double, std::milli>(Clock::now() - s.queue.front().t_submit).count();
                const int open = std::max(0, s.o.max_inflight_ligands - s.inflight_ligs);
                const int q = (int)s.queue.size();
                const int want = std::min({q, open, s.o.max_batch_ligands, (int)s.free_flags.size()});
                const bool go = want > 0 && (q > open || want >= s.o.max_batch_ligands || s.stopping ||
                                             waited >= s.o.max_wait_ms);
                if (go) {
                    std::vector<ServeReq> take;
                    size_t bytes = 0;
                    const int cap = want;
                    size_t t_stage = 0, t_ws = 0;
                    int t_chains = 1, t_shape = 0;
                    while (!s.queue.empty() && (int)take.size() < cap) {
                        ServeReq& r = s.queue.front();
                        if (!take.empty() && !same_params(r.p, take[0].p)) break;
                        // ligands that would force fewer chains per block on the
                        // launch wait for one of their own
                        const size_t n_stage = std::max(t_stage, r.stage), n_ws = std::max(t_ws, r.ws);
                        const int n_chains = std::max(t_chains, r.job.num_chains);
                        const int shape = serve_shape(s, n_stage, n_ws, n_chains);
                        if (!take.empty() && shape < t_shape) break;
                        t_stage = n_stage;
                        t_ws = n_ws;
                        t_chains = n_chains;
                        t_shape = shape;
                        if (s.inflight_bytes + bytes + r.bytes > s.o.hbm_budget_bytes &&
                            !(take.empty() && s.inflight.empty()))
                            break;
                        bytes += r.bytes;
                        take.push_back(std::move(r));
                        s.queue.pop_front();
                    }
                    if (!take.empty()) {
                        launch_batch(s, std::move(take));
                        busy = true;
                    }
                }
            }
            // 2. ligands whose chains are done: merge, then one refinement launch for all
            std::vector<std::pair<SvBatch*, SvLig*>> fin;
            for (auto& b : s.inflight)
                for (auto& L : b->ligs)
                    if (L.state == 0 && s.flags[L.flag]) {
                        fetch_merge(s, *b, L);
                        fin.emplace_back(b.get(), &L);
                        ++b->flagged;
                    }
            if (!fin.empty()) {
                launch_refines(s, fin);
                busy = true;
            }
            // refinements that finished: publish their ligands
            for (size_t i = 0; i < s.refining.size();) {
                RefineGroup& g = *s.refining[i];
                if (!g.ev || event_done(g.ev)) {
                    for (size_t k = 0; k < g.ligs.size(); k++) {
                        publish(s, g, k);
                        g.ligs[k]->batch->published++;
                    }
                    if (g.ev) cudaEventDestroy(g.ev);
                    pin_put(s, g.pin, g.pin_cap);
                    s.refining.erase(s.refining.begin() + i);
                    s.cv_done.notify_all();
                    busy = true;
                } else {
                    i++;
                }
            }
            // 3. retire batches whose ligands are all published (their chains
            // have signalled completion, their last access to the batch)
            for (size_t i = 0; i < s.inflight.size();) {
                SvBatch& b = *s.inflight[i];
                if (b.flagged == (int)b.ligs.size() && b.published == (int)b.ligs.size()) {
                    cuda_check(cudaFreeAsync(b.dmem, s.feed_stream), "serve: free batch");
                    pin_put(s, b.pin, b.pin_cap);
                    s.inflight_bytes -= b.bytes;
                    s.inflight.erase(s.inflight.begin() + i);
                    busy = true;
                } else {
                    i++;
                }
            }
            // device errors (overlap in a refinement) end the server; the pinned
            // copy is read without a CUDA call, so nothing waits on running kernels
            if (!busy && Clock::now() - s.last_err_check > std::chrono::milliseconds(10)) {
                s.last_err_check = Clock::now();
                const int herr = *s.h_err;
                if (herr != kDevOk)
                    throw EngineError(herr == kDevOverlap ? SG_ERR_OVERLAP : SG_ERR_ARG,
                                      "serve: device reported error " + std::to_string(herr));
                // a grid that failed on the device never raises its flags: its
                // stream reports the error instead
                for (cudaStream_t c : s.grid_streams) {
                    const cudaError_t q = cudaStreamQuery(c);
                    if (q != cudaSuccess && q != cudaErrorNotReady) cuda_check(q, "serve: search grid");
                }
            }
        } catch (EngineError& x) {
            fail_all(s, x.code, x.what());
        } catch (std::exception& x) {
            fail_all(s, SG_ERR_ARG, x.what());
        }
        if (s.stopping && s.queue.empty() && s.inflight.empty() && s.refining.empty()) break;
        // let submit / poll in between passes, busy or not
        lk.unlock();
        if (busy) std::this_thread::yield();
        else std::this_thread::sleep_for(std::chrono::microseconds(100));
        lk.lock();
    }
}

// Ends the serving grids (their blocks see stop within one sleep step, or
// leave after their idle time) and frees the ring.
static void stop_grids(Server& s) {
    if (s.d_ctrl) {
        const unsigned one = 1;
        cudaMemcpy(&s.d_ctrl->stop, &one, sizeof(unsigned), cudaMemcpyHostToDevice);
    }
    for (cudaStream_t c : s.grid_streams) {
        cudaStreamSynchronize(c);
        cudaStreamDestroy(c);
    }
    s.grid_streams.clear();
    if (s.feed_stream) cudaStreamSynchronize(s.feed_stream);
    if (s.ctrl_stream) cudaStreamSynchronize(s.ctrl_stream);
    if (s.feed_stream) cudaStreamDestroy(s.feed_stream);
    if (s.ctrl_stream) cudaStreamDestroy(s.ctrl_stream);
    if (s.ctrl_ev) cudaEventDestroy(s.ctrl_ev);
    if (s.d_ring) cudaFree(s.d_ring);
    if (s.d_ctrl) cudaFree(s.d_ctrl);
    if (s.h_ctrl) cudaFreeHost(s.h_ctrl);
    s.feed_stream = s.ctrl_stream = nullptr;
    s.ctrl_ev = nullptr;
    s.d_ring = nullptr;
    s.d_ctrl = nullptr;
    s.h_ctrl = nullptr;
}

}  // namespace sg

using namespace sg;

static std::mutex g_srv_mu;
static std::map<const sg_engine*, std::unique_ptr<Server>> g_servers;

static Server* server_of(const sg_engine* e) {
    std::lock_guard<std::mutex> lk(g_srv_mu);
    auto it = g_servers.find(e);
    return it == g_servers.end() ? nullptr : it->second.get();
}

// Stops the engine's server, if any (sg_destroy calls this first).
void sg::serve_shutdown(sg_engine* e) {
    Server* s = server_of(e);
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    if (s->th.joinable()) s->th.join();
    stop_grids(*s);
    std::lock_guard<std::mutex> lk(g_srv_mu);
    g_servers.erase(e);
}

extern "C" {

int sg_serve_start(sg_engine* e, const sg_serve_opts* o) {
    return guarded(e, [&] {
        require(e->precision != SG_PREC_FP64, "serve needs an engine created with SG_PREC_FP32 or SG_PREC_FP32_H16");
        require(e->has_tables, "no tables set");
        require(!server_of(e), "serve: already started");
        auto s = std::make_unique<Server>();
        s->e = e;
        if (o) s->o = *o;
        if (s->o.max_batch_ligands <= 0) s->o.max_batch_ligands = 64;
        if (s->o.max_wait_ms <= 0) s->o.max_wait_ms = 20.0;
        // resident 8-chain blocks, less a few slots so that refinements find room beside the search
        if (s->o.max_inflight_ligands <= 0) s->o.max_inflight_ligands = std::max(1, 2 * e->num_sms - 16);
        if (s->o.hbm_budget_bytes == 0) {
            size_t fr = 0, tot = 0;
            cuda_check(cudaMemGetInfo(&fr, &tot), "serve: memory info");
            s->o.hbm_budget_bytes = fr / 4;
        }
        // Every search launch takes the same shared memory per block, set once
        // here so that no kernel attribute changes while launches run.  By
        // default it is the most that still fits two blocks per SM (the SM's
        // shared memory, less per block the kernel's static shared memory and
        // the driver's reserve), so that the largest ligands also run eight
        // chains per block; block_smem_bytes overrides it.
        size_t dyn_max = 0, two_per_sm = 0;
        cuda_check(mc32_feed_max_dynamic_smem((size_t)e->max_smem, &dyn_max), "serve: kernel attributes");
        int per_sm = 0, reserved = 0;
        cuda_check(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, e->device), "serve");
        cuda_check(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, e->device), "serve");
        cuda_check(mc32_feed_max_dynamic_smem((size_t)std::max(0, per_sm / 2 - reserved), &two_per_sm), "serve");
        if (s->o.block_smem_bytes > 0) {
            require((size_t)s->o.block_smem_bytes <= dyn_max, "serve: block_smem_bytes above the device's limit");
            s->smem_block = (size_t)s->o.block_smem_bytes;
        } else {
            s->smem_block = std::min(dyn_max, two_per_sm & ~(size_t)1023);
        }
        require(s->smem_block >= 4096, "serve: too little shared memory per block");
        cuda_check(mc32_feed_reserve_smem(s->smem_block), "serve: kernel attributes");
        {   // serving blocks the device holds at once (8-warp blocks at the fixed
            // shared memory), less 16, so that the FP64 refinements find room
            int per = 0;
            cuda_check(mc32_feed_occupancy(8, s->smem_block, &per), "serve: occupancy");
            require(per > 0, "serve: the serving block does not fit an SM");
            s->target_blocks = std::max(1, per * e->num_sms - 16);
        }
        cuda_check(cudaMalloc((void**)&s->d_ring, (size_t)Server::kRing * sizeof(FeedItem32)), "serve: work ring");
        cuda_check(cudaMalloc((void**)&s->d_ctrl, sizeof(FeedCtrl32)), "serve: work ring");
        cuda_check(cudaMemset(s->d_ctrl, 0, sizeof(FeedCtrl32)), "serve: work ring");
        cuda_check(cudaHostAlloc((void**)&s->h_ctrl, sizeof(FeedCtrl32), cudaHostAllocDefault), "serve: work ring");
        std::memset(s->h_ctrl, 0, sizeof(FeedCtrl32));
        cuda_check(cudaEventCreateWithFlags(&s->ctrl_ev, cudaEventDisableTiming), "serve: event");
        cuda_check(cudaStreamCreateWithFlags(&s->feed_stream, cudaStreamNonBlocking), "serve: stream");
        cuda_check(cudaStreamCreateWithFlags(&s->ctrl_stream, cudaStreamNonBlocking), "serve: stream");
        cuda_check(cudaStreamCreateWithFlags(&s->refine_stream, cudaStreamNonBlocking), "serve: stream");
        cuda_check(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking), "serve: stream");
        unsigned* hf = nullptr;
        cuda_check(cudaHostAlloc((void**)&hf, Server::kFlags * sizeof(unsigned), cudaHostAllocMapped), "serve: flags");
        std::memset(hf, 0, Server::kFlags * sizeof(unsigned));
        s->flags = hf;
        cuda_check(cudaHostGetDevicePointer((void**)&s->dflags, hf, 0), "serve: flags");
        for (int i = Server::kFlags - 1; i >= 0; i--) s->free_flags.push_back(i);
        cuda_check(cudaMalloc((void**)&s->d_err, sizeof(int)), "serve: error word");
        cuda_check(cudaMemset(s->d_err, 0, sizeof(int)), "serve: error word");
        int* he = nullptr;
        cuda_check(cudaHostAlloc((void**)&he, sizeof(int), cudaHostAllocDefault), "serve: error word");
        *he = kDevOk;
        s->h_err = he;
        Server* raw = s.get();
        {
            std::lock_guard<std::mutex> lk(g_srv_mu);
            g_servers[e] = std::move(s);
        }
        raw->th = std::thread(worker, raw);
    });
}

int sg_serve_submit(sg_engine* e, int rid, const sg_model_desc* m, const sg_ligand_job* job, const sg_mc_params* p,
                    uint64_t* ticket) {
    return guarded(e, [&] {
        Server* s = server_of(e);
        require(s, "serve: not started");
        require(m && job && p && ticket, "serve: bad arguments");
        require(job->num_chains >= 1 && job->num_chains <= 4096 && job->maxiters >= 0, "serve: bad ligand job");
        require(p->num_saved_mins >= 1 && p->num_saved_mins <= 1024 && p->temperature > 0, "serve: bad search parameters");
        require(!p->visited, "the QuickVina 2 history (visited) runs on the plain path only");
        require(m->num_atoms <= 255, "mixed-precision path: at most 255 atoms per model");
        RecState& r = receptor_for(e, rid);
        ServeReq q;
        q.m = std::make_shared<ModelCopy>(*m);
        q.rid = rid;
        q.job = *job;
        q.job.model = 0;
        q.p = *p;
        q.bytes = req_bytes(*m, *job, p->num_saved_mins);
        {   // its staged model and workspace in shared memory (the launch shape it needs)
            ModelImage probe;
            pack_models_image(m, 1, reinterpret_cast<char*>(uintptr_t(1) << 20), probe);  // never dereferenced
            const DModel& h = probe.host[0];
            require(h.npchunks >= 0, "mixed-precision path: at most 255 atoms per model");
            q.ws = (ws32_bytes(h) + 15) & ~(size_t)15;
            q.stage = (size_t)stage32_bytes(h.natoms, h.nframes, h.nheavy, h.npchunks, h.nlig, h.nblocks, h.ntors);
            require(serve_shape(*s, q.stage, q.ws, job->num_chains) > 0,
                    "serve: model too large for the mixed-precision path's shared memory");
        }
        std::unique_lock<std::mutex> lk(s->mu);
        require(s->error == SG_OK, "serve: stopped after an error: " + s->error_text);
        require(!s->stopping, "serve: stopping");
        require(q.bytes <= s->o.hbm_budget_bytes, "serve: the request needs more device memory than the budget");
        lk.unlock();
        // the receptor's maps for this ligand's types (built once, then resident)
        {
            std::vector<int> types;
            for (int i = 0; i < m->num_movable; i++)
                if (m->atom_type[i] < kNumTypes && !is_h(m->atom_type[i])) types.push_back(m->atom_type[i]);
            bool missing = false;
            for (int t : types) missing = missing || !r.built[t];
            if (missing) {
                lk.lock();  // the worker reads receptor state while launching
                ensure_maps(e, r, types.data(), (int)types.size());
                lk.unlock();
            }
        }
        lk.lock();
        q.ticket = s->next_ticket++;
        q.t_submit = Clock::now();
        *ticket = q.ticket;
        s->queue.push_back(std::move(q));
    });
}

int sg_serve_poll(sg_engine* e, sg_serve_done* out, int max, int wait_ms, int* nout) {
    return guarded(e, [&] {
        Server* s = server_of(e);
        require(s, "serve: not started");
        require(out && nout && max >= 0, "serve: bad arguments");
        std::unique_lock<std::mutex> lk(s->mu);
        if (s->done_order.empty() && wait_ms > 0)
            s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->done_order.empty(); });
        int n = 0;
        while (n < max && !s->done_order.empty()) {
            const uint64_t t = s->done_order.front();
            s->done_order.pop_front();
            out[n++] = s->done[t].info;
        }
        *nout = n;
    });
}

int sg_serve_fetch(sg_engine* e, uint64_t ticket, sg_ligand_result* out) {
    return guarded(e, [&] {
        Server* s = server_of(e);
        require(s, "serve: not started");
        require(out, "serve: bad arguments");
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->done.find(ticket);
        require(it != s->done.end(), "serve: unknown or already fetched ticket");
        const ServeDone& d = it->second;
        out->count = d.info.count;
        out->evals = d.info.evals;
        if (d.info.count > 0) {
            require(out->e && out->conf && out->coords, "serve: null result arrays");
            std::memcpy(out->e, d.e.data(), d.e.size() * sizeof(double));
            std::memcpy(out->conf, d.conf.data(), d.conf.size() * sizeof(double));
            std::memcpy(out->coords, d.coords.data(), d.coords.size() * sizeof(double));
        }
        s->done.erase(it);
    });
}

int sg_serve_stats(const sg_engine* e, int* queued, int* inflight_ligands, uint64_t* inflight_bytes) {
    Server* s = server_of(e);
    if (!s) return SG_ERR_STATE;
    std::lock_guard<std::mutex> lk(s->mu);
    if (queued) *queued = (int)s->queue.size();
    int n = 0;
    for (auto& b : s->inflight)
        for (auto& L : b->ligs) n += L.state != 2;
    if (inflight_ligands) *inflight_ligands = n;
    if (inflight_bytes) *inflight_bytes = s->inflight_bytes;
    return SG_OK;
}

int sg_serve_stop(sg_engine* e) {
    return guarded(e, [&] {
        Server* s = server_of(e);
        require(s, "serve: not started");
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stopping = true;
        }
        if (s->th.joinable()) s->th.join();
        stop_grids(*s);
        cudaStreamSynchronize(s->refine_stream);
        cudaStreamSynchronize(s->copy_stream);
        cudaStreamDestroy(s->refine_stream);
        cudaStreamDestroy(s->copy_stream);
        cudaFreeHost((void*)s->flags);
        cudaFree(s->d_err);
        cudaFreeHost((void*)s->h_err);
        for (char* p : s->pin_all) cudaFreeHost(p);
        const int err = s->error;
        const std::string why = s->error_text;
        {
            std::lock_guard<std::mutex> lk(g_srv_mu);
            g_servers.erase(e);
        }
        if (err != SG_OK) throw EngineError(err, why);
    });
}

}  // extern "C"
