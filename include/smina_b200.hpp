/*
 * smina_b200.hpp - C++ interface of the B200 docking engine, shaped like the
 * reference's GPU drop-in gpusmina::GpuDocking (src/gpu/gpu_docking.h:24-114):
 * the same settings, method names, argument meaning and error behaviour
 * (std::runtime_error carrying the engine's message, as the reference's
 * cuda_check and flatteners throw), written over the C ABI of smina_b200.h
 * and smina_b200_host.h.  Header-only; link libsmina_b200.so.
 *
 * What differs, and why:
 *   - smina's model, precalculate and output_container are this project's
 *     sgh_model, sgh_tables and a vector of Pose; the receptor, which the
 *     reference reads from the model's grid atoms, is passed as an
 *     sgh_receptor with its grid_dims.
 *   - smina's rng& becomes an int seed.  parallel_mc draws one seed per task
 *     from the generator (parallel_mc.cpp:89); here sgh_seed_chains seeds
 *     every task from `seed` on the host, start conf and mt19937 state alike.
 *     For FP64 engines these are the states the plain kernels start from, as
 *     the reference's --gpu_fp64 chains start from the host's.  FP32 engines
 *     key their counter-based streams by (seed, ligand index).
 *   - The reference's --fast search (not smina's): chain_split and
 *     step_fraction (0: automatic) and dock_batch's first-pass budget,
 *     planned by sgh_fast_chains; early_stop on FP32 engines (the batched
 *     search in phases, sg_set_early_stop, with the reference's rule and
 *     checkpoints); skip_visited on FP64 engines.  Refused at construction
 *     with a message: threads_per_chain above 32 with FP64, skip_visited with FP32
 *     engines (QuickVina 2's history runs on the FP64 path only) and
 *     early_stop with FP64 engines (the plain path does not run in phases).
 *
 * Precision follows the reference: the search runs in FP32 (mixed
 * precision, batched) unless settings.fp64; refinement and local
 * optimisation always run in FP64 (gpu_docking.h:60-64).
 *
 * Threading: one GpuDocking per host thread, like the reference's engines;
 * with several devices, dock_batch runs each device's share of the jobs on
 * its own thread.
 */
#ifndef SMINA_B200_HPP
#define SMINA_B200_HPP

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "smina_b200.h"
#include "smina_b200_host.h"

namespace smina_b200 {

/* GpuSettings (gpu_docking.h:24-48). */
struct GpuSettings {
    std::vector<int> devices{0};
    bool fp64 = false;
    int threads_per_chain = 0;  /* 0: automatic (by the batch's size), or 32, 64, 128 */
    int chain_split = 1;        /* chains per search task (0: automatic, --fast) */
    double step_fraction = 1;   /* fraction of smina's steps (0: automatic, --fast) */
    bool skip_visited = false;
    enum { EARLY_STOP_OFF, EARLY_STOP_FULL, EARLY_STOP_ALWAYS };
    int early_stop = EARLY_STOP_OFF;
};

/* parse_devices (gpu_docking.h:51): "0,1" -> {0, 1}. */
inline std::vector<int> parse_devices(const std::string& s) {
    std::vector<int> out;
    std::stringstream ss(s);
    std::string item;
    while (std::getline(ss, item, ',')) {
        size_t used = 0;
        int d = -1;
        try {
            d = std::stoi(item, &used);
        } catch (const std::exception&) {
            used = 0;
        }
        if (used == 0 || used != item.size() || d < 0) throw std::runtime_error("bad device list: " + s);
        out.push_back(d);
    }
    if (out.empty()) throw std::runtime_error("bad device list: " + s);
    return out;
}

/* output_type: energy, conf (smina's flat layout), heavy-atom coordinates. */
struct Pose {
    double e = 0;
    std::vector<double> conf;
    std::vector<double> coords;  /* [heavy][3] */
};
typedef std::vector<Pose> OutputContainer;

/* parallel_mc (parallel_mc.h:28-35): exhaustiveness and the monte_carlo
 * parameters (sgh_search_params gives smina's). */
struct ParallelMC {
    int num_tasks = 8;
    sg_mc_params mc{};
};

/* minimization_params. */
struct MinParams {
    int maxiters = 0;
    int accurate_line = 0;
    int early_term = 0;
};

namespace detail {
inline void check_host(int rc, const char* what) {
    if (rc != SG_OK) throw std::runtime_error(std::string(what) + ": " + sgh_last_error());
}
inline sg_model_desc desc_of(const sgh_model* m) {
    sg_model_desc d;
    check_host(sgh_model_desc(m, &d), "model");
    return d;
}
inline sg_tables_desc desc_of(const sgh_tables* t) {
    sg_tables_desc d;
    check_host(sgh_tables_desc(t, &d), "tables");
    return d;
}
inline bool same_dims(const sg_grid_dims& a, const sg_grid_dims& b) {
    for (int i = 0; i < 3; i++)
        if (a.begin[i] != b.begin[i] || a.end[i] != b.end[i] || a.n[i] != b.n[i]) return false;
    return true;
}
}  // namespace detail

class GpuDocking {
    /* one device: its search engine and, created on first use, an FP64 one
     * for local optimisation; the tables and receptor each has resident */
    struct Device {
        int ordinal = 0;
        sg_engine* search = nullptr;
        sg_engine* local = nullptr;
        const sgh_tables* tables[2] = {nullptr, nullptr};
        const sgh_receptor* receptor[2] = {nullptr, nullptr};
        sg_grid_dims gd[2]{};
    };
    GpuSettings settings_;
    std::vector<Device> dev_;

    static void check(sg_engine* e, int rc, const char* what) {
        if (rc != SG_OK) throw std::runtime_error(std::string(what) + ": " + sg_last_error(e));
    }
    /* the engine of device k (search or local), with the caller's tables and
     * receptor resident (re-sent when they change, as the reference's
     * engines cache them by identity, gpu_docking.cpp:270-332) */
    sg_engine* prepare(size_t k, bool local, const sgh_tables* p, sgh_receptor* rec, const sg_grid_dims& gd) {
        Device& d = dev_[k];
        const int w = local ? 1 : 0;
        sg_engine*& e = local ? d.local : d.search;
        if (!e) {
            if (sg_create(d.ordinal, SG_PREC_FP64, &e) != SG_OK)
                throw std::runtime_error("CUDA device " + std::to_string(d.ordinal) + " is not usable");
            d.tables[w] = nullptr;
            d.receptor[w] = nullptr;
        }
        if (d.tables[w] != p) {
            const sg_tables_desc t = detail::desc_of(p);
            check(e, sg_set_tables(e, &t), "tables");
            d.tables[w] = p;
            d.receptor[w] = nullptr;  /* new tables drop the maps */
        }
        if (d.receptor[w] != rec || !detail::same_dims(d.gd[w], gd)) {
            sg_receptor_desc r;
            detail::check_host(sgh_receptor_desc(rec, &r), "receptor");
            check(e, sg_set_receptor(e, 0, &r, &gd), "receptor");
            d.receptor[w] = rec;
            d.gd[w] = gd;
        }
        return e;
    }

    GpuDocking(const GpuDocking&) = delete;
    GpuDocking& operator=(const GpuDocking&) = delete;

public:
    explicit GpuDocking(const GpuSettings& s) : settings_(s) {
        if (s.devices.empty()) throw std::runtime_error("no CUDA device given");
        if (s.chain_split < 0) throw std::runtime_error("chain_split must be 0 (automatic) or positive");
        if (!(s.step_fraction >= 0 && s.step_fraction <= 1))
            throw std::runtime_error("step_fraction must lie in [0, 1] (0: automatic)");
        if (s.early_stop < GpuSettings::EARLY_STOP_OFF || s.early_stop > GpuSettings::EARLY_STOP_ALWAYS)
            throw std::runtime_error("early_stop: unknown mode");
        if (s.early_stop != GpuSettings::EARLY_STOP_OFF && s.fp64)
            throw std::runtime_error("early_stop needs the FP32 search (the FP64 path does not run in phases)");
        if (!(s.threads_per_chain == 0 || s.threads_per_chain == 32 || s.threads_per_chain == 64 ||
              s.threads_per_chain == 128))
            throw std::runtime_error("threads_per_chain: 0 (automatic), 32, 64 or 128");
        if (s.fp64 && s.threads_per_chain > 32)
            throw std::runtime_error("threads_per_chain above 32 needs the FP32 search (the FP64 path runs one warp "
                                     "per chain, bit for bit as the CPU search)");
        if (s.skip_visited && !s.fp64)
            throw std::runtime_error("skip_visited needs the double precision search (fp64)");
        for (size_t i = 0; i < s.devices.size(); i++) {
            const int d = s.devices[i];
            if (d < 0) throw std::runtime_error("bad CUDA device " + std::to_string(d));
            if (std::find(s.devices.begin(), s.devices.begin() + i, d) != s.devices.begin() + i)
                throw std::runtime_error("CUDA device " + std::to_string(d) + " given twice");
        }
        for (int d : s.devices) {
            Device x;
            x.ordinal = d;
            const int prec = s.fp64 ? SG_PREC_FP64 : SG_PREC_FP32;
            if (sg_create(d, prec, &x.search) != SG_OK) {
                for (Device& y : dev_) sg_destroy(y.search);
                dev_.clear();
                throw std::runtime_error("CUDA device " + std::to_string(d) + " is not usable");
            }
            if (!s.fp64) sg_set_threads_per_chain(x.search, s.threads_per_chain);
            dev_.push_back(x);
        }
    }

    ~GpuDocking() {
        for (Device& d : dev_) {
            sg_destroy(d.search);
            sg_destroy(d.local);
        }
    }

    /* parallel_mc::operator() (parallel_mc.cpp:80-98): num_tasks chains of
     * model m seeded from `seed`, merged into `out` with min_rmsd 2 and at
     * most mc.num_saved_mins poses, sorted by energy.  Not refined. */
    void parallel_mc(const ParallelMC& par, const sgh_model* m, OutputContainer& out, const sgh_tables* p,
                     sgh_receptor* rec, const sg_grid_dims& gd, int seed) {
        search_on(0, par, m, out, p, rec, gd, seed);
    }

    /* refine_structure for every pose (main.cpp:165-190): FP64, against
     * the receptor atoms in the box gd; poses updated in place (conf, e,
     * heavy-atom coords). */
    void refine(const sgh_model* m, const sgh_tables* p, sgh_receptor* rec, const sg_grid_dims& gd,
                std::vector<Pose*>& poses, const double cap[3], const MinParams& minparm) {
        refine_on(0, m, p, rec, gd, poses, cap, minparm);
    }

    /* DockJob (gpu_docking.h:80-85): a ligand, its search parameters, its
     * merged and refined poses. */
    struct DockJob {
        const sgh_model* m = nullptr;
        ParallelMC par;
        OutputContainer out;
    };

    /* dock_batch (gpu_docking.h:86-94): for every job, parallel_mc then
     * refine_structure of every pose (FP64, cap as the refinement's curl
     * cap), poses sorted by energy.  FP32 engines run all jobs of a device
     * in one persistent launch; jobs are split over the devices in
     * contiguous ranges, one host thread per device.  budget > 0: that
     * fraction of smina's steps (a first pass of two-pass screening). */
    void dock_batch(std::vector<DockJob*>& jobs, const sgh_tables* p, sgh_receptor* rec, const sg_grid_dims& gd,
                    int seed, const double cap[3], double budget = 0) {
        if (!(budget >= 0 && budget <= 1)) throw std::runtime_error("dock_batch: budget must lie in [0, 1]");
        if (jobs.empty()) return;
        const size_t nd = std::min(dev_.size(), jobs.size());
        std::vector<std::string> errors(nd);
        auto run = [&](size_t k, size_t lo, size_t hi) {
            try {
                dock_range(k, jobs, lo, hi, p, rec, gd, seed, cap, budget);
            } catch (const std::exception& ex) {
                errors[k] = ex.what();
            }
        };
        std::vector<std::thread> th;
        for (size_t k = 0; k < nd; k++) {
            const size_t lo = jobs.size() * k / nd, hi = jobs.size() * (k + 1) / nd;
            if (nd == 1) run(k, lo, hi);
            else th.emplace_back(run, k, lo, hi);
        }
        for (std::thread& t : th) t.join();
        for (const std::string& s : errors)
            if (!s.empty()) throw std::runtime_error(s);
    }

    /* top_score (main.cpp:355-373): the best final score finish_docking
     * would report for a job's refined poses -- the conf-independent terms
     * applied to each pose's energy on the direct receptor sum less the
     * intramolecular energy of the best pose (FP64, sg_score on the first
     * device); max double for a job without poses. */
    double top_score(const DockJob& job, const sgh_tables* p, sgh_receptor* rec, const sg_grid_dims& gd,
                     const double cap[3], double slope = 1e6) {
        const int n = int(job.out.size());
        if (n == 0) return std::numeric_limits<double>::max();
        sg_engine* e = prepare(0, true, p, rec, gd);
        const sg_model_desc d = detail::desc_of(job.m);
        const int heavy = sgh_model_heavy(job.m);
        std::vector<const Pose*> sorted;
        for (const Pose& q : job.out) sorted.push_back(&q);
        std::stable_sort(sorted.begin(), sorted.end(), [](const Pose* a, const Pose* b) { return a->e < b->e; });
        std::vector<double> c(size_t(n) * d.conf_size), tot(n), intra(n);
        std::vector<int> pm(n, 0);
        for (int i = 0; i < n; i++) std::copy(sorted[i]->conf.begin(), sorted[i]->conf.end(), c.begin() + size_t(i) * d.conf_size);
        check(e, sg_score(e, 0, &d, 1, pm.data(), n, c.data(), d.conf_size, cap, slope, tot.data(), intra.data(), nullptr,
                          heavy),
              "top score");
        double inputs[7];
        detail::check_host(sgh_model_conf_independent_inputs(job.m, inputs), "conf-independent inputs");
        double best = std::numeric_limits<double>::max();
        for (int i = 0; i < n; i++) {
            if (!(sorted[i]->e < std::numeric_limits<double>::max())) continue;
            double v = 0;
            detail::check_host(sgh_tables_conf_independent(p, inputs, tot[i] - intra[0], &v), "conf-independent terms");
            best = std::min(best, v);
        }
        return best;
    }

    /* Two-pass screening (--fast_top, main.cpp:1563-1597; not smina's search):
     * once top_history and the batch hold at least 20 ligands and 0 <
     * fast_top < 1, every job is docked briefly (fast_first of smina's
     * steps), scored with top_score and its score added to top_history; the
     * jobs scoring within fast_top_margin of the best fast_top fraction of
     * top_history get the full search (their poses replaced).  Otherwise one
     * full pass.  Returns how many jobs got the full search. */
    size_t dock_batch_two_pass(std::vector<DockJob*>& jobs, const sgh_tables* p, sgh_receptor* rec,
                               const sg_grid_dims& gd, int seed, const double cap[3], double fast_top,
                               double fast_top_margin, double fast_first, std::vector<double>& top_history) {
        if (!(fast_top > 0 && fast_top < 1) || top_history.size() + jobs.size() < 20) {
            dock_batch(jobs, p, rec, gd, seed, cap);
            return jobs.size();
        }
        if (!(fast_first > 0 && fast_first <= 1)) throw std::runtime_error("two-pass: fast_first must lie in (0, 1]");
        dock_batch(jobs, p, rec, gd, seed, cap, fast_first);
        std::vector<double> score(jobs.size());
        for (size_t k = 0; k < jobs.size(); k++) score[k] = top_score(*jobs[k], p, rec, gd, cap);
        top_history.insert(top_history.end(), score.begin(), score.end());
        std::vector<double> sorted(top_history);
        const size_t q = std::max<size_t>(1, size_t(std::ceil(fast_top * sorted.size()))) - 1;
        std::nth_element(sorted.begin(), sorted.begin() + q, sorted.end());
        const double cutoff = sorted[q] + fast_top_margin;
        std::vector<DockJob*> again;
        for (size_t k = 0; k < jobs.size(); k++)
            if (score[k] <= cutoff) {
                jobs[k]->out.clear();
                again.push_back(jobs[k]);
            }
        if (!again.empty()) dock_batch(again, p, rec, gd, seed, cap);
        return again.size();
    }

    /* MinimizeJob (gpu_docking.h:96-103): a pose refined in its own box
     * with its own minimisation parameters (in: conf; out: conf, e, heavy
     * atom coords). */
    struct MinimizeJob {
        const sgh_model* m = nullptr;
        sg_grid_dims gd{};
        MinParams minparm;
        Pose* out = nullptr;
    };

    /* minimize_batch (gpu_docking.h:104-105, gpu_docking.cpp:690-742), FP64
     * on the first device.  Every job's box must lie inside `gd`, the box
     * the receptor is resident for; the line search settings are the first
     * job's. */
    void minimize_batch(std::vector<MinimizeJob>& jobs, const sgh_tables* p, sgh_receptor* rec,
                        const sg_grid_dims& gd, const double cap[3]) {
        if (jobs.empty()) return;
        sg_engine* e = prepare(0, true, p, rec, gd);
        const int n = int(jobs.size());
        std::vector<sg_model_desc> models;
        std::vector<const sgh_model*> seen;
        std::vector<int> pm(n), iters(n);
        int cs = 0, hs = 0;
        for (int k = 0; k < n; k++) {
            const auto it = std::find(seen.begin(), seen.end(), jobs[k].m);
            if (it == seen.end()) {
                seen.push_back(jobs[k].m);
                models.push_back(detail::desc_of(jobs[k].m));
                cs = std::max(cs, models.back().conf_size);
                hs = std::max(hs, sgh_model_heavy(jobs[k].m));
            }
            pm[k] = int(std::find(seen.begin(), seen.end(), jobs[k].m) - seen.begin());
            iters[k] = jobs[k].minparm.maxiters;
        }
        std::vector<double> c(size_t(n) * cs, 0.0), boxes(size_t(n) * 6), en(n), xyz(size_t(n) * hs * 3);
        for (int k = 0; k < n; k++) {
            const Pose& q = *jobs[k].out;
            if (int(q.conf.size()) != models[pm[k]].conf_size) throw std::runtime_error("minimize: conf size mismatch");
            std::copy(q.conf.begin(), q.conf.end(), c.begin() + size_t(k) * cs);
            for (int i = 0; i < 3; i++) {
                boxes[6 * k + i] = jobs[k].gd.begin[i];
                boxes[6 * k + 3 + i] = jobs[k].gd.end[i];
            }
        }
        check(e, sg_minimize(e, 0, models.data(), int(models.size()), pm.data(), n, c.data(), cs, boxes.data(), cap,
                             iters.data(), jobs[0].minparm.accurate_line, jobs[0].minparm.early_term, en.data(),
                             xyz.data(), hs),
              "minimize");
        for (int k = 0; k < n; k++) {
            Pose& q = *jobs[k].out;
            const int h = sgh_model_heavy(jobs[k].m);
            q.e = en[k];
            q.conf.assign(c.begin() + size_t(k) * cs, c.begin() + size_t(k) * cs + models[pm[k]].conf_size);
            q.coords.assign(xyz.begin() + size_t(k) * hs * 3, xyz.begin() + size_t(k) * hs * 3 + size_t(h) * 3);
        }
    }

    /* chains_per_batch (gpu_docking.h:107-109): search chains that keep
     * every device busy.  The FP32 search keeps two blocks of eight chains
     * per SM; the FP64 search runs one chain per 32-thread block, at most 32
     * blocks per SM. */
    size_t chains_per_batch() const {
        size_t total = 0;
        for (const Device& d : dev_) {
            int sms = 0;
            sg_device_info(d.search, nullptr, &sms, nullptr);
            total += size_t(sms) * (settings_.fp64 ? 32 : 16);
        }
        return total;
    }

    std::string description() const {
        std::stringstream ss;
        ss << "B200 engine (" << (settings_.fp64 ? "FP64 search" : "mixed-precision FP32 search, FP64 refinement")
           << (settings_.skip_visited ? ", QuickVina 2 history check" : "") << ") on device";
        ss << (dev_.size() > 1 ? "s" : "");
        for (size_t k = 0; k < dev_.size(); k++) {
            int sms = 0;
            sg_device_info(dev_[k].search, nullptr, &sms, nullptr);
            ss << (k ? ", " : " ") << dev_[k].ordinal << " (" << sms << " SMs)";
        }
        return ss.str();
    }

private:
    static void append(OutputContainer& out, int count, const std::vector<double>& e, const std::vector<double>& conf,
                       const std::vector<double>& xyz, int conf_size, int heavy) {
        for (int i = 0; i < count; i++) {
            Pose q;
            q.e = e[i];
            q.conf.assign(conf.begin() + size_t(i) * conf_size, conf.begin() + size_t(i + 1) * conf_size);
            q.coords.assign(xyz.begin() + size_t(i) * heavy * 3, xyz.begin() + size_t(i + 1) * heavy * 3);
            out.push_back(q);
        }
    }

    /* jobs [lo, hi) on device k */
    void dock_range(size_t k, std::vector<DockJob*>& jobs, size_t lo, size_t hi, const sgh_tables* p,
                    sgh_receptor* rec, const sg_grid_dims& gd, int seed, const double cap[3], double budget) {
        long long tasks = 0;  /* search tasks docked at once on this device: they set the automatic split */
        for (size_t j = lo; j < hi; j++) tasks += jobs[j]->par.num_tasks;
        if (settings_.fp64) {
            for (size_t j = lo; j < hi; j++) {
                DockJob& job = *jobs[j];
                OutputContainer poses;
                search_on(k, job.par, job.m, poses, p, rec, gd, seed, tasks, budget);
                std::vector<Pose*> ptr;
                for (Pose& q : poses) ptr.push_back(&q);
                MinParams mp{job.par.mc.maxiters, job.par.mc.accurate_line, job.par.mc.early_term};
                refine_on(k, job.m, p, rec, gd, ptr, cap, mp);
                std::stable_sort(poses.begin(), poses.end(), [](const Pose& a, const Pose& b) { return a.e < b.e; });
                job.out.insert(job.out.end(), poses.begin(), poses.end());
            }
            return;
        }
        sg_engine* e = prepare(k, false, p, rec, gd);
        const size_t n = hi - lo;
        std::vector<sg_model_desc> models(n);
        std::vector<sg_ligand_job> lj(n);
        std::vector<sg_ligand_result> res(n);
        std::vector<std::vector<double> > e_(n), c_(n), x_(n);
        std::vector<int> heavy(n);
        sg_mc_params mc = jobs[lo]->par.mc;
        for (size_t j = 0; j < n; j++) {
            const DockJob& job = *jobs[lo + j];
            if (job.par.mc.num_saved_mins != mc.num_saved_mins)
                throw std::runtime_error("dock_batch: every job must keep the same number of poses");
            models[j] = detail::desc_of(job.m);
            heavy[j] = sgh_model_heavy(job.m);
            const Plan f = plan(k, tasks, budget, job.par.mc.num_steps);
            lj[j] = sg_ligand_job{int(j), job.par.num_tasks * f.split, f.steps, job.par.mc.maxiters, uint64_t(seed),
                                  uint64_t(lo + j)};
            const int S = mc.num_saved_mins;
            e_[j].assign(S, 0.0);
            c_[j].assign(size_t(S) * models[j].conf_size, 0.0);
            x_[j].assign(size_t(S) * heavy[j] * 3, 0.0);
            res[j] = sg_ligand_result{0, e_[j].data(), c_[j].data(), x_[j].data(), 0};
        }
        for (int i = 0; i < 3; i++)  /* the batched search refines at authentic_v */
            if (mc.authentic_v[i] != cap[i])
                throw std::runtime_error("dock_batch: with the FP32 search the refinement cap must be authentic_v");
        apply_early_stop(e, plan(k, tasks, budget, mc.num_steps), budget);
        check(e, sg_dock_batch32(e, 0, models.data(), int(n), lj.data(), int(n), &mc, 1, res.data()), "dock_batch");
        for (size_t j = 0; j < n; j++)
            append(jobs[lo + j]->out, res[j].count, e_[j], c_[j], x_[j], models[j].conf_size, heavy[j]);
    }

    /* --fast's chain split for `tasks` tasks docked at once on device k */
    struct Plan {
        int split = 1;
        unsigned steps = 1;
        double fraction = 1;
    };
    Plan plan(size_t k, long long tasks, double budget, unsigned steps) const {
        Plan f;
        int sms = 0;
        sg_device_info(dev_[k].search, nullptr, &sms, nullptr);
        const long long capacity = (long long)sms * (settings_.fp64 ? 32 : 16);
        detail::check_host(sgh_fast_chains(tasks, capacity, settings_.chain_split, settings_.step_fraction, budget,
                                           steps, &f.split, &f.steps, &f.fraction),
                           "chain split");
        return f;
    }

    /* the early stop of device k's FP32 search for a plan (GpuDocking's
     * stops / stop_for, gpu_docking.cpp:170-188): never on a first pass;
     * EARLY_STOP_FULL only for splits below 32 (the GPU full); checks after
     * every tenth of smina's steps the chains run, from the second on */
    void apply_early_stop(sg_engine* e, const Plan& f, double budget) const {
        const bool on = !(budget > 0) && (settings_.early_stop == GpuSettings::EARLY_STOP_ALWAYS ||
                                          (settings_.early_stop == GpuSettings::EARLY_STOP_FULL && f.split < 32));
        if (!on) {
            check(e, sg_set_early_stop(e, nullptr), "early stop");
            return;
        }
        sg_early_stop es;
        es.first = 2;
        es.checkpoints = std::max(es.first + 1, int(std::lround(10 * f.fraction)));
        es.fraction = 0.5;
        es.eps = 0.05;
        es.chains_per_unit = f.split;
        check(e, sg_set_early_stop(e, &es), "early stop");
    }

    void search_on(size_t k, const ParallelMC& par, const sgh_model* m, OutputContainer& out, const sgh_tables* p,
                   sgh_receptor* rec, const sg_grid_dims& gd, int seed, long long tasks = 0, double budget = 0) {
        if (par.num_tasks <= 0) throw std::runtime_error("parallel_mc: no tasks");
        sg_engine* e = prepare(k, false, p, rec, gd);
        const sg_model_desc d = detail::desc_of(m);
        const Plan f = plan(k, tasks > 0 ? tasks : par.num_tasks, budget, par.mc.num_steps);
        const int heavy = sgh_model_heavy(m), S = par.mc.num_saved_mins, n = par.num_tasks * f.split;
        sg_mc_params mc = par.mc;
        mc.num_steps = f.steps;
        mc.visited = settings_.skip_visited ? 1 : 0;
        std::vector<double> e_(S), conf(size_t(S) * d.conf_size), xyz(size_t(S) * heavy * 3);
        int count = 0;
        if (settings_.fp64) {
            std::vector<double> c0(size_t(n) * d.conf_size);
            std::vector<uint32_t> mt(size_t(n) * 625);
            detail::check_host(sgh_seed_chains(m, seed, n, &gd, c0.data(), mt.data()), "seed chains");
            std::vector<sg_chain_input> in(n);
            std::vector<sg_chain_result> res(n);
            std::vector<double> re(size_t(n) * S), rc(size_t(n) * S * d.conf_size), rx(size_t(n) * S * heavy * 3);
            for (int j = 0; j < n; j++) {
                in[j] = sg_chain_input{0, mc.num_steps, &c0[size_t(j) * d.conf_size], &mt[size_t(j) * 625], 0};
                res[j] = sg_chain_result{0, &re[size_t(j) * S], &rc[size_t(j) * S * d.conf_size],
                                         &rx[size_t(j) * S * heavy * 3], 0};
            }
            check(e, sg_dock(e, 0, &d, 1, in.data(), n, &mc, res.data()), "parallel_mc");
            detail::check_host(sgh_merge_chains(res.data(), n, d.conf_size, heavy, 2.0, S, e_.data(), conf.data(),
                                                xyz.data(), &count),
                               "merge");
        } else {
            const sg_ligand_job job{0, n, mc.num_steps, mc.maxiters, uint64_t(seed), 0};
            sg_ligand_result r{0, e_.data(), conf.data(), xyz.data(), 0};
            apply_early_stop(e, f, budget);
            check(e, sg_dock_batch32(e, 0, &d, 1, &job, 1, &mc, 0, &r), "parallel_mc");
            count = r.count;
        }
        append(out, count, e_, conf, xyz, d.conf_size, heavy);
    }

    void refine_on(size_t k, const sgh_model* m, const sgh_tables* p, sgh_receptor* rec, const sg_grid_dims& gd,
                   std::vector<Pose*>& poses, const double cap[3], const MinParams& minparm) {
        if (poses.empty()) return;
        sg_engine* e = prepare(k, true, p, rec, gd);
        const sg_model_desc d = detail::desc_of(m);
        const int heavy = sgh_model_heavy(m), n = int(poses.size());
        std::vector<double> c(size_t(n) * d.conf_size), en(n), xyz(size_t(n) * heavy * 3);
        std::vector<int> pm(n, 0);
        for (int j = 0; j < n; j++) {
            if (int(poses[j]->conf.size()) != d.conf_size) throw std::runtime_error("refine: conf size mismatch");
            std::copy(poses[j]->conf.begin(), poses[j]->conf.end(), c.begin() + size_t(j) * d.conf_size);
        }
        check(e, sg_refine(e, 0, &d, 1, pm.data(), n, c.data(), cap, minparm.maxiters, minparm.accurate_line,
                           minparm.early_term, en.data(), xyz.data()),
              "refine");
        for (int j = 0; j < n; j++) {
            poses[j]->e = en[j];
            poses[j]->conf.assign(c.begin() + size_t(j) * d.conf_size, c.begin() + size_t(j + 1) * d.conf_size);
            poses[j]->coords.assign(xyz.begin() + size_t(j) * heavy * 3, xyz.begin() + size_t(j + 1) * heavy * 3);
        }
    }
};

}  // namespace smina_b200

#endif /* SMINA_B200_HPP */
