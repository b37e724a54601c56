// Host-side checks of the C++ interface (include/smina_b200.hpp), in the
// manner of the reference's own C++ test programs (src/gpu/tests): settings
// out of range, or that the reference accepts but this engine does not
// build, are refused at construction with std::runtime_error; --fast's
// chain split and step fraction are accepted; device lists parse like the
// reference's parse_devices, and a machine without a usable device gets an
// exception from the constructor instead of a half-built engine.
// On a device, the class's searches, refinement and minimisation are checked
// bit for bit against the same work done through the C ABI directly.
//
//   gpu_docking_api_test host          (no device present)
//   gpu_docking_api_test device        (device 0 present)
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "smina_b200.hpp"

using smina_b200::GpuDocking;
using smina_b200::GpuSettings;

static int failures = 0;

static void expect(bool ok, const char* what) {
    if (!ok) {
        std::printf("FAIL: %s\n", what);
        failures++;
    }
}

static void expect_throw(const std::function<void()>& f, const char* needle, const char* what) {
    try {
        f();
        std::printf("FAIL: %s (no exception)\n", what);
        failures++;
    } catch (const std::runtime_error& e) {
        if (!std::strstr(e.what(), needle)) {
            std::printf("FAIL: %s (message \"%s\" lacks \"%s\")\n", what, e.what(), needle);
            failures++;
        }
    }
}

static GpuSettings with(const std::function<void(GpuSettings&)>& f) {
    GpuSettings s;
    f(s);
    return s;
}


// ---- device mode ---------------------------------------------------------------------------
static bool same(const double* a, const double* b, size_t n) { return n == 0 || std::memcmp(a, b, n * sizeof(double)) == 0; }

// a pose list against C-ABI arrays (count poses, conf_size, heavy atoms)
static void expect_poses(const smina_b200::OutputContainer& out, int count, const double* e, const double* conf,
                         const double* xyz, int cs, int heavy, const char* what) {
    if (int(out.size()) != count) {
        std::printf("FAIL: %s (%zu poses, C ABI %d)\n", what, out.size(), count);
        failures++;
        return;
    }
    for (int i = 0; i < count; i++) {
        const smina_b200::Pose& q = out[i];
        const bool ok = same(&q.e, e + i, 1) && int(q.conf.size()) == cs && same(q.conf.data(), conf + size_t(i) * cs, cs) &&
                        int(q.coords.size()) == 3 * heavy && same(q.coords.data(), xyz + size_t(i) * heavy * 3, 3 * heavy);
        if (!ok) {
            std::printf("FAIL: %s (pose %d differs: %.17g vs %.17g)\n", what, i, q.e, e[i]);
            failures++;
            return;
        }
    }
}

static void require_ok(int rc, const char* what) {
    if (rc != SG_OK) {
        std::printf("FAIL: %s (rc %d: %s)\n", what, rc, sgh_last_error());
        std::exit(2);
    }
}

static sgh_model* ligand(int heavy, int rotors, uint64_t seed, const double c[3]) {
    const int need = sgh_make_ligand_pdbqt(heavy, rotors, seed, c, nullptr, 0);
    std::vector<char> buf(size_t(need > 0 ? need : 1) + 1);
    require_ok(sgh_make_ligand_pdbqt(heavy, rotors, seed, c, buf.data(), int(buf.size())), "ligand text");
    sgh_model* m = nullptr;
    require_ok(sgh_model_from_pdbqt(buf.data(), &m), "ligand model");
    return m;
}

static sg_engine* engine(int prec, const sgh_tables* T, sgh_receptor* R, const sg_grid_dims& gd) {
    sg_engine* e = nullptr;
    require_ok(sg_create(0, prec, &e), "engine");
    sg_tables_desc t;
    sg_receptor_desc r;
    require_ok(sgh_tables_desc(T, &t), "tables desc");
    require_ok(sgh_receptor_desc(R, &r), "receptor desc");
    require_ok(sg_set_tables(e, &t), "set tables");
    require_ok(sg_set_receptor(e, 0, &r, &gd), "set receptor");
    return e;
}

static void device_checks() {
    const double c[3] = {0.5, 0.25, -0.3}, size[3] = {16, 16, 16};
    sgh_tables* T = nullptr;
    sgh_receptor* R = nullptr;
    sg_grid_dims gd;
    require_ok(sgh_tables_create("vina", "", 32.0, &T), "tables");
    require_ok(sgh_make_receptor(1500, 3, c, 8.0, &R), "receptor");
    require_ok(sgh_make_box(c, size, 0.375, &gd), "box");
    sgh_model* m1 = ligand(14, 3, 2, c);
    sgh_model* m2 = ligand(22, 5, 9, c);
    sg_model_desc d1, d2;
    require_ok(sgh_model_desc(m1, &d1), "desc 1");
    require_ok(sgh_model_desc(m2, &d2), "desc 2");
    const int h1 = sgh_model_heavy(m1), h2 = sgh_model_heavy(m2);
    sg_mc_params mc;
    require_ok(sgh_search_params(m1, 9, &mc), "search params");
    mc.num_steps = 12;
    const int S = mc.num_saved_mins, tasks = 4, seed = 7;
    sg_engine* e32 = engine(SG_PREC_FP32, T, R, gd);
    sg_engine* e64 = engine(SG_PREC_FP64, T, R, gd);
    // the class's default threads_per_chain (0: automatic), so that its
    // results and the C ABI's are the same searches
    require_ok(sg_set_threads_per_chain(e32, 0), "automatic threads per chain");

    // FP32 engine: parallel_mc = one batched job, not refined
    GpuDocking g32(GpuSettings{});
    expect(g32.chains_per_batch() > 0, "chains_per_batch");
    expect(g32.description().find("device 0") != std::string::npos, "description names the device");
    smina_b200::ParallelMC par;
    par.num_tasks = tasks;
    par.mc = mc;
    smina_b200::OutputContainer out32;
    g32.parallel_mc(par, m1, out32, T, R, gd, seed);
    {
        std::vector<double> e(S), conf(size_t(S) * d1.conf_size), xyz(size_t(S) * h1 * 3);
        const sg_ligand_job job{0, tasks, mc.num_steps, mc.maxiters, uint64_t(seed), 0};
        sg_ligand_result r{0, e.data(), conf.data(), xyz.data(), 0};
        require_ok(sg_dock_batch32(e32, 0, &d1, 1, &job, 1, &mc, 0, &r), "C ABI dock_batch32");
        expect(r.count > 0, "FP32 search found poses");
        expect_poses(out32, r.count, e.data(), conf.data(), xyz.data(), d1.conf_size, h1, "parallel_mc (FP32)");
    }
    // dock_batch: two ligands in one persistent launch, merged and refined
    {
        GpuDocking::DockJob j1, j2;
        j1.m = m1;
        j2.m = m2;
        j1.par = par;
        j2.par = par;
        sg_mc_params mc2;
        require_ok(sgh_search_params(m2, 9, &mc2), "search params 2");
        j2.par.mc.maxiters = mc2.maxiters;
        std::vector<GpuDocking::DockJob*> jobs{&j1, &j2};
        g32.dock_batch(jobs, T, R, gd, seed, mc.authentic_v);
        const sg_model_desc ds[2] = {d1, d2};
        const int hs[2] = {h1, h2};
        std::vector<double> e[2], conf[2], xyz[2];
        sg_ligand_result r[2];
        sg_ligand_job lj[2];
        for (int k = 0; k < 2; k++) {
            e[k].assign(S, 0.0);
            conf[k].assign(size_t(S) * ds[k].conf_size, 0.0);
            xyz[k].assign(size_t(S) * hs[k] * 3, 0.0);
            r[k] = sg_ligand_result{0, e[k].data(), conf[k].data(), xyz[k].data(), 0};
            lj[k] = sg_ligand_job{k, tasks, mc.num_steps, k ? mc2.maxiters : mc.maxiters, uint64_t(seed), uint64_t(k)};
        }
        require_ok(sg_dock_batch32(e32, 0, ds, 2, lj, 2, &mc, 1, r), "C ABI dock_batch32 refined");
        expect_poses(j1.out, r[0].count, e[0].data(), conf[0].data(), xyz[0].data(), d1.conf_size, h1, "dock_batch job 1");
        expect_poses(j2.out, r[1].count, e[1].data(), conf[1].data(), xyz[1].data(), d2.conf_size, h2, "dock_batch job 2");
    }
    // refine: FP64 refine_structure of the FP32 search's poses
    {
        smina_b200::OutputContainer poses = out32;
        std::vector<smina_b200::Pose*> ptr;
        for (auto& q : poses) ptr.push_back(&q);
        smina_b200::MinParams mp;
        mp.maxiters = mc.maxiters;
        g32.refine(m1, T, R, gd, ptr, mc.authentic_v, mp);
        const int n = int(out32.size());
        std::vector<double> cf(size_t(n) * d1.conf_size), en(n), xyz(size_t(n) * h1 * 3);
        std::vector<int> pm(n, 0);
        for (int i = 0; i < n; i++) std::copy(out32[i].conf.begin(), out32[i].conf.end(), cf.begin() + size_t(i) * d1.conf_size);
        require_ok(sg_refine(e64, 0, &d1, 1, pm.data(), n, cf.data(), mc.authentic_v, mc.maxiters, 0, 0, en.data(),
                             xyz.data()),
                   "C ABI refine");
        expect_poses(poses, n, en.data(), cf.data(), xyz.data(), d1.conf_size, h1, "refine");
        // minimize_batch: each pose in its own box (a 12 A box around the centre), own iteration count
        sg_grid_dims small;
        const double s12[3] = {12, 12, 12};
        require_ok(sgh_make_box(c, s12, 0.375, &small), "small box");
        smina_b200::OutputContainer mposes = out32;
        std::vector<GpuDocking::MinimizeJob> mj(n);
        std::vector<double> boxes(size_t(n) * 6);
        std::vector<int> iters(n);
        for (int i = 0; i < n; i++) {
            mj[i].m = m1;
            mj[i].gd = (i % 2) ? small : gd;
            mj[i].minparm.maxiters = 4 + i;
            mj[i].out = &mposes[i];
            for (int a = 0; a < 3; a++) {
                boxes[6 * i + a] = mj[i].gd.begin[a];
                boxes[6 * i + 3 + a] = mj[i].gd.end[a];
            }
            iters[i] = 4 + i;
            std::copy(out32[i].conf.begin(), out32[i].conf.end(), cf.begin() + size_t(i) * d1.conf_size);
        }
        g32.minimize_batch(mj, T, R, gd, mc.authentic_v);
        require_ok(sg_minimize(e64, 0, &d1, 1, pm.data(), n, cf.data(), d1.conf_size, boxes.data(), mc.authentic_v,
                               iters.data(), 0, 0, en.data(), xyz.data(), h1),
                   "C ABI minimize");
        expect_poses(mposes, n, en.data(), cf.data(), xyz.data(), d1.conf_size, h1, "minimize_batch");
    }
    // early stop (--fast, ALWAYS, chain split 2): the class applies the reference's rule and checkpoints
    {
        GpuSettings se;
        se.early_stop = GpuSettings::EARLY_STOP_ALWAYS;
        se.chain_split = 2;
        GpuDocking ges(se);
        smina_b200::ParallelMC p2 = par;
        p2.mc.num_steps = 40;
        smina_b200::OutputContainer out_es;
        ges.parallel_mc(p2, m1, out_es, T, R, gd, seed);
        int sms = 0, split = 0;
        unsigned chain_steps = 0;
        double fraction = 0;
        sg_device_info(e32, nullptr, &sms, nullptr);
        require_ok(sgh_fast_chains(tasks, (long long)sms * 16, 2, 1.0, 0, p2.mc.num_steps, &split, &chain_steps, &fraction),
                   "fast chains");
        sg_early_stop es;
        es.first = 2;
        es.checkpoints = std::max(3, int(std::lround(10 * fraction)));
        es.fraction = 0.5;
        es.eps = 0.05;
        es.chains_per_unit = split;
        require_ok(sg_set_early_stop(e32, &es), "early stop");
        std::vector<double> e(S), conf(size_t(S) * d1.conf_size), xyz(size_t(S) * h1 * 3);
        const sg_ligand_job job{0, tasks * split, chain_steps, p2.mc.maxiters, uint64_t(seed), 0};
        sg_ligand_result r{0, e.data(), conf.data(), xyz.data(), 0};
        require_ok(sg_dock_batch32(e32, 0, &d1, 1, &job, 1, &p2.mc, 0, &r), "C ABI dock_batch32 with early stop");
        require_ok(sg_set_early_stop(e32, nullptr), "early stop off");
        expect_poses(out_es, r.count, e.data(), conf.data(), xyz.data(), d1.conf_size, h1, "parallel_mc with early stop");
    }
    // two-pass screening: 24 ligands, the full search for those within the
    // margin of the best quarter; the others keep their first pass
    {
        GpuDocking g2(GpuSettings{});
        const int nl = 24;
        std::vector<sgh_model*> lm;
        std::vector<GpuDocking::DockJob> tj(nl), first(nl), full(nl);
        for (int k = 0; k < nl; k++) {
            lm.push_back(ligand(12 + (k % 5) * 4, k % 4, 300 + k, c));
            for (auto* v : {&tj, &first, &full}) {
                (*v)[k].m = lm.back();
                (*v)[k].par = par;
                (*v)[k].par.mc.num_steps = 60;
                sg_mc_params mk;
                require_ok(sgh_search_params(lm.back(), 9, &mk), "search params");
                (*v)[k].par.mc.maxiters = mk.maxiters;
            }
        }
        auto ptrs = [](std::vector<GpuDocking::DockJob>& v) {
            std::vector<GpuDocking::DockJob*> r;
            for (auto& j : v) r.push_back(&j);
            return r;
        };
        std::vector<double> hist;
        std::vector<GpuDocking::DockJob*> tp = ptrs(tj);
        const size_t nfull = g2.dock_batch_two_pass(tp, T, R, gd, seed, mc.authentic_v, 0.25, 0.3, 0.1, hist);
        expect(hist.size() == size_t(nl), "two-pass keeps every first-pass score");
        expect(nfull >= 6 && nfull <= size_t(nl), "two-pass: at least the best quarter gets the full search");
        std::vector<GpuDocking::DockJob*> fp = ptrs(first);
        g2.dock_batch(fp, T, R, gd, seed, mc.authentic_v, 0.1);
        std::vector<double> sorted(hist);
        std::sort(sorted.begin(), sorted.end());
        const double cutoff = sorted[5] + 0.3;
        std::vector<GpuDocking::DockJob*> sel;
        for (int k = 0; k < nl; k++) {
            expect(hist[k] == g2.top_score(first[k], T, R, gd, mc.authentic_v), "first-pass score");
            if (hist[k] <= cutoff) sel.push_back(&full[k]);
        }
        expect(sel.size() == nfull, "two-pass selects by the cutoff");
        g2.dock_batch(sel, T, R, gd, seed, mc.authentic_v);
        for (int k = 0; k < nl; k++) {
            const GpuDocking::DockJob& want = hist[k] <= cutoff ? full[k] : first[k];
            bool same = want.out.size() == tj[k].out.size();
            for (size_t i = 0; same && i < want.out.size(); i++)
                same = want.out[i].e == tj[k].out[i].e && want.out[i].conf == tj[k].out[i].conf;
            expect(same, "two-pass poses: the full search for selected ligands, the first pass for the others");
        }
        for (sgh_model* x : lm) sgh_model_free(x);
    }
    // FP64 engine: parallel_mc = host-seeded mt19937 chains, merged with min_rmsd 2
    {
        GpuSettings s64;
        s64.fp64 = true;
        GpuDocking g64(s64);
        smina_b200::OutputContainer out64;
        g64.parallel_mc(par, m1, out64, T, R, gd, seed);
        std::vector<double> c0(size_t(tasks) * d1.conf_size);
        std::vector<uint32_t> mt(size_t(tasks) * 625);
        require_ok(sgh_seed_chains(m1, seed, tasks, &gd, c0.data(), mt.data()), "seed chains");
        std::vector<sg_chain_input> in(tasks);
        std::vector<sg_chain_result> res(tasks);
        std::vector<double> re(size_t(tasks) * S), rc(size_t(tasks) * S * d1.conf_size), rx(size_t(tasks) * S * h1 * 3);
        for (int j = 0; j < tasks; j++) {
            in[j] = sg_chain_input{0, mc.num_steps, &c0[size_t(j) * d1.conf_size], &mt[size_t(j) * 625], 0};
            res[j] = sg_chain_result{0, &re[size_t(j) * S], &rc[size_t(j) * S * d1.conf_size], &rx[size_t(j) * S * h1 * 3], 0};
        }
        require_ok(sg_dock(e64, 0, &d1, 1, in.data(), tasks, &mc, res.data()), "C ABI dock");
        std::vector<double> e(S), conf(size_t(S) * d1.conf_size), xyz(size_t(S) * h1 * 3);
        int count = 0;
        require_ok(sgh_merge_chains(res.data(), tasks, d1.conf_size, h1, 2.0, S, e.data(), conf.data(), xyz.data(), &count),
                   "merge");
        expect(count > 0, "FP64 search found poses");
        expect_poses(out64, count, e.data(), conf.data(), xyz.data(), d1.conf_size, h1, "parallel_mc (FP64)");
    }
    sg_destroy(e32);
    sg_destroy(e64);
    sgh_model_free(m1);
    sgh_model_free(m2);
    sgh_receptor_free(R);
    sgh_tables_free(T);
}

int main(int argc, char** argv) {
    const std::string mode = argc > 1 ? argv[1] : "host";
    // parse_devices
    expect(smina_b200::parse_devices("0") == std::vector<int>{0}, "parse 0");
    expect(smina_b200::parse_devices("0,1,3") == (std::vector<int>{0, 1, 3}), "parse 0,1,3");
    expect_throw([] { smina_b200::parse_devices(""); }, "bad device list", "empty list");
    expect_throw([] { smina_b200::parse_devices("0,x"); }, "bad device list", "non-numeric device");
    expect_throw([] { smina_b200::parse_devices("1a"); }, "bad device list", "trailing characters");
    expect_throw([] { smina_b200::parse_devices("-1"); }, "bad device list", "negative device");
    // settings this engine does not build
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.chain_split = -1; })); }, "chain_split",
                 "negative chain_split");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.step_fraction = 1.5; })); }, "step_fraction",
                 "step_fraction above 1");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.early_stop = GpuSettings::EARLY_STOP_FULL; s.fp64 = true; })); },
                 "early_stop", "early_stop with fp64");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.early_stop = 7; })); }, "early_stop", "unknown early_stop");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.threads_per_chain = 256; })); }, "threads_per_chain",
                 "threads_per_chain 256");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.threads_per_chain = 48; })); }, "threads_per_chain",
                 "threads_per_chain 48");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.threads_per_chain = 64; s.fp64 = true; })); },
                 "FP32 search", "threads_per_chain 64 with fp64");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.skip_visited = true; })); }, "fp64",
                 "skip_visited without fp64");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.devices.clear(); })); }, "no CUDA device",
                 "no devices");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.devices = {0, 0}; })); }, "given twice",
                 "duplicate device");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.devices = {-2}; })); }, "bad CUDA device",
                 "negative device ordinal");
    if (mode == "host") {
        // without a usable device the constructor throws (cuda_check in the reference)
        expect_throw([] { GpuDocking g(GpuSettings{}); }, "not usable", "no device present");
        expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.chain_split = 0; s.step_fraction = 0; })); },
                     "not usable", "--fast settings pass validation");
        expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.fp64 = true; })); }, "not usable",
                     "no device present, fp64");
        expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.threads_per_chain = 128; })); }, "not usable",
                     "threads_per_chain 128 passes validation");
        expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.early_stop = GpuSettings::EARLY_STOP_ALWAYS; })); },
                     "not usable", "early_stop passes validation on FP32");
    }
    if (mode == "device") device_checks();
    std::printf("%s: %d failure(s)\n", mode.c_str(), failures);
    return failures ? 1 : 0;
}
