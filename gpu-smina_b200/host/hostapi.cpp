/*
 * C entry points of the host library (sgh_*): building models, receptors,
 * pair tables, boxes, search parameters and chain seeds as the flat
 * descriptors of include/smina_b200.h.  Errors come back as a non-zero
 * status with a message in sgh_last_error().
 */
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include "sg_host.h"
#include "../../include/smina_b200_host.h"

struct sgh_model { sgh::Model m; };
struct sgh_receptor {
    sgh::Receptor r;
    std::vector<double> xyz, q;
    std::vector<int> t;
};
struct sgh_tables {
    sgh::Tables t;
    std::vector<std::string> ci_names;  // conf-independent terms, in order, and their weights
    std::vector<double> ci_w;
};

static thread_local std::string g_err;

template <typename F>
static int guarded(F f) {
    try {
        f();
        return SG_OK;
    } catch (std::exception& e) {
        g_err = e.what();
        return SG_ERR_ARG;
    }
}

extern "C" {

const char* sgh_last_error(void) { return g_err.c_str(); }

int sgh_model_from_pdbqt(const char* text, sgh_model** out) {
    *out = nullptr;
    return guarded([&] {
        sgh_model* m = new sgh_model();
        try { m->m = sgh::read_pdbqt_ligand(text); } catch (...) { delete m; throw; }
        *out = m;
    });
}
void sgh_model_free(sgh_model* m) { delete m; }
int sgh_model_from_pdbqt_flex(const char* ligand_text, const char* flex_text, sgh_model** out) {
    *out = nullptr;
    return guarded([&] {
        if (!ligand_text || !flex_text) throw std::runtime_error("model: null text");
        auto* m = new sgh_model{sgh::read_pdbqt_flex(ligand_text, flex_text)};
        *out = m;
    });
}

int sgh_make_flex_pdbqt(int residues, uint64_t seed, const double center[3], double shell, char* buf, int buflen) {
    std::string t;
    int rc = guarded([&] { t = sgh::make_flex_pdbqt(residues, seed, center, shell > 0 ? shell : 9.0); });
    if (rc) return -1;
    if ((int)t.size() + 1 > buflen) return (int)t.size() + 1;
    std::memcpy(buf, t.c_str(), t.size() + 1);
    return 0;
}

int sgh_model_desc(const sgh_model* m, sg_model_desc* out) {
    *out = m->m.desc();
    return SG_OK;
}
int sgh_model_heavy(const sgh_model* m) { return m->m.num_heavy_movable(); }
int sgh_model_torsdof(const sgh_model* m) { return m->m.torsdof; }

int sgh_make_receptor(int heavy_atoms, uint64_t seed, const double center[3], double cavity_radius,
                      sgh_receptor** out) {
    *out = nullptr;
    return guarded([&] {
        sgh_receptor* r = new sgh_receptor();
        r->r = sgh::make_receptor(heavy_atoms, seed, center, cavity_radius);
        *out = r;
    });
}
void sgh_receptor_free(sgh_receptor* r) { delete r; }
int sgh_receptor_desc(sgh_receptor* r, sg_receptor_desc* out) {
    *out = r->r.desc(r->xyz, r->t, r->q);
    return SG_OK;
}
int sgh_receptor_pdbqt(const sgh_receptor* r, char* buf, int buflen) {
    std::string s = sgh::receptor_pdbqt(r->r);
    if ((int)s.size() + 1 > buflen) return (int)s.size() + 1;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return 0;
}

int sgh_sdf_count(const char* text) {
    int n = -1;
    if (guarded([&] {
            if (!text) throw std::runtime_error("sdf_count: null text");
            n = sgh::sdf_count(text);
        }))
        return -1;
    return n;
}

int sgh_sdf_offsets(const char* text, int64_t* offsets, int max) {
    int n = -1;
    if (guarded([&] {
            if (!text || max < 0 || (max > 0 && !offsets)) throw std::runtime_error("sdf_offsets: bad arguments");
            const std::vector<size_t> st = sgh::sdf_starts(text);
            for (int k = 0; k < (int)st.size() && k < max; k++) offsets[k] = (int64_t)st[k];
            n = (int)st.size();
        }))
        return -1;
    return n;
}

int sgh_pdbqt_from_sdf(const char* text, int index, int add_hydrogens, char* buf, int buflen) {
    std::string s;
    if (guarded([&] {
            if (!text || index < 0) throw std::runtime_error("pdbqt_from_sdf: bad arguments");
            s = sgh::pdbqt_from_sdf(text, index, add_hydrogens != 0);
        }))
        return -1;
    if ((int)s.size() + 1 > buflen) return (int)s.size() + 1;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return 0;
}

int sgh_model_from_sdf(const char* text, int index, int add_hydrogens, sgh_model** out) {
    *out = nullptr;
    return guarded([&] {
        if (!text || index < 0) throw std::runtime_error("model_from_sdf: bad arguments");
        sgh_model* m = new sgh_model();
        try { m->m = sgh::read_pdbqt_ligand(sgh::pdbqt_from_sdf(text, index, add_hydrogens != 0)); } catch (...) { delete m; throw; }
        *out = m;
    });
}

int sgh_make_ligand_pdbqt(int heavy, int rotors, uint64_t seed, const double center[3], char* buf, int buflen) {
    std::string s;
    int rc = guarded([&] { s = sgh::make_ligand_pdbqt(heavy, rotors, seed, center); });
    if (rc) return -1;
    if ((int)s.size() + 1 > buflen) return (int)s.size() + 1;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return 0;
}

int sgh_tables_create(const char* builtin_name, const char* custom_text, double factor, sgh_tables** out) {
    *out = nullptr;
    return guarded([&] {
        sgh::Scoring sf;
        if (custom_text && *custom_text) sgh::scoring_from_text(custom_text, sf);
        else if (!sgh::builtin_scoring(builtin_name ? builtin_name : "vina", sf))
            throw std::runtime_error(std::string("unknown builtin scoring function ") + builtin_name);
        if (sf.indep.empty() && sf.dep.empty()) throw std::runtime_error("scoring function has no distance terms");
        sgh_tables* t = new sgh_tables();
        sgh::build_linear_tables(sf, factor, t->t);
        t->ci_names = sf.conf_indep_names;
        t->ci_w = sf.conf_indep_w;
        *out = t;
    });
}
void sgh_tables_free(sgh_tables* t) { delete t; }
int sgh_tables_desc(const sgh_tables* t, sg_tables_desc* out) {
    *out = t->t.desc();
    return SG_OK;
}

int sgh_model_conf_independent_inputs(const sgh_model* m, double out[7]) {
    if (!m || !out) return SG_ERR_ARG;
    std::copy(m->m.ci, m->m.ci + 7, out);
    return SG_OK;
}

int sgh_tables_conf_independent(const sgh_tables* t, const double inputs[7], double x, double* out) {
    if (!t || !inputs || !out) return SG_ERR_ARG;
    return guarded([&] { *out = sgh::conf_independent(t->ci_names, t->ci_w, inputs, x); });
}

// finish_docking (main.cpp:257-324) for one ligand's refined poses
int sgh_finish_docking(const sgh_tables* t, const double inputs[7], int n, const double* e_refined,
                       const double* e_total, const double* e_intra, const double* coords, int heavy,
                       double out_min_rmsd, int num_modes, double energy_range, int* out_index, double* out_e,
                       int* out_count) {
    if (!t || !inputs || n < 0 || heavy < 0 || !out_count || (n > 0 && (!e_refined || !e_total || !e_intra ||
                                                                         !coords || !out_index || !out_e)))
        return SG_ERR_ARG;
    return guarded([&] {
        *out_count = 0;
        if (n == 0) return;
        auto not_max = [](double x) { return x < 0.1 * DBL_MAX; };
        std::vector<int> order(n);
        for (int k = 0; k < n; k++) order[k] = k;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return e_refined[a] < e_refined[b]; });
        // the best mode's intramolecular energy, then every pose's adjusted energy
        const double intra = e_intra[order[0]];
        std::vector<double> e(n);
        for (int k = 0; k < n; k++)
            e[k] = not_max(e_refined[k]) ? sgh::conf_independent(t->ci_names, t->ci_w, inputs, e_total[k] - intra)
                                         : e_refined[k];
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return e[a] < e[b]; });
        // remove_redundant (main.cpp:204-210): add_to_output_container (coords.cpp:25-58) pose by pose
        auto rmsd = [&](int a, int b) {  // rmsd_upper_bound over heavy-atom coords
            double acc = 0;
            for (int i = 0; i < heavy; i++)
                for (int d = 0; d < 3; d++) {
                    const double x = coords[((size_t)a * heavy + i) * 3 + d] - coords[((size_t)b * heavy + i) * 3 + d];
                    acc += x * x;
                }
            return heavy > 0 ? std::sqrt(acc / heavy) : 0.0;
        };
        std::vector<int> kept;
        for (int k : order) {
            size_t ci = kept.size();
            double cr = DBL_MAX;
            for (size_t i = 0; i < kept.size(); i++) {
                const double r = rmsd(k, kept[i]);
                if (i == 0 || r < cr) { ci = i; cr = r; }
            }
            if (ci < kept.size() && cr < out_min_rmsd) {
                if (e[k] < e[kept[ci]]) kept[ci] = k;
            } else if ((int)kept.size() < n) {
                kept.push_back(k);
            } else if (!kept.empty() && e[k] < e[kept.back()]) {
                kept.back() = k;
            }
            std::stable_sort(kept.begin(), kept.end(), [&](int a, int b) { return e[a] < e[b]; });
        }
        // the modes written: at most num_modes, none at max energy or past energy_range
        int how_many = 0;
        for (size_t i = 0; i < kept.size(); i++) {
            const double ei = e[kept[i]];
            if (how_many >= num_modes || !not_max(ei) || ei > e[kept[0]] + energy_range) break;
            out_index[how_many] = kept[i];
            out_e[how_many] = ei;
            how_many++;
        }
        *out_count = how_many;
    });
}

int sgh_make_box(const double center[3], const double size[3], double granularity, sg_grid_dims* out) {
    *out = sgh::make_box(center, size, granularity);
    return SG_OK;
}

int sgh_search_params(const sgh_model* m, int num_modes, sg_mc_params* out) {
    *out = sgh::search_params(m->m, num_modes);
    return SG_OK;
}

int sgh_fast_chains(long long tasks, long long capacity, int chain_split, double step_fraction, double budget,
                    unsigned steps, int* split, unsigned* chain_steps, double* fraction) {
    if (tasks < 0 || capacity < 0 || chain_split < 0 || !(step_fraction >= 0) || !(budget >= 0) ||
        step_fraction > 1 || budget > 1 || !split || !chain_steps)
        return SG_ERR_ARG;
    const sgh::FastPlan f = sgh::fast_plan((size_t)tasks, (size_t)capacity, chain_split, step_fraction, budget, steps);
    *split = f.split;
    *chain_steps = f.steps;
    if (fraction) *fraction = f.fraction;
    return SG_OK;
}

int sgh_seed_chains(const sgh_model* m, int seed, int tasks, const sg_grid_dims* box, double* confs, uint32_t* mt) {
    return guarded([&] {
        std::vector<sgh::ChainStart> cs = sgh::seed_chains(m->m, seed, tasks, *box);
        for (int k = 0; k < tasks; k++) {
            std::memcpy(confs + (size_t)k * m->m.conf_size, cs[k].conf.data(), m->m.conf_size * sizeof(double));
            std::memcpy(mt + (size_t)k * 625, cs[k].mt, 625 * sizeof(uint32_t));
        }
    });
}

// merge_output_containers (parallel_mc.cpp:64-76): every chain's poses in
// chain order through add_to_output_container (coords.cpp:25-58)
int sgh_merge_chains(const sg_chain_result* chains, int nchains, int conf_size, int nheavy, double min_rmsd,
                     int max_size, double* out_e, double* out_conf, double* out_coords, int* out_count) {
    return guarded([&] {
        if (!chains || nchains < 0 || conf_size <= 0 || nheavy < 0 || max_size <= 0 || !out_e || !out_conf ||
            !out_coords || !out_count)
            throw std::runtime_error("merge: bad arguments");
        struct Pose { double e; std::vector<double> c, x; };
        std::vector<Pose> out;
        const size_t H3 = (size_t)nheavy * 3;
        for (int k = 0; k < nchains; k++)
            for (int j = 0; j < chains[k].count; j++) {
                Pose t;
                t.e = chains[k].e[j];
                t.c.assign(chains[k].conf + (size_t)j * conf_size, chains[k].conf + (size_t)(j + 1) * conf_size);
                t.x.assign(chains[k].coords + j * H3, chains[k].coords + (j + 1) * H3);
                size_t ci = out.size();
                double cr = DBL_MAX;
                for (size_t i = 0; i < out.size(); i++) {
                    double acc = 0;
                    for (size_t a = 0; a < H3; a++) acc += (t.x[a] - out[i].x[a]) * (t.x[a] - out[i].x[a]);
                    const double r = H3 ? std::sqrt(acc / (double)nheavy) : 0.0;
                    if (i == 0 || r < cr) { ci = i; cr = r; }
                }
                if (ci < out.size() && cr < min_rmsd) {
                    if (t.e < out[ci].e) out[ci] = std::move(t);
                } else if ((int)out.size() < max_size) {
                    out.push_back(std::move(t));
                } else if (!out.empty() && t.e < out.back().e) {
                    out.back() = std::move(t);
                }
                std::stable_sort(out.begin(), out.end(), [](const Pose& a, const Pose& b) { return a.e < b.e; });
            }
        for (size_t i = 0; i < out.size(); i++) {
            out_e[i] = out[i].e;
            std::memcpy(out_conf + i * conf_size, out[i].c.data(), conf_size * sizeof(double));
            std::memcpy(out_coords + i * H3, out[i].x.data(), H3 * sizeof(double));
        }
        *out_count = (int)out.size();
    });
}

}  // extern "C"
