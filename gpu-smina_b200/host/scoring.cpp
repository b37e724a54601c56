/*
 * Atom types, scoring terms and precalculate_linear tables.
 *
 * The per-type constants are smina's (atom_constants.h:134-183 default,
 * builtinscoring.cpp:8-61 vinardo); they are data and have to match.  Term
 * formulas follow everything.h:49-545 and their combination
 * weighted_terms.cpp:52-62; tables follow precalculate.h:92-308.
 */
#include "sg_host.h"
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <limits>
#include <regex>
#include <sstream>
#include <stdexcept>

namespace sgh {

enum { EL_H, EL_C, EL_N, EL_O, EL_S, EL_P, EL_F, EL_Cl, EL_Br, EL_I, EL_Met };

// name, ad, el, ad_radius, ad_depth, ad_solvation, ad_volume, covalent, xs_radius, hydrophobe, donor, acceptor, hetero
static const TypeInfo kDefault[NumTypes] = {
    {"Hydrogen", "H", EL_H, 1.0, 0.02, 0.00051, 0.0, 0.37, 0.0, false, false, false, false},
    {"PolarHydrogen", "HD", EL_H, 1.0, 0.02, 0.00051, 0.0, 0.37, 0.0, false, false, false, false},
    {"AliphaticCarbonXSHydrophobe", "C", EL_C, 2.0, 0.15, -0.00143, 33.5103, 0.77, 1.9, true, false, false, false},
    {"AliphaticCarbonXSNonHydrophobe", "C", EL_C, 2.0, 0.15, -0.00143, 33.5103, 0.77, 1.9, false, false, false, false},
    {"AromaticCarbonXSHydrophobe", "A", EL_C, 2.0, 0.15, -0.00052, 33.5103, 0.77, 1.9, true, false, false, false},
    {"AromaticCarbonXSNonHydrophobe", "A", EL_C, 2.0, 0.15, -0.00052, 33.5103, 0.77, 1.9, false, false, false, false},
    {"Nitrogen", "N", EL_N, 1.75, 0.16, -0.00162, 22.4493, 0.75, 1.8, false, false, false, true},
    {"NitrogenXSDonor", "N", EL_N, 1.75, 0.16, -0.00162, 22.4493, 0.75, 1.8, false, true, false, true},
    {"NitrogenXSDonorAcceptor", "NA", EL_N, 1.75, 0.16, -0.00162, 22.4493, 0.75, 1.8, false, true, true, true},
    {"NitrogenXSAcceptor", "NA", EL_N, 1.75, 0.16, -0.00162, 22.4493, 0.75, 1.8, false, false, true, true},
    {"Oxygen", "O", EL_O, 1.6, 0.2, -0.00251, 17.1573, 0.73, 1.7, false, false, false, true},
    {"OxygenXSDonor", "O", EL_O, 1.6, 0.2, -0.00251, 17.1573, 0.73, 1.7, false, true, false, true},
    {"OxygenXSDonorAcceptor", "OA", EL_O, 1.6, 0.2, -0.00251, 17.1573, 0.73, 1.7, false, true, true, true},
    {"OxygenXSAcceptor", "OA", EL_O, 1.6, 0.2, -0.00251, 17.1573, 0.73, 1.7, false, false, true, true},
    {"Sulfur", "S", EL_S, 2.0, 0.2, -0.00214, 33.5103, 1.02, 2.0, false, false, false, true},
    {"SulfurAcceptor", "SA", EL_S, 2.0, 0.2, -0.00214, 33.5103, 1.02, 2.0, false, false, false, true},
    {"Phosphorus", "P", EL_P, 2.1, 0.2, -0.0011, 38.7924, 1.06, 2.1, false, false, false, true},
    {"Fluorine", "F", EL_F, 1.545, 0.08, -0.0011, 15.448, 0.71, 1.5, true, false, false, true},
    {"Chlorine", "Cl", EL_Cl, 2.045, 0.276, -0.0011, 35.8235, 0.99, 1.8, true, false, false, true},
    {"Bromine", "Br", EL_Br, 2.165, 0.389, -0.0011, 42.5661, 1.14, 2.0, true, false, false, true},
    {"Iodine", "I", EL_I, 2.36, 0.55, -0.0011, 55.0585, 1.33, 2.2, true, false, false, true},
    {"Magnesium", "Mg", EL_Met, 0.65, 0.875, -0.0011, 1.56, 1.3, 1.2, false, true, false, true},
    {"Manganese", "Mn", EL_Met, 0.65, 0.875, -0.0011, 2.14, 1.39, 1.2, false, true, false, true},
    {"Zinc", "Zn", EL_Met, 0.74, 0.55, -0.0011, 1.7, 1.31, 1.2, false, true, false, true},
    {"Calcium", "Ca", EL_Met, 0.99, 0.55, -0.0011, 2.77, 1.74, 1.2, false, true, false, true},
    {"Iron", "Fe", EL_Met, 0.65, 0.01, -0.0011, 1.84, 1.25, 1.2, false, true, false, true},
    {"GenericMetal", "M", EL_Met, 1.2, 0.0, -0.0011, 22.4493, 1.75, 1.2, false, true, false, true},
};

static TypeInfo g_active[NumTypes];
static bool g_init = false;
static void ensure_table() {
    if (!g_init) { std::copy(kDefault, kDefault + NumTypes, g_active); g_init = true; }
}
const TypeInfo& type_info(int t) { ensure_table(); return g_active[t]; }

// vinardo's own radii and hydrophobicity (builtinscoring.cpp:8-61)
void use_type_table(bool vinardo) {
    std::copy(kDefault, kDefault + NumTypes, g_active);
    g_init = true;
    if (!vinardo) return;
    const double xs[NumTypes] = {0, 0, 2.0, 2.0, 1.9, 1.9, 1.7, 1.7, 1.7, 1.7, 1.6, 1.6, 1.6, 1.6,
                                 2.0, 2.0, 2.1, 1.5, 1.8, 2.0, 2.2, 1.2, 1.2, 1.2, 1.2, 1.2, 1.2};
    for (int t = 0; t < NumTypes; t++) g_active[t].xs_radius = xs[t];
    g_active[AromaticCarbonXSNonHydrophobe].xs_hydrophobe = true;
    g_active[SulfurAcceptor].xs_hydrophobe = true;
}

int type_from_ad_name(const std::string& ad) {
    ensure_table();
    for (int t = 0; t < NumTypes; t++)
        if (ad == g_active[t].ad) return t;
    if (ad == "Se") return type_from_ad_name("S");
    static const char* metals[] = {"Cu", "Fe", "Na", "K", "Hg", "Co", "U", "Cd", "Ni"};
    for (const char* m : metals)
        if (ad == m) return GenericMetal;
    return NumTypes;
}

// string_to_smina_type (atom_constants.h:294-327): two characters or fewer
// name an AD4 type, longer names a smina type (atom_type_* scoring terms)
int type_from_name(const std::string& name) {
    if (name.size() <= 2) return type_from_ad_name(name);
    ensure_table();
    for (int t = 0; t < NumTypes; t++)
        if (name == g_active[t].name) return t;
    return NumTypes;
}

int adjust_type(int t, bool hb, bool het) {
    switch (t) {
        case AliphaticCarbonXSHydrophobe:
        case AliphaticCarbonXSNonHydrophobe:
            return het ? AliphaticCarbonXSNonHydrophobe : AliphaticCarbonXSHydrophobe;
        case AromaticCarbonXSHydrophobe:
        case AromaticCarbonXSNonHydrophobe:
            return het ? AromaticCarbonXSNonHydrophobe : AromaticCarbonXSHydrophobe;
        case NitrogenXSDonor:
        case Nitrogen:
            return hb ? NitrogenXSDonor : Nitrogen;
        case NitrogenXSDonorAcceptor:
        case NitrogenXSAcceptor:
            return hb ? NitrogenXSDonorAcceptor : NitrogenXSAcceptor;
        case OxygenXSDonor:
        case Oxygen:
            return hb ? OxygenXSDonor : Oxygen;
        case OxygenXSDonorAcceptor:
        case OxygenXSAcceptor:
            return hb ? OxygenXSDonorAcceptor : OxygenXSAcceptor;
        default:
            return t;
    }
}

// ---- term primitives (everything.h) ------------------------------------------
static const double kEps = std::numeric_limits<double>::epsilon();
static double optimal_distance(int a, int b) { return type_info(a).xs_radius + type_info(b).xs_radius; }
static double gaussian(double x, double w) { double q = x / w; return std::exp(-(q * q)); }
static double slope_step(double bad, double good, double x) {
    if (bad < good) {
        if (x <= bad) return 0;
        if (x >= good) return 1;
    } else {
        if (x >= bad) return 0;
        if (x <= good) return 1;
    }
    return (x - bad) / (good - bad);
}
static double ipow(double x, int n) {  // int_pow<n>: ((1*x)*x)...
    double r = 1;
    for (int i = 0; i < n; i++) r = r * x;
    return r;
}
static bool hb_possible(int a, int b) {
    const TypeInfo &A = type_info(a), &B = type_info(b);
    return (A.xs_donor && B.xs_acceptor) || (B.xs_donor && A.xs_acceptor);
}
static bool anti_hb(int a, int b) {
    const TypeInfo &A = type_info(a), &B = type_info(b);
    if (A.xs_donor && !A.xs_acceptor) return B.xs_donor && !B.xs_acceptor;
    if (!A.xs_donor && A.xs_acceptor) return !B.xs_donor && B.xs_acceptor;
    return false;
}
static void vdw_coeffs(int n, int m, double pos, double depth, double& cn, double& cm) {
    cn = ipow(pos, n) * depth * m / ((double)n - (double)m);
    cm = ipow(pos, m) * depth * n / ((double)m - (double)n);
}

struct GaussT : Term { double o, w; double eval(int a, int b, double r) const override { return gaussian(r - (optimal_distance(a, b) + o), w); } };
struct RepulsionT : Term { double o; double eval(int a, int b, double r) const override { double d = r - (optimal_distance(a, b) + o); return d > 0 ? 0 : d * d; } };
struct HydrophobicT : Term {
    double g, b; bool non;
    double eval(int t1, int t2, double r) const override {
        bool h1 = type_info(t1).xs_hydrophobe, h2 = type_info(t2).xs_hydrophobe;
        bool ok = non ? (!h1 && !h2) : (h1 && h2);
        return ok ? slope_step(b, g, r - optimal_distance(t1, t2)) : 0;
    }
};
struct HBondT : Term { double g, b; double eval(int t1, int t2, double r) const override { return hb_possible(t1, t2) ? slope_step(b, g, r - optimal_distance(t1, t2)) : 0; } };
struct VdwT : Term {
    int i, j; double s, cap;
    double eval(int t1, int t2, double r) const override {
        double d0 = optimal_distance(t1, t2), ci, cj;
        vdw_coeffs(i, j, d0, 1, ci, cj);
        if (r > d0 + s) r -= s;
        else if (r < d0 - s) r += s;
        else r = d0;
        double ri = ipow(r, i), rj = ipow(r, j);
        if (ri > kEps && rj > kEps) return std::min(cap, ci / ri + cj / rj);
        return cap;
    }
};
struct HBondLJT : Term {
    double o, cap;
    double eval(int t1, int t2, double r) const override {
        if (!hb_possible(t1, t2)) return 0;
        double d0 = optimal_distance(t1, t2) + o, ci, cj;
        vdw_coeffs(10, 12, d0, 5, ci, cj);
        double ri = ipow(r, 10), rj = ipow(r, 12);
        if (ri > kEps && rj > kEps) return std::min(cap, ci / ri + cj / rj);
        return cap;
    }
};
struct QuadT : Term {  // anti-h-bond / donor-donor / acceptor-acceptor quadratic
    double o; int kind;
    double eval(int t1, int t2, double r) const override {
        bool ok = kind == 0 ? anti_hb(t1, t2)
                : kind == 1 ? (type_info(t1).xs_donor && type_info(t2).xs_donor)
                            : (type_info(t1).xs_acceptor && type_info(t2).xs_acceptor);
        if (!ok) return 0;
        double d = r - (optimal_distance(t1, t2) + o);
        return d > 0 ? 0 : d * d;
    }
};
struct ElectroT : Term {
    int p; double cap;
    bool charge_dependent() const override { return true; }
    double eval(int, int, double) const override { return 0; }
    void eval_components(int, int, double r, double out[4]) const override {
        out[0] = out[1] = out[2] = 0;
        double t = ipow(r, p);
        out[3] = t < kEps ? cap : std::min(cap, 1 / t);
    }
};
struct SolvT : Term {
    double sigma, q;
    bool charge_dependent() const override { return true; }
    double eval(int, int, double) const override { return 0; }
    void eval_components(int t1, int t2, double r, double out[4]) const override {
        const TypeInfo &A = type_info(t1), &B = type_info(t2);
        double x = r / (2 * sigma);
        double df = std::exp(-(x * x));
        out[0] = out[1] = out[2] = out[3] = 0;
        out[0] += A.ad_solvation * B.ad_volume * df;
        out[1] += q * B.ad_volume * df;
        out[0] += B.ad_solvation * A.ad_volume * df;
        out[2] += q * A.ad_volume * df;
    }
};
struct PairTypeT : Term {  // atom_type_* terms
    int a, b, kind; double p1, p2, cap; int power;
    bool match(int x, int y) const { return (x == a && y == b) || (x == b && y == a); }
    double eval(int t1, int t2, double r) const override {
        if (!match(t1, t2)) return 0;
        switch (kind) {
            case 0: return gaussian(r - (optimal_distance(a, b) + p1), p2);
            case 1: return slope_step(p2, p1, r - optimal_distance(a, b));
            case 2: { double d = r - (optimal_distance(a, b) + p1); return d > 0 ? 0 : d * d; }
            default: { double t = ipow(r, power); return t < kEps ? cap : std::min(cap, 1 / t); }
        }
    }
};

double Scoring::cutoff() const {
    double c = 0;
    for (auto& t : indep) c = std::max(c, t->cutoff);
    for (auto& t : dep) c = std::max(c, t->cutoff);
    return c;
}

// weighted_terms::eval_fast (weighted_terms.cpp:52-62)
void Scoring::eval_fast(int t1, int t2, double r, double out[4]) const {
    out[0] = out[1] = out[2] = out[3] = 0;
    for (size_t i = 0; i < indep.size(); i++) out[0] += indep_w[i] * indep[i]->eval(t1, t2, r);
    for (size_t i = 0; i < dep.size(); i++) {
        double c[4];
        dep[i]->eval_components(t1, t2, r, c);
        for (int k = 0; k < 4; k++) c[k] *= dep_w[i];
        for (int k = 0; k < 4; k++) out[k] += c[k];
    }
}

static std::vector<std::string> split_args(const std::string& inside) {
    std::vector<std::string> out;
    std::stringstream ss(inside);
    std::string tok;
    while (std::getline(ss, tok, ',')) out.push_back(tok);
    return out;
}
static double argval(const std::string& kv) {
    size_t eq = kv.find('=');
    if (eq == std::string::npos) throw std::runtime_error("bad term parameter: " + kv);
    return std::stod(kv.substr(eq + 1));
}
static std::string argstr(const std::string& kv) {
    size_t eq = kv.find('=');
    if (eq == std::string::npos) throw std::runtime_error("bad term parameter: " + kv);
    return kv.substr(eq + 1);
}

// term names and parameter syntax of everything.h (regex per term)
void Scoring::add(const std::string& desc, double w) {
    static const char* conf_terms[] = {"num_tors_add", "num_tors_sqr", "num_tors_sqrt", "num_tors_div",
                                       "num_tors_div_simple", "ligand_length", "num_ligands", "num_heavy_atoms_div",
                                       "num_heavy_atoms", "num_hydrophobic_atoms", "constant_term"};
    for (const char* c : conf_terms)
        if (desc == c) { conf_indep_names.push_back(desc); conf_indep_w.push_back(w); return; }
    size_t lp = desc.find('(');
    if (lp == std::string::npos || desc.back() != ')') throw std::runtime_error("Unknown term " + desc);
    std::string name = desc.substr(0, lp);
    std::vector<std::string> a = split_args(desc.substr(lp + 1, desc.size() - lp - 2));
    std::unique_ptr<Term> t;
    auto need = [&](size_t n) { if (a.size() != n) throw std::runtime_error("Could not convert parameters. " + desc); };
    if (name == "gauss") {
        need(3); auto* g = new GaussT; g->o = argval(a[0]); g->w = argval(a[1]); g->cutoff = argval(a[2]); t.reset(g);
    } else if (name == "repulsion") {
        need(2); auto* g = new RepulsionT; g->o = argval(a[0]); g->cutoff = argval(a[1]); t.reset(g);
    } else if (name == "hydrophobic" || name == "non_hydrophobic") {
        need(3); auto* g = new HydrophobicT; g->g = argval(a[0]); g->b = argval(a[1]); g->cutoff = argval(a[2]);
        g->non = name == "non_hydrophobic"; t.reset(g);
    } else if (name == "non_dir_h_bond") {
        need(3); auto* g = new HBondT; g->g = argval(a[0]); g->b = argval(a[1]); g->cutoff = argval(a[2]); t.reset(g);
    } else if (name == "vdw") {
        need(5); auto* g = new VdwT;
        const double vi = argval(a[0]), vj = argval(a[1]);
        if (!((vi == 4 && vj == 8) || (vi == 6 && vj == 12)))
            throw std::runtime_error("Unsupported LJ exponents: try <4,8> or <6,12>.");
        g->i = (int)vi; g->j = (int)vj; g->s = argval(a[2]); g->cap = argval(a[3]); g->cutoff = argval(a[4]);
        t.reset(g);
    } else if (name == "non_dir_h_bond_lj") {
        need(3); auto* g = new HBondLJT; g->o = argval(a[0]); g->cap = argval(a[1]); g->cutoff = argval(a[2]); t.reset(g);
    } else if (name == "non_dir_anti_h_bond_quadratic" || name == "donor_donor_quadratic" ||
               name == "acceptor_acceptor_quadratic") {
        need(2); auto* g = new QuadT; g->o = argval(a[0]); g->cutoff = argval(a[1]);
        g->kind = name[0] == 'n' ? 0 : name[0] == 'd' ? 1 : 2; t.reset(g);
    } else if (name == "electrostatic") {
        need(3); auto* g = new ElectroT;
        const double i = argval(a[0]);
        if (i != 1 && i != 2) throw std::runtime_error("Invalid exponent: 1 or 2 only");
        g->p = (int)i; g->cap = argval(a[1]); g->cutoff = argval(a[2]);
        t.reset(g);
    } else if (name == "ad4_solvation") {
        need(3); auto* g = new SolvT; g->sigma = argval(a[0]); g->q = argval(a[1]); g->cutoff = argval(a[2]); t.reset(g);
    } else if (name.rfind("atom_type_", 0) == 0) {
        auto* g = new PairTypeT;
        std::string n1 = argstr(a.at(0)), n2 = argstr(a.at(1));
        g->a = type_from_name(n1); g->b = type_from_name(n2);
        if (g->a == NumTypes || g->b == NumTypes) throw std::runtime_error("Invalid atom type: " + desc);
        if (name == "atom_type_gaussian") { need(5); g->kind = 0; g->p1 = argval(a[2]); g->p2 = argval(a[3]); g->cutoff = argval(a[4]); }
        else if (name == "atom_type_linear") { need(5); g->kind = 1; g->p1 = argval(a[2]); g->p2 = argval(a[3]); g->cutoff = argval(a[4]); }
        else if (name == "atom_type_quadratic") { need(4); g->kind = 2; g->p1 = argval(a[2]); g->cutoff = argval(a[3]); }
        else if (name == "atom_type_inverse_power") {
            need(5);
            g->kind = 3;
            const double i = argval(a[2]);
            if (i != 1 && i != 2) throw std::runtime_error("Invalid exponent: 1 or 2 only");
            g->power = (int)i; g->cap = argval(a[3]); g->cutoff = argval(a[4]);
        }
        else throw std::runtime_error("Unknown term " + desc);
        t.reset(g);
    } else {
        throw std::runtime_error("Unknown term " + desc);
    }
    t->name = desc;
    if (t->charge_dependent()) { dep.push_back(std::move(t)); dep_w.push_back(w); }
    else { indep.push_back(std::move(t)); indep_w.push_back(w); }
}

// builtinscoring.cpp:63-105
bool builtin_scoring(const std::string& name, Scoring& s) {
    auto add = [&](const char* t, double w) { s.add(t, w); };
    if (name == "vina" || name == "default") {
        add("gauss(o=0,_w=0.5,_c=8)", -0.035579);
        add("gauss(o=3,_w=2,_c=8)", -0.005156);
        add("repulsion(o=0,_c=8)", 0.840245);
        add("hydrophobic(g=0.5,_b=1.5,_c=8)", -0.035069);
        add("non_dir_h_bond(g=-0.7,_b=0,_c=8)", -0.587439);
        add("num_tors_div", 5 * 0.05846 / 0.1 - 1);
    } else if (name == "vinardo") {
        add("gauss(o=0,_w=0.8,_c=8)", -0.045);
        add("repulsion(o=0,_c=8)", 0.80);
        add("hydrophobic(g=0.0,_b=2.5,_c=8)", -0.035);
        add("non_dir_h_bond(g=-0.6,_b=0,_c=8)", -0.60);
        add("num_tors_div", 5 * 0.02 / 0.1 - 1);
        s.vinardo_types = true;
    } else if (name == "dkoes_scoring") {
        add("vdw(i=4,_j=8,_s=0,_^=100,_c=8)", 0.009900);
        add("non_dir_h_bond(g=-0.7,_b=0,_c=8)", -0.153055);
        add("ad4_solvation(d-sigma=3.6,_s/q=0.01097,_c=8)", 0.048934);
        add("num_tors_sqr", 0.317267);
        add("constant_term", -2.469020);
    } else if (name == "dkoes_scoring_old") {
        add("vdw(i=4,_j=8,_s=0,_^=100,_c=8)", 0.010607);
        add("non_dir_h_bond(g=-0.7,_b=0,_c=8)", 0.197201);
        add("num_tors_sqr", .285035);
        add("constant_term", -2.585651);
    } else if (name == "dkoes_fast") {
        add("vdw(i=4,_j=8,_s=0,_^=100,_c=8)", 0.008962);
        add("non_dir_h_bond(g=-0.7,_b=0,_c=8)", 0.387739);
        add("num_tors_sqr", .285035);
        add("constant_term", -2.467357);
    } else if (name == "ad4_scoring") {
        add("vdw(i=6,_j=12,_s=0,_^=100,_c=8)", 0.1560);
        add("non_dir_h_bond_lj(o=-0.7,_^=100,_c=8)", -0.0974);
        add("ad4_solvation(d-sigma=3.5,_s/q=0.01097,_c=8)", 0.1159);
        add("electrostatic(i=1,_^=100,_c=8)", 0.1465);
        add("num_tors_add", 0.2744);
    } else {
        return false;
    }
    return true;
}

// custom_terms::add_terms_from_file (custom_terms.cpp:56-71)
void scoring_from_text(const std::string& text, Scoring& s) {
    std::stringstream in(text);
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::stringstream ls(line);
        double w = 0;
        std::string name;
        if ((ls >> w >> name) && !name.empty()) s.add(name, w);
    }
}

sg_tables_desc Tables::desc() const {
    sg_tables_desc d;
    d.num_types = NumTypes;
    d.num_components = nc;
    d.n = n;
    d.factor = factor;
    d.cutoff_sqr = cutoff_sqr;
    d.smooth = smooth.data();
    d.fast = fast.data();
    return d;
}

// precalculate_linear ctor + init_from_smooth_fst (precalculate.h:153-180, 206-237)
void build_linear_tables(const Scoring& sf, double factor, Tables& T) {
    use_type_table(sf.vinardo_types);
    const double cutoff = sf.cutoff();
    T.cutoff_sqr = cutoff * cutoff;
    T.factor = factor;
    T.nc = sf.num_components();
    T.n = (int)(size_t)(factor * T.cutoff_sqr) + 3;
    const int n = T.n, nc = T.nc;
    std::vector<double> rs(n + 2);
    for (int i = 0; i < n + 2; i++) rs[i] = std::sqrt((size_t)i / factor);
    const int np = NumTypes * (NumTypes + 1) / 2;
    T.smooth.assign((size_t)np * n * nc * 2, 0.0);
    T.fast.assign((size_t)np * n * nc, 0.0);
    double res[4];
    for (int t1 = 0; t1 < NumTypes; t1++)
        for (int t2 = t1; t2 < NumTypes; t2++) {
            const int p = t1 + t2 * (t2 + 1) / 2;
            double* S = &T.smooth[(size_t)p * n * nc * 2];
            double* F = &T.fast[(size_t)p * n * nc];
            auto e_at = [&](int i, int c) -> double& { return S[((size_t)i * nc + c) * 2]; };
            auto d_at = [&](int i, int c) -> double& { return S[((size_t)i * nc + c) * 2 + 1]; };
            for (int i = 0; i < n; i++) {
                sf.eval_fast(t1, t2, rs[i], res);
                for (int c = 0; c < nc; c++) e_at(i, c) = res[c];
            }
            for (int c = 0; c < nc; c++)
                for (int i = 0; i < n; i++) {
                    double& dor = d_at(i, c);
                    if (i == 0 || i == n - 1) dor = 0;
                    else {
                        double delta = rs[i + 1] - rs[i - 1];
                        double r = rs[i];
                        dor = (e_at(i + 1, c) - e_at(i - 1, c)) / (delta * r);
                    }
                    double f1 = e_at(i, c);
                    double f2 = (i + 1 >= n) ? 0 : e_at(i + 1, c);
                    F[(size_t)i * nc + c] = (f2 + f1) / 2;
                }
        }
}

// smooth_div (everything.h:55-59)
static double smooth_div(double x, double y) {
    if (std::abs(x) < DBL_EPSILON) return 0;
    if (std::abs(y) < DBL_EPSILON) return (x * y > 0) ? DBL_MAX : -DBL_MAX;
    return x / y;
}

// weighted_terms::conf_independent (weighted_terms.cpp:74-80): the enabled
// conf-independent terms in order (terms.cpp:311-318), each with its own
// weight, formulas of everything.h:730-1000.  in: num_tors, num_rotors,
// num_heavy_atoms, num_hydrophobic_atoms, ligand_max_num_h_bonds,
// num_ligands, ligand_lengths_sum.
double conf_independent(const std::vector<std::string>& names, const std::vector<double>& weights, const double in[7],
                        double x) {
    for (size_t k = 0; k < names.size(); k++) {
        const std::string& n = names[k];
        const double r = weights[k];
        if (n == "num_tors_add") {
            x = x + r * in[0];
        } else if (n == "num_tors_sqr") {
            const double w = 0.1 * r;
            x = x + w * (in[0] * in[0]) / 5;
        } else if (n == "num_tors_sqrt") {
            const double w = 0.1 * r;
            x = x + w * std::sqrt(in[0]) / std::sqrt(5.0);
        } else if (n == "num_tors_div") {
            const double w = 0.1 * (r + 1);
            x = smooth_div(x, 1 + w * in[0] / 5.0);
        } else if (n == "num_tors_div_simple") {
            x = smooth_div(x, 1 + r * in[0]);
        } else if (n == "ligand_length") {
            x = x + r * in[6];
        } else if (n == "num_ligands") {
            const double w = 1 * r;
            x = x + w * in[5];
        } else if (n == "num_heavy_atoms_div") {
            const double w = 0.05 * r;
            x = smooth_div(x, 1 + w * in[2]);
        } else if (n == "num_heavy_atoms") {
            const double w = 0.05 * r;
            x = x + w * in[2];
        } else if (n == "num_hydrophobic_atoms") {
            const double w = 0.05 * r;
            x = x + w * in[3];
        } else if (n == "constant_term") {
            x = x + r;
        } else {
            throw std::runtime_error("unknown conf-independent term " + n);
        }
    }
    return x;
}

}  // namespace sgh

