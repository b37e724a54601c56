/*
 * Host side of the B200 docking engine (C++17, no Boost).
 *
 * Covers what smina's CPU library does around the GPU search: atom typing,
 * scoring terms and their precalculated pair tables, ligand torsion trees
 * read from PDBQT, search parameters, chain seeding, output merging, and the
 * synthetic receptors/ligands used for benchmarking.  Everything here feeds
 * the flat descriptors of include/smina_b200.h.
 */
#ifndef SG_HOST_H
#define SG_HOST_H

#include <cstdint>
#include <memory>
#include <string>
#include <vector>
#include "../../include/smina_b200.h"

namespace sgh {

// ---- atom types (atom_constants.h:85-376) --------------------------------
enum Smt {
    Hydrogen, PolarHydrogen, AliphaticCarbonXSHydrophobe, AliphaticCarbonXSNonHydrophobe,
    AromaticCarbonXSHydrophobe, AromaticCarbonXSNonHydrophobe, Nitrogen, NitrogenXSDonor,
    NitrogenXSDonorAcceptor, NitrogenXSAcceptor, Oxygen, OxygenXSDonor, OxygenXSDonorAcceptor,
    OxygenXSAcceptor, Sulfur, SulfurAcceptor, Phosphorus, Fluorine, Chlorine, Bromine, Iodine,
    Magnesium, Manganese, Zinc, Calcium, Iron, GenericMetal, NumTypes
};
struct TypeInfo {
    const char* name;
    const char* ad;
    int el;  // element class (EL_TYPE_*)
    double ad_radius, ad_depth, ad_solvation, ad_volume, covalent_radius, xs_radius;
    bool xs_hydrophobe, xs_donor, xs_acceptor, ad_heteroatom;
};
// active table (default or vinardo parameters, like smina_atom_type::data)
const TypeInfo& type_info(int t);
void use_type_table(bool vinardo);
int type_from_ad_name(const std::string& ad);  // string_to_smina_type for <= 2 chars
int type_from_name(const std::string& name);   // string_to_smina_type
int adjust_type(int t, bool h_bonded, bool hetero_bonded);  // adjust_smina_type
inline bool is_hydrogen(int t) { return t == Hydrogen || t == PolarHydrogen; }

// ---- scoring function (everything.h, weighted_terms.cpp) -------------------
struct Term {
    virtual ~Term() {}
    virtual bool charge_dependent() const { return false; }
    // charge-independent value, or the 4 components for charge-dependent terms
    virtual double eval(int t1, int t2, double r) const = 0;
    virtual void eval_components(int t1, int t2, double r, double out[4]) const {
        out[0] = eval(t1, t2, r); out[1] = out[2] = out[3] = 0;
    }
    double cutoff = 8;
    std::string name;
};
struct Scoring {
    std::vector<std::unique_ptr<Term>> indep, dep;   // charge independent / dependent, in file order
    std::vector<double> indep_w, dep_w;
    std::vector<std::string> conf_indep_names;       // num_tors_div ...
    std::vector<double> conf_indep_w;
    bool vinardo_types = false;
    double cutoff() const;
    int num_components() const { return dep.empty() ? 1 : 4; }
    void eval_fast(int t1, int t2, double r, double out[4]) const;  // weighted_terms::eval_fast
    // add "weight term(...)"; throws std::runtime_error on unknown terms
    void add(const std::string& term, double weight);
};
// builtin sets "vina"/"default", "vinardo", "dkoes_scoring", "ad4_scoring" ...
bool builtin_scoring(const std::string& name, Scoring& s);
// custom scoring file: "<weight> <term>" per line, '#' comments
void scoring_from_text(const std::string& text, Scoring& s);

// precalculate_linear tables (precalculate.h:187-308)
struct Tables {
    int nc = 1, n = 0;
    double factor = 32, cutoff_sqr = 64;
    std::vector<double> smooth, fast;
    sg_tables_desc desc() const;
};
void build_linear_tables(const Scoring& sf, double factor, Tables& out);
// weighted_terms::conf_independent: the conf-independent terms in order
double conf_independent(const std::vector<std::string>& names, const std::vector<double>& weights, const double in[7],
                        double x);

// ---- molecules --------------------------------------------------------------
struct Atom {
    int number = 0;   // PDBQT serial
    int type = NumTypes;
    double charge = 0;
    double xyz[3] = {0, 0, 0};
    std::string name, resname;
};

// A docking model: ligand(s) (+ flexible residues) flattened in smina order.
struct Model {
    int num_movable = 0;
    std::vector<int> type;
    std::vector<double> charge, local, lab;      // 3 per atom
    std::vector<int> fkind, fparent, fbegin, fend, fconf, fdof;
    std::vector<double> forigin, faxis, finit;   // 3 per frame
    std::vector<int> lig_pair_end, lig_begin, lig_end, lig_root;
    std::vector<int> pairs;                      // 2 per pair
    int num_other_pairs = 0;
    int num_ligands = 0, num_flex = 0, conf_size = 0, dof = 0;
    int torsdof = 0;                              // TORSDOF of the ligand
    // conf_independent_inputs of the ligand(s): num_tors, num_rotors,
    // num_heavy_atoms, num_hydrophobic_atoms, ligand_max_num_h_bonds,
    // num_ligands, ligand_lengths_sum
    double ci[7] = {0, 0, 0, 0, 0, 0, 0};
    std::string name;
    sg_model_desc desc() const;
    int num_heavy_movable() const;
    int num_torsions() const { return dof - 6 * num_ligands; }
};

// Reads one PDBQT ligand (ROOT/BRANCH/TORSDOF) the way parse_pdbqt.cpp:209-353
// does, types it (model.cpp:448-566) and builds its pairs (model.cpp:598-624).
// Throws std::runtime_error on malformed input.
Model read_pdbqt_ligand(const std::string& text);
// SDF / MOL V2000 records: how many, and record `index` as the PDBQT the
// reference's converter writes (sdf.cpp)
int sdf_count(const std::string& text);
std::vector<size_t> sdf_starts(const std::string& text);  // byte offset of each record
std::string pdbqt_from_sdf(const std::string& text, int index, bool add_hydrogens);
// A ligand with the receptor's flexible residues (smina --flex): residues in
// PDBQT BEGIN_RES/END_RES blocks (parse_pdbqt.cpp:412-437), the ligand
// appended as model::append does.
Model read_pdbqt_flex(const std::string& ligand_text, const std::string& flex_text);

// ---- synthetic workloads ---------------------------------------------------
struct Receptor {
    std::vector<Atom> atoms;  // heavy atoms and polar H, typed
    sg_receptor_desc desc(std::vector<double>& xyz, std::vector<int>& t, std::vector<double>& q) const;
};
// Seeded random-walk chains of 1.5 A bonds with >= 3.0 A non-bonded spacing
// around `center`, an 8 A cavity carved at the centre, polar H on donors.
Receptor make_receptor(int heavy_atoms, uint64_t seed, const double center[3], double cavity_radius = 8.0);
std::string receptor_pdbqt(const Receptor& r);
// Acyclic drug-like ligand: `heavy` heavy atoms, exactly `rotors` torsions,
// placed near `center`; returned as PDBQT text.
std::string make_ligand_pdbqt(int heavy, int rotors, uint64_t seed, const double center[3]);
// `residues` flexible side chains with 2..4 chi torsions each, CA on a shell
// of radius `shell` around `center`, side chains pointing into the cavity;
// returned as flex PDBQT (BEGIN_RES ... END_RES).
std::string make_flex_pdbqt(int residues, uint64_t seed, const double center[3], double shell = 9.0);

// grid_dims for a cubic box of `size` A at granularity 0.375 (main.cpp:801-809)
sg_grid_dims make_box(const double center[3], const double size[3], double granularity = 0.375);

// ---- search parameters and seeding -------------------------------------------
// setup_search (main.cpp:513-529): steps, maxiters, ...
sg_mc_params search_params(const Model& m, int num_modes = 9);
struct FastPlan {
    int split = 1;
    double fraction = 1;
    unsigned steps = 1;
};
FastPlan fast_plan(size_t tasks, size_t capacity, int chain_split, double step_fraction, double budget,
                   unsigned steps);
unsigned search_steps(const Model& m);

// mt19937 (Boost semantics)
struct MT {
    uint32_t x[624];
    int i;
    void seed(uint32_t s);
    uint32_t next();
};
double random_fl(double a, double b, MT& g);
int random_int(int a, int b, MT& g);
// standard normal by the Marsaglia polar method (Marsaglia & Bray 1964)
double random_normal(MT& g);

// A chain of the plain path: start conf and the generator state after
// conf::randomize (conf.h:355-360); the orientation uses random_normal.
struct ChainStart {
    std::vector<double> conf;
    uint32_t mt[625];
};
ChainStart make_chain(const Model& m, uint32_t seed, const sg_grid_dims& box);
// parallel_mc seeding (parallel_mc.cpp:80-98): a generator seeded with `seed`
// hands each of `tasks` chains random_int(0, 1000000)
std::vector<ChainStart> seed_chains(const Model& m, int seed, int tasks, const sg_grid_dims& box);

}  // namespace sgh
#endif
