/*
 * PDBQT ligand reader and model flattening.
 *
 * Restates smina's PDBQT tree semantics (parse_pdbqt.cpp:209-353,
 * parsing.h:111-232): BRANCH blocks hang off the atom they name; the
 * branch's axis atom ("immobile atom") is stored in the parent's frame;
 * branches that move only hydrogens are merged into their parent; frames
 * are numbered depth-first.  Bond perception (model.cpp:448-529), typing
 * (model.cpp:555-566, adjust_smina_type) and the intramolecular pair list
 * (model.cpp:598-624) follow the reference.
 */
#include "sg_host.h"
#include <algorithm>
#include <array>
#include <cmath>
#include <functional>
#include <sstream>
#include <stdexcept>

namespace sgh {

namespace {

struct PS;
struct PNode {
    Atom a;
    std::vector<PS> ps;
};
struct PS {  // parsing_struct
    std::vector<PNode> atoms;
    int immobile = -1;
    int axis_begin = -1, axis_end = -1;
    bool essentially_empty() const {
        for (size_t i = 0; i < atoms.size(); i++) {
            if (immobile >= 0 && immobile != (int)i) return false;
            if (!atoms[i].ps.empty()) return false;
        }
        return true;
    }
    bool mobile_hydrogens_only() const {
        for (size_t i = 0; i < atoms.size(); i++) {
            if (!atoms[i].ps.empty()) return false;
            if (immobile >= 0 && immobile != (int)i && !is_hydrogen(atoms[i].a.type)) return false;
        }
        return true;
    }
    void merge_into(const PS& from) {
        for (const PNode& n : from.atoms) { PNode c; c.a = n.a; atoms.push_back(c); }
    }
};

bool starts(const std::string& s, const char* p) { return s.rfind(p, 0) == 0; }
std::string sub(const std::string& s, size_t a, size_t b) {  // 1-based inclusive columns
    if (s.size() < a) return "";
    return s.substr(a - 1, std::min(b, s.size()) - a + 1);
}
std::string trim(const std::string& s) {
    size_t b = s.find_first_not_of(" \t\r"), e = s.find_last_not_of(" \t\r");
    return b == std::string::npos ? "" : s.substr(b, e - b + 1);
}

// parse_pdbqt_atom_string (parse_pdbqt.cpp:107-121)
Atom parse_atom(const std::string& s) {
    Atom a;
    try {
        a.number = std::stoi(trim(sub(s, 7, 11)));
        a.xyz[0] = std::stod(trim(sub(s, 31, 38)));
        a.xyz[1] = std::stod(trim(sub(s, 39, 46)));
        a.xyz[2] = std::stod(trim(sub(s, 47, 54)));
        std::string q = trim(sub(s, 69, 76));
        a.charge = q.empty() ? 0 : std::stod(q);
    } catch (...) {
        throw std::runtime_error("ATOM syntax incorrect: " + s);
    }
    a.name = trim(sub(s, 13, 16));
    a.resname = trim(sub(s, 18, 20));
    std::string t = trim(sub(s, 78, 79));
    a.type = type_from_ad_name(t);
    if (a.type == NumTypes) throw std::runtime_error("\"" + t + "\" is not a valid AutoDock type.");
    return a;
}

struct Reader {
    std::istringstream in;
    int torsdof = -1;
    explicit Reader(const std::string& t) : in(t) {}
    bool ignorable(const std::string& s) {
        return trim(s).empty() || starts(s, "WARNING") || starts(s, "REMARK") || starts(s, "USER") || starts(s, "TER");
    }
    void branch_aux(const std::string& line, PS& p) {
        std::istringstream ls(line.substr(6));
        int first = -1, second = -1;
        ls >> first >> second;
        if (!ls || first < 0 || second < 0) throw std::runtime_error("Syntax error: " + line);
        for (PNode& n : p.atoms)
            if (n.a.number == first) {
                PS b;
                branch(b, first, second);
                if (b.mobile_hydrogens_only()) p.merge_into(b);
                else n.ps.push_back(std::move(b));
                return;
            }
        throw std::runtime_error("No atom number " + std::to_string(first) + " in this branch");
    }
    void branch(PS& p, int from, int to) {
        std::string s;
        while (std::getline(in, s)) {
            if (trim(s).empty() || starts(s, "WARNING") || starts(s, "REMARK") || starts(s, "USER")) continue;
            if (starts(s, "BRANCH")) branch_aux(s, p);
            else if (starts(s, "ENDBRANCH")) {
                std::istringstream ls(s.substr(9));
                int a = -1, b = -1;
                ls >> a >> b;
                if (a != from || b != to) throw std::runtime_error("Inconsistent branch numbers");
                if (p.immobile < 0) throw std::runtime_error("Atom " + std::to_string(to) + " has not been found in this branch");
                return;
            } else if (starts(s, "ATOM  ") || starts(s, "HETATM")) {
                Atom a = parse_atom(s);
                if (a.number == to) p.immobile = (int)p.atoms.size();
                PNode n; n.a = a; p.atoms.push_back(n);
            } else if (starts(s, "MODEL")) throw std::runtime_error("Unexpected multi-MODEL input");
            else throw std::runtime_error("Unknown or inappropriate tag: " + s);
        }
        throw std::runtime_error("unterminated BRANCH");
    }
    void ligand(PS& p) {
        std::string s;
        bool root = false;
        while (std::getline(in, s)) {
            if (ignorable(s)) continue;
            if (starts(s, "ROOT")) { root = true; break; }
            throw std::runtime_error("Unknown or inappropriate tag: " + s);
        }
        if (!root) throw std::runtime_error("No atoms in the ligand");
        while (std::getline(in, s)) {
            if (ignorable(s)) continue;
            if (starts(s, "ENDROOT")) break;
            if (starts(s, "ATOM  ") || starts(s, "HETATM")) { PNode n; n.a = parse_atom(s); p.atoms.push_back(n); }
            else throw std::runtime_error("Unknown or inappropriate tag: " + s);
        }
        while (std::getline(in, s)) {
            if (ignorable(s)) continue;
            if (starts(s, "BRANCH")) branch_aux(s, p);
            else if (starts(s, "TORSDOF")) {
                if (torsdof >= 0) throw std::runtime_error("TORSDOF can occur only once");
                torsdof = std::stoi(trim(s.substr(7)));
            } else if (starts(s, "MODEL")) throw std::runtime_error("Unexpected multi-MODEL input");
            else throw std::runtime_error("Unknown or inappropriate tag: " + s);
        }
        if (p.atoms.empty()) throw std::runtime_error("No atoms in the ligand");
        if (torsdof < 0) throw std::runtime_error("Missing TORSDOF");
    }
    // parse_pdbqt_residue (parse_pdbqt.cpp:407-410): ROOT, BRANCHes, END_RES
    void residue(PS& p) {
        std::string s;
        bool root = false;
        while (std::getline(in, s)) {
            if (ignorable(s)) continue;
            if (starts(s, "ROOT")) { root = true; break; }
            throw std::runtime_error("Unknown or inappropriate tag: " + s);
        }
        if (!root) throw std::runtime_error("residue without ROOT");
        while (std::getline(in, s)) {
            if (ignorable(s)) continue;
            if (starts(s, "ENDROOT")) break;
            if (starts(s, "ATOM  ") || starts(s, "HETATM")) { PNode n; n.a = parse_atom(s); p.atoms.push_back(n); }
            else throw std::runtime_error("Unknown or inappropriate tag: " + s);
        }
        while (std::getline(in, s)) {
            if (ignorable(s)) continue;
            if (starts(s, "BRANCH")) branch_aux(s, p);
            else if (starts(s, "END_RES")) return;
            else if (starts(s, "MODEL")) throw std::runtime_error("Unexpected multi-MODEL input");
            else throw std::runtime_error("Unknown or inappropriate tag: " + s);
        }
        throw std::runtime_error("residue without END_RES");
    }
};

enum { D_FIXED = 0, D_ROTOR = 1, D_VARIABLE = 2 };

struct Flattener {
    std::vector<Atom> atoms;   // nr.atoms
    std::vector<double> rel;   // relative coords (3 per atom)
    std::vector<int> fparent, fbegin, fend;
    std::vector<double> forigin_lab, faxis_lab;  // lab origin / axis per frame
    std::vector<double> frel_origin;
    std::vector<std::array<int, 3>> mob_fixed;  // (i, j, type) entries to set
    std::vector<std::vector<char>> mob;

    void push_atom(PNode& n, const double* origin, PS* owner_children) {
        (void)owner_children;
        for (PS& c : n.ps) c.axis_begin = (int)atoms.size();
        atoms.push_back(n.a);
        for (int k = 0; k < 3; k++) rel.push_back(n.a.xyz[k] - origin[k]);
    }
    void insert_immobiles(PNode& n, const double* origin) {
        for (PS& c : n.ps)
            if (!c.atoms.empty()) {
                c.axis_end = (int)atoms.size();
                push_atom(c.atoms[c.immobile], origin, nullptr);
            }
    }
    void grow_mob() {
        size_t n = atoms.size();
        for (auto& r : mob) r.resize(n, D_VARIABLE);
        while (mob.size() < n) mob.emplace_back(n, D_VARIABLE);
    }
    void setm(int i, int j, char v) { mob[std::min(i, j)][std::max(i, j)] = v; }
    // postprocess_branch (parse_pdbqt.cpp:306-340)
    void branch(PS& p, int frame) {
        const double* origin = &forigin_lab[3 * frame];
        fbegin[frame] = (int)atoms.size();
        for (size_t i = 0; i < p.atoms.size(); i++) {
            PNode& nd = p.atoms[i];
            if (!(p.immobile >= 0 && (int)i == p.immobile)) push_atom(nd, origin, nullptr);
            insert_immobiles(nd, origin);
        }
        fend[frame] = (int)atoms.size();
        grow_mob();
        if (p.axis_begin >= 0)
            for (int i = fbegin[frame]; i < fend[frame]; i++) setm(p.axis_begin, i, D_FIXED);
        if (p.axis_end >= 0)
            for (int i = fbegin[frame]; i < fend[frame]; i++) setm(p.axis_end, i, D_FIXED);
        if (p.axis_begin >= 0 && p.axis_end >= 0) setm(p.axis_begin, p.axis_end, D_ROTOR);
        for (int i = fbegin[frame]; i < fend[frame]; i++)
            for (int j = i + 1; j < fend[frame]; j++) setm(i, j, D_FIXED);
        for (size_t i = 0; i < p.atoms.size(); i++) {
            PNode& nd = p.atoms[i];
            for (PS& c : nd.ps) {
                if (c.essentially_empty()) continue;
                // segment(origin = immobile atom, axis root = this atom)
                const double* o = c.atoms[c.immobile].a.xyz;
                const double* root = nd.a.xyz;
                double diff[3] = {o[0] - root[0], o[1] - root[1], o[2] - root[2]};
                double nrm = std::sqrt(diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2]);
                if (nrm < 2.220446049250313e-16) throw std::runtime_error("zero-length rotatable bond");
                double inv = 1 / nrm;
                int f = (int)fparent.size();
                fparent.push_back(frame);
                fbegin.push_back(0);
                fend.push_back(0);
                for (int k = 0; k < 3; k++) {
                    forigin_lab.push_back(o[k]);
                    faxis_lab.push_back(inv * diff[k]);
                    frel_origin.push_back(o[k] - forigin_lab[3 * frame + k]);
                }
                branch(c, f);
            }
        }
    }
};

// Flexible residues (parse_pdbqt.cpp:360-380, 412-437): the atoms of a
// residue's ROOT and the axis atom of every ROOT branch are "inflex" (part
// of the model, never moving); every ROOT branch becomes a first_segment
// frame turning about (root atom -> axis atom) at the axis atom, and its
// sub-branches become segments.  Atom references that can point at either
// list are (index, inflex).
struct Ref {
    int i = -1;
    bool inflex = false;
    bool valid() const { return i >= 0; }
};

struct FlexFlattener {
    std::vector<Atom> mov, inflex;
    std::vector<double> rel;  // 3 per movable atom
    std::vector<int> fparent, fbegin, fend, fkind;
    std::vector<double> forigin_lab, faxis_lab, frel_origin;
    std::vector<std::vector<char>> mm, mi, ii;  // mobility: movable x movable, movable x inflex, inflex x inflex

    void grow() {
        const size_t m = mov.size(), n = inflex.size();
        for (auto& r : mm) r.resize(m, D_VARIABLE);
        while (mm.size() < m) mm.emplace_back(m, D_VARIABLE);
        for (auto& r : mi) r.resize(n, D_VARIABLE);
        while (mi.size() < m) mi.emplace_back(n, D_VARIABLE);
        for (auto& r : ii) r.resize(n, D_FIXED);
        while (ii.size() < n) ii.emplace_back(n, D_FIXED);
    }
    void set_mm(int a, int b, char v) { mm[std::min(a, b)][std::max(a, b)] = v; }
    void set_ii(int a, int b, char v) { ii[std::min(a, b)][std::max(a, b)] = v; }
    void add_bonds(Ref r, int b, int e) {  // add_bonds (parse_pdbqt.cpp:270-279)
        if (!r.valid()) return;
        for (int i = b; i < e; i++) {
            if (r.inflex) mi[i][r.i] = D_FIXED;
            else set_mm(r.i, i, D_FIXED);
        }
    }
    void set_rotor(Ref a, Ref b) {  // set_rotor (parse_pdbqt.cpp:281-296)
        if (!a.valid() || !b.valid()) return;
        if (b.inflex) {
            if (!a.inflex) throw std::runtime_error("flexible residue: atom-inflex rotor");
            set_ii(a.i, b.i, D_ROTOR);
        } else if (a.inflex) {
            mi[b.i][a.i] = D_ROTOR;
        } else {
            set_mm(a.i, b.i, D_ROTOR);
        }
    }
    // postprocess_branch (parse_pdbqt.cpp:306-340) with refs that may be inflex
    void branch(PS& p, Ref axis_begin, Ref axis_end, int frame) {
        const double* origin = &forigin_lab[3 * frame];
        fbegin[frame] = (int)mov.size();
        std::vector<std::vector<Ref>> begins(p.atoms.size());
        std::vector<std::vector<Ref>> ends(p.atoms.size());
        for (size_t i = 0; i < p.atoms.size(); i++) {
            PNode& nd = p.atoms[i];
            if (!(p.immobile >= 0 && (int)i == p.immobile)) {
                for (size_t c = 0; c < nd.ps.size(); c++) begins[i].push_back(Ref{(int)mov.size(), false});
                mov.push_back(nd.a);
                for (int k = 0; k < 3; k++) rel.push_back(nd.a.xyz[k] - origin[k]);
            } else {
                for (size_t c = 0; c < nd.ps.size(); c++) begins[i].push_back(immobile_ref);
            }
            for (PS& c : nd.ps) {  // insert_immobile: the child's axis atom joins this frame
                if (c.atoms.empty()) { ends[i].push_back(Ref{}); continue; }
                ends[i].push_back(Ref{(int)mov.size(), false});
                mov.push_back(c.atoms[c.immobile].a);
                for (int k = 0; k < 3; k++) rel.push_back(c.atoms[c.immobile].a.xyz[k] - origin[k]);
            }
        }
        fend[frame] = (int)mov.size();
        grow();
        add_bonds(axis_begin, fbegin[frame], fend[frame]);
        add_bonds(axis_end, fbegin[frame], fend[frame]);
        set_rotor(axis_begin, axis_end);
        for (int i = fbegin[frame]; i < fend[frame]; i++)
            for (int j = i + 1; j < fend[frame]; j++) set_mm(i, j, D_FIXED);
        for (size_t i = 0; i < p.atoms.size(); i++) {
            PNode& nd = p.atoms[i];
            for (size_t c = 0; c < nd.ps.size(); c++) {
                PS& ch = nd.ps[c];
                if (ch.essentially_empty()) continue;
                const double* o = ch.atoms[ch.immobile].a.xyz;
                const double* root = nd.a.xyz;
                double diff[3] = {o[0] - root[0], o[1] - root[1], o[2] - root[2]};
                const double nrm = std::sqrt(diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2]);
                if (nrm < 2.220446049250313e-16) throw std::runtime_error("zero-length rotatable bond");
                const int f = (int)fparent.size();
                fparent.push_back(frame);
                fkind.push_back(SG_FRAME_SEGMENT);
                fbegin.push_back(0);
                fend.push_back(0);
                for (int k = 0; k < 3; k++) {
                    forigin_lab.push_back(o[k]);
                    faxis_lab.push_back(diff[k] / nrm);
                    frel_origin.push_back(o[k] - forigin_lab[3 * frame + k]);
                }
                const Ref saved = immobile_ref;
                immobile_ref = ends[i][c];
                branch(ch, begins[i][c], ends[i][c], f);
                immobile_ref = saved;
            }
        }
    }
    Ref immobile_ref;  // where this frame's own axis atom lives (for its grandchildren's axis_begin)

    // postprocess_residue (parse_pdbqt.cpp:360-380)
    void residue(PS& p) {
        std::vector<Ref> root_ref(p.atoms.size());
        std::vector<std::vector<Ref>> imm(p.atoms.size());
        for (size_t i = 0; i < p.atoms.size(); i++) {  // insert_inflex
            root_ref[i] = Ref{(int)inflex.size(), true};
            inflex.push_back(p.atoms[i].a);
        }
        for (size_t i = 0; i < p.atoms.size(); i++)  // insert_immobiles_inflex
            for (PS& c : p.atoms[i].ps) {
                if (c.atoms.empty()) { imm[i].push_back(Ref{}); continue; }
                imm[i].push_back(Ref{(int)inflex.size(), true});
                inflex.push_back(c.atoms[c.immobile].a);
            }
        grow();
        for (size_t i = 0; i < p.atoms.size(); i++)
            for (size_t c = 0; c < p.atoms[i].ps.size(); c++) {
                PS& ch = p.atoms[i].ps[c];
                if (ch.essentially_empty()) continue;
                const double* o = ch.atoms[ch.immobile].a.xyz;
                const double* root = p.atoms[i].a.xyz;
                double diff[3] = {o[0] - root[0], o[1] - root[1], o[2] - root[2]};
                const double nrm = std::sqrt(diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2]);
                if (nrm < 2.220446049250313e-16) throw std::runtime_error("zero-length rotatable bond");
                const int f = (int)fparent.size();
                fparent.push_back(-1);
                fkind.push_back(SG_FRAME_FIRST_SEGMENT);
                fbegin.push_back(0);
                fend.push_back(0);
                for (int k = 0; k < 3; k++) {
                    forigin_lab.push_back(o[k]);
                    faxis_lab.push_back(diff[k] / nrm);
                    frel_origin.push_back(o[k]);
                }
                immobile_ref = imm[i][c];
                branch(ch, root_ref[i], imm[i][c], f);
            }
    }
};

}  // namespace

Model read_pdbqt_ligand(const std::string& text) {
    Reader rd(text);
    PS root;
    rd.ligand(root);
    Flattener F;
    F.fparent.push_back(-1);
    F.fbegin.push_back(0);
    F.fend.push_back(0);
    for (int k = 0; k < 3; k++) {
        F.forigin_lab.push_back(root.atoms[0].a.xyz[k]);
        F.faxis_lab.push_back(0);
        F.frel_origin.push_back(root.atoms[0].a.xyz[k]);
    }
    F.branch(root, 0);
    const int N = (int)F.atoms.size();
    const int nf = (int)F.fparent.size();

    // assign_bonds (model.cpp:448-529): distance-based within non-variable pairs
    auto mobility = [&](int i, int j) -> int { return i == j ? (int)D_FIXED : F.mob[std::min(i, j)][std::max(i, j)]; };
    auto d2 = [&](int i, int j) {
        double s = 0;
        for (int k = 0; k < 3; k++) { double d = F.atoms[i].xyz[k] - F.atoms[j].xyz[k]; s += d * d; }
        return s;
    };
    double max_cov = 0;
    for (int t = 0; t < NumTypes; t++) max_cov = std::max(max_cov, type_info(t).covalent_radius);
    std::vector<std::vector<int>> bonds(N);
    for (int i = 0; i < N; i++) {
        const double ci = type_info(F.atoms[i].type).covalent_radius;
        std::vector<int> relevant;
        for (int j = 0; j < N; j++) {
            if (j == i || mobility(i, j) == D_VARIABLE) continue;
            double lim = 1.1 * (ci + max_cov);
            if (d2(i, j) < lim * lim) relevant.push_back(j);
        }
        for (int j : relevant) {
            if (j <= i) continue;
            double bl = ci + type_info(F.atoms[j].type).covalent_radius;
            double r2 = d2(i, j);
            double lim = 1.1 * bl;
            if (!(r2 < lim * lim)) continue;
            bool between = false;
            for (int c : relevant) {
                if (c == i || c == j) continue;
                if (mobility(i, c) != D_VARIABLE && mobility(j, c) != D_VARIABLE && d2(i, c) < r2 && d2(j, c) < r2) {
                    between = true;
                    break;
                }
            }
            if (!between) { bonds[i].push_back(j); bonds[j].push_back(i); }
        }
    }
    for (auto& b : bonds) std::sort(b.begin(), b.end());
    // assign_types (model.cpp:555-566)
    for (int i = 0; i < N; i++) {
        bool hb = false, het = false;
        for (int j : bonds[i]) {
            if (F.atoms[j].type == PolarHydrogen) hb = true;
            if (type_info(F.atoms[j].type).ad_heteroatom) het = true;
        }
        F.atoms[i].type = adjust_type(F.atoms[i].type, hb, het);
    }
    // initialize_pairs (model.cpp:598-624) with bonded_to(i, 3) (model.cpp:576-596)
    Model m;
    std::function<void(int, int, std::vector<int>&)> bonded_to = [&](int a, int n, std::vector<int>& out) {
        if (std::find(out.begin(), out.end(), a) != out.end()) return;
        out.push_back(a);
        if (n > 0)
            for (int b : bonds[a]) bonded_to(b, n - 1, out);
    };
    for (int i = 0; i < N; i++) {
        std::vector<int> near;
        bonded_to(i, 3, near);
        for (int j = i + 1; j < N; j++) {
            if (mobility(i, j) != D_VARIABLE) continue;
            if (std::find(near.begin(), near.end(), j) != near.end()) continue;
            int t1 = F.atoms[i].type, t2 = F.atoms[j].type;
            if (t1 < NumTypes && t2 < NumTypes && !is_hydrogen(t1) && !is_hydrogen(t2)) {
                m.pairs.push_back(i);
                m.pairs.push_back(j);
            }
        }
    }
    // conf_independent_inputs (terms.cpp:83-120): counts over the ligand's
    // heavy atoms; a rotatable bond is one across a branch axis (DISTANCE_ROTOR)
    auto nbh = [&](int i) {  // num_bonded_heavy_atoms (terms.cpp:40-53)
        int c = 0;
        for (int j : bonds[i]) c += !is_hydrogen(F.atoms[j].type);
        return c;
    };
    for (int i = 0; i < N; i++) {
        const int t = F.atoms[i].type;
        if (is_hydrogen(t)) continue;
        unsigned ar = 0;  // atom_rotors (terms.cpp:55-81), rotable hydrogens fixed
        for (int j : bonds[i])
            if (mobility(i, j) == D_ROTOR && !is_hydrogen(F.atoms[j].type) && nbh(j) > 1 && nbh(i) > 1) ar++;
        m.ci[0] += 0.5 * ar;                   // num_tors
        m.ci[1] += ar > 2 ? 0.5 : 0.5 * ar;    // num_rotors
        m.ci[2] += 1;                          // num_heavy_atoms
        if (type_info(t).xs_hydrophobe) m.ci[3] += 1;
        if (type_info(t).xs_acceptor || type_info(t).xs_donor) m.ci[4] += 1;
    }
    m.ci[5] = 1;  // num_ligands
    // ligand_length: get_branch_metrics(...).corner2corner over the branch tree (model.cpp:62-109)
    std::function<std::pair<long, long>(int)> metrics = [&](int f) -> std::pair<long, long> {
        long c2c_max = 0;
        std::vector<long> lengths;
        for (int c = 0; c < nf; c++)
            if (F.fparent[c] == f) {
                auto r = metrics(c);
                c2c_max = std::max(c2c_max, r.second);
                lengths.push_back(r.first + 1);
            }
        if (lengths.empty()) return {0, 0};
        std::sort(lengths.begin(), lengths.end());
        long len = lengths.back(), c2c = len;
        if (lengths.size() >= 2) c2c += lengths[lengths.size() - 1];  // as the reference adds it
        if (c2c < c2c_max) c2c = c2c_max;
        return {len, c2c};
    };
    m.ci[6] = (double)metrics(0).second;  // ligand_lengths_sum
    m.num_other_pairs = 0;
    m.num_ligands = 1;
    m.num_flex = 0;
    m.num_movable = N;
    m.lig_pair_end = {(int)(m.pairs.size() / 2)};
    m.lig_begin = {0};
    m.lig_end = {N};
    m.lig_root = {0};
    for (int i = 0; i < N; i++) {
        m.type.push_back(F.atoms[i].type);
        m.charge.push_back(F.atoms[i].charge);
        for (int k = 0; k < 3; k++) {
            m.local.push_back(F.rel[3 * i + k]);
            m.lab.push_back(F.atoms[i].xyz[k]);
        }
    }
    int tors = 0;
    for (int f = 0; f < nf; f++) {
        m.fkind.push_back(f == 0 ? SG_FRAME_RIGID : SG_FRAME_SEGMENT);
        m.fparent.push_back(F.fparent[f]);
        m.fbegin.push_back(F.fbegin[f]);
        m.fend.push_back(F.fend[f]);
        if (f == 0) { m.fconf.push_back(0); m.fdof.push_back(0); }
        else { m.fconf.push_back(7 + tors); m.fdof.push_back(6 + tors); tors++; }
        for (int k = 0; k < 3; k++) {
            m.forigin.push_back(F.frel_origin[3 * f + k]);
            m.faxis.push_back(F.faxis_lab[3 * f + k]);
            m.finit.push_back(F.forigin_lab[3 * f + k]);
        }
    }
    m.conf_size = 7 + tors;
    m.dof = 6 + tors;
    m.torsdof = rd.torsdof;
    return m;
}

// The combined model of `smina --flex`: the receptor's flexible residues as
// one model (model::initialize over its movable and inflex atoms), with the
// ligand appended (model::append, model.cpp:302-347).  Atom order follows
// append: flexible movable atoms, ligand atoms, inflex atoms; frames and
// confs list the ligand first, then one block per ROOT branch of a residue.
// Other pairs: the residues' own pairs, then every (residue atom, ligand
// atom) pair of typed atoms in append's loop order; then the ligand's pairs.
Model read_pdbqt_flex(const std::string& ligand_text, const std::string& flex_text) {
    Model L = read_pdbqt_ligand(ligand_text);
    Reader rd(flex_text);
    FlexFlattener F;
    std::string line;
    while (std::getline(rd.in, line)) {
        if (rd.ignorable(line)) continue;
        if (starts(line, "BEGIN_RES")) {
            PS p;
            rd.residue(p);
            F.residue(p);
        } else if (starts(line, "MODEL")) {
            throw std::runtime_error("Unexpected multi-MODEL input");
        } else {
            throw std::runtime_error("Unknown or inappropriate tag: " + line);
        }
    }
    if (F.fparent.empty()) throw std::runtime_error("flexible residues: no rotatable branch");
    const int Mf = (int)F.mov.size(), If = (int)F.inflex.size(), Nf = Mf + If;
    std::vector<Atom> at(F.mov);
    at.insert(at.end(), F.inflex.begin(), F.inflex.end());
    auto mobility = [&](int i, int j) -> int {
        if (i == j) return D_FIXED;
        if (i > j) std::swap(i, j);
        if (j < Mf) return F.mm[i][j];
        if (i < Mf) return F.mi[i][j - Mf];
        return F.ii[i - Mf][j - Mf];
    };
    auto d2 = [&](int i, int j) {
        double s = 0;
        for (int k = 0; k < 3; k++) { double d = at[i].xyz[k] - at[j].xyz[k]; s += d * d; }
        return s;
    };
    // assign_bonds and assign_types over the residues' atoms (model.cpp:448-566)
    double max_cov = 0;
    for (int t = 0; t < NumTypes; t++) max_cov = std::max(max_cov, type_info(t).covalent_radius);
    std::vector<std::vector<int>> bonds(Nf);
    for (int i = 0; i < Nf; i++) {
        const double ci = type_info(at[i].type).covalent_radius;
        std::vector<int> relevant;
        for (int j = 0; j < Nf; j++) {
            if (j == i || mobility(i, j) == D_VARIABLE) continue;
            const double lim = 1.1 * (ci + max_cov);
            if (d2(i, j) < lim * lim) relevant.push_back(j);
        }
        for (int j : relevant) {
            if (j <= i) continue;
            const double lim = 1.1 * (ci + type_info(at[j].type).covalent_radius);
            const double r2 = d2(i, j);
            if (!(r2 < lim * lim)) continue;
            bool between = false;
            for (int c : relevant) {
                if (c == i || c == j) continue;
                if (mobility(i, c) != D_VARIABLE && mobility(j, c) != D_VARIABLE && d2(i, c) < r2 && d2(j, c) < r2) {
                    between = true;
                    break;
                }
            }
            if (!between) { bonds[i].push_back(j); bonds[j].push_back(i); }
        }
    }
    for (auto& b : bonds) std::sort(b.begin(), b.end());
    std::vector<int> ftype(Nf);
    for (int i = 0; i < Nf; i++) {
        bool hb = false, het = false;
        for (int j : bonds[i]) {
            if (at[j].type == PolarHydrogen) hb = true;
            if (type_info(at[j].type).ad_heteroatom) het = true;
        }
        ftype[i] = adjust_type(at[i].type, hb, het);
    }
    std::function<void(int, int, std::vector<int>&)> bonded_to = [&](int a, int n, std::vector<int>& out) {
        if (std::find(out.begin(), out.end(), a) != out.end()) return;
        out.push_back(a);
        if (n > 0)
            for (int b : bonds[a]) bonded_to(b, n - 1, out);
    };
    // initialize_pairs of the residues' model (model.cpp:598-624): all other pairs
    std::vector<int> fpairs;
    for (int i = 0; i < Nf; i++) {
        std::vector<int> near;
        bonded_to(i, 3, near);
        for (int j = i + 1; j < Nf; j++) {
            if (i >= Mf && j >= Mf) continue;  // inflex-inflex
            if (mobility(i, j) != D_VARIABLE) continue;
            if (std::find(near.begin(), near.end(), j) != near.end()) continue;
            const int t1 = ftype[i], t2 = ftype[j];
            if (t1 < NumTypes && t2 < NumTypes && !is_hydrogen(t1) && !is_hydrogen(t2)) {
                fpairs.push_back(i);
                fpairs.push_back(j);
            }
        }
    }
    // append the ligand
    const int Ml = L.num_movable;
    auto fmap = [&](int i) { return i < Mf ? i : i + Ml; };
    Model m;
    m.num_movable = Mf + Ml;
    m.num_ligands = 1;
    for (int i = 0; i < Mf; i++) {
        m.type.push_back(ftype[i]);
        m.charge.push_back(at[i].charge);
        for (int k = 0; k < 3; k++) { m.local.push_back(F.rel[3 * i + k]); m.lab.push_back(at[i].xyz[k]); }
    }
    for (int i = 0; i < Ml; i++) {
        m.type.push_back(L.type[i]);
        m.charge.push_back(L.charge[i]);
        for (int k = 0; k < 3; k++) { m.local.push_back(L.local[3 * i + k]); m.lab.push_back(L.lab[3 * i + k]); }
    }
    for (int i = Mf; i < Nf; i++) {  // inflex: lab coordinates
        m.type.push_back(ftype[i]);
        m.charge.push_back(at[i].charge);
        for (int k = 0; k < 3; k++) { m.local.push_back(at[i].xyz[k]); m.lab.push_back(at[i].xyz[k]); }
    }
    const int nlf = (int)L.fkind.size();
    for (int f = 0; f < nlf; f++) {
        m.fkind.push_back(L.fkind[f]);
        m.fparent.push_back(L.fparent[f]);
        m.fbegin.push_back(L.fbegin[f] + Mf);
        m.fend.push_back(L.fend[f] + Mf);
        m.fconf.push_back(L.fconf[f]);
        m.fdof.push_back(L.fdof[f]);
        for (int k = 0; k < 3; k++) {
            m.forigin.push_back(L.forigin[3 * f + k]);
            m.faxis.push_back(L.faxis[3 * f + k]);
            m.finit.push_back(L.finit[3 * f + k]);
        }
    }
    for (size_t f = 0; f < F.fparent.size(); f++) {
        m.fkind.push_back(F.fkind[f]);
        m.fparent.push_back(F.fparent[f] < 0 ? -1 : F.fparent[f] + nlf);
        m.fbegin.push_back(F.fbegin[f]);
        m.fend.push_back(F.fend[f]);
        m.fconf.push_back(L.conf_size + (int)f);
        m.fdof.push_back(L.dof + (int)f);
        for (int k = 0; k < 3; k++) {
            m.forigin.push_back(F.frel_origin[3 * f + k]);
            m.faxis.push_back(F.faxis_lab[3 * f + k]);
            m.finit.push_back(F.forigin_lab[3 * f + k]);
        }
        if (F.fkind[f] == SG_FRAME_FIRST_SEGMENT) m.num_flex++;
    }
    m.conf_size = L.conf_size + (int)F.fparent.size();
    m.dof = L.dof + (int)F.fparent.size();
    m.torsdof = L.torsdof;
    std::copy(L.ci, L.ci + 7, m.ci);  // conf-independent inputs count ligand atoms only
    for (size_t k = 0; k < fpairs.size(); k += 2) {
        m.pairs.push_back(fmap(fpairs[k]));
        m.pairs.push_back(fmap(fpairs[k + 1]));
    }
    for (int i = 0; i < Nf; i++)  // append's cross pairs: typed atoms, hydrogens included
        for (int j = 0; j < Ml; j++)
            if (ftype[i] < NumTypes && L.type[j] < NumTypes) {
                m.pairs.push_back(fmap(i));
                m.pairs.push_back(Mf + j);
            }
    m.num_other_pairs = (int)(m.pairs.size() / 2);
    for (size_t k = 0; k < L.pairs.size(); k++) m.pairs.push_back(L.pairs[k] + Mf);
    m.lig_pair_end = {(int)(m.pairs.size() / 2)};
    m.lig_begin = {Mf};
    m.lig_end = {Mf + Ml};
    m.lig_root = {0};
    return m;
}

sg_model_desc Model::desc() const {
    sg_model_desc d;
    d.num_atoms = (int)type.size();
    d.num_movable = num_movable;
    d.num_frames = (int)fkind.size();
    d.num_ligands = num_ligands;
    d.num_flex = num_flex;
    d.conf_size = conf_size;
    d.dof = dof;
    d.num_pairs = (int)(pairs.size() / 2);
    d.num_other_pairs = num_other_pairs;
    d.lig_pair_end = lig_pair_end.data();
    d.ligand_atom_begin = lig_begin.data();
    d.ligand_atom_end = lig_end.data();
    d.ligand_root = lig_root.data();
    d.atom_type = type.data();
    d.atom_charge = charge.data();
    d.atom_local = local.data();
    d.atom_lab = lab.data();
    d.frame_kind = fkind.data();
    d.frame_parent = fparent.data();
    d.frame_begin = fbegin.data();
    d.frame_end = fend.data();
    d.frame_conf = fconf.data();
    d.frame_dof = fdof.data();
    d.frame_origin = forigin.data();
    d.frame_axis = faxis.data();
    d.frame_init_origin = finit.data();
    d.pairs = pairs.data();
    return d;
}

int Model::num_heavy_movable() const {
    int h = 0;
    for (int i = 0; i < num_movable; i++)
        if (!is_hydrogen(type[i])) h++;
    return h;
}

}  // namespace sgh
