/*
 * SDF / MOL (V2000 and V3000) ligands.  The reference reads them through OpenBabel
 * (molgetter.cpp:103-125) and turns the molecule into smina's parse tree
 * with its own converter (SminaConverter.cpp:87-130, PDBQTUtilities.cpp:
 * 50-627): hydrogens added, non-polar hydrogens deleted with their partial
 * charges moved to their heavy atom, rigid fragments cut at rotatable
 * bonds, the root fragment the one holding the atom whose removal leaves
 * the smallest largest piece, branches depth first, AutoDock types (after
 * StripSalts, which keeps the largest connected piece).  This
 * file does the same steps without OpenBabel, writing the PDBQT text that
 * the PDBQT reader then builds the model from.  What OpenBabel perceived
 * is perceived here by these rules:
 *   - aromatic atoms: bonds typed aromatic (4) in the file, and rings of 5
 *     or 6 atoms with 6 pi electrons in their Kekule form (a ring atom gives
 *     1 for a double bond inside the ring or to an aromatic neighbour, 2 for
 *     a lone pair: 3-connected N without a double bond, 2-connected O or S;
 *     an exocyclic double bond to O, N or S gives 0; anything else stops
 *     the ring), repeated until no ring changes (fused systems);
 *   - N is an acceptor (NA) unless it is 4-connected, or 3-connected and
 *     planar (aromatic, double-bonded, or bonded to a double-bonded or
 *     aromatic atom: amides, anilines, pyrrole N); S is SA when negatively
 *     charged; every O is OA, aromatic C is A, hydrogens left are HD;
 *   - rotatable: a single bond, not amide (C(=O)-N), not in a ring, both
 *     atoms with another heavy neighbour (IsRotBond_PDBQT);
 *   - hydrogens are added only where the file has fewer than N (3), O (2)
 *     and S (2) bonds allow (formal charges counted; aromatic bonds count
 *     1.5), on N, O and S, since carbon hydrogens are deleted anyway; an
 *     added hydrogen sits 1.0 A from its atom, away from its neighbours;
 *   - partial charges: Gasteiger-Marsili PEOE (Gasteiger and Marsili,
 *     Tetrahedron 36, 3219 (1980)): 6 rounds, damping 1/2, the paper's
 *     electronegativity polynomials by element and hybridisation, starting
 *     from the formal charges.  Charges matter only to charge-dependent
 *     scoring (ad4); vina's terms do not read them.
 * Atom order: fragment by fragment in tree order, file order within one.
 */
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <functional>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#include "sg_host.h"

namespace sgh {

namespace {

struct MAtom {
    double x[3];
    std::string el;  // element symbol as in the file (first letter upper case)
    int charge = 0;  // formal charge
    bool aromatic = false;
    int hyb = 3;     // 1 sp, 2 sp2, 3 sp3
    double q = 0;    // partial charge
};
struct MBond {
    int a, b, order;  // order 1, 2, 3; 4 aromatic
};
struct Mol {
    std::string name;
    std::vector<MAtom> atoms;
    std::vector<MBond> bonds;
};

std::string field(const std::string& s, size_t a, size_t n) { return a < s.size() ? s.substr(a, n) : std::string(); }
std::string strip(const std::string& s) {
    const size_t b = s.find_first_not_of(" \t\r"), e = s.find_last_not_of(" \t\r");
    return b == std::string::npos ? std::string() : s.substr(b, e - b + 1);
}
int to_int(const std::string& s, const char* what) {
    const std::string t = strip(s);
    if (t.empty()) return 0;
    try {
        size_t k = 0;
        const int v = std::stoi(t, &k);
        if (k != t.size()) throw std::invalid_argument(t);
        return v;
    } catch (...) {
        throw std::runtime_error(std::string("SDF: bad ") + what + " field \"" + t + "\"");
    }
}
double to_double(const std::string& s, const char* what) {
    const std::string t = strip(s);
    try {
        size_t k = 0;
        const double v = std::stod(t, &k);
        if (k != t.size()) throw std::invalid_argument(t);
        return v;
    } catch (...) {
        throw std::runtime_error(std::string("SDF: bad ") + what + " field \"" + t + "\"");
    }
}

std::string element_symbol(std::string el) {
    if (el.empty() || !std::isalpha((unsigned char)el[0])) throw std::runtime_error("SDF: atom without element");
    el[0] = (char)std::toupper((unsigned char)el[0]);
    for (size_t k = 1; k < el.size(); k++) el[k] = (char)std::tolower((unsigned char)el[k]);
    if (el == "D" || el == "T") el = "H";
    return el;
}

// the connection table of a V3000 record: "M  V30" lines (a trailing "-"
// continues a line), COUNTS, the ATOM block (index, element, x, y, z,
// map, then KEY=VALUE fields of which CHG is read) and the BOND block
// (index, type, atom, atom)
Mol parse_v3000(const std::vector<std::string>& L, const std::string& name) {
    std::vector<std::string> v;
    for (size_t k = 4; k < L.size(); k++) {
        const std::string& l = L[k];
        if (l.compare(0, 6, "M  END") == 0) break;
        if (l.compare(0, 7, "M  V30 ") != 0) continue;
        std::string body = strip(l.substr(7));
        if (!v.empty() && !v.back().empty() && v.back().back() == '-') {
            v.back().pop_back();
            v.back() += body;
        } else {
            v.push_back(body);
        }
    }
    Mol m;
    m.name = name;
    int na = -1, nb = -1;
    enum { NONE, ATOMS, BONDS } block = NONE;
    std::map<int, int> index_of;  // the file's atom index -> position
    for (const std::string& line : v) {
        std::istringstream ls(line);
        std::string w;
        ls >> w;
        if (w == "COUNTS") {
            ls >> na >> nb;
            if (!ls || na <= 0 || nb < 0) throw std::runtime_error("SDF: bad V3000 COUNTS line");
        } else if (w == "BEGIN" || w == "END") {
            std::string what;
            ls >> what;
            block = w == "END" ? NONE : what == "ATOM" ? ATOMS : what == "BOND" ? BONDS : NONE;
        } else if (block == ATOMS) {
            MAtom t;
            std::string el;
            int map = 0;
            ls >> el >> t.x[0] >> t.x[1] >> t.x[2] >> map;
            if (!ls) throw std::runtime_error("SDF: bad V3000 atom line \"" + line + "\"");
            t.el = element_symbol(el);
            std::string kv;
            while (ls >> kv)
                if (kv.compare(0, 4, "CHG=") == 0) t.charge = to_int(kv.substr(4), "CHG");
            index_of[to_int(w, "atom index")] = (int)m.atoms.size();
            m.atoms.push_back(t);
        } else if (block == BONDS) {
            int type = 0, a = 0, b = 0;
            ls >> type >> a >> b;
            if (!ls || !index_of.count(a) || !index_of.count(b) || a == b)
                throw std::runtime_error("SDF: bad V3000 bond line \"" + line + "\"");
            m.bonds.push_back(MBond{index_of[a], index_of[b], (type < 1 || type > 4) ? 1 : type});
        }
    }
    if (na <= 0 || (int)m.atoms.size() != na || (int)m.bonds.size() != nb)
        throw std::runtime_error("SDF: V3000 counts do not match the atom and bond blocks");
    return m;
}

// one MOL record (ctab V2000, or V3000): header, counts, atom block, bond
// block, M CHG
Mol parse_mol(const std::string& rec) {
    std::istringstream in(rec);
    std::vector<std::string> L;
    std::string s;
    while (std::getline(in, s)) L.push_back(s);
    if (L.size() < 4) throw std::runtime_error("SDF: record shorter than its header and counts line");
    Mol m;
    m.name = strip(L[0]);
    const std::string& c = L[3];
    if (c.find("V3000") != std::string::npos) return parse_v3000(L, m.name);
    const int na = to_int(field(c, 0, 3), "atom count"), nb = to_int(field(c, 3, 3), "bond count");
    if (na <= 0 || nb < 0 || (size_t)(4 + na + nb) > L.size())
        throw std::runtime_error("SDF: counts line does not match the record");
    static const int chg_code[8] = {0, 3, 2, 1, 0, -1, -2, -3};
    for (int i = 0; i < na; i++) {
        const std::string& a = L[4 + i];
        MAtom t;
        t.x[0] = to_double(field(a, 0, 10), "x");
        t.x[1] = to_double(field(a, 10, 10), "y");
        t.x[2] = to_double(field(a, 20, 10), "z");
        t.el = element_symbol(strip(field(a, 31, 3)));
        const int cc = to_int(field(a, 36, 3), "charge");
        if (cc < 0 || cc > 7) throw std::runtime_error("SDF: bad charge code");
        t.charge = chg_code[cc];
        m.atoms.push_back(t);
    }
    for (int i = 0; i < nb; i++) {
        const std::string& b = L[4 + na + i];
        MBond t{to_int(field(b, 0, 3), "bond atom") - 1, to_int(field(b, 3, 3), "bond atom") - 1,
                to_int(field(b, 6, 3), "bond type")};
        if (t.a < 0 || t.b < 0 || t.a >= na || t.b >= na || t.a == t.b)
            throw std::runtime_error("SDF: bond to a missing atom");
        if (t.order < 1 || t.order > 4) t.order = 1;  // query bond types read as single
        m.bonds.push_back(t);
    }
    bool chg_reset = false;
    for (size_t k = 4 + na + nb; k < L.size(); k++) {
        const std::string& p = L[k];
        if (p.compare(0, 6, "M  END") == 0) break;
        if (p.compare(0, 6, "M  CHG") == 0) {
            if (!chg_reset) {  // any M CHG line supersedes the atom block's charges
                for (MAtom& a : m.atoms) a.charge = 0;
                chg_reset = true;
            }
            const int n = to_int(field(p, 6, 3), "M CHG count");
            for (int e = 0; e < n; e++) {
                const int ai = to_int(field(p, 9 + 8 * e, 4), "M CHG atom") - 1;
                const int v = to_int(field(p, 13 + 8 * e, 4), "M CHG charge");
                if (ai < 0 || ai >= na) throw std::runtime_error("SDF: M CHG names a missing atom");
                m.atoms[ai].charge = v;
            }
        }
    }
    return m;
}

struct Graph {
    std::vector<std::vector<std::pair<int, int>>> nb;  // (neighbour, bond index)
    explicit Graph(const Mol& m) : nb(m.atoms.size()) {
        for (size_t k = 0; k < m.bonds.size(); k++) {
            nb[m.bonds[k].a].push_back({m.bonds[k].b, (int)k});
            nb[m.bonds[k].b].push_back({m.bonds[k].a, (int)k});
        }
    }
};

bool is_h(const MAtom& a) { return a.el == "H"; }

// hydrogens the file leaves out on N, O and S
void add_polar_hydrogens(Mol& m) {
    const Graph g(m);
    const size_t n0 = m.atoms.size();
    for (size_t i = 0; i < n0; i++) {
        const MAtom a = m.atoms[i];
        int val;
        if (a.el == "N") val = 3 + a.charge;
        else if (a.el == "O" || a.el == "S") val = 2 + a.charge;
        else continue;
        double used = 0;
        bool high = false;
        for (auto [j, k] : g.nb[i]) {
            const int o = m.bonds[k].order;
            used += o == 4 ? 1.5 : o;
            if (a.el == "S" && o == 2 && !is_h(m.atoms[j])) high = true;  // S=X: no hydrogen added
        }
        const int nh = high ? 0 : val - (int)std::floor(used + 1e-9);
        if (nh <= 0) continue;
        double u[3] = {0, 0, 0};
        for (auto [j, k] : g.nb[i]) {
            double d[3], r = 0;
            for (int c = 0; c < 3; c++) { d[c] = m.atoms[j].x[c] - a.x[c]; r += d[c] * d[c]; }
            r = std::sqrt(r);
            if (r > 1e-6)
                for (int c = 0; c < 3; c++) u[c] -= d[c] / r;
        }
        double r = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        if (r < 1e-3) { u[0] = 1; u[1] = 0; u[2] = 0; r = 1; }
        for (double& v : u) v /= r;
        // a unit vector perpendicular to u
        double t[3] = {std::fabs(u[0]) < 0.9 ? 1.0 : 0.0, std::fabs(u[0]) < 0.9 ? 0.0 : 1.0, 0};
        double p[3] = {u[1] * t[2] - u[2] * t[1], u[2] * t[0] - u[0] * t[2], u[0] * t[1] - u[1] * t[0]};
        const double pr = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        for (double& v : p) v /= pr;
        const double q[3] = {u[1] * p[2] - u[2] * p[1], u[2] * p[0] - u[0] * p[2], u[0] * p[1] - u[1] * p[0]};
        const double tilt = nh == 1 ? 0.0 : nh == 2 ? 54.75 : 70.5;
        for (int h = 0; h < nh; h++) {
            const double phi = 2 * M_PI * h / nh, th = tilt * M_PI / 180;
            MAtom H;
            H.el = "H";
            for (int c = 0; c < 3; c++)
                H.x[c] = a.x[c] + 1.0 * (std::cos(th) * u[c] + std::sin(th) * (std::cos(phi) * p[c] + std::sin(phi) * q[c]));
            m.atoms.push_back(H);
            m.bonds.push_back(MBond{(int)i, (int)m.atoms.size() - 1, 1});
        }
    }
}

// bonds on a ring: an edge whose removal keeps its ends connected
std::vector<char> ring_bonds(const Mol& m, const Graph& g) {
    const int n = (int)m.atoms.size();
    std::vector<int> disc(n, -1), low(n, 0);
    std::vector<char> ring(m.bonds.size(), 1);
    int timer = 0;
    std::function<void(int, int)> dfs = [&](int v, int via) {
        disc[v] = low[v] = timer++;
        for (auto [w, k] : g.nb[v]) {
            if (k == via) continue;
            if (disc[w] < 0) {
                dfs(w, k);
                low[v] = std::min(low[v], low[w]);
                if (low[w] > disc[v]) ring[k] = 0;  // a bridge
            } else {
                low[v] = std::min(low[v], disc[w]);
            }
        }
    };
    for (int v = 0; v < n; v++)
        if (disc[v] < 0) dfs(v, -1);
    return ring;
}

// the smallest ring through each ring bond (atom lists, deduplicated)
std::vector<std::vector<int>> small_rings(const Mol& m, const Graph& g, const std::vector<char>& ring) {
    std::set<std::vector<int>> seen;
    std::vector<std::vector<int>> out;
    const int n = (int)m.atoms.size();
    for (size_t k = 0; k < m.bonds.size(); k++) {
        if (!ring[k]) continue;
        const int s = m.bonds[k].a, t = m.bonds[k].b;
        std::vector<int> prev(n, -2);
        std::vector<int> q{s};
        prev[s] = -1;
        for (size_t h = 0; h < q.size() && prev[t] == -2; h++) {
            const int v = q[h];
            for (auto [w, kk] : g.nb[v]) {
                if ((int)kk == (int)k || prev[w] != -2) continue;
                prev[w] = v;
                q.push_back(w);
            }
        }
        if (prev[t] == -2) continue;
        std::vector<int> cyc;
        for (int v = t; v != -1; v = prev[v]) cyc.push_back(v);
        if (cyc.size() > 7) continue;
        std::vector<int> key(cyc);
        std::sort(key.begin(), key.end());
        if (seen.insert(key).second) out.push_back(cyc);
    }
    return out;
}

void perceive_aromatic(Mol& m, const Graph& g, const std::vector<std::vector<int>>& rings) {
    for (const MBond& b : m.bonds)
        if (b.order == 4) m.atoms[b.a].aromatic = m.atoms[b.b].aromatic = true;
    auto bond_between = [&](int a, int b) {
        for (auto [w, k] : g.nb[a])
            if (w == b) return k;
        return -1;
    };
    // lone-pair donor: 3-connected N, 2-connected O or S, without a double bond
    auto donor = [&](int a) {
        const MAtom& A = m.atoms[a];
        for (auto [w, k] : g.nb[a])
            if (m.bonds[k].order == 2) return false;
        const size_t deg = g.nb[a].size();
        return (A.el == "N" && deg == 3) || ((A.el == "O" || A.el == "S") && deg == 2);
    };
    std::vector<char> done(rings.size(), 0);
    for (bool changed = true; changed;) {
        changed = false;
        for (size_t r = 0; r < rings.size(); r++) {
            const std::vector<int>& R = rings[r];
            if (done[r] || (R.size() != 5 && R.size() != 6)) continue;
            int pi = 0;
            bool ok = true;
            for (size_t i = 0; i < R.size() && ok; i++) {
                const int a = R[i];
                const int o1 = m.bonds[bond_between(a, R[(i + 1) % R.size()])].order;
                const int o2 = m.bonds[bond_between(a, R[(i + R.size() - 1) % R.size()])].order;
                if (o1 == 4 || o2 == 4) {  // typed aromatic in the file
                    pi += donor(a) ? 2 : 1;
                } else if (o1 == 2 || o2 == 2) {  // a double bond inside the ring
                    pi += 1;
                } else {
                    int exo = -1;  // an exocyclic double bond
                    for (auto [w, k] : g.nb[a])
                        if (m.bonds[k].order == 2) exo = w;
                    if (exo >= 0) {
                        const std::string& ex = m.atoms[exo].el;
                        if (m.atoms[exo].aromatic) pi += 1;  // into a fused aromatic ring
                        else if (!(ex == "O" || ex == "N" || ex == "S")) ok = false;
                    } else if (donor(a)) {
                        pi += 2;
                    } else {
                        ok = false;
                    }
                }
            }
            if (ok && pi == 6) {
                done[r] = 1;
                changed = true;
                for (int a : R) m.atoms[a].aromatic = true;
            }
        }
    }
}

void assign_hybridisation(Mol& m, const Graph& g) {
    for (size_t i = 0; i < m.atoms.size(); i++) {
        MAtom& a = m.atoms[i];
        int dbl = 0, tri = 0;
        for (auto [w, k] : g.nb[i]) {
            dbl += m.bonds[k].order == 2;
            tri += m.bonds[k].order == 3;
        }
        if (tri || dbl >= 2) a.hyb = 1;
        else if (dbl || a.aromatic) a.hyb = 2;
        else a.hyb = 3;
    }
    // 3-connected N next to a double-bonded or aromatic atom is planar (amide, aniline)
    for (size_t i = 0; i < m.atoms.size(); i++) {
        MAtom& a = m.atoms[i];
        if (a.el != "N" || a.hyb != 3) continue;
        for (auto [w, k] : g.nb[i]) {
            const MAtom& b = m.atoms[w];
            bool conj = b.aromatic;
            for (auto [x, kk] : g.nb[w]) conj = conj || m.bonds[kk].order == 2 || m.bonds[kk].order == 3;
            if (conj) { a.hyb = 2; break; }
        }
    }
}

// Gasteiger-Marsili PEOE
void gasteiger(Mol& m, const Graph& g) {
    struct P { double a, b, c; };
    auto par = [](const MAtom& t) -> P {
        const std::string& e = t.el;
        if (e == "H") return {7.17, 6.24, -0.56};
        if (e == "C") return t.hyb == 1 ? P{10.39, 9.45, 0.73} : t.hyb == 2 ? P{8.79, 9.32, 1.51} : P{7.98, 9.18, 1.88};
        if (e == "N") return t.hyb == 1 ? P{15.68, 11.70, -0.27} : t.hyb == 2 ? P{12.87, 11.15, 0.85} : P{11.54, 10.82, 1.36};
        if (e == "O") return t.hyb == 3 ? P{14.18, 12.92, 1.39} : P{17.07, 13.79, 0.47};
        if (e == "S") return {10.14, 9.13, 1.38};
        if (e == "F") return {14.66, 13.85, 2.31};
        if (e == "Cl") return {11.00, 9.69, 1.35};
        if (e == "Br") return {10.08, 8.47, 1.16};
        if (e == "I") return {9.90, 7.96, 0.96};
        if (e == "P") return {8.90, 8.24, 0.96};
        return {0, 0, 0};  // no parameters: takes no part
    };
    const int n = (int)m.atoms.size();
    std::vector<P> p(n);
    std::vector<double> q(n), chi(n);
    for (int i = 0; i < n; i++) {
        p[i] = par(m.atoms[i]);
        q[i] = m.atoms[i].charge;
    }
    double damp = 1.0;
    for (int it = 0; it < 6; it++) {
        damp *= 0.5;
        for (int i = 0; i < n; i++) chi[i] = p[i].a + q[i] * (p[i].b + q[i] * p[i].c);
        std::vector<double> dq(n, 0.0);
        for (const MBond& b : m.bonds) {
            const int i = b.a, j = b.b;
            if (p[i].a == 0 || p[j].a == 0) continue;
            // electrons move toward the more electronegative atom, scaled by the
            // cation electronegativity of the one giving them (hydrogen: 20.02)
            const int lo = chi[i] < chi[j] ? i : j, hi = lo == i ? j : i;
            const double cation = m.atoms[lo].el == "H" ? 20.02 : p[lo].a + p[lo].b + p[lo].c;
            if (cation <= 0) continue;
            const double t = (chi[hi] - chi[lo]) / cation * damp;
            dq[lo] += t;
            dq[hi] -= t;
        }
        for (int i = 0; i < n; i++) q[i] += dq[i];
    }
    for (int i = 0; i < n; i++) m.atoms[i].q = q[i];
}

}  // namespace

// byte offsets at which the records of an SDF text start (a record ends at
// a "$$$$" line; lines that are all blank do not make a record)
std::vector<size_t> sdf_starts(const std::string& text) {
    std::vector<size_t> out;
    size_t pos = 0, start = 0;
    bool any = false;
    while (pos < text.size()) {
        size_t end = text.find('\n', pos);
        if (end == std::string::npos) end = text.size();
        const std::string line = text.substr(pos, end - pos);
        if (line.compare(0, 4, "$$$$") == 0) {
            if (any) out.push_back(start);
            any = false;
            start = end + 1;
        } else if (!strip(line).empty()) {
            any = true;
        }
        pos = end + 1;
    }
    if (any) out.push_back(start);
    return out;
}

int sdf_count(const std::string& text) { return (int)sdf_starts(text).size(); }

// record `index`; scans no further than its end
static std::string sdf_record(const std::string& text, int index) {
    size_t pos = 0, start = 0;
    bool any = false;
    int k = 0;
    while (pos < text.size()) {
        size_t end = text.find('\n', pos);
        if (end == std::string::npos) end = text.size();
        if (text.compare(pos, 4, "$$$$") == 0) {
            if (any) {
                if (k == index) return text.substr(start, pos - start);
                k++;
            }
            any = false;
            start = end + 1;
        } else if (!strip(text.substr(pos, end - pos)).empty()) {
            any = true;
        }
        pos = end + 1;
    }
    if (any && k == index) return text.substr(start);
    throw std::runtime_error("SDF: no record " + std::to_string(index));
}

// The largest connected piece of the molecule (most atoms; the first of
// equal ones), as the reference's StripSalts before conversion
// (molgetter.cpp:107): counter-ions and solvent of a salt record go.
Mol largest_piece(const Mol& m) {
    const Graph g(m);
    const int n = (int)m.atoms.size();
    std::vector<int> comp(n, -1);
    std::vector<int> size;
    for (int s = 0; s < n; s++) {
        if (comp[s] >= 0) continue;
        const int c = (int)size.size();
        size.push_back(0);
        std::vector<int> st{s};
        comp[s] = c;
        while (!st.empty()) {
            const int v = st.back();
            st.pop_back();
            size[c]++;
            for (auto [w, k] : g.nb[v])
                if (comp[w] < 0) {
                    comp[w] = c;
                    st.push_back(w);
                }
        }
    }
    if (size.size() <= 1) return m;
    const int keep = (int)(std::max_element(size.begin(), size.end()) - size.begin());
    Mol out;
    out.name = m.name;
    std::vector<int> at(n, -1);
    for (int i = 0; i < n; i++)
        if (comp[i] == keep) {
            at[i] = (int)out.atoms.size();
            out.atoms.push_back(m.atoms[i]);
        }
    for (const MBond& b : m.bonds)
        if (at[b.a] >= 0 && at[b.b] >= 0) out.bonds.push_back(MBond{at[b.a], at[b.b], b.order});
    return out;
}

std::string pdbqt_from_sdf(const std::string& text, int index, bool add_hydrogens) {
    Mol m = largest_piece(parse_mol(sdf_record(text, index)));
    if (add_hydrogens) add_polar_hydrogens(m);
    {
        const Graph g(m);
        const std::vector<char> ring = ring_bonds(m, g);
        perceive_aromatic(m, g, small_rings(m, g, ring));
        assign_hybridisation(m, g);
        gasteiger(m, g);
    }
    // delete non-polar hydrogens (bonded to anything but N, O, S, P), their
    // charge moved to the heavy atom (DeleteHydrogens, PDBQTUtilities.cpp:285-300)
    const Graph g0(m);
    const int n0 = (int)m.atoms.size();
    std::vector<int> keep_idx(n0, -1);
    std::vector<char> drop(n0, 0);
    for (int i = 0; i < n0; i++) {
        if (!is_h(m.atoms[i])) continue;
        int heavy = -1;
        for (auto [w, k] : g0.nb[i])
            if (!is_h(m.atoms[w])) heavy = w;
        const std::string e = heavy >= 0 ? m.atoms[heavy].el : std::string();
        if (!(e == "N" || e == "O" || e == "S" || e == "P")) {
            drop[i] = 1;
            if (heavy >= 0) m.atoms[heavy].q += m.atoms[i].q;
        }
    }
    Mol h;
    h.name = m.name;
    for (int i = 0; i < n0; i++)
        if (!drop[i]) {
            keep_idx[i] = (int)h.atoms.size();
            h.atoms.push_back(m.atoms[i]);
        }
    for (const MBond& b : m.bonds)
        if (keep_idx[b.a] >= 0 && keep_idx[b.b] >= 0) h.bonds.push_back(MBond{keep_idx[b.a], keep_idx[b.b], b.order});
    const int n = (int)h.atoms.size();
    if (n == 0) throw std::runtime_error("SDF: no atoms left");
    const Graph g(h);
    std::vector<int> heavy_deg(n, 0);
    for (int i = 0; i < n; i++)
        for (auto [w, k] : g.nb[i]) heavy_deg[i] += !is_h(h.atoms[w]);
    // connected pieces of the graph without `cut_atom` and the bonds in `cut`
    auto pieces = [&](int cut_atom, const std::vector<char>& cut) {
        std::vector<int> comp(n, -1);
        std::vector<std::vector<int>> out;
        for (int s = 0; s < n; s++) {
            if (s == cut_atom || comp[s] >= 0) continue;
            std::vector<int> st{s}, members;
            comp[s] = (int)out.size();
            while (!st.empty()) {
                const int v = st.back();
                st.pop_back();
                members.push_back(v);
                for (auto [w, k] : g.nb[v])
                    if (w != cut_atom && comp[w] < 0 && !cut[k]) {
                        comp[w] = comp[s];
                        st.push_back(w);
                    }
            }
            std::sort(members.begin(), members.end());
            out.push_back(members);
        }
        return out;
    };
    const std::vector<char> none(h.bonds.size(), 0);
    if (pieces(-1, none).size() != 1) throw std::runtime_error("SDF: the molecule is not connected");
    // best root atom: its removal leaves the smallest largest piece (first such atom)
    int best_root = 0;
    size_t best = (size_t)n + 1;
    for (int i = 0; i < n; i++) {
        size_t big = 0;
        for (auto& p : pieces(i, none)) big = std::max(big, p.size());
        if (big < best) { best = big; best_root = i; }
    }
    // rotatable bonds (IsRotBond_PDBQT, PDBQTUtilities.cpp:145-170)
    const std::vector<char> ring = ring_bonds(h, g);
    auto carbonyl_c = [&](int c) {
        if (h.atoms[c].el != "C") return false;
        for (auto [w, k] : g.nb[c])
            if (h.atoms[w].el == "O" && h.bonds[k].order == 2) return true;
        return false;
    };
    std::vector<char> rot(h.bonds.size(), 0);
    int nrot = 0;
    for (size_t k = 0; k < h.bonds.size(); k++) {
        const MBond& b = h.bonds[k];
        if (b.order != 1 || ring[k]) continue;
        const bool amide = (h.atoms[b.a].el == "N" && carbonyl_c(b.b)) || (h.atoms[b.b].el == "N" && carbonyl_c(b.a));
        if (amide || heavy_deg[b.a] <= 1 || heavy_deg[b.b] <= 1) continue;
        rot[k] = 1;
        nrot++;
    }
    std::vector<std::vector<int>> frags = pieces(-1, rot);
    std::vector<int> frag_of(n);
    for (size_t f = 0; f < frags.size(); f++)
        for (int a : frags[f]) frag_of[a] = (int)f;
    // tree: depth first from the root fragment; a fragment's children in
    // fragment order, each through the first bond found (ConstructTree)
    struct Node { int frag, parent_atom, child_atom; std::vector<int> kids; };
    std::vector<Node> tree{{frag_of[best_root], -1, -1, {}}};
    std::vector<char> used(frags.size(), 0);
    used[frag_of[best_root]] = 1;
    std::function<void(int)> grow = [&](int t) {
        for (bool more = true; more;) {
            more = false;
            for (size_t f = 0; f < frags.size() && !more; f++) {
                if (used[f]) continue;
                for (int a : frags[tree[t].frag]) {
                    for (auto [w, k] : g.nb[a])
                        if (frag_of[w] == (int)f) {
                            used[f] = 1;
                            tree.push_back(Node{(int)f, a, w, {}});
                            const int c = (int)tree.size() - 1;
                            tree[t].kids.push_back(c);
                            grow(c);
                            more = true;
                            break;
                        }
                    if (more) break;
                }
            }
        }
    };
    grow(0);
    // serial numbers in output order
    std::vector<int> serial(n, 0);
    int next = 1;
    std::function<void(int)> number = [&](int t) {
        for (int a : frags[tree[t].frag]) serial[a] = next++;
        for (int c : tree[t].kids) number(c);
    };
    number(0);
    auto ad_type = [&](int i) -> std::string {
        const MAtom& a = h.atoms[i];
        if (a.el == "H") return "HD";
        if (a.el == "C") return a.aromatic ? "A" : "C";
        if (a.el == "O") return "OA";
        if (a.el == "N") {
            const size_t deg = g.nb[i].size();
            if (deg >= 4 || (deg == 3 && a.hyb <= 2)) return "N";
            return "NA";
        }
        if (a.el == "S") return a.charge < 0 ? "SA" : "S";
        return a.el;
    };
    std::string out;
    char buf[160];
    if (!h.name.empty()) out += "REMARK  Name = " + h.name + "\n";
    std::snprintf(buf, sizeof buf, "REMARK  %d active torsions\n", nrot);
    out += buf;
    auto atom_line = [&](int i) {
        const std::string t = ad_type(i);
        std::string name = h.atoms[i].el + std::to_string(serial[i]);
        if (name.size() > 4) name = name.substr(0, 4);
        std::snprintf(buf, sizeof buf, "ATOM  %5d %-4s UNL A   1    %8.3f%8.3f%8.3f  0.00  0.00    %+6.3f %-2s\n",
                      serial[i] % 100000, name.c_str(), h.atoms[i].x[0], h.atoms[i].x[1], h.atoms[i].x[2],
                      h.atoms[i].q, t.c_str());
        out += buf;
    };
    out += "ROOT\n";
    for (int a : frags[tree[0].frag]) atom_line(a);
    out += "ENDROOT\n";
    std::function<void(int)> emit = [&](int t) {
        for (int c : tree[t].kids) {
            std::snprintf(buf, sizeof buf, "BRANCH %3d %3d\n", serial[tree[c].parent_atom], serial[tree[c].child_atom]);
            out += buf;
            for (int a : frags[tree[c].frag]) atom_line(a);
            emit(c);
            std::snprintf(buf, sizeof buf, "ENDBRANCH %3d %3d\n", serial[tree[c].parent_atom], serial[tree[c].child_atom]);
            out += buf;
        }
    };
    emit(0);
    std::snprintf(buf, sizeof buf, "TORSDOF %d\n", nrot);
    out += buf;
    return out;
}

}  // namespace sgh
