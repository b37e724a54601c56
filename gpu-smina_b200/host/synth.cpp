/*
 * Synthetic receptors and ligands with the shapes the benchmark configs ask
 * for (no public dataset is available offline):
 *   receptor R(n): seeded random-walk chains of 1.5 A bonds, element mix
 *     C 63 / N 17 / O 19 / S 1 %, >= 3.0 A between non-bonded atoms, an
 *     8 A cavity carved at the box centre, polar H on N/O donors;
 *   ligand L(h, r): acyclic drug-like tree of h heavy atoms with standard
 *     bond lengths and tetrahedral angles, polar H on heteroatoms, exactly r
 *     rotatable bonds, written as a PDBQT torsion tree.
 * A private splitmix64 stream keeps every draw identical on every compiler.
 */
#include "sg_host.h"
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <functional>
#include <map>
#include <stdexcept>
#include <unordered_map>

namespace sgh {

namespace {

struct Rng {  // splitmix64 (Steele, Lea, Flood 2014)
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed * 0x9E3779B97F4A7C15ull + 0x1234567ull) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uni() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    int below(int n) { return (int)(uni() * n); }
};

struct P3 {
    double x, y, z;
};
P3 operator+(P3 a, P3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
P3 operator-(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
P3 operator*(double s, P3 a) { return {s * a.x, s * a.y, s * a.z}; }
double dotp(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
P3 crossp(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double len(P3 a) { return std::sqrt(dotp(a, a)); }
P3 unit(P3 a) { return (1.0 / len(a)) * a; }
P3 rand_unit(Rng& r) {
    for (;;) {
        P3 p{2 * r.uni() - 1, 2 * r.uni() - 1, 2 * r.uni() - 1};
        double l = len(p);
        if (l > 1e-3 && l <= 1) return (1.0 / l) * p;
    }
}
// a direction making `angle` with `back` (unit), rotated by `dihedral` around it
P3 cone_dir(P3 back, double angle, double dihedral, Rng& r) {
    P3 t = rand_unit(r);
    P3 u = crossp(back, t);
    while (len(u) < 1e-3) { t = rand_unit(r); u = crossp(back, t); }
    u = unit(u);
    P3 w = crossp(back, u);
    return std::cos(angle) * back + std::sin(angle) * (std::cos(dihedral) * u + std::sin(dihedral) * w);
}

struct Hash {  // 3 A spatial hash of placed atoms
    double cell = 3.0;
    std::unordered_map<int64_t, std::vector<int>> m;
    int64_t key(int i, int j, int k) const { return ((int64_t)(i + 4096) << 26) | ((int64_t)(j + 4096) << 13) | (k + 4096); }
    void add(const P3& p, int idx) {
        m[key((int)std::floor(p.x / cell), (int)std::floor(p.y / cell), (int)std::floor(p.z / cell))].push_back(idx);
    }
    template <typename F>
    void near(const P3& p, F f) const {
        int ci = (int)std::floor(p.x / cell), cj = (int)std::floor(p.y / cell), ck = (int)std::floor(p.z / cell);
        for (int a = -1; a <= 1; a++)
            for (int b = -1; b <= 1; b++)
                for (int c = -1; c <= 1; c++) {
                    auto it = m.find(key(ci + a, cj + b, ck + c));
                    if (it != m.end())
                        for (int i : it->second) f(i);
                }
    }
};

void pdbqt_line(std::string& out, int serial, const char* name, const char* res, const P3& p, double q, const char* ad) {
    char buf[128];
    std::snprintf(buf, sizeof buf, "ATOM  %5d %-4s %3s A   1    %8.3f%8.3f%8.3f  1.00  0.00    %+6.3f %-2s\n", serial % 100000,
                  name, res, p.x, p.y, p.z, q, ad);
    out += buf;
}

}  // namespace

// ---- receptor -------------------------------------------------------------------
Receptor make_receptor(int heavy_atoms, uint64_t seed, const double center[3], double cavity_radius) {
    Rng r(seed);
    const P3 c{center[0], center[1], center[2]};
    const double density = 0.033;  // heavy atoms per A^3 reachable with 3 A spacing
    const double r_in = cavity_radius;
    const double r_out = std::cbrt(r_in * r_in * r_in + heavy_atoms / (density * 4.0 / 3.0 * M_PI));
    std::vector<P3> pos;
    std::vector<std::vector<int>> nb;
    Hash h;
    auto in_shell = [&](const P3& p) { double d = len(p - c); return d >= r_in && d <= r_out; };
    auto clear_of = [&](const P3& p, int ex1, int ex2) {
        bool ok = true;
        h.near(p, [&](int i) {
            if (i == ex1 || i == ex2) return;
            P3 d = pos[i] - p;
            if (dotp(d, d) < 9.0) ok = false;
        });
        return ok;
    };
    int stall = 0;
    while ((int)pos.size() < heavy_atoms && stall < 200000) {
        P3 s{c.x + (2 * r.uni() - 1) * r_out, c.y + (2 * r.uni() - 1) * r_out, c.z + (2 * r.uni() - 1) * r_out};
        if (!in_shell(s) || !clear_of(s, -1, -1)) { stall++; continue; }
        int prev = (int)pos.size(), pprev = -1;
        pos.push_back(s);
        nb.emplace_back();
        h.add(s, prev);
        int chain = 10 + r.below(40);
        for (int k = 1; k < chain && (int)pos.size() < heavy_atoms; k++) {
            bool placed = false;
            for (int t = 0; t < 30 && !placed; t++) {
                P3 d = pprev < 0 ? rand_unit(r)
                                 : cone_dir(unit(pos[prev] - pos[pprev]), M_PI - 109.5 * M_PI / 180, 2 * M_PI * r.uni(), r);
                P3 q = pos[prev] + 1.5 * d;
                if (!in_shell(q) || !clear_of(q, prev, pprev)) continue;
                int idx = (int)pos.size();
                pos.push_back(q);
                nb.emplace_back();
                nb[idx].push_back(prev);
                nb[prev].push_back(idx);
                h.add(q, idx);
                pprev = prev;
                prev = idx;
                placed = true;
            }
            if (!placed) break;
        }
    }
    const int n = (int)pos.size();
    std::vector<int> el(n);  // 0 C, 1 N, 2 O, 3 S
    for (int i = 0; i < n; i++) {
        double u = r.uni();
        el[i] = u < 0.63 ? 0 : u < 0.80 ? 1 : u < 0.99 ? 2 : 3;
    }
    Receptor rec;
    std::vector<int> polarH(n, 0);
    std::vector<P3> hpos(n);
    for (int i = 0; i < n; i++) {
        if (el[i] != 1 && el[i] != 2) continue;
        int maxdeg = el[i] == 1 ? 3 : 2;
        if ((int)nb[i].size() >= maxdeg) continue;
        if (r.uni() > (el[i] == 1 ? 0.6 : 0.5)) continue;
        P3 away{0, 0, 0};
        for (int j : nb[i]) away = away + unit(pos[i] - pos[j]);
        P3 dir = len(away) > 1e-3 ? unit(unit(away) + 0.3 * rand_unit(r)) : rand_unit(r);
        P3 hp = pos[i] + 1.0 * dir;
        bool ok = true;
        h.near(hp, [&](int k) {
            if (k == i) return;
            P3 d = pos[k] - hp;
            if (dotp(d, d) < 4.0) ok = false;
        });
        if (ok) { polarH[i] = 1; hpos[i] = hp; }
    }
    for (int i = 0; i < n; i++) {
        Atom a;
        a.xyz[0] = pos[i].x; a.xyz[1] = pos[i].y; a.xyz[2] = pos[i].z;
        bool het = false;
        for (int j : nb[i]) het |= el[j] != 0;
        if (el[i] == 0) { a.type = het ? AliphaticCarbonXSNonHydrophobe : AliphaticCarbonXSHydrophobe; a.name = "C"; }
        else if (el[i] == 1) {
            bool acc = r.uni() < 0.5;
            a.type = acc ? (polarH[i] ? NitrogenXSDonorAcceptor : NitrogenXSAcceptor) : (polarH[i] ? NitrogenXSDonor : Nitrogen);
            a.name = "N";
        } else if (el[i] == 2) { a.type = polarH[i] ? OxygenXSDonorAcceptor : OxygenXSAcceptor; a.name = "O"; }
        else { a.type = SulfurAcceptor; a.name = "S"; }
        a.resname = "REC";
        rec.atoms.push_back(a);
        if (polarH[i]) {
            Atom hh;
            hh.type = PolarHydrogen;
            hh.name = "H";
            hh.resname = "REC";
            hh.xyz[0] = hpos[i].x; hh.xyz[1] = hpos[i].y; hh.xyz[2] = hpos[i].z;
            rec.atoms.push_back(hh);
        }
    }
    for (size_t i = 0; i < rec.atoms.size(); i++) rec.atoms[i].number = (int)i + 1;
    return rec;
}

sg_receptor_desc Receptor::desc(std::vector<double>& xyz, std::vector<int>& t, std::vector<double>& q) const {
    xyz.clear(); t.clear(); q.clear();
    for (const Atom& a : atoms) {
        xyz.insert(xyz.end(), a.xyz, a.xyz + 3);
        t.push_back(a.type);
        q.push_back(a.charge);
    }
    sg_receptor_desc d;
    d.num_atoms = (int)atoms.size();
    d.coords = xyz.data();
    d.type = t.data();
    d.charge = q.data();
    return d;
}

std::string receptor_pdbqt(const Receptor& rec) {
    std::string out = "REMARK  synthetic receptor\n";
    for (const Atom& a : rec.atoms)
        pdbqt_line(out, a.number, a.name.c_str(), "REC", P3{a.xyz[0], a.xyz[1], a.xyz[2]}, a.charge, type_info(a.type).ad);
    return out;
}

// ---- ligand ------------------------------------------------------------------------
std::string make_ligand_pdbqt(int heavy, int rotors, uint64_t seed, const double center[3]) {
    if (heavy < 1) throw std::runtime_error("a ligand needs at least one heavy atom");
    // an acyclic tree of h heavy atoms has at most h - 3 bonds between two
    // non-terminal atoms
    rotors = std::max(0, std::min(rotors, heavy - 3));
    const P3 c{center[0], center[1], center[2]};
    for (int attempt = 0; attempt < 2000; attempt++) {
        Rng r(seed * 1000003ull + attempt);
        // elements: 0 C, 1 N, 2 O, 3 S, 4 F, 5 Cl, 6 Br
        static const int valence[] = {4, 3, 2, 2, 1, 1, 1};
        static const double cov[] = {0.77, 0.75, 0.73, 1.02, 0.71, 0.99, 1.14};
        std::vector<int> el, parent;
        std::vector<P3> pos;
        std::vector<std::vector<int>> nb;
        el.push_back(0); parent.push_back(-1); pos.push_back(c); nb.emplace_back();
        bool failed = false;
        for (int k = 1; k < heavy && !failed; k++) {
            double u = r.uni();
            int e = u < 0.70 ? 0 : u < 0.82 ? 1 : u < 0.95 ? 2 : u < 0.97 ? 3 : u < 0.98 ? 4 : u < 0.995 ? 5 : 6;
            bool placed = false;
            // grow chains (attach to the newest atom) more often when many
            // rotatable bonds are wanted
            const double linear = std::min(0.9, (double)rotors / std::max(1, heavy - 3) + attempt * 0.002);
            for (int t = 0; t < 60 && !placed; t++) {
                int p = (t < 20 && r.uni() < linear) ? (int)pos.size() - 1 : r.below((int)pos.size());
                if ((int)nb[p].size() >= valence[el[p]] - (el[p] == 0 ? 0 : 0)) continue;
                if (el[p] >= 4) continue;
                double bl = el[p] == 0 && e == 0 ? 1.54 : cov[el[p]] + cov[e];
                P3 d;
                if (nb[p].empty()) d = rand_unit(r);
                else {
                    P3 back = unit(pos[nb[p][0]] - pos[p]);
                    d = cone_dir(back, 109.5 * M_PI / 180, 2 * M_PI * r.uni(), r);
                }
                P3 q = pos[p] + bl * d;
                bool ok = true;
                for (size_t i = 0; i < pos.size() && ok; i++) {
                    if ((int)i == p) continue;
                    bool one_three = std::find(nb[p].begin(), nb[p].end(), (int)i) != nb[p].end();
                    double lim = one_three ? 2.2 : 2.9;
                    P3 dd = pos[i] - q;
                    if (dotp(dd, dd) < lim * lim) ok = false;
                }
                if (!ok) continue;
                int idx = (int)pos.size();
                el.push_back(e); parent.push_back(p); pos.push_back(q); nb.emplace_back();
                nb[idx].push_back(p); nb[p].push_back(idx);
                placed = true;
            }
            if (!placed) failed = true;
        }
        if (failed) continue;
        const int n = (int)pos.size();
        // eligible torsions: bonds between two atoms with >= 2 heavy neighbours
        std::vector<int> eligible;  // child index (bond child-parent)
        for (int i = 1; i < n; i++)
            if (nb[i].size() >= 2 && nb[parent[i]].size() >= 2) eligible.push_back(i);
        if ((int)eligible.size() < rotors) continue;
        for (int i = (int)eligible.size() - 1; i > 0; i--) std::swap(eligible[i], eligible[r.below(i + 1)]);
        std::vector<char> rot(n, 0);
        for (int k = 0; k < rotors; k++) rot[eligible[k]] = 1;
        // polar hydrogens on heteroatoms with free valence (one per atom)
        std::vector<int> hn(n, -1);
        std::vector<P3> hp;
        for (int i = 0; i < n; i++) {
            if (el[i] != 1 && el[i] != 2) continue;
            if ((int)nb[i].size() >= valence[el[i]]) continue;
            if (el[i] == 1 && r.uni() < 0.4) continue;
            P3 away{0, 0, 0};
            for (int j : nb[i]) away = away + unit(pos[i] - pos[j]);
            P3 dir = len(away) > 1e-3 ? unit(away) : rand_unit(r);
            P3 q = pos[i] + 1.0 * dir;
            bool ok = true;
            for (int j = 0; j < n && ok; j++)
                if (j != i) { P3 dd = pos[j] - q; if (dotp(dd, dd) < 2.0 * 2.0) ok = false; }
            for (const P3& o : hp) { P3 dd = o - q; if (dotp(dd, dd) < 2.0 * 2.0) ok = false; }
            if (!ok) continue;
            hn[i] = (int)hp.size();
            hp.push_back(q);
        }
        // fragments split at rotatable bonds
        std::vector<int> frag(n, -1);
        int nfrag = 0;
        for (int s = 0; s < n; s++) {
            if (frag[s] >= 0) continue;
            std::vector<int> st{s};
            frag[s] = nfrag;
            while (!st.empty()) {
                int a = st.back(); st.pop_back();
                for (int b : nb[a]) {
                    bool rb = (parent[b] == a && rot[b]) || (parent[a] == b && rot[a]);
                    if (!rb && frag[b] < 0) { frag[b] = nfrag; st.push_back(b); }
                }
            }
            nfrag++;
        }
        std::vector<int> fsize(nfrag, 0);
        for (int i = 0; i < n; i++) fsize[frag[i]]++;
        int rootf = (int)(std::max_element(fsize.begin(), fsize.end()) - fsize.begin());
        // serial numbers and PDBQT text, depth-first from the root fragment
        std::vector<int> serial(n, 0), hserial(hp.size(), 0);
        int next_serial = 1;
        std::string out = "REMARK  synthetic ligand\n";
        auto elname = [&](int i) -> const char* {
            static const char* nm[] = {"C", "N", "O", "S", "F", "Cl", "Br"};
            return nm[el[i]];
        };
        auto adname = [&](int i) -> const char* {
            switch (el[i]) {
                case 0: return "C";
                case 1: return (i % 2) ? "NA" : "N";
                case 2: return "OA";
                case 3: return "SA";
                case 4: return "F";
                case 5: return "Cl";
                default: return "Br";
            }
        };
        auto emit_atom = [&](int i) {
            serial[i] = next_serial++;
            pdbqt_line(out, serial[i], elname(i), "LIG", pos[i], 0.0, adname(i));
            if (hn[i] >= 0) {
                hserial[hn[i]] = next_serial++;
                pdbqt_line(out, hserial[hn[i]], "H", "LIG", hp[hn[i]], 0.0, "HD");
            }
        };
        std::function<void(int, int)> emit_frag = [&](int f, int first) {
            if (first >= 0) emit_atom(first);
            for (int i = 0; i < n; i++)
                if (frag[i] == f && i != first) emit_atom(i);
            for (int i = 0; i < n; i++) {
                if (frag[i] != f) continue;
                for (int b : nb[i]) {
                    if (frag[b] == f) continue;
                    bool rb = (parent[b] == i && rot[b]) || (parent[i] == b && rot[i]);
                    if (!rb || serial[b] != 0) continue;
                    // BRANCH parent_serial child_serial; child serial is assigned inside
                    size_t mark = out.size();
                    out += "BRANCH PLACEHOLDER\n";
                    emit_frag(frag[b], b);
                    char buf[64];
                    std::snprintf(buf, sizeof buf, "BRANCH %3d %3d\n", serial[i], serial[b]);
                    out.replace(mark, std::string("BRANCH PLACEHOLDER\n").size(), buf);
                    std::snprintf(buf, sizeof buf, "ENDBRANCH %3d %3d\n", serial[i], serial[b]);
                    out += buf;
                }
            }
        };
        out += "ROOT\n";
        size_t root_end_mark = 0;
        {
            for (int i = 0; i < n; i++)
                if (frag[i] == rootf) emit_atom(i);
            out += "ENDROOT\n";
            root_end_mark = out.size();
            (void)root_end_mark;
            for (int i = 0; i < n; i++) {
                if (frag[i] != rootf) continue;
                for (int b : nb[i]) {
                    if (frag[b] == rootf || serial[b] != 0) continue;
                    size_t mark = out.size();
                    out += "BRANCH PLACEHOLDER\n";
                    emit_frag(frag[b], b);
                    char buf[64];
                    std::snprintf(buf, sizeof buf, "BRANCH %3d %3d\n", serial[i], serial[b]);
                    out.replace(mark, std::string("BRANCH PLACEHOLDER\n").size(), buf);
                    std::snprintf(buf, sizeof buf, "ENDBRANCH %3d %3d\n", serial[i], serial[b]);
                    out += buf;
                }
            }
        }
        char buf[32];
        std::snprintf(buf, sizeof buf, "TORSDOF %d\n", rotors);
        out += buf;
        return out;
    }
    throw std::runtime_error("could not place a ligand with the requested rotors");
}

// ---- flexible residues ---------------------------------------------------------------
std::string make_flex_pdbqt(int residues, uint64_t seed, const double center[3], double shell) {
    if (residues < 1 || residues > 32) throw std::runtime_error("flexible residues: 1..32");
    Rng r(seed * 7919ull + 17);
    const P3 c{center[0], center[1], center[2]};
    std::string out;
    std::vector<P3> placed;  // every side-chain atom so far, for spacing
    int serial = 1;
    auto line = [&](int n, const char* name, const char* res, int resnum, const P3& p, double q, const char* ad) {
        char buf[128];
        std::snprintf(buf, sizeof buf, "ATOM  %5d  %-3s %3s A%4d    %8.3f%8.3f%8.3f  1.00  0.00    %+6.3f %-2s\n", n,
                      name, res, resnum, p.x, p.y, p.z, q, ad);
        out += buf;
    };
    static const char* names[] = {"CB", "CG", "CD", "CE", "CZ"};
    for (int k = 0; k < residues; k++) {
        const int chis = 2 + (int)r.below(3);  // 2..4
        // the residue's CA on the shell, directions spread over the sphere
        P3 dir{0, 0, 0};
        for (int t = 0; t < 200; t++) {
            P3 d = rand_unit(r);
            bool ok = true;
            for (const P3& q : placed) {
                P3 e = (c + shell * d) - q;
                if (dotp(e, e) < 5.0 * 5.0) { ok = false; break; }
            }
            dir = d;
            if (ok) break;
        }
        std::vector<P3> pos{c + shell * dir};
        P3 back = unit(pos[0] - c);  // points away from the centre
        pos.push_back(pos[0] + 1.53 * (-1.0 * back));
        for (int a = 2; a < chis + 2; a++) {  // X2 .. X(chis+1), growing into the cavity
            P3 best{0, 0, 0};
            double best_d = 1e30;
            const P3 b = unit(pos[a - 2] - pos[a - 1]);
            for (int t = 0; t < 24; t++) {
                P3 q = pos[a - 1] + 1.53 * cone_dir(b, 109.5 * M_PI / 180, 2 * M_PI * r.uni(), r);
                bool ok = true;
                for (int i = 0; i + 2 < a && ok; i++) {
                    P3 e = pos[i] - q;
                    if (dotp(e, e) < 2.4 * 2.4) ok = false;
                }
                for (const P3& o : placed) {
                    P3 e = o - q;
                    if (dotp(e, e) < 3.2 * 3.2) { ok = false; break; }
                }
                P3 e = q - c;
                const double dc = dotp(e, e) + (ok ? 0 : 1e6);
                if (dc < best_d) { best_d = dc; best = q; }
            }
            pos.push_back(best);
        }
        const bool amine = r.uni() < 0.5;  // terminal N-H or O-H
        const P3 hdir = unit(pos.back() - pos[pos.size() - 2]);
        const P3 h = pos.back() + 1.0 * hdir;
        const int resnum = 10 + 7 * k;
        const char* res = amine ? "LYS" : "SER";
        char head[64];
        std::snprintf(head, sizeof head, "BEGIN_RES %s A%4d\n", res, resnum);
        out += head;
        out += "ROOT\n";
        const int ca = serial++;
        line(ca, "CA", res, resnum, pos[0], 0.0, "C");
        out += "ENDROOT\n";
        std::vector<int> sn(pos.size());
        sn[0] = ca;
        for (size_t a = 1; a < pos.size(); a++) sn[a] = serial++;
        const int hs = serial++;
        const int last = (int)pos.size() - 1;  // X(chis+1)
        for (int b = 1; b <= chis; b++) {  // BRANCH X(b-1) X(b)
            char br[64];
            std::snprintf(br, sizeof br, "BRANCH %3d %3d\n", sn[b - 1], sn[b]);
            out += br;
            const bool tip = b == last - 1;
            line(sn[b], names[b - 1], res, resnum, pos[b], 0.0, "C");
            if (tip) {
                line(sn[last], amine ? "NZ" : "OG", res, resnum, pos[last], amine ? -0.3 : -0.4, amine ? "N" : "OA");
                line(hs, amine ? "HZ" : "HG", res, resnum, h, 0.2, "HD");
            }
        }
        for (int b = chis; b >= 1; b--) {
            char br[64];
            std::snprintf(br, sizeof br, "ENDBRANCH %3d %3d\n", sn[b - 1], sn[b]);
            out += br;
        }
        std::snprintf(head, sizeof head, "END_RES %s A%4d\n", res, resnum);
        out += head;
        for (const P3& q : pos) placed.push_back(q);
    }
    return out;
}

sg_grid_dims make_box(const double center[3], const double size[3], double granularity) {
    sg_grid_dims gd;
    for (int i = 0; i < 3; i++) {
        gd.n[i] = (int)(size_t)std::ceil(size[i] / granularity);
        double real_span = granularity * gd.n[i];
        gd.begin[i] = center[i] - real_span / 2;
        gd.end[i] = gd.begin[i] + real_span;
    }
    return gd;
}

}  // namespace sgh
