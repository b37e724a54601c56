/*
 * ORACLE (test infrastructure only): CPU FP64 restatement of smina's docking
 * search, used as the checker for the CUDA path and as the timed CPU
 * baseline.  Nothing in the product includes, links or executes it.
 *
 * Every function names the reference file:line it follows (paths inside the
 * reference project).  Arithmetic keeps the reference's operand order and is
 * compiled with -ffp-contract=off so results are deterministic.
 */
#ifndef OR_CORE_H
#define OR_CORE_H

#include <cstdint>
#include <vector>
#include <map>
#include <array>
#include <limits>
#include "or_math.h"
#include "../include/smina_b200.h"

namespace orc {

const double PI = 3.1415926535897931;            // common.h:227
const double EPS = std::numeric_limits<double>::epsilon();
const double MAXF = std::numeric_limits<double>::max();

// ---- vec / mat / quaternion in the operand order of common.h ----------
struct V3 {
    double d[3];
    V3() : d{0, 0, 0} {}
    V3(double x, double y, double z) : d{x, y, z} {}
    double& operator[](int i) { return d[i]; }
    double operator[](int i) const { return d[i]; }
};
inline V3 operator+(const V3& a, const V3& b) { return V3(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
inline V3 operator-(const V3& a, const V3& b) { return V3(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
inline V3 operator*(double s, const V3& v) { return V3(s * v[0], s * v[1], s * v[2]); }
inline void addto(V3& a, const V3& b) { a[0] += b[0]; a[1] += b[1]; a[2] += b[2]; }
inline void subfrom(V3& a, const V3& b) { a[0] -= b[0]; a[1] -= b[1]; a[2] -= b[2]; }
inline double sqr(double x) { return x * x; }
inline double sqrv(const V3& v) { return sqr(v[0]) + sqr(v[1]) + sqr(v[2]); }
inline double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline double dist2(const V3& a, const V3& b) { return sqr(a[0] - b[0]) + sqr(a[1] - b[1]) + sqr(a[2] - b[2]); }
inline V3 cross(const V3& a, const V3& b) {
    return V3(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}
struct M3 { double d[9]; };  // column-major, common.h:173-205
inline V3 mul(const M3& m, const V3& v) {
    return V3(m.d[0] * v[0] + m.d[3] * v[1] + m.d[6] * v[2],
              m.d[1] * v[0] + m.d[4] * v[1] + m.d[7] * v[2],
              m.d[2] * v[0] + m.d[5] * v[1] + m.d[8] * v[2]);
}
struct Q { double a, b, c, d; };
inline Q qmul(const Q& l, const Q& r) {  // boost::math::quaternion operator*=
    return Q{l.a * r.a - l.b * r.b - l.c * r.c - l.d * r.d,
             l.a * r.b + l.b * r.a + l.c * r.d - l.d * r.c,
             l.a * r.c - l.b * r.d + l.c * r.a + l.d * r.b,
             l.a * r.d + l.b * r.c - l.c * r.b + l.d * r.a};
}
void normalize_angle(double& x);                              // common.h:262-281
Q angle_to_quaternion(const V3& axis, double angle);          // quaternion.cpp:42-49
Q angle_to_quaternion(const V3& rotation);                    // quaternion.cpp:51-61
V3 quaternion_to_angle(const Q& q);                           // quaternion.cpp:63-81
M3 quaternion_to_r3(const Q& q);                              // quaternion.cpp:83-118
void quaternion_normalize_approx(Q& q);                       // quaternion.h:86-97
void quaternion_increment(Q& q, const V3& rotation);          // quaternion.cpp:135-139
template <typename T> void curl(double& e, T& deriv, double v);  // curl.h:30-37
void curl(double& e, double v);                                   // curl.h:38-43

// ---- flattened model --------------------------------------------------
struct Block {  // one ligand_conf or residue_conf inside a conf
    bool rigid;
    int conf_off, dof_off, ntors;
};

struct Model {
    int num_atoms = 0, num_movable = 0, num_frames = 0, num_ligands = 0, num_flex = 0;
    int conf_size = 0, dof = 0, num_pairs = 0, num_other_pairs = 0;
    std::vector<int> lig_pair_end, lig_begin, lig_end, lig_root;
    std::vector<int> type;
    std::vector<double> charge;
    std::vector<V3> local;  // frame-local (movable) / lab (inflex)
    std::vector<V3> lab;    // coords as read
    std::vector<int> fkind, fparent, fbegin, fend, fconf, fdof;
    std::vector<V3> forigin, faxis, finit;
    std::vector<Block> blocks;
    std::vector<std::vector<int>> children;
    std::vector<std::array<int, 2>> pairs;
    std::vector<int> heavy;  // movable non-hydrogen atoms
    void load(const sg_model_desc& m);
};

// the model's mutable state (model::coords, frame origins/orientations)
struct State {
    std::vector<V3> coords, minus_forces;
    std::vector<V3> origin, axis;
    std::vector<Q> q;
    std::vector<M3> rot;
};

struct Tables {
    int nt = 0, nc = 1, n = 0;
    double factor = 0, cutoff_sqr = 0;
    std::vector<double> smooth, fast;
    void load(const sg_tables_desc& t);
    int pair_index(int t1, int t2) const { return t1 <= t2 ? t1 + t2 * (t2 + 1) / 2 : t2 + t1 * (t1 + 1) / 2; }
};

// grid geometry of grid::init (grid.cpp:57-75)
struct GridGeom {
    int dim[3];
    V3 init, factor, factor_inv, dim_fl_minus_1;
    sg_grid_dims gd;
    void init_from(const sg_grid_dims& g);
    V3 index_to_argument(int x, int y, int z) const;
};

struct Grid {  // one type's maps
    std::vector<double> data, chargedata;
};

struct Receptor {
    std::vector<V3> xyz;
    std::vector<int> type;
    std::vector<double> charge;
};

// szv_grid_cache + szv_grid (szv_grid.h:55-221): lazily built 3 A cell
// lists; `full_cells` makes every list the one of the full brick
struct CellLists {
    const Receptor* r = nullptr;
    double cutoff_sqr = 0;
    std::vector<int> relevant;
    std::map<std::array<int, 3>, std::vector<int>> cache;
    bool full_cells = false;
    void init(const Receptor& rec, double cut2, const sg_grid_dims& gd);
    const std::vector<int>& get(const V3& coord);
};

// a user grid (--user_grid; grid::init(gd, user_in, ...), grid.cpp:78-110):
// its own geometry and values, x fastest
struct UserGrid {
    bool init = false;
    GridGeom geom;
    std::vector<double> data;
    double slope = 1e6;  // the cache's slope, used when it is added to the maps
};

struct Ctx {
    Tables tab;
    Receptor rec;
    GridGeom geom;
    std::vector<Grid> grids;  // by type
    std::vector<bool> built;
    bool has_receptor = false;
    bool full_cells = false;  // non_cache cell semantics
    UserGrid ug;
};

// evaluations
void model_set(const Model& m, const double* conf, State& s);                               // model.cpp:837-841
double eval_deriv(const Ctx& c, const Model& m, const double* conf, const double v[3], double slope,
                  State& s, double* g, uint64_t* evals);                                    // model.cpp:969-985
double eval_direct_deriv(Ctx& c, CellLists& cl, const Model& m, const double* conf, const double v[3],
                         double slope, State& s, double* g, bool* overlap, const sg_grid_dims* box = nullptr);                  // non_cache.cpp:109-191
void populate(Ctx& c, const int* types, int ntypes);                                        // cache.cpp:116-206

// search
struct Out { std::vector<double> c; double e; std::vector<V3> coords; };
struct Container { std::vector<Out> v; };
void add_to_output_container(Container& out, const Out& t, double min_rmsd, int max_size);  // coords.cpp:43-58
struct MinParams { int maxiters; int accurate_line; int early_term; };
// finish_docking's energies of one pose: model::eval on the direct sum and
// model::eval_intramolecular, fast table (main.cpp:257-282)
void score_pose(Ctx& c, const Model& m, const double* conf, const double v[3], double slope, double& e_out,
                double& intra_out, std::vector<V3>& coords_out);
}  // namespace orc
#endif
