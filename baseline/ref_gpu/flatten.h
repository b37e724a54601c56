/*
 * Conversion of this project's descriptors (include/smina_b200.h) to the
 * reference's flat structures (src/gpu/gpu_flatten_data.h), with host-side
 * index checks, so that the reference's own device library can be run on
 * the same inputs as this engine: by the oracle's pinning harness
 * (oracle/ref_gpu.cu, FP64) and by the reference GPU baseline
 * (baseline/ref_gpu/ref_search32.cu, FP32).  Needs the reference's headers
 * (src/gpu) on the include path.
 *
 * It restates the reference's flattener, src/gpu/gpu_flatten.cpp:
 * flatten_model :83-237, flatten_tables :239-271, flatten_receptor
 * :405-445, flatten_receptor_for_grid :447-486 and grid_geometry :488-503,
 * plus grid::init (src/lib/grid.cpp:57-75) and brick_distance_sqr
 * (src/lib/brick.h:28-45).  check_model and check_receptor verify every
 * index the reference's kernels read before anything is uploaded.
 */
#ifndef SMINA_B200_REF_FLATTEN_H
#define SMINA_B200_REF_FLATTEN_H

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "gpu_flatten_data.h"
#include "../../include/smina_b200.h"

namespace refflat {

using namespace gpusmina;

inline void need(bool ok, const char* what) {
    if (!ok) throw std::runtime_error(what);
}

// ---- grid geometry (grid::init, gpu_model_flattener::grid_geometry) --------------------------------
inline FlatGridGeometry geometry(const sg_grid_dims& gd) {
    FlatGridGeometry g;
    for (int i = 0; i < 3; i++) {
        // at least two points per axis: evaluate_aux reads corners a and a + 1 with a <= dim - 2
        need(gd.n[i] >= 1 && gd.end[i] > gd.begin[i], "grid: bad dimensions");
        g.dim[i] = gd.n[i] + 1;
        g.init[i] = gd.begin[i];
        const double range = gd.end[i] - gd.begin[i];
        g.dim_fl_minus_1[i] = double(g.dim[i]) - 1.0;
        g.factor[i] = g.dim_fl_minus_1[i] / range;
        g.factor_inv[i] = 1 / g.factor[i];
        g.gd_begin[i] = gd.begin[i];
        g.gd_end[i] = gd.end[i];
        g.gd_enabled[i] = gd.n[i] > 0;
    }
    return g;
}

// ---- tables (flatten_tables, linear) ------------------------------------------------------------------
inline FlatTables tables(const sg_tables_desc& t) {
    need(t.num_types == NUM_TYPES, "tables: 27 types expected");
    need(t.num_components >= 1 && t.num_components <= MAX_COMPONENTS && t.n > 0, "tables: bad sizes");
    need(t.smooth && t.fast, "tables: null arrays");
    FlatTables f;
    f.kind = FlatTables::Linear;
    f.num_components = t.num_components;
    f.cutoff_sqr = t.cutoff_sqr;
    f.cutoff = std::sqrt(t.cutoff_sqr);
    f.factor = t.factor;
    f.n = t.n;
    const size_t cells = size_t(NUM_TYPE_PAIRS) * t.n * t.num_components;
    f.lin_fast.assign(t.fast, t.fast + cells);
    f.lin_smooth.assign(t.smooth, t.smooth + 2 * cells);
    return f;
}

// ---- receptor cell lists (flatten_receptor, flatten_receptor_for_grid) ---------------------------------
inline double closest_between(double b, double e, double x) { return x <= b ? b : (x >= e ? e : x); }

inline double brick_distance_sqr(const double lo[3], const double hi[3], const double* v) {
    double c[3];
    for (int i = 0; i < 3; i++) c[i] = closest_between(lo[i], hi[i], v[i]);
    const double d0 = c[0] - v[0], d1 = c[1] - v[1], d2 = c[2] - v[2];
    return d0 * d0 + d1 * d1 + d2 * d2;
}

inline bool usable(int t) { return t >= 0 && t < NUM_TYPES && !type_is_hydrogen(t); }

inline void add_atoms(const sg_receptor_desc& r, const std::vector<int>& idx, FlatReceptor& out) {
    for (int i : idx) {
        for (int d = 0; d < 3; d++) out.coords.push_back(r.coords[3 * i + d]);
        out.type.push_back(r.type[i]);
        out.charge.push_back(r.charge ? r.charge[i] : 0.0);
    }
}

inline void build_cells(const FlatReceptor& rr, double cutoff_sqr, const std::vector<double> lower[3],
                 const std::vector<double> upper[3], FlatReceptor& r) {
    const int natoms = int(rr.type.size());
    r.cell_start.assign(1, 0);
    r.cell_atoms.clear();
    for (int z = 0; z < r.dims[2]; z++)
        for (int y = 0; y < r.dims[1]; y++)
            for (int x = 0; x < r.dims[0]; x++) {
                const double lo[3] = {lower[0][x], lower[1][y], lower[2][z]};
                const double hi[3] = {upper[0][x], upper[1][y], upper[2][z]};
                for (int a = 0; a < natoms; a++)
                    if (brick_distance_sqr(lo, hi, &rr.coords[3 * a]) < cutoff_sqr) r.cell_atoms.push_back(a);
                r.cell_start.push_back(int(r.cell_atoms.size()));
            }
}

// non_cache's receptor: every usable heavy atom, cells over its bounding box
inline FlatReceptor receptor_full(const sg_receptor_desc& rd, double cutoff_sqr) {
    FlatReceptor r;
    std::vector<int> idx;
    for (int i = 0; i < rd.num_atoms; i++)
        if (usable(rd.type[i])) idx.push_back(i);
    add_atoms(rd, idx, r);
    const double cutoff = std::sqrt(cutoff_sqr);
    double lo[3] = {1.79769313486231570e308, 1.79769313486231570e308, 1.79769313486231570e308};
    double hi[3] = {-lo[0], -lo[1], -lo[2]};
    for (size_t k = 0; k < idx.size(); k++)
        for (int d = 0; d < 3; d++) {
            lo[d] = std::min(lo[d], r.coords[3 * k + d]);
            hi[d] = std::max(hi[d], r.coords[3 * k + d]);
        }
    std::vector<double> lower[3], upper[3];
    for (int d = 0; d < 3; d++) {
        if (idx.empty()) lo[d] = hi[d] = 0;
        r.offset[d] = int(std::floor((lo[d] - cutoff) / 3.0));
        r.dims[d] = int(std::ceil((hi[d] + cutoff) / 3.0)) - r.offset[d] + 1;
        for (int i = 0; i < r.dims[d]; i++) {
            lower[d].push_back((r.offset[d] + i) * 3.0);
            upper[d].push_back((r.offset[d] + i + 1) * 3.0);
        }
    }
    FlatReceptor atoms = r;
    build_cells(atoms, cutoff_sqr, lower, upper, r);
    return r;
}

// cache::populate's receptor: atoms within the cutoff of the box; each 3 A
// cell's brick is that of the first grid point that falls into it
inline FlatReceptor receptor_for_grid(const sg_receptor_desc& rd, const sg_grid_dims& gd, const FlatGridGeometry& geo,
                               double cutoff_sqr) {
    FlatReceptor r;
    std::vector<int> idx;
    for (int i = 0; i < rd.num_atoms; i++)
        if (usable(rd.type[i]) && brick_distance_sqr(gd.begin, gd.end, rd.coords + 3 * i) < cutoff_sqr)
            idx.push_back(i);
    add_atoms(rd, idx, r);
    for (int d = 0; d < 3; d++) {
        r.offset[d] = int(std::floor(gd.begin[d] / 3.0));
        r.dims[d] = int(std::ceil(gd.end[d] / 3.0)) - r.offset[d] + 1;
    }
    std::vector<double> lower[3], upper[3];
    for (int d = 0; d < 3; d++) {
        lower[d].assign(r.dims[d], 0);
        upper[d].assign(r.dims[d], 0);
        std::vector<char> seen(r.dims[d], 0);
        for (int i = 0; i <= gd.n[d]; i++) {
            const double c = geo.init[d] + geo.factor_inv[d] * double(i);
            const int cell = int(std::floor(c / 3.0)) - r.offset[d];
            need(cell >= 0 && cell < r.dims[d], "receptor: grid point outside the cell range");
            if (!seen[cell]) {
                seen[cell] = 1;
                lower[d][cell] = std::floor(c / 3.0) * 3.0;
                upper[d][cell] = std::ceil(c / 3.0) * 3.0;
            }
        }
    }
    FlatReceptor atoms = r;
    build_cells(atoms, cutoff_sqr, lower, upper, r);
    return r;
}

inline void check_receptor(const FlatReceptor& r) {
    const int n = int(r.type.size());
    need(r.coords.size() == size_t(3 * n) && r.charge.size() == size_t(n), "receptor: array sizes");
    need(r.dims[0] > 0 && r.dims[1] > 0 && r.dims[2] > 0, "receptor: empty cell grid");
    const size_t cells = size_t(r.dims[0]) * r.dims[1] * r.dims[2];
    need(r.cell_start.size() == cells + 1 && r.cell_start[0] == 0, "receptor: cell_start size");
    for (size_t c = 0; c < cells; c++) need(r.cell_start[c] <= r.cell_start[c + 1], "receptor: cell_start order");
    need(size_t(r.cell_start[cells]) == r.cell_atoms.size(), "receptor: cell_atoms size");
    for (int a : r.cell_atoms) need(a >= 0 && a < n, "receptor: cell atom out of range");
    for (int t : r.type) need(t >= 0 && t < NUM_TYPES, "receptor: atom type out of range");
}

// ---- model (flatten_model) ------------------------------------------------------------------------------
inline int ref_kind(int k) {  // this project's frame kinds -> the reference's FrameKind
    if (k == SG_FRAME_RIGID) return FRAME_RIGID;
    if (k == SG_FRAME_FIRST_SEGMENT) return FRAME_FIRST_SEGMENT;
    if (k == SG_FRAME_SEGMENT) return FRAME_SEGMENT;
    throw std::runtime_error("model: bad frame kind");
}

inline FlatModel flatten(const sg_model_desc& d) {
    const int N = d.num_atoms, M = d.num_movable, F = d.num_frames, P = d.num_pairs;
    need(N > 0 && M > 0 && M <= N && F > 0 && P >= 0, "model: counts");
    need(d.num_ligands >= 0 && d.num_flex >= 0 && d.num_other_pairs >= 0 && d.num_other_pairs <= P, "model: counts");
    need(d.atom_type && d.atom_charge && d.atom_local && d.atom_lab && d.frame_kind && d.frame_parent &&
             d.frame_begin && d.frame_end && d.frame_conf && d.frame_dof && d.frame_origin && d.frame_axis &&
             d.frame_init_origin && (P == 0 || d.pairs) &&
             (d.num_ligands == 0 || (d.lig_pair_end && d.ligand_atom_begin && d.ligand_atom_end && d.ligand_root)),
         "model: null arrays");
    FlatModel fm;
    fm.num_movable = M;
    fm.num_atoms = N;
    for (int i = 0; i < M; i++) {
        const int t = d.atom_type[i];
        need(t >= 0 && t < NUM_TYPES, "model: movable atom type out of range");
        fm.atom_type.push_back(t);
        fm.atom_charge.push_back(d.atom_charge[i]);
        for (int k = 0; k < 3; k++) {
            fm.atom_local.push_back(d.atom_local[3 * i + k]);
            fm.init_coords.push_back(d.atom_lab[3 * i + k]);
        }
        if (!type_is_hydrogen(t)) fm.heavy.push_back(i);
    }
    for (int i = M; i < N; i++)
        for (int k = 0; k < 3; k++) fm.inflex_coords.push_back(d.atom_lab[3 * i + k]);
    // frames in the order given (depth-first pre-order, ligands then flex)
    std::vector<int> depth(F, 0);
    for (int f = 0; f < F; f++) {
        Frame<double> fr;
        fr.parent = d.frame_parent[f];
        need(fr.parent < f, "model: frames must be in pre-order");
        fr.kind = ref_kind(d.frame_kind[f]);
        fr.begin = d.frame_begin[f];
        fr.end = d.frame_end[f];
        fr.child_begin = fr.child_end = 0;
        fr.conf_idx = d.frame_conf[f];
        fr.change_idx = d.frame_dof[f];
        for (int k = 0; k < 3; k++) {
            fr.rel_origin[k] = fr.rel_axis[k] = fr.origin[k] = fr.axis[k] = 0;
            if (fr.kind == FRAME_SEGMENT) {
                fr.rel_origin[k] = d.frame_origin[3 * f + k];
                fr.rel_axis[k] = d.frame_axis[3 * f + k];
            } else if (fr.kind == FRAME_FIRST_SEGMENT) {
                fr.origin[k] = d.frame_origin[3 * f + k];
                fr.axis[k] = d.frame_axis[3 * f + k];
            }
            fm.init_frame_origin.push_back(d.frame_init_origin[3 * f + k]);
        }
        depth[f] = fr.parent < 0 ? 0 : depth[fr.parent] + 1;
        fm.frames.push_back(fr);
    }
    // conf blocks: ligands (in ligand order), then flexible residues (in frame order)
    std::vector<int> root_of(F);
    for (int f = 0; f < F; f++) root_of[f] = d.frame_parent[f] < 0 ? f : root_of[d.frame_parent[f]];
    auto tree_frames = [&](int root) {
        int n = 0;
        for (int f = 0; f < F; f++) n += root_of[f] == root && f != root;
        return n;
    };
    for (int l = 0; l < d.num_ligands; l++) {
        const int root = d.ligand_root[l];
        need(root >= 0 && root < F && fm.frames[root].kind == FRAME_RIGID, "model: ligand root");
        ConfBlock b;
        b.conf_offset = d.frame_conf[root];
        b.change_offset = d.frame_dof[root];
        b.ntors = tree_frames(root);
        b.is_ligand = 1;
        b.root_frame = root;
        b.atom_begin = d.ligand_atom_begin[l];
        b.atom_end = d.ligand_atom_end[l];
        fm.blocks.push_back(b);
    }
    for (int f = 0; f < F; f++) {
        if (fm.frames[f].kind != FRAME_FIRST_SEGMENT) continue;
        ConfBlock b;
        b.conf_offset = d.frame_conf[f];
        b.change_offset = d.frame_dof[f];
        b.ntors = 1 + tree_frames(f);
        b.is_ligand = 0;
        b.root_frame = f;
        b.atom_begin = b.atom_end = 0;
        fm.blocks.push_back(b);
    }
    fm.conf_size = d.conf_size;
    fm.change_size = d.dof;
    fm.num_ligands = d.num_ligands;
    fm.num_flex = d.num_flex;
    // children in branch (frame) order, then depth levels
    for (int f = 0; f < F; f++) {
        fm.frames[f].child_begin = int(fm.children.size());
        for (int c = f + 1; c < F; c++)
            if (d.frame_parent[c] == f) fm.children.push_back(c);
        fm.frames[f].child_end = int(fm.children.size());
    }
    const int maxdepth = *std::max_element(depth.begin(), depth.end());
    fm.level_start.push_back(0);
    for (int lv = 0; lv <= maxdepth; lv++) {
        for (int f = 0; f < F; f++)
            if (depth[f] == lv) fm.level_frames.push_back(f);
        fm.level_start.push_back(int(fm.level_frames.size()));
    }
    fm.atom_frame.assign(M, -1);
    for (int f = 0; f < F; f++) {
        need(fm.frames[f].begin >= 0 && fm.frames[f].begin <= fm.frames[f].end && fm.frames[f].end <= M,
             "model: frame atom range");
        for (int i = fm.frames[f].begin; i < fm.frames[f].end; i++) {
            need(fm.atom_frame[i] < 0, "model: frames overlap");
            fm.atom_frame[i] = f;
        }
    }
    for (int i = 0; i < M; i++) need(fm.atom_frame[i] >= 0, "model: atom without frame");
    // pair lists: other pairs, then each ligand's
    fm.list_start.push_back(0);
    fm.list_start.push_back(d.num_other_pairs);
    for (int l = 0; l < d.num_ligands; l++) fm.list_start.push_back(d.lig_pair_end[l]);
    need(fm.list_start.back() == P, "model: pair lists do not cover the pairs");
    for (int k = 0; k < P; k++) {
        const int a = d.pairs[2 * k], b = d.pairs[2 * k + 1];
        need(a >= 0 && a < N && b >= 0 && b < N && a != b, "model: pair atom out of range");
        const int ta = d.atom_type[a], tb = d.atom_type[b];
        need(ta >= 0 && ta < NUM_TYPES && tb >= 0 && tb < NUM_TYPES, "model: pair atom type out of range");
        Pair<double> p;
        p.a = a;
        p.b = b;
        p.tpair = tri_index_permissive(ta, tb);
        p.swapped = ta > tb;
        p.abs_qa = std::abs(d.atom_charge[a]);
        p.abs_qb = std::abs(d.atom_charge[b]);
        p.qab = d.atom_charge[a] * d.atom_charge[b];
        fm.pairs.push_back(p);
    }
    // atom-centric view of the pairs
    std::vector<std::vector<int> > per_atom(M);
    for (int k = 0; k < P; k++) {
        const Pair<double>& p = fm.pairs[k];
        const int list0 = k < fm.list_start[1];
        const bool a_mov = p.a < M, b_mov = p.b < M;
        if (a_mov) per_atom[p.a].push_back((k << 3) | (list0 << 1) | (1 << 2));
        if (b_mov) per_atom[p.b].push_back((k << 3) | 1 | (list0 << 1) | ((a_mov ? 0 : 1) << 2));
    }
    fm.nbr_start.push_back(0);
    for (int i = 0; i < M; i++) {
        fm.nbr.insert(fm.nbr.end(), per_atom[i].begin(), per_atom[i].end());
        fm.nbr_start.push_back(int(fm.nbr.size()));
    }
    return fm;
}

inline void check_model(const FlatModel& m) {
    const int M = m.num_movable, N = m.num_atoms, F = int(m.frames.size()), P = int(m.pairs.size());
    need(int(m.atom_type.size()) == M && int(m.atom_charge.size()) == M && int(m.atom_local.size()) == 3 * M &&
             int(m.init_coords.size()) == 3 * M && int(m.atom_frame.size()) == M &&
             int(m.inflex_coords.size()) == 3 * (N - M) && int(m.init_frame_origin.size()) == 3 * F,
         "flat model: array sizes");
    need(int(m.children.size()) == F - int(m.blocks.size()), "flat model: children count");
    for (int c : m.children) need(c > 0 && c < F, "flat model: child out of range");
    need(m.level_start.front() == 0 && m.level_start.back() == F && int(m.level_frames.size()) == F,
         "flat model: levels");
    for (int f : m.level_frames) need(f >= 0 && f < F, "flat model: level frame out of range");
    int ntors = 0;
    for (int f = 0; f < F; f++) {
        const Frame<double>& fr = m.frames[f];
        need(fr.parent >= -1 && fr.parent < f, "flat model: parent");
        need(fr.child_begin >= 0 && fr.child_begin <= fr.child_end && fr.child_end <= int(m.children.size()),
             "flat model: child range");
        if (fr.kind == FRAME_RIGID)
            need(fr.conf_idx >= 0 && fr.conf_idx + 7 <= m.conf_size && fr.change_idx >= 0 &&
                     fr.change_idx + 6 <= m.change_size, "flat model: rigid offsets");
        else {
            need(fr.conf_idx >= 0 && fr.conf_idx < m.conf_size && fr.change_idx >= 0 && fr.change_idx < m.change_size,
                 "flat model: torsion offsets");
            ntors++;
        }
    }
    int block_tors = 0, ligands = 0;
    for (const ConfBlock& b : m.blocks) {
        need(b.root_frame >= 0 && b.root_frame < F && m.frames[b.root_frame].parent < 0, "flat model: block root");
        need(b.conf_offset >= 0 && b.conf_offset + (b.is_ligand ? 7 : 0) + b.ntors <= m.conf_size &&
                 b.change_offset >= 0 && b.change_offset + (b.is_ligand ? 6 : 0) + b.ntors <= m.change_size,
             "flat model: block offsets");
        if (b.is_ligand) {
            need(b.atom_begin >= 0 && b.atom_begin <= b.atom_end && b.atom_end <= M, "flat model: ligand atoms");
            ligands++;
        }
        block_tors += b.ntors;
    }
    need(block_tors == ntors && ligands == m.num_ligands && int(m.blocks.size()) == m.num_ligands + m.num_flex,
         "flat model: blocks");
    need(int(m.list_start.size()) == m.num_ligands + 2 && m.list_start.front() == 0 && m.list_start.back() == P,
         "flat model: lists");
    for (size_t l = 0; l + 1 < m.list_start.size(); l++) need(m.list_start[l] <= m.list_start[l + 1], "flat model: list order");
    for (const Pair<double>& p : m.pairs)
        need(p.a >= 0 && p.a < N && p.b >= 0 && p.b < N && p.tpair >= 0 && p.tpair < NUM_TYPE_PAIRS,
             "flat model: pair");
    need(int(m.nbr_start.size()) == M + 1 && m.nbr_start.back() == int(m.nbr.size()), "flat model: nbr");
    for (int e : m.nbr) need((e >> 3) >= 0 && (e >> 3) < P, "flat model: nbr entry");
    for (int h : m.heavy) need(h >= 0 && h < M, "flat model: heavy atom");
}

}  // namespace refflat

#endif
