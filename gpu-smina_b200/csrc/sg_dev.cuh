// Device-resident data of the engine: pair tables, receptor + grid maps,
// packed docking models, and the launch parameters of the kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include "../../include/smina_b200.h"
#include "sg_math.cuh"

namespace sg {

constexpr int kNumTypes = SG_NUM_TYPES;
constexpr int kNumTypePairs = kNumTypes * (kNumTypes + 1) / 2;

SG_HD int tri_index(int i, int j) { return i + j * (j + 1) / 2; }  // i <= j
SG_HD bool is_h(int t) { return t == 0 || t == 1; }

// precalculate_linear tables
struct DTables {
    int nc, n;
    double factor, cutoff_sqr;
    const double* smooth;  // [pair][n][nc][2]
    const double* fast;    // [pair][n][nc]
};

// grid_dims + grid::init geometry
struct DGeom {
    int dim[3];                  // n + 1 samples per axis
    double init[3], factor[3], factor_inv[3], dim_fl_minus_1[3];
    double gd_begin[3], gd_end[3];
    int gd_n[3];
    // 3 A receptor cell lists (szv_grid)
    int cell_off[3], cell_dim[3];
};

struct DReceptor {
    int natoms;
    const double* xyz;     // [n][3]
    const int* type;
    const double* charge;
    // cell lists for grid construction (first-query bricks) and for the
    // direct evaluation (full 3 A bricks)
    const int* pop_start;   // [ncells + 1]
    const int* pop_atoms;
    const int* full_start;  // [ncells + 1]
    const int* full_atoms;
    DGeom g;
    const double* map[kNumTypes];        // FP64 maps or null
    const double* cmap[kNumTypes];       // FP64 charge maps or null
    const float4* map32[kNumTypes];      // packed-corner FP32 copies
    const float4* cmap32[kNumTypes];
    const uint4* map16[kNumTypes];       // packed-corner FP16 copies
    // user grid (--user_grid): its own geometry, values x fastest; null: none
    const double* ugrid;
    DGeom ug;
};

// A docking model packed for the device.  Arrays index into three pools
// (ints, doubles, floats); see pack_one() in engine.cu for the layout.
struct __align__(16) DModel {
    int natoms, nmov, nframes, nlig, nflex, conf_size, dof, npairs, nother, nheavy, nlevels, nblocks;
    const int* type;
    const double* charge;
    const double* local;      // [natoms][3]
    const double* lab;        // [natoms][3]
    const int* atom_frame;    // [natoms], -1 for inflex
    const int* fkind;
    const int* fparent;
    const int* fbegin;
    const int* fend;
    const int* fconf;
    const int* fdof;
    const double* forigin;    // [F][3]
    const double* faxis;
    const double* finit;
    const int* level_start;   // [nlevels + 1]
    const int* level_frames;  // frames by depth
    const int* child_start;   // [F + 1]
    const int* child_list;
    const int* pairs;         // [P][2]
    const int* pair_group;    // [P] 0 = other pairs (v[2]), l + 1 = ligand l (v[0])
    const int* csr_start;     // [natoms + 1]
    const int* csr;           // (pair << 1) | (atom is b)
    const int* heavy;         // [nheavy]
    const int* lig_begin;
    const int* lig_end;
    const int* lig_root;
    const int* lig_pair_end;
    const int* blk_rigid;     // [nblocks] conf blocks: ligands then flex
    const int* blk_conf;
    const int* blk_dof;
    const int* blk_ntors;
    int ntors;
    const int* tor_conf;      // [ntors] conf index of each torsion (block order)
    const int* tor_dof;       // [ntors] change index
    const int* tor_frame;     // [ntors] frame of each torsion
    // mixed-precision copies
    const float4* local32;    // [natoms] (x, y, z, charge); lab coords for inflex
    const float4* lab32;      // [natoms] coords as read
    const float4* forigin32;  // [F]
    const float4* faxis32;    // [F]
    const float4* finit32;    // [F]
    const int* pair_tp;       // [P] type-pair index, bit 30 set when the pair's types are swapped
    const int* fsub_end;      // [F] end of the atom range of the frame's subtree (depth-first layout)
    // mixed-precision pair schedule: npchunks chunks of 32 slots; within a
    // chunk every atom is at most once the first and once the second atom.
    // Slot: a | b << 8 | type pair << 16 | swapped << 25 | intramolecular
    // (v[0]) << 26; unused slots kSlotEmpty (type pair 0x1ff, atoms 0 and 0,
    // so their loads stay in range).  Null when the model has more
    // than 255 atoms.
    const uint32_t* pslot;    // [npchunks * 32]
    int cost;                 // relative cost of one evaluation (atoms + pairs + frames)
    int npchunks;
    int pad_[2];
};

constexpr uint32_t kSlotEmpty = 0x1ffu << 16;
constexpr uint32_t kSlotPairMask = 0x1ffu;  // (slot >> 16) & mask: type pair, 0x1ff when empty
constexpr uint32_t kSlotSwap = 1u << 25, kSlotIntra = 1u << 26;

// FP32 pair table: per (type pair, sample i, component) the float4
// (e_i, dor_i, e_i+1, dor_i+1), so one interpolation is one 16 B load
struct DTables32 {
    int nc, n;
    float factor, cutoff_sqr;
    const float4* tab;  // [pair][n][nc]
};

// packed-corner grid maps: each cell's 8 corner values contiguous
// FP32: 2 x float4 = (f000 f100 f010 f110)(f001 f101 f011 f111); FP16: 1 x uint4
struct __align__(16) DMaps32 {
    int cdim[3];  // cells per axis (dim - 1)
    float init[3], factor[3], factor_inv[3], dim_fl_minus_1[3];
    const float4* m32[kNumTypes];
    const float4* c32[kNumTypes];
    const uint4* m16[kNumTypes];
    int half;
};

// Chain bookkeeping of the batched mixed-precision path
struct __align__(16) Chain32 {
    int model;
    unsigned steps;
    int maxiters;            // BFGS iterations of this ligand's search
    uint32_t key0, key1;     // request seed (Philox key)
    uint32_t lig, chain;     // Philox counter words
    double* out_e;           // [S]
    double* out_conf;        // [S][conf_size]
    float* out_coords;       // [S][nheavy][3]
    int* out_order;          // [S]
    int* out_count;
    unsigned long long* evals;
    unsigned long long* hits;  // [2]: grid lookups, in-cutoff pair lookups
    // completion signal (serving; null otherwise): the last of the ligand's
    // lig_chains chains to finish sets *host_flag (host-mapped memory)
    unsigned* done_count;
    volatile unsigned* host_flag;
    int lig_chains;
    const double* box;  // search box (lo xyz, hi xyz) of this chain's receptor; null: the launch's
    unsigned long long* span;  // [2] device clock (ns) at the chain's start and end; null: not recorded
    // phased runs (early stop): this launch runs steps [begin, end) (end 0:
    // all steps), resuming from and saving to resume (resume32_doubles);
    // null resume: one run of all steps
    unsigned begin, end;
    double* resume;
};
// a phased chain's saved state: conf, current and best energy, the Philox
// draw index, then (16-byte aligned) its atoms' and frames' positions
SG_HD int resume32_coords_at(int conf_size) { return (conf_size + 4) & ~1; }
SG_HD size_t resume32_doubles(int conf_size, int natoms, int nframes) {
    return (size_t)resume32_coords_at(conf_size) + 2 * (size_t)(natoms + nframes);
}

struct __align__(16) MCParams32;

// A serving grid's unit of work, published by the host in a ring while the
// grid runs: up to a block's worth of chains of one ligand, with everything
// the block needs to run them (all in the memory of the ligand's batch)
struct __align__(16) FeedItem32 {
    const DModel* model;
    const Chain32* chains;     // [count]
    const DMaps32* maps;       // the ligand's receptor's map set
    const MCParams32* params;
    int count;                 // chains of this item
    int stage_stride;          // shared-memory layout of the item's block
    int ws_stride;
    int team;                  // warps per chain: 1, 2 or 4
};
// The ring's control words (device memory): the host advances tail after
// copying items in; blocks claim items by advancing head
struct FeedCtrl32 {
    unsigned head, tail;
    unsigned started, exited, waiting;  // blocks of serving grids
    unsigned stop;                      // set by the host to end the grids
    unsigned pad_[2];
};

// A block's unit of work: chains [first, first + count) of one model
struct Item32 {
    int model, first, count;
    int rec;  // receptor slot in the launch's map table (0 when the launch has one receptor)
};

// per-warp workspace (bytes, 16 B aligned)
struct Ws32 {
    int coords, force, origin, axis, quat, rot;                  // float4 arrays (rot: 3 rows per frame)
    int x_tmp, x_cand, x_new, x_orig, g, g_new, g_orig, p, y, mhy, h;  // double arrays (h: n x n)
    int pf, pc;                                                  // prefix sums over atoms (float4)
    int scratch;                                                 // counters: 32 + 32 + 1 words
    int total;
};
SG_HD Ws32 ws32_layout(int natoms, int nframes, int conf, int dof) {
    Ws32 w;
    int o = 0;
    auto take = [&](int bytes) { int r = o; o += (bytes + 15) & ~15; return r; };
    w.coords = take(16 * natoms);
    w.force = take(16 * natoms);
    w.origin = take(16 * nframes);
    w.axis = take(16 * nframes);
    w.quat = take(16 * nframes);
    w.rot = take(48 * nframes);
    w.x_tmp = take(8 * conf);
    w.x_cand = take(8 * conf);
    w.x_new = take(8 * conf);
    w.x_orig = take(8 * conf);
    w.g = take(8 * dof);
    w.g_new = take(8 * dof);
    w.g_orig = take(8 * dof);
    w.p = take(8 * dof);
    w.y = take(8 * dof);
    w.mhy = take(8 * dof);
    w.h = take(8 * dof * dof);
    w.pf = take(16 * (natoms + 1));
    w.pc = take(16 * (natoms + 1));
    w.scratch = take(4 * 65);
    w.total = o;
    return w;
}

// The block-shared copy of a model for the mixed-precision kernels: counts,
// then the byte offsets (in the kernel's dynamic shared memory) of the
// arrays the search reads.  Arrays read once per chain or only for trees
// of more than 32 frames stay in global memory.
struct SModel {
    int natoms, nmov, nframes, nlig, conf_size, dof, nheavy, nlevels, nblocks, ntors, npchunks;
    int local32, type, atom_frame, forigin32, faxis32, fkind, fparent, fbegin, fsub_end, fconf, fdof, heavy, pslot,
        lig_root, lig_begin, lig_end, blk_rigid, blk_conf, blk_ntors, tor_conf, tor_dof;
    const float4* lab32;
    const float4* finit32;
    const int* level_start;
    const int* level_frames;
    Ws32 L;  // every warp's workspace layout (all warps of a block run this model)
};

// Bytes of the staged model (SModel + arrays), 16 B aligned pieces
SG_HD int stage32_bytes(int natoms, int nframes, int nheavy, int npchunks, int nlig, int nblocks, int ntors) {
    auto r = [](int b) { return (b + 15) & ~15; };
    return r((int)sizeof(SModel)) + r(16 * natoms) + 2 * r(4 * natoms) + 2 * r(16 * nframes) + 6 * r(4 * nframes) +
           r(4 * nheavy) + r(128 * npchunks) + 3 * r(4 * nlig) + 3 * r(4 * nblocks) + 2 * r(4 * ntors);
}

struct __align__(16) MCParams32 {
    float hunt[3], auth[3];
    float slope;
    double temperature, amplitude, min_rmsd;
    int num_saved, maxiters, accurate_line, early_term;
    double box[6];  // search box: lo xyz, hi xyz
};

// Per-warp FP64 workspace layout in shared memory (offsets in doubles)
struct Ws64 {
    int coords, mf, eatom, origin, axis, q, rot, fF, fT, pe, pf, pin;
    int x_tmp, x_cand, x_new, x_orig, g, g_new, g_orig, p, y, mhy, h, bcast, rmsd, mt;
    int total;  // doubles
};

SG_HD Ws64 ws64_layout(int natoms, int nframes, int npairs, int conf, int dof) {
    Ws64 w;
    int o = 0;
    auto take = [&](int n) { int r = o; o += (n + 1) & ~1; return r; };
    w.coords = take(3 * natoms);
    w.mf = take(3 * natoms);
    w.eatom = take(natoms);
    w.origin = take(3 * nframes);
    w.axis = take(3 * nframes);
    w.q = take(4 * nframes);
    w.rot = take(9 * nframes);
    w.fF = take(3 * nframes);
    w.fT = take(3 * nframes);
    w.pe = take(npairs);
    w.pf = take(3 * npairs);
    w.pin = take((npairs + 7) / 8);  // one byte per pair
    w.x_tmp = take(conf);
    w.x_cand = take(conf);
    w.x_new = take(conf);
    w.x_orig = take(conf);
    w.g = take(dof);
    w.g_new = take(dof);
    w.g_orig = take(dof);
    w.p = take(dof);
    w.y = take(dof);
    w.mhy = take(dof);
    w.h = take(dof * (dof + 1) / 2);
    w.bcast = take(16);
    w.rmsd = take(64);
    w.mt = take(313);  // 625 uint32 words + padding
    w.total = o;
    return w;
}

// Chain bookkeeping for the plain path (global memory)
// A chain's QuickVina 2 history (plain path, MCParams::visited) over n <=
// kHistMaxN change coordinates: the last 5n points, stored coordinate-major
// (coordinate i of slot e at x[i * 5n + e]), their energies, two gradient-sign
// masks per point (bit i: gradient i nonzero / positive) and the count of
// points added so far (the next slot is that count mod 5n; the ring is full
// once it reaches 5n).  Only the count needs zeroing before a chain starts.
constexpr int kHistMaxN = 64;
struct Hist64 {
    double* x;                 // [n][5n]
    double* f;                 // [5n]
    unsigned long long* mask;  // [5n][2]: nonzero, positive
    unsigned long long* adds;  // [1]
};
SG_HD size_t hist64_doubles(int n) { return (size_t)5 * n * (n + 1); }
SG_HD size_t hist64_words(int n) { return (size_t)10 * n + 1; }

struct Chain64 {
    int model;
    unsigned steps;
    int maxiters;
    double* hist;                    // history doubles (hist64_doubles(dof)), or null: no history
    unsigned long long* hist_words;  // history masks and count (hist64_words(dof), zeroed)
    const double* conf0;
    uint32_t* mt;        // [625] state (read + written)
    double* out_e;       // [num_saved]
    double* out_conf;    // [num_saved][conf_size]
    double* out_coords;  // [num_saved][nheavy][3]
    int* out_order;      // [num_saved] sorted order of the slots
    int* out_count;
    unsigned long long* evals;
};

struct MCParams64 {
    unsigned num_steps;
    double temperature, amplitude, min_rmsd;
    int num_saved;
    double hunt[3], auth[3];
    int maxiters, accurate_line, early_term;
    double slope;
};

// device error word (bounded failures report here instead of trapping)
enum : int { kDevOk = 0, kDevOverlap = 1, kDevBadModel = 2 };

}  // namespace sg
