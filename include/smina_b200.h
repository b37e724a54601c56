/*
 * smina_b200.h - C ABI of the B200 docking engine.
 *
 * The engine runs smina's docking search (Monte Carlo chains, each doing
 * BFGS local optimisation of a ligand conformation scored against receptor
 * grid maps and an intramolecular pair table) on one B200.  Everything that
 * crosses this boundary is plain data: pointers, sizes and int status codes.
 * No exception, C++ type or torch type crosses it.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   sg_create / sg_destroy       gpusmina::GpuDocking ctor/dtor          src/gpu/gpu_docking.h:51-114
 *                                (Engine<T> per device                   src/gpu/gpu_docking.cpp:237-264)
 *   sg_set_tables                Engine::ensure_tables / flatten_tables src/gpu/gpu_flatten.cpp:239-332
 *   sg_set_receptor              ensure_receptor / DeviceGrids::build   src/gpu/gpu_device.cu:199-250
 *                                (cache::populate                       src/lib/cache.cpp:116-206)
 *   sg_build_grids               build_grids_kernel                     src/gpu/gpu_device.cu:133-186
 *   sg_set_user_grid             the user_grid argument of GpuDocking    src/gpu/gpu_docking.h:71,77,93,107
 *                                (FlatUserGrid                          src/gpu/gpu_flatten_data.h:90-96)
 *   sg_eval                      eval_confs (model::eval_deriv)          src/gpu/gpu_kernels.h:22-126,
 *                                                                        src/lib/model.cpp:969-985
 *   sg_dock                      run_monte_carlo (monte_carlo::operator()) src/gpu/gpu_kernels_impl.cuh:659-885,
 *                                                                        src/lib/monte_carlo.cpp:95-130
 *   sg_refine                    run_refine (refine_structure)          src/gpu/gpu_kernels_impl.cuh:999-1098,
 *                                                                        src/main/main.cpp:165-190
 *   sg_minimize                  GpuDocking::minimize_batch             src/gpu/gpu_docking.cpp:690-742
 *   sg_score                     finish_docking's rescoring energies    src/main/main.cpp:257-282
 *   sg_dock_batch32              GpuDocking::dock_batch (batched screen) src/gpu/gpu_docking.cpp:756-831
 *   sg_serve_*                   (no counterpart: continuous-batching request loop)
 *   sg_dock_batch32_noalloc      (no counterpart: the batched search without device allocation)
 *   sg_last_error                the std::runtime_error text the reference throws
 *
 * Conventions
 *   - All energies, coordinates, confs and changes are double on the ABI.
 *   - A conf is laid out per ligand as position(3), orientation quaternion
 *     (4: a, b, c, d = R_component_1..4), torsions; then the torsions of
 *     each flexible residue.  A change (gradient) is laid out per ligand as
 *     position(3), orientation(3), torsions; then flex torsions
 *     (conf.h: change::operator()(index)).
 *   - Atom order, frame order and pair order are smina's model order (see
 *     sg_model_desc).
 */
#ifndef SMINA_B200_H
#define SMINA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define SG_OK            0
#define SG_ERR_ARG       1  /* bad argument / unsupported input            */
#define SG_ERR_CUDA      2  /* CUDA runtime error                          */
#define SG_ERR_NOMEM     3  /* device allocation failed / admission refused*/
#define SG_ERR_OVERLAP   4  /* ligand atom exactly overlaps receptor atom  */
#define SG_ERR_TIMEOUT   5  /* bounded device wait gave up / cancelled     */
#define SG_ERR_STATE     6  /* call out of order (e.g. no tables set)      */

/* ---- precision modes -------------------------------------------------- */
#define SG_PREC_FP64      0  /* plain path: bit-exact with the CPU restatement */
#define SG_PREC_FP32      1  /* FP32 eval/tree, FP64 BFGS update + Armijo test */
#define SG_PREC_FP32_H16  2  /* as FP32, grid maps stored as FP16             */

#define SG_NUM_TYPES 27       /* smina_atom_type::NumTypes */

/* frame kinds of the torsion tree (tree.h) */
#define SG_FRAME_RIGID          0  /* rigid_body: ligand root            */
#define SG_FRAME_SEGMENT        1  /* segment: branch below a parent     */
#define SG_FRAME_FIRST_SEGMENT  2  /* first_segment: flex residue root   */

/* grid_dims: n[i] intervals, n[i]+1 sample points per axis */
typedef struct sg_grid_dims {
    double begin[3];
    double end[3];
    int n[3];
} sg_grid_dims;

/* precalculate_linear tables (precalculate.h:187-308).  Type pair index
 * for types i <= j is i + j*(j+1)/2 (triangular_matrix_index). */
typedef struct sg_tables_desc {
    int num_types;        /* SG_NUM_TYPES                                   */
    int num_components;   /* 1, or 4 with charge-dependent terms            */
    int n;                /* samples per type pair: int(factor*cutoff_sqr)+3 */
    double factor;        /* samples per A^2 (default 32)                   */
    double cutoff_sqr;    /* scoring cutoff squared (64)                    */
    const double* smooth; /* [npairs][n][nc][2]: (e, dor)                    */
    const double* fast;   /* [npairs][n][nc]: midpoint energies (grid build) */
} sg_tables_desc;

/* rigid receptor atoms (model::grid_atoms); hydrogens and untyped atoms
 * are allowed and skipped exactly as smina skips them */
typedef struct sg_receptor_desc {
    int num_atoms;
    const double* coords; /* [num_atoms][3] */
    const int* type;      /* smina type, SG_NUM_TYPES = unassigned */
    const double* charge;
} sg_receptor_desc;

/* The movable part of one smina `model`: its ligands and flexible
 * residues, flattened in model order.
 *   atoms:  [0, num_movable) move (ligand atoms, then flex side chains);
 *           [num_movable, num_atoms) are "inflex" atoms with fixed lab
 *           coordinates.
 *   frames: every tree node in depth-first pre-order, ligands first, then
 *           flexible residues; a frame's atoms are [begin, end).
 *   pairs:  other_pairs first (ligand-flex, flex-flex, flex-inflex ...,
 *           curled with v[2]), then each ligand's internal pairs in
 *           ligand order (curled with v[0]); lig_pair_end[l] is the end of
 *           ligand l's pairs. */
typedef struct sg_model_desc {
    int num_atoms;
    int num_movable;
    int num_frames;
    int num_ligands;
    int num_flex;
    int conf_size;
    int dof;
    int num_pairs;
    int num_other_pairs;
    const int*    lig_pair_end;      /* [num_ligands]                        */
    const int*    ligand_atom_begin; /* [num_ligands] ligand atom range      */
    const int*    ligand_atom_end;   /* [num_ligands]                        */
    const int*    ligand_root;       /* [num_ligands] root frame index       */
    const int*    atom_type;         /* [num_atoms]                          */
    const double* atom_charge;       /* [num_atoms]                          */
    const double* atom_local;        /* [num_atoms][3] frame-local coords (movable);
                                        lab coords (inflex)                  */
    const double* atom_lab;          /* [num_atoms][3] the model's coords as
                                        read (model::coords before any set)  */
    const int*    frame_kind;        /* [num_frames] SG_FRAME_*              */
    const int*    frame_parent;      /* [num_frames] -1 for roots            */
    const int*    frame_begin;       /* [num_frames]                         */
    const int*    frame_end;         /* [num_frames]                         */
    const int*    frame_conf;        /* rigid: position offset in conf; else torsion offset */
    const int*    frame_dof;         /* rigid: position offset in change; else torsion offset */
    const double* frame_origin;      /* [num_frames][3] rigid: initial origin;
                                        segment: origin relative to parent;
                                        first_segment: lab origin           */
    const double* frame_axis;        /* [num_frames][3] segment: relative axis;
                                        first_segment: lab axis             */
    const double* frame_init_origin; /* [num_frames][3] lab origin as read   */
    const int*    pairs;             /* [num_pairs][2] atom indices a < b     */
} sg_model_desc;

/* monte_carlo + minimization_params (monte_carlo.h:29-37, main.cpp:513-529) */
typedef struct sg_mc_params {
    unsigned num_steps;
    double temperature;         /* 1.2                                    */
    double mutation_amplitude;  /* 2                                      */
    double min_rmsd;            /* 1.0 during the search                  */
    int num_saved_mins;         /* max(20, num_modes)                     */
    double hunt_cap[3];         /* (10, 10, 10)                           */
    double authentic_v[3];      /* (1000, 1000, 1000)                     */
    int maxiters;               /* BFGS iterations: (25 + N_movable) / 3  */
    int accurate_line;          /* 1: accurate_line_search                */
    int early_term;             /* minimization_params::early_term        */
    double cache_slope;         /* grid out-of-box slope (1e6)            */
    int visited;                /* 1: QuickVina 2's history check skips
                                   local optimisations it deems redundant
                                   (MCParams::visited, gpu_mc_structs.h:30-33;
                                   not smina's search).  Plain path only.   */
} sg_mc_params;

/* One chain of the plain (FP64) path: its starting conf and the
 * mt19937 state after randomisation (624 words + index). */
typedef struct sg_chain_input {
    int model;          /* index into the models array                   */
    unsigned num_steps;
    const double* conf; /* [conf_size]                                   */
    const uint32_t* mt; /* [625]: state words then index (0..624)        */
    int maxiters;       /* BFGS iterations; 0: sg_mc_params.maxiters
                           (ChainInput::maxiters, gpu_kernels.h)         */
} sg_chain_input;

/* Result container of one chain (output_container, sorted ascending). */
typedef struct sg_chain_result {
    int count;          /* entries written, <= num_saved_mins            */
    double* e;          /* [num_saved_mins]                              */
    double* conf;       /* [num_saved_mins][conf_size]                   */
    double* coords;     /* [num_saved_mins][num_heavy_movable][3]        */
    uint64_t evals;     /* eval_deriv calls this chain made              */
} sg_chain_result;

typedef struct sg_engine sg_engine;

/* ---- engine ----------------------------------------------------------- */
int  sg_create(int device, int precision, sg_engine** out);
void sg_destroy(sg_engine* e);
const char* sg_last_error(const sg_engine* e);
int  sg_precision(const sg_engine* e);
/* The engine's device ordinal, its SM count and the shared memory a block
 * may opt in to (read at sg_create; no device work).  Any pointer may be
 * NULL.  Callers size batches from it, as the reference's
 * GpuDocking::chains_per_batch does from the device's residency
 * (src/gpu/gpu_docking.h:109-111). */
int  sg_device_info(const sg_engine* e, int* device, int* num_sms, int* smem_optin);

/* Pair tables (copied to the device). */
int sg_set_tables(sg_engine* e, const sg_tables_desc* t);

/* Receptor + box.  Keeps the receptor resident under `receptor_id`
 * (0..SG_MAX_RECEPTORS-1) and builds grid maps on demand. */
#define SG_MAX_RECEPTORS 16
int sg_set_receptor(sg_engine* e, int receptor_id, const sg_receptor_desc* r,
                    const sg_grid_dims* gd);
/* Build the maps of the listed ligand atom types (cache::populate). */
int sg_build_grids(sg_engine* e, int receptor_id, const int* types, int ntypes);
/* Copy one built map back: data [(n0+1)(n1+1)(n2+1)] (x fastest) and, with
 * charge-dependent terms, chargedata (NULL otherwise). */
int sg_get_grid(sg_engine* e, int receptor_id, int type, double* data, double* chargedata);
/* Drop a receptor and its maps. */
int sg_drop_receptor(sg_engine* e, int receptor_id);
/* A user grid (--user_grid) for receptor `receptor_id`: its own box `gd`
 * and values data [(n0+1)(n1+1)(n2+1)], x fastest, as smina holds them
 * after reading the grid file.  It is added to every map at the map point's
 * index coordinates with `cache_slope` (cache::populate, cache.cpp:204-205),
 * and to the direct receptor sum at each atom with its derivative
 * (non_cache::eval_deriv, non_cache.cpp:180-184), so refinement and
 * sg_minimize see it; the rescoring of sg_score does not (non_cache::eval
 * has no user-grid term).  gd == NULL or data == NULL clears it.  Maps built
 * before are dropped and rebuilt on demand. */
int sg_set_user_grid(sg_engine* e, int receptor_id, const sg_grid_dims* gd, const double* data,
                     double cache_slope);

/* model::eval_deriv for nconfs confs of one model against receptor maps
 * (cache) of `receptor_id`.  out_e [nconfs], out_g [nconfs][dof],
 * out_coords [nconfs][num_movable][3] (may be NULL).  FP32 engines run the
 * mixed-precision evaluation the batched search uses. */
int sg_eval(sg_engine* e, int receptor_id, const sg_model_desc* m, int nconfs,
            const double* confs, const double v[3], double slope,
            double* out_e, double* out_g, double* out_coords);

/* Direct receptor evaluation (non_cache::eval_deriv) with box penalty
 * slope; returns SG_ERR_OVERLAP like smina's exception. */
int sg_eval_direct(sg_engine* e, int receptor_id, const sg_model_desc* m, int nconfs,
                   const double* confs, const double v[3], double slope,
                   double* out_e, double* out_g);

/* monte_carlo::operator() for every chain, all chains in one launch. */
int sg_dock(sg_engine* e, int receptor_id, const sg_model_desc* models, int nmodels,
            const sg_chain_input* chains, int nchains, const sg_mc_params* p,
            sg_chain_result* out);

/* quasi_newton (BFGS, bfgs.h:202-282) of each conf against the maps;
 * confs [n][conf_size] updated in place, out_e [n].  FP32 engines run the
 * batched search's mixed-precision BFGS (FP32 energies and gradients; FP64
 * conf, inverse Hessian and acceptance tests), so its local optimisations
 * can be compared with the plain path's from the same starts. */
int sg_bfgs(sg_engine* e, int receptor_id, const sg_model_desc* m, int nconfs, double* confs,
            const double v[3], double slope, int maxiters, int accurate_line, int early_term,
            double* out_e);

/* refine_structure for each pose: BFGS on the direct receptor sum with box
 * slope 10, 100, ... (<= 5 tries) until every movable heavy atom is inside
 * the box.  confs [n][max conf_size over models] in/out, out_e [n] (max
 * double if it never got inside), out_coords [n][max heavy atoms][3]
 * (may be NULL; rows past a pose's own heavy-atom count are 0). */
int sg_refine(sg_engine* e, int receptor_id, const sg_model_desc* models, int nmodels,
              const int* pose_model, int nposes, double* confs, const double cap[3],
              int maxiters, int accurate_line, int early_term,
              double* out_e, double* out_coords);

/* Batched local optimisation (--minimize / --local_only): replaces
 * GpuDocking::minimize_batch (src/gpu/gpu_docking.h:96-107,
 * gpu_docking.cpp:690-742): refine_structure of every pose in FP64 against
 * the direct receptor sum, each pose in its own box (boxes [n][6]: lo xyz,
 * hi xyz, inside the receptor's box; NULL: the receptor's box) with its own
 * BFGS iteration count (maxiters [n]).  confs [n][conf_stride] in/out,
 * out_e [n] (max double if a pose never got inside its box), out_coords
 * [n][coord_stride][3] heavy atoms (may be NULL; rows past a pose's own
 * heavy-atom count are 0). */
int sg_minimize(sg_engine* e, int receptor_id, const sg_model_desc* models, int nmodels,
                const int* pose_model, int nposes, double* confs, int conf_stride,
                const double* boxes, const double cap[3], const int* maxiters,
                int accurate_line, int early_term, double* out_e, double* out_coords,
                int coord_stride);

/* The mixed-precision path's pair schedule for one model, computed on the
 * host (no device needed): chunks of 32 slots, slot = a | b << 8 |
 * type pair << 16 | swap << 25 | intra << 26, empty slots with type pair
 * 0x1ff.  Within a chunk no atom is twice a first (a) or twice a second (b)
 * atom; within each 8-slot quarter the a's are distinct modulo 8 and so are
 * the b's.  *nchunks gets the chunk count; out [cap] gets the slots when
 * cap >= 32 * *nchunks.  No counterpart in the reference (its FP32 kernels
 * gather pair forces per atom, gpu_flatten.cpp:217-235). */
int sg_pair_schedule(const sg_model_desc* m, uint32_t* out, int cap, int* nchunks);

/* Final rescoring of docked poses (finish_docking, src/main/main.cpp:257-282):
 * for every pose, model::eval on the direct receptor sum with the fast
 * table (model.cpp:938-967, non_cache::eval non_cache.cpp:34-91) into
 * out_e, and model::eval_intramolecular (model.cpp:1027-1079) into
 * out_intra, both with terms curled at v (authentic_v in the reference) and
 * the out-of-box penalty at `slope`; FP64, bit-exact with the CPU
 * algorithm.  confs [n][conf_stride]; out_coords [n][coord_stride][3] heavy
 * atoms (may be NULL; rows past a pose's heavy count are 0).  The rescored
 * energy of a pose is then conf_independent(out_e - out_intra of the best
 * pose): see sgh_finish_docking. */
int sg_score(sg_engine* e, int receptor_id, const sg_model_desc* models, int nmodels,
             const int* pose_model, int nposes, const double* confs, int conf_stride,
             const double v[3], double slope, double* out_e, double* out_intra,
             double* out_coords, int coord_stride);

/* ---- batched mixed-precision docking (virtual screening) ---------------
 * Replaces GpuDocking::dock_batch (src/gpu/gpu_docking.h:91-94,
 * gpu_docking.cpp:756): for every ligand job, its Monte Carlo chains,
 * merge_output_containers with min_rmsd 2 (gpu_docking.cpp:576-599), then
 * refine_structure of every pose in FP64 (main.cpp:165-200).  Needs an
 * engine created with SG_PREC_FP32 or SG_PREC_FP32_H16. */
typedef struct sg_ligand_job {
    int model;           /* index into the models array                    */
    int num_chains;      /* independent chains (exhaustiveness)            */
    unsigned num_steps;  /* Monte Carlo steps per chain                    */
    int maxiters;        /* BFGS iterations; 0: sg_mc_params.maxiters      */
    uint64_t seed;       /* request seed (Philox key)                      */
    uint64_t ligand_key; /* names the ligand's random streams: the same
                            (seed, ligand_key) docks the same way alone or
                            inside any batch                              */
} sg_ligand_job;

typedef struct sg_ligand_result {
    int count;           /* poses written, <= num_saved_mins, by energy    */
    double* e;           /* [num_saved_mins]                               */
    double* conf;        /* [num_saved_mins][conf_size]                    */
    double* coords;      /* [num_saved_mins][num_heavy_movable][3]         */
    uint64_t evals;      /* eval_deriv calls of the search (all chains)    */
} sg_ligand_result;

/* refine: 0 skips refine_structure (poses come straight from the merge). */
int sg_dock_batch32(sg_engine* e, int receptor_id, const sg_model_desc* models, int nmodels,
                    const sg_ligand_job* jobs, int njobs, const sg_mc_params* p, int refine,
                    sg_ligand_result* out);

/* sg_dock_batch32 with refine = 0, for callers that must not have device
 * memory allocated or freed while the call runs.  No counterpart in the
 * reference.  A serving loop may have promised the rest of the GPU's memory
 * to requests in flight or to a caching allocator, so an allocation here
 * could fail or fragment it; and cudaFree waits for the whole device to go
 * idle, stalling the caller's other streams.  This call places everything
 * the search kernel writes (its copy of the models, chain and work tables,
 * the queue counter, the chains' result slots) in one fixed 8 MiB array per
 * device that is part of the library's image.  Limits and rules:
 *   - a batch that needs more than the 8 MiB is refused with SG_ERR_ARG
 *     (for example 16 ligands of 50 heavy atoms x 8 chains fit);
 *   - the receptor's maps for the ligands' atom types must already be
 *     built (sg_build_grids), since building them allocates;
 *   - the array is claimed when a mixed-precision engine is created
 *     (sg_create with SG_PREC_FP32 or SG_PREC_FP32_H16): 8 MiB of device
 *     memory per device, held until the process exits.  Engine creation
 *     also loads the search kernel and raises its shared-memory limit, so a
 *     call loads no module and sets no kernel attribute;
 *   - the launch shape is the one sg_dock_batch32 would pick, including a
 *     shape set by sg_set_chains_per_block or sg_autotune32;
 *   - every call reuses the same array, so calls that overlap on one GPU
 *     (two engines, or two host threads) corrupt each other: keep them
 *     apart.
 * Results are the same as sg_dock_batch32's with refine = 0. */
int sg_dock_batch32_noalloc(sg_engine* e, int receptor_id, const sg_model_desc* models, int nmodels,
                            const sg_ligand_job* jobs, int njobs, const sg_mc_params* p,
                            sg_ligand_result* out);

/* The gather bandwidth the search kernel's roofline divides by (no
 * counterpart in the reference): independent random loads of
 * bytes_per_lookup (16: a pair table entry, 32: a packed grid cell) bytes,
 * aligned to their size, over a zero-filled device buffer of
 * working_set_bytes (1 MiB .. 64 GiB) with every SM full; the best of three
 * passes after one that brings the buffer into cache.  *out_gbs gets GB/s
 * (1e9 bytes per second).  Allocates and frees the buffer itself. */
int sg_probe_gather(sg_engine* e, uint64_t working_set_bytes, int bytes_per_lookup, double* out_gbs);

/* --fast's early stop for sg_dock_batch32 (not smina's search; EarlyStop,
 * src/gpu/gpu_kernels.h:45-56, applied as run_monte_carlo does,
 * src/gpu/gpu_kernels_impl.cuh:607-657,740-810): the chains run in phases
 * ending at first / checkpoints, (first + 1) / checkpoints, ... of their
 * steps, each phase resuming exactly where the previous one stopped; after
 * every phase but the last, a ligand whose chains form u >= 2 units of
 * chains_per_unit consecutive chains stops when at least
 * max(2, ceil(fraction * u)) of its units' best energies are within eps of
 * its best.  A ligand that never stops gets the results it gets without
 * early stop, bit for bit.  es == NULL turns it off; the setting stays on
 * the engine for later sg_dock_batch32 calls.  FP32 engines only. */
typedef struct sg_early_stop {
    int checkpoints;      /* phases end at (first + k) / checkpoints (10)     */
    int first;            /* the first check (2)                              */
    double fraction;      /* share of a ligand's units that must agree (0.5)  */
    double eps;           /* kcal/mol within the ligand's best (0.05)         */
    int chains_per_unit;  /* consecutive chains of a job that form a unit
                             (the --fast chain split; 1: every chain)         */
} sg_early_stop;
int sg_set_early_stop(sg_engine* e, const sg_early_stop* es);

/* Timing and launch shape of the last sg_dock_batch32 call. */
int sg_batch_stats(const sg_engine* e, double* mc_ms, double* refine_ms,
                   int* chains_per_block, int* blocks);

/* Work counters of the last sg_dock_batch32 call: eval_deriv calls, grid
 * map lookups (one packed cell each), in-cutoff pair table lookups, and
 * bytes copied host to device and device to host. */
int sg_batch_counters(const sg_engine* e, uint64_t* evals, uint64_t* grid_lookups,
                      uint64_t* pair_lookups, uint64_t* h2d_bytes, uint64_t* d2h_bytes);

/* Chains per block of the search kernel: 1, 2, 4 or 8 (at most 8 warps
 * per block, so 2 with 128 threads per chain), or 0 to pick the shape with
 * the most resident chains per SM (the default; a batch of at most one
 * chain per SM then runs one chain per block).  The chains of one block
 * share one copy of their ligand's model. */
int sg_set_chains_per_block(sg_engine* e, int n);

/* Threads per chain of the batched search (sg_dock_batch32, and the FP32
 * sg_eval / sg_bfgs): 32 (the default), 64 or 128 -- the reference's
 * threads_per_chain (gpu_kernels_impl.cuh:572-605) -- or 0 to pick, per
 * call, the most (128, 64, 32) at which the batch's chains all stay
 * resident at once.  More threads per chain shorten each chain (its grid
 * and pair terms are shared out among the warps) when the device has warps
 * to spare, such as for a lone ligand; they do not raise a full device's
 * throughput.  Results depend on the setting (the order of FP32 additions
 * changes with the team size) but, for a given value, not on the batch or
 * the launch shape; with 0 the value follows the batch's size.  A serving
 * loop (sg_serve_*) reads the setting at each upload; with 0 it picks, per
 * upload, the most at which the work items already on the device and the
 * new batch's all have a block (each result reports its value).  FP64
 * engines ignore it: the plain path runs one warp per chain.
 * sg_threads_per_chain reports the setting and the last batch's value. */
int sg_set_threads_per_chain(sg_engine* e, int threads);
int sg_threads_per_chain(const sg_engine* e, int* configured, int* last_batch);

/* Launch-shape autotuner for the search kernel: runs the given jobs with
 * their step counts scaled by step_fraction (0 < f <= 1, at least one step
 * each; no refinement) once per shape of 8, 4, 2 and 1 chains per block,
 * times each search launch with CUDA events and keeps the fastest shape
 * (as sg_set_chains_per_block would).  evals_per_s[4] (may be null) gets
 * each shape's eval_deriv calls per second, 0 for a shape that cannot run;
 * *chosen the shape kept.  Results of later calls do not depend on the
 * shape.  The reference picks its launch shape (threads per chain) from the
 * occupancy calculator alone: Residency / mc_residency,
 * src/gpu/gpu_kernels.h:70-88. */
int sg_autotune32(sg_engine* e, int receptor_id, const sg_model_desc* models, int nmodels, const sg_ligand_job* jobs,
                  int njobs, const sg_mc_params* p, double step_fraction, double* evals_per_s, int* chosen);

/* ---- serving: a request loop with continuous batching ------------------
 * No counterpart in the reference (its screens are offline batches).
 * Requests (one ligand against one resident receptor) are queued by
 * sg_serve_submit; a worker thread uploads them in small batches as they
 * arrive and publishes their work items (a group of chains of one ligand
 * each) to a ring in device memory.  A resident serving grid takes items
 * from the ring while it runs, so a ligand's chains start as soon as a
 * block is free, whatever batch it came with; ligands of different
 * receptors mix freely.  Blocks that find no work for a while leave, and
 * the worker starts blocks again when items wait and none is free.
 * Admission keeps the device memory held for requests in flight under
 * hbm_budget_bytes.  Each ligand is merged and refined (FP64) as soon as its
 * own chains finish.  A result equals sg_dock_batch32's (refine = 1) for the
 * same (seed, ligand_key), alone or in any mix.  While a server runs, the
 * engine's other entry points must not be called except sg_serve_*. */
typedef struct sg_serve_opts {
    uint64_t hbm_budget_bytes;  /* 0: a quarter of the free device memory   */
    int max_batch_ligands;      /* ligands per upload batch (0: 64)          */
    double max_wait_ms;         /* under light load, how long the oldest
                                   request may wait for others to share its
                                   batch (0: 20 ms)                          */
    int max_inflight_ligands;   /* at most this many ligands on the device;
                                   later requests wait in the server's queue
                                   (0: two per SM, what the device holds at
                                   once with 8 chains per ligand, less 16
                                   kept for refinements)                     */
    int block_smem_bytes;       /* dynamic shared memory of every search
                                   launch's blocks (0: the most that keeps two
                                   blocks per SM)                            */
} sg_serve_opts;

typedef struct sg_serve_done {
    uint64_t ticket;
    int status;                /* SG_OK, or the error that ended the request */
    int count;                 /* poses (merged, refined, by energy)        */
    int conf_size, num_heavy;  /* sizes for sg_serve_fetch's arrays         */
    uint64_t evals;            /* eval_deriv calls of the search            */
    double latency_ms;         /* submit to result                          */
    uint64_t launch;           /* the upload batch it came with (1, 2, ...) */
    uint64_t device_start_ns;  /* device clock (%globaltimer, ns) when its
                                  first chain started ...                   */
    uint64_t device_end_ns;    /* ... and when its last chain ended; two
                                  requests of different launches whose
                                  spans overlap were on the device at once  */
    double queue_ms;           /* submit to upload (waiting in the server's
                                  queue)                                    */
    double searched_ms;        /* submit to the worker seeing its chains
                                  done (then merge and FP64 refinement)     */
    int threads_per_chain;     /* its search's threads per chain (32, 64,
                                  128): the engine's sg_set_threads_per_chain
                                  setting at its upload, or with 0 there the
                                  most at which everything on the device
                                  then had a block at once                  */
    int pad_;
} sg_serve_done;

int sg_serve_start(sg_engine* e, const sg_serve_opts* opts);
/* job->model is ignored; the model is copied, so the caller may free it. */
int sg_serve_submit(sg_engine* e, int receptor_id, const sg_model_desc* m, const sg_ligand_job* job,
                    const sg_mc_params* p, uint64_t* ticket);
/* Up to max finished requests (waits up to wait_ms for the first one). */
int sg_serve_poll(sg_engine* e, sg_serve_done* out, int max, int wait_ms, int* nout);
/* Copies a finished request's poses (arrays sized by its sg_serve_done)
 * and forgets the ticket. */
int sg_serve_fetch(sg_engine* e, uint64_t ticket, sg_ligand_result* out);
int sg_serve_stats(const sg_engine* e, int* queued, int* inflight_ligands, uint64_t* inflight_bytes);
/* Finishes every submitted request, then stops the worker. */
int sg_serve_stop(sg_engine* e);

#ifdef __cplusplus
}
#endif
#endif /* SMINA_B200_H */
