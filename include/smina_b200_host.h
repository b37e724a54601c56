/*
 * smina_b200_host.h - C ABI of the host library that prepares inputs for the
 * engine (include/smina_b200.h): PDBQT ligand models, receptors, pair tables,
 * boxes, search parameters and chain seeds.
 *
 * Reference functions restated (paths inside the reference project):
 *   sgh_model_from_pdbqt   parse_ligand_stream_pdbqt + model::initialize
 *                          src/lib/parse_pdbqt.cpp:209-353,487-495,
 *                          src/lib/model.cpp:448-636
 *   sgh_tables_create      precalculate_linear(weighted_terms, factor)
 *                          src/lib/precalculate.h:187-308, src/main/main.cpp:1408-1421;
 *                          builtin / custom scoring src/lib/builtinscoring.cpp:63-105,
 *                          src/lib/custom_terms.cpp:56-71
 *   sgh_make_box           grid_dims from center/size src/main/main.cpp:801-809
 *   sgh_search_params      setup_search src/main/main.cpp:513-529
 *   sgh_seed_chains        parallel_mc task seeding src/lib/parallel_mc.cpp:80-98 and
 *                          conf::randomize src/lib/conf.h:355-360
 *   sgh_make_receptor /    synthetic inputs (no counterpart: the reference reads
 *   sgh_make_ligand_pdbqt  files through OpenBabel)
 */
#ifndef SMINA_B200_HOST_H
#define SMINA_B200_HOST_H

#include <stdint.h>
#include "smina_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sgh_model sgh_model;
typedef struct sgh_receptor sgh_receptor;
typedef struct sgh_tables sgh_tables;

const char* sgh_last_error(void);

int  sgh_model_from_pdbqt(const char* text, sgh_model** out);
/* SDF / MOL (V2000 or V3000) ligands, the reference's OpenBabel route
 * (molgetter.cpp:103-125 with SminaConverter.cpp:87-130 and
 * PDBQTUtilities.cpp:50-627) without OpenBabel: record `index` (0-based;
 * records end at "$$$$") typed, charged (Gasteiger) and cut into a
 * torsion tree, written as PDBQT, and read by the PDBQT reader.
 * add_hydrogens: add the hydrogens N, O and S lack (the reference's
 * default adds them).  sgh_sdf_count returns the records in the text (or
 * -1); sgh_pdbqt_from_sdf returns 0, -1 on error, or the buffer size
 * needed. */
int  sgh_sdf_count(const char* text);
/* Byte offsets of the records (up to max written; returns the count, or
 * -1).  For a large file, pass text + offsets[k] with index 0: a call then
 * reads only that record, where index k scans the k records before it. */
int  sgh_sdf_offsets(const char* text, int64_t* offsets, int max);
int  sgh_pdbqt_from_sdf(const char* text, int index, int add_hydrogens, char* buf, int buflen);
int  sgh_model_from_sdf(const char* text, int index, int add_hydrogens, sgh_model** out);
/* A ligand plus the receptor's flexible residues (smina --flex; flex PDBQT
 * with BEGIN_RES/END_RES blocks, parse_pdbqt.cpp:412-437), combined as
 * model::append does (model.cpp:302-347). */
int  sgh_model_from_pdbqt_flex(const char* ligand_text, const char* flex_text, sgh_model** out);
void sgh_model_free(sgh_model* m);
/* descriptor pointing into the model (valid while the model lives) */
int  sgh_model_desc(const sgh_model* m, sg_model_desc* out);
int  sgh_model_heavy(const sgh_model* m);
int  sgh_model_torsdof(const sgh_model* m);
/* conf_independent_inputs of the model's ligand (terms.cpp:83-120):
 * out[7] = num_tors, num_rotors, num_heavy_atoms, num_hydrophobic_atoms,
 * ligand_max_num_h_bonds, num_ligands, ligand_lengths_sum */
int  sgh_model_conf_independent_inputs(const sgh_model* m, double out[7]);

int  sgh_make_receptor(int heavy_atoms, uint64_t seed, const double center[3], double cavity_radius,
                       sgh_receptor** out);
void sgh_receptor_free(sgh_receptor* r);
int  sgh_receptor_desc(sgh_receptor* r, sg_receptor_desc* out);
/* returns 0, or the buffer size needed */
int  sgh_receptor_pdbqt(const sgh_receptor* r, char* buf, int buflen);
/* returns 0, -1 on error, or the buffer size needed */
int  sgh_make_ligand_pdbqt(int heavy, int rotors, uint64_t seed, const double center[3], char* buf, int buflen);
/* `residues` synthetic flexible side chains (2..4 chi torsions each) with
 * their CA on a shell of radius `shell` (0: 9 A) around `center`.  Like
 * sgh_make_ligand_pdbqt: returns the size needed when buflen is too small,
 * 0 when written, -1 on error. */
int  sgh_make_flex_pdbqt(int residues, uint64_t seed, const double center[3], double shell, char* buf, int buflen);

/* builtin_name: "vina"/"default", "vinardo", "dkoes_scoring", "dkoes_scoring_old", "dkoes_fast",
 * "ad4_scoring"; custom_text (if non-empty) takes precedence */
int  sgh_tables_create(const char* builtin_name, const char* custom_text, double factor, sgh_tables** out);
void sgh_tables_free(sgh_tables* t);
int  sgh_tables_desc(const sgh_tables* t, sg_tables_desc* out);
/* weighted_terms::conf_independent (weighted_terms.cpp:74-80): the scoring
 * function's conf-independent terms (num_tors_div, ...) applied to x in
 * order; inputs as sgh_model_conf_independent_inputs gives them */
int  sgh_tables_conf_independent(const sgh_tables* t, const double inputs[7], double x, double* out);
/* finish_docking (src/main/main.cpp:257-324) for one ligand: poses sorted by
 * their refined energy; every pose not at max energy rescored as
 * conf_independent(e_total - e_intra of the best pose) with e_total and
 * e_intra from sg_score; sorted again; remove_redundant at out_min_rmsd over
 * the heavy-atom coords [n][heavy][3]; at most num_modes poses, none at max
 * energy or more than energy_range above the best.  out_index / out_e get
 * the kept poses (indices into the inputs) and their final energies;
 * *out_count how many. */
int  sgh_finish_docking(const sgh_tables* t, const double inputs[7], int n, const double* e_refined,
                        const double* e_total, const double* e_intra, const double* coords, int heavy,
                        double out_min_rmsd, int num_modes, double energy_range, int* out_index, double* out_e,
                        int* out_count);

int  sgh_make_box(const double center[3], const double size[3], double granularity, sg_grid_dims* out);
int  sgh_search_params(const sgh_model* m, int num_modes, sg_mc_params* out);
/* --fast's chain split and step fraction (not smina's search; the
 * reference's GpuSettings::chain_split / step_fraction and dock_batch's
 * budget, src/gpu/gpu_docking.cpp:87-112,168-220): every search task
 * becomes *split chains of *chain_steps steps each.  chain_split 0 picks the
 * split from the tasks docked at once and the device's resident chain
 * capacity (the largest power of two from 32 down to 4 within 4 waves);
 * step_fraction 0 picks 1/2 for splits 4..31, else 1; budget > 0 (a
 * first pass) overrides the fraction.  *fraction (may be NULL) gets the
 * fraction used.  Host arithmetic only. */
int  sgh_fast_chains(long long tasks, long long capacity, int chain_split, double step_fraction, double budget,
                     unsigned steps, int* split, unsigned* chain_steps, double* fraction);
/* confs [tasks][conf_size], mt [tasks][625] */
int  sgh_seed_chains(const sgh_model* m, int seed, int tasks, const sg_grid_dims* box, double* confs, uint32_t* mt);

/* merge_output_containers (parallel_mc.cpp:64-76): the chains' sorted
 * containers merged in chain order with the given min_rmsd (2 in
 * parallel_mc) into at most max_size poses; out arrays sized max_size. */
int  sgh_merge_chains(const sg_chain_result* chains, int nchains, int conf_size, int nheavy, double min_rmsd,
                      int max_size, double* out_e, double* out_conf, double* out_coords, int* out_count);

#ifdef __cplusplus
}
#endif
#endif
