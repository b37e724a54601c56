"""Python binding of the B200 docking engine (ctypes over the C ABI).

The compute lives in ``libsmina_b200.so`` (CUDA kernels for sm_100a plus the
C++ host library); this module only marshals numpy arrays into the flat
descriptors of ``include/smina_b200.h`` / ``include/smina_b200_host.h``.
There is no CPU fallback: :func:`load` raises if the library is missing.

Reference interfaces mirrored (paths inside the reference project):
  Engine.eval        model::eval_deriv                 src/lib/model.cpp:969-985
  Engine.dock        monte_carlo::operator() per chain  src/lib/monte_carlo.cpp:95-130
  Engine.dock_batch  GpuDocking::dock_batch            src/gpu/gpu_docking.cpp:756
  Engine.refine      refine_structure                  src/main/main.cpp:165-190
  Engine.grid        cache::populate                   src/lib/cache.cpp:116-206
  GpuDocking         gpusmina::GpuDocking              src/gpu/gpu_docking.h:51-114
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libsmina_b200.so")

SG_OK, SG_ERR_ARG, SG_ERR_CUDA, SG_ERR_NOMEM, SG_ERR_OVERLAP, SG_ERR_TIMEOUT, SG_ERR_STATE = range(7)
PREC_FP64, PREC_FP32, PREC_FP32_H16 = 0, 1, 2
NUM_TYPES = 27

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_up = C.POINTER(C.c_uint32)


class GridDims(C.Structure):
    _fields_ = [("begin", C.c_double * 3), ("end", C.c_double * 3), ("n", C.c_int * 3)]


class TablesDesc(C.Structure):
    _fields_ = [("num_types", C.c_int), ("num_components", C.c_int), ("n", C.c_int),
                ("factor", C.c_double), ("cutoff_sqr", C.c_double), ("smooth", _dp), ("fast", _dp)]


class ReceptorDesc(C.Structure):
    _fields_ = [("num_atoms", C.c_int), ("coords", _dp), ("type", _ip), ("charge", _dp)]


class ModelDesc(C.Structure):
    _fields_ = [("num_atoms", C.c_int), ("num_movable", C.c_int), ("num_frames", C.c_int),
                ("num_ligands", C.c_int), ("num_flex", C.c_int), ("conf_size", C.c_int), ("dof", C.c_int),
                ("num_pairs", C.c_int), ("num_other_pairs", C.c_int),
                ("lig_pair_end", _ip), ("ligand_atom_begin", _ip), ("ligand_atom_end", _ip), ("ligand_root", _ip),
                ("atom_type", _ip), ("atom_charge", _dp), ("atom_local", _dp), ("atom_lab", _dp),
                ("frame_kind", _ip), ("frame_parent", _ip), ("frame_begin", _ip), ("frame_end", _ip),
                ("frame_conf", _ip), ("frame_dof", _ip), ("frame_origin", _dp), ("frame_axis", _dp),
                ("frame_init_origin", _dp), ("pairs", _ip)]


class MCParams(C.Structure):
    _fields_ = [("num_steps", C.c_uint), ("temperature", C.c_double), ("mutation_amplitude", C.c_double),
                ("min_rmsd", C.c_double), ("num_saved_mins", C.c_int), ("hunt_cap", C.c_double * 3),
                ("authentic_v", C.c_double * 3), ("maxiters", C.c_int), ("accurate_line", C.c_int),
                ("early_term", C.c_int), ("cache_slope", C.c_double), ("visited", C.c_int)]


class ChainInput(C.Structure):
    _fields_ = [("model", C.c_int), ("num_steps", C.c_uint), ("conf", _dp), ("mt", _up), ("maxiters", C.c_int)]


class ChainResult(C.Structure):
    _fields_ = [("count", C.c_int), ("e", _dp), ("conf", _dp), ("coords", _dp), ("evals", C.c_uint64)]


class LigandJob(C.Structure):
    _fields_ = [("model", C.c_int), ("num_chains", C.c_int), ("num_steps", C.c_uint), ("maxiters", C.c_int),
                ("seed", C.c_uint64), ("ligand_key", C.c_uint64)]


class LigandResult(C.Structure):
    _fields_ = [("count", C.c_int), ("e", _dp), ("conf", _dp), ("coords", _dp), ("evals", C.c_uint64)]


class EarlyStop(C.Structure):
    _fields_ = [("checkpoints", C.c_int), ("first", C.c_int), ("fraction", C.c_double), ("eps", C.c_double),
                ("chains_per_unit", C.c_int)]


class ServeOpts(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_batch_ligands", C.c_int), ("max_wait_ms", C.c_double),
                ("max_inflight_ligands", C.c_int), ("block_smem_bytes", C.c_int)]


class ServeDone(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("status", C.c_int), ("count", C.c_int), ("conf_size", C.c_int),
                ("num_heavy", C.c_int), ("evals", C.c_uint64), ("latency_ms", C.c_double), ("launch", C.c_uint64),
                ("device_start_ns", C.c_uint64), ("device_end_ns", C.c_uint64), ("queue_ms", C.c_double),
                ("searched_ms", C.c_double), ("threads_per_chain", C.c_int), ("pad_", C.c_int)]


_lib = None


def load(path: str = LIB_PATH):
    """Load libsmina_b200.so; raises OSError if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise OSError(f"{path} missing: run __graft_entry__.build() first")
        _lib = C.CDLL(path)
        _declare(_lib)
    return _lib


def _declare(L):
    vp = C.c_void_p
    L.sgh_last_error.restype = C.c_char_p
    L.sg_last_error.restype = C.c_char_p
    L.sg_last_error.argtypes = [vp]
    for name, args in {
        "sgh_model_from_pdbqt": [C.c_char_p, C.POINTER(vp)],
        "sgh_sdf_count": [C.c_char_p],
        "sgh_sdf_offsets": [C.c_char_p, C.POINTER(C.c_int64), C.c_int],
        "sgh_pdbqt_from_sdf": [C.c_char_p, C.c_int, C.c_int, C.c_char_p, C.c_int],
        "sgh_model_from_sdf": [C.c_char_p, C.c_int, C.c_int, C.POINTER(vp)],
        "sgh_model_desc": [vp, C.POINTER(ModelDesc)],
        "sgh_model_heavy": [vp], "sgh_model_torsdof": [vp],
        "sgh_make_receptor": [C.c_int, C.c_uint64, C.c_double * 3, C.c_double, C.POINTER(vp)],
        "sgh_receptor_desc": [vp, C.POINTER(ReceptorDesc)],
        "sgh_receptor_pdbqt": [vp, C.c_char_p, C.c_int],
        "sgh_make_ligand_pdbqt": [C.c_int, C.c_int, C.c_uint64, C.c_double * 3, C.c_char_p, C.c_int],
        "sgh_make_flex_pdbqt": [C.c_int, C.c_uint64, C.c_double * 3, C.c_double, C.c_char_p, C.c_int],
        "sgh_model_from_pdbqt_flex": [C.c_char_p, C.c_char_p, C.POINTER(vp)],
        "sgh_tables_create": [C.c_char_p, C.c_char_p, C.c_double, C.POINTER(vp)],
        "sgh_tables_desc": [vp, C.POINTER(TablesDesc)],
        "sgh_make_box": [C.c_double * 3, C.c_double * 3, C.c_double, C.POINTER(GridDims)],
        "sgh_search_params": [vp, C.c_int, C.POINTER(MCParams)],
        "sgh_seed_chains": [vp, C.c_int, C.c_int, C.POINTER(GridDims), _dp, _up],
        "sgh_fast_chains": [C.c_longlong, C.c_longlong, C.c_int, C.c_double, C.c_double, C.c_uint, _ip,
                            C.POINTER(C.c_uint), _dp],
        "sgh_merge_chains": [C.POINTER(ChainResult), C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, _dp, _dp, _dp,
                             _ip],
        "sg_create": [C.c_int, C.c_int, C.POINTER(vp)],
        "sg_device_info": [vp, _ip, _ip, _ip],
        "sg_set_tables": [vp, C.POINTER(TablesDesc)],
        "sg_set_receptor": [vp, C.c_int, C.POINTER(ReceptorDesc), C.POINTER(GridDims)],
        "sg_build_grids": [vp, C.c_int, _ip, C.c_int],
        "sg_get_grid": [vp, C.c_int, C.c_int, _dp, _dp],
        "sg_drop_receptor": [vp, C.c_int],
        "sg_set_user_grid": [vp, C.c_int, C.POINTER(GridDims), _dp, C.c_double],
        "sg_eval": [vp, C.c_int, C.POINTER(ModelDesc), C.c_int, _dp, C.c_double * 3, C.c_double, _dp, _dp, _dp],
        "sg_eval_direct": [vp, C.c_int, C.POINTER(ModelDesc), C.c_int, _dp, C.c_double * 3, C.c_double, _dp, _dp],
        "sg_dock": [vp, C.c_int, C.POINTER(ModelDesc), C.c_int, C.POINTER(ChainInput), C.c_int,
                    C.POINTER(MCParams), C.POINTER(ChainResult)],
        "sg_refine": [vp, C.c_int, C.POINTER(ModelDesc), C.c_int, _ip, C.c_int, _dp, C.c_double * 3,
                      C.c_int, C.c_int, C.c_int, _dp, _dp],
        "sg_bfgs": [vp, C.c_int, C.POINTER(ModelDesc), C.c_int, _dp, C.c_double * 3, C.c_double, C.c_int, C.c_int,
                    C.c_int, _dp],
        "sg_score": [vp, C.c_int, C.POINTER(ModelDesc), C.c_int, _ip, C.c_int, _dp, C.c_int, C.c_double * 3, C.c_double,
                     _dp, _dp, _dp, C.c_int],
        "sg_pair_schedule": [C.POINTER(ModelDesc), _up, C.c_int, _ip],
        "sgh_model_conf_independent_inputs": [vp, _dp],
        "sgh_tables_conf_independent": [vp, _dp, C.c_double, _dp],
        "sgh_finish_docking": [vp, _dp, C.c_int, _dp, _dp, _dp, _dp, C.c_int, C.c_double, C.c_int, C.c_double, _ip, _dp,
                               _ip],
        "sg_minimize": [vp, C.c_int, C.POINTER(ModelDesc), C.c_int, _ip, C.c_int, _dp, C.c_int, _dp, C.c_double * 3,
                        _ip, C.c_int, C.c_int, _dp, _dp, C.c_int],
        "sg_dock_batch32": [vp, C.c_int, C.POINTER(ModelDesc), C.c_int, C.POINTER(LigandJob), C.c_int,
                            C.POINTER(MCParams), C.c_int, C.POINTER(LigandResult)],
        "sg_dock_batch32_noalloc": [vp, C.c_int, C.POINTER(ModelDesc), C.c_int, C.POINTER(LigandJob), C.c_int,
                                    C.POINTER(MCParams), C.POINTER(LigandResult)],
        "sg_batch_stats": [vp, _dp, _dp, _ip, _ip],
        "sg_batch_counters": [vp] + [C.POINTER(C.c_uint64)] * 5,
        "sg_set_chains_per_block": [vp, C.c_int],
        "sg_set_threads_per_chain": [vp, C.c_int],
        "sg_threads_per_chain": [vp, _ip, _ip],
        "sg_set_early_stop": [vp, C.c_void_p],
        "sg_autotune32": [vp, C.c_int, C.POINTER(ModelDesc), C.c_int, C.POINTER(LigandJob), C.c_int,
                          C.POINTER(MCParams), C.c_double, _dp, _ip],
        "sg_serve_start": [vp, C.POINTER(ServeOpts)],
        "sg_serve_submit": [vp, C.c_int, C.POINTER(ModelDesc), C.POINTER(LigandJob), C.POINTER(MCParams),
                            C.POINTER(C.c_uint64)],
        "sg_serve_poll": [vp, C.POINTER(ServeDone), C.c_int, C.c_int, _ip],
        "sg_serve_fetch": [vp, C.c_uint64, C.POINTER(LigandResult)],
        "sg_serve_stats": [vp, _ip, _ip, C.POINTER(C.c_uint64)],
        "sg_serve_stop": [vp],
        "sg_probe_gather": [vp, C.c_uint64, C.c_int, C.POINTER(C.c_double)],
    }.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    L.sg_destroy.argtypes = [vp]
    L.sg_destroy.restype = None
    for name in ("sgh_model_free", "sgh_receptor_free", "sgh_tables_free"):
        getattr(L, name).argtypes = [vp]
        getattr(L, name).restype = None


def dptr(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def uptr(a):
    return a.ctypes.data_as(_up) if a is not None else None


def vec3(x):
    return (C.c_double * 3)(*[float(v) for v in x])


class SminaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _check_host(rc):
    if rc != 0:
        raise SminaError(rc, load().sgh_last_error().decode())


# ---- host-side objects -------------------------------------------------------------
class Model:
    """A docking model (ligand torsion tree, pairs) read from PDBQT text; with
    ``flex`` (flex PDBQT text) the receptor's flexible residues join it."""

    def __init__(self, pdbqt: str, flex: str | None = None):
        L = load()
        h = C.c_void_p()
        if flex is None:
            _check_host(L.sgh_model_from_pdbqt(pdbqt.encode(), C.byref(h)))
        else:
            _check_host(L.sgh_model_from_pdbqt_flex(pdbqt.encode(), flex.encode(), C.byref(h)))
        self._h = h
        self.pdbqt = pdbqt
        self.desc = ModelDesc()
        L.sgh_model_desc(h, C.byref(self.desc))
        self.heavy = L.sgh_model_heavy(h)
        self.torsdof = L.sgh_model_torsdof(h)

    @property
    def conf_size(self):
        return self.desc.conf_size

    @property
    def dof(self):
        return self.desc.dof

    @property
    def num_movable(self):
        return self.desc.num_movable

    def types(self):
        return [self.desc.atom_type[i] for i in range(self.desc.num_movable)]

    def search_params(self, num_modes=9) -> MCParams:
        p = MCParams()
        load().sgh_search_params(self._h, num_modes, C.byref(p))
        return p

    def pair_schedule(self):
        """The mixed-precision path's pair chunks (sg_pair_schedule): uint32 [nchunks][32]."""
        n = C.c_int()
        L = load()
        _check_host(L.sg_pair_schedule(C.byref(self.desc), None, 0, C.byref(n)))
        out = np.zeros(32 * n.value, dtype=np.uint32)
        _check_host(L.sg_pair_schedule(C.byref(self.desc), uptr(out), len(out), C.byref(n)))
        return out.reshape(n.value, 32)

    def conf_independent_inputs(self):
        """num_tors, num_rotors, num_heavy_atoms, num_hydrophobic_atoms,
        ligand_max_num_h_bonds, num_ligands, ligand_lengths_sum (terms.cpp:83-120)."""
        out = np.zeros(7)
        _check_host(load().sgh_model_conf_independent_inputs(self._h, dptr(out)))
        return out

    def seed_chains(self, seed: int, tasks: int, box: GridDims):
        confs = np.zeros((tasks, self.conf_size))
        mt = np.zeros((tasks, 625), dtype=np.uint32)
        _check_host(load().sgh_seed_chains(self._h, seed, tasks, C.byref(box), dptr(confs), uptr(mt)))
        return confs, mt

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.sgh_model_free(self._h)
            self._h = None


class Receptor:
    def __init__(self, heavy_atoms: int, seed: int, center=(0.0, 0.0, 0.0), cavity_radius=8.0):
        L = load()
        h = C.c_void_p()
        _check_host(L.sgh_make_receptor(heavy_atoms, seed, vec3(center), cavity_radius, C.byref(h)))
        self._h = h
        self.desc = ReceptorDesc()
        L.sgh_receptor_desc(h, C.byref(self.desc))
        n = self.desc.num_atoms
        self.coords = np.ctypeslib.as_array(self.desc.coords, shape=(n, 3)).copy()
        self.types = np.ctypeslib.as_array(self.desc.type, shape=(n,)).copy()

    def pdbqt(self) -> str:
        L = load()
        need = L.sgh_receptor_pdbqt(self._h, None, 0)
        buf = C.create_string_buffer(need)
        L.sgh_receptor_pdbqt(self._h, buf, need)
        return buf.value.decode()

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.sgh_receptor_free(self._h)
            self._h = None


def sdf_count(text: str) -> int:
    """Records in SDF text (sgh_sdf_count)."""
    L = load()
    n = L.sgh_sdf_count(text.encode())
    if n < 0:
        raise SminaError(SG_ERR_ARG, L.sgh_last_error().decode())
    return n


def sdf_records(text: str) -> list:
    """The records of SDF text, each as its own text (sgh_sdf_offsets); pass
    them one at a time to ``pdbqt_from_sdf`` for a large file."""
    L = load()
    raw = text.encode()
    n = L.sgh_sdf_offsets(raw, None, 0)
    if n < 0:
        raise SminaError(SG_ERR_ARG, L.sgh_last_error().decode())
    off = (C.c_int64 * max(n, 1))()
    L.sgh_sdf_offsets(raw, off, n)
    ends = list(off[1:n]) + [len(raw)]
    return [raw[off[k]:ends[k]].decode() for k in range(n)]


def pdbqt_from_sdf(text: str, index: int = 0, add_hydrogens: bool = True) -> str:
    """SDF record ``index`` as the PDBQT the reference's converter writes
    (sgh_pdbqt_from_sdf); ``Model(pdbqt_from_sdf(...))`` docks it."""
    L = load()
    need = L.sgh_pdbqt_from_sdf(text.encode(), index, int(add_hydrogens), None, 0)
    if need < 0:
        raise SminaError(SG_ERR_ARG, L.sgh_last_error().decode())
    buf = C.create_string_buffer(need)
    L.sgh_pdbqt_from_sdf(text.encode(), index, int(add_hydrogens), buf, need)
    return buf.value.decode()


def make_ligand_pdbqt(heavy: int, rotors: int, seed: int, center=(0.0, 0.0, 0.0)) -> str:
    L = load()
    need = L.sgh_make_ligand_pdbqt(heavy, rotors, seed, vec3(center), None, 0)
    if need < 0:
        raise SminaError(SG_ERR_ARG, L.sgh_last_error().decode())
    buf = C.create_string_buffer(need)
    L.sgh_make_ligand_pdbqt(heavy, rotors, seed, vec3(center), buf, need)
    return buf.value.decode()


def make_flex_pdbqt(residues: int, seed: int, center=(0.0, 0.0, 0.0), shell=9.0) -> str:
    L = load()
    need = L.sgh_make_flex_pdbqt(residues, seed, vec3(center), shell, None, 0)
    if need < 0:
        raise SminaError(SG_ERR_ARG, L.sgh_last_error().decode())
    buf = C.create_string_buffer(need)
    L.sgh_make_flex_pdbqt(residues, seed, vec3(center), shell, buf, need)
    return buf.value.decode()


class Tables:
    """precalculate_linear tables for a builtin or custom scoring function."""

    def __init__(self, builtin: str = "vina", custom_text: str | None = None, factor: float = 32.0):
        L = load()
        h = C.c_void_p()
        _check_host(L.sgh_tables_create(builtin.encode(), (custom_text or "").encode(), factor, C.byref(h)))
        self._h = h
        self.desc = TablesDesc()
        L.sgh_tables_desc(h, C.byref(self.desc))

    def conf_independent(self, inputs, x: float) -> float:
        """The scoring function's conf-independent terms applied to x."""
        out = C.c_double()
        _check_host(load().sgh_tables_conf_independent(self._h, dptr(np.ascontiguousarray(inputs, dtype=np.float64)),
                                                         float(x), C.byref(out)))
        return out.value

    def finish_docking(self, inputs, e_refined, e_total, e_intra, coords, out_min_rmsd=1.0, num_modes=9,
                       energy_range=3.0):
        """finish_docking for one ligand's refined poses (sgh_finish_docking):
        returns (indices of the kept poses, their final energies)."""
        er = np.ascontiguousarray(e_refined, dtype=np.float64)
        n = len(er)
        xyz = np.ascontiguousarray(coords, dtype=np.float64).reshape(n, -1, 3)
        idx, e, cnt = np.zeros(max(n, 1), np.int32), np.zeros(max(n, 1)), C.c_int()
        _check_host(load().sgh_finish_docking(self._h, dptr(np.ascontiguousarray(inputs, dtype=np.float64)), n,
                                              dptr(er), dptr(np.ascontiguousarray(e_total, dtype=np.float64)),
                                              dptr(np.ascontiguousarray(e_intra, dtype=np.float64)), dptr(xyz),
                                              xyz.shape[1], out_min_rmsd, num_modes, energy_range, iptr(idx), dptr(e),
                                              C.byref(cnt)))
        return idx[:cnt.value].copy(), e[:cnt.value].copy()

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.sgh_tables_free(self._h)
            self._h = None


def make_box(center, size, granularity=0.375) -> GridDims:
    gd = GridDims()
    load().sgh_make_box(vec3(center), vec3(size), granularity, C.byref(gd))
    return gd


def grid_points(gd: GridDims) -> int:
    return (gd.n[0] + 1) * (gd.n[1] + 1) * (gd.n[2] + 1)


@dataclass
class ChainBatch:
    """Owns the arrays behind an array of sg_chain_input / sg_chain_result."""
    inputs: object
    results: object
    keep: list = field(default_factory=list)
    e: np.ndarray = None
    conf: np.ndarray = None
    coords: np.ndarray = None
    count: np.ndarray = None


def make_chain_batch(models, model_of_chain, confs, mts, steps, num_saved, heavy_of_model, maxiters=None):
    n = len(model_of_chain)
    ins = (ChainInput * n)()
    outs = (ChainResult * n)()
    keep = []
    max_conf = max(m.conf_size for m in models)
    max_heavy = max(heavy_of_model)
    e = np.zeros((n, num_saved))
    conf = np.zeros((n, num_saved, max_conf))
    coords = np.zeros((n, num_saved, max_heavy, 3))
    for k in range(n):
        c = np.ascontiguousarray(confs[k], dtype=np.float64)
        m = np.ascontiguousarray(mts[k], dtype=np.uint32)
        keep += [c, m]
        ins[k].model = int(model_of_chain[k])
        ins[k].num_steps = int(steps[k] if hasattr(steps, "__len__") else steps)
        ins[k].maxiters = int(maxiters[k]) if maxiters is not None else 0
        ins[k].conf = dptr(c)
        ins[k].mt = uptr(m)
        outs[k].e = e[k].ctypes.data_as(_dp)
        outs[k].conf = conf[k].ctypes.data_as(_dp)
        outs[k].coords = coords[k].ctypes.data_as(_dp)
    return ChainBatch(ins, outs, keep, e, conf, coords)


def fast_chains(tasks, capacity, chain_split=0, step_fraction=0.0, budget=0.0, steps=1):
    """sgh_fast_chains: (split, steps per chain, fraction) of --fast's chain
    split for `tasks` search tasks on a device holding `capacity` chains."""
    sp, st, fr = C.c_int(), C.c_uint(), C.c_double()
    _check_host(load().sgh_fast_chains(int(tasks), int(capacity), int(chain_split), float(step_fraction),
                                       float(budget), int(steps), C.byref(sp), C.byref(st), C.byref(fr)))
    return sp.value, st.value, fr.value


def fast_jobs(models, num_tasks, seed, capacity, chain_split=0, step_fraction=0.0, budget=0.0, key_base=0,
              num_modes=9):
    """LigandJobs of the reference's --fast search (not smina's): every
    ligand's num_tasks tasks become `split` chains each, with the steps
    sgh_fast_chains plans for all the screen's tasks on a device holding
    `capacity` chains; BFGS iterations stay smina's."""
    tasks = num_tasks * len(models)
    jobs = []
    for k, m in enumerate(models):
        p = m.search_params(num_modes)
        split, steps, _ = fast_chains(tasks, capacity, chain_split, step_fraction, budget, p.num_steps)
        jobs.append(LigandJob(model=k, num_chains=num_tasks * split, num_steps=steps, maxiters=p.maxiters, seed=seed,
                              ligand_key=key_base + k))
    return jobs


def merge_chains(batch, model, first=0, n=None, min_rmsd=2.0, max_size=20):
    """merge_output_containers over chains [first, first + n) of a ChainBatch."""
    n = len(batch.count) - first if n is None else n
    e = np.zeros(max_size)
    conf = np.zeros((max_size, model.conf_size))
    xyz = np.zeros((max_size, model.heavy, 3))
    cnt = C.c_int()
    res = C.cast(C.byref(batch.results, first * C.sizeof(ChainResult)), C.POINTER(ChainResult))
    _check_host(load().sgh_merge_chains(res, n, model.conf_size, model.heavy, min_rmsd, max_size, dptr(e), dptr(conf),
                                        dptr(xyz), C.byref(cnt)))
    return e[:cnt.value], conf[:cnt.value], xyz[:cnt.value]


# ---- engine ---------------------------------------------------------------------------
class Engine:
    """One device engine (sg_create).  precision: PREC_FP64 / PREC_FP32 / PREC_FP32_H16."""

    def __init__(self, device: int = 0, precision: int = PREC_FP64):
        L = load()
        h = C.c_void_p()
        rc = L.sg_create(device, precision, C.byref(h))
        if rc != 0:
            raise SminaError(rc, f"sg_create failed on device {device}")
        self._h = h
        self.precision = precision

    def _check(self, rc):
        if rc != 0:
            raise SminaError(rc, load().sg_last_error(self._h).decode())

    def set_tables(self, t: Tables):
        self._check(load().sg_set_tables(self._h, C.byref(t.desc)))

    def set_receptor(self, rid: int, r: Receptor, gd: GridDims):
        self._check(load().sg_set_receptor(self._h, rid, C.byref(r.desc), C.byref(gd)))

    def set_user_grid(self, rid: int, gd, data, cache_slope=1e6):
        """sg_set_user_grid: a user grid (--user_grid) over ``gd``, values x
        fastest; ``data`` None clears it.  Maps built before are dropped."""
        if data is None or gd is None:
            self._ug = None
            self._check(load().sg_set_user_grid(self._h, rid, None, None, cache_slope))
            return
        self._ug = np.ascontiguousarray(data, dtype=np.float64).ravel()
        need = (gd.n[0] + 1) * (gd.n[1] + 1) * (gd.n[2] + 1)
        if self._ug.size != need:
            raise ValueError(f"user grid holds {self._ug.size} values, its box needs {need}")
        self._check(load().sg_set_user_grid(self._h, rid, C.byref(gd), dptr(self._ug), cache_slope))

    def build_grids(self, rid: int, types):
        t = np.ascontiguousarray(sorted(set(int(x) for x in types)), dtype=np.int32)
        self._check(load().sg_build_grids(self._h, rid, iptr(t), len(t)))

    def grid(self, rid: int, typ: int, gd: GridDims, charged=False):
        n = grid_points(gd)
        d = np.zeros(n)
        c = np.zeros(n) if charged else None
        self._check(load().sg_get_grid(self._h, rid, typ, dptr(d), dptr(c)))
        return d, c

    def eval(self, rid, m: Model, confs, v=(10, 10, 10), slope=1e6, coords=False):
        confs = np.ascontiguousarray(confs, dtype=np.float64).reshape(-1, m.conf_size)
        n = len(confs)
        e = np.zeros(n)
        g = np.zeros((n, m.dof))
        xyz = np.zeros((n, m.num_movable, 3)) if coords else None
        self._check(load().sg_eval(self._h, rid, C.byref(m.desc), n, dptr(confs), vec3(v), slope, dptr(e), dptr(g),
                                   dptr(xyz)))
        return (e, g, xyz) if coords else (e, g)

    def eval_direct(self, rid, m: Model, confs, v=(1000, 1000, 1000), slope=10.0):
        confs = np.ascontiguousarray(confs, dtype=np.float64).reshape(-1, m.conf_size)
        n = len(confs)
        e = np.zeros(n)
        g = np.zeros((n, m.dof))
        self._check(load().sg_eval_direct(self._h, rid, C.byref(m.desc), n, dptr(confs), vec3(v), slope, dptr(e),
                                          dptr(g)))
        return e, g

    def bfgs(self, rid, m: Model, confs, v=(10, 10, 10), slope=1e6, maxiters=10, accurate=0, early=0):
        confs = np.ascontiguousarray(confs, dtype=np.float64).reshape(-1, m.conf_size).copy()
        e = np.zeros(len(confs))
        self._check(load().sg_bfgs(self._h, rid, C.byref(m.desc), len(confs), dptr(confs), vec3(v), slope, maxiters,
                                   accurate, early, dptr(e)))
        return confs, e

    def dock(self, rid, models, model_of_chain, confs, mts, params: MCParams, steps=None, maxiters=None):
        """Plain FP64 chains (sg_dock); steps and maxiters may be per chain."""
        descs = (ModelDesc * len(models))(*[m.desc for m in models])
        heavy = [m.heavy for m in models]
        batch = make_chain_batch(models, model_of_chain, confs, mts,
                                 params.num_steps if steps is None else steps, params.num_saved_mins, heavy, maxiters)
        self._check(load().sg_dock(self._h, rid, descs, len(models), batch.inputs, len(model_of_chain),
                                   C.byref(params), batch.results))
        batch.count = np.array([batch.results[k].count for k in range(len(model_of_chain))])
        batch.evals = np.array([batch.results[k].evals for k in range(len(model_of_chain))], dtype=np.uint64)
        return batch

    def refine(self, rid, models, pose_model, confs, cap=(1000, 1000, 1000), maxiters=10, accurate_line=0,
               early_term=0):
        descs = (ModelDesc * len(models))(*[m.desc for m in models])
        pm = np.ascontiguousarray(pose_model, dtype=np.int32)
        confs = np.ascontiguousarray(confs, dtype=np.float64).copy()
        n = len(pm)
        e = np.zeros(n)
        H = max(m.heavy for m in models)
        xyz = np.zeros((n, H, 3))
        self._check(load().sg_refine(self._h, rid, descs, len(models), iptr(pm), n, dptr(confs), vec3(cap), maxiters,
                                     accurate_line, early_term, dptr(e), dptr(xyz)))
        return confs, e, xyz

    def dock_batch(self, rid, models, jobs, params: MCParams, refine=True):
        """Batched mixed-precision docking (sg_dock_batch32).  ``jobs`` is a list
        of :class:`LigandJob`; returns one dict per job with ``e`` [count],
        ``conf`` [count][conf_size], ``coords`` [count][heavy][3], ``evals``."""
        descs = (ModelDesc * len(models))(*[m.desc for m in models])
        J = (LigandJob * len(jobs))(*jobs)
        S = params.num_saved_mins
        bufs = []
        outs = (LigandResult * len(jobs))()
        for k, j in enumerate(jobs):
            m = models[j.model]
            e = np.zeros(S)
            conf = np.zeros((S, m.conf_size))
            xyz = np.zeros((S, m.heavy, 3))
            bufs.append((e, conf, xyz))
            outs[k].e, outs[k].conf, outs[k].coords = dptr(e), dptr(conf), dptr(xyz)
        self._check(load().sg_dock_batch32(self._h, rid, descs, len(models), J, len(jobs), C.byref(params),
                                           1 if refine else 0, outs))
        res = []
        for k, (e, conf, xyz) in enumerate(bufs):
            n = outs[k].count
            res.append({"e": e[:n].copy(), "conf": conf[:n].copy(), "coords": xyz[:n].copy(), "evals": int(outs[k].evals)})
        return res

    def dock_batch_noalloc(self, rid, models, jobs, params: MCParams):
        """The batched search and merge without device allocation inside the
        call (sg_dock_batch32_noalloc); same results as
        ``dock_batch(..., refine=False)``.  For callers that must not have
        memory allocated or freed mid-request; the batch must fit the fixed
        8 MiB scratch array and overlapping calls on one GPU must be avoided."""
        descs = (ModelDesc * len(models))(*[m.desc for m in models])
        J = (LigandJob * len(jobs))(*jobs)
        S = params.num_saved_mins
        bufs = []
        outs = (LigandResult * len(jobs))()
        for k, j in enumerate(jobs):
            m = models[j.model]
            e, conf, xyz = np.zeros(S), np.zeros((S, m.conf_size)), np.zeros((S, m.heavy, 3))
            bufs.append((e, conf, xyz))
            outs[k].e, outs[k].conf, outs[k].coords = dptr(e), dptr(conf), dptr(xyz)
        self._check(load().sg_dock_batch32_noalloc(self._h, rid, descs, len(models), J, len(jobs), C.byref(params),
                                                   outs))
        return [{"e": e[:outs[k].count].copy(), "conf": conf[:outs[k].count].copy(),
                 "coords": xyz[:outs[k].count].copy(), "evals": int(outs[k].evals)}
                for k, (e, conf, xyz) in enumerate(bufs)]

    def device_info(self):
        """sg_device_info: device ordinal, SM count, opt-in shared memory per block."""
        d, sms, smem = C.c_int(), C.c_int(), C.c_int()
        self._check(load().sg_device_info(self._h, C.byref(d), C.byref(sms), C.byref(smem)))
        return {"device": d.value, "num_sms": sms.value, "smem_optin": smem.value}

    def batch_stats(self):
        """Timing and counters of the last dock_batch call."""
        mc, rf = C.c_double(), C.c_double()
        wpb, blocks = C.c_int(), C.c_int()
        self._check(load().sg_batch_stats(self._h, C.byref(mc), C.byref(rf), C.byref(wpb), C.byref(blocks)))
        ctr = [C.c_uint64() for _ in range(5)]
        self._check(load().sg_batch_counters(self._h, *[C.byref(c) for c in ctr]))
        return {"mc_ms": mc.value, "refine_ms": rf.value, "chains_per_block": wpb.value, "blocks": blocks.value,
                "evals": ctr[0].value, "grid_lookups": ctr[1].value, "pair_lookups": ctr[2].value,
                "h2d_bytes": ctr[3].value, "d2h_bytes": ctr[4].value}

    # ---- serving (continuous batching) ----------------------------------------
    def probe_gather(self, working_set_bytes, bytes_per_lookup):
        """GB/s of random gathers of bytes_per_lookup bytes over a working set of that size."""
        g = C.c_double()
        self._check(load().sg_probe_gather(self._h, int(working_set_bytes), int(bytes_per_lookup), C.byref(g)))
        return g.value

    def serve_start(self, hbm_budget_bytes=0, max_batch_ligands=0, max_wait_ms=0.0, max_inflight_ligands=0,
                    block_smem_bytes=0):
        o = ServeOpts(hbm_budget_bytes, max_batch_ligands, max_wait_ms, max_inflight_ligands, block_smem_bytes)
        self._check(load().sg_serve_start(self._h, C.byref(o)))

    def serve_submit(self, rid, m: Model, job: LigandJob, params: MCParams) -> int:
        """Queues one ligand against receptor ``rid``; returns its ticket."""
        t = C.c_uint64()
        self._check(load().sg_serve_submit(self._h, rid, C.byref(m.desc), C.byref(job), C.byref(params), C.byref(t)))
        return t.value

    def serve_poll(self, max_n=256, wait_ms=0, spans=False):
        """Finished requests as (ticket, status, count, latency_ms, evals, conf_size, num_heavy) tuples;
        with spans, each tuple also carries (launch, device_start_ns, device_end_ns, queue_ms, searched_ms,
        threads_per_chain)."""
        buf = (ServeDone * max_n)()
        n = C.c_int()
        self._check(load().sg_serve_poll(self._h, buf, max_n, wait_ms, C.byref(n)))
        out = []
        for i in range(n.value):
            d = buf[i]
            t = (d.ticket, d.status, d.count, d.latency_ms, d.evals, d.conf_size, d.num_heavy)
            out.append(t + (d.launch, d.device_start_ns, d.device_end_ns, d.queue_ms, d.searched_ms,
                            d.threads_per_chain) if spans else t)
        return out

    def serve_fetch(self, ticket, count, conf_size, num_heavy):
        e, conf, xyz = np.zeros(max(count, 1)), np.zeros((max(count, 1), conf_size)), np.zeros((max(count, 1), num_heavy, 3))
        out = LigandResult(0, dptr(e), dptr(conf), dptr(xyz), 0)
        self._check(load().sg_serve_fetch(self._h, ticket, C.byref(out)))
        return {"e": e[:count].copy(), "conf": conf[:count].copy(), "coords": xyz[:count].copy(), "evals": int(out.evals)}

    def serve_stats(self):
        q, n, b = C.c_int(), C.c_int(), C.c_uint64()
        self._check(load().sg_serve_stats(self._h, C.byref(q), C.byref(n), C.byref(b)))
        return {"queued": q.value, "inflight": n.value, "inflight_bytes": b.value}

    def serve_stop(self):
        self._check(load().sg_serve_stop(self._h))

    def set_chains_per_block(self, n: int):
        self._check(load().sg_set_chains_per_block(self._h, n))

    def set_threads_per_chain(self, threads: int):
        """Threads per chain of the batched search and the serving loop: 32, 64, 128, or 0 (by load)."""
        self._check(load().sg_set_threads_per_chain(self._h, threads))

    def threads_per_chain(self):
        """(setting, the last batch's threads per chain)."""
        a, b = C.c_int(), C.c_int()
        self._check(load().sg_threads_per_chain(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_early_stop(self, checkpoints=10, first=2, fraction=0.5, eps=0.05, chains_per_unit=1, off=False):
        """--fast's early stop for later dock_batch calls (sg_set_early_stop); off=True turns it off."""
        if off:
            self._check(load().sg_set_early_stop(self._h, None))
        else:
            es = EarlyStop(checkpoints, first, fraction, eps, chains_per_unit)
            self._check(load().sg_set_early_stop(self._h, C.cast(C.byref(es), C.c_void_p)))

    def autotune(self, rid, models, jobs, params: MCParams, step_fraction=0.01):
        """Times the search at 8, 4, 2 and 1 chains per block on ``jobs`` with
        scaled step counts and keeps the fastest shape (sg_autotune32).
        Returns (chosen, {shape: eval_deriv calls per second})."""
        descs = (ModelDesc * len(models))(*[m.desc for m in models])
        J = (LigandJob * len(jobs))(*jobs)
        rate = np.zeros(4)
        chosen = C.c_int()
        self._check(load().sg_autotune32(self._h, rid, descs, len(models), J, len(jobs), C.byref(params),
                                         float(step_fraction), dptr(rate), C.byref(chosen)))
        return chosen.value, {c: float(v) for c, v in zip((8, 4, 2, 1), rate)}

    def score(self, rid, models, pose_model, confs, v=(1000, 1000, 1000), slope=1e6):
        """finish_docking's energies per pose (sg_score): model::eval on the
        direct receptor sum and model::eval_intramolecular, FP64.  Returns
        (e_total [n], e_intra [n], heavy coords [n][H][3])."""
        descs = (ModelDesc * len(models))(*[m.desc for m in models])
        pm = np.ascontiguousarray(pose_model, dtype=np.int32)
        n = len(pm)
        cs = max(m.conf_size for m in models)
        H = max(m.heavy for m in models)
        c = np.zeros((n, cs))
        src = np.asarray(confs, dtype=np.float64).reshape(n, -1)
        c[:, :src.shape[1]] = src
        e, intra, xyz = np.zeros(n), np.zeros(n), np.zeros((n, H, 3))
        self._check(load().sg_score(self._h, rid, descs, len(models), iptr(pm), n, dptr(c), cs, vec3(v), slope, dptr(e),
                                    dptr(intra), dptr(xyz), H))
        return e, intra, xyz

    def minimize(self, rid, models, pose_model, confs, boxes=None, cap=(1000, 1000, 1000), maxiters=10,
                 accurate_line=0, early_term=0):
        """Batched local optimisation (sg_minimize): each pose refined in FP64 in
        its own box (``boxes`` [n][6] lo xyz, hi xyz; None: the receptor's)."""
        descs = (ModelDesc * len(models))(*[m.desc for m in models])
        pm = np.ascontiguousarray(pose_model, dtype=np.int32)
        n = len(pm)
        cs = max(m.conf_size for m in models)
        H = max(m.heavy for m in models)
        c = np.zeros((n, cs))
        src = np.asarray(confs, dtype=np.float64).reshape(n, -1)
        c[:, :src.shape[1]] = src
        mi = np.ascontiguousarray(np.broadcast_to(np.asarray(maxiters, dtype=np.int32), (n,)))
        bx = None if boxes is None else np.ascontiguousarray(boxes, dtype=np.float64).reshape(n, 6)
        e = np.zeros(n)
        xyz = np.zeros((n, H, 3))
        self._check(load().sg_minimize(self._h, rid, descs, len(models), iptr(pm), n, dptr(c), cs, dptr(bx), vec3(cap),
                                       iptr(mi), accurate_line, early_term, dptr(e), dptr(xyz), H))
        return c, e, xyz

    def close(self):
        if getattr(self, "_h", None):
            load().sg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
