"""ctypes wrapper of the CPU oracle (oracle/liboracle.so) -- the checker.

Test infrastructure only: tests and bench.py's CPU baseline use it to check
and to time; the product never imports it.  The descriptors are the same C
structs the engine takes (include/smina_b200.h).
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
import sys  # noqa: E402

sys.path.insert(0, os.path.join(ROOT, "gpu-smina_b200"))
import smina_b200 as sb  # noqa: E402

ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
        L = C.CDLL(ORACLE_SO)
        vp = C.c_void_p
        L.or_create.restype = vp
        L.or_destroy.argtypes = [vp]
        L.or_last_error.restype = C.c_char_p
        L.or_last_error.argtypes = [vp]
        sig = {
            "or_set_tables": [vp, C.POINTER(sb.TablesDesc)],
            "or_set_receptor": [vp, C.POINTER(sb.ReceptorDesc), C.POINTER(sb.GridDims), C.c_int],
            "or_build_grids": [vp, sb._ip, C.c_int],
            "or_set_user_grid": [vp, C.POINTER(sb.GridDims), sb._dp, C.c_double],
            "or_get_grid": [vp, C.c_int, sb._dp, sb._dp],
            "or_eval": [vp, C.POINTER(sb.ModelDesc), C.c_int, sb._dp, C.c_double * 3, C.c_double, sb._dp, sb._dp, sb._dp],
            "or_eval_direct": [vp, C.POINTER(sb.ModelDesc), C.c_int, sb._dp, C.c_double * 3, C.c_double, sb._dp, sb._dp],
            "or_bfgs": [vp, C.POINTER(sb.ModelDesc), C.c_int, sb._dp, C.c_double * 3, C.c_double, C.c_int, C.c_int,
                        C.c_int, sb._dp],
            "or_dock": [vp, C.POINTER(sb.ModelDesc), C.c_int, C.POINTER(sb.ChainInput), C.c_int,
                        C.POINTER(sb.MCParams), C.POINTER(sb.ChainResult), C.c_int],
            "or_merge": [C.POINTER(sb.ChainResult), C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, sb._dp, sb._dp,
                         sb._dp],
            "or_refine": [vp, C.POINTER(sb.ModelDesc), sb._ip, C.c_int, sb._dp, C.c_double * 3, C.c_int, C.c_int,
                          C.c_int, sb._dp, sb._dp],
            "or_score": [vp, C.POINTER(sb.ModelDesc), sb._ip, C.c_int, sb._dp, C.c_int, C.c_double * 3, C.c_double,
                         sb._dp, sb._dp, sb._dp, C.c_int],
            "or_minimize": [vp, C.POINTER(sb.ModelDesc), sb._ip, C.c_int, sb._dp, C.c_int, sb._dp, C.c_double * 3,
                            sb._ip, C.c_int, C.c_int, sb._dp, sb._dp, C.c_int],
        }
        for k, a in sig.items():
            getattr(L, k).argtypes = a
            getattr(L, k).restype = C.c_int
        L.or_pm_eval.argtypes = [C.c_int, sb._dp, sb._dp, C.c_int]
        L.or_pm_eval.restype = None
        L.or_quat_probe.argtypes = [sb._dp, sb._dp, sb._dp, C.c_int]
        L.or_quat_probe.restype = None
        L.or_mt_probe.argtypes = [C.c_uint32, C.c_int, sb._up, C.c_double, C.c_double, sb._dp, C.c_int, C.c_int, sb._ip]
        L.or_mt_probe.restype = None
        _lib = L
    return _lib


class Oracle:
    def __init__(self, tables, receptor=None, box=None, full_cells=True):
        L = load()
        self.h = L.or_create()
        self.tables = tables
        L.or_set_tables(self.h, C.byref(tables.desc))
        if receptor is not None:
            self.set_receptor(receptor, box, full_cells)

    def _check(self, rc):
        if rc != 0:
            raise sb.SminaError(rc, load().or_last_error(self.h).decode())

    def set_receptor(self, receptor, box, full_cells=True):
        self.box = box
        self._built = set()
        load().or_set_receptor(self.h, C.byref(receptor.desc), C.byref(box), int(full_cells))

    def set_user_grid(self, gd, data, cache_slope=1e6):
        """A user grid (--user_grid) over `gd`, values x fastest; None clears it."""
        self._built = set()
        if data is None:
            self._check(load().or_set_user_grid(self.h, None, None, cache_slope))
            return
        self._ug = np.ascontiguousarray(data, dtype=np.float64).ravel(order="F") if np.ndim(data) == 3 else \
            np.ascontiguousarray(data, dtype=np.float64)
        self._check(load().or_set_user_grid(self.h, C.byref(gd), sb.dptr(self._ug), cache_slope))

    def build_grids(self, types):
        t = np.ascontiguousarray(sorted(set(int(x) for x in types)), dtype=np.int32)
        self._check(load().or_build_grids(self.h, sb.iptr(t), len(t)))

    def grid(self, typ, charged=False):
        n = sb.grid_points(self.box)
        d = np.zeros(n)
        c = np.zeros(n) if charged else None
        self._check(load().or_get_grid(self.h, typ, sb.dptr(d), sb.dptr(c)))
        return d, c

    def ensure(self, models):
        types = sorted({t for m in models for t in m.types() if 1 < t < 27})
        missing = [t for t in types if t not in getattr(self, "_built", set())]
        if missing:
            self.build_grids(missing)
            self._built = getattr(self, "_built", set()) | set(missing)

    def eval(self, m, confs, v=(10, 10, 10), slope=1e6, coords=False):
        self.ensure([m])
        confs = np.ascontiguousarray(confs, dtype=np.float64).reshape(-1, m.conf_size)
        n = len(confs)
        e, g = np.zeros(n), np.zeros((n, m.dof))
        x = np.zeros((n, m.num_movable, 3)) if coords else None
        self._check(load().or_eval(self.h, C.byref(m.desc), n, sb.dptr(confs), sb.vec3(v), slope, sb.dptr(e),
                                   sb.dptr(g), sb.dptr(x)))
        return (e, g, x) if coords else (e, g)

    def eval_direct(self, m, confs, v=(1000, 1000, 1000), slope=10.0):
        confs = np.ascontiguousarray(confs, dtype=np.float64).reshape(-1, m.conf_size)
        n = len(confs)
        e, g = np.zeros(n), np.zeros((n, m.dof))
        self._check(load().or_eval_direct(self.h, C.byref(m.desc), n, sb.dptr(confs), sb.vec3(v), slope, sb.dptr(e),
                                          sb.dptr(g)))
        return e, g

    def bfgs(self, m, confs, v=(10, 10, 10), slope=1e6, maxiters=10, accurate=0, early=0):
        self.ensure([m])
        confs = np.ascontiguousarray(confs, dtype=np.float64).reshape(-1, m.conf_size).copy()
        e = np.zeros(len(confs))
        self._check(load().or_bfgs(self.h, C.byref(m.desc), len(confs), sb.dptr(confs), sb.vec3(v), slope, maxiters,
                                   accurate, early, sb.dptr(e)))
        return confs, e

    def dock(self, models, model_of_chain, confs, mts, params, steps=None, threads=1, maxiters=None):
        self.ensure(models)
        descs = (sb.ModelDesc * len(models))(*[m.desc for m in models])
        batch = sb.make_chain_batch(models, model_of_chain, confs, mts, params.num_steps if steps is None else steps,
                                    params.num_saved_mins, [m.heavy for m in models], maxiters)
        self._check(load().or_dock(self.h, descs, len(models), batch.inputs, len(model_of_chain), C.byref(params),
                                   batch.results, threads))
        batch.count = np.array([batch.results[k].count for k in range(len(model_of_chain))])
        batch.evals = np.array([batch.results[k].evals for k in range(len(model_of_chain))], dtype=np.uint64)
        return batch

    def refine(self, models, pose_model, confs, cap=(1000, 1000, 1000), maxiters=10, accurate=0, early=0):
        descs = (sb.ModelDesc * len(models))(*[m.desc for m in models])
        pm = np.ascontiguousarray(pose_model, dtype=np.int32)
        confs = np.ascontiguousarray(confs, dtype=np.float64).copy()
        n = len(pm)
        e = np.zeros(n)
        H = max(m.heavy for m in models)
        x = np.zeros((n, H, 3))
        self._check(load().or_refine(self.h, descs, sb.iptr(pm), n, sb.dptr(confs), sb.vec3(cap), maxiters, accurate,
                                     early, sb.dptr(e), sb.dptr(x)))
        return confs, e, x

    def minimize(self, models, pose_model, confs, boxes=None, cap=(1000, 1000, 1000), maxiters=10, accurate=0,
                 early=0):
        descs = (sb.ModelDesc * len(models))(*[m.desc for m in models])
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
        x = np.zeros((n, H, 3))
        self._check(load().or_minimize(self.h, descs, sb.iptr(pm), n, sb.dptr(c), cs, sb.dptr(bx), sb.vec3(cap),
                                       sb.iptr(mi), accurate, early, sb.dptr(e), sb.dptr(x), H))
        return c, e, x

    def score(self, models, pose_model, confs, v=(1000, 1000, 1000), slope=1e6):
        descs = (sb.ModelDesc * len(models))(*[m.desc for m in models])
        pm = np.ascontiguousarray(pose_model, dtype=np.int32)
        n = len(pm)
        cs = max(m.conf_size for m in models)
        H = max(m.heavy for m in models)
        c = np.zeros((n, cs))
        src = np.asarray(confs, dtype=np.float64).reshape(n, -1)
        c[:, :src.shape[1]] = src
        e, intra, x = np.zeros(n), np.zeros(n), np.zeros((n, H, 3))
        self._check(load().or_score(self.h, descs, sb.iptr(pm), n, sb.dptr(c), cs, sb.vec3(v), slope, sb.dptr(e),
                                    sb.dptr(intra), sb.dptr(x), H))
        return e, intra, x

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.or_destroy(self.h)
            self.h = None


def merge(batch, model, min_rmsd=2.0, max_size=20):
    """merge_output_containers over every chain of one model."""
    n = len(batch.count)
    e = np.zeros(n * max_size)
    conf = np.zeros((n * max_size, model.conf_size))
    xyz = np.zeros((n * max_size, model.heavy, 3))
    cnt = load().or_merge(batch.results, n, model.conf_size, model.heavy, min_rmsd, max_size, sb.dptr(e),
                          sb.dptr(conf), sb.dptr(xyz))
    return e[:cnt], conf[:cnt], xyz[:cnt]


def pm_eval(fn, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros_like(x)
    load().or_pm_eval(fn, sb.dptr(x), sb.dptr(y), len(x))
    return y


def mt_probe(seed, n, a=-1.0, b=1.0, lo=0, hi=1000000):
    raw = np.zeros(n, np.uint32)
    fl = np.zeros(n)
    it = np.zeros(n, np.int32)
    load().or_mt_probe(seed, n, sb.uptr(raw), a, b, sb.dptr(fl), lo, hi, sb.iptr(it))
    return raw, fl, it


def quat_probe(inp, q0):
    """The oracle's quaternion / angle math on rows of in[7] and q0[4] (out[22])."""
    inp = np.ascontiguousarray(inp, dtype=np.float64).reshape(-1, 7)
    q0 = np.ascontiguousarray(q0, dtype=np.float64).reshape(-1, 4)
    out = np.zeros((len(inp), 22))
    load().or_quat_probe(sb.dptr(inp), sb.dptr(q0), sb.dptr(out), len(inp))
    return out
