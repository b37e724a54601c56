"""Records the reference's own FP64 outputs that pin the oracle's search path.

The reference's FP64 device library (src/gpu/gpu_device.cu and
src/gpu/gpu_kernels_f64.cu, its validation path that reproduces CPU smina)
is compiled by `make -C oracle ref` into oracle/_ref/libref_gpu.so, behind
the C entry points of oracle/ref_gpu.cu.  The reference tree is needed only
to build it.  This script runs it on a GPU over seeded synthetic inputs and
writes one compressed archive of its outputs:

  grid maps      sampled points of every map the models need (cache::populate)
  eval           energy and gradient of 24 confs per model, two curl caps
  eval_direct    energy and gradient against the receptor atoms (non_cache)
  bfgs           quasi_newton from 8 confs, both line searches
  dock           4 Monte Carlo chains of 40 steps per model
  refine         refine_structure of 8 poses per model

next to SHA-256 digests of every input, so a reader can tell that it
rebuilds the same inputs.  It then runs the oracle on the same inputs and
prints how many values agree bit for bit and the largest difference; with
--engine it does the same for this engine's FP64 path on the GPU.

    python tests/golden/make_ref_golden.py --engine --out tests/golden/ref_fp64.npz

Cases: default (vina) scoring and the charge-dependent ad4_scoring tables;
a 1,500-atom receptor with a 14 A box at 0.375 A; ligands of 14/3, 24/5 and
40/10 heavy atoms/rotors, and the 24/5 ligand with flexible residues; the
24/5 ligand with a user grid (--user_grid) added to the maps and the direct
sum; and ad4_scoring with seeded partial charges on the receptor, the ligand
and the flexible residues (ad4_q).
"""
import argparse
import ctypes as C
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "gpu-smina_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import smina_b200 as sb  # noqa: E402
import workloads as W  # noqa: E402

REF_SO = os.path.join(ROOT, "oracle", "_ref", "libref_gpu.so")
GRID_SAMPLES = 1024
EVAL_CONFS, DIRECT_CONFS, BFGS_CONFS, CHAINS, STEPS, POSES = 24, 12, 8, 4, 40, 8


# ---- inputs ---------------------------------------------------------------------------------------
def cases():
    """(name, tables, receptor, box, models) of every case, rebuilt from seeds."""
    R = W.receptor(1500, 3)
    gd = W.box(14.0)
    lig = [W.ligand(14, 3, 2), W.ligand(24, 5, 11), W.ligand(40, 10, 5)]
    flex = sb.Model(sb.make_ligand_pdbqt(24, 5, 11, W.CENTER), sb.make_flex_pdbqt(4, 3, W.CENTER))
    # charge-dependent terms with non-zero charges on both sides
    Rq = W.charged_receptor(1500, 3, 2)
    flex_q = sb.Model(W.with_charges(sb.make_ligand_pdbqt(24, 5, 11, W.CENTER), 1),
                      W.with_charges(sb.make_flex_pdbqt(4, 3, W.CENTER), 3))
    return [("vina", W.tables(), R, gd, lig + [flex]),
            ("ad4", sb.Tables("ad4_scoring"), R, gd, [lig[1]]),
            ("vina_ug", W.tables(), R, gd, [lig[1]]),
            ("ad4_q", sb.Tables("ad4_scoring"), Rq, gd, [W.charged_ligand(24, 5, 11, 1), flex_q])]


def user_grid_for(name, gd):
    """(GridDims, values x fastest) of a case's user grid, or None.  Values
    as smina holds them after reading a user grid file (grid.cpp:78-110
    fills x, y, z < n and leaves the last plane of each axis at 0)."""
    if name != "vina_ug":
        return None
    n = 16
    g = sb.GridDims()
    for i in range(3):
        g.begin[i], g.end[i], g.n[i] = gd.begin[i] - 4.0, gd.end[i] + 4.0, n
    v = 0.5 * np.random.default_rng(77).normal(size=(n + 1, n + 1, n + 1))  # [z][y][x]
    v[n, :, :] = v[:, n, :] = v[:, :, n] = 0.0
    return g, np.ascontiguousarray(v.ravel())


def oracle_for(name, T, R, gd):
    from oracle_lib import Oracle
    o = Oracle(T, R, gd, full_cells=True)
    ug = user_grid_for(name, gd)
    if ug is not None:
        o.set_user_grid(*ug)
    return o


def grid_types(models):
    return sorted({t for m in models for t in m.types() if 1 < t < 27})


def model_inputs(m, gd, k):
    """Confs, chain seeds and poses of model k of a case (all seeded)."""
    confs = W.random_confs(m, gd, EVAL_CONFS, 100 + k)
    direct = W.random_confs(m, gd, DIRECT_CONFS, 200 + k, spread=0.3)
    start = W.random_confs(m, gd, BFGS_CONFS, 300 + k)
    c0, mt = m.seed_chains(400 + k, CHAINS, gd)
    poses = W.random_confs(m, gd, POSES, 500 + k, spread=0.4)
    return confs, direct, start, c0, mt, poses


def _arr(ptr, n, dtype):
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype) if n else np.zeros(0, dtype)


def digest(T, R, gd, models, ug=None):
    h = hashlib.sha256()
    if ug is not None:
        h.update(np.array(list(ug[0].begin) + list(ug[0].end), np.float64).tobytes())
        h.update(np.array(list(ug[0].n), np.int64).tobytes() + ug[1].tobytes())
    t = T.desc
    cells = 351 * t.n * t.num_components
    h.update(np.array([t.num_types, t.num_components, t.n], np.int64).tobytes())
    h.update(np.array([t.factor, t.cutoff_sqr], np.float64).tobytes())
    h.update(_arr(t.fast, cells, np.float64).tobytes())
    h.update(_arr(t.smooth, 2 * cells, np.float64).tobytes())
    r = R.desc
    h.update(_arr(r.coords, 3 * r.num_atoms, np.float64).tobytes())
    h.update(_arr(r.type, r.num_atoms, np.int32).tobytes())
    if r.charge:
        h.update(_arr(r.charge, r.num_atoms, np.float64).tobytes())
    h.update(np.array(list(gd.begin) + list(gd.end), np.float64).tobytes() + np.array(list(gd.n), np.int64).tobytes())
    for m in models:
        d = m.desc
        h.update(np.array([d.num_atoms, d.num_movable, d.num_frames, d.num_ligands, d.num_flex, d.conf_size, d.dof,
                           d.num_pairs, d.num_other_pairs], np.int64).tobytes())
        for name, n, dt in [("atom_type", d.num_atoms, np.int32), ("atom_charge", d.num_atoms, np.float64),
                            ("atom_local", 3 * d.num_atoms, np.float64), ("atom_lab", 3 * d.num_atoms, np.float64),
                            ("frame_kind", d.num_frames, np.int32), ("frame_parent", d.num_frames, np.int32),
                            ("frame_begin", d.num_frames, np.int32), ("frame_end", d.num_frames, np.int32),
                            ("frame_conf", d.num_frames, np.int32), ("frame_dof", d.num_frames, np.int32),
                            ("frame_origin", 3 * d.num_frames, np.float64), ("frame_axis", 3 * d.num_frames, np.float64),
                            ("frame_init_origin", 3 * d.num_frames, np.float64), ("pairs", 2 * d.num_pairs, np.int32)]:
            h.update(_arr(getattr(d, name), n, dt).tobytes())
    for k, m in enumerate(models):
        for a in model_inputs(m, gd, k):
            h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def grid_sample(gd, seed):
    n = sb.grid_points(gd)
    return np.sort(np.random.default_rng(seed).choice(n, size=min(GRID_SAMPLES, n), replace=False))


# ---- the reference (oracle/_ref/libref_gpu.so) ----------------------------------------------------------
class Ref:
    def __init__(self, T, R, gd, types, ug=None):
        L = C.CDLL(REF_SO)
        vp, dp, ip = C.c_void_p, sb._dp, sb._ip
        L.refg_last_error.restype = C.c_char_p
        sig = {
            "refg_create": [C.POINTER(sb.TablesDesc), C.POINTER(sb.ReceptorDesc), C.POINTER(sb.GridDims), ip, C.c_int,
                            C.c_double, C.POINTER(sb.GridDims), dp, C.POINTER(vp)],
            "refg_get_grid": [vp, C.c_int, dp, dp],
            "refg_eval": [vp, C.POINTER(sb.ModelDesc), C.c_int, dp, C.c_double * 3, C.c_int, C.c_double, dp, dp, dp],
            "refg_bfgs": [vp, C.POINTER(sb.ModelDesc), C.c_int, dp, C.c_double * 3, C.c_int, C.c_int, C.c_int, dp],
            "refg_dock": [vp, C.POINTER(sb.ModelDesc), C.c_int, C.POINTER(sb.ChainInput), C.c_int,
                          C.POINTER(sb.MCParams), C.POINTER(sb.ChainResult)],
            "refg_refine": [vp, C.POINTER(sb.ModelDesc), C.c_int, ip, C.c_int, dp, C.c_double * 3, C.c_int, C.c_int,
                            C.c_int, dp, dp],
        }
        for k, a in sig.items():
            getattr(L, k).argtypes = a
            getattr(L, k).restype = C.c_int
        L.refg_destroy.argtypes = [vp]
        L.refg_destroy.restype = None
        self.L, self.gd = L, gd
        self.h = vp()
        t = np.ascontiguousarray(types, np.int32)
        self._ug = None if ug is None else np.ascontiguousarray(ug[1], np.float64)
        self._check(L.refg_create(C.byref(T.desc), C.byref(R.desc), C.byref(gd), sb.iptr(t), len(t), 1e6,
                                  None if ug is None else C.byref(ug[0]), None if ug is None else sb.dptr(self._ug),
                                  C.byref(self.h)))

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(f"reference harness: {self.L.refg_last_error().decode()} (status {rc})")

    def grid(self, typ, charged):
        n = sb.grid_points(self.gd)
        d = np.zeros(n)
        c = np.zeros(n) if charged else None
        self._check(self.L.refg_get_grid(self.h, typ, sb.dptr(d), sb.dptr(c)))
        return d, c

    def eval(self, m, confs, v, use_cache, slope):
        confs = np.ascontiguousarray(confs, np.float64)
        n = len(confs)
        e, g = np.zeros(n), np.zeros((n, m.dof))
        self._check(self.L.refg_eval(self.h, C.byref(m.desc), n, sb.dptr(confs), sb.vec3(v), use_cache, slope,
                                     sb.dptr(e), sb.dptr(g), None))
        return e, g

    def bfgs(self, m, confs, v, maxiters, accurate):
        x = np.ascontiguousarray(confs, np.float64).copy()
        e = np.zeros(len(x))
        self._check(self.L.refg_bfgs(self.h, C.byref(m.desc), len(x), sb.dptr(x), sb.vec3(v), maxiters, accurate, 0,
                                     sb.dptr(e)))
        return x, e

    def dock(self, m, c0, mt, p, steps):
        descs = (sb.ModelDesc * 1)(m.desc)
        b = sb.make_chain_batch([m], [0] * len(c0), c0, mt, steps, p.num_saved_mins, [m.heavy])
        self._check(self.L.refg_dock(self.h, descs, 1, b.inputs, len(c0), C.byref(p), b.results))
        b.count = np.array([b.results[k].count for k in range(len(c0))])
        return b

    def refine(self, m, poses, cap, maxiters):
        descs = (sb.ModelDesc * 1)(m.desc)
        x = np.ascontiguousarray(poses, np.float64).copy()
        pm = np.zeros(len(x), np.int32)
        e, xyz = np.zeros(len(x)), np.zeros((len(x), m.heavy, 3))
        self._check(self.L.refg_refine(self.h, descs, 1, sb.iptr(pm), len(x), sb.dptr(x), sb.vec3(cap), maxiters, 0,
                                       0, sb.dptr(e), sb.dptr(xyz)))
        return x, e, xyz

    def close(self):
        self.L.refg_destroy(self.h)


class EngineSide:
    """This engine's plain FP64 path with the oracle's method names, so that
    outputs() records it the same way (a third side of the comparison)."""

    def __init__(self, T, R, gd, ug=None):
        self.e = sb.Engine(0, sb.PREC_FP64)
        self.e.set_tables(T)
        self.e.set_receptor(0, R, gd)
        if ug is not None:
            self.e.set_user_grid(0, *ug)
        self.gd = gd

    def build_grids(self, types):
        self.e.build_grids(0, types)

    def grid(self, t, charged):
        return self.e.grid(0, t, self.gd, charged)

    def eval(self, m, confs, v, slope):
        return self.e.eval(0, m, confs, v=v, slope=slope)

    def eval_direct(self, m, confs, slope):
        return self.e.eval_direct(0, m, confs, slope=slope)

    def bfgs(self, m, confs, v, slope, maxiters, accurate):
        return self.e.bfgs(0, m, confs, v=v, slope=slope, maxiters=maxiters, accurate=accurate)

    def dock(self, models, moc, c0, mt, p, steps):
        return self.e.dock(0, models, moc, c0, mt, p, steps=steps)

    def refine(self, models, pm, poses, cap, maxiters):
        return self.e.refine(0, models, pm, poses, cap=cap, maxiters=maxiters)

    def close(self):
        self.e.close()


# ---- one side's outputs (the reference's, the oracle's or this engine's) --------------------------------
def outputs(side, T, gd, models, tag):
    """Every recorded quantity of a case, as {key: array}; `side` is a Ref
    or a tests/oracle_lib.Oracle (same method names)."""
    out = {}
    charged = T.desc.num_components > 1
    is_ref = isinstance(side, Ref)
    if not is_ref:
        side.build_grids(grid_types(models))
    idx = grid_sample(gd, 7)
    for t in grid_types(models):
        d, c = side.grid(t, charged)
        out[f"{tag}/grid{t}"] = d[idx]
        if charged:
            out[f"{tag}/grid{t}_charge"] = c[idx]
    for k, m in enumerate(models):
        p = m.search_params()
        confs, direct, start, c0, mt, poses = model_inputs(m, gd, k)
        for vn, v in (("hunt", (10.0, 10.0, 10.0)), ("auth", (1000.0, 1000.0, 1000.0))):
            e, g = side.eval(m, confs, v, 1, 1e6) if is_ref else side.eval(m, confs, v=v, slope=1e6)
            out[f"{tag}/m{k}/eval_{vn}_e"], out[f"{tag}/m{k}/eval_{vn}_g"] = e, g
        e, g = side.eval(m, direct, (1000.0,) * 3, 0, 10.0) if is_ref else side.eval_direct(m, direct, slope=10.0)
        out[f"{tag}/m{k}/direct_e"], out[f"{tag}/m{k}/direct_g"] = e, g
        for acc in (0, 1):
            x, e = (side.bfgs(m, start, (10.0,) * 3, p.maxiters, acc) if is_ref else
                    side.bfgs(m, start, v=(10.0,) * 3, slope=1e6, maxiters=p.maxiters, accurate=acc))
            out[f"{tag}/m{k}/bfgs{acc}_x"], out[f"{tag}/m{k}/bfgs{acc}_e"] = x, e
        b = side.dock(m, c0, mt, p, STEPS) if is_ref else side.dock([m], [0] * CHAINS, c0, mt, p, steps=STEPS)
        out[f"{tag}/m{k}/dock_count"] = np.asarray(b.count, np.int64)
        out[f"{tag}/m{k}/dock_e"] = np.where(np.arange(p.num_saved_mins)[None, :] < b.count[:, None], b.e, 0.0)
        conf = np.zeros((CHAINS, p.num_saved_mins, m.conf_size))
        for c in range(CHAINS):
            conf[c, :b.count[c]] = b.conf[c, :b.count[c], :m.conf_size]
        out[f"{tag}/m{k}/dock_conf"] = conf
        x, e, xyz = (side.refine(m, poses, (1000.0,) * 3, p.maxiters) if is_ref else
                     side.refine([m], np.zeros(POSES, np.int32), poses, cap=(1000.0,) * 3, maxiters=p.maxiters))
        out[f"{tag}/m{k}/refine_x"], out[f"{tag}/m{k}/refine_e"] = x, e
        out[f"{tag}/m{k}/refine_xyz"] = np.asarray(xyz, np.float64).reshape(POSES, -1)
    return out


def compare(ref, mine):
    """(values, bit-identical values, largest relative difference, worst key)."""
    total = same = 0
    worst, worst_key = 0.0, ""
    for k, a in ref.items():
        b = np.asarray(mine[k])
        a = np.asarray(a)
        assert a.shape == b.shape, (k, a.shape, b.shape)
        total += a.size
        if a.dtype.kind == "f":
            same += int(np.sum(a.view(np.uint64) == np.ascontiguousarray(b, np.float64).view(np.uint64)))
            rel = np.abs(a - b) / np.maximum(np.abs(a), 1.0)
            if rel.size and rel.max() > worst:
                worst, worst_key = float(rel.max()), k
        else:
            same += int(np.sum(a == b))
    return total, same, worst, worst_key


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_fp64.npz"))
    ap.add_argument("--engine", action="store_true", help="also compare this engine's FP64 path on the GPU")
    args = ap.parse_args()
    rec = {}
    for name, T, R, gd, models in cases():
        ug = user_grid_for(name, gd)
        ref = Ref(T, R, gd, grid_types(models), ug)
        r = outputs(ref, T, gd, models, name)
        ref.close()
        rec.update(r)
        rec[f"{name}/sha256"] = np.array(digest(T, R, gd, models, ug))
        o = outputs(oracle_for(name, T, R, gd), T, gd, models, name)
        total, same, worst, key = compare(r, o)
        print(f"{name}: oracle: {same}/{total} values bit-identical to the reference; largest relative "
              f"difference {worst:.3g} ({key or 'none'})", flush=True)
        if args.engine:
            eng = EngineSide(T, R, gd, ug)
            g = outputs(eng, T, gd, models, name)
            eng.close()
            total, same, worst, key = compare(r, g)
            print(f"{name}: this engine (FP64): {same}/{total} values bit-identical to the reference; largest "
                  f"relative difference {worst:.3g} ({key or 'none'})", flush=True)
    np.savez_compressed(args.out, **rec)
    print(f"wrote {args.out} ({os.path.getsize(args.out)} bytes)")


if __name__ == "__main__":
    main()
