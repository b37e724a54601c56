"""Mixed-precision (FP32) path vs the FP64 oracle, and the batched search.

Single evaluations must agree with FP64 to 1e-4 kcal/mol relative (energy
relative to max(|E|, 1 kcal/mol); gradient relative to its largest
component) under the reference's FP32 acceptance rule: at least 99% of the
evaluations within 1e-4, and every evaluation that is not at a
discontinuity of the scoring function within 10 x 1e-4.  Discontinuities:
a pair within float precision of the hard cutoff, and a heavy atom just
outside the grid box, where the 1e6 kcal/mol/A out-of-box slope turns the
float coordinate precision (~1e-6 A) into ~1 kcal/mol.  The batched search is checked for determinism, for
independence from the batch it runs in and from the launch shape, for
bit-exact FP64 refinement of its merged poses (against the oracle's
refine_structure), and for pose quality against the plain FP64 search.
Reference checks mirrored: gpu_eval_test.cpp:173-433 (FP32 tolerance
mode), gpu_mc_test.cpp:645-711 (search outcome), gpu_docking.cpp:560-625
(merge + refine of a batch).
"""
import numpy as np
import pytest

import smina_b200 as sb
import workloads as W
from oracle_lib import Oracle, merge

pytestmark = pytest.mark.gpu

TOL = 1e-4        # relative, energy and gradient
FRAC = 0.99       # share of evaluations that must be within TOL
OUTSIDE_A = 1e-2  # heavy atom closer than this outside the box: at the box-face kink
CUT_A2 = 2e-4     # pair with |r^2 - cutoff^2| below this: at the cutoff


@pytest.fixture(scope="module")
def base():
    T = W.tables()
    R = W.receptor()
    gd = W.box()
    orc = Oracle(T, R, gd, full_cells=True)
    engines = {}

    def engine(prec, tables=T, receptor=R):
        key = (prec, id(tables), id(receptor))
        if key not in engines:
            e = sb.Engine(0, prec)
            e.set_tables(tables)
            e.set_receptor(0, receptor, gd)
            engines[key] = e
        return engines[key]
    return engine, orc, gd, R


def _rel_err(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1.0)


def _grad_err(g, ref):
    scale = np.maximum(np.abs(ref).max(axis=1), 1.0)
    return np.abs(g - ref).max(axis=1) / scale


def at_discontinuity(m, gd, xyz, cutoff_sqr):
    """Confs (by oracle coords) at the hard pair cutoff or just outside the box."""
    d = m.desc
    flags = np.zeros(len(xyz), bool)
    if d.num_pairs:
        pr = np.ctypeslib.as_array(d.pairs, shape=(2 * d.num_pairs,)).reshape(-1, 2)
        full = xyz
        if d.num_atoms > xyz.shape[1]:  # fixed atoms of flexible residues keep their input coords
            lab = np.ctypeslib.as_array(d.atom_lab, shape=(3 * d.num_atoms,)).reshape(-1, 3)
            fixed = np.broadcast_to(lab[xyz.shape[1]:], (len(xyz),) + lab[xyz.shape[1]:].shape)
            full = np.concatenate([xyz, fixed], axis=1)
        r2 = ((full[:, pr[:, 1]] - full[:, pr[:, 0]]) ** 2).sum(-1)
        flags |= (np.abs(r2 - cutoff_sqr) < CUT_A2).any(1)
    heavy = np.where(np.array(m.types())[:m.num_movable] > 1)[0]
    lo, hi = np.array(gd.begin[:]), np.array(gd.end[:])
    out = np.maximum(lo - xyz[:, heavy], xyz[:, heavy] - hi)
    flags |= ((out > 0) & (out < OUTSIDE_A)).any((1, 2))
    return flags


def check_fp32(e, g, e64, g64, flags, tol=TOL):
    er, gr = _rel_err(e, e64), _grad_err(g, g64)
    ok = (er <= tol) & (gr <= tol)
    assert ok.mean() >= FRAC, f"{ok.mean():.4f} within {tol} (energy max {er.max():.3g}, gradient max {gr.max():.3g})"
    if (~flags).any():
        assert er[~flags].max() <= 10 * tol, f"energy rel err {er[~flags].max():.3g} away from discontinuities"
        assert gr[~flags].max() <= 10 * tol, f"gradient rel err {gr[~flags].max():.3g} away from discontinuities"


@pytest.mark.parametrize("heavy,rotors,seed", [(24, 5, 11), (12, 0, 3), (40, 10, 5), (50, 12, 4), (60, 40, 9)])
def test_eval_fp32_within_tolerance(base, heavy, rotors, seed):
    engine, orc, gd, _ = base
    m = W.ligand(heavy, rotors, seed)
    confs = W.random_confs(m, gd, 256, seed + 100)
    eng = engine(sb.PREC_FP32)
    e32, g32, x32 = eng.eval(0, m, confs, coords=True)
    e64, g64, x64 = orc.eval(m, confs, coords=True)
    assert np.abs(x32 - x64).max() < 1e-4  # torsion tree in FP32
    check_fp32(e32, g32, e64, g64, at_discontinuity(m, gd, x64, W.tables().desc.cutoff_sqr))


def test_eval_fp32_charge_dependent_tables(base):
    """nc = 4 tables (charge-weighted components, charge maps)."""
    engine, _, gd, R = base
    T4 = sb.Tables("ad4_scoring")
    Rq = W.charged_receptor()
    orc = Oracle(T4, Rq, gd, full_cells=True)
    m = W.charged_ligand(24, 5, 11)
    confs = W.random_confs(m, gd, 128, 7)
    eng = engine(sb.PREC_FP32, T4, Rq)
    e32, g32 = eng.eval(0, m, confs)
    e64, g64, x64 = orc.eval(m, confs, coords=True)
    check_fp32(e32, g32, e64, g64, at_discontinuity(m, gd, x64, T4.desc.cutoff_sqr))


def test_eval_fp16_maps_error_stated(base):
    """FP16 map storage: interpolation stays FP32; the error is the maps'
    half-precision rounding (relative 2^-11 of each corner value)."""
    engine, orc, gd, _ = base
    m = W.ligand(24, 5, 11)
    confs = W.random_confs(m, gd, 64, 21)
    e16, _ = engine(sb.PREC_FP32_H16).eval(0, m, confs)
    e64, _, x64 = orc.eval(m, confs, coords=True)
    er = _rel_err(e16, e64)[~at_discontinuity(m, gd, x64, W.tables().desc.cutoff_sqr)]
    assert er.max() <= 2e-3, f"fp16 maps: rel err max {er.max():.3g}"


def _jobs(models, chains=4, steps=30, seed=42, keys=None):
    return [sb.LigandJob(model=k, num_chains=chains, num_steps=steps, maxiters=0, seed=seed,
                         ligand_key=(keys[k] if keys else 1000 + k)) for k in range(len(models))]


def _params(m):
    return m.search_params()


def test_batch_deterministic_and_shape_independent(base):
    engine, _, _, _ = base
    eng = engine(sb.PREC_FP32)
    models = [W.ligand(24, 5, 11), W.ligand(12, 0, 3), W.ligand(40, 10, 5)]
    p = _params(models[0])
    jobs = _jobs(models)
    a = eng.dock_batch(0, models, jobs, p)
    b = eng.dock_batch(0, models, jobs, p)
    try:
        eng.set_chains_per_block(1)
        c = eng.dock_batch(0, models, jobs, p)
        assert eng.batch_stats()["chains_per_block"] == 1
    finally:
        eng.set_chains_per_block(0)
    for x, y, z in zip(a, b, c):
        assert len(x["e"]) > 0
        for k in ("e", "conf", "coords"):
            assert np.array_equal(x[k], y[k]) and np.array_equal(x[k], z[k]), k
        assert x["evals"] == y["evals"] == z["evals"] > 0


def test_autotune_keeps_a_shape_and_results(base):
    """The launch-shape autotuner times every shape that fits and keeps the
    fastest; docking results do not depend on the shape it keeps."""
    engine, _, _, _ = base
    eng = engine(sb.PREC_FP32)
    models = [W.ligand(24, 5, 11), W.ligand(12, 0, 3), W.ligand(40, 10, 5)]
    p = _params(models[0])
    jobs = _jobs(models)
    a = eng.dock_batch(0, models, jobs, p)
    try:
        chosen, rates = eng.autotune(0, models, jobs, p, step_fraction=0.5)
        assert chosen in (8, 4, 2, 1) and rates[chosen] == max(rates.values()) > 0
        b = eng.dock_batch(0, models, jobs, p)
        assert eng.batch_stats()["chains_per_block"] == chosen
    finally:
        eng.set_chains_per_block(0)
    for x, y in zip(a, b):
        for k in ("e", "conf", "coords"):
            assert np.array_equal(x[k], y[k]), k


def test_batch_alone_equals_in_mix(base):
    engine, _, _, _ = base
    eng = engine(sb.PREC_FP32)
    models = [W.ligand(24, 5, 11), W.ligand(12, 0, 3), W.ligand(40, 10, 5)]
    p = _params(models[0])
    mix = eng.dock_batch(0, models, _jobs(models, keys=[7, 8, 9]), p)
    alone = eng.dock_batch(0, [models[2]], [sb.LigandJob(model=0, num_chains=4, num_steps=30, maxiters=0, seed=42,
                                                          ligand_key=9)], p)
    for k in ("e", "conf", "coords"):
        assert np.array_equal(mix[2][k], alone[0][k]), k


def test_batch_refine_matches_oracle(base):
    """The merged poses go through FP64 refine_structure bit-exactly."""
    engine, orc, _, _ = base
    eng = engine(sb.PREC_FP32)
    models = [W.ligand(24, 5, 11), W.ligand(30, 8, 2)]
    p = _params(models[0])
    jobs = _jobs(models, chains=3, steps=20)
    raw = eng.dock_batch(0, models, jobs, p, refine=False)
    ref = eng.dock_batch(0, models, jobs, p, refine=True)
    for k, m in enumerate(models):
        assert len(raw[k]["e"]) == len(ref[k]["e"]) > 0
        confs, e, _ = orc.refine([m], np.zeros(len(raw[k]["e"]), np.int32), raw[k]["conf"],
                                 cap=tuple(p.authentic_v), maxiters=p.maxiters, accurate=p.accurate_line,
                                 early=p.early_term)
        order = np.argsort(e, kind="stable")
        assert np.array_equal(np.sort(e), ref[k]["e"])
        assert np.array_equal(confs[order], ref[k]["conf"])
        # merged poses are sorted and at least 2 A apart
        assert np.all(np.diff(raw[k]["e"]) >= 0)


def test_batch_counters(base):
    engine, _, _, _ = base
    eng = engine(sb.PREC_FP32)
    models = [W.ligand(24, 5, 11), W.ligand(12, 0, 3)]
    res = eng.dock_batch(0, models, _jobs(models, chains=2, steps=10), _params(models[0]), refine=False)
    st = eng.batch_stats()
    assert st["evals"] == sum(r["evals"] for r in res) > 0
    assert st["grid_lookups"] >= st["evals"] * 10  # every eval looks up every heavy atom
    assert st["pair_lookups"] > 0
    assert st["mc_ms"] > 0 and st["blocks"] > 0
    assert st["h2d_bytes"] > 0 and st["d2h_bytes"] > 0


def test_batch_pose_quality_vs_fp64(base):
    """Same ligand, same chains and steps: the FP32 batched search reaches the
    plain FP64 search's best refined energy.  The streams differ, and one
    short search lands in one of several near-degenerate minima, so each side
    runs 4 independent searches of 8 chains and their best results are
    compared, within a margin."""
    engine, orc, gd, _ = base
    m = W.ligand(24, 5, 11)
    p = _params(m)
    chains, steps, runs = 8, 400, 4
    eng64 = engine(sb.PREC_FP64)
    confs, mts = m.seed_chains(5, chains * runs, gd)
    b = eng64.dock(0, [m], np.zeros(chains * runs, np.int32), confs, mts, p, steps=steps)
    best64 = []
    for k in range(runs):
        sub = sb.merge_chains(b, m, first=chains * k, n=chains, max_size=p.num_saved_mins)
        _, e64, _ = eng64.refine(0, [m], np.zeros(len(sub[0]), np.int32), sub[1], cap=tuple(p.authentic_v),
                                 maxiters=p.maxiters, accurate_line=p.accurate_line, early_term=p.early_term)
        best64.append(float(np.min(e64)))
    jobs = [sb.LigandJob(model=0, num_chains=chains, num_steps=steps, maxiters=0, seed=5, ligand_key=1 + k)
            for k in range(runs)]
    r32 = engine(sb.PREC_FP32).dock_batch(0, [m], jobs, p)
    best32 = [float(r["e"][0]) for r in r32]
    assert min(best32) <= min(best64) + 0.5, (best32, best64)


def test_batch_rejects_fp64_engine(base):
    engine, _, _, _ = base
    m = W.ligand(24, 5, 11)
    with pytest.raises(sb.SminaError):
        engine(sb.PREC_FP64).dock_batch(0, [m], _jobs([m]), _params(m))


@pytest.mark.parametrize("heavy,rotors,seed", [(24, 5, 11), (40, 10, 5)])
def test_mixed_precision_bfgs(base, heavy, rotors, seed):
    """sg_bfgs on an FP32 engine runs the batched search's own BFGS (FP32
    energies and gradients; FP64 conf, inverse Hessian and acceptance
    tests): it never returns an energy above its starting energy, it lowers
    the energy of some of the random starts (many start far outside the box
    or in clashes that its line search cannot leave within the iterations), the energy it returns for a pose is that
    pose's energy (FP64 evaluation of the returned conf, within the FP32
    rule), and a second run gives the same bits."""
    engine, _, gd, _ = base
    m = W.ligand(heavy, rotors, seed)
    e64, e32 = engine(sb.PREC_FP64), engine(sb.PREC_FP32)
    starts = W.random_confs(m, gd, 128, 23)
    maxit = m.search_params().maxiters
    c32, f32 = e32.bfgs(0, m, starts, maxiters=maxit)
    e0, _ = e32.eval(0, m, starts)
    assert (f32 <= e0).all()
    assert (f32 < e0).mean() >= 0.1
    ev64, _ = e64.eval(0, m, c32)
    rel = np.abs(f32 - ev64) / np.maximum(np.abs(ev64), 1.0)
    assert (rel <= TOL).mean() >= FRAC, np.percentile(rel, [50, 99, 100])
    c32b, f32b = e32.bfgs(0, m, starts, maxiters=maxit)
    assert np.array_equal(c32b, c32) and np.array_equal(f32b, f32)
