"""Plain (FP64) CUDA path vs the CPU oracle: bit-exact.

Mirrors the reference's validation executables: grid maps and single
evaluations (gpu_eval_test.cpp:173-433, FP64 strict), BFGS alone
(gpu_mc_test.cpp:454-530), whole Monte Carlo chains (:645-711) and
refinement (:187-293, with full cell bricks as GPU_TEST_FULL_CELLS).  Here
"strict" is bit-for-bit: every double is compared by its bit pattern.
"""
import numpy as np
import pytest

import smina_b200 as sb
import workloads as W
from oracle_lib import Oracle, merge

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def assert_bitwise(a, b, what):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    assert a.shape == b.shape, what
    diff = bits(a) != bits(b)
    if diff.any():
        i = np.argwhere(diff)[0]
        raise AssertionError(f"{what}: {diff.sum()} of {a.size} differ, first at {tuple(i)}: "
                             f"{a[tuple(i)]!r} vs {b[tuple(i)]!r}")


@pytest.fixture(scope="module")
def setup():
    T = W.tables()
    R = W.receptor()
    gd = W.box()
    eng = sb.Engine(0, sb.PREC_FP64)
    eng.set_tables(T)
    eng.set_receptor(0, R, gd)
    orc = Oracle(T, R, gd, full_cells=True)
    return eng, orc, gd


@pytest.mark.parametrize("heavy,rotors,seed", [(24, 5, 11), (12, 0, 3), (40, 10, 5)])
def test_grid_maps_bit_exact(setup, heavy, rotors, seed):
    eng, orc, gd = setup
    m = W.ligand(heavy, rotors, seed)
    types = sorted({t for t in m.types() if t > 1})
    eng.build_grids(0, types)
    orc.build_grids(types)
    for t in types:
        g, _ = eng.grid(0, t, gd)
        o, _ = orc.grid(t)
        assert_bitwise(g, o, f"map of type {t}")
        assert np.abs(o).max() > 0


@pytest.mark.parametrize("heavy,rotors,seed", [(24, 5, 11), (12, 0, 3), (40, 10, 5)])
def test_eval_bit_exact(setup, heavy, rotors, seed):
    eng, orc, gd = setup
    m = W.ligand(heavy, rotors, seed)
    confs = W.random_confs(m, gd, 64, seed)
    for v in ((10, 10, 10), (1000, 1000, 1000)):
        for slope in (1e6, 10.0):
            e1, g1, x1 = eng.eval(0, m, confs, v, slope, coords=True)
            e0, g0, x0 = orc.eval(m, confs, v, slope, coords=True)
            assert_bitwise(x1, x0, "coords")
            assert_bitwise(e1, e0, f"energy v={v} slope={slope}")
            assert_bitwise(g1, g0, f"gradient v={v} slope={slope}")


def test_eval_direct_bit_exact(setup):
    eng, orc, gd = setup
    m = W.ligand()
    confs = W.random_confs(m, gd, 32, 99)
    e1, g1 = eng.eval_direct(0, m, confs, (1000, 1000, 1000), 10.0)
    e0, g0 = orc.eval_direct(m, confs, (1000, 1000, 1000), 10.0)
    assert_bitwise(e1, e0, "direct energy")
    assert_bitwise(g1, g0, "direct gradient")


@pytest.mark.parametrize("accurate", [0, 1])
def test_bfgs_bit_exact(setup, accurate):
    eng, orc, gd = setup
    m = W.ligand()
    confs = W.random_confs(m, gd, 32, 5)
    c1, e1 = eng.bfgs(0, m, confs, (10, 10, 10), 1e6, 17, accurate, 0)
    c0, e0 = orc.bfgs(m, confs, (10, 10, 10), 1e6, 17, accurate, 0)
    assert_bitwise(e1, e0, "bfgs energy")
    assert_bitwise(c1, c0, "bfgs conf")


@pytest.mark.parametrize("heavy,rotors,seed,steps", [(24, 5, 11, 60), (16, 3, 21, 40)])
def test_mc_chains_bit_exact(setup, heavy, rotors, seed, steps):
    eng, orc, gd = setup
    m = W.ligand(heavy, rotors, seed)
    p = m.search_params()
    confs, mts = m.seed_chains(1234, 8, gd)
    b1 = eng.dock(0, [m], [0] * 8, confs, mts, p, steps=steps)
    b0 = orc.dock([m], [0] * 8, confs, mts, p, steps=steps, threads=8)
    assert (b1.count == b0.count).all()
    assert (b1.evals == b0.evals).all()
    for k in range(8):
        c = b0.count[k]
        assert c > 0
        assert_bitwise(b1.e[k, :c], b0.e[k, :c], f"chain {k} energies")
        assert_bitwise(b1.conf[k, :c, :m.conf_size], b0.conf[k, :c, :m.conf_size], f"chain {k} confs")
        assert_bitwise(b1.coords[k, :c, :m.heavy], b0.coords[k, :c, :m.heavy], f"chain {k} coords")


def test_mixed_ligands_with_own_iteration_counts_bit_exact(setup):
    """Chains of several ligands in one launch, each with its ligand's own
    step and BFGS-iteration counts (ChainInput::maxiters)."""
    eng, orc, gd = setup
    models = [W.ligand(24, 5, 11), W.ligand(12, 0, 3), W.ligand(40, 10, 5)]
    p = models[0].search_params()
    confs, mts, moc, steps, its = [], [], [], [], []
    for k, m in enumerate(models):
        c, mt = m.seed_chains(50 + k, 2, gd)
        cm = np.zeros((2, max(x.conf_size for x in models)))
        cm[:, :m.conf_size] = c
        confs += list(cm)
        mts += list(mt)
        moc += [k, k]
        steps += [8 + 3 * k] * 2
        its += [m.search_params().maxiters] * 2
    b1 = eng.dock(0, models, moc, confs, mts, p, steps=steps, maxiters=its)
    b0 = orc.dock(models, moc, confs, mts, p, steps=steps, maxiters=its, threads=6)
    assert (b1.count == b0.count).all() and (b1.evals == b0.evals).all()
    assert_bitwise(b1.e, b0.e, "energies")
    e, conf, _ = sb.merge_chains(b1, models[2], first=4, n=2)
    assert len(e) > 0 and np.all(np.diff(e) >= 0)


def test_refine_bit_exact(setup):
    eng, orc, gd = setup
    m = W.ligand()
    p = m.search_params()
    confs, mts = m.seed_chains(77, 4, gd)
    b0 = orc.dock([m], [0] * 4, confs, mts, p, steps=30, threads=4)
    e, conf, _ = merge(b0, m)
    poses = conf
    c1, e1, x1 = eng.refine(0, [m], [0] * len(poses), poses, maxiters=p.maxiters)
    c0, e0, x0 = orc.refine([m], [0] * len(poses), poses, maxiters=p.maxiters)
    assert_bitwise(e1, e0, "refined energies")
    assert_bitwise(c1, c0, "refined confs")
    assert_bitwise(x1, x0, "refined coords")


def test_minimize_in_own_boxes_bit_exact(setup):
    """Batched local optimisation (minimize_batch): each pose in its own box
    with its own iteration count, FP64 against the checker bit for bit;
    poses outside their box are pulled in or get max energy."""
    eng, orc, gd = setup
    models = [W.ligand(24, 5, 11), W.ligand(40, 10, 5)]
    rng = np.random.default_rng(5)
    confs, pm, boxes, its = [], [], [], []
    lo, hi = np.array(gd.begin[:]), np.array(gd.end[:])
    for k in range(8):
        mi = k % 2
        m = models[mi]
        c = W.random_confs(m, gd, 1, 200 + k)[0]
        centre = c[:3]
        half = rng.uniform(4.0, 8.0)
        b = np.concatenate([np.maximum(lo, centre - half), np.minimum(hi, centre + half)])
        cm = np.zeros(max(x.conf_size for x in models))
        cm[:m.conf_size] = c
        confs.append(cm)
        pm.append(mi)
        boxes.append(b)
        its.append(5 + 3 * k)
    c1, e1, x1 = eng.minimize(0, models, pm, confs, boxes=boxes, maxiters=its)
    c0, e0, x0 = orc.minimize(models, pm, confs, boxes=boxes, maxiters=its)
    assert_bitwise(e1, e0, "energies")
    assert_bitwise(c1, c0, "confs")
    assert_bitwise(x1, x0, "coords")
    # no boxes: the receptor's box, like refine_structure
    c2, e2, _ = eng.minimize(0, models, pm, confs, maxiters=its)
    c3, e3, _ = orc.minimize(models, pm, confs, maxiters=its)
    assert_bitwise(e2, e3, "energies (receptor box)")


@pytest.mark.parametrize("heavy,rotors,seed", [(24, 5, 11), (40, 10, 5)])
def test_mc_chains_with_visited_history_bit_exact(setup, heavy, rotors, seed):
    """MCParams::visited (QuickVina 2's history, the reference's
    gpu_mc.cuh:144-264; not smina's search): chains skip local optimisations
    the history deems redundant.  Bit-exact against the checker, and fewer
    evaluations than the same chains without the history."""
    eng, orc, gd = setup
    m = W.ligand(heavy, rotors, seed)
    p = m.search_params()
    confs, mts = m.seed_chains(99, 4, gd)
    plain = eng.dock(0, [m], [0] * 4, confs, mts, p, steps=80)
    p.visited = 1
    b1 = eng.dock(0, [m], [0] * 4, confs, mts, p, steps=80)
    b0 = orc.dock([m], [0] * 4, confs, mts, p, steps=80, threads=4)
    assert (b1.count == b0.count).all() and (b1.evals == b0.evals).all()
    for k in range(4):
        c = b0.count[k]
        assert_bitwise(b1.e[k, :c], b0.e[k, :c], f"chain {k} energies")
        assert_bitwise(b1.conf[k, :c, :m.conf_size], b0.conf[k, :c, :m.conf_size], f"chain {k} confs")
    assert b1.evals.sum() < plain.evals.sum()


def test_visited_history_is_refused_on_the_mixed_precision_path():
    T, R, gd = W.tables(), W.receptor(), W.box()
    eng = sb.Engine(0, sb.PREC_FP32)
    eng.set_tables(T)
    eng.set_receptor(0, R, gd)
    m = W.ligand(12, 0, 3)
    p = m.search_params()
    p.visited = 1
    with pytest.raises(sb.SminaError):
        eng.dock_batch(0, [m], [sb.LigandJob(model=0, num_chains=2, num_steps=2, maxiters=0, seed=1, ligand_key=1)], p)
