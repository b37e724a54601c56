"""User grids (--user_grid) in the engine, against the oracle bit for bit.

smina adds a user grid to every receptor map at the map point's index
coordinates, with the cache's slope (cache::populate, cache.cpp:204-205),
and to the direct receptor sum at each heavy atom's own coordinates with its
derivative (non_cache::eval_deriv, non_cache.cpp:180-184).  The oracle's
restatement is pinned to the reference's device library by
tests/test_ref_pinning.py (case vina_ug); here the engine's FP64 path is
held to the oracle on other inputs: a user grid whose box covers the index
coordinates of the maps (so every map point takes an interpolated value, not
the out-of-grid penalty), charge-dependent tables with non-zero partial
charges, and a model with flexible residues.  The mixed-precision path reads maps built the same way.
"""
import numpy as np
import pytest

import smina_b200 as sb
import workloads as W
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def assert_bitwise(a, b, what):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    assert a.shape == b.shape, what
    diff = bits(a) != bits(b)
    assert not diff.any(), f"{what}: {diff.sum()} of {a.size} differ"


def user_grid(lo, hi, n, seed):
    g = sb.GridDims()
    for i in range(3):
        g.begin[i], g.end[i], g.n[i] = lo[i], hi[i], n
    v = 0.4 * np.random.default_rng(seed).normal(size=(n + 1) ** 3)
    return g, v


def _sides(tables, gd, ug, slope=1e6):
    R = W.charged_receptor(1500, 3, 2) if tables.desc.num_components > 1 else W.receptor(1500, 3)
    eng = sb.Engine(0, sb.PREC_FP64)
    eng.set_tables(tables)
    eng.set_receptor(0, R, gd)
    eng.set_user_grid(0, ug[0], ug[1], slope)
    orc = Oracle(tables, R, gd, full_cells=True)
    orc.set_user_grid(ug[0], ug[1], slope)
    return eng, orc


# a user grid over the maps' index coordinates (the box has 38 points per axis)
INDEX_GRID = ((-1.0, -1.0, -1.0), (40.0, 40.0, 40.0), 12, 5)
# a user grid over the box in Angstrom, 4 A larger on each side
def _around(gd):
    return (tuple(gd.begin[i] - 4.0 for i in range(3)), tuple(gd.end[i] + 4.0 for i in range(3)), 16, 77)


@pytest.mark.parametrize("tables,where", [("vina", "index"), ("vina", "around"), ("ad4_scoring", "index")])
def test_user_grid_maps_eval_direct_refine_bit_exact(tables, where):
    gd = W.box(14.0)
    T = W.tables(tables)
    lo, hi, n, seed = INDEX_GRID if where == "index" else _around(gd)
    eng, orc = _sides(T, gd, user_grid(lo, hi, n, seed))
    charged = T.desc.num_components > 1
    q = W.with_charges if charged else (lambda text, seed: text)
    models = [W.charged_ligand(24, 5, 11) if charged else W.ligand(24, 5, 11),
              sb.Model(q(sb.make_ligand_pdbqt(24, 5, 11, W.CENTER), 1), q(sb.make_flex_pdbqt(4, 3, W.CENTER), 3))]
    try:
        for k, m in enumerate(models):
            types = sorted({t for t in m.types() if 1 < t < 27})
            eng.build_grids(0, types)
            orc.build_grids(types)
            for t in types:
                g1, c1 = eng.grid(0, t, gd, charged)
                g0, c0 = orc.grid(t, charged)
                assert_bitwise(g1, g0, f"map {t}")
                if charged:
                    assert_bitwise(c1, c0, f"charge map {t}")
            confs = W.random_confs(m, gd, 24, 30 + k)
            for v in ((10, 10, 10), (1000, 1000, 1000)):
                e1, g1 = eng.eval(0, m, confs, v, 1e6)
                e0, g0 = orc.eval(m, confs, v, 1e6)
                assert_bitwise(e1, e0, f"eval energy v={v}")
                assert_bitwise(g1, g0, f"eval gradient v={v}")
            near = W.random_confs(m, gd, 12, 40 + k, spread=0.3)
            e1, g1 = eng.eval_direct(0, m, near, (1000, 1000, 1000), 10.0)
            e0, g0 = orc.eval_direct(m, near, (1000, 1000, 1000), 10.0)
            assert_bitwise(e1, e0, "direct energy")
            assert_bitwise(g1, g0, "direct gradient")
            p = m.search_params()
            c1, e1, x1 = eng.refine(0, [m], [0] * len(near), near, maxiters=p.maxiters)
            c0, e0, x0 = orc.refine([m], [0] * len(near), near, maxiters=p.maxiters)
            assert_bitwise(e1, e0, "refined energies")
            assert_bitwise(c1, c0, "refined confs")
    finally:
        eng.close()


def test_user_grid_changes_maps_and_clearing_restores_them():
    gd = W.box(14.0)
    T = W.tables()
    R = W.receptor(1500, 3)
    m = W.ligand(24, 5, 11)
    types = sorted({t for t in m.types() if 1 < t < 27})
    eng = sb.Engine(0, sb.PREC_FP64)
    try:
        eng.set_tables(T)
        eng.set_receptor(0, R, gd)
        eng.build_grids(0, types)
        plain = [eng.grid(0, t, gd)[0] for t in types]
        eng.set_user_grid(0, *user_grid(*INDEX_GRID))
        eng.build_grids(0, types)
        with_ug = [eng.grid(0, t, gd)[0] for t in types]
        assert all(not np.array_equal(a, b) for a, b in zip(plain, with_ug))
        eng.set_user_grid(0, None, None)
        eng.build_grids(0, types)
        for a, t in zip(plain, types):
            assert_bitwise(eng.grid(0, t, gd)[0], a, f"map {t} after clearing")
        bad_gd, bad = user_grid(*INDEX_GRID)
        with pytest.raises(sb.SminaError):
            eng.set_user_grid(0, bad_gd, np.full_like(bad, np.nan))
        with pytest.raises(ValueError):
            eng.set_user_grid(0, bad_gd, bad[:-1])
    finally:
        eng.close()


def test_user_grid_mixed_precision_eval_within_the_fp32_rule():
    """The FP32 path reads packed copies of maps that carry the user grid:
    its evaluations meet the reference's FP32 rule against the oracle."""
    gd = W.box(14.0)
    T = W.tables()
    ug = user_grid(*INDEX_GRID)
    R = W.receptor(1500, 3)
    eng = sb.Engine(0, sb.PREC_FP32)
    try:
        eng.set_tables(T)
        eng.set_receptor(0, R, gd)
        eng.set_user_grid(0, *ug)
        orc = Oracle(T, R, gd, full_cells=True)
        orc.set_user_grid(*ug)
        m = W.ligand(24, 5, 11)
        confs = W.random_confs(m, gd, 128, 8)
        e1, _ = eng.eval(0, m, confs)
        e0, _ = orc.eval(m, confs)
        rel = np.abs(e1 - e0) / np.maximum(np.abs(e0), 1.0)
        assert (rel <= 1e-4).mean() >= 0.99, np.sort(rel)[-5:]
    finally:
        eng.close()
