"""User grids (--user_grid) in the oracle, checked on the CPU against a
direct numpy restatement of grid::evaluate_aux (grid.cpp:111-236):
cache::populate adds the user grid to every map at the map point's index
coordinates (cache.cpp:204-205, with the cache's slope) and
non_cache::eval_deriv adds it at each heavy atom's coordinates
(non_cache.cpp:180-184).  Without a user grid the oracle is unchanged."""
import numpy as np
import pytest

import smina_b200 as sb
import workloads as W
from oracle_lib import Oracle


def evaluate_user(gd, data, loc, slope, v=1000.0):
    """grid::evaluate_user without derivative: evaluate_aux with curl cap v."""
    n = np.array(gd.n[:], int)
    init, end = np.array(gd.begin[:]), np.array(gd.end[:])
    dfm1 = n.astype(float)
    factor = dfm1 / (end - init)
    s = (np.asarray(loc, float) - init) * factor
    miss = np.zeros(3)
    a = np.zeros(3, int)
    for i in range(3):
        if s[i] < 0:
            miss[i], a[i], s[i] = -s[i], 0, 0.0
        elif s[i] >= dfm1[i]:
            miss[i], a[i], s[i] = s[i] - dfm1[i], n[i] - 1, 1.0
        else:
            a[i] = int(s[i])
            s[i] -= a[i]
    penalty = slope * float(miss @ (1 / factor))
    D = data.reshape(n[2] + 1, n[1] + 1, n[0] + 1)  # [z][y][x]
    f = 0.0
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                w = (s[0] if dx else 1 - s[0]) * (s[1] if dy else 1 - s[1]) * (s[2] if dz else 1 - s[2])
                f += w * D[a[2] + dz, a[1] + dy, a[0] + dx]
    if f > 0:
        f *= v / (v + f)
    return f + penalty


@pytest.fixture(scope="module")
def setup():
    T = W.tables()
    R = W.receptor(1500, 3)
    gd = W.box(12.0)
    return T, R, gd


def _user_grid(lo, hi, n, seed, zero=False):
    g = sb.GridDims()
    for i in range(3):
        g.begin[i], g.end[i], g.n[i] = lo[i], hi[i], n
    data = np.zeros((n + 1) ** 3) if zero else np.random.default_rng(seed).normal(size=(n + 1) ** 3)
    return g, data


def test_maps_gain_the_user_grid_at_index_coordinates(setup):
    T, R, gd = setup
    t = 2  # carbon: every screen ligand needs it
    a = Oracle(T, R, gd)
    a.build_grids([t])
    base, _ = a.grid(t)
    ug, data = _user_grid((-1.0, -1.0, -1.0), (40.0, 40.0, 40.0), 20, 5)
    b = Oracle(T, R, gd)
    b.set_user_grid(ug, data)
    b.build_grids([t])
    with_ug, _ = b.grid(t)
    dims = [gd.n[i] + 1 for i in range(3)]
    rng = np.random.default_rng(1)
    for idx in rng.choice(len(base), 400, replace=False):
        x, y, z = idx % dims[0], (idx // dims[0]) % dims[1], idx // (dims[0] * dims[1])
        u = evaluate_user(ug, data, (x, y, z), 1e6)
        assert abs((with_ug[idx] - base[idx]) - u) <= 1e-9 * max(1.0, abs(base[idx]), abs(u)), (idx, u)


def test_direct_sum_gains_the_user_grid_at_each_heavy_atom(setup):
    T, R, gd = setup
    m = W.ligand(24, 5, 11)
    confs = W.random_confs(m, gd, 16, 3, spread=0.3)
    lo = [gd.begin[i] - 6 for i in range(3)]
    hi = [gd.end[i] + 6 for i in range(3)]
    ug, data = _user_grid(lo, hi, 24, 9)
    a = Oracle(T, R, gd)
    b = Oracle(T, R, gd)
    b.set_user_grid(ug, data)
    v = (1e300, 1e300, 1e300)  # curl of the atom terms is then the identity
    ea, _ = a.eval_direct(m, confs, v=v, slope=10.0)
    eb, _ = b.eval_direct(m, confs, v=v, slope=10.0)
    _, _, xyz = a.eval(m, confs, coords=True)
    heavy = [i for i, t in enumerate(m.types()[:m.num_movable]) if t > 1]
    for k in range(len(confs)):
        u = sum(evaluate_user(ug, data, xyz[k, i], 10.0) for i in heavy)
        assert abs((eb[k] - ea[k]) - u) <= 1e-9 * max(1.0, abs(ea[k]), abs(u)), (k, eb[k] - ea[k], u)


def test_a_zero_user_grid_inside_its_box_changes_nothing(setup):
    T, R, gd = setup
    m = W.ligand(24, 5, 11)
    confs = W.random_confs(m, gd, 8, 4, spread=0.3)
    lo = [gd.begin[i] - 6 for i in range(3)]
    hi = [gd.end[i] + 6 for i in range(3)]
    ug, data = _user_grid(lo, hi, 12, 0, zero=True)
    a = Oracle(T, R, gd)
    b = Oracle(T, R, gd)
    b.set_user_grid(ug, data)
    ea, ga = a.eval_direct(m, confs)
    eb, gb = b.eval_direct(m, confs)
    assert np.array_equal(ea, eb) and np.array_equal(ga, gb)


def test_clearing_the_user_grid_restores_the_maps(setup):
    T, R, gd = setup
    a = Oracle(T, R, gd)
    a.build_grids([2])
    base, _ = a.grid(2)
    ug, data = _user_grid((-1.0, -1.0, -1.0), (40.0, 40.0, 40.0), 8, 2)
    a.set_user_grid(ug, data)
    a.build_grids([2])
    changed, _ = a.grid(2)
    a.set_user_grid(None, None)
    a.build_grids([2])
    again, _ = a.grid(2)
    assert not np.array_equal(base, changed)
    assert np.array_equal(base.view(np.uint64), again.view(np.uint64))
