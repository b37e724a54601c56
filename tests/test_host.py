"""Host library: PDBQT torsion trees, typing, pair lists, tables and search
parameters, checked against smina's documented rules on small inputs."""
import math

import numpy as np
import pytest

import smina_b200 as sb
import workloads as W

LIG = """REMARK tiny test ligand
ROOT
ATOM      1  C1  LIG A   1       0.000   0.000   0.000  1.00  0.00    +0.000 C
ATOM      2  C2  LIG A   1       1.540   0.000   0.000  1.00  0.00    +0.000 C
ENDROOT
BRANCH   2   3
ATOM      3  C3  LIG A   1       2.053   1.452   0.000  1.00  0.00    +0.000 C
ATOM      4  O4  LIG A   1       3.483   1.452   0.000  1.00  0.00    +0.000 OA
ATOM      5  H5  LIG A   1       3.816   2.395   0.000  1.00  0.00    +0.000 HD
BRANCH   3   6
ATOM      6  C6  LIG A   1       1.540   2.178   1.258  1.00  0.00    +0.000 C
ATOM      7  N7  LIG A   1       1.540   3.648   1.258  1.00  0.00    +0.000 NA
ENDBRANCH   3   6
ENDBRANCH   2   3
BRANCH   1   8
ATOM      8  C8  LIG A   1      -0.513  -1.452   0.000  1.00  0.00    +0.000 C
ATOM      9  H9  LIG A   1      -1.513  -1.452   0.000  1.00  0.00    +0.000 HD
ENDBRANCH   1   8
TORSDOF 2
"""


def test_tree_layout_follows_smina():
    m = sb.Model(LIG)
    d = m.desc
    # branch 1->8 moves only hydrogens besides its axis atom: merged (parse_pdbqt.cpp:239-244)
    assert d.num_frames == 3
    assert m.conf_size == 7 + 2 and m.dof == 6 + 2
    kinds = [d.frame_kind[f] for f in range(3)]
    parents = [d.frame_parent[f] for f in range(3)]
    assert kinds == [0, 1, 1] and parents == [-1, 0, 1]
    # each branch's axis atom lives in its parent's frame (parsing.h:136-146)
    ranges = [(d.frame_begin[f], d.frame_end[f]) for f in range(3)]
    assert ranges[0][0] == 0 and ranges[1][0] == ranges[0][1] and ranges[2][0] == ranges[1][1]
    assert m.num_movable == 9 and m.heavy == 7
    # typing (adjust_smina_type): O bonded to HD is a donor-acceptor; C bonded to O is not hydrophobic
    types = m.types()
    assert 12 in types  # OxygenXSDonorAcceptor
    assert 3 in types  # AliphaticCarbonXSNonHydrophobe


def test_pairs_exclude_near_bonded_and_rigid():
    m = sb.Model(LIG)
    d = m.desc
    pairs = [(d.pairs[2 * k], d.pairs[2 * k + 1]) for k in range(d.num_pairs)]
    assert pairs == sorted(pairs)
    for a, b in pairs:
        assert d.atom_type[a] > 1 and d.atom_type[b] > 1  # no hydrogens
        fa = next(f for f in range(d.num_frames) if d.frame_begin[f] <= a < d.frame_end[f])
        fb = next(f for f in range(d.num_frames) if d.frame_begin[f] <= b < d.frame_end[f])
        assert fa != fb  # atoms of one rigid fragment never pair


def test_generated_ligands_have_requested_shape():
    for heavy, rotors, seed in [(24, 5, 11), (10, 0, 1), (50, 12, 4)]:
        m = W.ligand(heavy, rotors, seed)
        assert m.heavy == heavy
        assert m.dof == 6 + rotors
        assert m.torsdof == rotors


def test_search_params_formula():
    m = W.ligand(24, 5, 11)
    p = m.search_params()
    heuristic = m.num_movable + 10 * m.dof
    assert p.num_steps == 70 * 3 * (50 + heuristic) // 2
    assert p.maxiters == (25 + m.num_movable) // 3
    assert p.num_saved_mins == 20 and p.min_rmsd == 1.0
    assert list(p.hunt_cap) == [10, 10, 10]


def _vina_pair(t1, t2, r):
    """Independent restatement of vina's weighted terms for two atom types."""
    xs = {2: 1.9, 3: 1.9, 6: 1.8, 7: 1.8, 8: 1.8, 9: 1.8, 10: 1.7, 11: 1.7, 12: 1.7, 13: 1.7}
    hyd = {2}
    don = {7, 8, 11, 12}
    acc = {8, 9, 12, 13}
    s = r - (xs[t1] + xs[t2])
    g1 = math.exp(-(s / 0.5) ** 2)
    g2 = math.exp(-((s - 3) / 2.0) ** 2)
    rep = s * s if s < 0 else 0.0

    def step(bad, good, x):
        if bad < good:
            return 0.0 if x <= bad else 1.0 if x >= good else (x - bad) / (good - bad)
        return 0.0 if x >= bad else 1.0 if x <= good else (x - bad) / (good - bad)
    h = step(1.5, 0.5, s) if (t1 in hyd and t2 in hyd) else 0.0
    hb = step(0, -0.7, s) if ((t1 in don and t2 in acc) or (t2 in don and t1 in acc)) else 0.0
    return -0.035579 * g1 - 0.005156 * g2 + 0.840245 * rep - 0.035069 * h - 0.587439 * hb


def test_vina_tables_match_independent_terms():
    T = W.tables()
    d = T.desc
    n = d.n
    smooth = np.ctypeslib.as_array(d.smooth, shape=(351 + 27, n, 1, 2))
    fast = np.ctypeslib.as_array(d.fast, shape=(378, n, 1))
    assert n == int(32 * 64) + 3
    for t1, t2 in [(2, 2), (2, 13), (8, 12), (3, 9), (7, 13)]:
        p = t1 + t2 * (t2 + 1) // 2
        for i in (1, 17, 200, 1000, 2000):
            r = math.sqrt(i / 32.0)
            assert smooth[p, i, 0, 0] == pytest.approx(_vina_pair(t1, t2, r), rel=1e-12, abs=1e-14)
        # dor is the centred difference over r, fast the midpoint (precalculate.h:153-180)
        i = 300
        rs = [math.sqrt(k / 32.0) for k in (i - 1, i, i + 1)]
        dor = (smooth[p, i + 1, 0, 0] - smooth[p, i - 1, 0, 0]) / ((rs[2] - rs[0]) * rs[1])
        assert smooth[p, i, 0, 1] == pytest.approx(dor, rel=1e-12)
        assert fast[p, i, 0] == pytest.approx((smooth[p, i, 0, 0] + smooth[p, i + 1, 0, 0]) / 2, rel=1e-14)


def test_custom_scoring_matches_builtin():
    text = ("-0.035579 gauss(o=0,_w=0.5,_c=8)\n-0.005156 gauss(o=3,_w=2,_c=8)\n0.840245 repulsion(o=0,_c=8)\n"
            "-0.035069 hydrophobic(g=0.5,_b=1.5,_c=8)\n-0.587439 non_dir_h_bond(g=-0.7,_b=0,_c=8)\n"
            "1.923 num_tors_div\n")
    a, b = W.tables(), W.custom_tables(text)
    n = a.desc.n
    sa = np.ctypeslib.as_array(a.desc.smooth, shape=(378 * n * 2,))
    sb_ = np.ctypeslib.as_array(b.desc.smooth, shape=(378 * n * 2,))
    assert np.array_equal(sa, sb_)


def test_charge_dependent_tables_have_four_components():
    t = sb.Tables("ad4_scoring")
    assert t.desc.num_components == 4


def test_box_dims():
    gd = W.box(22.0)
    assert list(gd.n) == [59, 59, 59]
    assert gd.end[0] - gd.begin[0] == pytest.approx(59 * 0.375)


def test_chain_seeding_deterministic():
    m = W.ligand()
    gd = W.box()
    c1, m1 = m.seed_chains(42, 4, gd)
    c2, m2 = m.seed_chains(42, 4, gd)
    assert np.array_equal(c1, c2) and np.array_equal(m1, m2)
    q = c1[:, 3:7]
    assert np.allclose(np.linalg.norm(q, axis=1), 1.0)
    lo, hi = np.array(gd.begin[:]), np.array(gd.end[:])
    assert ((c1[:, :3] >= lo) & (c1[:, :3] <= hi)).all()
    assert (np.abs(c1[:, 7:]) <= np.pi).all()
