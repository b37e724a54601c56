"""Flexible receptor side chains (smina --flex): a ligand plus synthetic
flexible residues (first_segment trees, inflex atoms, cross pairs with the
ligand).  The plain FP64 path must match the checker bit for bit (eval,
BFGS, whole chains, refinement); the FP32 path must meet the reference's
FP32 tolerance rule and dock the combined model reproducibly.
"""
import numpy as np
import pytest

import smina_b200 as sb
import workloads as W
from oracle_lib import Oracle
from test_fp32 import at_discontinuity, check_fp32
from test_plain_parity import assert_bitwise


@pytest.fixture(scope="module")
def flex_model():
    flex = sb.make_flex_pdbqt(4, 3, W.CENTER)
    return sb.Model(sb.make_ligand_pdbqt(24, 5, 11, W.CENTER), flex)


def test_flex_model_layout(flex_model):
    """model::append layout: flexible movable atoms, ligand atoms, inflex
    atoms; ligand frames first; one first_segment per residue branch."""
    m = flex_model
    d = m.desc
    kinds = [d.frame_kind[f] for f in range(d.num_frames)]
    assert kinds[0] == 0 and kinds.count(2) == d.num_flex == 4
    mf = d.ligand_atom_begin[0]
    assert mf > 0 and d.ligand_atom_end[0] == d.num_movable < d.num_atoms
    ntors = sum(1 for k in kinds if k != 0)
    assert d.conf_size == 7 + ntors and d.dof == 6 + ntors
    # a residue tree's atoms lie before the ligand's, the ligand tree's after
    for f in range(d.num_frames):
        root = f
        while d.frame_parent[root] >= 0:
            root = d.frame_parent[root]
        if kinds[root] == 2:
            assert d.frame_end[f] <= mf
        else:
            assert d.frame_begin[f] >= mf
    # cross pairs: every typed residue atom (movable and inflex) with every ligand atom
    pairs = np.ctypeslib.as_array(d.pairs, shape=(2 * d.num_pairs,)).reshape(-1, 2)
    lig = set(range(mf, d.num_movable))
    cross = [(a, b) for a, b in pairs[:d.num_other_pairs] if (a in lig) != (b in lig)]
    n_res_atoms = d.num_atoms - (d.num_movable - mf)
    assert len(cross) == n_res_atoms * (d.num_movable - mf)


@pytest.mark.gpu
def test_flex_plain_path_bit_exact(flex_model):
    m = flex_model
    T, R, gd = W.tables(), W.receptor(), W.box()
    eng = sb.Engine(0, sb.PREC_FP64)
    eng.set_tables(T)
    eng.set_receptor(0, R, gd)
    orc = Oracle(T, R, gd, full_cells=True)
    confs = W.random_confs(m, gd, 48, 31)
    e1, g1, x1 = eng.eval(0, m, confs, coords=True)
    e0, g0, x0 = orc.eval(m, confs, coords=True)
    assert_bitwise(x1, x0, "coords")
    assert_bitwise(e1, e0, "energy")
    assert_bitwise(g1, g0, "gradient")
    c1, b1 = eng.bfgs(0, m, confs[:16], maxiters=20)
    c0, b0 = orc.bfgs(m, confs[:16], maxiters=20)
    assert_bitwise(b1, b0, "bfgs energy")
    assert_bitwise(c1, c0, "bfgs conf")
    p = m.search_params()
    cs, mts = m.seed_chains(9, 4, gd)
    d1 = eng.dock(0, [m], [0] * 4, cs, mts, p, steps=15)
    d0 = orc.dock([m], [0] * 4, cs, mts, p, steps=15, threads=4)
    assert (d1.count == d0.count).all() and (d1.evals == d0.evals).all()
    assert_bitwise(d1.e, d0.e, "chain energies")
    e, conf, _ = sb.merge_chains(d1, m)
    r1 = eng.refine(0, [m], np.zeros(len(e), np.int32), conf, maxiters=p.maxiters)
    r0 = orc.refine([m], np.zeros(len(e), np.int32), conf, maxiters=p.maxiters)
    assert_bitwise(r1[1], r0[1], "refined energies")


@pytest.mark.gpu
def test_flex_fp32_eval_and_batched_search(flex_model):
    m = flex_model
    T, R, gd = W.tables(), W.receptor(), W.box()
    eng = sb.Engine(0, sb.PREC_FP32)
    eng.set_tables(T)
    eng.set_receptor(0, R, gd)
    orc = Oracle(T, R, gd, full_cells=True)
    confs = W.random_confs(m, gd, 256, 41)
    e32, g32 = eng.eval(0, m, confs)
    e64, g64, x64 = orc.eval(m, confs, coords=True)
    check_fp32(e32, g32, e64, g64, at_discontinuity(m, gd, x64, T.desc.cutoff_sqr))
    p = m.search_params()
    job = sb.LigandJob(model=0, num_chains=4, num_steps=20, maxiters=0, seed=5, ligand_key=77)
    a = eng.dock_batch(0, [m], [job], p)[0]
    b = eng.dock_batch(0, [m, W.ligand(24, 5, 11)], [job, sb.LigandJob(model=1, num_chains=4, num_steps=20,
                                                                       maxiters=0, seed=5, ligand_key=78)], p)[0]
    assert len(a["e"]) > 0
    for k in ("e", "conf", "coords"):
        assert np.array_equal(a[k], b[k]), k
