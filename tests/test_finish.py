"""Final rescoring and clustering of docked poses (finish_docking,
src/main/main.cpp:257-324).

CPU: the conf-independent inputs the PDBQT reader derives (terms.cpp:83-120,
model.cpp:62-109) against an independent reading of the PDBQT text; the
conf-independent terms (everything.h:730-1000) against a restatement here;
sgh_finish_docking's sort / rescore / remove_redundant / num_modes logic
against a restatement here.  GPU: sg_score's energies (model::eval on the
direct sum and model::eval_intramolecular, fast table) bit for bit against
the checker, for ligands, charge-dependent tables and flexible residues.
"""
import math

import numpy as np
import pytest

import smina_b200 as sb
import workloads as W
from oracle_lib import Oracle
from test_plain_parity import assert_bitwise


# ---- conf-independent inputs -----------------------------------------------------------
def _read(pdbqt):
    """Atoms (element, xyz), BRANCH bonds and the branch tree of a PDBQT text."""
    atoms, serial_to_idx, rot, parent, stack, frame_of = [], {}, [], [-1], [0], []
    for line in pdbqt.splitlines():
        if line.startswith(("ATOM", "HETATM")):
            serial = int(line[6:11])
            xyz = np.array([float(line[30:38]), float(line[38:46]), float(line[46:54])])
            el = {"A": "C", "NA": "N", "NS": "N", "OA": "O", "OS": "O", "SA": "S", "HD": "H", "HS": "H", "CL": "Cl",
                  "BR": "Br"}.get(line[77:79].strip(), line[77:79].strip())
            serial_to_idx[serial] = len(atoms)
            atoms.append((el, xyz))
            frame_of.append(stack[-1])
        elif line.startswith("BRANCH"):
            a, b = int(line.split()[1]), int(line.split()[2])
            rot.append((a, b))
            parent.append(stack[-1])
            stack.append(len(parent) - 1)
        elif line.startswith("ENDBRANCH"):
            stack.pop()
    rot = [(serial_to_idx[a], serial_to_idx[b]) for a, b in rot]
    return atoms, rot, parent


def _expected_inputs(pdbqt):
    atoms, rot, parent = _read(pdbqt)
    heavy = [i for i, (el, _) in enumerate(atoms) if el != "H"]
    cov = {"C": 0.77, "N": 0.75, "O": 0.73, "S": 1.02, "F": 0.71, "Cl": 0.99, "Br": 1.14, "I": 1.33, "H": 0.37,
           "P": 1.06}
    nb = {i: [] for i in range(len(atoms))}
    for i in range(len(atoms)):
        for j in range(i + 1, len(atoms)):
            d = np.linalg.norm(atoms[i][1] - atoms[j][1])
            if d < 1.1 * (cov[atoms[i][0]] + cov[atoms[j][0]]):
                nb[i].append(j)
                nb[j].append(i)
    nbh = {i: sum(1 for j in nb[i] if j in heavy) for i in nb}
    rotset = {frozenset(p) for p in rot}
    num_tors = num_rotors = 0.0
    for i in heavy:
        ar = sum(1 for j in nb[i] if frozenset((i, j)) in rotset and j in heavy and nbh[j] > 1 and nbh[i] > 1)
        num_tors += 0.5 * ar
        num_rotors += 0.5 if ar > 2 else 0.5 * ar

    def metrics(f):
        kids = [c for c in range(len(parent)) if parent[c] == f]
        if not kids:
            return 0, 0
        res = [metrics(c) for c in kids]
        lengths = sorted(r[0] + 1 for r in res)
        length = lengths[-1]
        c2c = length + (lengths[-1] if len(lengths) >= 2 else 0)
        return length, max(c2c, max(r[1] for r in res))

    return num_tors, num_rotors, len(heavy), metrics(0)[1]


@pytest.mark.parametrize("heavy,rotors,seed", [(5, 1, 3), (24, 5, 11), (12, 0, 3), (40, 10, 5), (30, 12, 7)])
def test_conf_independent_inputs_follow_the_tree(heavy, rotors, seed):
    text = sb.make_ligand_pdbqt(heavy, rotors, seed, W.CENTER)
    got = sb.Model(text).conf_independent_inputs()
    tors, rotors_w, nheavy, length = _expected_inputs(text)
    assert got[0] == tors and got[1] == rotors_w and got[2] == nheavy == heavy
    assert got[5] == 1 and got[6] == length
    assert 0 <= got[3] <= nheavy and 0 <= got[4] <= nheavy


def test_flex_model_counts_only_ligand_atoms():
    text = sb.make_ligand_pdbqt(24, 5, 11, W.CENTER)
    lig = sb.Model(text).conf_independent_inputs()
    both = sb.Model(text, sb.make_flex_pdbqt(4, 3, W.CENTER)).conf_independent_inputs()
    assert np.array_equal(lig, both)


# ---- conf-independent terms --------------------------------------------------------------
def _smooth_div(x, y):
    if abs(x) < 2.220446049250313e-16:
        return 0.0
    if abs(y) < 2.220446049250313e-16:
        return 1.7976931348623157e308 if x * y > 0 else -1.7976931348623157e308
    return x / y


def _conf_indep(terms, inp, x):
    nt, _, nh, nhyd, _, nl, ll = inp
    for name, r in terms:
        if name == "num_tors_add":
            x = x + r * nt
        elif name == "num_tors_sqr":
            x = x + 0.1 * r * (nt * nt) / 5
        elif name == "num_tors_sqrt":
            x = x + 0.1 * r * math.sqrt(nt) / math.sqrt(5.0)
        elif name == "num_tors_div":
            x = _smooth_div(x, 1 + 0.1 * (r + 1) * nt / 5.0)
        elif name == "num_tors_div_simple":
            x = _smooth_div(x, 1 + r * nt)
        elif name == "ligand_length":
            x = x + r * ll
        elif name == "num_ligands":
            x = x + 1 * r * nl
        elif name == "num_heavy_atoms_div":
            x = _smooth_div(x, 1 + 0.05 * r * nh)
        elif name == "num_heavy_atoms":
            x = x + 0.05 * r * nh
        elif name == "num_hydrophobic_atoms":
            x = x + 0.05 * r * nhyd
        elif name == "constant_term":
            x = x + r
    return x


def test_vina_conf_independent_is_num_tors_div():
    T = sb.Tables("vina")
    inp = sb.Model(sb.make_ligand_pdbqt(40, 10, 5, W.CENTER)).conf_independent_inputs()
    w = 5 * 0.05846 / 0.1 - 1  # builtinscoring.cpp's num_tors_div weight
    for x in (-12.5, -3.25, 0.0, 4.0, 1e-20):
        assert T.conf_independent(inp, x) == _conf_indep([("num_tors_div", w)], inp, x)


def test_custom_conf_independent_terms_in_file_order():
    terms = [("num_tors_add", 0.2744), ("num_tors_sqr", 0.317267), ("num_tors_sqrt", -0.11),
             ("num_heavy_atoms_div", 0.3), ("num_heavy_atoms", -0.02), ("num_hydrophobic_atoms", 0.07),
             ("ligand_length", 0.01), ("num_ligands", 0.5), ("num_tors_div_simple", 0.04), ("constant_term", -0.25),
             ("num_tors_div", 0.9)]
    text = "-0.0356 gauss(o=0,_w=0.5,_c=8)\n" + "".join(f"{w} {n}\n" for n, w in terms)
    T = sb.Tables("vina", custom_text=text)
    inp = sb.Model(sb.make_ligand_pdbqt(30, 12, 7, W.CENTER)).conf_independent_inputs()
    for x in (-9.75, -0.5, 2.0):
        assert T.conf_independent(inp, x) == _conf_indep(terms, inp, x)


# ---- finish_docking ----------------------------------------------------------------------
def _finish(T, inp, er, et, ei, xyz, min_rmsd, num_modes, erange):
    MAX = 1.7976931348623157e308
    not_max = lambda x: x < 0.1 * MAX  # noqa: E731
    n = len(er)
    order = sorted(range(n), key=lambda k: er[k])
    intra = ei[order[0]]
    e = [T.conf_independent(inp, et[k] - intra) if not_max(er[k]) else er[k] for k in range(n)]
    order = sorted(order, key=lambda k: e[k])
    H = xyz.shape[1]
    rmsd = lambda a, b: math.sqrt(sum(((xyz[a] - xyz[b]) ** 2).ravel().tolist()) / H)  # noqa: E731
    kept = []
    for k in order:
        best = None
        for i, j in enumerate(kept):
            r = rmsd(k, j)
            if best is None or r < best[1]:
                best = (i, r)
        if best is not None and best[1] < min_rmsd:
            if e[k] < e[kept[best[0]]]:
                kept[best[0]] = k
        elif len(kept) < n:
            kept.append(k)
        elif kept and e[k] < e[kept[-1]]:
            kept[-1] = k
        kept.sort(key=lambda j: e[j])
    out = []
    for j in kept:
        if len(out) >= num_modes or not not_max(e[j]) or e[j] > e[kept[0]] + erange:
            break
        out.append(j)
    return out, [e[j] for j in out]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_finish_docking_sorts_rescores_clusters_and_cuts(seed):
    rng = np.random.default_rng(seed)
    T = sb.Tables("vina")
    inp = sb.Model(sb.make_ligand_pdbqt(24, 5, 11, W.CENTER)).conf_independent_inputs()
    n, H = 20, 24
    centres = rng.normal(size=(5, H, 3)) * 3
    xyz = centres[rng.integers(0, 5, n)] + rng.normal(size=(n, H, 3)) * rng.choice([0.05, 1.5], n)[:, None, None]
    er = rng.uniform(-11, -6, n)
    er[rng.integers(0, n)] = 1.7976931348623157e308  # a pose that never got inside the box
    et = er + rng.uniform(-1, 1, n)
    ei = rng.uniform(-2, 1, n)
    for num_modes, erange in ((9, 3.0), (3, 1.0), (20, 10.0)):
        idx, e = T.finish_docking(inp, er, et, ei, xyz, 1.0, num_modes, erange)
        ridx, re = _finish(T, inp, er, et, ei, xyz, 1.0, num_modes, erange)
        assert list(idx) == ridx and list(e) == re
        assert len(idx) <= num_modes and np.all(np.diff(e) >= 0)


# ---- sg_score on the GPU -----------------------------------------------------------------
@pytest.fixture(scope="module")
def setup():
    T, R, gd = W.tables(), W.receptor(), W.box()
    eng = sb.Engine(0, sb.PREC_FP64)
    eng.set_tables(T)
    eng.set_receptor(0, R, gd)
    return eng, Oracle(T, R, gd, full_cells=True), gd


@pytest.mark.gpu
def test_score_bit_exact(setup):
    eng, orc, gd = setup
    models = [W.ligand(24, 5, 11), W.ligand(12, 0, 3), W.ligand(40, 10, 5),
              sb.Model(sb.make_ligand_pdbqt(24, 5, 11, W.CENTER), sb.make_flex_pdbqt(4, 3, W.CENTER))]
    confs, pm = [], []
    for k, m in enumerate(models):
        for c in W.random_confs(m, gd, 6, 40 + k):
            cm = np.zeros(max(x.conf_size for x in models))
            cm[:m.conf_size] = c
            confs.append(cm)
            pm.append(k)
    for v, slope in (((1000, 1000, 1000), 1e6), ((10, 1.5, 10), 10.0)):
        e1, i1, x1 = eng.score(0, models, pm, confs, v, slope)
        e0, i0, x0 = orc.score(models, pm, confs, v, slope)
        assert_bitwise(e1, e0, f"e_total v={v}")
        assert_bitwise(i1, i0, f"e_intra v={v}")
        assert_bitwise(x1, x0, "coords")
    assert np.any(i0[-6:] != 0)  # the flexible residues' intramolecular part is exercised


@pytest.mark.gpu
def test_score_charge_dependent_tables_bit_exact():
    T4, R, gd = sb.Tables("ad4_scoring"), W.charged_receptor(), W.box()
    eng = sb.Engine(0, sb.PREC_FP64)
    eng.set_tables(T4)
    eng.set_receptor(0, R, gd)
    orc = Oracle(T4, R, gd, full_cells=True)
    m = W.charged_ligand(24, 5, 11)
    confs = W.random_confs(m, gd, 16, 9)
    e1, i1, _ = eng.score(0, [m], [0] * 16, confs)
    e0, i0, _ = orc.score([m], [0] * 16, confs)
    assert_bitwise(e1, e0, "e_total")
    assert_bitwise(i1, i0, "e_intra")


@pytest.mark.gpu
def test_dock_score_finish_end_to_end(setup):
    """dock_batch poses -> sg_score -> sgh_finish_docking, against the checker's
    energies of the same poses through the same finish logic."""
    eng32 = sb.Engine(0, sb.PREC_FP32)
    T, R, gd = W.tables(), W.receptor(), W.box()
    eng32.set_tables(T)
    eng32.set_receptor(0, R, gd)
    _, orc, _ = setup
    m = W.ligand(24, 5, 11)
    p = m.search_params()
    job = sb.LigandJob(model=0, num_chains=4, num_steps=40, maxiters=0, seed=3, ligand_key=5)
    r = eng32.dock_batch(0, [m], [job], p)[0]
    n = len(r["e"])
    assert n > 0
    e1, i1, x1 = eng32.score(0, [m], [0] * n, r["conf"])
    e0, i0, x0 = orc.score([m], [0] * n, r["conf"])
    assert_bitwise(e1, e0, "e_total")
    assert_bitwise(i1, i0, "e_intra")
    inp = m.conf_independent_inputs()
    idx, e = T.finish_docking(inp, r["e"], e1, i1, r["coords"])
    ridx, re = _finish(T, inp, r["e"], e0, i0, r["coords"], 1.0, 9, 3.0)
    assert list(idx) == ridx and list(e) == re and len(idx) > 0
