"""SDF / MOL ligands (sgh_pdbqt_from_sdf, sgh_model_from_sdf): the
reference's OpenBabel route (molgetter.cpp:103-125 through its converter,
SminaConverter.cpp:87-130, PDBQTUtilities.cpp:50-627) restated without
OpenBabel.  Checked here on molecules written by the test: typing (aromatic
carbon, acceptor nitrogen, polar hydrogens), rotatable bonds (single, not
amide, not in a ring, both ends with another heavy neighbour), the root
(the atom whose removal leaves the smallest largest piece), non-polar
hydrogens deleted with their charge moved to their heavy atom, Gasteiger
charges that sum to the formal charge, a salt stripped to its largest
piece, records of a multi-record file,
V3000 records read as their V2000 twins, and a round trip of the synthetic
ligands (PDBQT -> SDF -> PDBQT) that keeps every heavy atom where it was and
yields a model.
"""
import numpy as np
import pytest

import smina_b200 as sb

COV = {"C": 0.77, "N": 0.75, "O": 0.73, "S": 1.02, "H": 0.37, "Cl": 0.99, "F": 0.71, "Br": 1.14, "I": 1.33, "P": 1.06}


def sdf(name, atoms, bonds, charges=()):
    """V2000 record: atoms (element, x, y, z), bonds (i, j, order) 1-based."""
    out = [name, "  test", "", f"{len(atoms):3d}{len(bonds):3d}  0  0  0  0  0  0  0  0999 V2000"]
    for el, x, y, z in atoms:
        out.append(f"{x:10.4f}{y:10.4f}{z:10.4f} {el:<3} 0  0  0  0  0  0  0  0  0  0  0  0")
    for i, j, o in bonds:
        out.append(f"{i:3d}{j:3d}{o:3d}  0")
    if charges:
        out.append(f"M  CHG{len(charges):3d}" + "".join(f"{a:4d}{c:4d}" for a, c in charges))
    out.append("M  END")
    return "\n".join(out) + "\n$$$$\n"


def atoms_of(pdbqt):
    rows = []
    for line in pdbqt.splitlines():
        if line.startswith("ATOM"):
            rows.append((int(line[6:11]), line[77:79].strip(), float(line[30:38]), float(line[38:46]),
                         float(line[46:54]), float(line[68:76])))
    return rows


def torsdof(pdbqt):
    return int([ln for ln in pdbqt.splitlines() if ln.startswith("TORSDOF")][0].split()[1])


def chain(elements, step=1.53):
    """Atoms along a zig-zag, bonded in order."""
    atoms = [(el, 1.25 * k, 0.8 * (k % 2), 0.0) for k, el in enumerate(elements)]
    return atoms, [(k + 1, k + 2, 1) for k in range(len(elements) - 1)]


def ring6(el="C", r=1.39, z=0.0):
    return [(el, r * np.cos(np.pi / 3 * k), r * np.sin(np.pi / 3 * k), z) for k in range(6)]


def test_butane_one_torsion_about_its_centre():
    atoms, bonds = chain(["C", "C", "C", "C"])
    p = sb.pdbqt_from_sdf(sdf("butane", atoms, bonds))
    assert torsdof(p) == 1  # only C2-C3: the end bonds have a one-heavy-neighbour atom
    rows = atoms_of(p)
    assert [r[1] for r in rows] == ["C"] * 4
    lines = p.splitlines()
    root = lines[lines.index("ROOT") + 1:lines.index("ENDROOT")]
    assert len(root) == 2 and any(ln.startswith("BRANCH") for ln in lines)
    m = sb.Model(p)
    assert m.torsdof == 1


def test_toluene_aromatic_carbons_no_torsions():
    ring = ring6()
    atoms = ring + [("C", 2.9, 0.0, 0.0)]
    bonds = [(1, 2, 2), (2, 3, 1), (3, 4, 2), (4, 5, 1), (5, 6, 2), (6, 1, 1), (1, 7, 1)]
    p = sb.pdbqt_from_sdf(sdf("toluene", atoms, bonds))
    types = [r[1] for r in atoms_of(p)]
    assert types.count("A") == 6 and types.count("C") == 1
    assert torsdof(p) == 0
    # the same ring typed aromatic (bond type 4) in the file
    bonds4 = [(i, i % 6 + 1, 4) for i in range(1, 7)] + [(1, 7, 1)]
    assert [r[1] for r in atoms_of(sb.pdbqt_from_sdf(sdf("toluene4", atoms, bonds4)))].count("A") == 6


def test_cyclohexane_is_not_aromatic():
    atoms = ring6(r=1.53)
    bonds = [(i, i % 6 + 1, 1) for i in range(1, 7)]
    assert [r[1] for r in atoms_of(sb.pdbqt_from_sdf(sdf("chx", atoms, bonds)))] == ["C"] * 6


def test_pyridine_and_pyrrole_nitrogens():
    pyr = ring6()
    pyr[0] = ("N",) + pyr[0][1:]
    bonds = [(1, 2, 2), (2, 3, 1), (3, 4, 2), (4, 5, 1), (5, 6, 2), (6, 1, 1)]
    t = [r[1] for r in atoms_of(sb.pdbqt_from_sdf(sdf("pyridine", pyr, bonds)))]
    assert t.count("NA") == 1 and t.count("A") == 5
    five = [(("N" if k == 0 else "C"), 1.2 * np.cos(2 * np.pi / 5 * k), 1.2 * np.sin(2 * np.pi / 5 * k), 0.0)
            for k in range(5)]
    five.append(("H", 2.2, 0.0, 0.0))  # N-H
    bonds5 = [(1, 2, 1), (2, 3, 2), (3, 4, 1), (4, 5, 2), (5, 1, 1), (1, 6, 1)]
    t5 = [r[1] for r in atoms_of(sb.pdbqt_from_sdf(sdf("pyrrole", five, bonds5)))]
    assert t5.count("N") == 1 and t5.count("A") == 4 and t5.count("HD") == 1


def test_amide_bond_is_not_rotatable_and_its_nitrogen_is_not_an_acceptor():
    # CH3-C(=O)-NH-CH2-CH3: C(=O)-N is the amide; N-C(ethyl) rotates
    atoms = [("C", 0.0, 0.0, 0.0), ("C", 1.5, 0.0, 0.0), ("O", 2.1, 1.05, 0.0), ("N", 2.2, -1.2, 0.0),
             ("C", 3.65, -1.25, 0.0), ("C", 4.2, -2.6, 0.3), ("H", 1.7, -2.05, 0.0)]
    bonds = [(1, 2, 1), (2, 3, 2), (2, 4, 1), (4, 5, 1), (5, 6, 1), (4, 7, 1)]
    p = sb.pdbqt_from_sdf(sdf("nma", atoms, bonds))
    t = [r[1] for r in atoms_of(p)]
    assert t.count("N") == 1 and t.count("OA") == 1 and t.count("HD") == 1
    assert torsdof(p) == 1  # N-CH2 only (amide and the terminal bonds do not rotate)


def test_hydrogens_added_and_nonpolar_ones_deleted():
    # ethanol without hydrogens: the hydroxyl gets one (HD); carbon ones never appear
    atoms, bonds = chain(["C", "C", "O"])
    rows = atoms_of(sb.pdbqt_from_sdf(sdf("ethanol", atoms, bonds)))
    assert [r[1] for r in rows].count("HD") == 1 and len(rows) == 4
    o = [r for r in rows if r[1] == "OA"][0]
    h = [r for r in rows if r[1] == "HD"][0]
    assert abs(np.linalg.norm(np.subtract(o[2:5], h[2:5])) - 1.0) < 2e-3
    assert len(atoms_of(sb.pdbqt_from_sdf(sdf("ethanol", atoms, bonds), add_hydrogens=False))) == 3
    # explicit hydrogens: the carbon ones go, their charge moves to the carbon
    atoms_h = atoms + [("H", -0.5, -0.9, 0.0), ("H", -0.5, 0.5, 0.9), ("H", -0.5, 0.5, -0.9),
                       ("H", 1.25, 1.4, 0.9), ("H", 1.25, 1.4, -0.9), ("H", 3.0, 1.3, 0.0)]
    bonds_h = bonds + [(1, 4, 1), (1, 5, 1), (1, 6, 1), (2, 7, 1), (2, 8, 1), (3, 9, 1)]
    rows_h = atoms_of(sb.pdbqt_from_sdf(sdf("ethanol-h", atoms_h, bonds_h)))
    assert len(rows_h) == 4 and [r[1] for r in rows_h].count("HD") == 1
    assert abs(sum(r[5] for r in rows_h)) < 2e-3  # neutral: the kept charges sum to 0 (3 decimals each)


PEOE = {"C3": (7.98, 9.18, 1.88), "H": (7.17, 6.24, -0.56), "O3": (14.18, 12.92, 1.39)}


def peoe(el, bonds):
    """Gasteiger-Marsili PEOE (6 rounds, damping 1/2), restated for the check."""
    q = [0.0] * len(el)
    damp = 1.0
    for _ in range(6):
        damp *= 0.5
        chi = [PEOE[e][0] + q[i] * (PEOE[e][1] + q[i] * PEOE[e][2]) for i, e in enumerate(el)]
        dq = [0.0] * len(el)
        for i, j in bonds:
            lo, hi = (i, j) if chi[i] < chi[j] else (j, i)
            t = (chi[hi] - chi[lo]) / (20.02 if el[lo] == "H" else sum(PEOE[el[lo]])) * damp
            dq[lo] += t
            dq[hi] -= t
        q = [a + b for a, b in zip(q, dq)]
    return q


def test_gasteiger_charges():
    # the method's published charges for methane: C -0.078, H +0.019
    q = peoe(["C3", "H", "H", "H", "H"], [(0, k) for k in range(1, 5)])
    assert abs(q[0] + 0.078) < 5e-4 and abs(q[1] - 0.019) < 5e-4
    atoms = [("C", 0, 0, 0), ("H", 0.63, 0.63, 0.63), ("H", -0.63, -0.63, 0.63), ("H", -0.63, 0.63, -0.63),
             ("H", 0.63, -0.63, -0.63)]
    rows = atoms_of(sb.pdbqt_from_sdf(sdf("methane", atoms, [(1, k, 1) for k in range(2, 6)])))
    assert len(rows) == 1 and abs(rows[0][5]) < 1e-3  # hydrogens folded into the carbon: neutral
    # methanol with explicit hydrogens: the kept atoms carry the restated charges
    # (the carbon's with its three hydrogens folded in)
    atoms = [("C", 0, 0, 0), ("O", 1.43, 0, 0), ("H", 1.75, 0.9, 0), ("H", -0.36, 1.03, 0), ("H", -0.36, -0.5, 0.9),
             ("H", -0.36, -0.5, -0.9)]
    bonds = [(1, 2, 1), (2, 3, 1), (1, 4, 1), (1, 5, 1), (1, 6, 1)]
    q = peoe(["C3", "O3", "H", "H", "H", "H"], [(i - 1, j - 1) for i, j, _ in bonds])
    rows = atoms_of(sb.pdbqt_from_sdf(sdf("methanol", atoms, bonds)))
    got = {r[1]: r[5] for r in rows}
    assert abs(got["C"] - (q[0] + q[3] + q[4] + q[5])) < 1e-3
    assert abs(got["OA"] - q[1]) < 1e-3 and abs(got["HD"] - q[2]) < 1e-3
    # acetate: formal charge -1 on one oxygen, charges sum to -1
    atoms = [("C", 0, 0, 0), ("C", 1.5, 0, 0), ("O", 2.1, 1.05, 0), ("O", 2.1, -1.05, 0)]
    bonds = [(1, 2, 1), (2, 3, 2), (2, 4, 1)]
    rows = atoms_of(sb.pdbqt_from_sdf(sdf("acetate", atoms, bonds, charges=[(4, -1)])))
    assert abs(sum(r[5] for r in rows) + 1) < 3e-3
    ox = [r[5] for r in rows if r[1] == "OA"]
    assert len(ox) == 2 and all(q < 0 for q in ox)
    carbonyl = [r[5] for r in rows if r[1] == "C"]
    assert max(carbonyl) > 0  # the carboxyl carbon gives electrons to its oxygens


def test_records_of_a_file():
    a1, b1 = chain(["C", "C", "C", "C"])
    a2, b2 = chain(["C", "C", "O"])
    text = sdf("one", a1, b1) + sdf("two", a2, b2)
    assert sb.sdf_count(text) == 2
    assert "Name = two" in sb.pdbqt_from_sdf(text, 1)
    recs = sb.sdf_records(text + "\n\n")  # trailing blank lines are not a record
    assert len(recs) == 2 and recs[1].startswith("two")
    assert [sb.pdbqt_from_sdf(r) for r in recs] == [sb.pdbqt_from_sdf(text, 0), sb.pdbqt_from_sdf(text, 1)]
    with pytest.raises(sb.SminaError):
        sb.pdbqt_from_sdf(text, 2)


@pytest.mark.parametrize("bad", ["", "x\ny\nz\n  3  2  0  0  0  0  0  0  0  0999 V2000\n",
                                 "x\ny\nz\n  1  0  0  0  0  0  0  0  0  0999 V3000\nM  END\n"])
def test_malformed_records_refused(bad):
    with pytest.raises(sb.SminaError):
        sb.pdbqt_from_sdf(bad)


def _bonds_by_distance(atoms):
    bonds = []
    for i in range(len(atoms)):
        for j in range(i + 1, len(atoms)):
            d = np.linalg.norm(np.subtract(atoms[i][1:], atoms[j][1:]))
            if d < 1.1 * (COV[atoms[i][0]] + COV[atoms[j][0]]):
                bonds.append((i + 1, j + 1, 1))
    return bonds


@pytest.mark.parametrize("heavy,rotors,seed", [(14, 3, 5), (24, 5, 11), (40, 10, 5)])
def test_synthetic_ligand_round_trip(heavy, rotors, seed):
    src = sb.make_ligand_pdbqt(heavy, rotors, seed)
    rows = atoms_of(src)
    el = {"C": "C", "A": "C", "N": "N", "NA": "N", "OA": "O", "O": "O", "SA": "S", "S": "S", "HD": "H", "Cl": "Cl",
          "F": "F", "Br": "Br", "I": "I", "P": "P"}
    atoms = [(el[r[1]], r[2], r[3], r[4]) for r in rows]
    bonds = _bonds_by_distance(atoms)
    out = sb.pdbqt_from_sdf(sdf("syn", atoms, bonds), add_hydrogens=False)
    back = atoms_of(out)
    key = lambda r: (round(r[2], 3), round(r[3], 3), round(r[4], 3))  # noqa: E731
    assert sorted(key(r) for r in back) == sorted(key(r) for r in rows)  # every atom kept where it was
    # the rotatable bonds, counted here by the rule
    heavy_deg = np.zeros(len(atoms), int)
    for i, j, _ in bonds:
        heavy_deg[i - 1] += atoms[j - 1][0] != "H"
        heavy_deg[j - 1] += atoms[i - 1][0] != "H"
    want = sum(1 for i, j, _ in bonds if heavy_deg[i - 1] > 1 and heavy_deg[j - 1] > 1)  # acyclic chains
    assert torsdof(out) == want >= rotors
    m = sb.Model(out)
    assert m.num_movable == len(rows) and m.torsdof == want


NAPHTHALENE = [("C", 1.212, 0.7, 0), ("C", 0, 1.4, 0), ("C", -1.212, 0.7, 0), ("C", -1.212, -0.7, 0),
               ("C", 0, -1.4, 0), ("C", 1.212, -0.7, 0), ("C", 2.425, 1.4, 0), ("C", 3.637, 0.7, 0),
               ("C", 3.637, -0.7, 0), ("C", 2.425, -1.4, 0)]
NAPH_EDGES = [(1, 2), (2, 3), (3, 4), (4, 5), (5, 6), (6, 1), (1, 7), (7, 8), (8, 9), (9, 10), (10, 6)]


@pytest.mark.parametrize("doubles", [{(2, 3), (4, 5), (6, 1), (7, 8), (9, 10)},   # shared bond double
                                     {(1, 2), (3, 4), (5, 6), (7, 8), (9, 10)}])  # shared bond single: fused pass
def test_naphthalene_both_kekule_forms_aromatic(doubles):
    bonds = [(i, j, 2 if (i, j) in doubles else 1) for i, j in NAPH_EDGES]
    types = [r[1] for r in atoms_of(sb.pdbqt_from_sdf(sdf("naphthalene", NAPHTHALENE, bonds)))]
    assert types == ["A"] * 10


def test_biphenyl_one_torsion_phenol_and_chlorine():
    ring_a = ring6()
    ring_b = [(el, x + 4.29, y, z) for el, x, y, z in ring6()]
    kek = [(1, 2, 2), (2, 3, 1), (3, 4, 2), (4, 5, 1), (5, 6, 2), (6, 1, 1)]
    bonds = kek + [(i + 6, j + 6, o) for i, j, o in kek] + [(1, 10, 1)]  # ring A atom 1 to ring B atom 4
    atoms = ring_a + ring_b + [("O", -2.76, 0.0, 0.0), ("Cl", 5.0, 2.6, 0.0)]
    bonds += [(4, 13, 1), (8, 14, 1)]
    p = sb.pdbqt_from_sdf(sdf("biphenyl", atoms, bonds))
    t = [r[1] for r in atoms_of(p)]
    assert t.count("A") == 12 and t.count("OA") == 1 and t.count("HD") == 1 and t.count("Cl") == 1
    assert torsdof(p) == 1  # the ring-ring bond; C-O and C-Cl end at one-heavy-neighbour atoms
    m = sb.Model(p)
    assert m.torsdof == 1


def sdf3000(name, atoms, bonds, charges=(), split_at=None):
    """The same molecule as a V3000 record; ``split_at``: an atom whose line is
    continued onto a second one with a trailing "-"."""
    chg = dict(charges)
    out = [name, "  test", "", "  0  0  0     0  0            999 V3000", "M  V30 BEGIN CTAB",
           f"M  V30 COUNTS {len(atoms)} {len(bonds)} 0 0 0", "M  V30 BEGIN ATOM"]
    for k, (el, x, y, z) in enumerate(atoms, 1):
        line = f"M  V30 {k} {el} {x:.4f} {y:.4f} {z:.4f} 0" + (f" CHG={chg[k]}" if k in chg else "")
        if k == split_at:
            cut = len(line) // 2
            out += [line[:cut] + "-", "M  V30 " + line[cut:]]
        else:
            out.append(line)
    out += ["M  V30 END ATOM", "M  V30 BEGIN BOND"]
    out += [f"M  V30 {k} {o} {i} {j}" for k, (i, j, o) in enumerate(bonds, 1)]
    out += ["M  V30 END BOND", "M  V30 END CTAB", "M  END", "$$$$"]
    return "\n".join(out) + "\n"


def test_v3000_records_read_as_their_v2000_twins():
    atoms = [("C", 0, 0, 0), ("C", 1.5, 0, 0), ("O", 2.1, 1.05, 0), ("O", 2.1, -1.05, 0)]
    bonds = [(1, 2, 1), (2, 3, 2), (2, 4, 1)]
    for a, b, ch in [(atoms, bonds, [(4, -1)]), (NAPHTHALENE, [(i, j, 4) for i, j in NAPH_EDGES], [])]:
        assert sb.pdbqt_from_sdf(sdf3000("m", a, b, ch, split_at=2)) == sb.pdbqt_from_sdf(sdf("m", a, b, ch))
    src = sb.make_ligand_pdbqt(24, 5, 11)
    el = {"C": "C", "A": "C", "N": "N", "NA": "N", "OA": "O", "SA": "S", "HD": "H", "Cl": "Cl", "F": "F",
          "Br": "Br", "I": "I", "P": "P", "S": "S", "O": "O"}
    syn = [(el[r[1]], r[2], r[3], r[4]) for r in atoms_of(src)]
    sb_ = _bonds_by_distance(syn)
    assert sb.pdbqt_from_sdf(sdf3000("s", syn, sb_)) == sb.pdbqt_from_sdf(sdf("s", syn, sb_))
    with pytest.raises(sb.SminaError):  # counts that do not match the blocks
        sb.pdbqt_from_sdf(sdf3000("m", atoms, bonds).replace("COUNTS 4 3", "COUNTS 5 3"))


def test_salt_stripped_to_its_largest_piece():
    # sodium acetate: the Na+ counter-ion is a piece of its own and goes (StripSalts)
    atoms = [("C", 0, 0, 0), ("C", 1.5, 0, 0), ("O", 2.1, 1.05, 0), ("O", 2.1, -1.05, 0)]
    bonds = [(1, 2, 1), (2, 3, 2), (2, 4, 1)]
    salt = sdf("NaOAc", atoms + [("Na", 5.0, 0, 0)], bonds, charges=[(4, -1), (5, 1)])
    assert sb.pdbqt_from_sdf(salt).replace("NaOAc", "m") == sb.pdbqt_from_sdf(sdf("m", atoms, bonds, charges=[(4, -1)]))
