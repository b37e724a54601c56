"""The engine's precalculate_linear tables (host/scoring.cpp) against an
independent restatement of smina's terms and tables (tests/scoring_restated.py)
built on the reference's own type constants and builtin term lists
(tests/golden/scoring_ref.json, extracted from src/lib/atom_constants.h and
src/lib/builtinscoring.cpp): every type pair, every sample and every
component, bit for bit, for each builtin scoring function and for custom
scoring files that use every pair term smina has."""
import numpy as np
import pytest

import smina_b200 as sb
import scoring_restated as R

# every pair term, with type names in all the forms string_to_smina_type
# takes: AD4 names, smina names, the Se -> S equivalence and a non-AD metal
CUSTOM_ALL = """# every charge-independent pair term
-0.035579 gauss(o=0,_w=0.5,_c=8)
-0.005156 gauss(o=3,_w=2,_c=8)
0.840245 repulsion(o=0,_c=8)
0.3 repulsion(o=-0.25,_c=6)
-0.035069 hydrophobic(g=0.5,_b=1.5,_c=8)
0.02 non_hydrophobic(g=0.5,_b=1.5,_c=7.5)
-0.587439 non_dir_h_bond(g=-0.7,_b=0,_c=8)
0.0099 vdw(i=4,_j=8,_s=0,_^=100,_c=8)
0.0031 vdw(i=6,_j=12,_s=0.5,_^=20,_c=8)
-0.0974 non_dir_h_bond_lj(o=-0.7,_^=100,_c=8)
0.11 non_dir_anti_h_bond_quadratic(o=0.4,_c=8)
0.07 donor_donor_quadratic(o=0.2,_c=8)
0.05 acceptor_acceptor_quadratic(o=0.1,_c=8)
-0.4 atom_type_gaussian(t1=Zn,t2=OA,o=0,_w=1.2,_c=8)
-0.2 atom_type_linear(t1=NitrogenXSDonor,t2=Cl,g=-0.3,_b=0.6,_c=8)
0.25 atom_type_quadratic(t1=Se,t2=A,o=0.3,_c=8)
0.6 atom_type_inverse_power(t1=Cu,t2=N,i=2,_^=50,_c=8)
0.3 atom_type_inverse_power(t1=HD,t2=C,i=1,_^=10,_c=8)
1.923 num_tors_div
"""
CUSTOM_CHARGED = """# charge-dependent terms beside charge-independent ones, longest cutoff 9
0.1560 vdw(i=6,_j=12,_s=0,_^=100,_c=8)
0.1159 ad4_solvation(d-sigma=3.5,_s/q=0.01097,_c=9)
0.1465 electrostatic(i=1,_^=100,_c=8)
0.05 electrostatic(i=2,_^=30,_c=6)
-0.0974 non_dir_h_bond_lj(o=-0.7,_^=100,_c=8)
0.2744 num_tors_add
"""


def _engine_tables(t):
    d = t.desc
    np_, n, nc = R.NPAIRS, d.n, d.num_components
    smooth = np.ctypeslib.as_array(d.smooth, shape=(np_, n, nc, 2)).copy()
    fast = np.ctypeslib.as_array(d.fast, shape=(np_, n, nc)).copy()
    return smooth, fast, d


def _assert_same(t, expect, what):
    smooth, fast, d = _engine_tables(t)
    es, ef = expect
    assert smooth.shape == es.shape, (what, smooth.shape, es.shape)
    for c, name in ((0, "energies"), (1, "dor")):
        bad = np.flatnonzero(smooth[..., c].view(np.uint64) != es[..., c].view(np.uint64))
        if bad.size:
            k = np.unravel_index(bad[0], smooth[..., c].shape)
            pytest.fail(f"{what}: {name} differ at {bad.size} entries, first (pair, i, comp) {k}: "
                        f"{smooth[..., c][k]!r} vs {es[..., c][k]!r}")
    assert np.array_equal(fast.view(np.uint64), ef.view(np.uint64)), f"{what}: fast table"


def _terms_of(name):
    return R.REF["functions"][name]


@pytest.mark.parametrize("name", sorted(R.REF["functions"]))
def test_builtin_tables_match_restatement(name):
    """every builtin scoring function of the reference, by its own term list"""
    t = sb.Tables(name)
    _assert_same(t, R.tables(_terms_of(name), vinardo=name == "vinardo"), name)


@pytest.mark.parametrize("text", [CUSTOM_ALL, CUSTOM_CHARGED], ids=["every_pair_term", "charged"])
def test_custom_tables_match_restatement(text):
    t = sb.Tables("vina", text)
    _assert_same(t, R.tables(R.parse_custom(text)), "custom")


def test_table_geometry():
    """n = int(factor * cutoff^2) + 3 samples at r = sqrt(i / factor), for
    the longest cutoff of any term"""
    t = sb.Tables("vina", CUSTOM_CHARGED, factor=16.0)
    assert t.desc.n == int(16.0 * 81.0) + 3 and t.desc.cutoff_sqr == 81.0 and t.desc.num_components == 4
    _assert_same(t, R.tables(R.parse_custom(CUSTOM_CHARGED), factor=16.0), "custom, factor 16")


@pytest.mark.parametrize("bad", ["0.1 vdw(i=5,_j=8,_s=0,_^=100,_c=8)", "0.1 electrostatic(i=3,_^=100,_c=8)",
                                 "0.1 atom_type_gaussian(t1=Xx,t2=C,o=0,_w=1,_c=8)", "0.1 gaussian(o=0,_w=1,_c=8)",
                                 "0.1 atom_type_inverse_power(t1=C,t2=N,i=3,_^=10,_c=8)",
                                 "0.1 electrostatic(i=1.5,_^=100,_c=8)", "0.1 vdw(i=4.5,_j=8,_s=0,_^=100,_c=8)"])
def test_bad_terms_are_refused_like_the_reference(bad):
    with pytest.raises(ValueError):
        R.tables(R.parse_custom(bad))
    with pytest.raises(sb.SminaError):
        sb.Tables("vina", bad)
