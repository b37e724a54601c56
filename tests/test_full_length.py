"""The plain (FP64) search at full length, bit for bit against the oracle.

The single-ligand redock workload (a 24-heavy-atom ligand with 5 rotatable
bonds against the 3,000-atom receptor, 22 A box at 0.375 A, default
scoring): exhaustiveness 8, smina's own step and BFGS-iteration counts for
that ligand (monte_carlo.cpp:95-130 with main.cpp:513-529), so that the
rare branches of long chains run -- the output container replacing its
worst pose once 20 are kept, torsions wrapping at +-pi, the mt19937 state
regenerated many times over.  The oracle runs one thread per chain.  Then
the merged poses are refined on both sides, as the redock does.
"""
import numpy as np
import pytest

import workloads as W
from oracle_lib import merge
from test_plain_parity import assert_bitwise, setup  # noqa: F401  (module fixture)

pytestmark = pytest.mark.gpu


def test_full_length_chains_bit_exact(setup):  # noqa: F811
    eng, orc, gd = setup
    m = W.ligand(24, 5, 11)
    p = m.search_params()
    assert p.num_steps > 15000  # smina's count for this ligand, not a shortened chain
    nch = 8
    confs, mts = m.seed_chains(2024, nch, gd)
    b1 = eng.dock(0, [m], [0] * nch, confs, mts, p)
    b0 = orc.dock([m], [0] * nch, confs, mts, p, threads=nch)
    assert (b1.count == b0.count).all(), (b1.count, b0.count)
    assert (b1.evals == b0.evals).all(), (b1.evals, b0.evals)
    assert (b1.count == p.num_saved_mins).any(), "no chain filled its output container"
    for k in range(nch):
        c = b0.count[k]
        assert_bitwise(b1.e[k, :c], b0.e[k, :c], f"chain {k} energies")
        assert_bitwise(b1.conf[k, :c, :m.conf_size], b0.conf[k, :c, :m.conf_size], f"chain {k} confs")
        assert_bitwise(b1.coords[k, :c], b0.coords[k, :c], f"chain {k} coords")
    # merge (min_rmsd 2) and refine the merged poses, as the redock does
    e0, conf0, _ = merge(b0, m, max_size=p.num_saved_mins)
    _, er1, _ = eng.refine(0, [m], np.zeros(len(e0), np.int32), conf0, cap=tuple(p.authentic_v),
                           maxiters=p.maxiters)
    _, er0, _ = orc.refine([m], np.zeros(len(e0), np.int32), conf0, cap=tuple(p.authentic_v), maxiters=p.maxiters)
    assert_bitwise(er1, er0, "refined energies")
