"""The mixed-precision search's pair schedule (sg_pair_schedule), checked on
the host: every intramolecular / other pair of the model (model.cpp:598-624
pair lists) appears exactly once, with the type pair, charge-role (swap) and
curl-group (intra) bits the kernel reads; within a chunk no atom is twice a
first atom or twice a second atom (so a warp adds the forces without
atomics); within each 8-slot quarter the first atoms are distinct modulo 8
and so are the second atoms (distinct shared-memory bank groups)."""
import numpy as np
import pytest

import smina_b200 as sb
import workloads as W

EMPTY_TP = 0x1ff


def tri(i, j):
    return i + j * (j + 1) // 2


def _check(m):
    d = m.desc
    types = [d.atom_type[i] for i in range(d.num_atoms)]
    pairs = [(d.pairs[2 * k], d.pairs[2 * k + 1]) for k in range(d.num_pairs)]
    index = {}
    for k, (u, v) in enumerate(pairs):
        index[(u, v)] = k
        index[(v, u)] = k
    sched = m.pair_schedule()
    seen = np.zeros(len(pairs), int)
    for chunk in sched:
        firsts, seconds = [], []
        for q in range(4):
            amod, bmod = set(), set()
            for s in chunk[8 * q:8 * q + 8]:
                s = int(s)
                a, b, tp = s & 0xff, (s >> 8) & 0xff, (s >> 16) & 0x1ff
                swap, intra = (s >> 25) & 1, (s >> 26) & 1
                if tp == EMPTY_TP:
                    assert a == 0 and b == 0
                    continue
                k = index[(a, b)]
                seen[k] += 1
                ta, tb = types[a], types[b]
                assert tp == tri(min(ta, tb), max(ta, tb))
                # the charge roles: the table's A atom is the smaller type, or for equal
                # types the pair's own first atom (precalculate.h:245-260)
                u, v = pairs[k]
                canon_first = (u if types[u] <= types[v] else v)
                assert swap == int(a != canon_first)
                assert intra == int(k >= d.num_other_pairs)
                assert a % 8 not in amod and b % 8 not in bmod
                amod.add(a % 8)
                bmod.add(b % 8)
                firsts.append(a)
                seconds.append(b)
        assert len(set(firsts)) == len(firsts) and len(set(seconds)) == len(seconds)
    assert np.all(seen == 1)
    return sched


@pytest.mark.parametrize("heavy,rotors,seed", [(12, 0, 3), (24, 5, 11), (40, 10, 5), (50, 12, 9)])
def test_schedule_covers_every_pair_once_without_conflicts(heavy, rotors, seed):
    m = W.ligand(heavy, rotors, seed)
    sched = _check(m)
    assert len(sched) >= -(-m.desc.num_pairs // 32)


def test_schedule_of_a_model_with_flexible_residues():
    m = sb.Model(sb.make_ligand_pdbqt(24, 5, 11, W.CENTER), sb.make_flex_pdbqt(4, 3, W.CENTER))
    assert m.desc.num_other_pairs > 0
    _check(m)


def test_schedule_is_dense():
    """Chunks stay full enough that the pair loop does not run mostly empty
    slots: on the screen's ligand sizes, at least 60 % of slots hold a pair."""
    filled = total = 0
    for h, r, s in [(20, 3, 1), (30, 6, 2), (40, 9, 3), (50, 12, 4)]:
        sched = W.ligand(h, r, s).pair_schedule()
        filled += int(np.sum(((sched >> 16) & 0x1ff) != EMPTY_TP))
        total += sched.size
    assert filled / total >= 0.6
