"""Seeded synthetic workloads shared by the tests (small and full size).

Receptor R(n): random-walk chains, 8 A cavity at the box centre; ligands
L(h, r): acyclic drug-like trees with r torsions.  The box centre is kept
off multiples of 3 A so the 3 A cell bricks are never flat.
"""
import functools

import numpy as np

import smina_b200 as sb

CENTER = (0.5, 0.25, -0.3)


@functools.lru_cache(maxsize=None)
def receptor(n=3000, seed=7):
    return sb.Receptor(n, seed, CENTER)


@functools.lru_cache(maxsize=None)
def tables(name="vina", factor=32.0):
    return sb.Tables(name, factor=factor)


@functools.lru_cache(maxsize=None)
def custom_tables(text):
    return sb.Tables("vina", custom_text=text)


def box(size=22.0, center=CENTER):
    return sb.make_box(center, (size, size, size))


@functools.lru_cache(maxsize=None)
def ligand(heavy=24, rotors=5, seed=11):
    return sb.Model(sb.make_ligand_pdbqt(heavy, rotors, seed, CENTER))


def random_confs(m, gd, n, seed, spread=None):
    """Half random poses inside the box, half perturbed around the input pose
    (the split of gpu_eval_test.cpp:212-243)."""
    rng = np.random.default_rng(seed)
    out = np.zeros((n, m.conf_size))
    lo = np.array(gd.begin[:])
    hi = np.array(gd.end[:])
    init = np.array([m.desc.frame_init_origin[i] for i in range(3)])
    for k in range(n):
        if k % 2 == 0:
            pos = rng.uniform(lo, hi)
            q = rng.normal(size=4)
            q /= np.linalg.norm(q)
            tors = rng.uniform(-np.pi, np.pi, m.conf_size - 7)
        else:
            pos = init + rng.normal(scale=0.5 if spread is None else spread, size=3)
            ax = rng.normal(size=3)
            ax /= np.linalg.norm(ax)
            ang = rng.normal(scale=0.3)
            q = np.concatenate([[np.cos(ang / 2)], np.sin(ang / 2) * ax])
            tors = rng.normal(scale=0.5, size=m.conf_size - 7)
        out[k, :3] = pos
        out[k, 3:7] = q
        out[k, 7:] = tors
    return out


def with_charges(pdbqt, seed, sd=0.25):
    """The PDBQT text with seeded partial charges (normal, s.d. `sd`, within
    +-0.9) in the charge columns of its ATOM lines, so charge-dependent terms
    see non-zero charges through the reader."""
    rng = np.random.default_rng(seed)
    out = []
    for line in pdbqt.splitlines():
        if line.startswith(("ATOM", "HETATM")):
            q = float(np.clip(rng.normal(scale=sd), -0.9, 0.9))
            line = line[:66] + "    " + f"{q:+6.3f}" + line[76:]
        out.append(line)
    return "\n".join(out) + "\n"


@functools.lru_cache(maxsize=None)
def charged_ligand(heavy=24, rotors=5, seed=11, qseed=1):
    return sb.Model(with_charges(sb.make_ligand_pdbqt(heavy, rotors, seed, CENTER), qseed))


class ChargedReceptor:
    """A synthetic receptor with seeded partial charges (normal, s.d. 0.3,
    within +-0.9) in place of its zero charges; `desc` is what the engine and
    the oracle take."""

    def __init__(self, n, seed, qseed):
        self.base = sb.Receptor(n, seed, CENTER)
        d = self.base.desc
        self.q = np.clip(np.random.default_rng(qseed).normal(scale=0.3, size=d.num_atoms), -0.9, 0.9)
        self.desc = sb.ReceptorDesc(d.num_atoms, d.coords, d.type, sb.dptr(self.q))
        self.coords, self.types = self.base.coords, self.base.types


@functools.lru_cache(maxsize=None)
def charged_receptor(n=3000, seed=7, qseed=2):
    return ChargedReceptor(n, seed, qseed)
