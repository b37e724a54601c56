"""--fast's early stop on the batched search (sg_set_early_stop; not
smina's search: the reference's EarlyStop, src/gpu/gpu_kernels.h:45-56,
gpu_kernels_impl.cuh:607-657,740-810).  The chains run in phases that
resume exactly where the previous one stopped, so a ligand that never stops
docks bit for bit as without early stop, and one that stops at the first
check docks as if its chains had that many steps; with the rule in between,
some ligands stop and the search makes fewer evaluations."""
import math

import numpy as np
import pytest

import smina_b200 as sb
import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    T, R, gd = W.tables(), W.receptor(), W.box()
    e = sb.Engine(0, sb.PREC_FP32)
    e.set_tables(T)
    e.set_receptor(0, R, gd)
    models = [W.ligand(24, 5, 11), W.ligand(14, 2, 3), W.ligand(30, 8, 2)]
    yield e, models
    e.close()


def _jobs(models, steps, chains=8):
    return [sb.LigandJob(model=k, num_chains=chains, num_steps=steps, maxiters=0, seed=3, ligand_key=40 + k)
            for k in range(len(models))]


def _same(a, b):
    for x, y in zip(a, b):
        for k in ("e", "conf", "coords"):
            assert np.array_equal(x[k], y[k]), k
        assert x["evals"] == y["evals"]


def test_phases_that_never_stop_change_nothing(setup):
    e, models = setup
    p = models[0].search_params()
    jobs = _jobs(models, 120)
    e.set_early_stop(off=True)
    ref = e.dock_batch(0, models, jobs, p, refine=True)
    e.set_early_stop(checkpoints=7, first=2, fraction=0.5, eps=-1.0, chains_per_unit=2)  # no units ever agree
    try:
        got = e.dock_batch(0, models, jobs, p, refine=True)
    finally:
        e.set_early_stop(off=True)
    _same(got, ref)


def test_stopping_at_the_first_check_docks_as_the_shorter_search(setup):
    e, models = setup
    p = models[0].search_params()
    steps, n, first = 150, 10, 3
    e.set_early_stop(checkpoints=n, first=first, fraction=0.5, eps=1e9, chains_per_unit=1)  # every ligand agrees
    try:
        got = e.dock_batch(0, models, _jobs(models, steps), p, refine=True)
    finally:
        e.set_early_stop(off=True)
    ref = e.dock_batch(0, models, _jobs(models, math.ceil(steps * first / n)), p, refine=True)
    _same(got, ref)


def test_the_rule_stops_some_ligands(setup):
    e, models = setup
    p = models[0].search_params()
    jobs = _jobs(models, 200, chains=8)
    full = e.dock_batch(0, models, jobs, p, refine=True)
    e.set_early_stop(checkpoints=10, first=2, fraction=0.5, eps=1.0, chains_per_unit=2)
    try:
        es = e.dock_batch(0, models, jobs, p, refine=True)
    finally:
        e.set_early_stop(off=True)
    assert sum(r["evals"] for r in es) < sum(r["evals"] for r in full)
    assert all(len(r["e"]) > 0 for r in es)


def test_early_stop_is_refused_on_fp64_engines():
    e = sb.Engine(0, sb.PREC_FP64)
    try:
        with pytest.raises(sb.SminaError):
            e.set_early_stop()
    finally:
        e.close()
