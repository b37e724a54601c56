"""--fast's chain split and step fraction (sgh_fast_chains), on the host,
against a direct restatement of the reference's rules
(src/gpu/gpu_docking.cpp:87-112 auto_split / auto_fraction, :168-171
fraction_for, :217-220 chain_steps).  Not smina's search: the engine's
default (split 1, fraction 1) is the identity."""
import math

import pytest

import smina_b200 as sb


def ref_plan(tasks, capacity, chain_split, step_fraction, budget, steps):
    if chain_split > 0:
        split = chain_split
    else:
        split = 32
        while split > 4 and tasks * split > 4 * capacity:
            split //= 2
    if budget > 0:
        frac = budget
    elif step_fraction > 0:
        frac = step_fraction
    else:
        frac = 0.5 if 4 <= split < 32 else 1.0
    return split, max(1, int(math.ceil(steps * frac / split))), frac


@pytest.mark.parametrize("tasks", [1, 8, 64, 296, 2368, 8000, 80000])
@pytest.mark.parametrize("chain_split,step_fraction,budget", [(0, 0, 0), (0, 0, 0.25), (1, 1, 0), (2, 0, 0),
                                                               (8, 0.5, 0), (0, 0.75, 0), (3, 1, 0.1)])
def test_plan_matches_the_reference_rule(tasks, chain_split, step_fraction, budget):
    cap = 16 * 148
    for steps in (1, 7, 19635, 30135):
        got = sb.fast_chains(tasks, cap, chain_split, step_fraction, budget, steps)
        want = ref_plan(tasks, cap, chain_split, step_fraction, budget, steps)
        assert got[:2] == want[:2] and got[2] == want[2], (got, want)


def test_defaults_are_smina_search():
    assert sb.fast_chains(8, 2368, 1, 1.0, 0.0, 19635) == (1, 19635, 1.0)


def test_automatic_split_follows_the_load():
    # a few ligands leave the device idle: 32 chains per task; a screen fills it: 4
    assert sb.fast_chains(8, 2368)[0] == 32
    assert sb.fast_chains(8000, 2368)[0] == 4
    assert sb.fast_chains(8000, 2368, steps=19635)[1] == math.ceil(19635 * 0.5 / 4)


@pytest.mark.parametrize("args", [(-1, 10, 0, 0, 0), (1, 10, -2, 0, 0), (1, 10, 0, 1.5, 0), (1, 10, 0, 0, 2.0),
                                  (1, 10, 0, float("nan"), 0)])
def test_bad_arguments_are_refused(args):
    with pytest.raises(sb.SminaError):
        sb.fast_chains(*args)


def test_fast_jobs_shape_the_screen():
    import workloads as W
    models = [W.ligand(14, 3, 2), W.ligand(24, 5, 11)]
    jobs = sb.fast_jobs(models, 8, 42, capacity=16 * 148)
    for m, j in zip(models, jobs):
        p = m.search_params()
        assert j.num_chains == 8 * 32  # two ligands leave the device idle: 32 chains per task
        assert j.num_steps == max(1, math.ceil(p.num_steps / 32))
        assert j.maxiters == p.maxiters and j.seed == 42
    plain = sb.fast_jobs(models, 8, 42, capacity=16 * 148, chain_split=1, step_fraction=1.0)
    assert [j.num_chains for j in plain] == [8, 8]
    assert [j.num_steps for j in plain] == [m.search_params().num_steps for m in models]
