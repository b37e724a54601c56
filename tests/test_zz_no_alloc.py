"""sg_dock_batch32_noalloc: the batched search for callers that must not
have device memory allocated or freed during the call.

Who needs it: a serving loop that has already promised the rest of the
GPU's memory to requests in flight or to a caching allocator (an allocation
mid-request could fail or fragment that memory), and any caller that keeps
other streams busy, because cudaFree waits for the whole device to go idle.
The entry point keeps everything its kernel writes in one fixed array that
every call reuses, so these tests call it twice in a row on different
batches, check that the device's free memory is the same before and after
each call (the first call on the engine included), and check each result
against sg_dock_batch32 (refine off).  The batch path is deterministic, so
the comparison is exact, as in the other batch tests.  The file is named to
run last and builds its own engine, so it passes alone in a fresh process
and after the rest of the suite.
"""
import numpy as np
import pytest

import smina_b200 as sb
import workloads as W

pytestmark = pytest.mark.gpu


def _free_bytes():
    """The device's free memory as cudaMemGetInfo reports it."""
    import torch
    return torch.cuda.mem_get_info(0)[0]


@pytest.fixture(scope="module")
def engine():
    _free_bytes()  # the runtime used for the reading is set up before any reading
    eng = sb.Engine(0, sb.PREC_FP32)
    eng.set_tables(W.tables())
    eng.set_receptor(0, W.receptor(), W.box())
    models = [W.ligand(24, 5, 11), W.ligand(12, 0, 3), W.ligand(40, 10, 5)]
    eng.build_grids(0, sorted({t for m in models for t in m.types() if 1 < t < 27}))
    yield eng, models
    eng.close()


def _jobs(n, seed, chains=4, steps=20):
    return [sb.LigandJob(model=k, num_chains=chains, num_steps=steps, maxiters=0, seed=seed, ligand_key=50 + k)
            for k in range(n)]


def _same(a, b):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert len(x["e"]) > 0
        for k in ("e", "conf", "coords"):
            assert np.array_equal(x[k], y[k]), k
        assert x["evals"] == y["evals"]


def test_noalloc_matches_batched_entry_on_two_calls_in_a_row(engine):
    eng, models = engine
    p = models[0].search_params()
    first, second = _jobs(3, seed=11), _jobs(2, seed=12)
    free0 = _free_bytes()
    got1 = eng.dock_batch_noalloc(0, models, first, p)  # the engine's first search call
    free1 = _free_bytes()
    got2 = eng.dock_batch_noalloc(0, models[:2], second, p)  # reuses the array the first call filled
    free2 = _free_bytes()
    assert free0 == free1 == free2, (free0, free1, free2)
    _same(got1, eng.dock_batch(0, models, first, p, refine=False))
    _same(got2, eng.dock_batch(0, models[:2], second, p, refine=False))


def test_noalloc_follows_a_forced_launch_shape(engine):
    eng, models = engine
    p = models[0].search_params()
    jobs = _jobs(3, seed=21, chains=6)
    try:
        eng.set_chains_per_block(2)
        free0 = _free_bytes()
        got = eng.dock_batch_noalloc(0, models, jobs, p)
        assert _free_bytes() == free0
        _same(got, eng.dock_batch(0, models, jobs, p, refine=False))
        assert eng.batch_stats()["chains_per_block"] == 2
    finally:
        eng.set_chains_per_block(0)


def test_noalloc_refuses_a_batch_larger_than_its_array(engine):
    eng, models = engine
    p = models[0].search_params()
    big = [sb.LigandJob(model=2, num_chains=8, num_steps=1, maxiters=0, seed=1, ligand_key=k) for k in range(400)]
    with pytest.raises(sb.SminaError) as err:
        eng.dock_batch_noalloc(0, models, big, p)
    assert "scratch" in str(err.value)


def test_noalloc_needs_resident_maps(engine):
    eng, models = engine
    eng.set_receptor(1, W.receptor(), W.box())  # no maps built for receptor 1
    with pytest.raises(sb.SminaError) as err:
        eng.dock_batch_noalloc(1, models[:1], _jobs(1, seed=3), models[0].search_params())
    assert "sg_build_grids" in str(err.value)
    assert sb.load().sg_drop_receptor(eng._h, 1) == sb.SG_OK
