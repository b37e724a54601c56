"""Serving loop (sg_serve_*): continuous batching of docking requests over
resident receptors.  Each result must equal the batched entry point's for
the same (seed, ligand key) -- alone, or submitted in a mix with other
ligands and other receptors while earlier requests are still running.
"""
import time

import numpy as np
import pytest

import smina_b200 as sb
import workloads as W

pytestmark = pytest.mark.gpu


def _job(seed, key, chains=4, steps=25):
    return sb.LigandJob(model=0, num_chains=chains, num_steps=steps, maxiters=0, seed=seed, ligand_key=key)


def _collect(eng, tickets, timeout_s=120):
    got, t0 = {}, time.time()
    while len(got) < len(tickets) and time.time() - t0 < timeout_s:
        for (t, status, count, lat, evals, cs, nh, launch, d0, d1, qms, sms, tpc) in eng.serve_poll(64, wait_ms=50,
                                                                                                 spans=True):
            assert status == sb.SG_OK
            got[t] = eng.serve_fetch(t, count, cs, nh)
            got[t].update(latency_ms=lat, launch=launch, span=(d0, d1), queue_ms=qms)
            assert 0 <= qms <= sms <= lat
    assert len(got) == len(tickets), "requests did not finish"
    return got


@pytest.fixture(scope="module")
def setup():
    eng = sb.Engine(0, sb.PREC_FP32)
    eng.set_tables(W.tables())
    R2 = sb.Receptor(2000, 8, W.CENTER)
    eng.set_receptor(0, W.receptor(), W.box())
    eng.set_receptor(1, R2, W.box(26.0))
    models = [W.ligand(24, 5, 11), W.ligand(12, 0, 3), W.ligand(40, 10, 5), W.ligand(30, 8, 2)]
    yield eng, models
    eng.close()


def _reference(eng, rid, m, job, p):
    j = sb.LigandJob(model=0, num_chains=job.num_chains, num_steps=job.num_steps, maxiters=job.maxiters,
                     seed=job.seed, ligand_key=job.ligand_key)
    return eng.dock_batch(rid, [m], [j], p, refine=True)[0]


def _same(a, b):
    for k in ("e", "conf", "coords"):
        assert np.array_equal(a[k], b[k]), k
    assert a["evals"] == b["evals"]


def test_serving_matches_batched_entry_alone_and_in_a_mix(setup):
    eng, models = setup
    p = models[0].search_params()
    work = [(0, models[0], _job(3, 101)), (1, models[1], _job(3, 102)), (0, models[2], _job(4, 103)),
            (1, models[3], _job(5, 104)), (0, models[3], _job(6, 105))]
    refs = [_reference(eng, rid, m, j, p) for rid, m, j in work]
    eng.serve_start(max_batch_ligands=2, max_wait_ms=1.0)
    try:
        # alone
        t = eng.serve_submit(work[0][0], work[0][1], work[0][2], p)
        alone = _collect(eng, [t])[t]
        _same(alone, refs[0])
        # in a mix: staggered submissions, two receptors, several launches in flight
        tickets = []
        for rid, m, j in work:
            tickets.append(eng.serve_submit(rid, m, j, p))
            time.sleep(0.01)
        got = _collect(eng, tickets)
        for t, ref in zip(tickets, refs):
            _same(got[t], ref)
            assert got[t]["latency_ms"] > 0
    finally:
        eng.serve_stop()


def test_serving_rejects_requests_over_budget(setup):
    eng, models = setup
    p = models[0].search_params()
    eng.serve_start(hbm_budget_bytes=1 << 16)
    try:
        with pytest.raises(sb.SminaError):
            eng.serve_submit(0, models[2], _job(1, 1, chains=64), p)
    finally:
        eng.serve_stop()


def test_serving_launches_overlap_on_the_device(setup):
    """Requests that arrive while others run go out in launches of their own
    and share the device with them: the device-clock spans of requests from
    different launches overlap, and every result still equals the batched
    entry point's."""
    eng, models = setup
    p = models[0].search_params()
    work = [(k % 2, models[k % 4], _job(11, 200 + k, chains=4, steps=60)) for k in range(6)]
    refs = [_reference(eng, rid, m, j, p) for rid, m, j in work]
    eng.serve_start(max_batch_ligands=1, max_wait_ms=0.5)
    try:
        tickets = []
        for rid, m, j in work:
            tickets.append(eng.serve_submit(rid, m, j, p))
            time.sleep(0.005)
        got = _collect(eng, tickets)
    finally:
        eng.serve_stop()
    for t, ref in zip(tickets, refs):
        _same(got[t], ref)
        d0, d1 = got[t]["span"]
        assert 0 < d0 < d1
    res = [got[t] for t in tickets]
    assert len({r["launch"] for r in res}) >= 2
    overlapping = [(a["launch"], b["launch"]) for a in res for b in res
                   if a["launch"] < b["launch"] and b["span"][0] < a["span"][1] and a["span"][0] < b["span"][1]]
    assert overlapping, "no two launches were on the device at the same time"
