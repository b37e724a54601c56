"""Chains on teams of warps: 64 and 128 threads per chain (the reference's
threads_per_chain, gpu_kernels_impl.cuh:572-605; its automatic choice from
residency, gpu_kernels_impl.cuh:578-582).

A team's leader warp runs the chain; at every evaluation the team shares
out the grid and pair terms and the leader sums the warps' energies and
force arrays in team order.  So a team's evaluation differs from one warp's
only by the order of FP32 additions, and is held to the FP32 acceptance
rule against one warp (and against the FP64 oracle).  The batched search
on teams must be deterministic, independent of the batch and of the launch
shape for a given team size, reach the FP64 search's best energies, and
return poses whose energies are their confs' energies.  The automatic
setting must pick 128 threads for a lone ligand and 32 for a batch that
fills the device; serving must run a request on the team size set, with
the batched entry point's results.
"""
import time

import numpy as np
import pytest

import smina_b200 as sb
import workloads as W
from oracle_lib import Oracle
from test_fp32 import at_discontinuity, check_fp32

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engines():
    made = {}

    def engine(threads, tables=None, receptor=None, gd=None):
        key = (threads, id(tables), id(receptor))
        if key not in made:
            e = sb.Engine(0, sb.PREC_FP32)
            e.set_tables(tables or W.tables())
            e.set_receptor(0, receptor or W.receptor(), gd or W.box())
            e.set_threads_per_chain(threads)
            made[key] = e
        return made[key]
    yield engine
    for e in made.values():
        e.close()


@pytest.mark.parametrize("heavy,rotors,seed", [(24, 5, 11), (12, 0, 3), (50, 12, 4), (60, 40, 9)])
def test_team_eval_matches_one_warp(engines, heavy, rotors, seed):
    """60 heavy atoms with 40 rotors: more than 32 frames (model::set level by level)."""
    gd = W.box()
    m = W.ligand(heavy, rotors, seed)
    confs = W.random_confs(m, gd, 256, seed + 100)
    e1, g1, x1 = engines(32).eval(0, m, confs, coords=True)
    orc = Oracle(W.tables(), W.receptor(), gd, full_cells=True)
    e64, g64, x64 = orc.eval(m, confs, coords=True)
    flags = at_discontinuity(m, gd, x64, W.tables().desc.cutoff_sqr)
    for threads in (64, 128):
        e, g, x = engines(threads).eval(0, m, confs, coords=True)
        assert np.array_equal(x, x1)  # model::set is the leader's, as on one warp
        check_fp32(e, g, e1, g1, flags)
        check_fp32(e, g, e64, g64, flags)


def test_team_eval_charge_dependent_and_flex(engines):
    """nc = 4 tables with charge maps, and a model with flexible residues
    (other pairs, inflex atoms)."""
    gd = W.box()
    T4, Rq = sb.Tables("ad4_scoring"), W.charged_receptor()
    m = W.charged_ligand(24, 5, 11)
    confs = W.random_confs(m, gd, 128, 7)
    e1, g1 = engines(32, T4, Rq).eval(0, m, confs)
    _, _, x64 = Oracle(T4, Rq, gd, full_cells=True).eval(m, confs, coords=True)
    flags = at_discontinuity(m, gd, x64, T4.desc.cutoff_sqr)
    for threads in (64, 128):
        e, g = engines(threads, T4, Rq).eval(0, m, confs)
        check_fp32(e, g, e1, g1, flags)
    mf = sb.Model(sb.make_ligand_pdbqt(24, 5, 11, W.CENTER), sb.make_flex_pdbqt(4, 3, W.CENTER))
    confs = W.random_confs(mf, gd, 128, 8)
    e1, g1 = engines(32).eval(0, mf, confs)
    _, _, x64 = Oracle(W.tables(), W.receptor(), gd, full_cells=True).eval(mf, confs, coords=True)
    flags = at_discontinuity(mf, gd, x64, W.tables().desc.cutoff_sqr)
    for threads in (64, 128):
        e, g = engines(threads).eval(0, mf, confs)
        check_fp32(e, g, e1, g1, flags)


def _jobs(n, chains=4, steps=30, seed=42, keys=None):
    return [sb.LigandJob(model=k, num_chains=chains, num_steps=steps, maxiters=0, seed=seed,
                         ligand_key=(keys[k] if keys else 1000 + k)) for k in range(n)]


def _same(a, b):
    for k in ("e", "conf", "coords"):
        assert np.array_equal(a[k], b[k]), k
    assert a["evals"] == b["evals"]


@pytest.mark.parametrize("threads", [64, 128])
def test_team_batch_deterministic_alone_and_shape_independent(engines, threads):
    eng = engines(threads)
    models = [W.ligand(24, 5, 11), W.ligand(12, 0, 3), W.ligand(40, 10, 5)]
    p = models[0].search_params()
    jobs = _jobs(3, keys=[7, 8, 9])
    a = eng.dock_batch(0, models, jobs, p)
    assert eng.threads_per_chain() == (threads, threads)
    b = eng.dock_batch(0, models, jobs, p)
    try:
        eng.set_chains_per_block(2 if threads == 64 else 1)
        c = eng.dock_batch(0, models, jobs, p)
    finally:
        eng.set_chains_per_block(0)
    alone = eng.dock_batch(0, [models[2]], [sb.LigandJob(model=0, num_chains=4, num_steps=30, maxiters=0, seed=42,
                                                          ligand_key=9)], p)
    for x, y, z in zip(a, b, c):
        assert len(x["e"]) > 0 and x["evals"] > 0
        _same(x, y)
        _same(x, z)
    _same(a[2], alone[0])


def test_team_poses_carry_their_energies(engines):
    """Every unrefined pose's energy is its conf's authentic energy (the
    search's last BFGS on a team), evaluated again on one warp."""
    m = W.ligand(30, 8, 2)
    p = m.search_params()
    res = engines(128).dock_batch(0, [m], _jobs(1, chains=8, steps=60), p, refine=False)[0]
    assert len(res["e"]) > 1
    e1, g1 = engines(32).eval(0, m, res["conf"], v=tuple(p.authentic_v), slope=p.cache_slope)
    rel = np.abs(e1 - res["e"]) / np.maximum(np.abs(res["e"]), 1.0)
    assert rel.max() <= 1e-3, rel.max()


def test_team_search_quality_vs_fp64(engines):
    """As the one-warp search's check: 4 independent searches of 8 chains per
    side, best refined energies within a margin."""
    m = W.ligand(24, 5, 11)
    p = m.search_params()
    gd = W.box()
    chains, steps, runs = 8, 400, 4
    eng64 = sb.Engine(0, sb.PREC_FP64)
    try:
        eng64.set_tables(W.tables())
        eng64.set_receptor(0, W.receptor(), gd)
        confs, mts = m.seed_chains(5, chains * runs, gd)
        b = eng64.dock(0, [m], np.zeros(chains * runs, np.int32), confs, mts, p, steps=steps)
        best64 = []
        for k in range(runs):
            sub = sb.merge_chains(b, m, first=chains * k, n=chains, max_size=p.num_saved_mins)
            _, e64, _ = eng64.refine(0, [m], np.zeros(len(sub[0]), np.int32), sub[1], cap=tuple(p.authentic_v),
                                     maxiters=p.maxiters, accurate_line=p.accurate_line, early_term=p.early_term)
            best64.append(float(np.min(e64)))
    finally:
        eng64.close()
    jobs = [sb.LigandJob(model=0, num_chains=chains, num_steps=steps, maxiters=0, seed=5, ligand_key=1 + k)
            for k in range(runs)]
    for threads in (64, 128):
        r = engines(threads).dock_batch(0, [m], jobs, p)
        best = [float(x["e"][0]) for x in r]
        assert min(best) <= min(best64) + 0.5, (threads, best, best64)


def test_automatic_threads_per_chain(engines):
    eng = engines(0)
    m = W.ligand(20, 3, 5)
    p = m.search_params()
    eng.dock_batch(0, [m], _jobs(1, chains=8, steps=2), p, refine=False)
    assert eng.threads_per_chain() == (0, 128)  # a lone ligand
    n = 320  # 2,560 chains: more than the device holds at 64 threads per chain
    eng.dock_batch(0, [m] * n, _jobs(n, chains=8, steps=1), p, refine=False)
    assert eng.threads_per_chain() == (0, 32)


def test_bad_threads_per_chain_refused(engines):
    eng = engines(32)
    for bad in (16, 48, 96, 256, -1):
        with pytest.raises(sb.SminaError):
            eng.set_threads_per_chain(bad)
    assert eng.threads_per_chain()[0] == 32


def _collect(eng, tickets, timeout_s=120):
    got, t0 = {}, time.time()
    while len(got) < len(tickets) and time.time() - t0 < timeout_s:
        for (t, status, count, lat, evals, cs, nh, launch, d0, d1, qms, sms, tpc) in eng.serve_poll(64, wait_ms=50,
                                                                                                 spans=True):
            assert status == sb.SG_OK
            got[t] = eng.serve_fetch(t, count, cs, nh)
            got[t]["threads_per_chain"] = tpc
    assert len(got) == len(tickets), "requests did not finish"
    return got


def test_serving_on_teams(engines):
    """Serving at 128 threads per chain gives the batched entry point's
    results at 128; with the automatic setting a lone request on an idle
    device runs at 128."""
    models = [W.ligand(24, 5, 11), W.ligand(12, 0, 3)]
    p = models[0].search_params()
    jobs = [sb.LigandJob(model=0, num_chains=4, num_steps=25, maxiters=0, seed=3, ligand_key=201 + k)
            for k in range(2)]
    eng = engines(128)
    refs = [eng.dock_batch(0, [m], [j], p, refine=True)[0] for m, j in zip(models, jobs)]
    eng.serve_start(max_batch_ligands=2, max_wait_ms=1.0)
    try:
        tickets = [eng.serve_submit(0, m, j, p) for m, j in zip(models, jobs)]
        got = _collect(eng, tickets)
        for t, ref in zip(tickets, refs):
            assert got[t]["threads_per_chain"] == 128
            _same(got[t], ref)
    finally:
        eng.serve_stop()
    auto = engines(0)
    auto.serve_start(max_batch_ligands=2, max_wait_ms=1.0)
    try:
        t = auto.serve_submit(0, models[0], jobs[0], p)
        got = _collect(auto, [t])
        assert got[t]["threads_per_chain"] == 128
        _same(got[t], refs[0])
    finally:
        auto.serve_stop()
