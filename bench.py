"""Throughput of the batched mixed-precision docking search on B200.

Workload: the 1,000-ligand synthetic virtual screen -- one receptor of
3,000 heavy atoms (seeded random-walk chains, 8 A cavity), 22 A box at
0.375 A, ligands with heavy atoms uniform in [10, 50] and rotatable bonds
uniform in [0, 12], exhaustiveness 8, smina's own step and BFGS-iteration
counts per ligand, default (vina) scoring, FP32 evaluation with FP64 BFGS
update/acceptance.  One step = one persistent search launch over a batch of
ligands (default: the whole screen) followed by the FP64 refinement of the
merged poses.  Metric: ligands docked per second.

  value          ligands / device time of the step's launches (receptor
                 maps resident, CUDA events on the engine's stream)
  e2e            the same through the C-ABI call with host buffers
                 (model upload, result download, host merge included)
  roofline       algorithmic gather bytes of the search kernel (32 B per
                 packed grid cell, 16 B per in-cutoff pair table entry)
                 over its event-timed duration, against measured HBM
                 copy bandwidth
  cpu_baseline   the CPU restatement of smina's search (FP64, one thread
                 per chain) on a bounded sample of the screen's ligands

Multi-GPU: replicas only (every rank docks its own copy of the screen with
its own random streams; no collective on the data path).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpu-smina_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import smina_b200 as sb  # noqa: E402

METRIC = "ligands docked/sec on 1 B200 (batched FP32 vs plain FP64); p50/p99 latency"
UNIT = "ligands/s"
CENTER = (0.5, 0.25, -0.3)
G_BYTES = {sb.PREC_FP32: 32, sb.PREC_FP32_H16: 16}  # one packed grid cell
T_BYTES = 16  # one (e_i, dor_i, e_i+1, dor_i+1) table entry, nc = 1


def screen(n, seed):
    """The synthetic screen: (heavy, rotors, ligand seed) per ligand."""
    rng = np.random.default_rng(seed)
    heavy = rng.integers(10, 51, size=n)
    rotors = rng.integers(0, 13, size=n)
    return [(int(h), int(r), 10_000 + k) for k, (h, r) in enumerate(zip(heavy, rotors))]


def build_models(spec):
    return [sb.Model(sb.make_ligand_pdbqt(h, r, s, CENTER)) for h, r, s in spec]


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=10)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = [r.split(",") for r in self.out.strip().splitlines() if r.count(",") >= 7]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[4 + i] and "Not" not in r[4 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(rows[0][2]),
                "reasons": reasons, "samples": len(rows)}


def make_params(models):
    p = models[0].search_params(9)
    p.num_steps = 0
    return p


def jobs_for(models, idx, exh, seed, key_base, step_scale=1.0):
    jobs = []
    for j, k in enumerate(idx):
        sp = models[k].search_params(9)
        steps = max(1, int(sp.num_steps * step_scale)) if step_scale != 1.0 else sp.num_steps
        jobs.append(sb.LigandJob(model=k, num_chains=exh, num_steps=steps, maxiters=sp.maxiters,
                                 seed=seed, ligand_key=key_base + k))
    return jobs


def cpu_sample(models, gd, receptor, tables, exh, seed, nlig, threads, parallel=1):
    """CPU restatement of the same search (oracle: FP64, one thread per chain)
    over ``nlig`` ligands spread evenly over the screen; ligands/s."""
    from oracle_lib import Oracle, merge
    orc = Oracle(tables, receptor, gd, full_cells=True)
    idx = [int(i) for i in np.linspace(0, len(models) - 1, nlig)]
    orc.ensure([models[k] for k in idx])

    def one(k):
        m = models[k]
        p = m.search_params(9)
        confs, mts = m.seed_chains(seed + k, exh, gd)
        b = orc.dock([m], np.zeros(exh, np.int32), confs, mts, p, threads=threads)
        e, conf, _ = merge(b, m, 2.0, p.num_saved_mins)
        orc.refine([m], np.zeros(len(e), np.int32), conf, cap=tuple(p.authentic_v), maxiters=p.maxiters,
                   accurate=p.accurate_line, early=p.early_term)

    t0 = time.perf_counter()
    for base in range(0, len(idx), parallel):
        ts = [threading.Thread(target=one, args=(k,)) for k in idx[base:base + parallel]]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
    dt = time.perf_counter() - t0
    return len(idx) / dt, dt, idx


def run_accuracy(args):
    """Top-score agreement of the batched FP32 search with the plain FP64
    search on a sample of the screen (smina's full step counts, exhaustiveness
    8, merge + FP64 refinement on both sides), each path run with
    --acc-seeds seeds.  Reports the spread of best-energy differences FP32 -
    FP64 (every FP32 run against every FP64 run) next to the seed-to-seed
    spreads of FP64 and of FP32 (every pair of runs of one path), per-ligand
    spreads over the seeds with a Wilcoxon signed-rank test, and ligand
    bootstrap intervals of the spread ratios."""
    spec = screen(args.ligands, args.seed)
    idx = [int(i) for i in np.linspace(0, len(spec) - 1, args.accuracy)]
    models = build_models([spec[i] for i in idx])
    R = sb.Receptor(3000, 7, CENTER)
    T = sb.Tables("vina")
    gd = sb.make_box(CENTER, (22.0, 22.0, 22.0))
    types = sorted({t for m in models for t in m.types() if 1 < t < 27})
    e64 = sb.Engine(0, sb.PREC_FP64)
    e64.set_tables(T)
    e64.set_receptor(0, R, gd)
    e64.build_grids(0, types)
    e32 = sb.Engine(0, sb.PREC_FP32 if args.precision == "fp32" else sb.PREC_FP32_H16)
    e32.set_tables(T)
    e32.set_receptor(0, R, gd)
    e32.build_grids(0, types)
    p = make_params(models)
    exh = args.exhaustiveness
    cmax = max(m.conf_size for m in models)

    def best64(seed):
        confs, mts, moc, steps, its = [], [], [], [], []
        for k, m in enumerate(models):
            sp = m.search_params(9)
            c, mt = m.seed_chains(seed + k, exh, gd)
            cm = np.zeros((exh, cmax))
            cm[:, :m.conf_size] = c
            confs += list(cm)
            mts += list(mt)
            moc += [k] * exh
            steps += [sp.num_steps] * exh
            its += [sp.maxiters] * exh
        t0 = time.perf_counter()
        b = e64.dock(0, models, moc, confs, mts, p, steps=steps, maxiters=its)
        out = []
        for k, m in enumerate(models):
            sp = m.search_params(9)
            e, conf, _ = sb.merge_chains(b, m, first=exh * k, n=exh, max_size=p.num_saved_mins)
            _, er, _ = e64.refine(0, [m], np.zeros(len(e), np.int32), conf, cap=tuple(p.authentic_v),
                                  maxiters=sp.maxiters, accurate_line=p.accurate_line, early_term=p.early_term)
            out.append(float(np.min(er)))
        return np.array(out), time.perf_counter() - t0

    K = max(2, args.acc_seeds)
    seeds = [args.seed + 7919 * k for k in range(K)]
    A64, t64 = [], []
    for sd in seeds:
        v, t = best64(sd)
        A64.append(v)
        t64.append(t)
    A32, t32 = [], []
    for sd in seeds:
        jobs = jobs_for(models, list(range(len(models))), exh, sd, 0)
        t0 = time.perf_counter()
        r32 = e32.dock_batch(0, models, jobs, p, refine=True)
        t32.append(time.perf_counter() - t0)
        A32.append(np.array([float(r["e"][0]) for r in r32]))
    A64, A32 = np.array(A64), np.array(A32)

    def spread(X, Y, pairs):
        d = np.concatenate([X[k] - Y[l] for k, l in pairs])
        return {"mean": float(d.mean()), "sd": float(d.std(ddof=1)), "median_abs": float(np.median(np.abs(d))),
                "pairs": len(pairs)}

    within = [(k, l) for k in range(K) for l in range(K) if k < l]
    cross = [(k, l) for k in range(K) for l in range(K)]
    s64 = A64.std(axis=0, ddof=1)  # per-ligand spread over seeds
    s32 = A32.std(axis=0, ddof=1)
    rng = np.random.default_rng(1)
    boot_w, boot_c = [], []
    for _ in range(2000):  # ligands resampled with replacement
        i = rng.integers(0, len(models), len(models))
        ww64 = np.concatenate([A64[k, i] - A64[l, i] for k, l in within]).std(ddof=1)
        ww32 = np.concatenate([A32[k, i] - A32[l, i] for k, l in within]).std(ddof=1)
        cc = np.concatenate([A32[k, i] - A64[l, i] for k, l in cross]).std(ddof=1)
        boot_w.append(ww32 / ww64)
        boot_c.append(cc / ww64)
    try:
        from scipy.stats import wilcoxon
        p_w = float(wilcoxon(s32, s64).pvalue)
    except Exception:
        p_w = None
    print(json.dumps({
        "accuracy": f"top-score agreement, {len(models)} ligands spread over the screen, full smina steps, "
                    f"exhaustiveness {exh}, merge + FP64 refine on both sides, {K} seeds per path",
        "precision": args.precision,
        "target_sd_kcal_mol": 0.08,
        "fp32_minus_fp64": spread(A32, A64, cross),
        "fp64_seed_to_seed": spread(A64, A64, within),
        "fp32_seed_to_seed": spread(A32, A32, within),
        "sd_ratio_fp32_seed_to_seed_over_fp64": {
            "value": float(spread(A32, A32, within)["sd"] / spread(A64, A64, within)["sd"]),
            "ci95_ligand_bootstrap": [float(np.percentile(boot_w, 2.5)), float(np.percentile(boot_w, 97.5))]},
        "sd_ratio_fp32_minus_fp64_over_fp64_seed_to_seed": {
            "value": float(spread(A32, A64, cross)["sd"] / spread(A64, A64, within)["sd"]),
            "ci95_ligand_bootstrap": [float(np.percentile(boot_c, 2.5)), float(np.percentile(boot_c, 97.5))]},
        "per_ligand_sd_over_seeds": {"fp64_median": float(np.median(s64)), "fp32_median": float(np.median(s32)),
                                     "fp64_mean": float(s64.mean()), "fp32_mean": float(s32.mean()),
                                     "fraction_fp32_above": float((s32 > s64).mean()),
                                     "wilcoxon_p": p_w},
        "per_ligand_mean_fp32_minus_fp64": {"mean": float((A32.mean(0) - A64.mean(0)).mean()),
                                            "sd": float((A32.mean(0) - A64.mean(0)).std(ddof=1))},
        "best_energy_mean": {"fp32": float(A32.mean()), "fp64": float(A64.mean())},
        "wall_s": {"fp64_runs": t64, "fp32_runs": t32},
        "ligands_per_s": {"fp64_plain": len(models) / float(np.mean(t64)),
                          "fp32_batched": len(models) / float(np.mean(t32))},
        "best_energies": {"fp64": A64.round(4).tolist(), "fp32": A32.round(4).tolist()},
    }), flush=True)


def run_plain64(args):
    """The same screen through the plain FP64 path (the reference's
    --gpu_fp64 search): every chain of every ligand in one sg_dock launch
    with host-seeded mt19937 streams, then merge and FP64 refinement per
    ligand.  Prints ligands/s of device-and-host wall time, for the
    comparison with the batched FP32 search."""
    spec = screen(args.ligands, args.seed)
    models = build_models(spec)
    R = sb.Receptor(3000, 7, CENTER)
    T = sb.Tables("vina")
    gd = sb.make_box(CENTER, (22.0, 22.0, 22.0))
    eng = sb.Engine(0, sb.PREC_FP64)
    eng.set_tables(T)
    eng.set_receptor(0, R, gd)
    eng.build_grids(0, sorted({t for m in models for t in m.types() if 1 < t < 27}))
    p = make_params(models)
    p.visited = 1 if args.visited else 0
    exh = args.exhaustiveness
    cmax = max(m.conf_size for m in models)
    confs, mts, moc, steps, its = [], [], [], [], []
    for k, m in enumerate(models):
        sp = m.search_params(9)
        c, mt = m.seed_chains(args.seed + k, exh, gd)
        cm = np.zeros((exh, cmax))
        cm[:, :m.conf_size] = c
        confs += list(cm)
        mts += list(mt)
        moc += [k] * exh
        n = max(1, int(sp.num_steps * args.step_scale)) if args.step_scale != 1.0 else sp.num_steps
        steps += [n] * exh
        its += [sp.maxiters] * exh
    with Clocks(0) as clk:
        t0 = time.perf_counter()
        b = eng.dock(0, models, moc, confs, mts, p, steps=steps, maxiters=its)
        t_dock = time.perf_counter() - t0
        best = []
        for k, m in enumerate(models):
            sp = m.search_params(9)
            e, conf, _ = sb.merge_chains(b, m, first=exh * k, n=exh, max_size=p.num_saved_mins)
            _, er, _ = eng.refine(0, [m], np.zeros(len(e), np.int32), conf, cap=tuple(p.authentic_v),
                                  maxiters=sp.maxiters, accurate_line=p.accurate_line, early_term=p.early_term)
            best.append(float(np.min(er)) if len(er) else float("nan"))
        wall = time.perf_counter() - t0
    clocks = clk.summary()
    evals = int(np.sum(b.evals))
    print(json.dumps({
        "mode": "plain64", "metric": "ligands docked/sec, plain FP64 path", "value": len(models) / wall,
        "unit": UNIT, "n_gpus": 1, "dtype": "f64", "data": "synthetic", "wall_s": wall, "search_wall_s": t_dock,
        "evals_per_s": evals / t_dock, "evals": evals, "visited": bool(args.visited),
        "best_energy_mean": float(np.mean(best)),
        "config": {"workload": f"virtual screen, {args.ligands} ligands (heavy U[10,50], rotors U[0,12]), receptor "
                               f"3000 heavy atoms, 22 A box at 0.375 A, exhaustiveness {exh}, smina step counts"
                               + (f" x {args.step_scale}" if args.step_scale != 1.0 else "")
                               + ", all chains in one launch, merge + FP64 refine per ligand"},
        "clocks": {k_: clocks[k_] for k_ in ("sm_mhz", "sm_max_mhz", "reasons")},
    }), flush=True)


# config 5's custom scoring: the five distance terms of vina with user weights
CUSTOM_FLEX = ("-0.0400 gauss(o=0,_w=0.5,_c=8)\n-0.0060 gauss(o=3,_w=2,_c=8)\n0.8000 repulsion(o=0,_c=8)\n"
               "-0.0300 hydrophobic(g=0.5,_b=1.5,_c=8)\n-0.5500 non_dir_h_bond(g=-0.7,_b=0,_c=8)\n"
               "1.923 num_tors_div\n")


def run_flex(args):
    """Flexible residues, custom scoring and FP16 maps: ligands drawn from the
    20,000-ligand screen (heavy atoms U[10,50], rotors U[0,12]) docked with
    4 synthetic flexible side chains (2-4 chi torsions each) next to the
    cavity of the 3,000-atom receptor, a custom scoring file (vina's five
    distance terms with user weights), grid maps stored in FP16 and
    interpolated in FP32.  Times ``args.flex_screen`` evenly spaced ligands
    of that screen through the batched search (merge + FP64 refinement) and
    extrapolates to 20,000; then, on the first ``args.flex_acc`` of them,
    compares the top refined energies of the FP16 search with the plain FP64
    search (two seeds each, so FP64's own seed-to-seed spread stands beside
    the difference)."""
    spec = screen(20000, args.seed)
    idx = [int(i) for i in np.linspace(0, len(spec) - 1, args.flex_screen)]
    flex = sb.make_flex_pdbqt(4, args.seed, CENTER)
    models = [sb.Model(sb.make_ligand_pdbqt(*spec[i][:2], spec[i][2], CENTER), flex) for i in idx]
    R = sb.Receptor(3000, 7, CENTER)
    T = sb.Tables("vina", CUSTOM_FLEX)
    gd = sb.make_box(CENTER, (22.0, 22.0, 22.0))
    types = sorted({t for m in models for t in m.types() if 1 < t < 27})
    e16 = sb.Engine(0, sb.PREC_FP32_H16)
    e16.set_tables(T)
    e16.set_receptor(0, R, gd)
    e16.build_grids(0, types)
    p = make_params(models)
    exh = args.exhaustiveness
    jobs = jobs_for(models, list(range(len(models))), exh, args.seed, 0, args.step_scale)
    e16.dock_batch(0, models[:2], jobs_for(models, [0, 1], exh, args.seed, 0, 0.01), p, refine=True)  # warm-up
    with Clocks(0) as clk:
        t0 = time.perf_counter()
        r16 = e16.dock_batch(0, models, jobs, p, refine=True)
        wall = time.perf_counter() - t0
    clocks = clk.summary()
    lps = len(models) / wall
    print(f"flex: {len(models)} ligands searched in {wall:.1f} s", file=sys.stderr, flush=True)
    evals = int(sum(r["evals"] for r in r16))
    line = {
        "mode": "flex_fp16_custom", "metric": "ligands docked/sec, flexible residues + custom scoring + FP16 maps",
        "value": lps, "unit": UNIT, "n_gpus": 1, "dtype": "f32 (f16 maps)", "data": "synthetic",
        "ligands_timed": len(models), "chains": len(models) * exh, "wall_s": wall, "evals_per_s": evals / wall,
        "extrapolated_20000_ligands_s": 20000 / lps,
        "flex": {"residues": 4, "torsions_added": int(models[0].dof - 6 - models[0].torsdof)},
        "config": {"workload": f"{len(models)} of a 20,000-ligand screen (heavy U[10,50], rotors U[0,12]) with 4 "
                               "flexible side chains (2-4 chi each), receptor 3000 heavy atoms, 22 A box at 0.375 A, "
                               f"custom scoring (vina's five terms, user weights), FP16 maps, exhaustiveness {exh}, "
                               "smina step counts" + (f" x {args.step_scale}" if args.step_scale != 1.0 else "")
                               + ", one persistent launch, merge + FP64 refine"},
        "clocks": {k_: clocks[k_] for k_ in ("sm_mhz", "sm_max_mhz", "reasons")},
    }
    # accuracy on a subsample: FP16 batched (two seeds) against plain FP64 (two seeds)
    na = min(args.flex_acc, len(models))
    if na < 2:  # the rate alone
        print(json.dumps(line), flush=True)
        return
    sub = models[:na]
    e64 = sb.Engine(0, sb.PREC_FP64)
    e64.set_tables(T)
    e64.set_receptor(0, R, gd)
    e64.build_grids(0, types)
    cmax = max(m.conf_size for m in sub)

    def best64(seed):
        confs, mts, moc, steps, its = [], [], [], [], []
        for k, m in enumerate(sub):
            sp = m.search_params(9)
            c, mt = m.seed_chains(seed + k, exh, gd)
            cm = np.zeros((exh, cmax))
            cm[:, :m.conf_size] = c
            confs += list(cm)
            mts += list(mt)
            moc += [k] * exh
            n = max(1, int(sp.num_steps * args.step_scale)) if args.step_scale != 1.0 else sp.num_steps
            steps += [n] * exh
            its += [sp.maxiters] * exh
        b = e64.dock(0, sub, moc, confs, mts, p, steps=steps, maxiters=its)
        out = []
        for k, m in enumerate(sub):
            sp = m.search_params(9)
            e, conf, _ = sb.merge_chains(b, m, first=exh * k, n=exh, max_size=p.num_saved_mins)
            _, er, _ = e64.refine(0, [m], np.zeros(len(e), np.int32), conf, cap=tuple(p.authentic_v),
                                  maxiters=sp.maxiters, accurate_line=p.accurate_line, early_term=p.early_term)
            out.append(float(np.min(er)))
        return np.array(out)

    t1 = time.perf_counter()
    a64 = best64(args.seed)
    print(f"flex: FP64 run 1 of {na} ligands in {time.perf_counter() - t1:.1f} s", file=sys.stderr, flush=True)
    b64 = best64(args.seed + 7919)
    t64 = (time.perf_counter() - t1) / 2
    a16 = np.array([float(r["e"][0]) for r in r16[:na]])
    r16b = e16.dock_batch(0, sub, jobs_for(sub, list(range(na)), exh, args.seed + 7919, 0, args.step_scale), p,
                          refine=True)
    b16 = np.array([float(r["e"][0]) for r in r16b])
    d_cross = np.concatenate([a16 - a64, a16 - b64, b16 - a64, b16 - b64])

    def st(d):
        return {"mean": float(d.mean()), "sd": float(d.std(ddof=1)), "median_abs": float(np.median(np.abs(d)))}

    line["accuracy"] = {"ligands": na, "seeds_per_path": 2,
                     "fp16_minus_fp64": st(d_cross), "fp64_seed_to_seed": st(b64 - a64),
                     "fp16_seed_to_seed": st(b16 - a16), "target_sd_kcal_mol": 0.08,
                     "best_energy_mean": {"fp16": float(np.concatenate([a16, b16]).mean()),
                                          "fp64": float(np.concatenate([a64, b64]).mean())},
                     "fp64_wall_s_per_run": t64}
    print(json.dumps(line), flush=True)


def heavy_rmsd(a, b):
    """Heavy-atom RMSD of two poses of one model (same atom order, no
    symmetry matching), as smina's rmsd_upper_bound (coords.cpp:25-33)."""
    a, b = np.asarray(a, float).reshape(-1, 3), np.asarray(b, float).reshape(-1, 3)
    return float(np.sqrt(((a - b) ** 2).sum(1).mean())) if len(a) else 0.0


def run_lone(args):
    """A lone ligand's search latency at 32, 64 and 128 threads per chain:
    each ligand of ``args.lone`` ("heavy:rotors,...", synthetic, seed 11)
    docked alone through the batched entry point (exhaustiveness 8, smina's
    step counts, seed 5) against the 3,000-atom receptor (22 A box at
    0.375 A, default scoring), with the device otherwise idle.  For each it
    runs the previous launch shape (32 threads, 8 chains per block), then 32,
    64 and 128 threads with the automatic shape, and prints one JSON line per
    run with the search time (CUDA events, ``sg_batch_stats``)."""
    import workloads as W
    eng = sb.Engine(0, sb.PREC_FP32)
    eng.set_tables(W.tables())
    eng.set_receptor(0, W.receptor(), W.box())
    for spec in args.lone.split(","):
        heavy, rot = (int(x) for x in spec.split(":"))
        m = W.ligand(heavy, rot, 11)
        p = m.search_params()
        steps = max(1, int(p.num_steps * args.step_scale))
        job = sb.LigandJob(model=0, num_chains=args.exhaustiveness, num_steps=steps, maxiters=0, seed=5, ligand_key=1)
        eng.set_threads_per_chain(32)
        eng.dock_batch(0, [m], [sb.LigandJob(model=0, num_chains=args.exhaustiveness, num_steps=2, maxiters=0, seed=5,
                                             ligand_key=1)], p)  # warm-up
        for tpc, cpb in [(32, 8), (32, 0), (64, 0), (128, 0)]:
            eng.set_threads_per_chain(tpc)
            eng.set_chains_per_block(cpb)
            t0 = time.perf_counter()
            r = eng.dock_batch(0, [m], [job], p, refine=True)[0]
            wall = time.perf_counter() - t0
            st = eng.batch_stats()
            print(json.dumps({"mode": "lone", "heavy": heavy, "rotors": rot, "steps": steps, "threads_per_chain": tpc,
                              "chains_per_block": st["chains_per_block"], "search_ms": round(st["mc_ms"], 1),
                              "wall_s": round(wall, 2), "best_e": float(r["e"][0]), "evals": int(r["evals"])}),
                  flush=True)
        eng.set_chains_per_block(0)
    eng.close()


def run_redock(args):
    """The single-ligand redock: a 24-heavy-atom, 5-rotor ligand against the
    3,000-atom receptor (22 A box at 0.375 A, default scoring, smina's step
    and BFGS-iteration counts).  Plain FP64 at exhaustiveness 8 and the
    batched FP32 search at exhaustiveness 128, each repeated with
    ``args.redock`` seeds; both merge with min_rmsd 2 and refine every
    merged pose in FP64.  Reports, per seed, the FP32 top pose's energy
    difference and heavy-atom RMSD against the FP64 top pose of the same
    seed index, next to FP64's own seed-to-seed figures."""
    reps = args.redock
    m = sb.Model(sb.make_ligand_pdbqt(24, 5, args.seed, CENTER))
    R = sb.Receptor(3000, 7, CENTER)
    T = sb.Tables("vina")
    gd = sb.make_box(CENTER, (22.0, 22.0, 22.0))
    types = sorted({t for t in m.types() if 1 < t < 27})
    e64 = sb.Engine(0, sb.PREC_FP64)
    e64.set_tables(T)
    e64.set_receptor(0, R, gd)
    e64.build_grids(0, types)
    e32 = sb.Engine(0, sb.PREC_FP32 if args.precision == "fp32" else sb.PREC_FP32_H16)
    e32.set_tables(T)
    e32.set_receptor(0, R, gd)
    e32.build_grids(0, types)
    p = m.search_params(9)
    exh64, exh32 = 8, 128
    seeds = [args.seed + 1009 * r for r in range(reps)]
    confs, mts = [], []
    for s in seeds:
        c, mt = m.seed_chains(s, exh64, gd)
        confs += list(c)
        mts += list(mt)
    t0 = time.perf_counter()
    b = e64.dock(0, [m], [0] * (exh64 * reps), confs, mts, p)
    top64 = []
    for r in range(reps):
        e, conf, _ = sb.merge_chains(b, m, first=exh64 * r, n=exh64, max_size=p.num_saved_mins)
        _, er, xyz = e64.refine(0, [m], np.zeros(len(e), np.int32), conf, cap=tuple(p.authentic_v),
                                maxiters=p.maxiters, accurate_line=p.accurate_line, early_term=p.early_term)
        k = int(np.argmin(er))
        top64.append((float(er[k]), xyz[k, :m.heavy]))
    t64 = time.perf_counter() - t0
    jobs = [sb.LigandJob(model=0, num_chains=exh32, num_steps=p.num_steps, maxiters=p.maxiters, seed=s,
                         ligand_key=r) for r, s in enumerate(seeds)]
    t0 = time.perf_counter()
    r32 = e32.dock_batch(0, [m], jobs, p, refine=True)
    t32 = time.perf_counter() - t0
    top32 = []
    for res in r32:
        k = int(np.argmin(res["e"]))
        top32.append((float(res["e"][k]), res["coords"][k]))
    de = [top32[r][0] - top64[r][0] for r in range(reps)]
    rmsd = [heavy_rmsd(top32[r][1], top64[r][1]) for r in range(reps)]
    pairs = [(i, j) for i in range(reps) for j in range(i + 1, reps)]
    de64 = [top64[j][0] - top64[i][0] for i, j in pairs]
    rmsd64 = [heavy_rmsd(top64[i][1], top64[j][1]) for i, j in pairs]
    print(json.dumps({
        "mode": "redock",
        "config": {"workload": f"single-ligand redock: ligand 24 heavy atoms, 5 rotors (seed {args.seed}); receptor "
                               "3000 heavy atoms; 22 A box at 0.375 A; default scoring; smina step and iteration "
                               f"counts ({p.num_steps} steps, {p.maxiters} BFGS iterations); FP64 plain at "
                               f"exhaustiveness {exh64}, FP32 batched at exhaustiveness {exh32}; {reps} seeds; "
                               "merge min_rmsd 2 + FP64 refine on both sides"},
        "precision": args.precision,
        "top_energy": {"fp64": [t[0] for t in top64], "fp32": [t[0] for t in top32]},
        "fp32_minus_fp64_energy": de,
        "fp32_vs_fp64_rmsd": rmsd,
        "fp64_seed_to_seed_energy": de64,
        "fp64_seed_to_seed_rmsd": rmsd64,
        "wall_s": {"fp64_plain": t64, "fp32_batched": t32},
    }), flush=True)


def run_fast(args):
    """The reference's --fast search (not smina's) on the same screen: chain
    split and step fraction chosen automatically by sgh_fast_chains for the
    screen's tasks on this device (16 resident chains per SM), then merge and
    FP64 refinement as in the headline.  Reports ligands/s of the call and
    the mean best refined energy, beside the same for smina's search."""
    spec = screen(args.ligands, args.seed)
    models = build_models(spec)
    R = sb.Receptor(3000, 7, CENTER)
    T = sb.Tables("vina")
    gd = sb.make_box(CENTER, (22.0, 22.0, 22.0))
    eng = sb.Engine(0, sb.PREC_FP32)
    eng.set_tables(T)
    eng.set_receptor(0, R, gd)
    eng.build_grids(0, sorted({t for m in models for t in m.types() if 1 < t < 27}))
    p = make_params(models)
    cap = 16 * eng.device_info()["num_sms"]
    runs = {}
    for name, jobs in (("smina", jobs_for(models, list(range(len(models))), args.exhaustiveness, args.seed, 0)),
                       ("fast", sb.fast_jobs(models, args.exhaustiveness, args.seed, cap))):
        eng.dock_batch(0, models[:2], [sb.LigandJob(model=k, num_chains=2, num_steps=5, maxiters=j.maxiters,
                                                    seed=j.seed, ligand_key=j.ligand_key)
                                       for k, j in enumerate(jobs[:2])], p)  # warm
        with Clocks(0) as clk:
            t0 = time.perf_counter()
            r = eng.dock_batch(0, models, jobs, p)
            wall = time.perf_counter() - t0
        st = eng.batch_stats()
        runs[name] = {"ligands_per_s": len(models) / wall, "wall_s": wall, "search_ms": st["mc_ms"],
                      "refine_ms": st["refine_ms"], "chains_per_ligand": jobs[0].num_chains,
                      "steps_of_first_ligand": jobs[0].num_steps,
                      "mean_best_e": float(np.mean([x["e"][0] for x in r if len(x["e"])])),
                      "clocks": {k_: clk.summary()[k_] for k_ in ("sm_mhz", "sm_max_mhz", "reasons")}}
    print(json.dumps({
        "mode": "fast", "metric": "ligands docked/sec, --fast search (not smina's)", "unit": UNIT, "n_gpus": 1,
        "config": {"workload": f"virtual screen, {args.ligands} ligands (heavy U[10,50], rotors U[0,12]), receptor "
                               f"3000 heavy atoms, 22 A box at 0.375 A, exhaustiveness {args.exhaustiveness}; "
                               "automatic chain split and step fraction; merge + FP64 refine"},
        "runs": runs,
    }), flush=True)


REF_SEARCH_SO = os.path.join(ROOT, "baseline", "_ref", "libref_search32.so")


def run_ref_gpu(args):
    """The reference's own FP32 GPU search on this GPU, beside this engine's,
    on the same screen.  baseline/_ref/libref_search32.so holds the
    reference's device library (src/gpu/gpu_device.cu, gpu_kernels_f32.cu)
    compiled for sm_100a from its sources (make -C baseline/ref_gpu, which
    needs the reference tree).  Both searches get every chain of every
    ligand at once, smina's step counts (times --step-scale), no refinement;
    the reference's chains start from host-seeded confs and mt19937 states,
    this engine's from its own counter-based streams.  Reported: each
    search's time and ligands/s, and the mean best (unrefined) energy."""
    import ctypes as C
    if not os.path.exists(REF_SEARCH_SO):
        print(json.dumps({"mode": "reference_gpu", "unavailable": "baseline/_ref/libref_search32.so is not built "
                                                                   "(make -C baseline/ref_gpu needs the reference tree)"}))
        return
    L = C.CDLL(REF_SEARCH_SO)
    L.refs_last_error.restype = C.c_char_p
    L.refs_create.argtypes = [C.POINTER(sb.TablesDesc), C.POINTER(sb.ReceptorDesc), C.POINTER(sb.GridDims), sb._ip,
                              C.c_int, C.c_double, C.POINTER(C.c_void_p)]
    L.refs_dock.argtypes = [C.c_void_p, C.POINTER(sb.ModelDesc), C.c_int, C.POINTER(sb.ChainInput), C.c_int,
                            C.POINTER(sb.MCParams), C.POINTER(sb.ChainResult), C.POINTER(C.c_double)]
    L.refs_destroy.argtypes = [C.c_void_p]
    spec = screen(args.ligands, args.seed)
    models = build_models(spec)
    R = sb.Receptor(3000, 7, CENTER)
    T = sb.Tables("vina")
    gd = sb.make_box(CENTER, (22.0, 22.0, 22.0))
    types = np.array(sorted({t for m in models for t in m.types() if 1 < t < 27}), np.int32)
    p = make_params(models)
    exh = args.exhaustiveness

    def ref_chains(ms):
        confs, mts, moc, steps, its = [], [], [], [], []
        for k, m in enumerate(ms):
            sp = m.search_params(9)
            c, mt = m.seed_chains(args.seed + k, exh, gd)
            confs += list(c)
            mts += list(mt)
            moc += [k] * exh
            steps += [max(1, int(sp.num_steps * args.step_scale))] * exh
            its += [sp.maxiters] * exh
        return sb.make_chain_batch(ms, moc, confs, mts, steps, p.num_saved_mins, [m.heavy for m in ms], its)

    def ref_dock(ms, b):
        descs = (sb.ModelDesc * len(ms))(*[m.desc for m in ms])
        secs = C.c_double()
        rc = L.refs_dock(h, descs, len(ms), b.inputs, len(b.e), C.byref(p), b.results, C.byref(secs))
        if rc != 0:
            raise RuntimeError("reference search: " + L.refs_last_error().decode())
        return secs.value

    h = C.c_void_p()
    if L.refs_create(C.byref(T.desc), C.byref(R.desc), C.byref(gd), sb.iptr(types), len(types), 1e6, C.byref(h)):
        raise RuntimeError("reference maps: " + L.refs_last_error().decode())
    warm = models[:2]
    ref_dock(warm, ref_chains(warm))  # loads the reference's kernels
    b = ref_chains(models)
    t_ref = ref_dock(models, b)
    cnt = [b.results[c].count for c in range(len(b.e))]
    best_ref = []
    for k in range(len(models)):
        vals = [b.e[c, :cnt[c]].min() for c in range(exh * k, exh * (k + 1)) if cnt[c] > 0]
        best_ref.append(float(min(vals)) if vals else float("nan"))
    L.refs_destroy(h)
    eng = sb.Engine(0, sb.PREC_FP32)
    eng.set_tables(T)
    eng.set_receptor(0, R, gd)
    eng.build_grids(0, [int(t) for t in types])
    jobs = jobs_for(models, list(range(len(models))), exh, args.seed, 0, args.step_scale)
    eng.dock_batch(0, models[:2], jobs_for(models[:2], [0, 1], exh, args.seed, 0, 0.001), p, refine=False)
    t0 = time.perf_counter()
    r = eng.dock_batch(0, models, jobs, p, refine=False)
    t_ours_wall = time.perf_counter() - t0
    t_ours = eng.batch_stats()["mc_ms"] / 1000.0
    best_ours = [float(x["e"][0]) if len(x["e"]) else float("nan") for x in r]
    n = len(models)
    print(json.dumps({
        "mode": "reference_gpu",
        "config": {"workload": f"virtual screen, {n} ligands (heavy U[10,50], rotors U[0,12]), receptor 3000 heavy "
                               f"atoms, 22 A box at 0.375 A, exhaustiveness {exh}, smina step counts"
                               + (f" x {args.step_scale}" if args.step_scale != 1.0 else "")
                               + ", every chain at once, search only (no merge, no refinement)"},
        "reference_fp32": {"search_s": t_ref, "ligands_per_s": n / t_ref,
                           "how": "run_monte_carlo<float>, 32 threads per chain, wall time of the call",
                           "mean_best_e_unrefined": float(np.nanmean(best_ref))},
        "this_engine_fp32": {"search_s": t_ours, "ligands_per_s": n / t_ours, "call_wall_s": t_ours_wall,
                             "how": "k_mc32 persistent launch, CUDA-event time of the search launch",
                             "mean_best_e_unrefined": float(np.nanmean(best_ours))},
    }), flush=True)


SERVE_RECEPTORS = ((2000, 22.0), (3000, 26.0), (5000, 30.0))  # (heavy atoms, box edge in A)


def run_serve(args):
    """Serving: ``args.serve`` single-ligand requests with seeded Poisson
    arrivals at ``args.rate`` per second, spread round-robin over three
    resident receptors (2,000 / 3,000 / 5,000 heavy atoms in 22 / 26 / 30 A
    boxes), ligands with heavy atoms U[10, 60] and rotors U[0, 15],
    exhaustiveness 8.  Latency is the engine's own submit-to-result time of
    each request (queueing, search, merge and FP64 refinement)."""
    # more hardware queues for the server's many streams (read when the CUDA context is created)
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    rng = np.random.default_rng(args.seed)
    n = args.serve
    spec = [(int(rng.integers(10, 61)), int(rng.integers(0, 16)), 20_000 + k) for k in range(n)]
    models = build_models(spec)
    T = sb.Tables("vina")
    eng = sb.Engine(0, sb.PREC_FP32 if args.precision == "fp32" else sb.PREC_FP32_H16)
    eng.set_tables(T)
    types = sorted({t for m in models for t in m.types() if 1 < t < 27})
    for i, (na, edge) in enumerate(SERVE_RECEPTORS):
        eng.set_receptor(i, sb.Receptor(na, 7 + i, CENTER), sb.make_box(CENTER, (edge,) * 3))
        eng.build_grids(i, types)
    p = make_params(models)
    jobs = jobs_for(models, list(range(n)), args.exhaustiveness, args.seed, 0, args.step_scale)
    for j in jobs:
        j.model = 0
    if args.rates:  # piecewise-constant Poisson rates, cycling every rate_period seconds
        rates = [float(x) for x in args.rates.split(",")]
        arrivals, t = [], 0.0
        while len(arrivals) < n:
            seg = int(t // args.rate_period) % len(rates)
            t_next = t + rng.exponential(1.0 / rates[seg])
            seg_end = (t // args.rate_period + 1) * args.rate_period
            if t_next > seg_end:  # memoryless: restart at the segment boundary with the next rate
                t = seg_end
                continue
            t = t_next
            arrivals.append(t)
        arrivals = np.array(arrivals)
    else:
        arrivals = np.cumsum(rng.exponential(1.0 / args.rate, n))
    eng.set_threads_per_chain(args.threads_per_chain)
    eng.serve_start(block_smem_bytes=args.serve_block_smem)
    lat, evals, dev, queue, searched, done_at, tpcs = {}, 0, {}, {}, {}, {}, {}
    k = 0
    occupancy = []  # (queued, ligands in flight) sampled every 100 ms
    next_sample = 0.0
    with Clocks(0) as clk:
        t0 = time.perf_counter()
        while len(lat) < n:
            now = time.perf_counter() - t0
            while k < n and arrivals[k] <= now:
                eng.serve_submit(k % len(SERVE_RECEPTORS), models[k], jobs[k], p)
                k += 1
            if now >= next_sample:
                st = eng.serve_stats()
                occupancy.append((st["queued"], st["inflight"]))
                next_sample = now + 0.1
            wait = 1 if k < n else 20
            for (t, st, cnt, ms, ev, cs, nh, launch, d0, d1, qms, sms, tpc) in eng.serve_poll(256, wait_ms=wait,
                                                                                                spans=True):
                if st != 0:
                    raise RuntimeError(f"request {t} failed with status {st}")
                eng.serve_fetch(t, cnt, cs, nh)
                lat[t] = ms
                done_at[t] = time.perf_counter() - t0
                dev[t] = (launch, d0, d1)
                queue[t] = qms
                searched[t] = sms
                tpcs[t] = tpc
                evals += ev
        wall = time.perf_counter() - t0
    eng.serve_stop()
    v = np.array(list(lat.values()))
    dms = np.array([(d1 - d0) / 1e6 for (_, d0, d1) in dev.values()])
    tk = list(lat)
    launch_to_done = np.array([searched[t] - queue[t] for t in tk])
    after_search = np.array([lat[t] - searched[t] for t in tk])
    d0s = [d[1] for d in dev.values()]
    busy_s = (max(d[2] for d in dev.values()) - min(d0s)) / 1e9
    concurrency = float(dms.sum() / 1e3 / busy_s) if busy_s > 0 else None
    # completions per second over the middle 80 % of them (the ramp-up and the
    # drain of the last, longest ligands left out), and the device spans
    # inside that window
    tdone = np.sort(np.array(list(done_at.values())))
    t10, t90 = np.percentile(tdone, 10), np.percentile(tdone, 90)
    mid_rate = float(((tdone >= t10) & (tdone <= t90)).sum() / (t90 - t10)) if t90 > t10 else None
    launches = len({l for (l, _, _) in dev.values()})
    clocks = clk.summary()
    print(json.dumps({
        "mode": "serve", "metric": "request latency (p50/p99) and ligands/s under Poisson arrivals",
        "value": n / wall, "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
        "latency_ms": {"p50": float(np.percentile(v, 50)), "p99": float(np.percentile(v, 99)),
                       "max": float(v.max()), "mean": float(v.mean())},
        "device_search_ms": {"p50": float(np.percentile(dms, 50)), "p99": float(np.percentile(dms, 99)),
                             "mean": float(dms.mean())},
        "queue_ms": {"p50": float(np.percentile(list(queue.values()), 50)),
                     "p99": float(np.percentile(list(queue.values()), 99)), "mean": float(np.mean(list(queue.values())))},
        "launch_to_chains_done_ms": {"p50": float(np.percentile(launch_to_done, 50)),
                                     "mean": float(launch_to_done.mean())},
        "merge_refine_ms": {"p50": float(np.percentile(after_search, 50)), "mean": float(after_search.mean())},
        "ligands_searching_at_once": concurrency,
        "completions_per_s_middle_80pct": mid_rate,
        "launches": launches,
        "threads_per_chain": {str(c): int(sum(1 for x in tpcs.values() if x == c)) for c in sorted(set(tpcs.values()))},
        "requests": n, "offered_rate_per_s": args.rates or args.rate, "wall_s": wall, "evals_per_s": evals / wall,
        "inflight_ligands": {"mean": float(np.mean([o[1] for o in occupancy])),
                             "max": int(max(o[1] for o in occupancy)),
                             "mean_while_requests_wait": float(np.mean([o[1] for o in occupancy if o[0] > 0]))
                             if any(o[0] > 0 for o in occupancy) else None},
        "queued": {"mean": float(np.mean([o[0] for o in occupancy])), "max": int(max(o[0] for o in occupancy))},
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{n} requests, ligands heavy U[10,60] rotors U[0,15], receptors "
                               f"{[r[0] for r in SERVE_RECEPTORS]} heavy atoms in {[r[1] for r in SERVE_RECEPTORS]} A "
                               f"boxes at 0.375 A, exhaustiveness {args.exhaustiveness}, smina step counts"
                               + (f" x {args.step_scale}" if args.step_scale != 1.0 else ""),
                   "precision": args.precision,
                   "arrivals": (f"Poisson at rates {args.rates} per second, each for {args.rate_period} s in turn"
                                if args.rates else f"Poisson at {args.rate} per second") + f", seed {args.seed}",
                   "block_smem_bytes": args.serve_block_smem or "automatic",
                   "threads_per_chain": args.threads_per_chain or "automatic (by the blocks in flight)"},
        "clocks": {k_: clocks[k_] for k_ in ("sm_mhz", "sm_max_mhz", "reasons")},
    }), flush=True)


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=1800))
        pg = dist
    return world, rank, local, pg


def reduce_max(pg, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def run_reference(args, world, rank):
    """The reference arm: the CPU restatement of smina's search on all host
    cores, on the same workload, each step a bounded sample of ligands."""
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    parallel = max(1, cores // args.exhaustiveness)
    spec = screen(args.ligands, args.seed)
    models = build_models(spec)
    R = sb.Receptor(3000, 7, CENTER)
    T = sb.Tables("vina")
    gd = sb.make_box(CENTER, (22.0, 22.0, 22.0))
    times = []
    for s in range(args.warmup + args.steps):
        # ligands spread evenly over the screen, a different set each step
        total = (args.warmup + args.steps) * parallel
        stride = max(1, len(models) // total)
        sub = [models[((s * parallel + i) * stride) % len(models)] for i in range(parallel)]
        v, dt, _ = cpu_sample(sub, gd, R, T, args.exhaustiveness, args.seed, len(sub), args.exhaustiveness, parallel)
        if s >= args.warmup:
            times.append((len(sub), dt))
    n = sum(a for a, _ in times)
    t = sum(b for _, b in times)
    value = n / t
    sample = (f"{n} ligands spread over the screen ({parallel} at a time, {args.exhaustiveness} chains each at "
              f"smina's full step count, merge + refine)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * t / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"virtual screen, {args.ligands} ligands (heavy U[10,50], rotors U[0,12]), receptor "
                               "3000 heavy atoms, 22 A box, exhaustiveness 8", "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": parallel * args.exhaustiveness, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ligands", type=int, default=1000, help="ligands in the screen")
    ap.add_argument("--batch", type=int, default=0, help="ligands per step (0: the whole screen)")
    ap.add_argument("--exhaustiveness", type=int, default=8)
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp16"])
    ap.add_argument("--cpu-ligands", type=int, default=4, help="ligands in the CPU baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--chains-per-block", type=int, default=0)
    ap.add_argument("--threads-per-chain", type=int, default=32, choices=[0, 32, 64, 128],
                    help="threads per chain of the batched search and the serving loop (0: automatic)")
    ap.add_argument("--autotune", type=float, default=0.0,
                    help="autotune the launch shape first on the step's ligands at this fraction of their steps "
                         "(0: the occupancy rule; short samples overweight the wait for each block's slowest chain)")
    ap.add_argument("--step-scale", type=float, default=1.0,
                    help="scale every ligand's Monte Carlo step count (profiling cases; 1 = smina's counts)")
    ap.add_argument("--accuracy", type=int, default=0,
                    help="instead of timing: top-score agreement FP32 vs FP64 on this many ligands")
    ap.add_argument("--acc-seeds", type=int, default=4, help="with --accuracy: seeds per path (at least 2)")
    ap.add_argument("--serve", type=int, default=0,
                    help="instead of the screen: this many requests through the serving loop (p50/p99 latency)")
    ap.add_argument("--rate", type=float, default=20.0, help="offered request rate for --serve (per second)")
    ap.add_argument("--rates", default="",
                    help="with --serve: comma-separated Poisson rates (per second), each held for --rate-period s in turn")
    ap.add_argument("--rate-period", type=float, default=60.0)
    ap.add_argument("--serve-block-smem", type=int, default=0,
                    help="with --serve: dynamic shared memory per search block (0: the server's default)")
    ap.add_argument("--plain64", action="store_true",
                    help="instead of the batched search: the same screen through the plain FP64 path")
    ap.add_argument("--visited", action="store_true",
                    help="with --plain64: QuickVina 2's history check (not smina's search)")
    ap.add_argument("--fast", action="store_true",
                    help="instead of timing: the reference's --fast search (not smina's) beside smina's, same screen")
    ap.add_argument("--ref-gpu", action="store_true",
                    help="instead of timing: the reference's own FP32 GPU search (built from its sources into "
                         "baseline/_ref) beside this engine's, on the same screen")
    ap.add_argument("--flex-screen", type=int, default=0,
                    help="instead of timing the screen: this many ligands of the 20,000-ligand screen with 4 flexible "
                         "residues, custom scoring and FP16 maps, plus an accuracy check against FP64")
    ap.add_argument("--lone", default="",
                    help="heavy:rotors,... -- a lone ligand's search time at 32, 64 and 128 threads per chain")
    ap.add_argument("--flex-acc", type=int, default=24, help="with --flex-screen: ligands in the FP64 comparison")
    ap.add_argument("--redock", type=int, default=0,
                    help="instead of timing: the single-ligand redock (FP64 exhaustiveness 8, FP32 exhaustiveness "
                         "128) with this many seeds; top-pose energy and RMSD differences")
    args = ap.parse_args()
    assert args.warmup >= 3, "at least 3 warm-up steps"
    if args.accuracy:
        run_accuracy(args)
        return
    if args.redock:
        run_redock(args)
        return
    if args.flex_screen:
        run_flex(args)
        return
    if args.lone:
        run_lone(args)
        return
    if args.ref_gpu:
        run_ref_gpu(args)
        return
    if args.fast:
        run_fast(args)
        return
    if args.serve:
        run_serve(args)
        return
    if args.plain64:
        run_plain64(args)
        return
    world, rank, local, pg = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import torch
    torch.cuda.set_device(local)
    prec = sb.PREC_FP32 if args.precision == "fp32" else sb.PREC_FP32_H16
    spec = screen(args.ligands, args.seed)
    models = build_models(spec)
    R = sb.Receptor(3000, 7, CENTER)
    T = sb.Tables("vina")
    gd = sb.make_box(CENTER, (22.0, 22.0, 22.0))
    eng = sb.Engine(local, prec)
    eng.set_tables(T)
    eng.set_receptor(0, R, gd)
    types = sorted({t for m in models for t in m.types() if 1 < t < 27})
    eng.build_grids(0, types)
    p = make_params(models)
    B = args.batch or args.ligands
    tuned = None
    eng.set_threads_per_chain(args.threads_per_chain)
    if args.chains_per_block:
        eng.set_chains_per_block(args.chains_per_block)
    elif args.autotune > 0:  # launch shape timed on a short sample of the screen, before any timed step
        idx = list(range(B))  # one step's ligands, so the sample fills the device as a step does
        sample = jobs_for(models, idx, args.exhaustiveness, args.seed, 10_000_000)
        chosen, rates = eng.autotune(0, models[:B], sample, p, step_fraction=args.autotune)
        tuned = {"chosen": chosen, "evals_per_s": {str(c): round(v) for c, v in rates.items()},
                 "sample": f"{len(idx)} ligands at {args.autotune} of their steps"}
    nb = max(1, args.ligands // B)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > L2 (126 MB)
    key_base = 1_000_000 * rank

    def step(s):
        idx = list(range((s % nb) * B, (s % nb) * B + B))
        jobs = jobs_for(models, idx, args.exhaustiveness, args.seed, key_base, args.step_scale)
        sub = [models[k] for k in idx]
        for j, jb in enumerate(jobs):
            jb.model = j
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = eng.dock_batch(0, sub, jobs, p, refine=True)
        wall = time.perf_counter() - t0
        st = eng.batch_stats()
        return len(idx), wall, st, res

    for s in range(args.warmup):
        step(s)
    barrier(pg)
    torch.cuda.synchronize()
    recs = []
    with Clocks(local) as clk:
        for s in range(args.steps):
            recs.append(step(args.warmup + s))
    torch.cuda.synchronize()
    barrier(pg)
    n_lig = sum(r[0] for r in recs)
    dev_s = sum((r[2]["mc_ms"] + r[2]["refine_ms"]) / 1000 for r in recs)
    mc_s = sum(r[2]["mc_ms"] / 1000 for r in recs)
    wall_s = sum(r[1] for r in recs)
    dev_max = reduce_max(pg, dev_s)
    wall_max = reduce_max(pg, wall_s)
    value = n_lig * world / dev_max
    e2e = n_lig * world / wall_max
    gbytes = sum(r[2]["grid_lookups"] * G_BYTES[prec] + r[2]["pair_lookups"] * T_BYTES for r in recs)
    achieved = gbytes / mc_s / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak, peak_src = (peaks["hbm_gbs"], "measured") if "hbm_gbs" in peaks else (6650.0, "fallback")
    traffic = None
    tf = os.path.join(ROOT, "profiles", "k_mc32_traffic.json")
    if os.path.exists(tf):  # DRAM bytes of short-case ncu captures, extended to this launch by eval_deriv calls
        t = json.load(open(tf))
        if t.get("bytes_per_eval"):
            traffic = t.get("fixed_bytes", 0) + t["bytes_per_eval"] * sum(r[2]["evals"] for r in recs) / len(recs)
    # The gathers hit L2 (the maps of the screen's types and the table fit in
    # it), so their bound is the measured rate of random 32 B / 16 B gathers
    # over a working set of the same size, mixed in the kernel's proportion.
    roof_l2 = None
    if rank == 0:
        ncells = int(np.prod([gd.n[i] for i in range(3)]))
        ws = len(types) * ncells * G_BYTES[prec] + T.desc.n * 378 * T_BYTES
        g32 = eng.probe_gather(ws, 32) if G_BYTES[prec] == 32 else eng.probe_gather(ws, 16)
        g16 = eng.probe_gather(ws, 16)
        gb = sum(r[2]["grid_lookups"] * G_BYTES[prec] for r in recs)
        tb = sum(r[2]["pair_lookups"] * T_BYTES for r in recs)
        peak_l2 = (gb + tb) / (gb / g32 + tb / g16)
        roof_l2 = {"bound": "l2 gathers", "achieved": achieved, "peak": peak_l2, "unit": "GB/s",
                   "frac": achieved / peak_l2,
                   "peak_source": f"measured in this run: random {G_BYTES[prec]} B gathers {g32:.0f} GB/s and 16 B "
                                  f"gathers {g16:.0f} GB/s over {ws / 1e6:.0f} MB (sg_probe_gather), weighted by the "
                                  f"kernel's grid / table bytes"}
    evals = sum(r[2]["evals"] for r in recs)
    accuracy = None  # top-score agreement with the FP64 search, measured by the command it names
    af = os.path.join(ROOT, "profiles", "accuracy_fp32_vs_fp64_screen120.json")
    if os.path.exists(af):
        accuracy = json.load(open(af))
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = args.exhaustiveness
        v, dt, idx = cpu_sample(models, gd, R, T, args.exhaustiveness, args.seed, args.cpu_ligands, threads)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{len(idx)} ligands spread over the screen (indices {idx}), {args.exhaustiveness} chains "
                         f"each at smina's full step count, one thread per chain, merge + refine; {dt:.1f} s"}
    if rank == 0:
        clocks = clk.summary()
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * dev_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"virtual screen, {args.ligands} ligands (heavy U[10,50], rotors U[0,12]), "
                                   f"receptor 3000 heavy atoms, 22 A box at 0.375 A, exhaustiveness "
                                   f"{args.exhaustiveness}, smina step counts"
                                   + (f" x {args.step_scale}" if args.step_scale != 1.0 else "")
                                   + f", {B} ligands per step",
                       "precision": args.precision, "ligands_per_step": B, "global_batch": B * world,
                       "parallelism": f"replicas x{world}", "l2": "flushed between steps (256 MB write)",
                       "chains_per_block": recs[-1][2]["chains_per_block"], "blocks": recs[-1][2]["blocks"],
                       "autotune": tuned},
            "e2e": {"value": e2e, "unit": UNIT,
                    "h2d_bytes_per_step": int(sum(r[2]["h2d_bytes"] for r in recs) / len(recs)),
                    "d2h_bytes_per_step": int(sum(r[2]["d2h_bytes"] for r in recs) / len(recs))},
            "gpu_launches": 2 * args.steps,
            "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                         "kernel": "k_mc32"},
            "roofline_l2": roof_l2,
            "cpu_baseline": cpu,
            "accuracy": accuracy,
            "evals_per_s": evals / mc_s,
            "evals_per_step": evals / args.steps,
            "search_ms_per_step": 1000 * mc_s / args.steps,
        }), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
