"""Multi-GPU runs are replicas: every rank docks its own copy of the screen
with its own random streams, and the only cross-rank steps are a barrier and
the max-over-ranks time.  These checks run those host steps as two gloo ranks
on the CPU (no GPU): the reduction, the barrier, the per-rank ligand keys,
and the reference arm's rule that only rank 0 works."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    class A:
        pass

    w, r, local, pg = bench.dist_setup(A())
    assert (w, r, local) == (world, rank, rank) and pg is not None
    slowest = bench.reduce_max(pg, 10.0 + rank)  # each rank's own time
    bench.barrier(pg)

    class M:
        def search_params(self, n):
            class P:
                num_steps, maxiters = 100, 10
            return P()

    jobs = bench.jobs_for([M()] * 4, list(range(4)), 8, 42, 1_000_000 * rank)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"max": slowest, "keys": [j.ligand_key for j in jobs], "seeds": [j.seed for j in jobs]}, f)
    pg.destroy_process_group()


def test_two_gloo_ranks_reduce_max_and_use_disjoint_ligand_keys(tmp_path):
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r0 = json.load(open(tmp_path / "rank0.json"))
    r1 = json.load(open(tmp_path / "rank1.json"))
    assert r0["max"] == r1["max"] == 11.0  # the job's time is the slowest rank's
    assert not set(r0["keys"]) & set(r1["keys"])  # each replica docks with its own random streams
    assert r0["seeds"] == r1["seeds"]


def test_reference_arm_runs_on_rank_zero_only(tmp_path):
    """Under torchrun the reference arm prints from rank 0; other ranks exit 0
    without work."""
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(_free_port()))
    code = ("import sys; sys.path.insert(0, %r); import bench\n"
            "class A: ligands = 4; seed = 42; exhaustiveness = 8; warmup = 3; steps = 1\n"
            "bench.run_reference(A(), 2, 1)\n" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == ""
