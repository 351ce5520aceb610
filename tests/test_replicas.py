"""The multi-GPU form of the benchmark is replicas: one independent Markov
chain per rank, no exchange in the data path (the reference runs its chains
as separate jobs, rhmc/scan_in_beta.sh).  What crosses ranks is the timing:
every rank's elapsed time goes through a max-reduction, the job's figure is
the slowest rank's time over all ranks' trajectories, and each rank starts
its own generator seed.  Checked here on two gloo ranks on the CPU, through
the functions bench.py uses; the reference arm does no work on ranks other
than 0.
"""
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = 100.0 + 25.0 * rank                     # rank 1 is the slower one
        got = bench.max_over_ranks(ms, world, "cpu")
        dist.barrier()
        seed = bench.replica_seed(693764523745.0, rank)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{got!r} {seed!r}\n")
    finally:
        dist.destroy_process_group()


def test_two_replicas_reduce_the_slowest_time(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    vals = [open(tmp_path / f"rank{r}.txt").read().split() for r in range(world)]
    maxes = [float(v[0]) for v in vals]
    seeds = [float(v[1]) for v in vals]
    assert maxes == [125.0, 125.0]                 # every rank holds the slowest time
    assert seeds[0] == 693764523745.0              # rank 0: the single-GPU chain
    assert len(set(seeds)) == world                # independent chains


def test_whole_job_figure_and_single_rank():
    sys.path.insert(0, ROOT)
    import bench
    # 2 chains x 5 trajectories in 12.5 s (the slowest rank): 1.25 s a trajectory
    assert bench.seconds_per_trajectory(12500.0, 5, 2) == pytest.approx(1.25)
    assert bench.seconds_per_trajectory(12500.0, 5, 1) == pytest.approx(2.5)
    # a single rank needs no process group
    assert bench.max_over_ranks(42.0, 1, "cpu") == 42.0


def test_reference_arm_does_no_work_off_rank_zero(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        steps, warmup, L, Ls = 1, 0, 24, 24

    assert bench.run_reference(Args(), 1, 2) is None
    assert capsys.readouterr().out == ""
