"""Multi-GPU host logic on CPU: two gloo ranks stand in for two GPUs.

The path shards by samples (and a batch by jobs) with no exchange on the data
path; the collectives are the FP64 XYZ combination of a frame split by
samples and the max over ranks of the device time. Here each rank renders its
sample range with the CPU oracle, and the combined XYZ sums must equal one
process rendering all the samples."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from hdcodex_b200 import multigpu as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
W = H = 16
SPP = 2


def test_sample_ranges_are_disjoint_and_complete():
    for world in (1, 2, 3, 8):
        got = M.covered_samples(steps=3, world=world, spp=5)
        assert sorted(got) == list(range(3 * world * 5))


def test_job_shard_partitions_the_batch():
    for world in (1, 2, 4, 7):
        shards = [M.job_shard(64, world, r) for r in range(world)]
        assert sorted(j for s in shards for j in s) == list(range(64))
        assert max(map(len, shards)) - min(map(len, shards)) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]
    import torch.distributed as dist
    import oracle as O
    import ref_scenes as R
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = O.OracleTracer()
        t.set_scene(R.base_scene())
        s0 = M.sample_range(0, world, rank, SPP)
        _, xyz = t.render(R.base_camera(), W, H, s0, 8, SPP, want_xyz=True, threads=1)
        total, samples = M.combine_xyz_sums(xyz, SPP)
        slowest = M.max_over_ranks(float(rank + 1))
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), total)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{samples} {slowest}")
    finally:
        dist.destroy_process_group()


def test_two_ranks_combine_to_the_single_process_frame(oracle_lib, tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    import ref_scenes as R
    t = oracle_lib.OracleTracer()
    t.set_scene(R.base_scene())
    _, reference = t.render(R.base_camera(), W, H, 0, 8, world * SPP, want_xyz=True)
    for rank in range(world):
        total = np.load(tmp_path / f"rank{rank}.npy")
        samples, slowest = open(tmp_path / f"rank{rank}.txt").read().split()
        assert int(samples) == world * SPP
        assert float(slowest) == float(world)
        # The ranks' partial sums add in another order than one sequential sum.
        np.testing.assert_allclose(total, reference, rtol=1e-12, atol=1e-15)
