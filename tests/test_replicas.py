"""Multi-GPU host logic on CPU: two ranks over gloo (127.0.0.1).

The path shards by independent clouds (one process per GPU, no data-path
collective): each rank voxelizes its own contiguous run of clouds, and the
job's step time is the maximum over ranks.  Here each rank takes its shard of
an uneven batch, voxelizes it with the CPU oracle, and the ranks check with
collectives that the shards cover every cloud once, that the per-rank results
add up to the single-process results, and that the timing reduction takes the
slowest rank.
"""

import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _batch():
    from nanovdb_editor import workloads as W

    clouds, start, vs = W.batch_clouds(6, 11, 100, 600, vs_min=0.01, vs_max=0.03, max_clusters=3)
    return clouds, start, vs


def _rank_main(rank, world, port, out_dir):
    for p in (os.path.join(ROOT, "nanovdb-editor_b200"), os.path.join(ROOT, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime

    import torch.distributed as dist

    import oracle as O
    from nanovdb_editor import replicas as R

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        clouds, start, vs = _batch()
        c0, c1 = R.shard_clouds(start, rank, world)
        # voxelize this rank's clouds (the oracle stands in for the GPU here)
        pairs = voxels = 0
        for c in range(c0, c1):
            ref = O.OracleResult(clouds[c], float(vs[c]), 0.05, window_mode=0, nthreads=1)
            pairs += ref.counts["P"]
            voxels += ref.counts["V"]
            ref.close()
        shards = [None] * world
        dist.all_gather_object(shards, (c0, c1, pairs, voxels))
        slowest = R.max_over_ranks(10.0 + rank, dist)
        total_gaussians = R.sum_over_ranks(float(start[c1] - start[c0]), dist)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"),
                np.array([c0, c1, pairs, voxels, slowest, total_gaussians], dtype=np.float64))
        np.save(os.path.join(out_dir, f"shards{rank}.npy"), np.array(shards, dtype=np.float64))
    finally:
        dist.destroy_process_group()


def test_shard_clouds_partitions_and_balances():
    from nanovdb_editor import replicas as R

    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 8):
        sizes = rng.integers(1, 1000, size=37)
        start = np.concatenate([[0], np.cumsum(sizes)])
        shards = [R.shard_clouds(start, r, world) for r in range(world)]
        assert shards[0][0] == 0 and shards[-1][1] == len(sizes)
        for (a0, a1), (b0, b1) in zip(shards, shards[1:]):
            assert a1 == b0 and a0 <= a1
        loads = [int(start[b] - start[a]) for a, b in shards]
        assert max(loads) - min(loads) <= 2 * int(sizes.max())
    # fewer clouds than ranks: some ranks get none, all clouds still covered once
    start = np.array([0, 5, 9])
    shards = [R.shard_clouds(start, r, 4) for r in range(4)]
    assert sum(b - a for a, b in shards) == 2
    with pytest.raises(ValueError):
        R.shard_clouds(start, 4, 4)
    assert R.job_rate(2_000_000, 100.0) == pytest.approx(2e7)


def test_two_rank_replicas_gloo(tmp_path):
    world = 2
    port = _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    rows = [np.load(tmp_path / f"rank{r}.npy") for r in range(world)]
    clouds, start, vs = _batch()
    # the shards cover every cloud exactly once, in order
    assert rows[0][0] == 0 and rows[-1][1] == len(clouds) and rows[0][1] == rows[1][0]
    # every rank saw the same shard table and the slowest rank's time
    for r in range(world):
        shards = np.load(tmp_path / f"shards{r}.npy")
        np.testing.assert_array_equal(shards[:, :2], np.array([row[:2] for row in rows]))
        assert rows[r][4] == 10.0 + (world - 1)
        assert rows[r][5] == float(start[-1])
    # the replicas' results add up to one process voxelizing every cloud
    import oracle as O

    pairs = voxels = 0
    for c in range(len(clouds)):
        ref = O.OracleResult(clouds[c], float(vs[c]), 0.05, window_mode=0, nthreads=1)
        pairs += ref.counts["P"]
        voxels += ref.counts["V"]
        ref.close()
    assert sum(int(row[2]) for row in rows) == pairs
    assert sum(int(row[3]) for row in rows) == voxels
