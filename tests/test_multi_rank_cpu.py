"""The multi-GPU path's host logic on CPU: two gloo ranks.

bench.py gives every rank whole clouds (longest first onto the least-loaded
rank), with no collective in the data path, and reduces the timing as the
maximum over ranks.  Here two processes shard a small batch the same way,
each answers its clouds with the oracle (the CPU restatement of the path),
and rank 0 checks that the gathered rows equal the single-process answer for
the whole batch, that the shards are disjoint and cover every cloud, and that
the MAX reduction returns the slowest rank's time.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _batch():
    from flashknn_exprepo_b200 import synthetic as S
    rng = np.random.default_rng(3)
    counts = np.array([900, 2500, 400, 1700, 1200, 3000, 600])
    clouds = [rng.random((c, 3), dtype=np.float32) * np.float32(2) for c in counts]
    return S.Batch(np.concatenate(clouds), np.cumsum(counts), counts, ["uniform"] * 7, 0.05)


def _rank(rank, world, port, out_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        from oracle import oracle as O
        b = _batch()
        owner = bench.shard_clouds(b.counts, world)
        mine = [c for c in range(len(b.counts)) if owner[c] == rank]
        xyz, off = bench.take_clouds(b, mine)
        idx, d = O.knn_offsets(xyz, off, 8, 0.05, 2)
        # local -> global indices: each cloud's rows keep their cloud-local order
        starts = np.concatenate([[0], b.offsets[:-1]])
        local_starts = np.concatenate([[0], off[:-1]])
        rows = {}
        for j, c in enumerate(mine):
            s, e = local_starts[j], off[j]
            shift = starts[c] - s
            rows[c] = (np.where(idx[s:e] >= 0, idx[s:e] + shift, -1), d[s:e])
        gathered = [None] * world
        dist.all_gather_object(gathered, (rank, mine, rows))
        t = torch.tensor([10.0 * (rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            np.save(out_path, np.array([t.item()]))
            all_rows = {}
            seen = []
            for _, m, r in gathered:
                seen += m
                all_rows.update(r)
            assert sorted(seen) == list(range(len(b.counts)))
            gi = np.concatenate([all_rows[c][0] for c in range(len(b.counts))])
            gd = np.concatenate([all_rows[c][1] for c in range(len(b.counts))])
            oi, od = O.knn_offsets(b.xyz, b.offsets, 8, 0.05, 2)
            assert np.array_equal(gi, oi)
            assert np.array_equal(gd.view(np.uint32), od.view(np.uint32))
            np.save(out_path + ".ok.npy", np.array([1]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_whole_clouds(tmp_path):
    out = str(tmp_path / "max.npy")
    mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, join=True,
                       start_method="spawn")
    assert np.load(out)[0] == 20.0                 # MAX over ranks
    assert os.path.exists(out + ".ok.npy")


def test_shard_balance():
    import bench
    counts = np.array([200, 20, 150, 90, 60, 180, 30, 110])
    for world in (1, 2, 3, 4):
        owner = bench.shard_clouds(counts, world)
        load = np.bincount(owner, weights=counts, minlength=world)
        assert load.max() - load.min() <= counts.max()
        assert set(owner) <= set(range(world))
    with pytest.raises(Exception):
        bench.shard_clouds(counts, 0)
