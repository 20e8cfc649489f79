"""The N > 1 path on CPU: world_size-2 gloo ranks each match their contiguous
block of segments (the oracle stands in for the GPU), gather, and merge; the
result must equal the single-process match."""
import os
import socket

import numpy as np
import pytest

from ngap_b200 import shard

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _workload():
    """Dot-star set in which three patterns start at start-of-data states, which
    only global segment 0 may use."""
    from ngap_b200 import workloads as W
    anml, data = W.dotstar_set(seed=41, n_patterns=12, input_len=7 * 1500, plant_every=400)
    return anml.replace('start="all-input"', 'start="start-of-data"', 3), data


def _worker(rank, world, port, out_dir):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from datetime import timedelta

    from ngap_b200 import shard
    from oracle import frontend, oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    anml, data = _workload()
    nodes, adj = frontend.load_anml(anml)
    groups = frontend.build_groups(nodes, adj, 3)
    num_seg, seg_len = 7, 1500
    first, count = shard.rank_segments(num_seg, rank, world)
    block = data[first * seg_len:(first + count) * seg_len]
    rep, _ = oracle.match(groups, block, count, seg_len, first_segment=first)
    rep = shard.shift_offsets(rep, first * seg_len)
    parts = [None] * world
    dist.all_gather_object(parts, rep.tolist())
    if rank == 0:
        merged = shard.merge_reports([np.array(p, dtype=np.uint64) for p in parts])
        np.save(os.path.join(out_dir, "merged.npy"), merged)
    dist.barrier()
    dist.destroy_process_group()


def test_rank_segments_cover_stream():
    from ngap_b200 import shard
    for n in (1, 7, 16):
        for world in (1, 2, 3, 8):
            blocks = [shard.rank_segments(n, r, world) for r in range(world)]
            assert sum(c for _, c in blocks) == n
            pos = 0
            for f, c in blocks:
                assert f == pos
                pos += c


def test_two_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp

    from oracle import frontend, oracle
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2,
                       start_method="spawn", join=True)
    merged = np.load(tmp_path / "merged.npy")
    anml, data = _workload()
    nodes, adj = frontend.load_anml(anml)
    groups = frontend.build_groups(nodes, adj, 3)
    want, _ = oracle.match(groups, data, 7, 1500)
    assert len(want) > 0
    assert np.array_equal(merged, want)


def test_shift_offsets_keeps_ids_and_refuses_overflow():
    rep = np.array([(5 << 32) | 10, (7 << 32) | 0xFFFFFF00], dtype=np.uint64)
    got = shard.shift_offsets(rep, 0x10)
    assert got.tolist() == [(5 << 32) | 0x1A, (7 << 32) | 0xFFFFFF10]
    with pytest.raises(ValueError):
        shard.shift_offsets(rep, 0x100)  # the second offset would pass 2^32 - 1
