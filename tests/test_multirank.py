"""The multi-rank host logic on CPU: two processes with the gloo backend stand in for two GPUs.

Every (pixel, sample) is independent, so ranks render their own rows or sample ranges with no
data-path collective (repackshot_b200/shards.py). Checked here:
- the sample ranges and row bands of all ranks tile the frame exactly;
- a frame rendered as row bands, one per rank, and gathered equals the one-process film bit for
  bit (each pixel's samples stay on one rank, added in index order); the renderer here is the
  oracle, the CPU restatement of the reference, because no GPU is present;
- the job's time is the maximum over ranks.
"""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
WORLD = 2
W, H, SPP = 48, 40, 2


def small_scene_rsb():
    from repackshot_b200 import scenes
    s = scenes.cfg0_scene()
    s.width, s.height = W, H
    return scenes.to_rsb(s)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, port, out_dir):
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch.distributed as dist

    import oracle
    from repackshot_b200 import shards

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        # Ranges and bands of every rank, gathered.
        ranges, bands = [None] * WORLD, [None] * WORLD
        dist.all_gather_object(ranges, shards.sample_range(rank, WORLD, SPP))
        dist.all_gather_object(bands, shards.row_band(rank, WORLD, H))
        # This rank's band of the frame at every sample.
        first_row, rows = shards.row_band(rank, WORLD, H)
        o = oracle.OracleScene(small_scene_rsb())
        rgb, wt, al, l2, _ = o.render_film(0, SPP, 0, first_row, W, rows)
        parts = [None] * WORLD
        dist.all_gather_object(parts, (first_row, rgb, wt, al, l2))
        slowest = shards.max_over_ranks(1.5 + rank, dist)
        if rank == 0:
            np.save(Path(out_dir) / "result.npy", np.array([ranges, bands, parts, slowest], dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def gathered(tmp_path_factory, oracle_lib):
    import torch.multiprocessing as mp
    out = tmp_path_factory.mktemp("ranks")
    mp.start_processes(worker, args=(free_port(), str(out)), nprocs=WORLD, join=True, start_method="spawn")
    return np.load(out / "result.npy", allow_pickle=True)


def test_sample_ranges_and_bands_tile_the_frame(gathered):
    ranges, bands = gathered[0], gathered[1]
    assert [r[0] for r in ranges] == [k * SPP for k in range(WORLD)] and all(r[1] == SPP for r in ranges)
    rows = [r for first, n in bands for r in range(first, first + n)]
    assert rows == list(range(H))


def test_gathered_bands_equal_the_one_process_film(gathered, oracle_lib):
    parts = gathered[2]
    rgb, wt, al, l2, _ = oracle_lib.OracleScene(small_scene_rsb()).render_film(0, SPP)
    got = [np.zeros_like(a) for a in (rgb, wt, al, l2)]
    for first, *arrays in parts:
        for g, a in zip(got, arrays):
            g[first:first + a.shape[0]] = a
    for g, a in zip(got, (rgb, wt, al, l2)):
        assert np.array_equal(g.view(np.uint32), a.view(np.uint32))
    assert float(wt.sum()) == W * H * SPP


def test_time_is_the_slowest_rank(gathered):
    assert gathered[3] == 1.5 + (WORLD - 1)


def test_shard_arguments_are_checked():
    sys.path.insert(0, str(ROOT))
    from repackshot_b200 import shards
    with pytest.raises(ValueError):
        shards.sample_range(2, 2, 8)
    with pytest.raises(ValueError):
        shards.row_band(0, 2, -1)
    assert shards.row_band(2, 3, 2) == (2, 0)
    assert shards.max_over_ranks(3.0) == 3.0
