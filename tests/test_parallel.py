"""Data parallelism over binaries (``waveformx_b200.parallel``) on CPU: the
shard ranges partition a batch, ragged shards balance the frequencies, and
two ``gloo`` ranks that each evaluate their shard (the oracle stands in for
the kernels, which need a GPU) gather the same per-binary results as one
process evaluating the whole batch."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from waveformx_b200.parallel import gather_rows, rank_and_world, shard, shard_ragged


@pytest.mark.parametrize("batch", [0, 1, 5, 4096, 4099])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shards_partition_the_batch(batch, world):
    parts = [shard(batch, r, world) for r in range(world)]
    assert parts[0].start == 0 and parts[-1].stop == batch
    assert all(a.stop == b.start for a, b in zip(parts, parts[1:]))
    sizes = [p.stop - p.start for p in parts]
    assert max(sizes) - min(sizes) <= 1


def test_shard_errors():
    with pytest.raises(ValueError):
        shard(10, 2, 2)
    with pytest.raises(ValueError):
        shard_ragged([0, 5, 3], 0, 2)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_ragged_shards_balance_frequencies(world):
    lengths = np.random.default_rng(3).integers(1000, 130000, 16384)
    offsets = np.concatenate([[0], np.cumsum(lengths)])
    parts = [shard_ragged(offsets, r, world) for r in range(world)]
    assert parts[0].start == 0 and parts[-1].stop == len(lengths)
    assert all(a.stop == b.start for a, b in zip(parts, parts[1:]))
    work = [int(offsets[p.stop] - offsets[p.start]) for p in parts]
    assert sum(work) == offsets[-1]
    assert max(work) - min(work) <= 2 * lengths.max()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, params, grid, data, weights, out_dir):
    import torch
    import torch.distributed as dist

    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        assert rank_and_world() == (rank, world)
        mine = shard(len(params), rank, world)
        loss = oracle.batch_loss("IMRPhenomXAS", params[mine], grid, data, weights)
        gathered = gather_rows(torch.as_tensor(loss), len(params))
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), gathered.numpy())
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_the_whole_batch(tmp_path):
    import torch.multiprocessing as mp

    import oracle

    rng = np.random.default_rng(8)
    m = rng.uniform(5.0, 100.0, (7, 2))
    params = np.stack([m.max(1), m.min(1), rng.uniform(-0.9, 0.9, 7), rng.uniform(-0.9, 0.9, 7),
                       rng.uniform(100, 5000, 7), rng.uniform(0, 3, 7), rng.uniform(0, 6, 7), np.full(7, 20.0)], 1)
    grid = np.linspace(20.0, 512.0, 257)
    data = (rng.normal(size=257) + 1j * rng.normal(size=257)) * 1e-2
    weights = 1.0 / oracle.psd(grid)
    mp.start_processes(_rank_main, args=(2, _free_port(), params, grid, data, weights, str(tmp_path)), nprocs=2,
                       join=True, start_method="spawn")
    whole = oracle.batch_loss("IMRPhenomXAS", params, grid, data, weights)
    for rank in range(2):
        np.testing.assert_allclose(np.load(tmp_path / f"rank{rank}.npy"), whole, rtol=1e-13, atol=0)
