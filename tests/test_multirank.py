"""Several ranks on one frame (grrt_b200.multi), run as world_size-2 gloo
process groups on the CPU: the row shards cover the image exactly once, the
all-gather puts every rank's rows back in image order (also for a row count
that does not divide by the ranks), and the max over ranks is the largest
rank's value. The GPU side (NCCL, one process per GPU) runs the same calls."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

from grrt_b200 import multi


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, height: int, width: int) -> None:
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        row0, step, n = multi.shard_rows(height, world, rank)
        rows = torch.arange(row0, height, step, dtype=torch.float32)
        assert len(rows) == n
        # this rank's "render": each pixel holds its image row and column
        local = torch.stack([rows[:, None].expand(n, width), torch.arange(width, dtype=torch.float32)[None, :].expand(n, width)],
                            dim=-1)
        frame = multi.gather_frame(local.contiguous(), height, dist, world)
        assert frame.shape == (height, width, 2)
        want_rows = torch.arange(height, dtype=torch.float32)[:, None].expand(height, width)
        assert torch.equal(frame[..., 0], want_rows)
        assert torch.equal(frame[..., 1], torch.arange(width, dtype=torch.float32)[None, :].expand(height, width))
        assert multi.max_over_ranks(1.5 + rank, dist, "cpu") == 1.5 + world - 1
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("height", [16, 37])
def test_two_ranks_gather_one_frame(height):
    mp.start_processes(_rank_main, args=(2, _free_port(), height, 5), nprocs=2, join=True, start_method="spawn")


def test_shards_cover_rows_once():
    for world in (1, 2, 3, 8):
        for height in (1, 7, 16, 1024):
            if world > height:
                continue
            seen = []
            for rank in range(world):
                row0, step, n = multi.shard_rows(height, world, rank)
                seen += [row0 + k * step for k in range(n)]
            assert sorted(seen) == list(range(height))
    with pytest.raises(ValueError):
        multi.shard_rows(16, 2, 2)
