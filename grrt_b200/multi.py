"""One frame across several GPUs (one process per GPU, torch.distributed).

Every ray is independent, so a frame splits by rows with no exchange until
the end. Rank k renders the image rows k, k + N, k + 2N, ... (N ranks):
interleaved rows spread the costly ones (the disk, the shadow's edge) evenly,
where contiguous blocks would hand the middle ranks most of the work. Each
rank renders its rows in one launch (`Renderer.render_rows_device`), then one
all-gather brings every rank's rows together and they are put back in image
order. The collectives are the only data exchange.
"""
from __future__ import annotations


def shard_rows(height: int, world: int, rank: int) -> tuple:
    """(row0, row_step, n_rows) of rank's rows of a height-row image."""
    if not (0 <= rank < world) or height < 1:
        raise ValueError("bad shard")
    return rank, world, len(range(rank, height, world))


def assemble(parts, height: int, world: int):
    """parts[k]: rank k's rows (tensor [n_k, ...]) -> the frame [height, ...] in image order."""
    out = parts[0].new_empty((height,) + tuple(parts[0].shape[1:]))
    for k, p in enumerate(parts):
        n = len(range(k, height, world))
        if p.shape[0] < n:
            raise ValueError(f"rank {k} holds {p.shape[0]} rows, needs {n}")
        out[k::world] = p[:n]
    return out


def gather_frame(local, height: int, dist, world: int):
    """All-gather every rank's rows (local: this rank's [n_rows, ...] tensor)
    and return the whole frame on every rank. Row counts differ by at most one
    between ranks; each rank pads to the largest for the collective."""
    n_max = (height + world - 1) // world
    buf = local.new_zeros((n_max,) + tuple(local.shape[1:]))
    buf[: local.shape[0]] = local
    parts = [buf.new_empty(buf.shape) for _ in range(world)]
    dist.all_gather(parts, buf)
    return assemble(parts, height, world)


def max_over_ranks(value: float, dist, device) -> float:
    """The largest of every rank's value (e.g. a device time: a step ends when its slowest rank does)."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
