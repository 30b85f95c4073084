"""Ensemble pass across several GPUs (one process per GPU).

Pairs are sharded across ranks; each rank accumulates its own pairs into its own
sums.  One exchange per pass combines them: the AB/AA/BB plane sums are
reduce-scattered by window block (rank r owns windows [start_r, stop_r)), the
frame sums and the pair count are all-reduced (every rank needs the full mean
images for the background correlation of its windows).  Each rank then
finalises and fits only its window block, and the per-window fit results are
all-gathered.  Kahan-compensated FP32 sums cross the wire as FP64 (sum - comp),
so the exchange adds no rounding of its own.

The exchange is plain torch.distributed: NCCL over NVLink on GPUs, gloo on CPU
tensors (where a reduce-scatter is an all-reduce followed by a slice).
"""

from __future__ import annotations


def _host_side(t, group):
    """gloo runs its collectives on host tensors: stage device tensors through
    host memory there (NCCL works on device memory directly)."""
    import torch.distributed as dist

    return t.is_cuda and dist.get_backend(group) != "nccl"


def _all_reduce(t, group):
    import torch.distributed as dist

    if _host_side(t, group):
        h = t.cpu()
        dist.all_reduce(h, group=group)
        t.copy_(h)
    else:
        dist.all_reduce(t, group=group)


def window_blocks(n_win: int, world: int):
    """Contiguous window blocks, one per rank, sizes differing by at most one."""
    base, extra = divmod(n_win, world)
    out, start = [], 0
    for r in range(world):
        stop = start + base + (1 if r < extra else 0)
        out.append((start, stop))
        start = stop
    return out


def _reduce_scatter_blocks(flat, blocks, group):
    """flat: (3, n_win, hw) FP64 on every rank -> this rank's summed block."""
    import torch
    import torch.distributed as dist

    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    blk = max(b - a for a, b in blocks)
    hw = flat.shape[2]
    padded = flat.new_zeros((world, 3, blk, hw))
    for r, (a, b) in enumerate(blocks):
        padded[r, :, : b - a] = flat[:, a:b]
    if dist.get_backend(group) == "nccl":
        out = flat.new_empty((3, blk, hw))
        dist.reduce_scatter_tensor(out, padded.reshape(-1), group=group)
    else:
        _all_reduce(padded, group)
        out = padded[rank]
    a, b = blocks[rank]
    return out[:, : b - a].contiguous()


def exchange_sums(sums, comps, fsum, fcomp, n_pairs, n_win, hw, group=None):
    """Combine the ranks' accumulators.

    sums, comps: (3, n_win * hw) float32 Kahan sums and compensations;
    fsum, fcomp: (2, H * W) float32 frame sums and compensations.
    Returns (block_sums (3, n_block, hw) float32, frame_sums (2, H * W) float32,
    total pair count, (start, stop) of this rank's windows)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    blocks = window_blocks(n_win, world)
    flat = (sums.double() - comps.double()).reshape(3, n_win, hw)
    block = _reduce_scatter_blocks(flat, blocks, group).float()
    fr = fsum.double() - fcomp.double()
    _all_reduce(fr, group)
    n = torch.tensor([float(n_pairs)], dtype=torch.float64, device=sums.device)
    _all_reduce(n, group)
    return block, fr.float(), int(round(n.item())), blocks[rank]


def all_reduce_frame_sums(fsum, fcomp, n_pairs, group=None):
    """Frame sums (2, H * W) float32 with their Kahan compensations and the pair
    count, summed over the ranks (the first sweep of the 'image' background
    methods).  Returns (frame sums float32, total pair count)."""
    import torch

    fr = fsum.double() - fcomp.double()
    _all_reduce(fr, group)
    n = torch.tensor([float(n_pairs)], dtype=torch.float64, device=fsum.device)
    _all_reduce(n, group)
    return fr.float(), int(round(n.item()))


def gather_rows(local, n_win, group=None):
    """All-gather per-window rows (n_block, ...) of every rank into (n_win, ...)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    blocks = window_blocks(n_win, world)
    blk = max(b - a for a, b in blocks)
    pad = local.new_zeros((blk,) + tuple(local.shape[1:]))
    pad[: local.shape[0]] = local
    host = _host_side(pad, group)
    src = pad.cpu() if host else pad
    parts = [torch.empty_like(src) for _ in range(world)]
    dist.all_gather(parts, src, group=group)
    out = torch.cat([p[: b - a] for p, (a, b) in zip(parts, blocks)], dim=0)
    return out.to(local.device) if host else out
