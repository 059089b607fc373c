"""Multi-GPU all-PRN search: antennas sharded across ranks.

Every (antenna, PRN, Doppler bin) row of the search is independent, so a
multi-GPU search needs no collective on the data path: rank r searches the
antennas of its shard on its own GPU (one process per GPU, launched by
torchrun), and the per-cell results (64 bytes per antenna and PRN) are
gathered afterwards.  The merged cells are in the single-GPU order
(constellation, PRN, antenna), so the JSON output is identical.
"""
import numpy as np


def shard_antennas(antennas, world, rank):
    """Contiguous, balanced split of the antenna list; shard r of `world`."""
    antennas = list(antennas)
    n = len(antennas)
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return antennas[start:start + base + (1 if rank < extra else 0)]


def merge_cells(parts, antennas):
    """Merge per-rank cell record arrays into (constellation, PRN order,
    antenna order) -- the order tga_acquire_all returns for all antennas."""
    allc = np.concatenate([p for p in parts if len(p)]) if parts else np.zeros(0)
    if len(allc) == 0:
        return allc
    ant_pos = {a: i for i, a in enumerate(antennas)}
    # PRN order inside a constellation is the order of first appearance
    prn_pos = {}
    for c, prn in zip(allc["constellation"], allc["prn"]):
        prn_pos.setdefault((int(c), int(prn)), len(prn_pos))
    key = np.array([(int(c), prn_pos[(int(c), int(p))], ant_pos[int(a)])
                    for c, p, a in zip(allc["constellation"], allc["prn"], allc["antenna"])])
    order = np.lexsort((key[:, 2], key[:, 1], key[:, 0]))
    return allc[order]


def acquire_cells_sharded(ctx, packed_bits, sampling_freq, group=None, antennas=None, **kw):
    """Search this rank's antenna shard with `ctx` (a tga.Context on the
    rank's GPU) and all-gather the cells.  torch.distributed must be
    initialised (nccl on GPUs; gloo works for the gather as well)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    n_ant = np.asarray(packed_bits).shape[0]
    antennas = list(range(n_ant)) if antennas is None else list(antennas)
    mine = shard_antennas(antennas, world, rank)
    local = ctx.acquire_cells(packed_bits, sampling_freq, ant_filter=mine, **kw) if mine else \
        np.zeros(0, dtype=getattr(ctx, "cell_dtype", None) or __import__("tga").CELL_DTYPE)
    parts = [None] * world
    dist.all_gather_object(parts, local, group=group)
    return merge_cells(parts, antennas)
