"""World-size-2 gloo test of the multi-GPU host path (no GPU needed).

Each rank runs the sharded search with a stand-in context that produces
deterministic cells from (constellation, PRN, antenna) exactly as
tga_acquire_all orders them; the gathered, merged result must equal a
single-rank search over all antennas.  The real kernels are exercised by
the single-GPU parity tests; this covers sharding, gathering and ordering.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import tga
from multi_gpu import acquire_cells_sharded, merge_cells, shard_antennas


class FakeCtx:
    """Stand-in for tga.Context.acquire_cells (same output layout)."""

    cell_dtype = tga.CELL_DTYPE

    def acquire_cells(self, packed_bits, fs, mask=tga.ALL, ant_filter=None, prn_filter=None, **kw):
        n_ant = np.asarray(packed_bits).shape[0]
        ants = list(range(n_ant)) if ant_filter is None else list(ant_filter)
        rows = []
        for c in range(6):
            if not (mask >> c) & 1:
                continue
            lo, hi = {0: (1, 38), 1: (1, 50), 2: (1, 63), 3: (120, 158), 4: (1, 63), 5: (184, 206)}[c]
            for prn in (prn_filter if prn_filter is not None else range(lo, hi + 1)):
                for a in ants:
                    row = np.zeros(1, dtype=tga.CELL_DTYPE)
                    row["constellation"], row["prn"], row["antenna"] = c, prn, a
                    row["signal_strength"] = 1000.0 * c + prn + a / 100.0
                    row["best_codephase"] = (prn * 31 + a * 7) % 16368
                    rows.append(row)
        return np.concatenate(rows) if rows else np.zeros(0, dtype=tga.CELL_DTYPE)


def test_shard_antennas_balanced_cover():
    for n in (1, 5, 24, 25):
        for w in (1, 2, 3, 8):
            parts = [shard_antennas(range(n), w, r) for r in range(w)]
            assert sum(parts, []) == list(range(n))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1


def _worker(rank, world, port, out_q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    bits = np.zeros((24, 16), np.uint8)
    cells = acquire_cells_sharded(FakeCtx(), bits, 16.368e6, mask=(1 << tga.GPS) | (1 << tga.SBAS),
                                  prn_filter=None)
    out_q.put((rank, cells.tobytes(), len(cells)))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_gather_matches_single_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    bits = np.zeros((24, 16), np.uint8)
    single = FakeCtx().acquire_cells(bits, 16.368e6, mask=(1 << tga.GPS) | (1 << tga.SBAS))
    for rank, raw, n in res:
        got = np.frombuffer(raw, dtype=tga.CELL_DTYPE)
        assert n == len(single)
        assert np.array_equal(got, single), rank


def test_merge_cells_orders_like_single_rank():
    fake = FakeCtx()
    bits = np.zeros((5, 4), np.uint8)
    full = fake.acquire_cells(bits, 1.0, mask=1 << tga.QZSS, prn_filter=[190, 185])
    parts = [fake.acquire_cells(bits, 1.0, mask=1 << tga.QZSS, prn_filter=[190, 185], ant_filter=s)
             for s in ([3, 4], [0, 1, 2])]
    assert np.array_equal(merge_cells(parts, list(range(5))), full)
