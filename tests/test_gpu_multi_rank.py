"""The antenna-sharded search (multi_gpu.acquire_cells_sharded) with the real
kernels: two ranks, each a process with its own context, search their
halves of the antennas of the real TART recording and all-gather the cells
over gloo; the merged cells must equal one context's search of every
antenna, field for field.  Both ranks share the one GPU of this run; their
kernels never wait on each other (the only exchange is the host-side
gather), so they may run on one device.  On a multi-GPU node the same path
runs one rank per GPU with nccl."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import tga
from multi_gpu import acquire_cells_sharded

pytestmark = pytest.mark.gpu

MASK = (1 << tga.GPS) | (1 << tga.GALILEO)


def _rows():
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "tart_head.npz"))
    from test_gpu_parity import _real_bits_for_gpu
    return _real_bits_for_gpu(z["head"], z["ones"], int(z["row_bytes"]))[:8], float(z["sampling_frequency"])


def _worker(rank, world, port, precision, out_q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    rows, fs = _rows()
    with tga.Context(0) as ctx:
        ctx.set_precision(precision)
        cells = acquire_cells_sharded(ctx, rows, fs, mask=MASK, cn0=True)
    out_q.put((rank, cells.tobytes()))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("precision", [tga.PRECISION_FP32, tga.PRECISION_FP16_TC], ids=["fp32", "fp16tc"])
def test_sharded_search_equals_single_context(precision):
    mpc = mp.get_context("spawn")
    q = mpc.Queue()
    port = _free_port()
    procs = [mpc.Process(target=_worker, args=(r, 2, port, precision, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    rows, fs = _rows()
    with tga.Context(0) as ctx:
        ctx.set_precision(precision)
        want = ctx.acquire_cells(rows, fs, mask=MASK, cn0=True)
    for rank, raw in res:
        got = np.frombuffer(raw, dtype=tga.CELL_DTYPE)
        assert np.array_equal(got, want), rank
