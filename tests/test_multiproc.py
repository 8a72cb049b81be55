"""Host logic of the multi-GPU bench path with world_size 2 on CPU (gloo):
the max-over-ranks reduction of the timings and the rank-0-only reference
arm.  The GPU replicas themselves run one per GPU under torchrun."""

import contextlib
import io
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        vals = [1.0 + 3 * rank, 5.0 - 3 * rank, 3.0 + 3 * rank]   # r0 [1,5,3], r1 [4,2,6]
        got = bench.max_over_ranks(vals, ws)
        # the reference arm prints on rank 0 only; rank 1 returns at once
        buf = io.StringIO()
        if rank == 1:
            with contextlib.redirect_stdout(buf):
                bench.run_reference(type("A", (), dict(workload="lossy_256", dtype="float64",
                                                        steps=1, warmup=3, gpus=ws))())
        out.put((rank, got, buf.getvalue()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_max_and_rank0_reference():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict()
    for _ in range(2):
        r, got, printed = q.get(timeout=120)
        res[r] = (got, printed)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][0] == [4.0, 5.0, 6.0]
    assert res[1][0] == [4.0, 5.0, 6.0]
    assert res[1][1] == ""


def test_single_rank_max_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([1.5, 2.0], 1) == [1.5, 2.0]


def test_traffic_scales_with_the_cells_of_the_launch():
    """roofline.traffic: the ncu bytes per cell of the committed summary
    times the cells of the launch; None for a case it does not hold."""
    import json
    sys.path.insert(0, ROOT)
    import bench
    with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
        e = json.load(f)["lossy_256:float64:tma"]
    per_cell = (e["read_bytes_small"] + e["write_bytes_small"]) / e["cells_small"]
    assert 80.0 < per_cell < 96.5
    assert bench._traffic("lossy_256", "float64", "tma", e["cells_small"]) == \
        e["read_bytes_small"] + e["write_bytes_small"]
    assert bench._traffic("lossy_256", "float64", "tma", 256 * 256 * 512) == \
        int(round(per_cell * 256 * 256 * 512))
    assert bench._traffic("lossy_256", "float64", "no-such-schedule", 10) is None
