"""Multi-rank host logic of bench.py on CPU: two gloo ranks take the same
barrier / max-over-ranks steps the GPU run takes over NCCL, and the reference
arm runs on rank 0 only (other ranks exit 0 without work or output)."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    from datetime import timedelta

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        barrier, max_over_ranks = bench.rank_ops(dist, torch.device("cpu"))
        barrier()
        m = max_over_ranks(10.0 * (rank + 1) + 0.25)
        barrier()
        buf = io.StringIO()
        rc = None
        if rank != 0:
            args = type("A", (), dict(gpus=world, steps=1, warmup=0, config="small", impl="reference"))()
            with redirect_stdout(buf):
                rc = bench.run_reference(args)
        out.put((rank, m, rc, buf.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_rank_barrier_and_max():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 2
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert [r[1] for r in res] == [20.25, 20.25]
    # rank 1 of the reference arm: exit status 0, no JSON line, no work
    assert res[1][2] == 0 and res[1][3] == ""


def test_single_rank_ops_are_identity():
    sys.path.insert(0, ROOT)
    import bench
    barrier, mx = bench.rank_ops(None, None)
    barrier()
    assert mx(3.5) == 3.5


@pytest.mark.parametrize("rng", ["replay", "native"])
def test_reference_arm_line(rng, monkeypatch):
    """Rank 0 of the reference arm prints one JSON line with the contract's keys:
    the reference's host run of the small workload (one complete run), its
    cpu_baseline (kind "reference", the threads used: one with the reference's
    own generator) and an e2e block with no host-device copies."""
    import json
    sys.path.insert(0, ROOT)
    import bench
    from oracle import oracle as O
    if not O.ref_available(native_rng=rng == "native"):
        pytest.skip("oracle/_ref not built")
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    args = type("A", (), dict(gpus=1, steps=1, warmup=0, config="small", impl="reference", subset=0,
                              ref_rng=rng))()
    buf = io.StringIO()
    with redirect_stdout(buf):
        assert bench.run_reference(args) == 0
    line = json.loads(buf.getvalue().strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "samples/s" and line["value"] > 0
    assert line["config"]["rng"] == rng and line["config"]["targets_timed"] == 1
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == line["value"]
    if rng == "native":
        assert cb["cores"] == 1
    assert line["e2e"] == {"value": line["value"], "unit": "samples/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert 0.5 < line["dosage_r2"] <= 1.0
