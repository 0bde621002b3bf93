"""The multi-rank plumbing of bench.py on CPU: two gloo ranks agree on the
slowest rank's time, the whole-job value counts every rank's rays, and the
reference arm does its work on rank 0 only."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(1.0 + rank, ws, device="cpu")  # rank r took 1 + r ms
        v = bench.whole_job_mrays(2_000_000, ws, t)
        dist.barrier()

        class A:
            steps, warmup = 1, 3
        skipped = bench.run_reference_arm(A()) == 0 if rank > 0 else None
        out.put((rank, t, v, skipped))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t, v, skipped in res:
        assert t == 2.0                      # the slowest rank's time, on every rank
        assert v == pytest.approx(2 * 2_000_000 / 2.0 / 1e3)
    assert res[1][3] is True                 # rank 1 leaves the reference arm without work
