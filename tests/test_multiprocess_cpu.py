"""The multi-GPU host paths on CPU ranks (gloo, world size 2).

With N GPUs, bench.py runs N independent replicas and reports the whole-job
rate over the slowest rank's time (max over ranks).  Ensemble and serving
requests are dealt to the GPUs as whole runs (no data exchange), and the
per-run records are gathered on rank 0 for the percentiles.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    import bench
    from oraclev8_b200.serving import (RunRecord, draw_requests, gather_records,
                                       shard_requests, summarize)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # slowest replica's times, element-wise
        red = bench.max_over_ranks([1.0 + rank, 10.0 - rank], "cpu")
        reqs = draw_requests(40, 3, hours=2.0)
        mine = shard_requests(reqs, rank, world)
        recs = [RunRecord(r.rid, r.n, r.nz, r.precision, r.nsteps, r.cells, 0.0, admit_s=0.0,
                          done_s=1.0 + rank) for r in mine]
        allrecs = gather_records(recs)
        out.put((rank, red, [r.rid for r in mine], sum(r.cell_updates for r in mine),
                 None if allrecs is None else summarize(allrecs)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_replica_reductions_and_request_sharding_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(out.get(timeout=100) for _ in ps)
    for p in ps:
        p.join(timeout=30)
        assert p.exitcode == 0
    (r0, red0, ids0, cu0, sum0), (r1, red1, ids1, cu1, sum1) = res
    assert red0 == red1 == [2.0, 10.0]
    assert not set(ids0) & set(ids1) and len(ids0) + len(ids1) == 40
    assert abs(cu0 - cu1) <= 0.15 * (cu0 + cu1)  # balanced by cell-updates
    assert sum1 is None and sum0["runs"] == 40
    assert sum0["makespan_s"] == 2.0  # slowest rank's completion
