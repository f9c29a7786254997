"""The multi-GPU replica path on CPU: two gloo ranks (127.0.0.1) run the same
bookkeeping the benchmark runs over NCCL -- barriers, the max over ranks of
the per-rank timings, the whole-job rate, and the round-robin share of a
batch of instances."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from geowarp_b200.replicas import Replicas, aggregate_rate
    rep = Replicas("gloo", timeout_s=60)
    try:
        rep.barrier()
        # rank r "took" 10 + r ms for its steps and 5 * (r + 1) for another leg
        ms = rep.max_over_ranks([10.0 + rank, 5.0 * (rank + 1)])
        items = rep.share(list(range(7)))
        rate = aggregate_rate([4] * world, ms[0])
        q.put((rank, ms, items, rate))
    finally:
        rep.close()


def test_two_gloo_replicas():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(world))
    for rank, ms, items, rate in out:
        assert ms == [11.0, 10.0]                       # max over ranks, on every rank
        assert items == list(range(7))[rank::world]     # round-robin share
        assert abs(rate - 8 / 0.011) < 1e-9             # all ranks' units over the slowest time
    assert sorted(i for _, _, items, _ in out for i in items) == list(range(7))
