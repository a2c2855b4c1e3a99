"""Multi-rank host logic on the CPU: two gloo ranks (world size 2), as
bench.py --gpus 2 runs them over NCCL: the barrier, the max over ranks of the
elapsed time, disjoint trajectory blocks per rank and the weak-scaling
aggregate.  No GPU is needed."""
import os
import socket

import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from molspin_b200 import ranks
    from molspin_b200 import systems as S
    w, r, _ = ranks.init("gloo", timeout_s=60)
    ranks.barrier(w)
    elapsed = ranks.max_over_ranks(10.0 + 5.0 * r, w)  # the slower rank sets the time
    seed = ranks.block_seed(1.0, r)
    block = S.plain_small().system.trace_samples(8, seed)
    q.put((r, w, elapsed, seed, block[:, 0].copy(), ranks.aggregate(100.0, w, elapsed)))
    ranks.barrier(w)
    ranks.finish(w)


def test_two_gloo_ranks_weak_scaling():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        r, w, elapsed, seed, col, agg = q.get(timeout=180)
        out[r] = (w, elapsed, seed, col, agg)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == 2
    assert out[0][1] == out[1][1] == 15.0          # max over ranks
    assert out[0][2] != out[1][2]                  # distinct block seeds
    assert abs(out[0][3] - out[1][3]).max() > 1e-3  # disjoint trajectory samples
    assert out[0][4] == out[1][4] == 2 * 100.0 / 15.0
