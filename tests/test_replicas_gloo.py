"""The replica mode's host logic (cerebellum_simulation_b200.replicas) on two
gloo ranks on the CPU: max-over-ranks timing, whole-job throughput and
per-rank seeds, as bench.py --gpus N uses them over NCCL."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from cerebellum_simulation_b200 import replicas
    dist, r, w, local = replicas.init("gloo", timeout_s=60)
    assert (r, w, local) == (rank, world, rank)
    # rank 1 is the slower one for the first value, rank 0 for the second
    ms = replicas.max_over_ranks(dist, [10.0 + 5.0 * rank, 20.0 - 3.0 * rank])
    out.put((rank, ms, replicas.throughput(w, 1000, ms[0]), replicas.replica_seed(7, r)))
    replicas.finish(dist)


def test_two_gloo_ranks_agree_on_max_and_throughput():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, thr, seed in res:
        assert ms == [15.0, 20.0]
        assert thr == pytest.approx(2 * 1000 / 0.015)
        assert seed == 7 + rank


def test_single_process_is_identity():
    from cerebellum_simulation_b200 import replicas
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    dist, rank, world, local = replicas.init()
    assert dist is None and (rank, world, local) == (0, 1, 0)
    assert replicas.max_over_ranks(None, [3, 4]) == [3.0, 4.0]
    assert replicas.throughput(1, 500, 250.0) == 2000.0
