"""bench.py's replica aggregation over two gloo ranks on the CPU: the time
is the max over ranks and the work the sum (replicas only -- the path has no
data-path collective)."""
import os
import socket

import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2",
                      RANK=str(rank), LOCAL_RANK=str(rank))
    dist = bench.init_dist(2, "gloo")
    t, w = bench.reduce_max_sum(dist, float(rank + 1), 10.0 * (rank + 1))
    q.put((rank, t, w))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_max_time_sum_work():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, t, w in res:
        assert t == 2.0 and w == 30.0


def test_single_rank_passthrough():
    assert bench.reduce_max_sum(None, 3.0, 7.0) == (3.0, 7.0)


def test_l2_note_per_workload():
    """The bench says whether the SOR matrix exceeds the 126 MB L2: the
    64^3 cube (567 MB) and 32^3 20-node bricks stream from HBM, the sample
    mesh does not."""
    import bench
    from cpfem_code_b200 import generator
    assert bench.l2_note(generator.workload("cube64")).startswith("inputs larger than L2 (567 MB")
    assert bench.l2_note(generator.workload("brick20_32")).startswith("inputs larger than L2")
    assert "fits in L2" in bench.l2_note(generator.workload("brick20_10"))
