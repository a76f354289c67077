"""Multi-rank host logic on CPU (gloo, world size 2): the benchmark's
combination of per-rank timings (max time, summed units), disjoint per-rank
seeds, and the rule that every rank takes the same collective steps.  The
GPU path runs the same code over NCCL, one process per GPU."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "protein-structure-analysis_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from protein_physics_b200.dist import init, rank_info, rank_seed, reduce_timing
    init("gloo", timeout_s=60)
    r, w, lr = rank_info()
    ms, units = reduce_timing(10.0 + 5.0 * r, 100 * (r + 1))
    # a second round: collectives stay in step across ranks
    ms2, units2 = reduce_timing(1.0 if r == 0 else 3.0, 7)
    q.put((r, w, lr, ms, units, ms2, units2, rank_seed(3, r)))
    dist.barrier()
    dist.destroy_process_group()


def test_reduce_timing_world2():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for r, (rank, world, local, ms, units, ms2, units2, seed) in enumerate(res):
        assert (rank, world, local) == (r, 2, r)
        assert ms == 15.0 and units == 300.0  # max of 10/15 ms, 100 + 200 units
        assert ms2 == 3.0 and units2 == 14.0
    assert res[0][-1] != res[1][-1]  # disjoint seeds per rank


def test_single_process_is_identity():
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "protein-structure-analysis_b200"))
    from protein_physics_b200.dist import reduce_timing
    assert reduce_timing(12.5, 40) == (12.5, 40.0)
