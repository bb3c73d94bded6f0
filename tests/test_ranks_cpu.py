"""The multi-rank path of bench.py on the CPU: two gloo ranks (world size 2) -- the job time is
the slowest rank's (max over ranks), every rank searches its own pair (replicas, weak scaling),
and a rank that leaves before the reduction makes its peer's collective end with an error
within the process group's timeout instead of hanging."""
import datetime
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


def _worker(rank, world, port, fail_rank, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        if rank == fail_rank:
            raise SystemExit(3)  # leaves before the collective, as a crashed rank would
        t = bench.max_over_ranks(10.0 * (rank + 1), world, "cpu")
        out[rank] = (t, bench.rank_seed(rank, 100))
    except RuntimeError as e:  # the peer's collective gives up
        out[rank] = ("error", str(e)[:80])
    finally:
        if rank != fail_rank:
            dist.destroy_process_group()


def _run(fail_rank):
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        ps = [ctx.Process(target=_worker, args=(r, 2, port, fail_rank, out)) for r in range(2)]
        for p in ps:
            p.start()
        for p in ps:
            p.join(timeout=60)
        for p in ps:
            if p.is_alive():
                p.kill()
                pytest.fail("a rank did not finish")
        return dict(out), [p.exitcode for p in ps]


def test_max_over_ranks_and_seeds():
    out, codes = _run(fail_rank=-1)
    assert codes == [0, 0]
    assert out[0][0] == out[1][0] == 20.0
    assert out[0][1] != out[1][1]


def test_single_rank_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(7.5, 1, "cpu") == 7.5


def test_lost_rank_ends_the_peer_with_an_error():
    out, codes = _run(fail_rank=1)
    assert codes[1] == 3
    assert 0 in out and out[0][0] == "error"
