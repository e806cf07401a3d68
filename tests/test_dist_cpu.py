"""Multi-process plumbing of the N-GPU path on CPU (gloo, world size 2): instance shards,
the max-over-ranks timing reduction, and a rank that fails before the collective (the
survivor gets an error from the short process-group timeout instead of hanging)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, mode, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from dpcrypto_b200 import dist as D
    from oracle import oracle as O

    dist = D.init("gloo", timeout_s=5.0)
    try:
        first, n = D.shard(8, rank)
        coins = O.coins(n, 24, "enc", first=first)
        if mode == "fail" and rank == 1:
            raise SystemExit(3)  # leaves before the collective
        ms = D.max_over_ranks(10.0 * (rank + 1))
        q.put((rank, first, n, coins[0].tobytes(), ms, None))
    except Exception as e:  # noqa: BLE001 - report the collective error to the parent
        q.put((rank, None, None, None, None, type(e).__name__))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=60)
    for p in procs:
        if p.is_alive():
            p.kill()
    out = {}
    while not q.empty():
        r = q.get()
        out[r[0]] = r
    return out, [p.exitcode for p in procs]


def test_shards_and_max_over_ranks():
    from oracle import oracle as O

    out, codes = _run("ok")
    assert codes == [0, 0]
    assert out[0][1:3] == (0, 8) and out[1][1:3] == (8, 8)
    assert out[0][3] == O.coins(1, 24, "enc", first=0)[0].tobytes()
    assert out[1][3] == O.coins(1, 24, "enc", first=8)[0].tobytes()
    assert out[0][4] == out[1][4] == 20.0


def test_failed_rank_surfaces_as_error():
    out, codes = _run("fail")
    assert codes[1] == 3
    assert 0 in out and out[0][5] is not None  # rank 0's collective ended with an error
