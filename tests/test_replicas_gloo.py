"""The multi-GPU layer's host logic (b200enc.replicas, used by bench.py) with
world_size-2 gloo process groups on the CPU: disjoint streams per rank, the
barrier, the device time of the slowest rank on every rank, the whole-job
rate, and a rank whose peer never joins failing within its timeout instead of
hanging."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

PKG = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "bc250-vaapi_b200")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, ws, port):
    os.environ.update({"WORLD_SIZE": str(ws), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, PKG)


def _rank_main(rank, ws, port, q):
    _env(rank, ws, port)
    import torch.distributed as dist
    from b200enc import replicas
    g = replicas.Group("gloo", device="cpu", timeout_s=60)
    seeds = replicas.stream_seeds(g.rank, 8)
    synced = []
    g.barrier(lambda: synced.append(True))
    ms = 10.0 * (g.rank + 1)  # the ranks' device times differ
    mx = g.max(ms)
    every = [None] * ws
    dist.all_gather_object(every, seeds)
    rate = replicas.aggregate_rate(g.world_size, 8 * 5, mx)
    g.close()
    q.put((g.rank, mx, every, rate, bool(synced)))


def _lonely_rank(port, q):
    _env(1, 2, port)
    from b200enc import replicas
    try:
        replicas.Group("gloo", device="cpu", timeout_s=4)
        q.put("joined")
    except Exception as e:  # the rendezvous timed out: an error, not a hang
        q.put(type(e).__name__)


def _run(target, args_list, timeout=120):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=target, args=(*a, q)) for a in args_list]
    for p in ps:
        p.start()
    out = [q.get(timeout=timeout) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    codes = [p.exitcode for p in ps]
    for p in ps:
        if p.is_alive():
            p.kill()
    return out, codes


def test_two_gloo_ranks_barrier_max_and_rate():
    port = _free_port()
    out, codes = _run(_rank_main, [(r, 2, port) for r in range(2)])
    assert codes == [0, 0]
    assert sorted(o[0] for o in out) == [0, 1]
    for rank, mx, every, rate, synced in out:
        assert mx == 20.0  # every rank holds the slowest rank's time
        assert synced
        assert set(every[0]).isdisjoint(every[1]) and len(every[0]) == len(every[1]) == 8
        assert rate == pytest.approx(2 * 40 / 0.020)


def test_rank_without_peer_fails_within_timeout():
    out, codes = _run(_lonely_rank, [(_free_port(),)], timeout=90)
    assert out[0] != "joined"
    assert codes == [0]


def test_single_process_needs_no_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, PKG)
    from b200enc import replicas
    g = replicas.Group("nccl", device="cuda")  # one process: no group, no GPU touched
    calls = []
    g.barrier(lambda: calls.append(1))
    assert g.dist is None and calls == [1] and g.max(3.5) == 3.5
    assert replicas.stream_seeds(0, 3) == [0, 1, 2] and replicas.stream_seeds(2, 2) == [2000, 2001]
    with pytest.raises(ValueError):
        replicas.stream_seeds(0, 1001)
    with pytest.raises(ValueError):
        replicas.aggregate_rate(1, 10, 0.0)
    g.close()
