"""Multi-rank plumbing on CPU: two gloo ranks exercise the max-over-ranks
timing, the PRN sharding of the strong-scaling mode and the all-gather of
per-PRN results (no GPU, no data-path collective)."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        from pocketsdr_b200 import dist as D
        from pocketsdr_b200.synth import Group
        dist = D.init(backend="gloo", timeout_s=60)
        t = D.max_over_ranks(10.0 + rank, dist)
        groups = [Group("L1CA", list(range(1, 33)), 24e6, 0.0, 1e-3, 24000, 48000, 24000, 2,
                        np.zeros(3, np.float32)),
                  Group("E1B", list(range(1, 4)), 24e6, 0.0, 4e-3, 96000, 192000, 96000, 1,
                        np.zeros(5, np.float32))]
        mine, index = D.shard_groups(groups, rank, world)
        dt = np.dtype([("bin", np.int32), ("offset", np.int32), ("cn0", np.float32),
                       ("pmax", np.float32), ("pave", np.float64), ("fd", np.float64)])
        local = np.zeros(sum(len(g.prns) for g in mine), dt)
        k = 0
        for g in mine:     # a result that encodes the PRN, to check the placement
            for p in g.prns:
                local[k]["offset"] = p
                local[k]["bin"] = rank
                k += 1
        full = D.gather_results(local, index, groups, world, dist)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, t, [g.prns for g in mine], [a["offset"].tolist() for a in full],
               [a["bin"].tolist() for a in full]))
    except Exception as e:  # surfaced in the parent
        q.put((rank, "error", repr(e), None, None))


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        r = q.get(timeout=120)
        out[r[0]] = r
    for p in procs:
        p.join(timeout=60)
    for r in (0, 1):
        assert out[r][1] != "error", out[r][2]
        assert out[r][1] == 11.0                      # max over ranks
        assert out[r][3][0] == list(range(1, 33))     # every PRN back in order
        assert out[r][3][1] == [1, 2, 3]
        assert out[r][4][0] == [i % 2 for i in range(32)]   # dealt round-robin
    assert out[0][2][0] == list(range(1, 33, 2)) and out[1][2][0] == list(range(2, 33, 2))


def _search_worker(rank, world, port, q):
    """One rank of the strong mode with real search results: the reference
    search (the oracle's sdr_search_code + sdr_corr_max + sdr_fine_dop) over
    this rank's PRN shard, gathered as per-PRN result records."""
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        from oracle import oracle
        from pocketsdr_b200 import dist as D
        from pocketsdr_b200 import synth
        dist = D.init(backend="gloo", timeout_s=60)
        wl = _small_workload(synth)
        mine, index = D.shard_groups(wl.groups, rank, world)
        cfs = [synth.group_code_ffts(g) for g in mine]
        ref = oracle.search_groups(mine, wl.bufs, cfs, max_threads=2)
        full = D.gather_results(_records(ref["res"]), index, wl.groups, world, dist)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, np.concatenate(full).tobytes()))
    except Exception as e:  # surfaced in the parent
        q.put((rank, "error: " + repr(e)))


def _small_workload(synth):
    wl = synth.acq_multi_24mhz(seed=12, prn_limit=5, t_sum=2e-3)
    for g in wl.groups:
        g.fds = g.fds[::10].copy()
    return wl


def _records(r):
    dt = np.dtype([("bin", np.int32), ("offset", np.int32), ("cn0", np.float32),
                   ("pmax", np.float32), ("pave", np.float64), ("fd", np.float64)])
    out = np.zeros(len(r), dt)
    for f in ("bin", "offset", "cn0", "fd"):
        out[f] = r[f]
    out["pmax"] = r["pmax"]
    out["pave"] = r["pmean"]
    return out


def test_two_gloo_ranks_gather_real_search_results():
    """PRNs dealt over two ranks, each searching its share with the reference
    path on CPU; the gathered per-PRN results equal one process searching
    every PRN."""
    import torch.multiprocessing as mp
    from oracle import oracle
    from pocketsdr_b200 import synth
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_search_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
    for r in (0, 1):
        assert not isinstance(out[r], str), out[r]
    wl = _small_workload(synth)
    single = oracle.search_groups(wl.groups, wl.bufs, [synth.group_code_ffts(g) for g in wl.groups])
    want = _records(single["res"]).tobytes()
    assert out[0] == want and out[1] == want
