"""The strong-scaling split end to end on the GPU: two processes (ranks of a
gloo group, both on the one GPU of this host; their kernels never wait on
each other) each run the acquisition plan over their round-robin share of
every group's PRNs and all-gather the 32-byte per-PRN results; the gathered
results equal one process searching every PRN, bit for bit."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _workload(synth):
    return synth.acq_multi_24mhz(seed=13, prn_limit=6, t_sum=4e-3)


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK="0",
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        import torch
        torch.cuda.set_device(0)
        from pocketsdr_b200 import acquire, synth
        from pocketsdr_b200 import dist as D
        dist = D.init(backend="gloo", timeout_s=120)
        wl = _workload(synth)
        mine, index = D.shard_groups(wl.groups, rank, world)
        plan = acquire.AcqPlan(mine, [synth.group_code_ffts(g) for g in mine])
        res = plan.run_host(wl.bufs, wl.ix)
        plan.close()
        full = D.gather_results(res, index, wl.groups, world, dist)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, np.concatenate(full).tobytes()))
    except Exception as e:  # surfaced in the parent
        q.put((rank, "error: " + repr(e)))


def test_strong_split_two_processes_equals_one():
    import torch.multiprocessing as mp
    from pocketsdr_b200 import acquire, synth
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=600) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
    for r in (0, 1):
        assert not isinstance(out[r], str), out[r]
    wl = _workload(synth)
    plan = acquire.AcqPlan(wl.groups, [synth.group_code_ffts(g) for g in wl.groups])
    want = plan.run_host(wl.bufs, wl.ix).tobytes()
    plan.close()
    assert out[0] == want and out[1] == want
