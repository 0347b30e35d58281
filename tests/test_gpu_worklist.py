"""The work-list consumer (sdrg_acq_set_worklist): every group's (PRN,
Doppler bin) tasks consumed by one persistent launch against the per-group
launches on concurrent streams - the same arithmetic in another kernel, so
grids equal within FP32 rounding (1e-5 per cell of max(|P|, mean P)) and the
same peaks - including narrow units that straddle two groups and groups of
different sum counts; CUDA-graph replay of the work list, bit for bit against
its own stream launch; plans it cannot take."""
import numpy as np
import pytest

from pocketsdr_b200 import synth

pytestmark = pytest.mark.gpu


def _plan(wl):
    from pocketsdr_b200.acquire import AcqPlan
    return AcqPlan(wl.groups, [synth.group_code_ffts(g) for g in wl.groups])


def _grids(plan, wl):
    return [plan.grid(i).copy() for i in range(len(wl.groups))]


def test_worklist_equals_per_group_launches():
    wl = synth.acq_multi_24mhz(seed=31, prn_limit=5, t_sum=4e-3)
    wl.groups[2].n_sum = 2          # B1I: fewer sums than the other narrow groups
    assert [g.L for g in wl.groups] == [48000, 192000, 48000, 48000]
    plan = _plan(wl)
    try:
        assert plan.set_worklist(0) is False
        r0 = plan.run_host(wl.bufs, wl.ix)
        g0 = _grids(plan, wl)
        assert plan.set_worklist(1) is True
        r1 = plan.run_host(wl.bufs, wl.ix)
        g1 = _grids(plan, wl)
        for a, b in zip(g0, g1):
            floor = float(a.mean(dtype=np.float64))
            err = np.abs(a.astype(np.float64) - b) / np.maximum(np.abs(a), floor)
            assert err.max() <= 1e-5, float(err.max())
        assert np.array_equal(r0["bin"], r1["bin"]) and np.array_equal(r0["offset"], r1["offset"])
        assert np.abs(r0["cn0"] - r1["cn0"]).max() < 1e-3
        # a second run over the same buffers (queue heads re-armed): the same
        # kernels on the same data, bit for bit
        r2 = plan.run_host(wl.bufs, wl.ix)
        assert np.array_equal(r1, r2)
    finally:
        plan.close()


def test_worklist_graph_replay_and_narrow_only_plan():
    import torch
    from pocketsdr_b200 import acquire
    wl = synth.acq_l1ca_12mhz(seed=3)
    wl.groups[0].prns = wl.groups[0].prns[:11]      # 11 x 41 tasks: a partial last unit
    plan = _plan(wl)
    try:
        assert plan.set_worklist(1) is True
        ref = plan.run_host(wl.bufs, wl.ix)
        bufs = [torch.from_numpy(b).cuda() for b in wl.bufs]
        res = torch.empty(plan.n_res * acquire.RESULT_DTYPE.itemsize, dtype=torch.uint8,
                          device="cuda")
        st = torch.cuda.current_stream().cuda_stream
        for _ in range(3):
            plan.run_device([b.data_ptr() for b in bufs], [len(b) for b in wl.bufs], wl.ix,
                            res.data_ptr(), st, graph=True)
        torch.cuda.synchronize()
        got = np.frombuffer(res.cpu().numpy().tobytes(), dtype=acquire.RESULT_DTYPE)
        assert np.array_equal(got, ref)
        assert plan.graph_captures() == 1
    finally:
        plan.close()


def test_worklist_refused_for_staged_splits():
    from pocketsdr_b200.acquire import AcqPlan
    from pocketsdr_b200._lib import GpuError
    wl = synth.acq_long_48mhz(prn_limit=1, n_sum=1, bins=np.array([0.0], np.float32))
    plan = AcqPlan(wl.groups, [synth.long_code_ffts(g) for g in wl.groups])
    try:
        assert plan.set_worklist(-1) is False
        with pytest.raises(GpuError, match="24 000-point"):
            plan.set_worklist(1)
    finally:
        plan.close()
