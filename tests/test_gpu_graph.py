"""CUDA-graph launch of a batched search (sdrg_acq_run_graph): the replayed
graph gives the grids and peaks of the stream-launched run bit for bit, the
read position of a replay moves through the tables without a new capture,
new buffers are captured again, and the peaks agree with the reference's
sdr_search_code + sdr_corr_max (src/sdr_func.c:641-705) on the same input."""
import numpy as np
import pytest

from pocketsdr_b200 import synth

pytestmark = pytest.mark.gpu


def _device_run(plan, d_bufs, ix, graph, torch):
    from pocketsdr_b200._lib import torch_stream
    from pocketsdr_b200.acquire import RESULT_DTYPE
    res = torch.zeros(plan.n_res * RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    st = torch_stream()
    plan.run_device([b.data_ptr() for b in d_bufs], [b.numel() for b in d_bufs], ix,
                    res.data_ptr(), st, graph=graph)
    torch.cuda.synchronize()
    out = res.cpu().numpy().view(RESULT_DTYPE).copy()
    grids = [plan.grid(g) for g in range(len(plan.groups))]
    return out, grids


def _same(a, b):
    ra, ga = a
    rb, gb = b
    assert np.array_equal(ra.view(np.uint8), rb.view(np.uint8))
    for x, y in zip(ga, gb):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


def test_graph_replay_matches_stream_launch(gpu):
    torch = pytest.importorskip("torch")
    from pocketsdr_b200.acquire import AcqPlan
    wl = synth.acq_multi_24mhz(seed=5, prn_limit=3, t_sum=2e-3)
    plan = AcqPlan(wl.groups, [synth.group_code_ffts(g) for g in wl.groups])
    d = [torch.from_numpy(np.ascontiguousarray(b)).cuda() for b in wl.bufs]
    nb = len(d)
    assert plan.graph_captures() == 0
    n0 = min(len(x) for x in wl.bufs)
    for k in (0, 24000 * 3 + 17, n0 - 5000):      # the last one wraps
        ix = [k] * nb
        a = _device_run(plan, d, ix, False, torch)
        b = _device_run(plan, d, ix, True, torch)
        _same(a, b)
        assert plan.graph_captures() == 1
    # the same position twice: tables unchanged, a plain replay
    ix = [123] * nb
    _same(_device_run(plan, d, ix, True, torch), _device_run(plan, d, ix, True, torch))
    assert plan.graph_captures() == 1
    # other buffers: a new capture, results follow the new data
    d2 = [torch.flip(x, [0]).contiguous() for x in d]
    a = _device_run(plan, d2, [0] * nb, False, torch)
    b = _device_run(plan, d2, [0] * nb, True, torch)
    _same(a, b)
    assert plan.graph_captures() == 2
    plan.close()


def test_graph_staged_split_peaks_vs_reference(gpu, ref):
    """A 480 000-point search (20 x 24 000 staged through the scratch: several
    launches per sum inside the graph) against the reference's own grids."""
    torch = pytest.importorskip("torch")
    from pocketsdr_b200.acquire import AcqPlan
    wl = synth.acq_long_48mhz(seed=12, prn_limit=1, n_sum=2,
                              bins=np.array([-50, 0, 50], np.float32))
    cf = [synth.long_code_ffts(g) for g in wl.groups]
    plan = AcqPlan(wl.groups, cf)
    d = [torch.from_numpy(np.ascontiguousarray(b)).cuda() for b in wl.bufs]
    ix = [x + 1000 for x in wl.ix]
    a = _device_run(plan, d, ix, False, torch)
    b = _device_run(plan, d, ix, True, torch)
    _same(a, b)
    res = b[0]
    for gi, (g, c) in enumerate(zip(wl.groups, cf)):
        P = np.zeros((len(g.fds), g.L), np.float32)
        for s in range(g.n_sum):
            ref.search_code(c[0], wl.bufs[g.buf], (ix[g.buf] + s * g.N) % len(wl.bufs[g.buf]),
                            g.L, g.fs, g.fi, g.fds, P)
        P = P[:, :g.Nmax]
        G = b[1][gi][0]
        floor = float(np.mean(P))
        assert np.all(np.abs(G.astype(np.float64) - P) <= 1e-4 * np.maximum(np.abs(P), floor))
        cn0, pk = ref.corr_max(P, g.Nmax, g.Nmax, len(g.fds), g.T)
        r = res[plan.offsets[gi]]
        assert (int(r["bin"]), int(r["offset"])) == pk, g.sig
        assert abs(float(r["cn0"]) - cn0) < 0.1, g.sig
    plan.close()
