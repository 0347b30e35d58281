"""torch.ops.pocketsdr.search and torch.ops.pocketsdr.corr_batch on a B200
against the reference: the search grid within 1e-4 of sdr_search_code summed
over the same code periods with identical peaks and C/N0 within 0.1 dB
(src/sdr_func.c:641-706); the correlators bit-identical to sdr_mix_carr +
sdr_corr_std per channel (src/sdr_ch.c:725-733)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_prn", [4, 1])
def test_search_op_vs_reference(gpu, ref, n_prn):
    """n_prn = 1: 21 (PRN, bin) tasks, few enough for the plan to take a finer
    split of its 48 000-point transforms (8 ways), codes laid out for it."""
    torch = pytest.importorskip("torch")
    from pocketsdr_b200 import codes, ops, synth  # noqa: F401
    wl = synth.acq_multi_24mhz(seed=3, prn_limit=n_prn, t_sum=2e-3, sigs=(("L1CA", 0),))
    g = wl.groups[0]
    buf = wl.bufs[g.buf]
    chips = np.stack([codes.gen_code(g.sig, p) for p in g.prns])
    d = torch.from_numpy(buf).cuda()
    grid, b, off, cn0, fd = torch.ops.pocketsdr.search(
        d, 0, torch.from_numpy(chips).cuda(), [float(f) for f in g.fds], g.fs, g.fi, g.T,
        g.N, g.L - g.N, g.n_sum)
    grid, b, off, cn0 = grid.cpu().numpy(), b.cpu().numpy(), off.cpu().numpy(), cn0.cpu().numpy()
    for p, prn in enumerate(g.prns):
        cf = ref.gen_code_fft(chips[p], None, g.T, 0.0, g.fs, g.N, g.L - g.N)
        P = np.zeros((len(g.fds), g.L), np.float32)
        for s in range(g.n_sum):
            ref.search_code(cf, buf, (s * g.N) % len(buf), g.L, g.fs, g.fi, g.fds, P, g.T)
        P = P[:, :g.Nmax]
        floor = float(P.mean())
        assert np.all(np.abs(grid[p] - P) <= 1e-4 * np.maximum(np.abs(P), floor)), prn
        c, pk = ref.corr_max(P, g.Nmax, g.Nmax, len(g.fds), g.T)
        assert (int(b[p]), int(off[p])) == pk, prn
        assert abs(float(cn0[p]) - c) < 0.1, prn
    # a second call of the same shape reuses the plan and gives the same grid
    grid2 = torch.ops.pocketsdr.search(
        d, 0, torch.from_numpy(chips).cuda(), [float(f) for f in g.fds], g.fs, g.fi, g.T,
        g.N, g.L - g.N, g.n_sum)[0].cpu().numpy()
    assert np.array_equal(grid.view(np.uint32), grid2.view(np.uint32))
    ops.release_plans()


def test_corr_batch_op_bit_exact(gpu, orc):
    torch = pytest.importorskip("torch")
    from pocketsdr_b200 import codes, ops, synth, track  # noqa: F401
    fs, T = 24e6, 1e-3
    N = int(fs * T)
    sats = [synth.Sat("L1CA", p, (90.0 * p) % 1023, 250.0 * p - 1500, 0.1 * p, 45.0)
            for p in (2, 9, 23)]
    buf = synth.gen_if(5 * N, fs, {"L1CA": 4.0e6}, sats, iq=True, bits=3, seed=4)
    sc = T / 1023 * fs
    pos = [0.0, -0.5 * sc, 0.5 * sc, -120.0] + list(np.arange(-10, 10) * 0.05 * sc)
    banks = np.stack([track.code_bank(codes.gen_code("L1CA", s.prn), T, fs, N) for s in sats])
    ix = [N + 17 * k for k in range(len(sats))]
    fc = [4.0e6 + s.doppler for s in sats]
    phi = [0.3, -0.2, 0.05]
    coff = [(1023 - s.code_phase) / 1023 * N + 0.37 for s in sats]
    out = torch.ops.pocketsdr.corr_batch(torch.from_numpy(buf).cuda(), ix, fc, phi, coff,
                                         torch.from_numpy(banks).cuda(), pos, fs, N)
    out = out.cpu().numpy()
    for j in range(len(sats)):
        IQ = orc.mix_carr(buf, ix[j], N, fs, fc[j], phi[j])
        want, _ = orc.corr_std(IQ, banks[j], coff[j], np.asarray(pos), False)
        assert np.array_equal(out[j].view(np.uint32), want.view(np.uint32)), j


def test_ops_ordered_after_torch_default_stream(gpu):
    """The operators run on torch's current stream, the legacy default stream
    here: an IF buffer whose fill is still queued behind a 0.1 s spin on that
    stream is searched only once it is filled, and the grid's copy waits for
    the search."""
    torch = pytest.importorskip("torch")
    from pocketsdr_b200 import codes, ops, synth  # noqa: F401
    wl = synth.acq_multi_24mhz(seed=3, prn_limit=1, t_sum=2e-3, sigs=(("L1CA", 0),))
    g = wl.groups[0]
    chips = torch.from_numpy(np.stack([codes.gen_code(g.sig, p) for p in g.prns])).cuda()
    src = torch.from_numpy(wl.bufs[g.buf]).cuda()
    args = (chips, [float(f) for f in g.fds], g.fs, g.fi, g.T, g.N, g.L - g.N, g.n_sum)
    want = torch.ops.pocketsdr.search(src, 0, *args)[0].cpu().numpy()
    torch.cuda.synchronize()
    for _ in range(2):
        d = torch.zeros_like(src)
        torch.cuda._sleep(200_000_000)          # about 0.1 s of device time
        d.copy_(src)
        got = torch.ops.pocketsdr.search(d, 0, *args)[0].cpu().numpy()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    ops.release_plans()
