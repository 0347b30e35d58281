"""GPU parity through the C ABI against the oracle and the reference's golden
vectors.

Bars:
* mixing and standard correlators: bit-exact (integer stages and the FP32
  scaling, compared as raw float bits);
* FFT correlator / search grids (FP32): per cell
  |GPU - ref| <= 1e-4 * max(|ref|, mean(ref))   (POWER_RTOL below), and
  for complex correlations |GPU - ref| <= 1e-4 * max(|ref|, rms(ref));
* peaks (Doppler bin, code offset) identical; C/N0 within 0.1 dB.
"""
import numpy as np
import pytest

from pocketsdr_b200 import codes, synth

pytestmark = pytest.mark.gpu

POWER_RTOL = 1e-4
CPLX_RTOL = 1e-4


def assert_power_close(P, ref):
    floor = max(float(np.mean(ref)), 0.0)
    err = np.abs(P.astype(np.float64) - ref)
    bound = POWER_RTOL * np.maximum(np.abs(ref), floor)
    bad = err > bound
    assert not bad.any(), f"{bad.sum()} cells off; worst ratio {np.max(err / np.maximum(bound, 1e-30)):.3g}"


def assert_cplx_close(c, ref):
    rms = float(np.sqrt(np.mean(np.abs(ref) ** 2)))
    err = np.abs(c.astype(np.complex128) - ref)
    bound = CPLX_RTOL * np.maximum(np.abs(ref), rms)
    assert np.all(err <= bound), f"worst ratio {np.max(err / np.maximum(bound, 1e-30)):.3g}"


def pack_cpx8(re, im):
    return ((im & 0x0F) << 4) | (re & 0x0F)


def assert_same_peak(gpu_pk, ref_pk, Pref, period=None):
    """Peaks must be identical. The one exception is a replica tiled from a
    shorter periodic code (period = samples per code period): its grid has
    mathematically equal maxima `period` samples apart, and FP32 rounding
    picks one of them in either implementation - then the GPU's cell must be
    the same bin and offset modulo the period, and a near-exact tie
    (within 1e-5) in the reference's own grid."""
    gpu_pk = (int(gpu_pk[0]), int(gpu_pk[1]))
    if gpu_pk == tuple(ref_pk):
        return
    assert period, f"peak {gpu_pk} != reference {tuple(ref_pk)}"
    assert gpu_pk[0] == ref_pk[0] and gpu_pk[1] % period == ref_pk[1] % period, (gpu_pk, ref_pk)
    assert Pref[gpu_pk] >= (1 - 1e-5) * Pref[tuple(ref_pk)], (Pref[gpu_pk], Pref[tuple(ref_pk)])


# ---- carrier wipe-off -----------------------------------------------------------
def test_mix_known_answers(gpu):
    buf = np.array([pack_cpx8(1, -2), pack_cpx8(2, 1), pack_cpx8(-1, 3), pack_cpx8(0, -1)],
                   np.uint8)
    assert gpu.sdr_mix_carr(buf, 0, 2, 4.0, 0.0, 0.0).tolist() == [[11, -22], [22, 11]]
    assert gpu.sdr_mix_carr(buf, 3, 3, 4.0, 0.0, 0.0)[:2].tolist() == [[0, -11], [11, -22]]


def test_mix_full_table(gpu, orc):
    tb = np.repeat(np.arange(256, dtype=np.uint8), 256)
    assert np.array_equal(gpu.sdr_mix_carr(tb, 0, 65536, 256.0, 1.0, 0.0), orc.mix_table())


def test_mix_golden(gpu, golden):
    g = golden("mix.npz")
    off = 0
    for (ix, N, fs, fc, phi), n in zip(g["cases"], g["lens"]):
        o = gpu.sdr_mix_carr(g["buf"], int(ix), int(N), fs, fc, phi)
        assert np.array_equal(o, g["out"][off:off + n])
        off += n


def test_mix_random_vs_oracle(gpu, orc):
    rng = np.random.default_rng(11)
    for _ in range(40):
        L = int(rng.integers(100, 300000))
        N = int(rng.integers(1, L + 1))
        buf = rng.integers(0, 256, L, dtype=np.uint8)
        ix = int(rng.integers(0, L))
        fs = float(rng.uniform(1e6, 48e6))
        fc = float(rng.uniform(-0.49 * fs, 0.49 * fs))
        phi = float(rng.uniform(-5, 5))
        assert np.array_equal(gpu.sdr_mix_carr(buf, ix, N, fs, fc, phi),
                              orc.mix_carr(buf, ix, N, fs, fc, phi))


# ---- standard correlators -------------------------------------------------------
def test_corr_std_golden(gpu, golden):
    g = golden("corr_std.npz")
    for name, cpx in (("real", False), ("cpx", True)):
        off = 0
        for k, (coff, n) in enumerate(zip(g["coffs"], g["npos"])):
            pos = g["pos"][off:off + n]
            c, Cb = gpu.sdr_corr_std(g["IQ"], g[f"code_{name}"], float(coff), pos, cpx)
            assert np.array_equal(c.view(np.uint32), g[f"corr_{name}"][off:off + n].view(np.uint32))
            assert np.array_equal(Cb.view(np.uint32), g[f"C_{name}"][k].view(np.uint32))
            off += n


def test_corr_std_random_vs_oracle(gpu, orc):
    rng = np.random.default_rng(5)
    for t in range(40):
        N = int(rng.integers(16, 30000))
        IQ = rng.integers(-128, 128, (N, 2), dtype=np.int8)
        cpx = bool(t % 2)
        code = (rng.choice(np.array([-1, 0, 1], np.int8), (10 * N, 2)) if cpx else
                np.repeat(rng.choice(np.array([-1, 1], np.int8), (10 * N, 1)), 2, 1))
        n = int(rng.integers(3, 108))
        pos = np.concatenate([[0.0, -3.3, 3.3], rng.uniform(-N, N, n - 3)])
        coff = float(rng.uniform(0, N))
        a, A = gpu.sdr_corr_std(IQ, code, coff, pos, cpx)
        b, B = orc.corr_std(IQ, code, coff, pos, cpx)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), t
        assert np.array_equal(A.view(np.uint32), B.view(np.uint32)), t


def test_cpx_buffer_golden(gpu, golden):
    g = golden("cpx_buffer.npz")
    c = gpu.corr_std(g["buff"], 1700, 2000, 4e6, 1.1e6, 0.25, g["code"], g["pos"])
    assert np.array_equal(c.view(np.uint32), g["corr_std"].view(np.uint32))
    f = gpu.corr_fft(g["buff"], 900, 2000, 4e6, -0.7e6, 0.6, g["code_fft"])
    assert_cplx_close(f, g["corr_fft"])


# ---- FFT correlator ----------------------------------------------------------------
def test_corr_fft_zero_code(gpu):
    IQ = np.array([[1, 0], [2, -1], [3, -2], [4, -3]], np.int8)
    assert np.max(np.abs(gpu.sdr_corr_fft(IQ, np.zeros(4, np.complex64)))) <= 1e-6


def test_corr_fft_golden(gpu, golden):
    g = golden("search.npz")
    assert_cplx_close(gpu.sdr_corr_fft(g["IQm"], g["code_fft"]), g["corr"])


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 8, 30, 100, 1000, 2000, 4096, 12000,
                               24000, 25000, 48000, 64000, 96000, 120000, 192000,
                               240000, 384000, 480000])
def test_corr_fft_sizes_vs_oracle(gpu, orc, N):
    rng = np.random.default_rng(N)
    IQ = rng.integers(-100, 101, (N, 2), dtype=np.int8)
    cf = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    assert_cplx_close(gpu.sdr_corr_fft(IQ, cf), orc.corr_fft(IQ, cf))


# ---- search ----------------------------------------------------------------------------
def test_search_golden(gpu, golden):
    g = golden("search.npz")
    fs, fi, T = g["params"]
    Ns = int(fs * T)
    P = np.zeros_like(g["P"])
    for ix in g["ix"]:
        gpu.sdr_search_code(g["code_fft"], T, g["ifbuf"], int(ix), 2 * Ns, fs, fi, g["fds"], P)
    assert_power_close(P, g["P"])
    cn0, pk = gpu.sdr_corr_max(P, 2 * Ns, Ns, len(g["fds"]), T)
    assert pk == tuple(g["peak"])
    assert abs(cn0 - float(g["cn0"])) < 0.1
    assert abs(gpu.sdr_fine_dop(P, 2 * Ns, g["fds"], pk) - float(g["fd"])) < 0.5


def test_search_accumulates(gpu):
    buf = np.array([pack_cpx8(i + 1, -i) for i in range(4)], np.uint8)
    P = np.ones((1, 4), np.float32)
    gpu.sdr_search_code(np.zeros(4, np.complex64), 1.0, buf, 0, 4, 4.0, 0.0,
                        np.zeros(1, np.float32), P)
    assert np.allclose(P, 1.0, atol=1e-6)


def test_search_helpers_known_answers(gpu):
    P = np.array([1, 1, 1, 1, 1, 1, 4, 1, 1, 1, 1, 1], np.float32)
    cn0, ix = gpu.sdr_corr_max(P, 4, 4, 3, 0.001)
    assert cn0 > 0 and ix == (1, 2)
    fds = np.array([-500.0, 0.0, 500.0], np.float32)
    assert abs(gpu.sdr_fine_dop(P, 4, fds, ix)) < 1e-6
    assert abs(gpu.sdr_fine_dop(P, 4, fds, (0, 0)) + 500.0) < 1e-6
    assert abs(gpu.sdr_corr_max(np.zeros(4, np.float32), 4, 4, 1, 0.001)[0]) < 1e-6
    b = gpu.sdr_dop_bins(0.001, 0.0, 1000.0)
    assert b.tolist() == [-1000.0, -500.0, 0.0, 500.0, 1000.0]


def test_dop_bins_golden(gpu):
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "meta.json")) as f:
        meta = json.load(f)
    for key, vals in meta["dop_bins"].items():
        T, d, m = (float(x) for x in key.split("_"))
        assert gpu.sdr_dop_bins(T, d, m).tolist() == vals


def _oracle_group_grid(ref, g, code_fft, buf, ix0):
    """Reference grid of one PRN: sdr_search_code per sum (N = L), first Nmax
    columns kept."""
    P = np.zeros((len(g.fds), g.L), np.float32)
    for s in range(g.n_sum):
        ix = (ix0 + s * g.N) % len(buf)
        ref.search_code(code_fft, buf, ix, g.L, g.fs, g.fi, g.fds, P)
    return P[:, :g.Nmax]


def test_batched_acquisition_vs_oracle(gpu, ref):
    from pocketsdr_b200.acquire import AcqPlan
    wl = synth.acq_multi_24mhz(seed=3, prn_limit=3, t_sum=3e-3)
    cf = [synth.group_code_ffts(g) for g in wl.groups]
    plan = AcqPlan(wl.groups, cf)
    res = plan.run_host(wl.bufs, wl.ix)
    k = 0
    for gi, (g, c) in enumerate(zip(wl.groups, cf)):
        G = plan.grid(gi)
        for p in range(len(g.prns)):
            Pref = _oracle_group_grid(ref, g, c[p], wl.bufs[g.buf], wl.ix[g.buf])
            assert_power_close(G[p], Pref)
            cn0, pk = ref.corr_max(Pref, g.Nmax, g.Nmax, len(g.fds), g.T)
            r = res[k]
            assert (r["bin"], r["offset"]) == pk, (g.sig, g.prns[p])
            assert abs(float(r["cn0"]) - cn0) < 0.1, (g.sig, g.prns[p], float(r["cn0"]), cn0)
            k += 1


def test_e1b_cluster_sums_vs_oracle(gpu, ref):
    """Galileo E1-B (L = 192 000, clusters of 8 CTAs) over 3 sums of 4 ms: the
    power accumulator's first, middle and last sums against the reference's
    grid; identical peaks, C/N0 within 0.1 dB."""
    from pocketsdr_b200.acquire import AcqPlan
    wl = synth.acq_multi_24mhz(seed=21, prn_limit=2, t_sum=12e-3, sigs=(("E1B", 0),))
    g = wl.groups[0]
    g.fds = g.fds[::4]
    assert g.n_sum == 3 and g.L == 192000
    cf = synth.group_code_ffts(g)
    plan = AcqPlan([g], [cf])
    res = plan.run_host(wl.bufs, wl.ix)
    G = plan.grid(0)
    for p in range(len(g.prns)):
        Pref = _oracle_group_grid(ref, g, cf[p], wl.bufs[g.buf], wl.ix[g.buf])
        assert_power_close(G[p], Pref)
        cn0, pk = ref.corr_max(Pref, g.Nmax, g.Nmax, len(g.fds), g.T)
        assert_same_peak((res[p]["bin"], res[p]["offset"]), pk, Pref)
        assert abs(float(res[p]["cn0"]) - cn0) < 0.1


def test_batched_grid_matches_search_code(gpu):
    """The batched grid equals sdr_search_code accumulated over the sums."""
    from pocketsdr_b200.acquire import AcqPlan
    wl = synth.acq_multi_24mhz(seed=4, prn_limit=2, t_sum=2e-3, sigs=(("L1CA", 0),))
    g = wl.groups[0]
    cf = synth.group_code_ffts(g)
    plan = AcqPlan([g], [cf])
    plan.run_host(wl.bufs, wl.ix)
    G = plan.grid(0)
    assert G.shape == (len(g.prns), len(g.fds), g.Nmax)
    for p in range(len(g.prns)):
        P = np.zeros((len(g.fds), g.L), np.float32)
        for s in range(g.n_sum):
            gpu.sdr_search_code(cf[p], g.T, wl.bufs[0], s * g.N, g.L, g.fs, g.fi, g.fds, P)
        assert_power_close(G[p], P[:, :g.Nmax])


def test_real_front_end_data_vs_reference_fixture(gpu, golden):
    """Real data: 20 ms of the reference's own L1 sample (12 MHz, IF 3 MHz,
    2-bit) searched for GPS L1 C/A PRN 1-32, 4 ms coherent (code tiled x4,
    48 000-point circular correlation) x 5 sums, against the reference's
    sdr_search_code / sdr_corr_max / sdr_fine_dop results stored in the
    fixture. Detected PRNs (the reference finds 2, 5, 11, 13, 15, 18, 20, 29,
    30 at >= 38 dB-Hz): same Doppler bin, same code offset modulo the 1 ms
    period (the tiled replica makes the four maxima exactly equal), C/N0
    within 0.1 dB. Every PRN: peak power within 1e-4 and C/N0 within 0.1 dB."""
    from pocketsdr_b200.acquire import AcqPlan
    d = golden("real_l1ca.npz")
    fs, fi, T, N, n_sum = d["params"]
    N, n_sum = int(N), int(n_sum)
    g = synth.Group("L1CA", list(range(1, 33)), fs, fi, T, N, N, N, n_sum, d["fds"], 0, tile=4)
    plan = AcqPlan([g], [synth.group_code_ffts(g)])
    res = plan.run_host([d["buf"]], [0])
    ref_res = d["res"]
    det = [int(r["prn"]) for r in ref_res if r["cn0"] >= 38.0]
    assert det == [2, 5, 11, 13, 15, 18, 20, 29, 30]
    period = N // 4
    for r, e in zip(res, ref_res):
        assert abs(float(r["cn0"]) - float(e["cn0"])) < 0.1, (int(e["prn"]), r, e)
        assert float(r["pmax"]) == pytest.approx(float(e["pmax"]), rel=1e-4)
        if e["cn0"] >= 38.0:
            assert int(r["bin"]) == int(e["bin"]), (int(e["prn"]), r, e)
            assert int(r["offset"]) % period == int(e["offset"]) % period, (int(e["prn"]), r, e)
            assert float(r["fd"]) == pytest.approx(float(e["fd"]), abs=0.5)


def test_acq_l1ca_12mhz_peaks(gpu, ref):
    """The 12 MHz real-IF L1 C/A search (4 ms coherent x 5 sums) on the
    visible PRNs and a few absent ones: identical peaks, C/N0 within 0.1 dB."""
    from pocketsdr_b200.acquire import AcqPlan
    wl = synth.acq_l1ca_12mhz(seed=1)
    g = wl.groups[0]
    vis = sorted({s.prn for s in wl.sats})
    absent = [p for p in g.prns if p not in vis][:3]
    g.prns = vis + absent
    cf = synth.group_code_ffts(g)
    plan = AcqPlan([g], [cf])
    res = plan.run_host(wl.bufs, wl.ix)
    truth = {s.prn: s for s in wl.sats}
    period = int(round(g.fs * codes.code_cyc("L1CA")))   # replica tiled x4
    for p, prn in enumerate(g.prns):
        Pref = _oracle_group_grid(ref, g, cf[p], wl.bufs[0], 0)
        cn0, pk = ref.corr_max(Pref, g.Nmax, g.Nmax, len(g.fds), g.T)
        r = res[p]
        assert_same_peak((r["bin"], r["offset"]), pk, Pref, period)
        assert abs(float(r["cn0"]) - cn0) < 0.1, prn
        if prn in truth:   # the visible satellites are found at their Doppler
            s = truth[prn]
            assert abs(float(g.fds[r["bin"]]) - s.doppler) <= 250.0
            assert cn0 > 30.0


def test_long_coherent_search_vs_oracle(gpu, ref):
    """10 ms coherent integration at 48 MHz: 480 000-point transforms split
    20 x 24 000 (staged through the scratch), 2 sums, against the reference's
    own sdr_search_code grids; identical peaks, C/N0 within 0.1 dB."""
    from pocketsdr_b200.acquire import AcqPlan
    wl = synth.acq_long_48mhz(seed=8, prn_limit=2, n_sum=2,
                              bins=np.array([-9000, -150, -100, -50, 0, 50, 100], np.float32))
    cf = [synth.long_code_ffts(g) for g in wl.groups]
    plan = AcqPlan(wl.groups, cf)
    res = plan.run_host(wl.bufs, wl.ix)
    k = 0
    for gi, (g, c) in enumerate(zip(wl.groups, cf)):
        G = plan.grid(gi)
        for p in range(len(g.prns)):
            Pref = _oracle_group_grid(ref, g, c[p], wl.bufs[g.buf], wl.ix[g.buf])
            assert_power_close(G[p], Pref)
            cn0, pk = ref.corr_max(Pref, g.Nmax, g.Nmax, len(g.fds), g.T)
            r = res[k]
            assert_same_peak((r["bin"], r["offset"]), pk, Pref)
            assert abs(float(r["cn0"]) - cn0) < 0.1
            k += 1


def test_long_coherent_multi_chunk_vs_oracle(gpu, ref):
    """A staged search of more tasks than one scratch chunk holds (4 PRNs x 20
    bins = 80 (PRN, bin) tasks; a chunk of 480 000-point tasks holds 69): the
    grids of PRNs with tasks in both chunks within 1e-4 of the reference's
    sdr_search_code over the same sums, peaks identical, C/N0 within 0.1 dB."""
    from pocketsdr_b200.acquire import AcqPlan
    wl = synth.acq_long_48mhz(seed=13, prn_limit=4, n_sum=2,
                              bins=np.arange(-500, 500, 50, dtype=np.float32))
    wl.groups = wl.groups[:1]
    g = wl.groups[0]
    assert len(g.prns) * len(g.fds) == 80
    cf = [synth.long_code_ffts(g)]
    plan = AcqPlan([g], cf)
    res = plan.run_host(wl.bufs, wl.ix)
    G = plan.grid(0)
    for p in (0, 3):                  # tasks of both chunks (bin-major order)
        Pref = _oracle_group_grid(ref, g, cf[0][p], wl.bufs[g.buf], wl.ix[g.buf])
        assert_power_close(G[p], Pref)
        cn0, pk = ref.corr_max(Pref, g.Nmax, g.Nmax, len(g.fds), g.T)
        assert_same_peak((res[p]["bin"], res[p]["offset"]), pk, Pref)
        assert abs(float(res[p]["cn0"]) - cn0) < 0.1


@pytest.mark.parametrize("n_bins", [3, 72])
def test_search_code_staged_dropin(gpu, ref, n_bins):
    """The drop-in sdr_search_code at L = 480 000 (staged split, P in/out,
    accumulated onto the caller's values); 72 bins span two scratch chunks."""
    wl = synth.acq_long_48mhz(seed=9, prn_limit=1, n_sum=1,
                              bins=np.arange(n_bins, dtype=np.float32) * 50 - 50)
    g = wl.groups[0]
    cf = synth.long_code_ffts(g)[0]
    P = np.full((len(g.fds), g.L), 0.5, np.float32)
    Pr = P.copy()
    gpu.sdr_search_code(cf, g.T, wl.bufs[0], 1000, g.L, g.fs, g.fi, g.fds, P)
    ref.search_code(cf, wl.bufs[0], 1000, g.L, g.fs, g.fi, g.fds, Pr, g.T)
    assert_power_close(P, Pr)
