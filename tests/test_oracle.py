"""The oracle pinned before it is trusted (CPU only).

* known answers of the reference's own unit tests (test/src/test_sdr_func.c);
* the golden fixtures produced by the reference's own C build
  (tests/golden/make_golden.py);
* the reference build itself, where it was compiled on this machine.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import oracle

HAVE_REF = oracle.reference_available()


def pack_cpx8(re, im):
    # test/src/test_sdr_func.c:49-52
    return ((im & 0x0F) << 4) | (re & 0x0F)


def test_mix_known_answers(orc):
    # test/src/test_sdr_func.c:170-192
    buf = np.array([pack_cpx8(1, -2), pack_cpx8(2, 1), pack_cpx8(-1, 3), pack_cpx8(0, -1)],
                   np.uint8)
    out = orc.mix_carr(buf, 0, 2, 4.0, 0.0, 0.0)
    assert out.tolist() == [[11, -22], [22, 11]]
    out = orc.mix_carr(buf, 3, 3, 4.0, 0.0, 0.0)
    assert out[:2].tolist() == [[0, -11], [11, -22]]


def test_mix_table_hash(orc):
    with open(os.path.join(os.path.dirname(__file__), "golden", "meta.json")) as f:
        meta = json.load(f)
    assert hashlib.sha256(orc.mix_table().tobytes()).hexdigest() == meta["mix_table_sha256"]


def test_mix_golden(orc, golden):
    g = golden("mix.npz")
    out, off = g["out"], 0
    for (ix, N, fs, fc, phi), n in zip(g["cases"], g["lens"]):
        o = orc.mix_carr(g["buf"], int(ix), int(N), fs, fc, phi)
        assert np.array_equal(o, out[off:off + n])
        off += n


def test_corr_std_golden(orc, golden):
    g = golden("corr_std.npz")
    pos_all, npos = g["pos"], g["npos"]
    for name, cpx in (("real", False), ("cpx", True)):
        code = g[f"code_{name}"]
        off = 0
        for k, (coff, n) in enumerate(zip(g["coffs"], npos)):
            pos = pos_all[off:off + n]
            c, Cb = orc.corr_std(g["IQ"], code, float(coff), pos, cpx)
            exp = g[f"corr_{name}"][off:off + n]
            assert np.array_equal(c.view(np.uint32), exp.view(np.uint32)), (name, k)
            assert np.array_equal(Cb.view(np.uint32), g[f"C_{name}"][k].view(np.uint32))
            off += n


def test_cpx_buffer_golden(orc, golden):
    g = golden("cpx_buffer.npz")
    c = orc.corr_std_cpx(g["buff"], 1700, 2000, 4e6, 1.1e6, 0.25, g["code"], g["pos"])
    assert np.array_equal(c.view(np.uint32), g["corr_std"].view(np.uint32))
    f = orc.corr_fft_cpx(g["buff"], 900, 2000, 4e6, -0.7e6, 0.6, g["code_fft"])
    ref = g["corr_fft"]
    assert np.max(np.abs(f - ref)) <= 1e-5 * np.max(np.abs(ref))


def test_corr_fft_zero_code(orc):
    # test/src/test_sdr_func.c:231-235: a zero code DFT correlates to 0
    IQ = np.array([[1, 0], [2, -1], [3, -2], [4, -3]], np.int8)
    out = orc.corr_fft(IQ, np.zeros(4, np.complex64))
    assert np.max(np.abs(out)) <= 1e-6


def test_search_golden(orc, golden):
    g = golden("search.npz")
    fs, fi, T = g["params"]
    Ns = int(fs * T)
    P = np.zeros_like(g["P"])
    for ix in g["ix"]:
        orc.search_code(g["code_fft"], g["ifbuf"], int(ix), 2 * Ns, fs, fi, g["fds"], P)
    ref = g["P"]
    floor = max(float(ref.mean()), 0.0)
    assert np.all(np.abs(P - ref) <= 1e-4 * np.maximum(np.abs(ref), floor))
    cn0, pk = orc.corr_max(P, 2 * Ns, Ns, len(g["fds"]), T)
    assert pk == tuple(g["peak"])
    assert abs(cn0 - float(g["cn0"])) < 0.01
    assert abs(orc.fine_dop(P, 2 * Ns, g["fds"], pk) - float(g["fd"])) < 1e-3
    corr = orc.corr_fft(g["IQm"], g["code_fft"])
    assert np.max(np.abs(corr - g["corr"])) <= 1e-5 * np.max(np.abs(g["corr"]))


def test_search_real_data_golden(orc, golden):
    """The restatement on the reference's real L1 sample: for two detected
    PRNs, the peak over the reference's peak bin and its neighbours is the
    reference's (offset modulo the 1 ms period of the x4 tiled code) with the
    same power."""
    from pocketsdr_b200 import codes
    d = golden("real_l1ca.npz")
    fs, fi, T, N, n_sum = d["params"]
    N, n_sum = int(N), int(n_sum)
    for e in d["res"][[12, 28]]:                  # PRN 13 (47.8 dB-Hz), 29 (38.4)
        b = int(e["bin"])
        fds = d["fds"][b - 1: b + 2]
        cf = orc.gen_code_fft(np.tile(codes.gen_code("L1CA", int(e["prn"])), 4), None, T, 0.0,
                              fs, N, 0)
        P = np.zeros((3, N), np.float32)
        for s in range(n_sum):
            orc.search_code(cf, d["buf"], s * N, N, fs, fi, fds, P)
        i, j = np.unravel_index(int(np.argmax(P)), P.shape)
        assert i == 1 and j % (N // 4) == int(e["offset"]) % (N // 4)
        assert float(P[i, j]) == pytest.approx(float(e["pmax"]), rel=1e-5)


def test_search_accumulates(orc):
    # test/src/test_sdr_func.c:237-242: zero code DFT leaves P at 1.0
    buf = np.array([pack_cpx8(i + 1, -i) for i in range(4)], np.uint8)
    P = np.ones((1, 4), np.float32)
    orc.search_code(np.zeros(4, np.complex64), buf, 0, 4, 4.0, 0.0, np.zeros(1, np.float32), P)
    assert np.allclose(P, 1.0, atol=1e-6)


def test_search_helpers_known_answers(orc):
    # test/src/test_sdr_func.c:253-282
    P = np.array([1, 1, 1, 1, 1, 1, 4, 1, 1, 1, 1, 1], np.float32)
    cn0, ix = orc.corr_max(P, 4, 4, 3, 0.001)
    assert cn0 > 0 and ix == (1, 2)
    fds = np.array([-500.0, 0.0, 500.0], np.float32)
    assert abs(orc.fine_dop(P, 4, fds, ix)) < 1e-6
    assert abs(orc.fine_dop(P, 4, fds, (0, 0)) + 500.0) < 1e-6
    assert abs(orc.corr_max(np.zeros(4, np.float32), 4, 4, 1, 0.001)[0]) < 1e-6
    b = orc.dop_bins(0.001, 0.0, 1000.0)
    assert len(b) == 5 and b[0] == -1000.0 and b[2] == 0.0 and b[4] == 1000.0


def test_dop_bins_golden(orc):
    with open(os.path.join(os.path.dirname(__file__), "golden", "meta.json")) as f:
        meta = json.load(f)
    from pocketsdr_b200 import synth
    for key, vals in meta["dop_bins"].items():
        T, d, m = (float(x) for x in key.split("_"))
        assert synth.dop_bins(T, d, m).tolist() == vals


def test_fft_matches_numpy(orc):
    rng = np.random.default_rng(0)
    for n in (1, 2, 7, 12, 100, 1023, 4000, 24000):
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        assert np.allclose(orc.fft(x), np.fft.fft(x), atol=1e-9 * n)
        assert np.allclose(orc.fft(x, True), np.fft.ifft(x) * n, atol=1e-9 * n)


@pytest.mark.skipif(not HAVE_REF, reason="reference build (oracle/_ref) not present")
def test_restatement_vs_reference_random(orc):
    R = oracle.Reference()
    rng = np.random.default_rng(7)
    for _ in range(60):
        n = int(rng.integers(1, 2000))
        L = int(rng.integers(n, n + 300))
        buf = rng.integers(0, 256, L, dtype=np.uint8)
        ix = int(rng.integers(0, L))
        fs = float(rng.uniform(1e6, 30e6))
        fc = float(rng.uniform(-0.45 * fs, 0.45 * fs))
        assert np.array_equal(R.mix_carr(buf, ix, n, fs, fc, 0.3), orc.mix_carr(buf, ix, n, fs, fc, 0.3))
    for t in range(60):
        N = int(rng.integers(20, 2000))
        IQ = rng.integers(-128, 128, (N, 2), dtype=np.int8)
        cpx = bool(t % 2)
        code = (rng.choice(np.array([-1, 0, 1], np.int8), (10 * N, 2)) if cpx else
                np.repeat(rng.choice(np.array([-1, 1], np.int8), (10 * N, 1)), 2, 1))
        pos = rng.uniform(-N, N, int(rng.integers(3, 20)))
        coff = float(rng.uniform(0, N))
        a, A = R.corr_std(IQ, code, coff, pos, cpx)
        b, B = orc.corr_std(IQ, code, coff, pos, cpx)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
        assert np.array_equal(A.view(np.uint32), B.view(np.uint32))


@pytest.mark.skipif(not HAVE_REF, reason="reference build (oracle/_ref) not present")
def test_polarity_contraction_vs_reference(orc):
    """Cases where fused and unfused evaluation of the E/P/L polarity test
    differ in sign: the oracle must follow the reference build."""
    R = oracle.Reference()
    N = 32
    code = np.ones((10 * N, 2), np.int8)
    pos = np.array([0.0, 0.0, 0.0, 5.0])
    for a in range(-60, 61, 11):
        for b in range(-60, 61, 7):
            IQ = np.zeros((N, 2), np.int8)
            IQ[0] = (a, b)
            IQ[16] = (-b, a)
            x, _ = R.corr_std(IQ, code, 16.0, pos)
            y, _ = orc.corr_std(IQ, code, 16.0, pos)
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


@pytest.mark.skipif(not HAVE_REF, reason="reference build (oracle/_ref) not present")
def test_l1ca_codes_vs_reference():
    from pocketsdr_b200 import codes
    R = oracle.Reference()
    for prn in range(1, 33):
        assert np.array_equal(R.gen_code("L1CA", prn), codes.gen_code_L1CA(prn))
    c = R.gen_code("L1CA", 7)
    assert np.array_equal(R.res_code(c, None, 1e-3, -0.7 / 24e6, 24e6, 24000, 0),
                          codes.res_code(c, 1e-3, -0.7 / 24e6, 24e6, 24000, 0))


@pytest.mark.skipif(not HAVE_REF, reason="reference build (oracle/_ref) not present")
def test_replica_restatement_vs_reference(orc):
    """Resampled code banks (the tracking channel's -k/fs/10 offsets,
    src/sdr_ch.c:265-272) bit-exact and code DFTs within 1e-6 of the largest
    value: the restatement matches the reference build it stands in for."""
    R = oracle.Reference()
    rng = np.random.default_rng(12)
    for L, fs, T in ((1023, 24e6, 1e-3), (2046, 12e6, 1e-3), (10230, 20.46e6 * 1.25, 1e-3)):
        c = rng.choice(np.array([-1, 1], np.int8), L)
        q = rng.choice(np.array([-1, 1], np.int8), L)
        N = int(fs * T)
        for k in range(10):
            coff = -k / fs / 10
            assert np.array_equal(orc.res_code(c, None, T, coff, fs, N, 3),
                                  R.res_code(c, None, T, coff, fs, N, 3)), (L, k)
            assert np.array_equal(orc.res_code(c, q, T, coff, fs, N, 0),
                                  R.res_code(c, q, T, coff, fs, N, 0)), (L, k)
    c = rng.choice(np.array([-1, 1], np.int8), 1023)
    for N, Nz in ((6000, 6000), (4000, 0)):
        a = orc.gen_code_fft(c, None, 1e-3, 2e-4, N * 1000.0, N, Nz)
        b = R.gen_code_fft(c, None, 1e-3, 2e-4, N * 1000.0, N, Nz)
        assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max()


@pytest.mark.skipif(not HAVE_REF, reason="reference build (oracle/_ref) not present")
def test_psd_restatement_vs_reference(orc):
    """Welch PSD (src/sdr_func.c:1141-1182): the restatement within 1e-4 dB of
    the reference build, real and complex data, several FFT sizes, and the
    same NaN output when the data hold no full segment."""
    R = oracle.Reference()
    rng = np.random.default_rng(2)
    for N, IQ, n in ((4096, 2, 4096 * 30 + 17), (4096, 1, 4096 * 9), (6000, 2, 42000),
                     (1024, 1, 100)):
        x = (rng.integers(-7, 8, n) + 1j * rng.integers(-7, 8, n) * (IQ == 2)).astype(np.complex64)
        a, b = R.psd_cpx(x, N, 24e6, IQ), orc.psd_cpx(x, N, 24e6, IQ)
        assert np.array_equal(np.isnan(a), np.isnan(b))
        ok = ~np.isnan(a)
        assert np.all(np.abs(a[ok] - b[ok]) <= 1e-4), (N, IQ)


@pytest.mark.skipif(not os.path.exists(oracle.CH_SO), reason="reference channel build absent")
def test_csk_restatement_vs_reference(orc):
    """L6 CSK decode (src/sdr_ch.c:626-664): the restatement gives the
    reference's symbol and bit-identical taps on random correlations with a
    planted code-shift peak."""
    R = oracle.Channel()
    rng = np.random.default_rng(6)
    for _ in range(300):
        N = int(rng.choice([96000, 48000, 192000, 24000]))
        Lc = 20460
        corr = (rng.normal(size=N) + 1j * rng.normal(size=N)).astype(np.complex64)
        sc = N / (Lc / 2)
        corr[int(round(int(rng.integers(0, 256)) * sc)) % N] += np.complex64(40 + 30j)
        pos = np.array([0.0, -0.5 * sc, 0.5 * sc, -120.0] + list(rng.uniform(-3 * sc, 3 * sc, 3)))
        a, b = R.csk(corr, Lc, pos), orc.csk(corr, Lc, pos)
        assert a[0] == b[0] and np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))
    # no power anywhere: symbol of shift 0
    z = np.zeros(24000, np.complex64)
    assert R.csk(z, Lc, [0.0])[0] == orc.csk(z, Lc, [0.0])[0] == 255


@pytest.mark.skipif(not HAVE_REF, reason="reference build (oracle/_ref) not present")
def test_fine_dop_closed_form_matches_reference_lsq():
    """The library's sdr_fine_dop (host; the vertex of the parabola through
    three points, in closed form) against the reference's RTKLIB least-squares
    fit (src/sdr_func.c:709-744) on random grids, bins and spacings, at a
    local maximum along Doppler - what sdr_corr_max hands it: within 1e-9
    relative (the two FP64 evaluations differ by rounding only; far from a
    maximum the parabola flattens, its vertex runs off, and both fits lose
    digits to the conditioning)."""
    import ctypes as C
    from pocketsdr_b200 import _lib
    R = oracle.Reference()
    rng = np.random.default_rng(11)
    for _ in range(3000):
        step = float(rng.choice([50.0, 62.5, 125.0, 250.0, 500.0]))
        M, N = 41, 7
        fds = (np.arange(M) * step - 20 * step + float(rng.choice([0.0, 3.0]))).astype(np.float32)
        P = (rng.random((M, N)) * 1e6).astype(np.float32)
        b, o = int(rng.integers(0, M)), int(rng.integers(0, N))
        P[b, o] = P[max(b - 1, 0):b + 2, o].max() * np.float32(1.0 + rng.random())
        ix = np.array([b, o], np.int32)
        want = R.fine_dop(P, N, fds, (b, o))
        got = _lib.lib.sdr_fine_dop(C.c_void_p(P.ctypes.data), N, C.c_void_p(fds.ctypes.data), M,
                                    C.c_void_p(ix.ctypes.data))
        assert abs(got - want) <= 1e-9 * max(abs(want), 1.0), (b, o, got, want)


@pytest.mark.skipif(not oracle.track_run_available(), reason="tracking driver (oracle/_ref) absent")
def test_track_driver_matches_reference_calls():
    """The tracking baseline's C driver runs the same reference calls as the
    Python-level Reference.mix_carr + corr_std, result for result."""
    from pocketsdr_b200 import synth
    wl = synth.track_24mhz(seed=5)
    jobs = wl.jobs_at(0.0, [0] * len(wl.channels))[:24]
    chans = [c for c in wl.channels if abs(round(0.0 / c.T) * c.T) < 1e-9]
    for s, c in zip(jobs, chans):
        s["ch"] = wl.channels.index(c)
    banks = synth.track_banks(wl)
    corr = oracle.TrackRun(wl.bufs, jobs, banks).run(4)
    R = oracle.Reference()
    for k, s in enumerate(jobs):
        IQ = R.mix_carr(wl.bufs[s["buf"]], s["ix"], s["N"], s["fs"], s["fc"], s["phi"])
        c, _ = R.corr_std(IQ, banks[s["ch"]], s["coff"], s["pos"], False)
        assert np.array_equal(c, corr[k, :len(c)])

