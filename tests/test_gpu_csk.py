"""QZSS L6 CSK tracking on the GPU (sdrg_csk_decode, sdrg_l6_csk_batch)
against the reference channel's own CSK decoder (src/sdr_ch.c:626-664,
through oracle/ch_shim.c; the restatement when that build is absent) and its
sdr_mix_carr + sdr_corr_fft chain (reference build):
* decode alone on the reference's correlations: symbols and taps bit-identical;
* the whole batch: correlations within 1e-4 of the largest |value|, the same
  symbols, taps within 1e-4 of the largest tap."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-4


@pytest.fixture(scope="module")
def ch():
    from oracle import oracle
    return oracle.Channel() if os.path.exists(oracle.CH_SO) else oracle.Restatement()


def _l6_setup(ref, seed=3):
    """24 MHz complex IF with four L6D signals, each keyed
    by its own code shift, and the channels that track them."""
    from pocketsdr_b200 import codes, synth
    fs, fi, T = 24e6, 2.0e6, 4e-3
    N = int(fs * T)
    Lc = codes.SIGNALS["L6D"][0]
    rng = np.random.default_rng(seed)
    prns = [193, 195, 199, 202]
    shifts = [17, 200, 0, 255]
    sats = [synth.Sat("L6D", p, 2.0 * k + 0.25, float(rng.uniform(-3000, 3000)), 0.1 * i, 50.0)
            for i, (p, k) in enumerate(zip(prns, shifts))]
    buf = synth.gen_if(3 * N + 1000, fs, {"L6D": fi}, sats, iq=True, bits=3, seed=seed)
    sc = N / (Lc / 2)
    pos = np.array([0.0, -0.5 * sc, 0.5 * sc, -120.0] + list(np.arange(-4, 5) * 0.25 * sc))
    jobs = []
    for i, s in enumerate(sats):
        j = i % 10                                     # the channel's code bank
        chips = codes.gen_code("L6D", s.prn)
        cf = ref.gen_code_fft(chips, None, T, -j / fs / 10, fs, N, 0)
        ix = (i * 7919 + (2 * N + 900 if i == 3 else 0)) % len(buf)   # job 3 wraps
        jobs.append(dict(buf=0, ix=ix, N=N, fs=fs, fc=fi + s.doppler, phi=0.37 * i,
                         code_fft=cf, len_code=Lc, pos=pos))
    return buf, jobs


def _reference_chain(ref, ch, buf, jb):
    IQ = ref.mix_carr(buf, jb["ix"], jb["N"], jb["fs"], jb["fc"], jb["phi"])
    corr = ref.corr_fft(IQ, jb["code_fft"])
    sym, C = ch.csk(corr, jb["len_code"], jb["pos"])
    return corr, sym, C


def test_csk_decode_bit_exact(ref, ch, gpu):
    import ctypes as Cc
    torch = pytest.importorskip("torch")
    from pocketsdr_b200._lib import lib
    buf, jobs = _l6_setup(ref)
    corrs, want = [], []
    rng = np.random.default_rng(1)
    for jb in jobs:
        corr, sym, C = _reference_chain(ref, ch, buf, jb)
        corrs.append(corr)
        want.append((sym, C))
    # plus pure noise (no clear symbol) and an all-zero correlation
    N = jobs[0]["N"]
    corrs.append((rng.normal(size=N) + 1j * rng.normal(size=N)).astype(np.complex64))
    corrs.append(np.zeros(N, np.complex64))
    pos = jobs[0]["pos"]
    for c in corrs[len(jobs):]:
        want.append(ch.csk(c, jobs[0]["len_code"], pos))
    cd = torch.from_numpy(np.stack(corrs)).cuda()
    sym = torch.zeros(len(corrs), dtype=torch.uint8, device="cuda")
    C = torch.zeros((len(corrs), 107), dtype=torch.complex64, device="cuda")
    pos_np = np.ascontiguousarray(pos, np.float64)
    st = lib.sdrg_csk_decode(Cc.c_void_p(cd.data_ptr()), len(corrs), N, jobs[0]["len_code"],
                             Cc.c_void_p(pos_np.ctypes.data), len(pos_np),
                             Cc.c_void_p(sym.data_ptr()), Cc.c_void_p(C.data_ptr()), None)
    assert st == 0
    torch.cuda.synchronize()
    sym, C = sym.cpu().numpy(), C.cpu().numpy()
    for j, (ws, wC) in enumerate(want):
        assert int(sym[j]) == ws, (j, int(sym[j]), ws)
        assert np.array_equal(C[j, :len(pos)].view(np.uint32), wC.view(np.uint32)), j


def test_l6_batch_matches_reference_chain(ref, ch, gpu):
    torch = pytest.importorskip("torch")
    from pocketsdr_b200 import track
    buf, jobs = _l6_setup(ref, seed=8)
    specs = [dict(jb, code_fft=torch.from_numpy(jb["code_fft"]).cuda()) for jb in jobs]
    d = torch.from_numpy(buf).cuda()
    sym, taps, corr = track.l6_csk_batch(specs, [d.data_ptr()], [len(buf)])
    torch.cuda.synchronize()
    sym, taps, corr = sym.cpu().numpy(), taps.cpu().numpy(), corr.cpu().numpy()
    for j, jb in enumerate(jobs):
        wcorr, wsym, wC = _reference_chain(ref, ch, buf, jb)
        scale = np.abs(wcorr).max()
        assert np.abs(corr[j, :jb["N"]] - wcorr).max() <= TOL * scale, j
        assert int(sym[j]) == wsym, (j, int(sym[j]), wsym)
        assert np.abs(taps[j, :len(jb["pos"])] - wC).max() <= TOL * np.abs(wC).max(), j


def test_l6_batch_mixed_lengths_job_by_job(ref, ch, gpu):
    """Jobs of different lengths take the job-by-job path: same results."""
    torch = pytest.importorskip("torch")
    from pocketsdr_b200 import codes, track
    buf, jobs = _l6_setup(ref, seed=11)
    fs, T2 = jobs[0]["fs"], 2e-3                      # a half-period window of 48 000
    N2 = int(fs * T2)
    chips = codes.gen_code("L6D", 196)
    # P, E, L only: at this length the noise tap (-120 samples) would fall
    # before the +-280-chip window, which the library rejects
    extra = dict(jobs[1], N=N2, ix=12345, code_fft=ref.gen_code_fft(chips, None, T2, 0.0, fs, N2, 0),
                 pos=jobs[1]["pos"][:3])
    alljobs = jobs[:2] + [extra]
    specs = [dict(jb, code_fft=torch.from_numpy(jb["code_fft"]).cuda()) for jb in alljobs]
    d = torch.from_numpy(buf).cuda()
    sym, taps, corr = track.l6_csk_batch(specs, [d.data_ptr()], [len(buf)])
    torch.cuda.synchronize()
    sym, taps, corr = sym.cpu().numpy(), taps.cpu().numpy(), corr.cpu().numpy()
    for j, jb in enumerate(alljobs):
        wcorr, wsym, wC = _reference_chain(ref, ch, buf, jb)
        assert np.abs(corr[j, :jb["N"]] - wcorr).max() <= TOL * np.abs(wcorr).max(), j
        assert int(sym[j]) == wsym, j
        assert np.abs(taps[j, :len(jb["pos"])] - wC).max() <= TOL * np.abs(wC).max(), j
