"""The drop-ins called at once from many host threads, as the reference's
receiver calls them (one pthread per channel, src/sdr_rcv.c:495-520, each
running sdr_mix_carr + sdr_corr_std per code period, src/sdr_ch.c:725-733):
every thread's results are bit-identical to the oracle for mixing and the
correlators and within 1e-4 for the FFT correlator. ctypes releases the
interpreter lock during the calls, so the threads overlap inside the
library (one CUDA stream and staging area per thread)."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-4


def test_dropins_from_concurrent_channel_threads(gpu, orc):
    rng = np.random.default_rng(55)
    n_thr, n_ep, fs = 12, 6, 12e6
    sizes = [4000, 6000, 8000, 12000, 16000, 24000]
    cases = []
    for t in range(n_thr):
        N = sizes[t % len(sizes)]
        eps = []
        for _ in range(n_ep):
            n = int(rng.integers(3, 45))
            eps.append(dict(ix=int(rng.integers(0, 3 * N)), fc=float(rng.uniform(-3e6, 3e6)),
                            phi=float(rng.uniform(-1, 1)), coff=float(rng.uniform(0, N)),
                            pos=np.concatenate([[0.0, -1.5, 1.5], rng.uniform(-N, N, n - 3)])))
        cases.append(dict(N=N, buf=rng.integers(0, 256, 3 * N, dtype=np.uint8),
                          bank=np.repeat(rng.choice(np.array([-1, 1], np.int8), (10 * N, 1)), 2, 1),
                          cf=(rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64),
                          eps=eps))
    results, errors = [None] * n_thr, []
    start = threading.Barrier(n_thr)

    def channel(t):
        try:
            c = cases[t]
            out = []
            start.wait()
            for e in c["eps"]:
                IQ = gpu.sdr_mix_carr(c["buf"], e["ix"], c["N"], fs, e["fc"], e["phi"])
                corr, Cb = gpu.sdr_corr_std(IQ, c["bank"], e["coff"], e["pos"])
                out.append((IQ, corr, Cb, gpu.sdr_corr_fft(IQ, c["cf"])))
            results[t] = out
        except BaseException as ex:         # surfaced in the test thread
            errors.append(ex)

    threads = [threading.Thread(target=channel, args=(t,)) for t in range(n_thr)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    assert not errors, errors
    for t, c in enumerate(cases):
        for k, (e, (IQ, corr, Cb, cf)) in enumerate(zip(c["eps"], results[t])):
            want = orc.mix_carr(c["buf"], e["ix"], c["N"], fs, e["fc"], e["phi"])
            assert np.array_equal(IQ, want), (t, k)
            rc, rC = orc.corr_std(want, c["bank"], e["coff"], e["pos"], False)
            assert np.array_equal(corr.view(np.uint32), rc.view(np.uint32)), (t, k)
            assert np.array_equal(Cb.view(np.uint32), rC.view(np.uint32)), (t, k)
            rf = orc.corr_fft(want, c["cf"])
            assert np.abs(cf - rf).max() <= TOL * np.abs(rf).max(), (t, k)
