"""Batched search (sdrg_search_batch) against the reference receiver's own
per-channel search: for every request, search_sig (src/sdr_ch.c:398-450)
replayed with the reference build - sdr_search_code accumulated over the
code periods from ix, sdr_corr_max, the threshold decision, sdr_fine_dop and
the code offset - on the same IF bytes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _reference_search(ref, chips, T, fs, fi, N, fds, buf, ix, t_acq, thres):
    cf = ref.gen_code_fft(chips, None, T, 0.0, fs, N, N)
    P = np.zeros((len(fds), 2 * N), np.float32)
    n_sum = 0
    while True:
        ref.search_code(cf, buf, (ix + n_sum * N) % len(buf), 2 * N, fs, fi, fds, P, T)
        n_sum += 1
        if n_sum * T >= t_acq:
            break
    cn0, pk = ref.corr_max(P, 2 * N, N, len(fds), T)
    fd = ref.fine_dop(P, 2 * N, fds, pk)
    return dict(found=cn0 >= thres, bin=pk[0], offset=pk[1], cn0=cn0, fd=fd, coff=pk[1] / fs,
                n_sum=n_sum)


def test_search_batch_matches_reference_search_sig(ref, gpu):
    torch = pytest.importorskip("torch")
    from pocketsdr_b200 import codes, schedule, synth
    fs, fi, T = 12e6, 3.0e6, 1e-3
    N = int(fs * T)
    sats = [synth.Sat("L1CA", 4, 321.7, 1730.0, 0.1, 47.0),
            synth.Sat("L1CA", 9, 12.25, -2210.0, 0.6, 44.0),
            synth.Sat("L1CA", 17, 800.5, 330.0, 0.3, 41.0)]
    buf = synth.gen_if(16 * N, fs, {"L1CA": fi}, sats, iq=False, bits=2, seed=12)
    prns = [1, 4, 9, 17, 23, 30]
    chips = np.stack([codes.gen_code("L1CA", p) for p in prns])
    setups = [schedule.Setup(chips, T, fs, fi, max_dop=5000.0)]
    reqs = [schedule.Request(0, k) for k in range(len(prns))]
    reqs += [schedule.Request(0, 2, fd_ext=float(np.float32(-2210.0 + 180.0))),          # PRN 9
             schedule.Request(0, 3, fd_ext=float(np.float32(330.0 - 410.0)), fd_ext_n=7),  # PRN 17
             schedule.Request(0, 5, fd_ext=float(np.float32(1500.0)))]                    # absent
    ix, t_acq, thres = 2 * N + 77, 4e-3, 38.0
    got = schedule.search(setups, reqs, [torch.from_numpy(buf).cuda()], ix, t_acq, thres)
    full = np.asarray(ref.dop_bins(T, 0.0, 5000.0), np.float32)
    for i, r in enumerate(reqs):
        if r.fd_ext != 0.0:
            nw = r.fd_ext_n or 3
            fds = np.array([r.fd_ext + (k - nw // 2) * 0.5 / T for k in range(nw)]).astype(np.float32)
        else:
            fds = full
        w = _reference_search(ref, chips[r.prn], T, fs, fi, N, fds, buf, ix, t_acq, thres)
        g = got[i]
        assert bool(g["found"]) == w["found"], i
        assert (g["bin"], g["offset"]) == (w["bin"], w["offset"]), (i, g, w)
        assert abs(g["cn0"] - w["cn0"]) < 0.1 and g["n_sum"] == w["n_sum"], i
        assert abs(g["fd"] - w["fd"]) < 0.5 and g["coff"] == w["coff"], (i, g["fd"], w["fd"])
    assert got["found"][1] and got["found"][2]      # PRN 4 (47 dB-Hz) and 9 (44 dB-Hz)


def test_search_batch_reuses_plan_with_new_codes(ref, gpu):
    """Back-to-back calls with the same group structure reuse the cached plan
    but search the new requests' codes; a call with another structure (and
    sdrg_search_release) starts afresh - every result equals the reference's
    search_sig replay."""
    torch = pytest.importorskip("torch")
    from pocketsdr_b200 import codes, schedule, synth
    from pocketsdr_b200._lib import lib
    fs, fi, T = 12e6, 3.0e6, 1e-3
    N = int(fs * T)
    sats = [synth.Sat("L1CA", 6, 100.5, 900.0, 0.3, 46.0),
            synth.Sat("L1CA", 21, 700.25, -1500.0, 0.7, 45.0)]
    buf = synth.gen_if(12 * N, fs, {"L1CA": fi}, sats, iq=False, bits=2, seed=31)
    prns = list(range(1, 33))
    chips = np.stack([codes.gen_code("L1CA", p) for p in prns])
    setups = [schedule.Setup(chips, T, fs, fi, max_dop=5000.0)]
    d = torch.from_numpy(buf).cuda()
    full = np.asarray(ref.dop_bins(T, 0.0, 5000.0), np.float32)
    t_acq, thres, ix = 3e-3, 38.0, 1000
    for rows in ([0, 2, 4], [5, 20, 9], [5, 20], [1, 6, 11, 20]):
        reqs = [schedule.Request(0, r) for r in rows]
        got = schedule.search(setups, reqs, [d], ix, t_acq, thres)
        for i, r in enumerate(rows):
            w = _reference_search(ref, chips[r], T, fs, fi, N, full, buf, ix, t_acq, thres)
            assert (got[i]["bin"], got[i]["offset"]) == (w["bin"], w["offset"]), (rows, r)
            assert bool(got[i]["found"]) == w["found"] and abs(got[i]["cn0"] - w["cn0"]) < 0.1
    lib.sdrg_search_release()
