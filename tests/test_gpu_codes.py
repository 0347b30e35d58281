"""Replicas on the GPU against the reference build (the oracle restatement
when the reference build is absent): nearest-chip resampled banks
(sdr_res_code, src/sdr_code.c:2556-2568) bit-exact, conjugated code DFTs
(sdr_gen_code_fft, src/sdr_code.c:2589-2608) within 1e-4 of the largest
|value|, and an acquisition plan whose codes are computed on the device
against one given the reference's host DFTs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-4   # complex outputs: |d| <= TOL * max(|ref|, rms ref) per element


def _close(got, ref, tol=TOL):
    got = np.asarray(got)
    floor = max(float(np.sqrt(np.mean(np.abs(ref) ** 2))), 1e-30)
    err = np.abs(got - ref)
    bound = tol * np.maximum(np.abs(ref), floor)
    return bool(np.all(err <= bound)), float((err / np.maximum(np.abs(ref), floor)).max())


CASES = [  # (signal, fs, T, Nz)
    ("L1CA", 12e6, 1e-3, 0),
    ("L1CA", 24e6, 1e-3, 24000),
    ("E1B", 24e6, 4e-3, 0),
    ("B1I", 24e6, 1e-3, 0),
    ("L5I", 24e6, 1e-3, 0),
    ("L1CA", 2.046e6 * 1.5, 1e-3, 5),      # odd row length: scalar stores
]


@pytest.mark.parametrize("sig,fs,T,Nz", CASES)
def test_res_code_banks_bit_exact(ref, gpu, sig, fs, T, Nz):
    from pocketsdr_b200 import codes, replica
    prns = list(codes.PRN_SETS[sig])[:3]
    chips = np.stack([codes.gen_code(sig, p) for p in prns])
    N = int(fs * T)
    got = replica.res_code(chips, T, 0.0, fs, N, Nz, n_bank=replica.SDR_N_CODES).cpu().numpy()
    for c in range(len(prns)):
        for b in range(replica.SDR_N_CODES):
            want = ref.res_code(chips[c], None, T, -b / fs / replica.SDR_N_CODES, fs, N, Nz)
            assert np.array_equal(got[c, b], want), (sig, c, b)


def test_res_code_complex_and_offsets(ref, gpu):
    """Complex (I != Q) codes, positive code offsets, a single bank."""
    from pocketsdr_b200 import replica
    rng = np.random.default_rng(4)
    ci = rng.choice(np.array([-1, 1], np.int8), (2, 10230))
    cq = rng.choice(np.array([-1, 0, 1], np.int8), (2, 10230))
    fs, T, N = 20e6, 1e-3, 20000
    for coff in (0.0, 3.3e-7, 0.4e-3, 0.99e-3):
        got = replica.res_code(ci, T, coff, fs, N, 17, code_Q=cq).cpu().numpy()
        for c in range(2):
            assert np.array_equal(got[c, 0], ref.res_code(ci[c], cq[c], T, coff, fs, N, 17)), coff


def test_drop_in_res_code(ref, gpu):
    from pocketsdr_b200 import codes
    from pocketsdr_b200._lib import lib, ptr
    c = codes.gen_code("L1CA", 17)
    fs, T, N = 24e6, 1e-3, 24000
    for b in range(10):
        out = np.zeros((N + 100, 2), np.int8)
        lib.sdr_res_code(ptr(c), None, len(c), T, -b / fs / 10, fs, N, 100, ptr(out))
        assert np.array_equal(out, ref.res_code(c, None, T, -b / fs / 10, fs, N, 100)), b


FFT_CASES = [  # (signal, fs, T, N, Nz, tile): L = N + Nz exercises each split kind
    ("L1CA", 4e6, 1e-3, 4000, 0, 1),            # R = 1
    ("L1CA", 24e6, 1e-3, 24000, 24000, 1),      # R = 2 (receiver zero padding)
    ("L1CA", 12e6, 4e-3, 48000, 0, 4),          # R = 2, tiled code
    ("E1B", 24e6, 4e-3, 96000, 96000, 1),       # R = 8 cluster
    ("L1CA", 24e6, 10e-3, 240000, 0, 10),       # R = 10 staged
    ("B1I", 16e6, 1e-3, 16000, 0, 1),           # R = 1, another length
]


@pytest.mark.parametrize("sig,fs,T,N,Nz,tile", FFT_CASES)
def test_gen_code_fft_matches_reference(ref, gpu, sig, fs, T, N, Nz, tile):
    from pocketsdr_b200 import codes, replica
    prns = list(codes.PRN_SETS[sig])[:2]
    chips = np.stack([np.tile(codes.gen_code(sig, p), tile) for p in prns])
    got = replica.gen_code_fft(chips, T, 0.0, fs, N, Nz).cpu().numpy()
    for c in range(len(prns)):
        want = ref.gen_code_fft(chips[c], None, T, 0.0, fs, N, Nz)
        ok, worst = _close(got[c], want)
        assert ok, (sig, N, Nz, c, worst)


def test_gen_code_fft_complex_code_and_offset(ref, gpu):
    from pocketsdr_b200 import replica
    rng = np.random.default_rng(8)
    ci = rng.choice(np.array([-1, 1], np.int8), (1, 2046))
    cq = rng.choice(np.array([-1, 1], np.int8), (1, 2046))
    fs, T, N = 12e6, 1e-3, 12000
    got = replica.gen_code_fft(ci, T, 1.7e-4, fs, N, N, code_Q=cq).cpu().numpy()[0]
    ok, worst = _close(got, ref.gen_code_fft(ci[0], cq[0], T, 1.7e-4, fs, N, N))
    assert ok, worst


def test_drop_in_gen_code_fft(ref, gpu):
    from pocketsdr_b200 import codes
    from pocketsdr_b200._lib import lib, ptr
    c = codes.gen_code("L1CA", 5)
    fs, T, N = 12e6, 1e-3, 12000
    out = np.zeros(2 * N, np.complex64)
    lib.sdr_gen_code_fft(ptr(c), None, len(c), T, 0.0, fs, N, N, ptr(out))
    ok, worst = _close(out, ref.gen_code_fft(c, None, T, 0.0, fs, N, N))
    assert ok, worst


def test_bad_arguments_are_errors(gpu):
    """A code offset indexing before the code and an FFT length without a
    plan are rejected with a status (no kernel runs)."""
    import ctypes as C
    torch = pytest.importorskip("torch")
    from pocketsdr_b200 import _lib
    ci = torch.ones(1023, dtype=torch.int8, device="cuda")
    out = torch.empty(2 * 24000 * 2, dtype=torch.int8, device="cuda")
    st = _lib.lib.sdrg_res_code(C.c_void_p(ci.data_ptr()), None, 1023, 1, 1e-3, -1e-4, 24e6,
                                24000, 0, 1, C.c_void_p(out.data_ptr()), None)
    assert st == -1
    _lib.lib.sdr_gpu_clear_error()
    fo = torch.empty(7 * 11 * 13 * 2, dtype=torch.float32, device="cuda")
    st = _lib.lib.sdrg_gen_code_fft(C.c_void_p(ci.data_ptr()), None, 1023, 1, 1e-3, 0.0, 1.001e6,
                                    7 * 11 * 13, 0, C.c_void_p(fo.data_ptr()), None)
    assert st == -1
    _lib.lib.sdr_gpu_clear_error()


def test_plan_codes_from_device_chips(ref, gpu):
    """A multi-signal plan created without host DFTs and filled by
    sdrg_acq_set_codes gives the grid and peaks of the same plan built from
    the reference's sdr_gen_code_fft outputs."""
    torch = pytest.importorskip("torch")
    from pocketsdr_b200 import acquire, codes, synth
    wl = synth.acq_multi_24mhz(seed=3, prn_limit=4, t_sum=2e-3)
    host_cf = []
    for g in wl.groups:
        host_cf.append(np.stack([ref.gen_code_fft(codes.gen_code(g.sig, p), None, g.T, 0.0,
                                                  g.fs, g.N, g.L - g.N) for p in g.prns]))
    pa = acquire.AcqPlan(wl.groups, host_cf)
    pb = acquire.AcqPlan(wl.groups, [None] * len(wl.groups))
    for i, g in enumerate(wl.groups):
        pb.set_codes(i, np.stack([codes.gen_code(g.sig, p) for p in g.prns]), g.T)
    torch.cuda.synchronize()
    ra = pa.run_host(wl.bufs, wl.ix)
    rb = pb.run_host(wl.bufs, wl.ix)
    for i in range(len(wl.groups)):
        ga, gb = pa.grid(i), pb.grid(i)
        floor = float(ga.mean())
        assert np.all(np.abs(gb - ga) <= TOL * np.maximum(np.abs(ga), floor)), i
    assert np.array_equal(ra["bin"], rb["bin"]) and np.array_equal(ra["offset"], rb["offset"])
    assert np.all(np.abs(ra["cn0"] - rb["cn0"]) < 0.1)


def test_drop_in_empty_replica_is_zero_padding(ref, gpu):
    """N = 0: the reference fills the N + Nz outputs with zeros (no error)."""
    from pocketsdr_b200 import codes
    from pocketsdr_b200._lib import last_error, lib, ptr
    lib.sdr_gpu_clear_error()
    c = codes.gen_code("L1CA", 3)
    a = np.full((16, 2), 9, np.int8)
    lib.sdr_res_code(ptr(c), None, len(c), 1e-3, 0.0, 4e6, 0, 16, ptr(a))
    assert np.array_equal(a, ref.res_code(c, None, 1e-3, 0.0, 4e6, 0, 16))
    f = np.full(16, 9, np.complex64)
    lib.sdr_gen_code_fft(ptr(c), None, len(c), 1e-3, 0.0, 4e6, 0, 16, ptr(f))
    assert not f.any() and not ref.gen_code_fft(c, None, 1e-3, 0.0, 4e6, 0, 16).any()
    assert last_error()[0] == 0
