"""sdrg_corr_fft_noalloc: the FFT correlator for callers that cannot call
cudaMalloc - a real-time receiver channel thread that must not stall on the
device synchronisation an allocation may bring, or an application whose device
memory all comes from its own pool. It keeps every intermediate in one fixed
device array, so this test owns the input and output buffers (torch tensors)
and checks the entry point through the C ABI against the oracle's corr_fft
(the reference's sdr_corr_fft, src/sdr_func.c:1088-1102) and against the
library's allocating sdr_corr_fft, on calls in a row whose lengths alternate
(each call must rebuild the tables it reads in the shared array), within the
FFT-correlator tolerance of the other parity tests. Collected last on purpose
(file name), so a failure here comes after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CPLX_RTOL = 1e-4   # same bar as tests/test_gpu_parity.py


def _close(c, ref):
    rms = float(np.sqrt(np.mean(np.abs(ref) ** 2)))
    err = np.abs(c.astype(np.complex128) - ref)
    return bool(np.all(err <= CPLX_RTOL * np.maximum(np.abs(ref), rms)))


def _noalloc(lib, torch, IQ, cf, stream):
    N = IQ.shape[0]
    d_iq = torch.from_numpy(np.ascontiguousarray(IQ)).cuda()
    d_cf = torch.from_numpy(np.ascontiguousarray(cf).view(np.float32)).cuda()
    d_out = torch.zeros(2 * N, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rc = lib.sdrg_corr_fft_noalloc(C.c_void_p(d_iq.data_ptr()), C.c_void_p(d_cf.data_ptr()), N,
                                   C.c_void_p(d_out.data_ptr()), C.c_void_p(stream))
    torch.cuda.synchronize()
    return rc, d_out.cpu().numpy().view(np.complex64)


def test_corr_fft_noalloc_matches_oracle_and_allocating_entry():
    torch = pytest.importorskip("torch")
    from oracle import oracle
    from pocketsdr_b200 import sdr_func
    from pocketsdr_b200._lib import lib, torch_stream
    sdr_func.init()
    R = oracle.best()
    stream = torch_stream()
    rng = np.random.default_rng(2024)
    # calls in a row: a length, the same length with new data, another
    # length, back to the first (the shared array holds the previous call's
    # tables and data each time)
    for N in (48000, 48000, 4000, 48000, 65536, 6000):
        IQ = rng.integers(-100, 101, (N, 2), dtype=np.int8)
        cf = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
        rc, got = _noalloc(lib, torch, IQ, cf, stream)
        assert rc == 0, (N, rc)
        assert _close(got, R.corr_fft(IQ, cf)), N
        assert _close(got, sdr_func.sdr_corr_fft(IQ, cf)), N


def test_corr_fft_noalloc_ignores_schedules():
    """A schedule that sends a length to a staged split (R > 8) applies to
    sdr_corr_fft, not to this entry, which keeps the default cluster split."""
    torch = pytest.importorskip("torch")
    from oracle import oracle
    from pocketsdr_b200 import sdr_func
    from pocketsdr_b200._lib import lib, torch_stream
    sdr_func.init()
    R = oracle.best()
    N = 48000
    assert lib.sdrg_fft_schedule_set(N, 10, 256) == 0
    try:
        rng = np.random.default_rng(7)
        IQ = rng.integers(-100, 101, (N, 2), dtype=np.int8)
        cf = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
        rc, got = _noalloc(lib, torch, IQ, cf, torch_stream())
        assert rc == 0
        assert _close(got, R.corr_fft(IQ, cf))
    finally:
        lib.sdrg_fft_schedule_set(N, 0, 0)


def test_corr_fft_noalloc_rejects_oversize():
    torch = pytest.importorskip("torch")
    from pocketsdr_b200._lib import lib, last_error
    t = torch.zeros(16, dtype=torch.float32, device="cuda")
    p = C.c_void_p(t.data_ptr())
    rc = lib.sdrg_corr_fft_noalloc(p, p, 65536 * 2, p, None)
    assert rc == -1
    assert "outside" in last_error()[1]
    lib.sdr_gpu_clear_error()
