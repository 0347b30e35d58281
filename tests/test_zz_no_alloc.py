"""sdrg_corr_fft_noalloc: the FFT correlator for callers that cannot allocate
device memory when they call (inside a stream capture, on a real-time receiver
thread that must not stall on cudaMalloc's device synchronisation, or with
device memory from their own pool). It keeps every intermediate in one fixed
device array, so this test owns the input and output buffers (torch tensors)
and checks the entry point through the C ABI against the allocating
sdr_corr_fft on two calls in a row, within the FFT-correlator tolerance of the
other parity tests. Collected last on purpose (file name), so a failure here
comes after every other test has run.
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


def test_corr_fft_noalloc_matches_allocating_entry():
    torch = pytest.importorskip("torch")
    from pocketsdr_b200 import sdr_func
    from pocketsdr_b200._lib import lib, torch_stream
    sdr_func.init()
    stream = torch_stream()
    rng = np.random.default_rng(2024)
    # two calls in a row: a new length (tables uploaded), then the same length
    # with new data (array contents of the previous call left behind)
    for N in (48000, 48000, 4000):
        IQ = rng.integers(-100, 101, (N, 2), dtype=np.int8)
        cf = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
        expected = sdr_func.sdr_corr_fft(IQ, cf)
        rc, got = _noalloc(lib, torch, IQ, cf, stream)
        assert rc == 0, rc
        assert _close(got, expected), N


def test_corr_fft_noalloc_rejects_oversize():
    torch = pytest.importorskip("torch")
    from pocketsdr_b200._lib import lib, last_error
    t = torch.zeros(16, dtype=torch.float32, device="cuda")
    p = C.c_void_p(t.data_ptr())
    rc = lib.sdrg_corr_fft_noalloc(p, p, 65536 * 2, p, None)
    assert rc == -1
    assert "outside" in last_error()[1]
    lib.sdr_gpu_clear_error()
