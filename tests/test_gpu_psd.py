"""Welch PSD on the GPU (sdr_psd_cpx, sdrg_psd, sdrg_psd_if) against the
reference build's sdr_psd_cpx: within 1e-3 dB per bin (FP32 transforms of
noise-like IF data), real and complex data, FFT sizes that split over 1, 2,
4 and 8 CTAs, and the receiver's packed-buffer window with a wrap."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_DB = 1e-3


def _iq(rng, n, IQ):
    return (rng.integers(-7, 8, n) + 1j * rng.integers(-7, 8, n) * (IQ == 2)).astype(np.complex64)


@pytest.mark.parametrize("N,IQ,n", [(4096, 2, 4096 * 40 + 5), (4096, 1, 4096 * 12),
                                    (48000, 2, 48000 * 4), (65536, 1, 65536 * 3),
                                    (131072, 2, 131072 * 2), (3072, 2, 3072 * 100)])
def test_drop_in_psd_matches_reference(ref, gpu, N, IQ, n):
    rng = np.random.default_rng(N + IQ)
    x = _iq(rng, n, IQ)
    want = ref.psd_cpx(x, N, 24e6, IQ)
    got = gpu.psd(x, N, 24e6, IQ)
    assert got.shape == want.shape
    assert np.max(np.abs(got - want)) <= TOL_DB, np.max(np.abs(got - want))


def test_psd_short_data_is_nan_like_reference(ref, gpu):
    x = _iq(np.random.default_rng(1), 100, 2)
    assert np.all(np.isnan(gpu.psd(x, 1024, 24e6, 2))) and np.all(np.isnan(ref.psd_cpx(x, 1024, 24e6, 2)))


def test_psd_from_packed_if_buffer(ref, gpu):
    """sdrg_psd_if on a circular cpx8 buffer (window wrapping the end) equals
    the reference's PSD of the same samples unpacked to floats, as
    sdr_rcv_rfch_psd does (src/sdr_rcv.c:401-407)."""
    import ctypes as C
    torch = pytest.importorskip("torch")
    from pocketsdr_b200._lib import lib
    rng = np.random.default_rng(7)
    L, N, n, ix = 200000, 8192, 8192 * 20, 150000
    buf = rng.integers(0, 256, L, dtype=np.uint8)
    idx = (ix + np.arange(n)) % L
    b = buf[idx]
    x = (((b << 4).astype(np.int8) >> 4) + 1j * (b.astype(np.int8) >> 4)).astype(np.complex64)
    want = ref.psd_cpx(x, N, 16e6, 2)
    d = torch.from_numpy(buf).cuda()
    out = torch.empty(N, dtype=torch.float32, device="cuda")
    st = lib.sdrg_psd_if(C.c_void_p(d.data_ptr()), L, ix, n, N, 16e6, 2,
                         C.c_void_p(out.data_ptr()), None)
    assert st == 0
    torch.cuda.synchronize()
    assert np.max(np.abs(out.cpu().numpy() - want)) <= TOL_DB
