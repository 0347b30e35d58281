"""sdrg_mix_carr (carrier wipe-off on a device-resident circular IF buffer)
against the reference build's sdr_mix_carr (src/sdr_func.c:824-836), bit for
bit: aligned and unaligned windows, windows that wrap the buffer end, and
lengths that are not multiples of the 16-sample vector width."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("len_buf,ix,N", [
    (96000, 0, 96000), (96000, 16, 48000), (100003, 5, 50001), (96000, 95000, 30000),
    (100003, 99990, 100003), (64, 3, 61), (1 << 22, 1 << 20, 3 << 20)])
def test_mix_carr_device_matches_reference(ref, gpu, len_buf, ix, N):
    import torch
    from pocketsdr_b200._lib import lib, torch_stream
    rng = np.random.default_rng(len_buf + ix + N)
    buf = rng.integers(0, 256, len_buf, dtype=np.uint8)
    fs, fc, phi = 24e6, float(rng.uniform(-6e6, 6e6)), float(rng.uniform(-1.0, 1.0))
    want = ref.mix_carr(buf, ix, N, fs, fc, phi)
    d_buf = torch.from_numpy(buf).cuda()
    d_out = torch.zeros(2 * N, dtype=torch.int8, device="cuda")
    st = lib.sdrg_mix_carr(C.c_void_p(d_buf.data_ptr()), len_buf, ix, N, fs, fc, phi,
                           C.c_void_p(d_out.data_ptr()), C.c_void_p(torch_stream()))
    assert st == 0
    got = d_out.cpu().numpy().reshape(N, 2)
    assert np.array_equal(got, want)


def test_mix_carr_device_every_alignment(ref, gpu):
    """Every offset of the window start within a 16-byte block, with the
    buffer itself starting at each of 4 byte offsets from an aligned address
    (the kernel realigns 16-byte blocks), windows wrapping the buffer end."""
    import torch
    from pocketsdr_b200._lib import lib, torch_stream
    rng = np.random.default_rng(77)
    len_buf, N = 4099, 4000
    for off in range(4):
        buf = rng.integers(0, 256, len_buf, dtype=np.uint8)
        d_all = torch.from_numpy(np.concatenate([np.zeros(off, np.uint8), buf])).cuda()
        for ix in list(range(0, 33)) + [len_buf - 40, len_buf - 1]:
            fs, fc, phi = 24e6, float(rng.uniform(-6e6, 6e6)), float(rng.uniform(-1.0, 1.0))
            want = ref.mix_carr(buf, ix, N, fs, fc, phi)
            d_out = torch.zeros(2 * N, dtype=torch.int8, device="cuda")
            st = lib.sdrg_mix_carr(C.c_void_p(d_all.data_ptr() + off), len_buf, ix, N, fs, fc,
                                   phi, C.c_void_p(d_out.data_ptr()), C.c_void_p(torch_stream()))
            assert st == 0
            got = d_out.cpu().numpy().reshape(N, 2)
            assert np.array_equal(got, want), (off, ix)


def test_mix_carr_device_unaligned_output(ref, gpu):
    """An output array that does not start on a 16-byte boundary takes the
    sample-by-sample path; the result is the same."""
    import torch
    from pocketsdr_b200._lib import lib, torch_stream
    rng = np.random.default_rng(91)
    len_buf, ix, N = 50000, 333, 40000
    buf = rng.integers(0, 256, len_buf, dtype=np.uint8)
    want = ref.mix_carr(buf, ix, N, 24e6, 3.1e6, 0.7)
    d_buf = torch.from_numpy(buf).cuda()
    d_out = torch.zeros(2 * N + 16, dtype=torch.int8, device="cuda")
    for off in (2, 6):
        st = lib.sdrg_mix_carr(C.c_void_p(d_buf.data_ptr()), len_buf, ix, N, 24e6, 3.1e6, 0.7,
                               C.c_void_p(d_out.data_ptr() + off), C.c_void_p(torch_stream()))
        assert st == 0
        got = d_out.cpu().numpy()[off:off + 2 * N].reshape(N, 2)
        assert np.array_equal(got, want), off


def test_mix_carr_device_rejects_bad_window(gpu):
    from pocketsdr_b200._lib import lib, last_error
    p = C.c_void_p(1)
    assert lib.sdrg_mix_carr(p, 100, 100, 10, 1.0, 0.0, 0.0, p, None) == -1
    assert "bad window" in last_error()[1]
    lib.sdr_gpu_clear_error()
