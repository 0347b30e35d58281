"""FFT schedules, host side (no device work): set / get / save / load of a
length's split and CTA size, rejection of shapes the library cannot run, and
the file format - schedule lines only, so the reference's FFTW wisdom file
(which sdr_func_init(file) also receives) loads nothing."""
import os

import pytest

from pocketsdr_b200._lib import lib


def _get(L):
    import ctypes as C
    R, t = C.c_int(-1), C.c_int(-1)
    ok = lib.sdrg_fft_schedule_get(L, C.byref(R), C.byref(t))
    return (R.value, t.value) if ok else None


def test_set_get_clear():
    assert lib.sdrg_fft_schedule_set(48000, 4, 256) == 0
    assert _get(48000) == (4, 256)
    assert lib.sdrg_fft_schedule_set(48000, 0, 0) == 0
    assert _get(48000) is None


@pytest.mark.parametrize("L,R,t", [(48000, 7, 256), (48000, 1, 512), (48000, 2, 300),
                                   (1000003, 1, 256), (-5, 1, 256)])
def test_invalid_schedules_rejected(L, R, t):
    assert lib.sdrg_fft_schedule_set(L, R, t) == -1
    lib.sdr_gpu_clear_error()
    assert _get(L) is None


def test_save_load_roundtrip(tmp_path):
    p = str(tmp_path / "sched.txt")
    for L, R, t in ((48000, 2, 512), (192000, 8, 512), (96000, 4, 256)):
        assert lib.sdrg_fft_schedule_set(L, R, t) == 0
    assert lib.sdrg_fft_schedule_save(p.encode()) == 0
    text = open(p).read()
    assert "sdrg_fft 96000 4 256" in text
    for L in (48000, 192000, 96000):
        lib.sdrg_fft_schedule_set(L, 0, 0)
    assert lib.sdrg_fft_schedule_load(p.encode()) == 3
    assert _get(96000) == (4, 256) and _get(192000) == (8, 512)
    for L in (48000, 192000, 96000):
        lib.sdrg_fft_schedule_set(L, 0, 0)


def test_wisdom_file_loads_nothing(tmp_path):
    p = tmp_path / "fftw_wisdom.txt"
    p.write_text("(fftw-3.3.10 fftwf_wisdom #x7f2a #x1 #x2 #x3\n  (fftwf_codelet_n1_64 0 #x10bdd))\n")
    assert lib.sdrg_fft_schedule_load(str(p).encode()) == 0


def test_bad_entries_are_reported(tmp_path):
    p = tmp_path / "bad.txt"
    p.write_text("sdrg_fft 48000 7 256 0.1\nsdrg_fft 24000 1 512 0.2\n")
    assert lib.sdrg_fft_schedule_load(str(p).encode()) == -1
    lib.sdr_gpu_clear_error()
    assert _get(24000) == (1, 512)
    lib.sdrg_fft_schedule_set(24000, 0, 0)
