"""Link test: the reference's own programs relinked against the GPU library.

oracle/Makefile (target `linktest`) builds, from the reference sources,
* test/src/test_sdr_{func,code,ch}.c, the reference's unit tests of
  sdr_func.c, sdr_code.c and sdr_ch.c, and
* app/pocket_acq/pocket_acq.c, its acquisition app,
twice: `*_gpu` with the hot symbols of sdr_func.o / sdr_code.o renamed `*_cpu`
(objcopy) so that the calls resolve to libsdr_gpu.so, and `*_cpu` from the
unmodified objects. The GPU-linked unit tests must pass all of their tests;
the GPU-linked pocket_acq, run on 20 ms of the reference's own L1 sample
(sample/L1_20211125_004000_12MHz_I.bin as INT8, reconstructed from the
committed fixture), must print the same code offsets and Doppler for the
detected satellites as the CPU build and C/N0 within 0.1 dB for every PRN.
The binaries exist where the reference sources were present at build time.
"""
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "..", "oracle", "_ref")


def _bin(name):
    p = os.path.join(REF, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} not built (reference sources absent at build time)")
    return p


def _undefined(path):
    out = subprocess.run(["nm", "-u", path], capture_output=True, text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if ln.strip()}


UNIT = [  # (program, tests it runs, hot functions it reaches)
    ("test_sdr_func", 14, ("sdr_mix_carr", "sdr_corr_std", "sdr_corr_fft", "sdr_search_code",
                           "sdr_psd_cpx", "sdr_lpf_apply")),
    ("test_sdr_code", 7, ("sdr_res_code", "sdr_gen_code_fft")),
    # the channel: search (sdr_search_code via search_sig) and tracking
    # (sdr_mix_carr + sdr_corr_std via the correlator of a locked channel)
    ("test_sdr_ch", 7, ("sdr_search_code", "sdr_mix_carr", "sdr_corr_std")),
]


@pytest.mark.parametrize("prog,n_tests,hot", UNIT)
def test_reference_unit_tests_through_gpu_library(tmp_path, prog, n_tests, hot):
    exe = _bin(prog + "_gpu")
    # the hot functions are not in the executable: they come from libsdr_gpu.so
    und = _undefined(exe)
    for s in hot:
        assert s in und, s
    r = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    oks = [ln for ln in r.stdout.splitlines() if ln.endswith(" ... OK")]
    assert len(oks) == n_tests, r.stdout


_LINE = re.compile(r"SIG= (\S+)\s*, PRN=\s*(\d+), COFF=\s*([-\d.]+) ms, DOP=\s*([-\d]+) Hz, "
                   r"C/N0=\s*([-\d.]+) dB-Hz")


def _acq(exe, path):
    r = subprocess.run([exe, "-sig", "L1CA", "-prn", "1-32", "-tint", "19", "-fmt", "INT8",
                        "-f", "12", "-fi", "3", path], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    out = {}
    for ln in r.stdout.splitlines():
        m = _LINE.search(ln)
        if m:
            out[int(m.group(2))] = (m.group(3), int(m.group(4)), float(m.group(5)))
    return out


def test_pocket_acq_through_gpu_library(tmp_path, golden):
    gpu_exe, cpu_exe = _bin("pocket_acq_gpu"), _bin("pocket_acq_cpu")
    assert {"sdr_search_code", "sdr_gen_code_fft", "sdr_corr_max"} <= _undefined(gpu_exe)
    # 20 ms at 12 MHz: the fixture holds the low nibble of each INT8 sample
    # (values -3, -1, 1, 3), as the reference's sdr_read_data packs it
    nib = golden("real_l1ca.npz")["buf"].astype(np.int16)
    path = str(tmp_path / "L1_12MHz_I.bin")
    ((nib ^ 8) - 8).astype(np.int8).tofile(path)
    got, want = _acq(gpu_exe, path), _acq(cpu_exe, path)
    assert sorted(got) == list(range(1, 33)) and sorted(want) == list(range(1, 33))
    detected = [p for p, w in want.items() if w[2] >= 38.0]
    assert detected == [2, 5, 11, 13, 15, 18, 20, 29, 30]
    for prn, (coff, dop, cn0) in want.items():
        g = got[prn]
        assert abs(g[2] - cn0) <= 0.1 + 1e-9, (prn, g, (coff, dop, cn0))
        if prn in detected:
            assert g[0] == coff, (prn, g, (coff, dop, cn0))
            assert abs(g[1] - dop) <= 1, (prn, g, (coff, dop, cn0))
