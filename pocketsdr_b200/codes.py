"""Spreading-code chips, replicas and conjugated code DFTs.

* Chips come from the library's generators (``sdrg_gen_code`` /
  ``sdrg_sec_code`` in libsdr_gpu.so, host code): GPS L1 C/A, L5-I/Q, QZSS
  L6D/L6E, Galileo E1-B (BOC(1,1)) and BeiDou B1I, the same chips as the
  reference's sdr_gen_code / sdr_sec_code (src/sdr_code.c:2173-2182,
  :2274-2283), secondary codes included.
* res_code / gen_code_fft restate src/sdr_code.c:2556-2608 (nearest-chip
  resampling by (int)((coff*fs + i)*dx) % len_code); the DFT here is numpy's
  float64 FFT, rounded to complex64 (the device versions are in replica.py).
"""
from __future__ import annotations

import ctypes as C
import functools

import numpy as np

from . import _lib

# code length (values per period, sub-carrier or time multiplex included),
# period (s)
SIGNALS = {
    "L1CA": (1023, 1e-3),
    "E1B": (4092 * 2, 4e-3),      # BOC(1,1): two half-chips per chip
    "B1I": (2046, 1e-3),
    "L5I": (10230, 1e-3),
    "L5Q": (10230, 1e-3),
    "L6D": (10230 * 2, 4e-3),     # time-multiplexed with L6E: every other chip 0
    "L6E": (10230 * 2, 4e-3),
}
PRN_SETS = {
    "L1CA": range(1, 33), "E1B": range(1, 37), "B1I": range(1, 64),
    "L5I": range(1, 33), "L5Q": range(1, 33), "L6D": range(193, 203),
    "L6E": range(203, 213),
}


def _call(fn, sig: str, prn: int) -> np.ndarray:
    n = fn(sig.encode(), prn, None, 0)
    if n <= 0:
        _lib.check(f"{fn.__name__}({sig}, {prn})")
        raise ValueError(f"no code for {sig} PRN {prn}")
    out = np.empty(n, np.int8)
    if fn(sig.encode(), prn, C.c_void_p(out.ctypes.data), n) != n:
        _lib.check(f"{fn.__name__}({sig}, {prn})")
    return out


@functools.lru_cache(maxsize=None)
def _gen(sig: str, prn: int) -> bytes:
    return _call(_lib.lib.sdrg_gen_code, sig, prn).tobytes()


def gen_code(sig: str, prn: int) -> np.ndarray:
    """Chips of one primary code period: +1 / -1, 0 in the off slots of a
    time-multiplexed code (sdr_gen_code)."""
    return np.frombuffer(_gen(sig.upper(), prn), np.int8).copy()


def gen_code_L1CA(prn: int) -> np.ndarray:
    if not 1 <= prn <= 210:
        raise ValueError("L1CA PRN 1-210")
    return gen_code("L1CA", prn)


def sec_code(sig: str, prn: int) -> np.ndarray:
    """Secondary (overlay) code, one chip per primary period (sdr_sec_code)."""
    return _call(_lib.lib.sdrg_sec_code, sig.upper(), prn)


def code_cyc(sig: str) -> float:
    return SIGNALS[sig][1]


def res_code(code_I, T, coff, fs, N, Nz=0, code_Q=None) -> np.ndarray:
    """Nearest-chip resampled replica as int8 [N+Nz, 2] (I, Q), zero padded
    (src/sdr_code.c:2556-2568)."""
    code_I = np.asarray(code_I, np.int8)
    L = len(code_I)
    dx = L / T / fs
    j = (((coff * fs + np.arange(N, dtype=np.float64)) * dx).astype(np.int64)) % L
    out = np.zeros((N + Nz, 2), np.int8)
    out[:N, 0] = code_I[j]
    out[:N, 1] = (np.asarray(code_Q, np.int8)[j] if code_Q is not None else code_I[j])
    return out


def gen_code_fft(code_I, T, coff, fs, N, Nz=0, code_Q=None) -> np.ndarray:
    """Conjugated DFT of the resampled, zero-padded replica (complex64[N+Nz]);
    the replica's Q part is 0 for a real code (src/sdr_code.c:2589-2608)."""
    code_I = np.asarray(code_I, np.int8)
    L = len(code_I)
    dx = L / T / fs
    j = (((coff * fs + np.arange(N, dtype=np.float64)) * dx).astype(np.int64)) % L
    x = np.zeros(N + Nz, np.complex128)
    x[:N] = code_I[j]
    if code_Q is not None:
        x[:N] += 1j * np.asarray(code_Q, np.int8)[j]
    return np.conj(np.fft.fft(x)).astype(np.complex64)
