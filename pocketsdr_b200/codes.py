"""Spreading-code replicas and conjugated code DFTs for acquisition plans.

* GPS L1 C/A codes come from the standard G1/G2 10-stage LFSRs with the
  per-PRN G2 delays of the GPS interface specification (IS-GPS-200, table
  3-Ia) - the same definition the reference implements in
  src/sdr_code.c:771-824.
* For the other signals of the benchmark configurations (Galileo E1-B,
  BeiDou B1I, GPS L5-I/Q, QZSS L6D) this module provides STAND-IN codes: seeded
  +-1 sequences with the signal's code length, period and chip rate (E1-B
  with its BOC(1,1) sub-carrier, L6D time-multiplexed with zeros). Search cost
  does not depend on the chip values, and every parity test feeds the same
  replica to the GPU and to the oracle.
* res_code / gen_code_fft restate src/sdr_code.c:2556-2608 (nearest-chip
  resampling by (int)((coff*fs + i)*dx) % len_code); the DFT here is numpy's
  float64 FFT, rounded to complex64.
"""
from __future__ import annotations

import numpy as np

# IS-GPS-200 table 3-Ia: G2 delay (chips) for PRN 1-32
_L1CA_G2_DELAY = [5, 6, 7, 8, 17, 18, 139, 140, 141, 251, 252, 254, 255, 256, 257, 258,
                  469, 470, 471, 472, 473, 474, 509, 512, 513, 514, 515, 516, 859, 860,
                  861, 862]

# code length (chips per period after sub-carrier modulation), period (s)
SIGNALS = {
    "L1CA": (1023, 1e-3),
    "E1B": (4092 * 2, 4e-3),      # BOC(1,1): two half-chips per chip
    "B1I": (2046, 1e-3),
    "L5I": (10230, 1e-3),
    "L5Q": (10230, 1e-3),
    "L6D": (10230 * 2, 4e-3),     # time-multiplexed with L6E: every other chip 0
}
PRN_SETS = {
    "L1CA": range(1, 33), "E1B": range(1, 37), "B1I": range(1, 64),
    "L5I": range(1, 33), "L5Q": range(1, 33), "L6D": range(193, 203),
}


def _lfsr10(taps, n):
    """10-stage Fibonacci LFSR, all-ones start; output = stage 10; taps are
    1-based stage numbers XORed into stage 1."""
    reg = [1] * 10
    out = np.empty(n, np.int8)
    for i in range(n):
        out[i] = reg[9]
        fb = 0
        for t in taps:
            fb ^= reg[t - 1]
        reg = [fb] + reg[:9]
    return out


_G1 = None
_G2 = None


def gen_code_L1CA(prn: int) -> np.ndarray:
    global _G1, _G2
    if not 1 <= prn <= 32:
        raise ValueError("L1CA PRN 1-32")
    if _G1 is None:
        _G1 = _lfsr10([3, 10], 1023)
        _G2 = _lfsr10([2, 3, 6, 8, 9, 10], 1023)
    d = _L1CA_G2_DELAY[prn - 1]
    g2 = np.roll(_G2, d)
    bits = _G1 ^ g2
    return (1 - 2 * bits).astype(np.int8)       # 0 -> +1, 1 -> -1


def _standin(sig: str, prn: int) -> np.ndarray:
    n, _ = SIGNALS[sig]
    rng = np.random.default_rng(sum(map(ord, sig)) * 1000 + prn)
    if sig == "E1B":
        chips = rng.choice(np.array([-1, 1], np.int8), n // 2)
        return np.repeat(chips, 2) * np.tile(np.array([1, -1], np.int8), n // 2)
    if sig == "L6D":
        chips = rng.choice(np.array([-1, 1], np.int8), n // 2)
        out = np.zeros(n, np.int8)
        out[0::2] = chips
        return out
    return rng.choice(np.array([-1, 1], np.int8), n)


def gen_code(sig: str, prn: int) -> np.ndarray:
    """+-1 (or 0) chips of one code period."""
    if sig == "L1CA":
        return gen_code_L1CA(prn)
    if sig not in SIGNALS:
        raise ValueError(f"unknown signal {sig}")
    return _standin(sig, prn)


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
