"""GPU mirror of the hot-path functions of Pocket SDR's python/sdr_func.py.

Same names, arguments and return values as the reference module
(python/sdr_func.py:119-184), executed by libsdr_gpu.so:

  search_code(code_fft, T, buff, ix, fs, fi, fds) -> P      (:119-126)
  corr_max(P, T) -> (P_max, ix, cn0)                        (:129-134)
  fine_dop(P, fds, ix) -> fd                                (:137-141)
  shift_freq(sig, fcn, fi) -> fi                            (:144-149)
  dop_bins(T, dop, max_dop) -> fds                          (:152-153)
  corr_std(buff, ix, N, fs, fc, phi, code, pos) -> corr     (:156-171)
  corr_fft(buff, ix, N, fs, fc, phi, code_fft) -> corr      (:174-187)
  mix_carr(buff, ix, N, fs, fc, phi) -> int8 [N, 2]
  psd(data, N, fs, IQ) -> float32 [N/2 or N] (dB/Hz)          (:215-223)

`buff` is the complex64 IF array of the reference's Python layer. Like the
reference's C-library path (LIBSDR_ENA), samples are cast to int8 and packed
4+4 bits before mixing with the quantised carrier table, so results follow
the C library (the reference's numpy-only fallback mixes in float and differs
by a few percent of the peak, test/python/sdr_func_c_test.py:52-127).

The C-level drop-ins are exposed with their reference names too (sdr_*).
"""
from __future__ import annotations

import ctypes as C
from math import log10

import numpy as np

from ._lib import SdrBuff, check, lib, ptr

DOP_STEP = 0.5   # python/sdr_func.py:49



def init() -> None:
    """sdr_func_init(): selects the GPU and builds the carrier table (every
    entry point also initialises lazily)."""
    lib.sdr_func_init(b"")
    check("sdr_func_init")


# ---- reference python API -------------------------------------------------
def corr_fft(buff, ix, N, fs, fc, phi, code_fft):
    buff = np.ascontiguousarray(buff, np.complex64)
    code_fft = np.ascontiguousarray(code_fft, np.complex64)
    corr = np.empty(N, np.complex64)
    lib.sdr_corr_fft_cpx(ptr(buff), len(buff), int(ix), int(N), float(fs), float(fc),
                         float(phi), ptr(code_fft), ptr(corr))
    check("sdr_corr_fft_cpx")
    return corr


def corr_std(buff, ix, N, fs, fc, phi, code, pos):
    buff = np.ascontiguousarray(buff, np.complex64)
    code_real = np.ascontiguousarray(np.real(code), np.float32)
    pos = np.ascontiguousarray(pos, np.float64)
    corr = np.empty(len(pos), np.complex64)
    lib.sdr_corr_std_cpx(ptr(buff), len(buff), int(ix), int(N), float(fs), float(fc),
                         float(phi), ptr(code_real), ptr(pos), len(pos), ptr(corr))
    check("sdr_corr_std_cpx")
    return corr


def search_code(code_fft, T, buff, ix, fs, fi, fds):
    N = int(fs * T)
    P = np.zeros((len(fds), N), dtype="float32")
    for i in range(len(fds)):
        C_ = corr_fft(buff, ix, len(code_fft), fs, fi + fds[i], 0.0, code_fft)[:N]
        P[i] = np.abs(C_) ** 2
    return P


def psd(data, N, fs, IQ):
    """Welch PSD of IF data (sdr_psd_cpx): N/2 bins for IQ = 1, N for IQ = 2."""
    data = np.ascontiguousarray(data, np.complex64)
    out = np.zeros(N if IQ == 2 else N // 2, np.float32)
    lib.sdr_psd_cpx(ptr(data), len(data), int(N), float(fs), int(IQ), ptr(out))
    check("sdr_psd_cpx")
    return out


def corr_max(P, T):
    P = np.ascontiguousarray(P, np.float32)
    ix = np.zeros(2, np.int32)
    M, N = P.shape
    cn0 = lib.sdr_corr_max(ptr(P), N, N, M, float(T), ptr(ix))
    check("sdr_corr_max")
    return P[ix[0], ix[1]], (int(ix[0]), int(ix[1])), float(cn0)


def fine_dop(P, fds, ix):
    if ix == 0 or ix == len(fds) - 1:
        return fds[ix]
    x0, x1, x2 = (float(v) for v in fds[ix - 1:ix + 2])
    y0, y1, y2 = (float(v) for v in P[ix - 1:ix + 2])
    d01 = (y1 - y0) / (x1 - x0)
    d12 = (y2 - y1) / (x2 - x1)
    c = (d12 - d01) / (x2 - x0)
    b = d01 - c * (x0 + x1)
    return -b / (2.0 * c)


def shift_freq(sig, fcn, fi):
    if sig == "G1CA":
        fi += 0.5625e6 * fcn
    elif sig == "G2CA":
        fi += 0.4375e6 * fcn
    return fi


def dop_bins(T, dop, max_dop):
    return np.arange(dop - max_dop, dop + max_dop + DOP_STEP / T, DOP_STEP / T)


def mix_carr(buff, ix, N, fs, fc, phi):
    """Carrier wipe-off of the complex64 buffer through the C-library
    semantics (int8 cast, 4+4-bit pack, quantised carrier); int8 [N, 2]."""
    packed = pack_cpx8(np.asarray(buff)[(ix + np.arange(N)) % len(buff)])
    return sdr_mix_carr(packed, 0, N, fs, fc, phi)


def pack_cpx8(x) -> np.ndarray:
    """complex -> 4+4-bit packed bytes, as SDR_CPX8((int8)re, (int8)im)."""
    x = np.asarray(x, np.complex64)
    re = np.trunc(x.real).astype(np.int32).astype(np.int8)
    im = np.trunc(x.imag).astype(np.int32).astype(np.int8)
    return (((im.astype(np.uint8) & 0x0F) << 4) | (re.astype(np.uint8) & 0x0F)).astype(np.uint8)


# ---- C-level drop-ins -------------------------------------------------------
def _buff(data: np.ndarray):
    d = np.ascontiguousarray(data, np.uint8)
    return d, SdrBuff(d.ctypes.data_as(C.POINTER(C.c_uint8)), 2, len(d))


def sdr_mix_carr(buff_u8, ix, N, fs, fc, phi):
    d, sb = _buff(buff_u8)
    out = np.zeros((N, 2), np.int8)
    lib.sdr_mix_carr(C.byref(sb), int(ix), int(N), float(fs), float(fc), float(phi), ptr(out))
    check("sdr_mix_carr")
    return out


def sdr_corr_std(IQ, code, coff, pos, cpx_code=False):
    IQ = np.ascontiguousarray(IQ, np.int8)
    code = np.ascontiguousarray(code, np.int8)
    pos = np.ascontiguousarray(pos, np.float64)
    corr = np.zeros(len(pos), np.complex64)
    Cb = np.zeros(2, np.complex64)
    fn = lib.sdr_corr_std_cpx_code if cpx_code else lib.sdr_corr_std
    fn(ptr(IQ), ptr(code), IQ.shape[0], float(coff), ptr(pos), len(pos), ptr(corr), ptr(Cb))
    check("sdr_corr_std")
    return corr, Cb


def sdr_corr_fft(IQ, code_fft):
    IQ = np.ascontiguousarray(IQ, np.int8)
    code_fft = np.ascontiguousarray(code_fft, np.complex64)
    out = np.zeros(IQ.shape[0], np.complex64)
    lib.sdr_corr_fft(ptr(IQ), ptr(code_fft), IQ.shape[0], ptr(out))
    check("sdr_corr_fft")
    return out


def sdr_search_code(code_fft, T, buff_u8, ix, N, fs, fi, fds, P):
    code_fft = np.ascontiguousarray(code_fft, np.complex64)
    fds = np.ascontiguousarray(fds, np.float32)
    assert P.dtype == np.float32 and P.flags.c_contiguous and P.size >= len(fds) * N
    d, sb = _buff(buff_u8)
    lib.sdr_search_code(ptr(code_fft), float(T), C.byref(sb), int(ix), int(N), float(fs),
                        float(fi), ptr(fds), len(fds), ptr(P))
    check("sdr_search_code")
    return P


def sdr_corr_max(P, N, Nmax, M, T):
    P = np.ascontiguousarray(P, np.float32)
    ix = np.full(2, -1, np.int32)
    cn0 = lib.sdr_corr_max(ptr(P), int(N), int(Nmax), int(M), float(T), ptr(ix))
    check("sdr_corr_max")
    return float(cn0), (int(ix[0]), int(ix[1]))


def sdr_fine_dop(P, N, fds, ix):
    P = np.ascontiguousarray(P, np.float32)
    fds = np.ascontiguousarray(fds, np.float32)
    ixa = np.asarray(ix, np.int32)
    return float(lib.sdr_fine_dop(ptr(P), int(N), ptr(fds), len(fds), ptr(ixa)))


def sdr_dop_bins(T, dop, max_dop):
    n = C.c_int(0)
    p = lib.sdr_dop_bins(float(T), float(dop), float(max_dop), C.byref(n))
    out = np.ctypeslib.as_array(p, shape=(n.value,)).copy()
    C.CDLL(None).free(C.cast(p, C.c_void_p))
    return out
