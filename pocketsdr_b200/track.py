"""Batched tracking correlators on the GPU (sdrg_corr_batch C ABI).

One job is the per-channel, per-code-period work of the reference's tracking
loop (src/sdr_ch.c:725-733): carrier wipe-off of the channel's IF window
(sdr_mix_carr) and the multi-tap standard correlator (sdr_corr_std, or
sdr_corr_std_cpx_code for complex codes) against the channel's resampled code
bank. A batch runs every channel of an epoch in three launches; outputs are
bit-identical to the reference's two calls per channel.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib, torch_stream

SDR_N_CODES = 10
SDR_MAX_CORR = 107


class CorrJob(C.Structure):
    """sdrg_corr_job_t."""
    _fields_ = [("buf", C.c_int), ("ix", C.c_int), ("N", C.c_int),
                ("fs", C.c_double), ("fc", C.c_double), ("phi", C.c_double),
                ("coff", C.c_double), ("code", C.c_void_p), ("cpx_code", C.c_int),
                ("n", C.c_int), ("pos", C.POINTER(C.c_double))]


lib.sdrg_corr_batch.argtypes = [C.POINTER(CorrJob), C.c_int, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_void_p, C.c_void_p]
lib.sdrg_corr_batch.restype = C.c_int


def make_jobs(specs) -> tuple:
    """specs: iterable of dicts with keys buf, ix, N, fs, fc, phi, coff,
    code_ptr (device pointer of the bank), cpx_code, pos (sequence of floats).
    Returns (ctypes job array, keep-alive list)."""
    specs = list(specs)
    arr = (CorrJob * len(specs))()
    keep = []
    for j, s in zip(arr, specs):
        pos = np.ascontiguousarray(s["pos"], np.float64)
        keep.append(pos)
        j.buf, j.ix, j.N = int(s["buf"]), int(s["ix"]), int(s["N"])
        j.fs, j.fc, j.phi, j.coff = float(s["fs"]), float(s["fc"]), float(s["phi"]), float(s["coff"])
        j.code = C.c_void_p(int(s["code_ptr"]))
        j.cpx_code = int(bool(s.get("cpx_code", False)))
        j.n = len(pos)
        j.pos = pos.ctypes.data_as(C.POINTER(C.c_double))
    return arr, keep


def corr_batch(jobs, if_ptrs, lens, corr_ptr: int, C_ptr: int = 0, stream: int = 0) -> None:
    """Asynchronous batch on device buffers: jobs from make_jobs; if_ptrs /
    lens: device IF buffers; corr_ptr: [n_job][107] complex64 device buffer;
    C_ptr: [n_job][2] complex64 device buffer or 0."""
    arr, _ = jobs if isinstance(jobs, tuple) else (jobs, None)
    n = len(if_ptrs)
    ptrs = (C.c_void_p * n)(*if_ptrs)
    ls = (C.c_int * n)(*lens)
    st = lib.sdrg_corr_batch(arr, len(arr), ptrs, ls, C.c_void_p(corr_ptr),
                             C.c_void_p(C_ptr or None), C.c_void_p(stream or None))
    if st:
        check("sdrg_corr_batch")


def code_bank(code, T, fs, N, code_Q=None) -> np.ndarray:
    """The receiver's fractional-phase code bank (src/sdr_ch.c:265-272):
    bank k is the code resampled with offset -k / fs / SDR_N_CODES, as
    int8 [SDR_N_CODES * N, 2]."""
    from .codes import res_code
    banks = [res_code(code, T, -k / fs / SDR_N_CODES, fs, N, 0, code_Q) for k in range(SDR_N_CODES)]
    return np.concatenate(banks)


class L6Batch:
    """One epoch of QZSS L6 channels prepared for sdrg_l6_csk_batch: the job
    array and pointer arguments are built once, run() makes the call. specs
    are dicts with buf, ix, N, fs, fc, phi, code_fft (CUDA complex64 tensor:
    the bank's conjugated code DFT), len_code, pos. Results go to CUDA tensors
    (symbols uint8 [n], taps complex64 [n, SDR_MAX_CORR], correlations
    complex64 [n, max N]), the given `out` triple or new ones."""

    def __init__(self, specs, if_ptrs, lens, out=None):
        import torch
        from ._lib import L6Job
        specs = list(specs)
        self.n = n = len(specs)
        self.arr = arr = (L6Job * n)()
        self._keep = []
        for j, s in zip(arr, specs):
            pos = np.ascontiguousarray(s["pos"], np.float64)
            self._keep += [pos, s["code_fft"]]
            j.buf, j.ix, j.N = int(s["buf"]), int(s["ix"]), int(s["N"])
            j.fs, j.fc, j.phi = float(s["fs"]), float(s["fc"]), float(s["phi"])
            j.code_fft = C.c_void_p(s["code_fft"].data_ptr())
            j.len_code, j.n = int(s["len_code"]), len(pos)
            j.pos = pos.ctypes.data_as(C.POINTER(C.c_double))
        nmax = max(int(s["N"]) for s in specs)
        if out is None:
            out = (torch.empty(n, dtype=torch.uint8, device="cuda"),
                   torch.empty((n, SDR_MAX_CORR), dtype=torch.complex64, device="cuda"),
                   torch.empty((n, nmax), dtype=torch.complex64, device="cuda"))
        self.out = out
        self._args = ((C.c_void_p * len(if_ptrs))(*if_ptrs), (C.c_int * len(if_ptrs))(*lens),
                      C.c_void_p(out[0].data_ptr()), C.c_void_p(out[1].data_ptr()),
                      C.c_void_p(out[2].data_ptr()))

    def run(self, stream: int = 0):
        """Asynchronous on `stream` (0: torch's current stream)."""
        if not stream:
            stream = torch_stream()
        ptrs, ls, sym, taps, corr = self._args
        if lib.sdrg_l6_csk_batch(self.arr, self.n, ptrs, ls, sym, taps, corr, C.c_void_p(stream)):
            check("sdrg_l6_csk_batch")
        return self.out


def l6_csk_batch(specs, if_ptrs, lens, stream: int = 0, out=None):
    """QZSS L6 channels of one epoch (sdrg_l6_csk_batch); see L6Batch for the
    specs. Returns the CUDA tensors (symbols, taps, correlations), written
    into `out` when given; asynchronous."""
    return L6Batch(specs, if_ptrs, lens, out).run(stream)
