"""Spreading-code replicas on the GPU (sdrg_res_code / sdrg_gen_code_fft /
sdrg_acq_set_codes C ABI).

The receiver builds its replicas on the CPU: one FFT per PRN for acquisition
(sdr_gen_code_fft in acq_new, src/sdr_ch.c:192-201) and SDR_N_CODES resampled
banks per tracking channel (sdr_res_code in trk_new, src/sdr_ch.c:265-272).
These functions do the same for many codes at once on the device, from chips
(int8 +-1 / 0, codes.gen_code) to device tensors:

* res_code: bit-identical to sdr_res_code per (code, bank);
* gen_code_fft: sdr_gen_code_fft's conjugated DFT (FP32, natural order);
* AcqPlan.set_codes (acquire.py) writes the same DFTs straight into an
  acquisition plan.

All calls are asynchronous on torch's current CUDA stream.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib, torch_stream

SDR_N_CODES = 10


def _torch():
    import torch
    return torch


def device_chips(chips):
    """int8 [n_code, len_code] CUDA tensor from a (list of) numpy / torch array(s)."""
    torch = _torch()
    if isinstance(chips, torch.Tensor):
        t = chips
    else:
        a = np.asarray(chips if not isinstance(chips, (list, tuple)) else np.stack(chips), np.int8)
        t = torch.from_numpy(np.ascontiguousarray(a))
    if t.dim() == 1:
        t = t.unsqueeze(0)
    return t.to(device="cuda", dtype=torch.int8).contiguous()


def _stream() -> C.c_void_p:
    return C.c_void_p(torch_stream())


def res_code(chips, T: float, coff: float, fs: float, N: int, Nz: int = 0,
             n_bank: int = 1, code_Q=None):
    """Resampled replicas: int8 CUDA tensor [n_code, n_bank, N + Nz, 2] with
    bank b = sdr_res_code(code, coff - b / fs / n_bank). n_bank = SDR_N_CODES
    and coff = 0 give a tracking channel's code banks."""
    torch = _torch()
    ci = device_chips(chips)
    cq = device_chips(code_Q) if code_Q is not None else None
    if cq is not None and cq.shape != ci.shape:
        raise ValueError("code_Q must have the shape of chips")
    n_code, len_code = ci.shape
    out = torch.empty((n_code, n_bank, N + Nz, 2), dtype=torch.int8, device="cuda")
    st = lib.sdrg_res_code(C.c_void_p(ci.data_ptr()),
                           C.c_void_p(cq.data_ptr()) if cq is not None else None,
                           len_code, n_code, T, coff, fs, N, Nz, n_bank,
                           C.c_void_p(out.data_ptr()), _stream())
    if st:
        check("sdrg_res_code")
    return out


def gen_code_fft(chips, T: float, coff: float, fs: float, N: int, Nz: int = 0, code_Q=None):
    """Conjugated code DFTs: complex64 CUDA tensor [n_code, N + Nz], each equal
    to sdr_gen_code_fft(code, ..., coff, fs, N, Nz)."""
    torch = _torch()
    ci = device_chips(chips)
    cq = device_chips(code_Q) if code_Q is not None else None
    if cq is not None and cq.shape != ci.shape:
        raise ValueError("code_Q must have the shape of chips")
    n_code, len_code = ci.shape
    out = torch.empty((n_code, N + Nz), dtype=torch.complex64, device="cuda")
    st = lib.sdrg_gen_code_fft(C.c_void_p(ci.data_ptr()),
                               C.c_void_p(cq.data_ptr()) if cq is not None else None,
                               len_code, n_code, T, coff, fs, N, Nz,
                               C.c_void_p(out.data_ptr()), _stream())
    if st:
        check("sdrg_gen_code_fft")
    return out


def set_plan_codes(handle, g: int, chips, T: float, coff: float, N: int, code_Q=None) -> None:
    """Group g of an acquisition plan takes the DFTs of these chips (one code
    per PRN of the group, in the group's PRN order): an N-sample replica zero
    padded to the group's FFT length."""
    ci = device_chips(chips)
    cq = device_chips(code_Q) if code_Q is not None else None
    n_code, len_code = ci.shape
    st = lib.sdrg_acq_set_codes(C.c_void_p(handle), g, C.c_void_p(ci.data_ptr()),
                                C.c_void_p(cq.data_ptr()) if cq is not None else None,
                                len_code, T, coff, N, _stream())
    if st:
        check("sdrg_acq_set_codes")
