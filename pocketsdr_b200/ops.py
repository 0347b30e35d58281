"""PyTorch operators over the C ABI (torch.library custom ops).

The batched search and the tracking correlators as operators on CUDA tensors,
run on torch's current stream, so they compose with other torch work
(streams, CUDA graphs of the caller, shape inference through the fake
implementations):

* ``torch.ops.pocketsdr.search`` - parallel-code-phase search of one signal
  group: for every PRN the non-coherent grid of sdr_search_code over n_sum
  code periods, its peak and C/N0 (sdr_corr_max) and fine Doppler
  (sdr_fine_dop) - src/sdr_func.c:641-744, the receiver's search_sig
  (src/sdr_ch.c:398-450) for all PRNs at once.
* ``torch.ops.pocketsdr.corr_batch`` - the tracking correlators of many
  channels on one IF buffer: sdr_mix_carr then sdr_corr_std per channel
  (src/sdr_ch.c:725-733), bit-exact.

Importing this module registers the operators; the library must be built.
"""
import threading
from types import SimpleNamespace
from typing import List, Tuple

import numpy as np
import torch

from . import acquire, track
from ._lib import torch_stream

_plans: dict = {}
_plans_lock = threading.Lock()


def _plan(n_prn: int, fds: List[float], fs: float, fi: float, T: float, N: int, Nz: int,
          n_sum: int) -> acquire.AcqPlan:
    """One cached acquisition plan per search shape (its grid and spectra
    stay allocated for the next call of the same shape)."""
    key = (n_prn, tuple(float(f) for f in fds), fs, fi, T, N, Nz, n_sum)
    with _plans_lock:
        pl = _plans.get(key)
        if pl is None:
            g = SimpleNamespace(sig="", prns=list(range(n_prn)), fs=fs, fi=fi, T=T, N=N,
                                L=N + Nz, Nmax=N, n_sum=n_sum,
                                fds=np.asarray(fds, np.float32), buf=0)
            pl = acquire.AcqPlan([g], [None])
            _plans[key] = pl
        return pl


def _device_view(ptr: int, shape, typestr: str) -> torch.Tensor:
    """A tensor over device memory the library owns (no copy)."""
    class _View:
        __cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                    "data": (int(ptr), False), "version": 3}
    return torch.as_tensor(_View(), device="cuda")


@torch.library.custom_op("pocketsdr::search", mutates_args=())
def search(buf: torch.Tensor, ix: int, chips: torch.Tensor, fds: List[float], fs: float,
           fi: float, T: float, N: int, Nz: int, n_sum: int
           ) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor]:
    """buf: uint8 CUDA [len] packed IF samples (circular, as sdr_buff_t data);
    ix: first sample of sum 0 (sum s starts at ix + s N); chips: int8 CUDA
    [n_prn, len_code], one spreading code per PRN with code period T; N
    samples per period, zero padded by Nz (the receiver uses Nz = N); fds:
    Doppler bins (Hz). Returns grid float32 [n_prn, n_bin, N] (the
    accumulated correlation power of the N code offsets), bin int32 [n_prn],
    offset int32 [n_prn], cn0 float32 [n_prn] (dB-Hz) and fd float64 [n_prn]
    (Hz, the peak bin refined by the three-bin fit). Calls of the same shape
    share one cached plan (its grid and spectra): issue them on one stream."""
    if not (buf.is_cuda and chips.is_cuda):
        raise ValueError("pocketsdr::search takes CUDA tensors")
    buf = buf.contiguous()
    n_prn = int(chips.shape[0])
    pl = _plan(n_prn, fds, fs, fi, T, N, Nz, n_sum)
    pl.set_codes(0, chips, T)
    res = torch.empty(n_prn * acquire.RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    pl.run_device([buf.data_ptr()], [buf.numel()], [ix], res.data_ptr(),
                  torch_stream())
    grid = _device_view(pl.grid_ptr(0), (n_prn, len(fds), N), "<f4").clone()
    r32 = res.view(torch.int32).view(n_prn, 8)
    rf = res.view(torch.float32).view(n_prn, 8)
    rd = res.view(torch.float64).view(n_prn, 4)
    return grid, r32[:, 0].clone(), r32[:, 1].clone(), rf[:, 2].clone(), rd[:, 3].clone()


@search.register_fake
def _search_fake(buf, ix, chips, fds, fs, fi, T, N, Nz, n_sum):
    n_prn = chips.shape[0]
    return (buf.new_empty((n_prn, len(fds), N), dtype=torch.float32),
            buf.new_empty((n_prn,), dtype=torch.int32), buf.new_empty((n_prn,), dtype=torch.int32),
            buf.new_empty((n_prn,), dtype=torch.float32),
            buf.new_empty((n_prn,), dtype=torch.float64))


@torch.library.custom_op("pocketsdr::corr_batch", mutates_args=())
def corr_batch(buf: torch.Tensor, ix: List[int], fc: List[float], phi: List[float],
               coff: List[float], banks: torch.Tensor, pos: List[float], fs: float,
               N: int) -> torch.Tensor:
    """Channels j = 0 .. n-1 on one IF buffer: sdr_mix_carr(buf, ix[j], N, fs,
    fc[j], phi[j]) then sdr_corr_std with code bank banks[j] (int8 CUDA
    [n, SDR_N_CODES * N, 2], the receiver's fractional-phase banks of a real
    code), code offset coff[j] and tap positions pos (samples, P / E / L
    first). Returns complex64 [n, len(pos)], bit-identical to the reference
    calls."""
    if not (buf.is_cuda and banks.is_cuda):
        raise ValueError("pocketsdr::corr_batch takes CUDA tensors")
    n = len(ix)
    if banks.dtype != torch.int8 or tuple(banks.shape) != (n, track.SDR_N_CODES * N, 2):
        raise ValueError(f"banks must be int8 [{n}, {track.SDR_N_CODES * N}, 2]")
    if not 1 <= len(pos) <= track.SDR_MAX_CORR:
        raise ValueError(f"1 to {track.SDR_MAX_CORR} tap positions")
    buf, banks = buf.contiguous(), banks.contiguous()
    stride = banks.stride(0)
    specs = [dict(buf=0, ix=int(ix[j]), N=N, fs=fs, fc=float(fc[j]), phi=float(phi[j]),
                  coff=float(coff[j]), code_ptr=banks.data_ptr() + j * stride,
                  cpx_code=False, pos=pos) for j in range(n)]
    jobs = track.make_jobs(specs)
    out = torch.empty((n, track.SDR_MAX_CORR), dtype=torch.complex64, device="cuda")
    track.corr_batch(jobs, [buf.data_ptr()], [buf.numel()], out.data_ptr(), 0,
                     torch_stream())
    return out[:, :len(pos)].clone()


@corr_batch.register_fake
def _corr_batch_fake(buf, ix, fc, phi, coff, banks, pos, fs, N):
    return buf.new_empty((len(ix), len(pos)), dtype=torch.complex64)


def release_plans() -> None:
    """Frees the acquisition plans cached by pocketsdr::search."""
    with _plans_lock:
        for pl in _plans.values():
            pl.close()
        _plans.clear()


__all__ = ["search", "corr_batch", "release_plans"]
