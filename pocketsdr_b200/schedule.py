"""Batched signal search (sdrg_search_batch C ABI): every channel that is ready
to search, searched at once - the work the receiver does one channel at a time
with update_srch_ch (src/sdr_rcv.c:1222-1257) and search_sig
(src/sdr_ch.c:398-450), with the same per-channel decision and tracking seed.

    setups = [Setup(chips_L1CA, T=1e-3, fs=24e6, fi=..., max_dop=5000.0, buf=0), ...]
    reqs = [Request(setup=0, prn=k) for k in idle_L1CA] + [Request(1, 4, fd_ext=1234.0)]
    res = search(setups, reqs, [if_buf_tensor], ix, t_acq=20e-3, thres_cn0=35.0)
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import SrchReq, SrchRes, SrchSetup, check, lib, torch_stream

RESULT_DTYPE = np.dtype([("found", np.int32), ("bin", np.int32), ("offset", np.int32),
                         ("cn0", np.float32), ("fd", np.float64), ("coff", np.float64),
                         ("n_sum", np.int32)], align=True)
assert RESULT_DTYPE.itemsize == C.sizeof(SrchRes)


@dataclass
class Setup:
    chips: object          # int8 [n_prn, len_code] (numpy or CUDA tensor)
    T: float
    fs: float
    fi: float
    max_dop: float = 5000.0
    buf: int = 0
    N: int | None = None   # samples per code period (default round(fs * T))


@dataclass
class Request:
    setup: int
    prn: int               # code row in the setup
    fd_ext: float = 0.0
    fd_ext_n: int = 0


def _arrays(setups, reqs):
    from . import replica
    su = (SrchSetup * len(setups))()
    keep = []
    for s, d in zip(su, setups):
        c = replica.device_chips(d.chips)
        keep.append(c)
        s.code_dev = C.c_void_p(c.data_ptr())
        s.len_code, s.n_prn = c.shape[1], c.shape[0]
        s.T, s.fs, s.fi, s.max_dop, s.buf = d.T, d.fs, d.fi, d.max_dop, d.buf
        s.N = d.N if d.N is not None else int(round(d.fs * d.T))
    rq = (SrchReq * len(reqs))()
    for r, d in zip(rq, reqs):
        r.setup, r.prn, r.fd_ext, r.fd_ext_n = d.setup, d.prn, d.fd_ext, d.fd_ext_n
    return su, rq, keep


def groups(setups, reqs, t_acq):
    """(group of each request, sums per group, bins per group) - host only."""
    su, rq, keep = _arrays(setups, reqs)
    gi = np.zeros(len(reqs), np.int32)
    ns = np.zeros(len(reqs), np.int32)
    nf = np.zeros(len(reqs), np.int32)
    n = lib.sdrg_srch_groups(su, len(su), rq, len(rq), t_acq, C.c_void_p(gi.ctypes.data),
                             C.c_void_p(ns.ctypes.data), C.c_void_p(nf.ctypes.data))
    if n < 0:
        check("sdrg_srch_groups")
    return gi, ns[:n], nf[:n]


def search(setups, reqs, bufs, ix: int, t_acq: float, thres_cn0: float) -> np.ndarray:
    """Runs every request's search; bufs: CUDA uint8 tensors (IF buffers).
    Returns RESULT_DTYPE[len(reqs)]."""
    su, rq, keep = _arrays(setups, reqs)
    ptrs = (C.c_void_p * len(bufs))(*[b.data_ptr() for b in bufs])
    lens = (C.c_int * len(bufs))(*[b.numel() for b in bufs])
    res = (SrchRes * len(reqs))()
    st = torch_stream()
    if lib.sdrg_search_batch(su, len(su), rq, len(rq), ptrs, lens, int(ix), t_acq, thres_cn0,
                             res, C.c_void_p(st)):
        check("sdrg_search_batch")
    return np.frombuffer(bytes(res), RESULT_DTYPE).copy()
