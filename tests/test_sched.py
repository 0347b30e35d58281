"""Batched search scheduling, host side (no device work): the grouping
sdrg_search_batch uses - unaided channels of one code setup share the
receiver's sdr_dop_bins(T, 0, max_dop) bins, each Doppler-aided channel gets
fd_ext_n (default 3) bins, and every group accumulates the code periods
search_sig would (src/sdr_ch.c:398-450: stop once n_sum * T >= sdr_t_acq)."""
import ctypes as C

import numpy as np
import pytest

from pocketsdr_b200._lib import SrchReq, SrchSetup, lib


def _setups(specs):
    su = (SrchSetup * len(specs))()
    for s, (T, fs, n_prn, max_dop) in zip(su, specs):
        s.code_dev = None                  # not touched by the grouping
        s.len_code, s.n_prn, s.T, s.fs, s.fi = 1023, n_prn, T, fs, 0.0
        s.N, s.max_dop, s.buf = int(round(fs * T)), max_dop, 0
    return su


def _reqs(items):
    rq = (SrchReq * len(items))()
    for r, (su, prn, fd, n) in zip(rq, items):
        r.setup, r.prn, r.fd_ext, r.fd_ext_n = su, prn, fd, n
    return rq


def _groups(su, rq, t_acq):
    gi = np.zeros(len(rq), np.int32)
    ns = np.zeros(len(rq), np.int32)
    nf = np.zeros(len(rq), np.int32)
    n = lib.sdrg_srch_groups(su, len(su), rq, len(rq), t_acq, C.c_void_p(gi.ctypes.data),
                             C.c_void_p(ns.ctypes.data), C.c_void_p(nf.ctypes.data))
    return n, gi, ns[:max(n, 0)], nf[:max(n, 0)]


def _sums(T, t_acq):
    n = 1
    while n * T < t_acq:
        n += 1
    return n


def test_grouping_follows_the_receiver(ref):
    su = _setups([(1e-3, 24e6, 32, 5000.0), (4e-3, 24e6, 36, 5000.0), (10e-3, 12e6, 4, 2500.0)])
    items = [(0, p, 0.0, 0) for p in (3, 7, 9)] + [(1, 5, 0.0, 0), (0, 11, 1234.5, 0),
                                                    (1, 2, -870.25, 5), (2, 1, 0.0, 0), (0, 3, 0.0, 0)]
    rq = _reqs(items)
    for t_acq in (20e-3, 0.0105, 1e-3, 0.1):
        n, gi, ns, nf = _groups(su, rq, t_acq)
        assert n == 5
        # unaided requests of a setup share one group; aided ones are alone
        assert gi[0] == gi[1] == gi[2] == gi[7] and len({gi[0], gi[3], gi[4], gi[5], gi[6]}) == 5
        for i, (s, _, fd, nw) in enumerate(items):
            T = (1e-3, 4e-3, 10e-3)[s]
            assert ns[gi[i]] == _sums(T, t_acq)
            want = (nw or 3) if fd != 0.0 else len(ref.dop_bins(T, 0.0, su[s].max_dop))
            assert nf[gi[i]] == want, i


def test_bad_requests_are_rejected():
    su = _setups([(1e-3, 24e6, 32, 5000.0)])
    for bad in ([(1, 0, 0.0, 0)], [(0, 32, 0.0, 0)], [(0, -1, 0.0, 0)]):
        n, *_ = _groups(su, _reqs(bad), 20e-3)
        assert n == -1
        lib.sdr_gpu_clear_error()
    n, *_ = _groups(su, _reqs([(0, 1, 0.0, 0)]), 0.0)
    assert n == -1
    lib.sdr_gpu_clear_error()
