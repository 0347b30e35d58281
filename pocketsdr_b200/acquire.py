"""Batched parallel-code-phase acquisition on the GPU (sdrg_acq_* C ABI).

One AcqPlan holds every signal group of a search: the permuted code DFTs,
FFT tables, forward-transform and grid buffers live on the device; run()
executes forward FFTs (shared by all PRNs of a group), the fused
code-multiply / inverse FFT / power accumulation over all sums, and the
per-PRN peak, C/N0 and fine-Doppler reduction - the work that
src/sdr_ch.c:398-450 (search_sig) and app/pocket_acq/pocket_acq.c:152-192
do one PRN at a time with sdr_search_code + sdr_corr_max + sdr_fine_dop.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import AcqResult, AcqSig, GpuError, check, lib

RESULT_DTYPE = np.dtype([("bin", np.int32), ("offset", np.int32), ("cn0", np.float32),
                         ("pmax", np.float32), ("pave", np.float64), ("fd", np.float64)])
assert RESULT_DTYPE.itemsize == C.sizeof(AcqResult)


class AcqPlan:
    def __init__(self, groups, code_ffts):
        """groups: sequence of synth.Group-like objects (sig, prns, fs, fi, T, N,
        L, Nmax, n_sum, fds, buf); code_ffts: per group complex64 [n_prn, L],
        or None for a group whose codes come from set_codes (device chips)."""
        self.groups = list(groups)
        n = len(self.groups)
        sigs = (AcqSig * n)()
        self._keep = []
        for i, (g, cf) in enumerate(zip(self.groups, code_ffts)):
            fds = np.ascontiguousarray(g.fds, np.float32)
            if cf is not None:
                cf = np.ascontiguousarray(cf, np.complex64)
                if cf.shape != (len(g.prns), g.L):
                    raise ValueError(f"group {i}: code_fft shape {cf.shape} != {(len(g.prns), g.L)}")
            self._keep += [cf, fds]
            s = sigs[i]
            s.L, s.N, s.Nmax, s.n_sum = g.L, g.N, g.Nmax, g.n_sum
            s.n_prn, s.len_fds = len(g.prns), len(fds)
            s.fs, s.fi, s.T = g.fs, g.fi, g.T
            s.fds = fds.ctypes.data_as(C.POINTER(C.c_float))
            s.code_fft = C.c_void_p(cf.ctypes.data) if cf is not None else None
            s.buf = g.buf
        self.handle = lib.sdrg_acq_plan_new(sigs, n)
        if not self.handle:
            check("sdrg_acq_plan_new")
            raise GpuError("sdrg_acq_plan_new failed")
        self._keep = None      # the plan copied everything
        self.n_res = sum(len(g.prns) for g in self.groups)
        self.offsets = np.cumsum([0] + [len(g.prns) for g in self.groups])[:-1]

    def set_codes(self, g: int, chips, T: float, coff: float = 0.0, N: int | None = None,
                  code_Q=None) -> None:
        """Computes group g's code DFTs on the device (sdrg_acq_set_codes) from
        chips [n_prn, len_code] (one code per PRN, group order): the N-sample
        replica (default: the group's N) of code period T, zero padded to L.
        Asynchronous on torch's current stream, like run_device."""
        from . import replica
        gr = self.groups[g]
        ci = replica.device_chips(chips)
        if ci.shape[0] != len(gr.prns):
            raise ValueError(f"group {g}: {ci.shape[0]} codes for {len(gr.prns)} PRNs")
        replica.set_plan_codes(self.handle, g, ci, T, coff, gr.N if N is None else N, code_Q)

    @property
    def cells(self) -> int:
        return int(lib.sdrg_acq_plan_cells(self.handle))

    def run_host(self, bufs, ix=None) -> np.ndarray:
        """Synchronous run from host IF buffers; returns RESULT_DTYPE[n_res]."""
        bufs = [np.ascontiguousarray(b, np.uint8) for b in bufs]
        ix = list(ix) if ix is not None else [0] * len(bufs)
        ptrs = (C.c_void_p * len(bufs))(*[b.ctypes.data for b in bufs])
        lens = (C.c_int * len(bufs))(*[len(b) for b in bufs])
        ixs = (C.c_int * len(bufs))(*ix)
        res = np.zeros(self.n_res, RESULT_DTYPE)
        st = lib.sdrg_acq_run_host(self.handle, ptrs, lens, ixs, C.c_void_p(res.ctypes.data))
        if st:
            check("sdrg_acq_run_host")
        return res

    def run_device(self, buf_ptrs, lens, ix, res_ptr: int, stream: int = 0,
                   graph: bool = False) -> None:
        """Asynchronous run on device-resident IF buffers (raw device
        pointers, e.g. torch tensor data_ptr()) on a CUDA stream handle.
        graph=True replays the plan's captured CUDA graph (captured on the
        first call for these buffers)."""
        n = len(buf_ptrs)
        ptrs = (C.c_void_p * n)(*buf_ptrs)
        lens_ = (C.c_int * n)(*lens)
        ixs = (C.c_int * n)(*ix)
        fn = lib.sdrg_acq_run_graph if graph else lib.sdrg_acq_run
        st = fn(self.handle, ptrs, lens_, ixs, C.c_void_p(res_ptr), C.c_void_p(stream))
        if st:
            check("sdrg_acq_run_graph" if graph else "sdrg_acq_run")

    def set_worklist(self, mode: int = 1) -> bool:
        """Consumer issue mode (sdrg_acq_set_worklist): 1 the single
        persistent work-list launch, 0 (the plan's default) per-group launches
        on concurrent streams, -1 the work list where the plan allows it.
        Returns whether runs use the work list."""
        r = lib.sdrg_acq_set_worklist(self.handle, int(mode))
        if r < 0:
            check("sdrg_acq_set_worklist")
        return bool(r)

    def graph_captures(self) -> int:
        return int(lib.sdrg_acq_graph_captures(self.handle))

    def grid_ptr(self, g: int) -> int:
        return int(lib.sdrg_acq_grid(self.handle, g) or 0)

    def grid(self, g: int) -> np.ndarray:
        """Host copy of group g's grid, float32 [n_prn, len_fds, Nmax]."""
        gr = self.groups[g]
        out = np.empty((len(gr.prns), len(gr.fds), gr.Nmax), np.float32)
        if lib.sdrg_acq_grid_host(self.handle, g, C.c_void_p(out.ctypes.data)):
            check("sdrg_acq_grid_host")
        return out

    def profile(self, enable: bool = True) -> None:
        """Record CUDA events around every kernel launch of run()/run_device()."""
        if lib.sdrg_acq_profile(self.handle, int(enable)):
            check("sdrg_acq_profile")

    def profile_get(self) -> dict:
        """Kernel timing since the last call: {(group, kind): (ms, launches)}
        per launch family, and {('span', kind): (ms, runs)}, the per-run span
        of each kind over all (concurrent) groups; kind in fwd, cons, peak."""
        ng = len(self.groups)
        ms = np.zeros(3 * ng + 3, np.float64)
        n = np.zeros(3 * ng + 3, np.int64)
        if lib.sdrg_acq_profile_get(self.handle, C.c_void_p(ms.ctypes.data),
                                    C.c_void_p(n.ctypes.data)):
            check("sdrg_acq_profile_get")
        kinds = ("fwd", "cons", "peak")
        out = {(g, kinds[k]): (float(ms[3 * g + k]), int(n[3 * g + k]))
               for g in range(ng) for k in range(3)}
        out.update({("span", kinds[k]): (float(ms[3 * ng + k]), int(n[3 * ng + k]))
                    for k in range(3)})
        return out

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib.sdrg_acq_plan_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
