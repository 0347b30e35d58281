"""Differentiable refinement of code delay, Doppler and carrier phase on the
GPU (sdrg_refine_* C ABI), with a torch.autograd.Function around the block
correlations.

The reference has no counterpart: after the acquisition grid
(src/sdr_func.c:664-744: search, peak and the three-bin Doppler quadratic)
its receiver hands the signal to tracking loops (src/sdr_ch.c). Here the
grid peak seeds a batched Gauss-Newton refinement of
theta = (tau [s], fd [Hz], phi [cycles at t_ref]) for many signals at once;
the model (carrier, code linearly interpolated through the chip centres) is
documented in include/pocket_sdr_gpu.h and oracle/refine_oracle.c.

* RefinePlan   - signals (chips, nominal chip rate, IF, RF carrier), sampling
                 and span geometry (K blocks of Nb samples); sums / vjp / gn.
* CorrBlocks   - autograd Function: forward = per-block correlations C_k
                 (FP32), backward = hand-written adjoint that RECOMPUTES the
                 derivative sums from the IF samples (nothing per-sample is
                 stored between forward and backward).
* corr_power   - the correlation-power loss sum_k |C_k|^2 per signal.

All tensors live on the CUDA device; every call is asynchronous on torch's
current stream. There is no CPU path: without the library the import fails.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from ._lib import GpuError, RefineSig, check, lib, torch_stream

W = 12                      # sums per (signal, block)
MODEL_POWER, MODEL_COHERENT, MODEL_BLOCKS = 0, 1, 2


@dataclass
class RefineSpec:
    chips: np.ndarray       # int8 chip values of one code period
    rate: float             # nominal chip rate (chips/s)
    fi: float               # IF (Hz)
    fc: float = 0.0         # RF carrier (Hz) for the carrier-aided code rate


def _stream() -> C.c_void_p:
    return C.c_void_p(torch_stream())


def _dptr(t: torch.Tensor) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


class RefinePlan:
    def __init__(self, specs, fs: float, iq: bool, Nb: int, K: int):
        self.specs = list(specs)
        n = len(self.specs)
        arr = (RefineSig * n)()
        keep = []
        for a, s in zip(arr, self.specs):
            chips = np.ascontiguousarray(s.chips, np.int8)
            keep.append(chips)
            a.chips = C.c_void_p(chips.ctypes.data)
            a.Lc, a.rate, a.fi, a.fc = len(chips), float(s.rate), float(s.fi), float(s.fc)
        self.handle = lib.sdrg_refine_plan_new(arr, n, float(fs), int(bool(iq)), int(Nb), int(K))
        if not self.handle:
            check("sdrg_refine_plan_new")
            raise GpuError("sdrg_refine_plan_new failed")
        info = (C.c_int * 4)()
        lib.sdrg_refine_plan_info(self.handle, info)
        self.n, self.K, self.Nb, self.ctas_per_block = info[0], info[1], info[2], info[3]
        self.fs, self.iq = float(fs), bool(iq)
        self.rate_nom = torch.tensor([s.rate for s in self.specs], dtype=torch.float64)
        self.fc = torch.tensor([s.fc for s in self.specs], dtype=torch.float64)

    def t_ref(self, ix0: int) -> float:
        return (ix0 + 0.5 * self.K * self.Nb) / self.fs

    def carrier_aided_rate(self, theta: torch.Tensor) -> torch.Tensor:
        """rate_nom (1 + fd / fc) per signal (rate_nom where fc = 0)."""
        rn, fc = self.rate_nom.to(theta.device), self.fc.to(theta.device)
        safe = torch.where(fc > 0, fc, torch.ones_like(fc))
        return torch.where(fc > 0, rn * (1.0 + theta[:, 1] / safe), rn).contiguous()

    def _check(self, buf: torch.Tensor, theta: torch.Tensor, rate: torch.Tensor) -> None:
        if not (buf.is_cuda and buf.dtype == torch.uint8 and buf.is_contiguous()):
            raise ValueError("buf: contiguous uint8 CUDA tensor expected")
        if theta.shape != (self.n, 3) or theta.dtype != torch.float64 or not theta.is_cuda \
                or not theta.is_contiguous():
            raise ValueError(f"theta: contiguous float64 CUDA tensor [{self.n}, 3] expected")
        if rate.shape != (self.n,) or rate.dtype != torch.float64 or not rate.is_cuda \
                or not rate.is_contiguous():
            raise ValueError(f"rate: contiguous float64 CUDA tensor [{self.n}] expected")

    def sums(self, buf: torch.Tensor, ix0: int, theta: torch.Tensor, rate: torch.Tensor,
             mode: int = 1) -> torch.Tensor:
        """Block sums: mode 1 -> float32 [n, K, 12], mode 0 -> C only [n, K, 2]."""
        self._check(buf, theta, rate)
        out = torch.empty((self.n, self.K, W if mode else 2), dtype=torch.float32,
                          device=theta.device)
        st = lib.sdrg_refine_sums(self.handle, _dptr(buf), buf.numel(), int(ix0), _dptr(theta),
                                  _dptr(rate), int(mode), _dptr(out), _stream())
        if st:
            check("sdrg_refine_sums")
        return out

    def vjp(self, sums: torch.Tensor, g: torch.Tensor) -> torch.Tensor:
        """d/dtheta sum_k Re(conj(g_k) C_k) -> float64 [n, 3]."""
        sums = sums.contiguous()
        g = g.to(torch.float32).contiguous()
        if sums.shape != (self.n, self.K, W) or g.shape != (self.n, self.K, 2):
            raise ValueError("vjp: sums [n, K, 12] and g [n, K, 2] expected")
        grad = torch.empty((self.n, 3), dtype=torch.float64, device=sums.device)
        if lib.sdrg_refine_vjp(self.handle, _dptr(sums), _dptr(g), _dptr(grad), _stream()):
            check("sdrg_refine_vjp")
        return grad

    def from_peaks(self, res: torch.Tensor, ix_grid: int, ix0: int, theta: torch.Tensor,
                   rate: torch.Tensor) -> None:
        """theta / rate (in place) from device acquisition results (the
        sdrg_acq_result_t bytes an AcqPlan.run_device wrote), signal order =
        plan order."""
        if not res.is_cuda or res.numel() < 32 * self.n:
            raise ValueError("res: device buffer of n_sig acquisition results expected")
        if lib.sdrg_refine_from_peaks(self.handle, _dptr(res), int(ix_grid), int(ix0),
                                      _dptr(theta), _dptr(rate), _stream()):
            check("sdrg_refine_from_peaks")

    def gn(self, buf: torch.Tensor, ix0: int, theta: torch.Tensor, rate: torch.Tensor,
           models=(MODEL_COHERENT,) * 5, info: bool = True):
        """Gauss-Newton steps in place on theta / rate (one per entry of
        models); returns the float64 info tensor [steps, n, 5] or None."""
        self._check(buf, theta, rate)
        models = [int(m) for m in models]
        m_arr = (C.c_int * max(1, len(models)))(*models)
        inf = torch.zeros((len(models), self.n, 5), dtype=torch.float64, device=theta.device) \
            if info else None
        st = lib.sdrg_refine_gn(self.handle, _dptr(buf), buf.numel(), int(ix0), _dptr(theta),
                                _dptr(rate), m_arr, len(models),
                                _dptr(inf) if inf is not None else None, _stream())
        if st:
            check("sdrg_refine_gn")
        return inf

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib.sdrg_refine_plan_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CorrBlocks(torch.autograd.Function):
    """C = corr_blocks(theta): float32 [n, K, 2] (Re, Im of C_k); the
    backward recomputes the derivative sums and applies the hand-written
    adjoint (sdrg_refine_vjp). rate is a constant input."""

    @staticmethod
    def forward(ctx, theta, plan, buf, ix0, rate):
        ctx.plan, ctx.buf, ctx.ix0 = plan, buf, ix0
        ctx.save_for_backward(theta, rate)
        return plan.sums(buf, ix0, theta.detach(), rate, mode=0)

    @staticmethod
    def backward(ctx, gC):
        theta, rate = ctx.saved_tensors
        s = ctx.plan.sums(ctx.buf, ctx.ix0, theta.detach(), rate, mode=1)
        return ctx.plan.vjp(s, gC), None, None, None, None


def corr_blocks(plan: RefinePlan, buf, ix0: int, theta, rate=None) -> torch.Tensor:
    if rate is None:
        rate = plan.carrier_aided_rate(theta.detach())
    return CorrBlocks.apply(theta, plan, buf, ix0, rate)


def corr_power(plan: RefinePlan, buf, ix0: int, theta, rate=None) -> torch.Tensor:
    """Correlation-power loss per signal: sum_k |C_k|^2 (K coherent blocks,
    summed non-coherently). Its carrier-phase gradient is identically zero."""
    C_ = corr_blocks(plan, buf, ix0, theta, rate)
    return (C_ * C_).sum(dim=(1, 2))


def theta_from_peaks(offset, fd, ix_grid, fs: float, fc, t_ref: float) -> np.ndarray:
    """Starting theta from acquisition peaks: code phase 0 at sample
    ix_grid + offset, carrier-aided code rate, phase 0. Returns float64
    [n, 3]."""
    offset = np.asarray(offset, np.float64)
    fd = np.asarray(fd, np.float64)
    fc = np.asarray(fc, np.float64)
    t0 = (np.asarray(ix_grid, np.float64) + offset) / fs
    scale = np.where(fc > 0, fd / np.where(fc > 0, fc, 1.0), 0.0)
    tau = t0 + scale * (t0 - t_ref)
    return np.stack([tau, fd, np.zeros_like(fd)], axis=1)
