"""IF ingest on the GPU (sdrg_ingest_* C ABI): raw front-end blocks to packed
sdr_cpx8_t IF buffers, with the per-channel LPF and array beam-forming of the
receiver's write_buff (src/sdr_rcv.c:840-936), bit-identical.

    ing = Ingest(fmt=FMT_RAW16, N=24000, fs=24e6, IQ=[1, 1, 2, 2], bits=[3, 3, 2, 2],
                 lpf_fc=[5e6, 5e6, 0, 0])
    ing.run(raw_tensor, ix, [buf0, buf1, buf2, buf3], base)   # CUDA tensors
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import IngestCfg, check, lib, torch_stream

FMT_INT8, FMT_INT8X2, FMT_RAW8, FMT_RAW16, FMT_RAW16I, FMT_RAW32, FMT_CS8, FMT_CS16 = range(1, 9)
BYTES_PER_SAMPLE = {FMT_INT8: 1, FMT_INT8X2: 2, FMT_RAW8: 1, FMT_RAW16: 2, FMT_RAW16I: 2,
                    FMT_RAW32: 4, FMT_CS8: 2, FMT_CS16: 4}


def n_rfch(fmt: int) -> int:
    """RF channels a format carries (src/sdr_rcv.c:93-102)."""
    return {FMT_RAW8: 2, FMT_RAW16: 4, FMT_RAW16I: 8, FMT_RAW32: 8}.get(fmt, 1)


def lpf_taps(fc: float, fs: float):
    """The 9 Q13 taps sdr_lpf_new computes, or None for a cutoff outside (0, fs/2)."""
    h = np.zeros(9, np.int32)
    return h if lib.sdrg_lpf_taps(fc, fs, C.c_void_p(h.ctypes.data)) else None


class Ingest:
    def __init__(self, fmt: int, N: int, fs: float, IQ=None, bits=None, lut_off=(0.0, 0.0),
                 lut_scale=(1.0, 1.0), lpf_fc=None, w=None, arch_on=None):
        """w: int16 [narch, n_rf, 2] Q8 beam-forming weights (array channels,
        multi-channel RAW formats only); arch_on: per array channel flag."""
        cfg = IngestCfg()
        cfg.fmt, cfg.N, cfg.fs = fmt, N, fs
        nrf = n_rfch(fmt)
        for k in range(8):
            cfg.IQ[k] = int(IQ[k]) if IQ is not None and k < len(IQ) else 2
            cfg.bits[k] = int(bits[k]) if bits is not None and k < len(bits) else 2
            cfg.lpf_fc[k] = float(lpf_fc[k]) if lpf_fc is not None and k < len(lpf_fc) else 0.0
        cfg.lut_off[0], cfg.lut_off[1] = lut_off
        cfg.lut_scale[0], cfg.lut_scale[1] = lut_scale
        narch = 0 if w is None else len(w)
        cfg.narch = narch
        if narch:
            wa = np.asarray(w, np.int16).reshape(narch, nrf, 2)
            for m in range(narch):
                cfg.arch_on[m] = int(arch_on[m]) if arch_on is not None else 1
                for k in range(nrf):
                    cfg.w[(m * 8 + k) * 2] = int(wa[m, k, 0])
                    cfg.w[(m * 8 + k) * 2 + 1] = int(wa[m, k, 1])
        self.fmt, self.N, self.n_rf, self.narch = fmt, N, nrf, narch
        self.handle = lib.sdrg_ingest_new(C.byref(cfg))
        if not self.handle:
            check("sdrg_ingest_new")
            raise RuntimeError("sdrg_ingest_new failed")

    def run(self, raw, ix: int, bufs, base: int = 0, stream=None) -> None:
        """raw: CUDA uint8 tensor (N * bytes-per-sample); bufs: n_rf + narch CUDA
        uint8 tensors (IF buffers); asynchronous on torch's current stream."""
        if len(bufs) != self.n_rf + self.narch:
            raise ValueError(f"{self.n_rf + self.narch} buffers expected")
        for b in bufs:
            if b.numel() < base + self.N:
                raise ValueError("IF buffer shorter than base + N")
        if raw.numel() < self.N * BYTES_PER_SAMPLE[self.fmt]:
            raise ValueError("raw block shorter than N samples")
        ptrs = (C.c_void_p * len(bufs))(*[b.data_ptr() for b in bufs])
        st = stream if stream is not None else torch_stream()
        if lib.sdrg_ingest_run(self.handle, C.c_void_p(raw.data_ptr()), int(ix), ptrs, int(base),
                               C.c_void_p(st)):
            check("sdrg_ingest_run")

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib.sdrg_ingest_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
