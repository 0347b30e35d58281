"""ctypes binding of libsdr_gpu.so (the C ABI declared in include/pocket_sdr_gpu.h).

The library is required: importing this module without the built .so raises
ImportError (build it with ``python -m pocketsdr_b200.build``). There is no
CPU fallback anywhere in the package.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libsdr_gpu.so")

_p = C.c_void_p
_i = C.c_int
_d = C.c_double
_f = C.c_float


class SdrBuff(C.Structure):
    """sdr_buff_t (src/pocket_sdr.h:242-245)."""
    _fields_ = [("data", C.POINTER(C.c_uint8)), ("IQ", C.c_int), ("N", C.c_int)]


class AcqSig(C.Structure):
    """sdrg_acq_sig_t."""
    _fields_ = [("L", _i), ("N", _i), ("Nmax", _i), ("n_sum", _i), ("n_prn", _i),
                ("len_fds", _i), ("fs", _d), ("fi", _d), ("T", _d),
                ("fds", C.POINTER(_f)), ("code_fft", _p), ("buf", _i)]


class AcqResult(C.Structure):
    """sdrg_acq_result_t."""
    _fields_ = [("bin", _i), ("offset", _i), ("cn0", _f), ("pmax", _f),
                ("pave", _d), ("fd", _d)]


class IngestCfg(C.Structure):
    """sdrg_ingest_cfg_t."""
    _fields_ = [("fmt", _i), ("N", _i), ("fs", _d), ("IQ", _i * 8), ("bits", _i * 8),
                ("lut_off", _d * 2), ("lut_scale", _d * 2), ("lpf_fc", _d * 8),
                ("narch", _i), ("arch_on", _i * 8), ("w", C.c_int16 * (8 * 8 * 2))]


class SrchSetup(C.Structure):
    """sdrg_srch_setup_t."""
    _fields_ = [("code_dev", _p), ("len_code", _i), ("n_prn", _i), ("T", _d), ("fs", _d),
                ("fi", _d), ("N", _i), ("max_dop", _d), ("buf", _i)]


class SrchReq(C.Structure):
    """sdrg_srch_req_t."""
    _fields_ = [("setup", _i), ("prn", _i), ("fd_ext", _f), ("fd_ext_n", _i)]


class SrchRes(C.Structure):
    """sdrg_srch_res_t."""
    _fields_ = [("found", _i), ("bin", _i), ("offset", _i), ("cn0", _f), ("fd", _d),
                ("coff", _d), ("n_sum", _i)]


class L6Job(C.Structure):
    """sdrg_l6_job_t."""
    _fields_ = [("buf", _i), ("ix", _i), ("N", _i), ("fs", _d), ("fc", _d), ("phi", _d),
                ("code_fft", _p), ("len_code", _i), ("n", _i), ("pos", C.POINTER(_d))]


class RefineSig(C.Structure):
    """sdrg_refine_sig_t."""
    _fields_ = [("chips", _p), ("Lc", _i), ("rate", _d), ("fi", _d), ("fc", _d)]


# every exported entry point and its signature; tests check the library
# exports exactly these names
SIGNATURES = {
    "sdr_func_init": ([C.c_char_p], None),
    "sdr_mix_carr": ([C.POINTER(SdrBuff), _i, _i, _d, _d, _d, _p], None),
    "sdr_corr_std": ([_p, _p, _i, _d, _p, _i, _p, _p], None),
    "sdr_corr_std_cpx_code": ([_p, _p, _i, _d, _p, _i, _p, _p], None),
    "sdr_corr_std_cpx": ([_p, _i, _i, _i, _d, _d, _d, _p, _p, _i, _p], None),
    "sdr_corr_fft": ([_p, _p, _i, _p], None),
    "sdr_corr_fft_cpx": ([_p, _i, _i, _i, _d, _d, _d, _p, _p], None),
    "sdr_search_code": ([_p, _d, C.POINTER(SdrBuff), _i, _i, _d, _d, _p, _i, _p], None),
    "sdr_corr_max": ([_p, _i, _i, _i, _d, _p], _f),
    "sdr_fine_dop": ([_p, _i, _p, _i, _p], _d),
    "sdr_dop_bins": ([_d, _f, _f, C.POINTER(_i)], C.POINTER(_f)),
    "sdr_res_code": ([_p, _p, _i, _d, _d, _d, _i, _i, _p], None),
    "sdr_gen_code_fft": ([_p, _p, _i, _d, _d, _d, _i, _i, _p], None),
    "sdr_lpf_new": ([_d, _d], _p),
    "sdr_lpf_free": ([_p], None),
    "sdr_lpf_apply": ([_p, _p, _i], None),
    "sdr_psd_cpx": ([_p, _i, _i, _d, _i, _p], None),
    "sdr_gpu_last_error": ([C.c_char_p, _i], _i),
    "sdr_gpu_clear_error": ([], None),
    "sdrg_init": ([_i], _i),
    "sdrg_fft_supported": ([_i], _i),
    "sdrg_version": ([], C.c_char_p),
    "sdrg_inject_alloc_failure": ([_i], None),
    "sdrg_inject_stage_timeout": ([_i], _i),
    "sdrg_fft_autotune": ([_i, _p, _p, _p], _i),
    "sdrg_fft_schedule_set": ([_i, _i, _i], _i),
    "sdrg_fft_schedule_get": ([_i, _p, _p], _i),
    "sdrg_fft_schedule_save": ([C.c_char_p], _i),
    "sdrg_fft_schedule_load": ([C.c_char_p], _i),
    "sdrg_corr_fft_noalloc": ([_p, _p, _i, _p, _p], _i),
    "sdrg_acq_plan_new": ([C.POINTER(AcqSig), _i], _p),
    "sdrg_acq_plan_free": ([_p], None),
    "sdrg_acq_plan_cells": ([_p], C.c_int64),
    "sdrg_acq_run": ([_p, _p, _p, _p, _p, _p], _i),
    "sdrg_acq_run_graph": ([_p, _p, _p, _p, _p, _p], _i),
    "sdrg_acq_graph_captures": ([_p], _i),
    "sdrg_acq_set_worklist": ([_p, _i], _i),
    "sdrg_acq_grid": ([_p, _i], _p),
    "sdrg_acq_grid_host": ([_p, _i, _p], _i),
    "sdrg_acq_profile": ([_p, _i], _i),
    "sdrg_acq_profile_get": ([_p, _p, _p], _i),
    "sdrg_acq_run_host": ([_p, _p, _p, _p, _p], _i),
    "sdrg_corr_batch": ([_p, _i, _p, _p, _p, _p, _p], _i),
    "sdrg_mix_carr": ([_p, _i, _i, _i, _d, _d, _d, _p, _p], _i),
    "sdrg_gen_code": ([C.c_char_p, _i, _p, _i], _i),
    "sdrg_sec_code": ([C.c_char_p, _i, _p, _i], _i),
    "sdrg_res_code": ([_p, _p, _i, _i, _d, _d, _d, _i, _i, _i, _p, _p], _i),
    "sdrg_gen_code_fft": ([_p, _p, _i, _i, _d, _d, _d, _i, _i, _p, _p], _i),
    "sdrg_acq_set_codes": ([_p, _i, _p, _p, _i, _d, _d, _i, _p], _i),
    "sdrg_search_batch": ([C.POINTER(SrchSetup), _i, C.POINTER(SrchReq), _i, _p, _p, _i, _d, _d,
                           C.POINTER(SrchRes), _p], _i),
    "sdrg_search_release": ([], None),
    "sdrg_srch_groups": ([C.POINTER(SrchSetup), _i, C.POINTER(SrchReq), _i, _d, _p, _p, _p], _i),
    "sdrg_l6_csk_batch": ([C.POINTER(L6Job), _i, _p, _p, _p, _p, _p, _p], _i),
    "sdrg_csk_decode": ([_p, _i, _i, _i, _p, _i, _p, _p, _p], _i),
    "sdrg_psd": ([_p, _i, _i, _d, _i, _p, _p], _i),
    "sdrg_psd_if": ([_p, _i, _i, _i, _i, _d, _i, _p, _p], _i),
    "sdrg_ingest_new": ([C.POINTER(IngestCfg)], _p),
    "sdrg_ingest_free": ([_p], None),
    "sdrg_ingest_run": ([_p, _p, C.c_int64, _p, _i, _p], _i),
    "sdrg_lpf_taps": ([_d, _d, _p], _i),
    "sdrg_refine_plan_new": ([C.POINTER(RefineSig), _i, _d, _i, _i, _i], _p),
    "sdrg_refine_plan_free": ([_p], None),
    "sdrg_refine_plan_info": ([_p, _p], _i),
    "sdrg_refine_sums": ([_p, _p, _i, _i, _p, _p, _i, _p, _p], _i),
    "sdrg_refine_vjp": ([_p, _p, _p, _p, _p], _i),
    "sdrg_refine_gn": ([_p, _p, _i, _i, _p, _p, _p, _i, _p, _p], _i),
    "sdrg_refine_from_peaks": ([_p, _p, _i, _i, _p, _p, _p], _i),
}


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"pocketsdr_b200: {LIB_PATH} is missing; build it with "
            "`python -m pocketsdr_b200.build` (nvcc, sm_100a)")
    lib = C.CDLL(LIB_PATH)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


lib = _load()


class GpuError(RuntimeError):
    pass


def last_error() -> tuple[int, str]:
    buf = C.create_string_buffer(512)
    code = lib.sdr_gpu_last_error(buf, 512)
    return code, buf.value.decode(errors="replace")


def check(what: str = "") -> None:
    """Raises GpuError when the last call on this thread failed (and clears it)."""
    code, msg = last_error()
    if code:
        lib.sdr_gpu_clear_error()
        raise GpuError(f"{what}: {msg} (status {code})" if what else f"{msg} (status {code})")


def ptr(a) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


CUDA_STREAM_LEGACY = 1      # cudaStreamLegacy


def torch_stream() -> int:
    """Handle of torch's current CUDA stream for the C ABI. Torch's default
    stream is the legacy default stream, handle 0, but several entry points
    read a NULL stream as the calling thread's own non-blocking stream, which
    is not ordered with torch's work; the legacy stream is therefore named
    explicitly (cudaStreamLegacy), which every entry point reads the same way."""
    import torch
    return torch.cuda.current_stream().cuda_stream or CUDA_STREAM_LEGACY
