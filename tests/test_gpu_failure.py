"""Failure handling without faulting the GPU: a simulated allocation
failure (sdrg_inject_alloc_failure) makes the call fail cleanly - the
reference exits the process on allocation failure (src/sdr_func.c:150-153),
here the drop-in leaves its outputs zero-filled (P unchanged), records
SDRG_ERR_NOMEM with a message, and the next call works. Each case runs on a
fresh host thread so that the thread's staging buffers are allocated anew."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NOMEM = -3


def _on_fresh_thread(fn):
    out = {}

    def run():
        try:
            out["v"] = fn()
        except BaseException as e:       # surfaced in the calling thread
            out["e"] = e
    t = threading.Thread(target=run)
    t.start()
    t.join()
    if "e" in out:
        raise out["e"]
    return out["v"]


def test_search_code_alloc_failure_leaves_P_and_recovers(gpu):
    from pocketsdr_b200 import codes, synth
    from pocketsdr_b200._lib import last_error, lib, ptr
    fs, fi, T = 4e6, 1.0e6, 1e-3
    N = int(fs * T)
    buf = synth.gen_if(4 * N, fs, {"L1CA": fi}, [synth.Sat("L1CA", 9, 311.5, 1700.0, 0.2, 48.0)],
                       iq=False, bits=2, seed=5)
    cf = codes.gen_code_fft(codes.gen_code("L1CA", 9), T, 0.0, fs, N, N)
    fds = synth.dop_bins(T, 0.0, 5000.0)

    import ctypes as C
    from pocketsdr_b200._lib import SdrBuff
    cf = np.ascontiguousarray(cf, np.complex64)
    fds = np.ascontiguousarray(fds, np.float32)
    sb = SdrBuff(buf.ctypes.data_as(C.POINTER(C.c_uint8)), 2, len(buf))

    def search(P):      # the C call, as the reference's callers make it
        lib.sdr_search_code(ptr(cf), T, C.byref(sb), 0, 2 * N, fs, fi, ptr(fds), len(fds), ptr(P))

    def call():
        P = np.full((len(fds), 2 * N), 7.0, np.float32)
        lib.sdrg_inject_alloc_failure(0)
        search(P)
        code, msg = last_error()
        lib.sdr_gpu_clear_error()
        unchanged = bool(np.all(P == 7.0))
        search(P)                                   # recovers
        code2, _ = last_error()
        return code, msg, unchanged, code2, float(P.max())
    code, msg, unchanged, code2, pmax = _on_fresh_thread(call)
    assert code == NOMEM and "simulated allocation failure" in msg
    assert unchanged
    assert code2 == 0 and pmax > 7.0


def test_mix_carr_alloc_failure_zero_fills(gpu):
    import ctypes as C
    from pocketsdr_b200._lib import SdrBuff, last_error, lib, ptr

    def call():
        buf = (np.arange(5000) % 256).astype(np.uint8)
        sb = SdrBuff(buf.ctypes.data_as(C.POINTER(C.c_uint8)), 2, len(buf))
        out = np.full((4000, 2), 5, np.int8)
        lib.sdrg_inject_alloc_failure(0)
        lib.sdr_mix_carr(C.byref(sb), 10, 4000, 4e6, 1.0e6, 0.1, ptr(out))
        code, _ = last_error()
        lib.sdr_gpu_clear_error()
        return code, out
    code, out = _on_fresh_thread(call)
    assert code == NOMEM and not out.any()


def test_plan_alloc_failure_returns_null(gpu):
    from pocketsdr_b200 import acquire, synth
    from pocketsdr_b200._lib import GpuError, lib
    wl = synth.acq_multi_24mhz(seed=3, prn_limit=2, t_sum=2e-3)
    cfs = [synth.group_code_ffts(g) for g in wl.groups]
    lib.sdrg_inject_alloc_failure(0)
    with pytest.raises(GpuError, match="simulated allocation failure"):
        acquire.AcqPlan(wl.groups, cfs)
    plan = acquire.AcqPlan(wl.groups, cfs)        # and the next plan builds
    assert plan.cells > 0
    lib.sdrg_inject_alloc_failure(-1)


CUDA_ERR = -2


def test_staged_copy_wait_bound_reported_and_cleared(gpu, ref):
    """The bounded waits for the bulk copies of a staged split (480 000
    points = 20 x 24 000): with sdrg_inject_stage_timeout the first wait of
    each copy gives up at once (the copies still land and are waited for in
    full). The synchronous drop-ins then report SDRG_ERR_CUDA - sdr_corr_fft
    zero-fills its output, sdr_search_code leaves P unchanged - and the next
    call, with the normal bound, runs and matches the reference."""
    import ctypes as C
    from pocketsdr_b200 import codes
    from pocketsdr_b200._lib import SdrBuff, last_error, lib, ptr
    N = 480000
    rng = np.random.default_rng(17)
    IQ = rng.integers(-60, 61, (N, 2), dtype=np.int8)
    cf = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    corr = np.full(N, 3.0, np.complex64)

    def corr_fft():
        lib.sdr_corr_fft(ptr(IQ), ptr(cf), N, ptr(corr))
        code, msg = last_error()
        lib.sdr_gpu_clear_error()
        return code, msg

    assert lib.sdrg_inject_stage_timeout(1) == 0
    code, msg = corr_fft()
    assert code == CUDA_ERR and "bulk copy" in msg, (code, msg)
    assert not corr.any()
    code, _ = corr_fft()
    assert code == 0
    want = ref.corr_fft(IQ, cf)
    rms = float(np.sqrt(np.mean(np.abs(want) ** 2)))
    assert np.all(np.abs(corr - want) <= 1e-4 * np.maximum(np.abs(want), rms))

    # sdr_search_code over a 480 000-sample window, 2 bins
    fs, fi, T = 48e6, 0.0, 10e-3
    buf = ((rng.integers(-7, 8, N) & 0x0F) | ((rng.integers(-7, 8, N) & 0x0F) << 4)).astype(np.uint8)
    sb = SdrBuff(buf.ctypes.data_as(C.POINTER(C.c_uint8)), 2, len(buf))
    code_fft = np.ascontiguousarray(cf)
    fds = np.array([-50.0, 50.0], np.float32)
    P = np.full((2, N), 5.0, np.float32)
    assert lib.sdrg_inject_stage_timeout(1) == 0
    lib.sdr_search_code(ptr(code_fft), T, C.byref(sb), 0, N, fs, fi, ptr(fds), 2, ptr(P))
    code, msg = last_error()
    lib.sdr_gpu_clear_error()
    assert code == CUDA_ERR and "bulk copy" in msg
    assert np.all(P == 5.0)
    lib.sdr_search_code(ptr(code_fft), T, C.byref(sb), 0, N, fs, fi, ptr(fds), 2, ptr(P))
    assert last_error()[0] == 0
    Pr = np.full((2, N), 5.0, np.float32)
    ref.search_code(code_fft, buf, 0, N, fs, fi, fds, Pr, T)
    floor = float(Pr.mean())
    assert np.all(np.abs(P - Pr) <= 1e-4 * np.maximum(np.abs(Pr), floor))
    assert lib.sdrg_inject_stage_timeout(0) == 0
