"""FFT schedules on the GPU: the autotuner times the shapes of a length and
sets the fastest; plans built under a tuned or imposed schedule give the
oracle's grids and peaks (same bars as tests/test_gpu_parity.py)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batched_vs_oracle(ref, seed):
    import test_gpu_parity as tp
    from pocketsdr_b200 import synth
    from pocketsdr_b200.acquire import AcqPlan
    wl = synth.acq_multi_24mhz(seed=seed, prn_limit=2, t_sum=2e-3, sigs=(("L1CA", 0), ("E1B", 0)))
    cf = [synth.group_code_ffts(g) for g in wl.groups]
    plan = AcqPlan(wl.groups, cf)
    res = plan.run_host(wl.bufs, wl.ix)
    k = 0
    for gi, (g, c) in enumerate(zip(wl.groups, cf)):
        G = plan.grid(gi)
        for p in range(len(g.prns)):
            Pref = tp._oracle_group_grid(ref, g, c[p], wl.bufs[g.buf], wl.ix[g.buf])
            tp.assert_power_close(G[p], Pref)
            cn0, pk = ref.corr_max(Pref, g.Nmax, g.Nmax, len(g.fds), g.T)
            assert (res[k]["bin"], res[k]["offset"]) == pk and abs(float(res[k]["cn0"]) - cn0) < 0.1
            k += 1
    plan.close()


def test_autotune_then_parity(gpu, ref):
    from pocketsdr_b200._lib import lib
    R, t, ms = C.c_int(), C.c_int(), C.c_double()
    try:
        for L in (48000, 192000):
            assert lib.sdrg_fft_autotune(L, C.byref(R), C.byref(t), C.byref(ms)) == 0
            assert L % R.value == 0 and R.value <= 8 and t.value in (256, 512) and ms.value > 0
            Rg, tg = C.c_int(), C.c_int()
            assert lib.sdrg_fft_schedule_get(L, C.byref(Rg), C.byref(tg)) == 1
            assert (Rg.value, tg.value) == (R.value, t.value)
        _batched_vs_oracle(ref, seed=21)
    finally:
        for L in (48000, 192000):
            lib.sdrg_fft_schedule_set(L, 0, 0)


@pytest.mark.parametrize("shape", [(48000, 4, 256), (48000, 2, 256), (192000, 8, 256)])
def test_imposed_schedule_parity(gpu, ref, shape):
    from pocketsdr_b200._lib import lib
    L, R, t = shape
    try:
        assert lib.sdrg_fft_schedule_set(L, R, t) == 0
        _batched_vs_oracle(ref, seed=22)
    finally:
        lib.sdrg_fft_schedule_set(L, 0, 0)
