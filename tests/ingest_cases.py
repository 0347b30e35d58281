"""Shared IF-ingest test cases: seeded receiver configurations covering every
IF data format of src/pocket_sdr.h:85-92, real (fs/4 real-to-complex) and
complex channels, 2- and 3-bit samples, LPFs and array channels."""
import numpy as np

BPS = {1: 1, 2: 2, 3: 1, 4: 2, 5: 2, 6: 4, 7: 2, 8: 4}
NRF = {3: 2, 4: 4, 5: 8, 6: 8}


def cases(N=3000, seed=0):
    """Yields (name, cfg dict) with keys fmt, N, IQ, bits, off, scale, lpf_fc,
    fs, w, arch_on."""
    rng = np.random.default_rng(seed)
    fs = 24e6
    yield "int8_rtoc_lpf", dict(fmt=1, N=N, IQ=[1], bits=[8], off=(0.4, 0.0), scale=(9.5, 1.0),
                                lpf_fc=[0.45 * 0.5 * fs], fs=fs, w=None, arch_on=None)
    yield "int8_real", dict(fmt=1, N=N, IQ=[2], bits=[8], off=(-1.0, 0.0), scale=(3.3, 1.0),
                            lpf_fc=[0.0], fs=fs, w=None, arch_on=None)
    yield "int8x2", dict(fmt=2, N=N, IQ=[2], bits=[8], off=(0.0, 0.0), scale=(12.0, 1.0),
                         lpf_fc=[3e6], fs=fs, w=None, arch_on=None)
    yield "cs8", dict(fmt=7, N=N, IQ=[2], bits=[8], off=(1.5, 0.0), scale=(20.0, 1.0),
                      lpf_fc=[0.0], fs=fs, w=None, arch_on=None)
    yield "cs16", dict(fmt=8, N=N, IQ=[2, 2], bits=[16, 16], off=(12.0, -30.0),
                       scale=(900.0, 1100.0), lpf_fc=[5e6], fs=fs, w=None, arch_on=None)
    for fmt, name in ((3, "raw8"), (4, "raw16"), (6, "raw32"), (5, "raw16i")):
        nrf = NRF[fmt]
        IQ = [1 if (k % 3 != 2) else 2 for k in range(nrf)]
        bits = [3 if IQ[k] == 1 and k % 2 == 0 else 2 for k in range(nrf)]
        lpf = [float(rng.uniform(2e6, 10e6)) if k % 2 == 0 else 0.0 for k in range(nrf)]
        w = rng.integers(-300, 301, (3, nrf, 2)).astype(np.int16)
        yield name, dict(fmt=fmt, N=N, IQ=IQ, bits=bits, off=(0.0, 0.0), scale=(1.0, 1.0),
                         lpf_fc=lpf, fs=fs, w=w, arch_on=[1, 0, 1])


def raw_blocks(cfg, n_blocks, seed=1):
    rng = np.random.default_rng(seed)
    return [rng.integers(0, 256, cfg["N"] * BPS[cfg["fmt"]], dtype=np.uint8)
            for _ in range(n_blocks)]
