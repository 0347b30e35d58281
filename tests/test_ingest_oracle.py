"""IF-ingest checker pinned before it is trusted (CPU only): the plain-C
restatement (oracle/ingest_oracle.c) against the reference's own
src/sdr_rcv.c write_buff, table builders and src/sdr_func.c LPF, compiled
from the reference tree through oracle/rcv_shim.c; and the library's
host-side LPF taps (sdrg_lpf_taps, no device work) against the reference's
sdr_lpf_new."""
import os
import sys

import numpy as np
import pytest

from oracle import oracle

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import ingest_cases  # noqa: E402

HAVE_RCV = os.path.exists(oracle.RCV_SO)
need_ref = pytest.mark.skipif(not HAVE_RCV, reason="reference receiver build (oracle/_ref) absent")


@pytest.fixture(scope="module")
def chk():
    return oracle.Ingest("reference"), oracle.Ingest("port")


@need_ref
def test_tables_match_reference(chk):
    R, P = chk
    rng = np.random.default_rng(3)
    for fmt in (1, 2, 7, 8):
        for _ in range(20):
            off, scale = float(rng.uniform(-40, 40)), float(rng.uniform(0.01, 2000))
            assert np.array_equal(R.gen_lut8(fmt, off, scale), P.gen_lut8(fmt, off, scale))
        assert np.array_equal(R.gen_lut8(fmt, 0.0, 0.0), P.gen_lut8(fmt, 0.0, 0.0))
    for fmt in (3, 4, 5, 6):
        for k in range(8):
            for IQ in (1, 2):
                for bits in (2, 3):
                    for rtoc in (0, 1):
                        assert np.array_equal(R.gen_lutc(fmt, k, IQ, bits, rtoc),
                                              P.gen_lutc(fmt, k, IQ, bits, rtoc)), (fmt, k, IQ, bits)


@need_ref
def test_lpf_taps_match_reference(chk):
    """The restatement's and the library's taps (host code) equal the
    reference build's over a sweep of cutoffs and rates."""
    from pocketsdr_b200 import ingest
    R, P = chk
    rng = np.random.default_rng(5)
    for _ in range(400):
        fs = float(rng.choice([2.048e6, 4e6, 12e6, 24e6, 48e6, 64e6]) * rng.uniform(0.9, 1.1))
        fc = float(rng.uniform(-0.05, 0.55) * fs)
        r = R.lpf_taps(fc, fs)
        p = P.lpf_taps(fc, fs)
        g = ingest.lpf_taps(fc, fs)
        if r is None:
            assert p is None and g is None
        else:
            assert np.array_equal(r, p) and np.array_equal(r, g), (fc, fs, r, p, g)


@need_ref
@pytest.mark.parametrize("N", [3000, 5])
def test_write_buff_restatement_matches_reference(chk, N):
    R, P = chk
    for name, cfg in ingest_cases.cases(N=N):
        a = R.receiver(**cfg)
        b = P.receiver(**cfg)
        for ix, raw in enumerate(ingest_cases.raw_blocks(cfg, 4, seed=N)):
            x = a.write(raw, ix + 5)
            y = b.write(raw, ix + 5)
            assert np.array_equal(x, y), (name, ix)


@need_ref
def test_lpf_apply_restatement_matches_reference(chk):
    R, P = chk
    rng = np.random.default_rng(9)
    a, b = R.lpf(4e6, 16e6), P.lpf(4e6, 16e6)
    for n in (3, 1000, 2048, 7, 1, 5000):
        d = rng.integers(0, 256, n, dtype=np.uint8)
        assert np.array_equal(a.apply(d), b.apply(d)), n
