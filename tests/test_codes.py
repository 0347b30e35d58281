"""Spreading-code generators of the library (sdrg_gen_code / sdrg_sec_code,
host code, no device work) against the reference build's sdr_gen_code /
sdr_sec_code (src/sdr_code.c:2173-2182, :2274-2283): every PRN of every
signal generated, chip for chip."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle

HAVE_REF = oracle.reference_available()

SIGNAL_PRNS = [
    ("L1CA", range(1, 211), 1023),
    ("L5I", range(1, 211), 10230),
    ("L5Q", range(1, 211), 10230),
    ("L6D", range(193, 203), 20460),
    ("L6E", range(203, 213), 20460),
    ("E1B", range(1, 51), 8184),
    ("B1I", range(1, 64), 2046),
]


@pytest.mark.skipif(not HAVE_REF, reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("sig,prns,n", SIGNAL_PRNS, ids=[s[0] for s in SIGNAL_PRNS])
def test_primary_codes_match_reference(sig, prns, n):
    from pocketsdr_b200 import codes
    R = oracle.Reference()
    for prn in prns:
        got = codes.gen_code(sig, prn)
        assert len(got) == n
        assert np.array_equal(got, R.gen_code(sig, prn)), (sig, prn)


@pytest.mark.skipif(not HAVE_REF, reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("sig,prns,n", SIGNAL_PRNS, ids=[s[0] for s in SIGNAL_PRNS])
def test_secondary_codes_match_reference(sig, prns, n):
    from pocketsdr_b200 import codes
    R = oracle.Reference()
    for prn in prns:
        assert np.array_equal(codes.sec_code(sig, prn), R.sec_code(sig, prn)), (sig, prn)


def test_code_properties():
    """Size-independent facts of the codes, also without the reference build:
    balanced Gold / memory codes, BOC(1,1) half-chips of opposite sign, the
    time multiplex of L6D / L6E, the published overlays."""
    from pocketsdr_b200 import codes
    c = codes.gen_code("L1CA", 1)
    assert set(np.unique(c)) == {-1, 1} and abs(int(c.sum())) <= 65
    e = codes.gen_code("E1B", 11)
    assert np.array_equal(e[1::2], -e[0::2])
    d, f = codes.gen_code("L6D", 193), codes.gen_code("L6E", 203)
    assert not d[1::2].any() and not f[0::2].any() and np.all(np.abs(d[0::2]) == 1)
    bits = lambda s: np.array([-1 if ch == "1" else 1 for ch in s], np.int8)
    assert np.array_equal(codes.sec_code("L5I", 3), bits("0000110101"))
    assert np.array_equal(codes.sec_code("L5Q", 3), bits("00000100110101001110"))
    assert np.array_equal(codes.sec_code("B1I", 6), bits("00000100110101001110"))
    assert np.array_equal(codes.sec_code("B1I", 3), np.ones(1, np.int8))
    assert np.array_equal(codes.sec_code("L5I", 135), bits("01"))
    assert np.array_equal(codes.sec_code("e1b", 5), np.ones(1, np.int8))


def test_errors():
    from pocketsdr_b200 import _lib
    lib = _lib.lib
    buf = np.zeros(100, np.int8)
    for sig, prn in (("L1CA", 0), ("L1CA", 211), ("L6D", 192), ("E1B", 51), ("XYZ", 1)):
        assert lib.sdrg_gen_code(sig.encode(), prn, None, 0) == -1
        lib.sdr_gpu_clear_error()
    assert lib.sdrg_gen_code(b"l1ca", 1, None, 0) == 1023
    assert lib.sdrg_gen_code(b"L1CA", 1, C.c_void_p(buf.ctypes.data), 100) == -1
    assert "do not fit" in _lib.last_error()[1]
    lib.sdr_gpu_clear_error()
    assert not buf.any()
