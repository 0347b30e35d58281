"""The C-ABI library: builds, loads and exports every symbol the public
header declares (no compute calls - this runs without a GPU)."""
import ctypes as C
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pocket_sdr_gpu.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b(sdrg?_\w+)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if not n.endswith("_t")))


def test_header_parses():
    names = header_functions()
    for must in ("sdr_func_init", "sdr_mix_carr", "sdr_corr_std", "sdr_corr_std_cpx_code",
                 "sdr_corr_std_cpx", "sdr_corr_fft", "sdr_corr_fft_cpx", "sdr_search_code",
                 "sdr_corr_max", "sdr_fine_dop", "sdr_dop_bins", "sdrg_acq_run"):
        assert must in names


def test_library_exports_header_symbols():
    from pocketsdr_b200 import _lib
    lib = C.CDLL(_lib.LIB_PATH)
    for name in header_functions():
        assert hasattr(lib, name), name
    # and the python binding covers exactly the header
    assert sorted(_lib.SIGNATURES) == header_functions()


def test_exported_dynamic_symbols_are_the_abi():
    from pocketsdr_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if " T " in l)
    ours = {n for n in exported if n.startswith(("sdr_", "sdrg_"))}
    assert ours == set(header_functions())


def test_fft_plan_shapes_host_only():
    """Plan selection is host logic (no device needed)."""
    from pocketsdr_b200._lib import lib
    for n in (1, 2, 4, 12, 100, 2000, 4000, 12000, 24000, 48000, 96000, 192000, 64000, 4800):
        assert lib.sdrg_fft_supported(n) == 1, n
    for n in (7, 2046 * 2 * 11, 1000003):
        assert lib.sdrg_fft_supported(n) == 0, n
