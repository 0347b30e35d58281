"""Test-only CPU oracle for Pocket SDR's search / correlation hot path.

Two checkers live here, both test infrastructure (used by tests/, the smoke
check and the CPU-baseline leg of bench.py; never by the product path):

* ``Restatement`` - ctypes wrapper over ``_build/liboracle.so``, the plain C
  restatement in ``sdr_oracle.c`` (each function cites the reference lines it
  follows).
* ``Reference`` - ctypes wrapper over ``_ref/libsdr_ref.so``, the reference's
  own ``src/sdr_func.c`` + ``src/sdr_code.c`` compiled from source by
  ``oracle/Makefile`` with the reference's flags. Present wherever ``make ref``
  ran (the .so travels with the repository snapshot).

Both expose the same numpy-level API:
  mix_carr(buff_u8, ix, N, fs, fc, phi) -> int8[N, 2]
  corr_std(IQ_i8[N,2], code_i8[10*N,2], coff, pos, cpx_code) -> (corr c64[n], C c64[2])
  corr_fft(IQ_i8[N,2], code_fft_c64[N]) -> c64[N]
  search_code(code_fft_c64[N], buff_u8, ix, N, fs, fi, fds, P_f32[len_fds,N]) (in/out)
  corr_max(P, N, Nmax, M, T) -> (cn0, (bin, offset))
  fine_dop(P, N, fds, ix) -> float
  dop_bins(T, dop, max_dop) -> f32[]
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libsdr_ref.so")
ORC_SO = os.path.join(HERE, "_build", "liboracle.so")

_p = C.c_void_p
_i = C.c_int
_d = C.c_double
_f = C.c_float


def build(ref_root: str | None = None) -> None:
    """Compile the restatement and, given the Pocket SDR source tree (argument
    or the POCKETSDR_REF environment variable), the reference library."""
    ref_root = ref_root or os.environ.get("POCKETSDR_REF")
    targets = ["oracle"]
    if ref_root and os.path.isdir(os.path.join(ref_root, "src")):
        targets.append("ref")
        # the reference's unit test and pocket_acq relinked against the GPU
        # library (which the package build makes first)
        if os.path.exists(os.path.join(HERE, "..", "pocketsdr_b200", "lib", "libsdr_gpu.so")):
            targets.append("linktest")
    cmd = ["make", "-s", "-C", HERE] + targets
    if ref_root:
        cmd.append("REF=" + os.path.abspath(ref_root))
    subprocess.run(cmd, check=True)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_p)


class _SdrBuff(C.Structure):
    # sdr_buff_t layout (src/pocket_sdr.h:242-245)
    _fields_ = [("data", C.POINTER(C.c_uint8)), ("IQ", C.c_int), ("N", C.c_int)]


class Restatement:
    """The oracle's own C restatement (oracle/sdr_oracle.c)."""

    kind = "port"

    def __init__(self, path: str = ORC_SO):
        if not os.path.exists(path):
            build()
        L = self.lib = C.CDLL(path)
        L.orc_init.argtypes = []
        L.orc_mix_table.restype = C.POINTER(C.c_int8)
        L.orc_mix_carr.argtypes = [_p, _i, _i, _i, _d, _d, _d, _p]
        L.orc_mix_carr_cpx.argtypes = [_p, _i, _i, _i, _d, _d, _d, _p]
        L.orc_corr_std.argtypes = [_p, _p, _i, _d, _p, _i, _i, _p, _p]
        L.orc_corr_std_cpx.argtypes = [_p, _i, _i, _i, _d, _d, _d, _p, _p, _i, _p]
        L.orc_fft.argtypes = [_p, _i, _i, _p]
        L.orc_corr_fft.argtypes = [_p, _p, _i, _p]
        L.orc_corr_fft_cpx.argtypes = [_p, _i, _i, _i, _d, _d, _d, _p, _p]
        L.orc_psd_cpx.argtypes = [_p, _i, _i, _d, _i, _p]
        L.orc_csk.argtypes = [_p, _i, _i, _p, _i, _p, _p]
        L.orc_search_code.argtypes = [_p, _p, _i, _i, _i, _d, _d, _p, _i, _p]
        L.orc_corr_max.argtypes = [_p, _i, _i, _i, _d, _p]
        L.orc_corr_max.restype = _f
        L.orc_fine_dop.argtypes = [_p, _i, _p, _i, _p]
        L.orc_fine_dop.restype = _d
        L.orc_dop_bins.argtypes = [_d, _f, _f, _p]
        L.orc_res_code.argtypes = [_p, _p, _i, _d, _d, _d, _i, _i, _p]
        L.orc_gen_code_fft.argtypes = [_p, _p, _i, _d, _d, _d, _i, _i, _p]
        L.orc_refine_sums.argtypes = [_p, _i, _d, _d, _d, _p, _p, _i, _d, _i, _i, _i, _p]
        L.orc_refine_step.argtypes = [_p, _i, _i, _d, _d, _d, _i, _p, _p, _p]
        L.orc_init()

    def mix_table(self) -> np.ndarray:
        t = self.lib.orc_mix_table()
        return np.ctypeslib.as_array(t, shape=(65536, 2)).copy()

    def mix_carr(self, buff, ix, N, fs, fc, phi):
        buff = np.ascontiguousarray(buff, np.uint8)
        out = np.zeros((N, 2), np.int8)
        self.lib.orc_mix_carr(_ptr(buff), len(buff), ix, N, fs, fc, phi, _ptr(out))
        return out

    def mix_carr_cpx(self, buff, ix, N, fs, fc, phi):
        buff = np.ascontiguousarray(buff, np.complex64)
        out = np.zeros((N, 2), np.int8)
        self.lib.orc_mix_carr_cpx(_ptr(buff), len(buff), ix, N, fs, fc, phi, _ptr(out))
        return out

    def corr_std(self, IQ, code, coff, pos, cpx_code=False):
        IQ = np.ascontiguousarray(IQ, np.int8)
        code = np.ascontiguousarray(code, np.int8)
        pos = np.ascontiguousarray(pos, np.float64)
        N = IQ.shape[0]
        corr = np.zeros(len(pos), np.complex64)
        Cb = np.zeros(2, np.complex64)
        self.lib.orc_corr_std(_ptr(IQ), _ptr(code), N, coff, _ptr(pos), len(pos),
                              int(cpx_code), _ptr(corr), _ptr(Cb))
        return corr, Cb

    def corr_std_cpx(self, buff, ix, N, fs, fc, phi, code, pos):
        buff = np.ascontiguousarray(buff, np.complex64)
        code = np.ascontiguousarray(code, np.float32)
        pos = np.ascontiguousarray(pos, np.float64)
        corr = np.zeros(len(pos), np.complex64)
        self.lib.orc_corr_std_cpx(_ptr(buff), len(buff), ix, N, fs, fc, phi,
                                  _ptr(code), _ptr(pos), len(pos), _ptr(corr))
        return corr

    def fft(self, x, inverse=False):
        x = np.ascontiguousarray(x, np.complex128)
        out = np.zeros_like(x)
        self.lib.orc_fft(_ptr(x), len(x), int(inverse), _ptr(out))
        return out

    def corr_fft(self, IQ, code_fft):
        IQ = np.ascontiguousarray(IQ, np.int8)
        code_fft = np.ascontiguousarray(code_fft, np.complex64)
        out = np.zeros(IQ.shape[0], np.complex64)
        self.lib.orc_corr_fft(_ptr(IQ), _ptr(code_fft), IQ.shape[0], _ptr(out))
        return out

    def corr_fft_cpx(self, buff, ix, N, fs, fc, phi, code_fft):
        buff = np.ascontiguousarray(buff, np.complex64)
        code_fft = np.ascontiguousarray(code_fft, np.complex64)
        out = np.zeros(N, np.complex64)
        self.lib.orc_corr_fft_cpx(_ptr(buff), len(buff), ix, N, fs, fc, phi,
                                  _ptr(code_fft), _ptr(out))
        return out

    def psd_cpx(self, buff, N, fs, IQ):
        buff = np.ascontiguousarray(buff, np.complex64)
        out = np.zeros(N // 2 if IQ == 1 else N, np.float32)
        self.lib.orc_psd_cpx(_ptr(buff), len(buff), N, fs, IQ, _ptr(out))
        return out

    def csk(self, corr, len_code, pos):
        """L6 CSK decode: (symbol, taps complex64[len(pos)])."""
        corr = np.ascontiguousarray(corr, np.complex64)
        pos = np.ascontiguousarray(pos, np.float64)
        sym = np.zeros(1, np.uint8)
        C = np.zeros(len(pos), np.complex64)
        self.lib.orc_csk(_ptr(corr), len(corr), len_code, _ptr(pos), len(pos), _ptr(sym), _ptr(C))
        return int(sym[0]), C

    def search_code(self, code_fft, buff, ix, N, fs, fi, fds, P):
        code_fft = np.ascontiguousarray(code_fft, np.complex64)
        buff = np.ascontiguousarray(buff, np.uint8)
        fds = np.ascontiguousarray(fds, np.float32)
        assert P.dtype == np.float32 and P.flags.c_contiguous
        self.lib.orc_search_code(_ptr(code_fft), _ptr(buff), len(buff), ix, N, fs, fi,
                                 _ptr(fds), len(fds), _ptr(P))
        return P

    def corr_max(self, P, N, Nmax, M, T):
        P = np.ascontiguousarray(P, np.float32)
        ix = np.zeros(2, np.int32)
        cn0 = self.lib.orc_corr_max(_ptr(P), N, Nmax, M, T, _ptr(ix))
        return float(cn0), (int(ix[0]), int(ix[1]))

    def fine_dop(self, P, N, fds, ix):
        P = np.ascontiguousarray(P, np.float32)
        fds = np.ascontiguousarray(fds, np.float32)
        ixa = np.asarray(ix, np.int32)
        return float(self.lib.orc_fine_dop(_ptr(P), N, _ptr(fds), len(fds), _ptr(ixa)))

    def dop_bins(self, T, dop, max_dop):
        n = self.lib.orc_dop_bins(T, dop, max_dop, None)
        out = np.zeros(n, np.float32)
        self.lib.orc_dop_bins(T, dop, max_dop, _ptr(out))
        return out

    def res_code(self, code_I, code_Q, T, coff, fs, N, Nz):
        code_I = np.ascontiguousarray(code_I, np.int8)
        cq = None if code_Q is None else np.ascontiguousarray(code_Q, np.int8)
        out = np.zeros((N + Nz, 2), np.int8)
        self.lib.orc_res_code(_ptr(code_I), None if cq is None else _ptr(cq), len(code_I),
                              T, coff, fs, N, Nz, _ptr(out))
        return out

    def gen_code_fft(self, code_I, code_Q, T, coff, fs, N, Nz):
        code_I = np.ascontiguousarray(code_I, np.int8)
        cq = None if code_Q is None else np.ascontiguousarray(code_Q, np.int8)
        out = np.zeros(N + Nz, np.complex64)
        self.lib.orc_gen_code_fft(_ptr(code_I), None if cq is None else _ptr(cq),
                                  len(code_I), T, coff, fs, N, Nz, _ptr(out))
        return out

    # ---- refinement model (refine_oracle.c; FP64, no reference counterpart) --

    REFINE_W = 12

    def refine_sums(self, chips, rate_nom, rate, fi, theta, buf, iq, fs, ix0, Nb, K):
        """float64 [K, 12] block sums of one signal (see refine_oracle.c)."""
        chips = np.ascontiguousarray(chips, np.int8)
        buf = np.ascontiguousarray(buf, np.uint8)
        th = np.ascontiguousarray(theta, np.float64)
        if ix0 < 0 or ix0 + K * Nb > len(buf):
            raise ValueError("refine span outside the buffer")
        out = np.zeros((K, self.REFINE_W), np.float64)
        self.lib.orc_refine_sums(_ptr(chips), len(chips), rate_nom, rate, fi, _ptr(th),
                                 _ptr(buf), int(iq), fs, ix0, Nb, K, _ptr(out))
        return out

    def refine_step(self, sums, Nb, fs, rate_nom, fc, theta, rate, model=1):
        """One Gauss-Newton step (model 0 power, 1 coherent, 2 coherent with
        per-block signs): returns (theta', rate', info[5])."""
        sums = np.ascontiguousarray(sums, np.float64)
        th = np.array(theta, np.float64)
        r = np.array([rate], np.float64)
        info = np.zeros(5, np.float64)
        self.lib.orc_refine_step(_ptr(sums), sums.shape[0], Nb, fs, rate_nom, fc,
                                 int(model), _ptr(th), _ptr(r), _ptr(info))
        return th, float(r[0]), info

    @staticmethod
    def refine_corr(sums):
        """Complex C_k of block sums."""
        return sums[:, 0] + 1j * sums[:, 1]

    @staticmethod
    def refine_vjp(sums, g, rate_nom, Nb, fs):
        """FP64 vector-Jacobian product: d/dtheta of sum_k Re(conj(g_k) C_k)
        for upstream gradients g_k (complex) - the analytic gradient the GPU
        backward computes, from FP64 sums. dC/dtau = -rate_nom D,
        dC/dfd = -2 pi j (E + dt_k C), dC/dphi = -2 pi j C."""
        K = sums.shape[0]
        Cc = sums[:, 0] + 1j * sums[:, 1]
        D = sums[:, 2] + 1j * sums[:, 3]
        E = sums[:, 4] + 1j * sums[:, 5]
        dt = (np.arange(K) + 0.5 - 0.5 * K) * Nb / fs
        g = np.asarray(g, np.complex128)
        d_tau = np.sum(np.real(np.conj(g) * (-rate_nom * D)))
        d_fd = np.sum(np.real(np.conj(g) * (-2j * np.pi * (E + dt * Cc))))
        d_phi = np.sum(np.real(np.conj(g) * (-2j * np.pi * Cc)))
        return np.array([d_tau, d_fd, d_phi])

    def refine_gn(self, chips, rate_nom, fc, fi, theta, buf, iq, fs, ix0, Nb, K, models):
        """Gauss-Newton steps from theta, one per entry of `models` (the model
        of each step); the code rate follows the carrier. Returns
        (theta, rate, [info per step])."""
        th = np.array(theta, np.float64)
        rate = rate_nom * (1.0 + th[1] / fc) if fc > 0 else rate_nom
        infos = []
        for m in models:
            s = self.refine_sums(chips, rate_nom, rate, fi, th, buf, iq, fs, ix0, Nb, K)
            th, rate, info = self.refine_step(s, Nb, fs, rate_nom, fc, th, rate, model=m)
            infos.append(info)
        return th, rate, infos


class Reference:
    """The reference's own C functions, compiled from its sources."""

    kind = "reference"

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = self.lib = C.CDLL(path)
        L.sdr_func_init.argtypes = [C.c_char_p]
        L.sdr_mix_carr.argtypes = [C.POINTER(_SdrBuff), _i, _i, _d, _d, _d, _p]
        L.sdr_corr_std.argtypes = [_p, _p, _i, _d, _p, _i, _p, _p]
        L.sdr_corr_std_cpx_code.argtypes = [_p, _p, _i, _d, _p, _i, _p, _p]
        L.sdr_corr_std_cpx.argtypes = [_p, _i, _i, _i, _d, _d, _d, _p, _p, _i, _p]
        L.sdr_corr_fft.argtypes = [_p, _p, _i, _p]
        L.sdr_corr_fft_cpx.argtypes = [_p, _i, _i, _i, _d, _d, _d, _p, _p]
        L.sdr_search_code.argtypes = [_p, _d, C.POINTER(_SdrBuff), _i, _i, _d, _d, _p, _i, _p]
        L.sdr_corr_max.argtypes = [_p, _i, _i, _i, _d, _p]
        L.sdr_corr_max.restype = _f
        L.sdr_fine_dop.argtypes = [_p, _i, _p, _i, _p]
        L.sdr_fine_dop.restype = _d
        L.sdr_dop_bins.argtypes = [_d, _f, _f, C.POINTER(_i)]
        L.sdr_dop_bins.restype = C.POINTER(_f)
        L.sdr_gen_code.argtypes = [C.c_char_p, _i, C.POINTER(_i)]
        L.sdr_gen_code.restype = C.POINTER(C.c_int8)
        L.sdr_sec_code.argtypes = [C.c_char_p, _i, C.POINTER(_i)]
        L.sdr_sec_code.restype = C.POINTER(C.c_int8)
        L.sdr_code_cyc.argtypes = [C.c_char_p]
        L.sdr_code_cyc.restype = _d
        L.sdr_res_code.argtypes = [_p, _p, _i, _d, _d, _d, _i, _i, _p]
        L.sdr_gen_code_fft.argtypes = [_p, _p, _i, _d, _d, _d, _i, _i, _p]
        L.sdr_cpx_fft.argtypes = [_p, _i, _i, _p]
        L.sdr_cpx_fft.restype = _i
        L.sdr_free.argtypes = [_p]
        L.sdr_psd_cpx.argtypes = [_p, _i, _i, _d, _i, _p]
        L.sdr_func_init(b"")

    def _buff(self, buff):
        b = np.ascontiguousarray(buff, np.uint8)
        sb = _SdrBuff(b.ctypes.data_as(C.POINTER(C.c_uint8)), 2, len(b))
        return b, sb

    def mix_carr(self, buff, ix, N, fs, fc, phi):
        b, sb = self._buff(buff)
        out = np.zeros((N, 2), np.int8)
        self.lib.sdr_mix_carr(C.byref(sb), ix, N, fs, fc, phi, _ptr(out))
        return out

    def corr_std(self, IQ, code, coff, pos, cpx_code=False):
        IQ = np.ascontiguousarray(IQ, np.int8)
        code = np.ascontiguousarray(code, np.int8)
        pos = np.ascontiguousarray(pos, np.float64)
        corr = np.zeros(len(pos), np.complex64)
        Cb = np.zeros(2, np.complex64)
        fn = self.lib.sdr_corr_std_cpx_code if cpx_code else self.lib.sdr_corr_std
        fn(_ptr(IQ), _ptr(code), IQ.shape[0], coff, _ptr(pos), len(pos), _ptr(corr), _ptr(Cb))
        return corr, Cb

    def corr_std_cpx(self, buff, ix, N, fs, fc, phi, code, pos):
        buff = np.ascontiguousarray(buff, np.complex64)
        code = np.ascontiguousarray(code, np.float32)
        pos = np.ascontiguousarray(pos, np.float64)
        corr = np.zeros(len(pos), np.complex64)
        self.lib.sdr_corr_std_cpx(_ptr(buff), len(buff), ix, N, fs, fc, phi,
                                  _ptr(code), _ptr(pos), len(pos), _ptr(corr))
        return corr

    def fft(self, x, inverse=False):
        x = np.ascontiguousarray(x, np.complex64)
        out = np.zeros_like(x)
        self.lib.sdr_cpx_fft(_ptr(x), len(x), int(inverse), _ptr(out))
        return out

    def corr_fft(self, IQ, code_fft):
        IQ = np.ascontiguousarray(IQ, np.int8)
        code_fft = np.ascontiguousarray(code_fft, np.complex64)
        out = np.zeros(IQ.shape[0], np.complex64)
        self.lib.sdr_corr_fft(_ptr(IQ), _ptr(code_fft), IQ.shape[0], _ptr(out))
        return out

    def corr_fft_cpx(self, buff, ix, N, fs, fc, phi, code_fft):
        buff = np.ascontiguousarray(buff, np.complex64)
        code_fft = np.ascontiguousarray(code_fft, np.complex64)
        out = np.zeros(N, np.complex64)
        self.lib.sdr_corr_fft_cpx(_ptr(buff), len(buff), ix, N, fs, fc, phi,
                                  _ptr(code_fft), _ptr(out))
        return out

    def psd_cpx(self, buff, N, fs, IQ):
        buff = np.ascontiguousarray(buff, np.complex64)
        out = np.zeros(N // 2 if IQ == 1 else N, np.float32)
        self.lib.sdr_psd_cpx(_ptr(buff), len(buff), N, fs, IQ, _ptr(out))
        return out

    def sleep_cost(self, n: int = 40) -> float:
        """Mean seconds of the reference's sdr_sleep_msec(1), the CPU release
        sdr_search_code makes after every 22nd Doppler bin
        (src/sdr_func.c:681-683)."""
        import time
        self.lib.sdr_sleep_msec.argtypes = [_i]
        t0 = time.perf_counter()
        for _ in range(n):
            self.lib.sdr_sleep_msec(1)
        return (time.perf_counter() - t0) / n

    def search_code(self, code_fft, buff, ix, N, fs, fi, fds, P, T=1e-3):
        code_fft = np.ascontiguousarray(code_fft, np.complex64)
        b, sb = self._buff(buff)
        fds = np.ascontiguousarray(fds, np.float32)
        assert P.dtype == np.float32 and P.flags.c_contiguous
        self.lib.sdr_search_code(_ptr(code_fft), T, C.byref(sb), ix, N, fs, fi,
                                 _ptr(fds), len(fds), _ptr(P))
        return P

    def corr_max(self, P, N, Nmax, M, T):
        P = np.ascontiguousarray(P, np.float32)
        ix = np.zeros(2, np.int32)
        cn0 = self.lib.sdr_corr_max(_ptr(P), N, Nmax, M, T, _ptr(ix))
        return float(cn0), (int(ix[0]), int(ix[1]))

    def fine_dop(self, P, N, fds, ix):
        P = np.ascontiguousarray(P, np.float32)
        fds = np.ascontiguousarray(fds, np.float32)
        ixa = np.asarray(ix, np.int32)
        return float(self.lib.sdr_fine_dop(_ptr(P), N, _ptr(fds), len(fds), _ptr(ixa)))

    def dop_bins(self, T, dop, max_dop):
        n = _i(0)
        p = self.lib.sdr_dop_bins(T, dop, max_dop, C.byref(n))
        out = np.ctypeslib.as_array(p, shape=(n.value,)).copy()
        self.lib.sdr_free(C.cast(p, _p))
        return out

    def gen_code(self, sig: str, prn: int) -> np.ndarray:
        n = _i(0)
        p = self.lib.sdr_gen_code(sig.encode(), prn, C.byref(n))
        if not p:
            raise ValueError(f"no code for {sig} {prn}")
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy()

    def sec_code(self, sig: str, prn: int) -> np.ndarray:
        n = _i(0)
        p = self.lib.sdr_sec_code(sig.encode(), prn, C.byref(n))
        if not p:
            raise ValueError(f"no secondary code for {sig} {prn}")
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy()

    def code_cyc(self, sig: str) -> float:
        return float(self.lib.sdr_code_cyc(sig.encode()))

    def res_code(self, code_I, code_Q, T, coff, fs, N, Nz):
        code_I = np.ascontiguousarray(code_I, np.int8)
        cq = None if code_Q is None else np.ascontiguousarray(code_Q, np.int8)
        out = np.zeros((N + Nz, 2), np.int8)
        self.lib.sdr_res_code(_ptr(code_I), None if cq is None else _ptr(cq), len(code_I),
                              T, coff, fs, N, Nz, _ptr(out))
        return out

    def gen_code_fft(self, code_I, code_Q, T, coff, fs, N, Nz):
        code_I = np.ascontiguousarray(code_I, np.int8)
        cq = None if code_Q is None else np.ascontiguousarray(code_Q, np.int8)
        out = np.zeros(N + Nz, np.complex64)
        self.lib.sdr_gen_code_fft(_ptr(code_I), None if cq is None else _ptr(cq),
                                  len(code_I), T, coff, fs, N, Nz, _ptr(out))
        return out


def search_groups(groups, bufs, code_ffts, gpu_res=None, keep=None, max_threads=None) -> dict:
    """The reference's search path over every PRN of every signal group, on
    this host's cores: per (group, PRN), sdr_search_code over every
    non-coherent sum (src/sdr_func.c:664-687, with its 1 ms CPU release every
    22 bins) into one grid, then sdr_corr_max and sdr_fine_dop
    (src/sdr_func.c:690-744), as search_sig does per channel
    (src/sdr_ch.c:420-432); one PRN search per thread, the longest first.
    Groups are objects with prns, fs, fi, T, N (sum advance), L (FFT length),
    Nmax, n_sum, fds (float32) and buf (index into bufs); code_ffts[g] holds
    the conjugated code DFTs [n_prn, L].

    Returns wall_s, cores, kind, "res" (per PRN in group order: bin, offset,
    cn0, fd, pmax = the grid maximum, pmean = the grid mean over the Nmax kept
    columns and, with gpu_res - per-PRN results in the same order - at_gpu,
    the reference grid at the cell the GPU reported) and "grids"
    ({g: (prn index, grid[n_bin, Nmax])} for the rows named by keep =
    {g: prn index})."""
    import concurrent.futures as cf
    import time
    R = best()
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    threads = min(cores, max_threads or cores)
    keep = keep or {}
    offs = np.cumsum([0] + [len(g.prns) for g in groups])
    tasks = [(gi, pi) for gi, g in enumerate(groups) for pi in range(len(g.prns))]
    tasks.sort(key=lambda t: -len(groups[t[0]].fds) * groups[t[0]].n_sum * groups[t[0]].L)
    out = np.zeros(int(offs[-1]), [("bin", np.int32), ("offset", np.int32),
                                   ("cn0", np.float64), ("fd", np.float64),
                                   ("at_gpu", np.float64), ("pmax", np.float64),
                                   ("pmean", np.float64)])
    grids = {}

    def one(t):
        gi, pi = t
        g = groups[gi]
        buf = bufs[g.buf]
        fds = np.ascontiguousarray(g.fds, np.float32)
        P = np.zeros((len(fds), g.L), np.float32)
        for s in range(g.n_sum):
            R.search_code(code_ffts[gi][pi], buf, (s * g.N) % len(buf), g.L, g.fs, g.fi, fds, P,
                          g.T)
        cn0, (b, o) = R.corr_max(P, g.L, g.Nmax, len(fds), g.T)
        k = int(offs[gi]) + pi
        out[k]["bin"], out[k]["offset"], out[k]["cn0"] = b, o, cn0
        out[k]["fd"] = R.fine_dop(P, g.L, fds, (b, o))
        out[k]["pmax"] = float(P[b, o])
        out[k]["pmean"] = float(P[:, :g.Nmax].mean(dtype=np.float64))
        if gpu_res is not None:
            gb, go = int(gpu_res[k]["bin"]), int(gpu_res[k]["offset"])
            ok = 0 <= gb < len(fds) and 0 <= go < g.Nmax
            out[k]["at_gpu"] = float(P[gb, go]) if ok else np.nan
        if keep.get(gi) == pi:
            grids[gi] = (pi, P[:, :g.Nmax].copy())

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(one, tasks))
    return {"wall_s": time.perf_counter() - t0, "cores": threads, "kind": R.kind, "res": out,
            "grids": grids}


def reference_available() -> bool:
    return os.path.exists(REF_SO)


RCV_SO = os.path.join(HERE, "_ref", "librcv_ref.so")


class Ingest:
    """IF-ingest checker: raw front-end blocks -> packed cpx8 buffers with the
    per-channel LPF and the array combine. kind "reference": the reference's
    own src/sdr_rcv.c write_buff through rcv_shim.c (_ref/librcv_ref.so);
    kind "port": the restatement in ingest_oracle.c."""

    def __init__(self, kind: str | None = None):
        if kind is None:
            kind = "reference" if os.path.exists(RCV_SO) else "port"
        self.kind = kind
        if kind == "reference":
            L = C.CDLL(RCV_SO)
            names = dict(lut8="orr_gen_lut8", lutc="orr_gen_lutc", taps="orr_lpf_taps",
                         new="orr_rcv_new", write="orr_write_buff", free="orr_rcv_free",
                         lpf_new="orr_lpf_new", lpf_apply="orr_lpf_apply", lpf_free="orr_lpf_free")
        else:
            L = C.CDLL(ORC_SO)
            names = dict(lut8="orc_gen_lut8", lutc="orc_gen_lutc", taps="orc_lpf_taps",
                         new="orc_ingest_new", write="orc_ingest_write", free="orc_ingest_free",
                         lpf_new="orc_lpf_new", lpf_apply="orc_lpf_apply", lpf_free="orc_lpf_free")
        f = {k: getattr(L, v) for k, v in names.items()}
        f["lut8"].argtypes = [_i, _d, _d, _p]
        f["lutc"].argtypes = [_i, _i, _i, _i, _i, _p]
        f["taps"].argtypes = [_d, _d, _p]
        f["taps"].restype = _i
        f["new"].argtypes = [_i, _i, _p, _p, _p, _p, _p, _d, _i, _p, _p]
        f["new"].restype = _p
        f["write"].argtypes = [_p, _p, C.c_int64, _p]
        f["free"].argtypes = [_p]
        f["lpf_new"].argtypes = [_d, _d]
        f["lpf_new"].restype = _p
        f["lpf_apply"].argtypes = [_p, _p, _i]
        f["lpf_free"].argtypes = [_p]
        self.f, self.lib = f, L

    def gen_lut8(self, fmt, off, scale):
        out = np.zeros(65536 if fmt == 8 else 256, np.int8)
        self.f["lut8"](fmt, off, scale, _ptr(out))
        return out

    def gen_lutc(self, fmt, rfch, IQ, bits, rtoc):
        out = np.zeros(1024 if rtoc else 256, np.uint8)
        self.f["lutc"](fmt, rfch, IQ, bits, int(rtoc), _ptr(out))
        return out

    def lpf_taps(self, fc, fs):
        h = np.zeros(9, np.int32)
        return h if self.f["taps"](fc, fs, _ptr(h)) else None

    def receiver(self, fmt, N, IQ, bits, off=(0.0, 0.0), scale=(1.0, 1.0), lpf_fc=None, fs=1.0,
                 w=None, arch_on=None):
        return _IngestState(self, fmt, N, IQ, bits, off, scale, lpf_fc, fs, w, arch_on)

    def lpf(self, fc, fs):
        return _LpfState(self, fc, fs)


class _IngestState:
    def __init__(self, chk, fmt, N, IQ, bits, off, scale, lpf_fc, fs, w, arch_on):
        self.chk, self.N = chk, N
        self.nrf = {3: 2, 4: 4, 5: 8, 6: 8}.get(fmt, 1)
        iq = np.zeros(8, np.int32); iq[:len(IQ)] = IQ
        bt = np.zeros(8, np.int32); bt[:len(bits)] = bits
        fc = np.zeros(8, np.float64)
        if lpf_fc is not None:
            fc[:len(lpf_fc)] = lpf_fc
        self.narch = 0 if w is None else len(w)
        wa = np.zeros((max(self.narch, 1), self.nrf, 2), np.int16)
        if self.narch:
            wa[:] = np.asarray(w, np.int16).reshape(self.narch, self.nrf, 2)
        on = np.ones(8, np.int32)
        if arch_on is not None:
            on[:len(arch_on)] = arch_on
        o = np.asarray(off, np.float64)
        s = np.asarray(scale, np.float64)
        self._keep = (iq, bt, fc, wa, on, o, s)
        self.h = chk.f["new"](fmt, N, _ptr(iq), _ptr(bt), _ptr(o), _ptr(s), _ptr(fc), fs,
                              self.narch, _ptr(wa), _ptr(on))

    def write(self, raw, ix):
        """One block: uint8 [(n_rf + narch), N]."""
        raw = np.ascontiguousarray(raw, np.uint8)
        out = np.zeros((self.nrf + self.narch, self.N), np.uint8)
        self.chk.f["write"](self.h, _ptr(raw), int(ix), _ptr(out))
        return out

    def __del__(self):
        if getattr(self, "h", None):
            self.chk.f["free"](self.h)
            self.h = None


class _LpfState:
    def __init__(self, chk, fc, fs):
        self.chk = chk
        self.h = chk.f["lpf_new"](fc, fs)

    def apply(self, data):
        d = np.array(data, np.uint8)
        self.chk.f["lpf_apply"](self.h, _ptr(d), len(d))
        return d

    def __del__(self):
        if getattr(self, "h", None):
            self.chk.f["lpf_free"](self.h)
            self.h = None


CH_SO = os.path.join(HERE, "_ref", "libch_ref.so")


class Channel:
    """The reference channel's L6 CSK decoder (src/sdr_ch.c:636-664) through
    ch_shim.c (_ref/libch_ref.so), same API as Restatement.csk."""
    kind = "reference"

    def __init__(self):
        self.lib = C.CDLL(CH_SO)
        self.lib.orr_csk.argtypes = [_p, _i, _i, _p, _i, _p, _p]

    def csk(self, corr, len_code, pos):
        corr = np.ascontiguousarray(corr, np.complex64)
        pos = np.ascontiguousarray(pos, np.float64)
        sym = np.zeros(1, np.uint8)
        Cc = np.zeros(len(pos), np.complex64)
        self.lib.orr_csk(_ptr(corr), len(corr), len_code, _ptr(pos), len(pos), _ptr(sym), _ptr(Cc))
        return int(sym[0]), Cc


TRACK_SO = os.path.join(HERE, "_ref", "libtrack_ref.so")


class _TrackJob(C.Structure):
    # orc_track_job_t in track_bench.c
    _fields_ = [("buf", _i), ("ix", _i), ("N", _i), ("npos", _i),
                ("fs", _d), ("fc", _d), ("phi", _d), ("coff", _d),
                ("pos", _p), ("code", _p), ("corr", _p)]


class TrackRun:
    """The tracking benchmark's CPU baseline: the reference's own sdr_mix_carr
    + sdr_corr_std for every job of a list, run from C over a pthread pool
    (track_bench.c over _ref/libsdr_ref.so), so that no Python runs between
    the calls. ``jobs``: dicts with buf, ix, N, fs, fc, phi, coff, pos, ch;
    ``banks``: per channel int8 [10 N, 2] code banks."""
    kind = "reference"

    def __init__(self, bufs, jobs, banks):
        self.lib = C.CDLL(TRACK_SO)
        self.lib.orc_track_run.argtypes = [_p, _p, _i, _i]
        self.lib.orc_track_run.restype = _i
        self._keep = [np.ascontiguousarray(b, np.uint8) for b in bufs]
        self.bufs = (_SdrBuff * len(bufs))(
            *[_SdrBuff(b.ctypes.data_as(C.POINTER(C.c_uint8)), 2, len(b)) for b in self._keep])
        self._banks = [np.ascontiguousarray(b, np.int8) for b in banks]
        self.pos = [np.ascontiguousarray(j["pos"], np.float64) for j in jobs]
        self.corr = np.zeros((len(jobs), max((len(p) for p in self.pos), default=1)), np.complex64)
        self.jobs = (_TrackJob * max(len(jobs), 1))()
        for k, j in enumerate(jobs):
            t = self.jobs[k]
            t.buf, t.ix, t.N, t.npos = j["buf"], j["ix"], j["N"], len(self.pos[k])
            t.fs, t.fc, t.phi, t.coff = j["fs"], j["fc"], j["phi"], j["coff"]
            t.pos = self.pos[k].ctypes.data
            t.code = self._banks[j["ch"]].ctypes.data
            t.corr = self.corr[k].ctypes.data
        self.n = len(jobs)

    def run(self, threads: int) -> np.ndarray:
        """Runs every job once; returns the correlations [n_jobs, n_pos]."""
        if self.lib.orc_track_run(C.cast(self.bufs, _p), C.cast(self.jobs, _p), self.n,
                                  threads) != 0:
            raise RuntimeError("track_bench: a thread could not start")
        return self.corr


def track_run_available() -> bool:
    return os.path.exists(TRACK_SO)


def best():
    """The reference build when present, else the restatement."""
    return Reference() if reference_available() else Restatement()
