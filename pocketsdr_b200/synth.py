"""Seeded synthetic IF data and search workloads.

The reference measures on live or recorded front-end data; these generators
stand in for it with the same sample formats: every sample is one packed
4+4-bit byte (I low nibble, Q high nibble; Q = 0 for real sampling), values
quantised to 2-bit {-3,-1,1,3} or 3-bit {-7,...,7} odd levels. Each
satellite is code * carrier at its IF + Doppler with a carrier-aided code
Doppler, scaled to its C/N0 against unit-variance Gaussian noise.

Workloads:
  acq_l1ca_12mhz  - 12 MHz real IF at 3 MHz, 2-bit, 8 visible GPS L1 C/A
                    satellites; search 32 PRNs x 41 bins (+-5 kHz, 250 Hz) with
                    4 ms coherent (48,000-sample FFT, replica tiled x4) x 5 sums.
  acq_multi_24mhz - 24 MHz complex IQ, 3-bit, two RF buffers (L1/E1/B1 band
                    and L5 band), 10 satellites per signal; search every PRN of
                    L1CA (1 ms), E1-B (4 ms, BOC(1,1)), B1I (1 ms) and L5-I
                    (1 ms), zero-padded FFTs of 2N, Doppler bins by
                    sdr_dop_bins(T, 0, 5000), 20 ms of non-coherent sums.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import codes

CARRIER = {"L1CA": 1575.42e6, "E1B": 1575.42e6, "B1I": 1561.098e6,
           "L5I": 1176.45e6, "L5Q": 1176.45e6, "L6D": 1278.75e6}


@dataclass
class Sat:
    sig: str
    prn: int
    code_phase: float     # chips at sample 0
    doppler: float        # Hz
    phase: float          # cycles at sample 0
    cn0: float            # dB-Hz
    buf: int = 0


@dataclass
class Group:
    """One signal group of a search (one sdrg_acq_sig_t)."""
    sig: str
    prns: list
    fs: float
    fi: float
    T: float              # code period = coherent time (s)
    N: int                # samples per period / sum advance
    L: int                # FFT length
    Nmax: int             # code offsets kept
    n_sum: int
    fds: np.ndarray       # float32 Doppler bins
    buf: int = 0
    tile: int = 1         # replica periods per coherent block


@dataclass
class Workload:
    name: str
    fs: float
    iq: bool
    bufs: list            # packed uint8 IF buffers
    groups: list
    sats: list = field(default_factory=list)
    ix: list = field(default_factory=list)

    @property
    def cells(self) -> int:
        return sum(len(g.prns) * len(g.fds) * g.Nmax for g in self.groups)


def dop_bins(T: float, dop: float, max_dop: float) -> np.ndarray:
    """sdr_dop_bins (src/sdr_func.c:757-769), float32, with the fused
    multiply-add the reference build uses."""
    step = np.float32(0.5 / T)
    n = int(2.0 * max_dop / step) + 1
    i = np.arange(n, dtype=np.float64)
    return (i * np.float64(step) + np.float64(np.float32(dop) - np.float32(max_dop))).astype(np.float32)


def _quant(x: np.ndarray, bits: int) -> np.ndarray:
    """Nearest odd level of a mid-rise quantiser: 2-bit step 1 sigma,
    3-bit step 0.5 sigma, clipped."""
    step = 1.0 if bits == 2 else 0.5
    top = (1 << bits) - 1
    q = 2 * np.floor(x / step) + 1
    return np.clip(q, -top, top).astype(np.int8)


def pack(I: np.ndarray, Q: np.ndarray | None) -> np.ndarray:
    lo = I.astype(np.uint8) & 0x0F
    hi = (Q.astype(np.uint8) & 0x0F) << 4 if Q is not None else np.zeros_like(lo)
    return (hi | lo).astype(np.uint8)


def gen_if(n: int, fs: float, fi_of: dict, sats: list, *, iq: bool, bits: int,
           seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    t = np.arange(n, dtype=np.float64) / fs
    if iq:
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        n0 = 2.0 / fs
    else:
        x = rng.standard_normal(n).astype(np.complex128)
        n0 = 2.0 / fs
    for s in sats:
        chips = codes.gen_code(s.sig, s.prn).astype(np.float64)
        sec = codes.sec_code(s.sig, s.prn).astype(np.float64)
        L, T = codes.SIGNALS[s.sig]
        rate = L / T * (1.0 + s.doppler / CARRIER[s.sig])
        u = np.floor(s.code_phase + rate * t).astype(np.int64)
        # secondary code: the first whole primary period (the one after the
        # partial period at sample 0) carries its first chip
        c = chips[u % L] * sec[(u // L - 1) % len(sec)]
        ph = 2 * np.pi * ((fi_of[s.sig] + s.doppler) * t + s.phase)
        if iq:
            amp = np.sqrt(10 ** (s.cn0 / 10) * n0)
            x += amp * c * np.exp(1j * ph)
        else:
            amp = np.sqrt(2 * 10 ** (s.cn0 / 10) * n0)
            x += amp * c * np.cos(ph)
    I = _quant(x.real, bits)
    Q = _quant(x.imag, bits) if iq else None
    return pack(I, Q)


def tiled_code_fft(sig: str, prn: int, fs: float, tile: int, N: int, Nz: int) -> np.ndarray:
    chips = np.tile(codes.gen_code(sig, prn), tile)
    T = codes.code_cyc(sig) * tile
    return codes.gen_code_fft(chips, T, 0.0, fs, N, Nz)


def acq_l1ca_12mhz(seed: int = 1) -> Workload:
    fs, fi, bits = 12e6, 3e6, 2
    rng = np.random.default_rng(seed)
    vis = sorted(rng.choice(np.arange(1, 33), 8, replace=False).tolist())
    sats = [Sat("L1CA", int(p), float(rng.uniform(0, 1023)), float(rng.uniform(-4000, 4000)),
                float(rng.uniform(0, 1)), float(rng.uniform(38, 48))) for p in vis]
    N = int(fs * 4e-3)
    n_sum = 5
    buf = gen_if(N * n_sum, fs, {"L1CA": fi}, sats, iq=False, bits=bits, seed=seed + 100)
    fds = np.arange(-5000, 5001, 250, dtype=np.float32)
    g = Group("L1CA", list(range(1, 33)), fs, fi, 4e-3, N, N, N, n_sum, fds, 0, tile=4)
    return Workload("acq_l1ca_12mhz", fs, False, [buf], [g], sats, [0])


MULTI_SIGS = (("L1CA", 0), ("E1B", 0), ("B1I", 0), ("L5I", 1))


def acq_multi_24mhz(seed: int = 2, prn_limit: int | None = None, t_sum: float = 20e-3,
                    sigs=MULTI_SIGS) -> Workload:
    """prn_limit / t_sum shrink the search for parity tests."""
    fs, bits = 24e6, 3
    fi_of = {"L1CA": 7.161e6, "E1B": 7.161e6, "B1I": -7.161e6, "L5I": 2.0e6}
    rng = np.random.default_rng(seed)
    sats, groups = [], []
    n_buf = max(b for _, b in sigs) + 1
    n_samp = 0
    for sig, b in sigs:
        T = codes.code_cyc(sig)
        N = int(round(fs * T))
        n_sum = max(1, int(round(t_sum / T)))
        n_samp = max(n_samp, N * (n_sum + 1))
        prns = list(codes.PRN_SETS[sig])
        if prn_limit:
            prns = prns[:prn_limit]
        vis = sorted(rng.choice(prns, min(10, len(prns)), replace=False).tolist())
        for p in vis:
            L_code = codes.SIGNALS[sig][0]
            sats.append(Sat(sig, int(p), float(rng.uniform(0, L_code)), float(rng.uniform(-5000, 5000)),
                            float(rng.uniform(0, 1)), float(rng.uniform(35, 48)), b))
        groups.append(Group(sig, prns, fs, fi_of[sig], T, N, 2 * N, N, n_sum,
                            dop_bins(T, 0.0, 5000.0), b))
    bufs = []
    for b in range(n_buf):
        bsats = [s for s in sats if s.buf == b]
        bufs.append(gen_if(n_samp, fs, fi_of, bsats, iq=True, bits=bits, seed=seed * 10 + b))
    return Workload("acq_multi_24mhz", fs, True, bufs, groups, sats, [0] * n_buf)


def long_replica_fft(sig: str, prn: int, fs: float, t_coh: float, L: int) -> np.ndarray:
    """Conjugated DFT of a t_coh-second replica for long coherent integration:
    the primary code repeated over t_coh with the signal's secondary code
    overlaid, one secondary chip per primary period from its first chip (L5-Q:
    NH20), and, for codes longer than t_coh allows to repeat whole (L6D, 4 ms
    in 10 ms), truncated."""
    chips = codes.gen_code(sig, prn).astype(np.float64)
    sec = codes.sec_code(sig, prn).astype(np.float64)
    Lc, T = codes.SIGNALS[sig]
    n = int(round(fs * t_coh))
    t = np.arange(n, dtype=np.float64)
    per = np.floor(t * (1.0 / (T * fs))).astype(np.int64)            # primary period index
    idx = (np.floor(t * (Lc / (T * fs))).astype(np.int64)) % Lc
    x = np.zeros(L, np.complex128)
    x[:n] = chips[idx] * sec[per % len(sec)]
    return np.conj(np.fft.fft(x)).astype(np.complex64)


def acq_long_48mhz(seed: int = 6, prn_limit: int | None = None, n_sum: int = 20,
                   bins: np.ndarray | None = None) -> Workload:
    """Weak-signal long coherent search: 48 MHz complex IQ, 3-bit, GPS L5-Q
    (1 ms primary code with the NH20 secondary code) and QZSS L6D (4 ms code,
    time-multiplexed) at C/N0 25-32 dB-Hz; 10 ms coherent (480 000-sample
    FFTs) x n_sum non-coherent sums over +-10 kHz in 50 Hz bins. The coherent
    windows start 20 ms apart - one NH20 period, five L6D periods - so that
    every sum meets the replica's secondary-code and code phase (with 10 ms
    steps, every other window would carry the other half of NH20 and start
    half an L6D period later)."""
    fs, bits, t_coh, t_step = 48e6, 3, 10e-3, 20e-3
    fi_of = {"L5Q": 0.0, "L6D": 5.0e6}
    rng = np.random.default_rng(seed)
    L = int(round(fs * t_coh))
    step = int(round(fs * t_step))
    fds = np.arange(-10000, 10001, 50, dtype=np.float32) if bins is None else np.asarray(bins, np.float32)
    sats, groups = [], []
    for sig in ("L5Q", "L6D"):
        prns = list(codes.PRN_SETS[sig])
        if prn_limit:
            prns = prns[:prn_limit]
        vis = sorted(rng.choice(prns, min(4, len(prns)), replace=False).tolist())
        for p in vis:
            sats.append(Sat(sig, int(p), float(rng.uniform(0, codes.SIGNALS[sig][0])),
                            float(rng.uniform(-9000, 9000)), float(rng.uniform(0, 1)),
                            float(rng.uniform(25, 32)), 0))
        groups.append(Group(sig, prns, fs, fi_of[sig], t_coh, step, L, L, n_sum, fds, 0))
    buf = gen_if(step * n_sum + L, fs, fi_of, sats, iq=True, bits=bits, seed=seed * 10)
    return Workload("acq_long_48mhz", fs, True, [buf], groups, sats, [0])


@dataclass
class RefineSat:
    sig: str
    prn: int
    tau: float            # code delay (s): code phase rate_nom (t_ref - tau) at t_ref
    doppler: float        # Hz
    phase: float          # carrier phase at t_ref (cycles)
    cn0: float            # dB-Hz


@dataclass
class RefineWorkload:
    """Delay / Doppler / phase refinement: one IF record, the satellites in
    it, the acquisition groups that give the starting grid peaks and the
    refinement span (K blocks of Nb samples from ix0)."""
    name: str
    fs: float
    fi: float
    iq: bool
    buf: np.ndarray
    sats: list
    groups: list
    Nb: int
    K: int
    ix0: int = 0

    @property
    def t_ref(self) -> float:
        return (self.ix0 + 0.5 * self.K * self.Nb) / self.fs


def code_rate(sig: str) -> float:
    L, T = codes.SIGNALS[sig]
    return L / T


def refine_signal(sig: str, prn: int, fs: float, fi: float, n: int, tau: float, fd: float,
                  phi: float, t_ref: float) -> np.ndarray:
    """Unit-amplitude complex signal of one satellite: rectangular chips at
    the carrier-aided code rate, chip phase rate_nom (t_ref - tau) at t_ref,
    carrier phase fi t + fd (t - t_ref) + phi cycles."""
    chips = codes.gen_code(sig, prn).astype(np.float64)
    Lc = len(chips)
    rn = code_rate(sig)
    rate = rn * (1.0 + fd / CARRIER[sig])
    t = np.arange(n, dtype=np.float64) / fs
    u = rate * (t - t_ref) + rn * (t_ref - tau)
    idx = np.floor(u).astype(np.int64) % Lc
    cyc = fi * t + fd * (t - t_ref) + phi
    return chips[idx] * np.exp(2j * np.pi * (cyc - np.floor(cyc)))


def refine_12mhz(seed: int = 4, n_l1ca: int = 32, n_e1b: int = 32,
                 cn0=(30.0, 45.0)) -> RefineWorkload:
    """12 MHz real IF at 3 MHz, 2-bit, GPS L1 C/A and Galileo E1-B (BOC(1,1))
    satellites at C/N0 U[30, 45] dB-Hz with off-grid delay
    and Doppler (U[-4500, 4500] Hz); refinement over 10 ms coherent x 4
    blocks. Starting grid: L1 C/A 10 ms coherent (N = 120 000, 2N FFT) x 4
    sums in 50 Hz bins, E1-B 8 ms (two code periods, N = 96 000) x 5 sums in
    62.5 Hz bins (coherent windows must advance by whole code periods), both
    over +-5 kHz. No data-bit modulation."""
    fs, fi, bits = 12e6, 3e6, 2
    Nb, K = 120000, 4
    rng = np.random.default_rng(seed)
    n = 5 * Nb
    t_ref = 0.5 * K * Nb / fs
    sats = []
    for sig, cnt in (("L1CA", n_l1ca), ("E1B", n_e1b)):
        T = codes.code_cyc(sig)
        for p in list(codes.PRN_SETS[sig])[:cnt]:
            sats.append(RefineSat(sig, int(p), float(rng.uniform(0, T)),
                                  float(rng.uniform(-4500, 4500)), float(rng.uniform(0, 1)),
                                  float(rng.uniform(*cn0))))
    x = rng.standard_normal(n)
    n0 = 2.0 / fs
    for s in sats:
        amp = np.sqrt(2 * 10 ** (s.cn0 / 10) * n0)
        x += amp * refine_signal(s.sig, s.prn, fs, fi, n, s.tau, s.doppler, s.phase, t_ref).real
    buf = pack(_quant(x, bits), None)
    groups = []
    for sig, T, n_sum in (("L1CA", 10e-3, 4), ("E1B", 8e-3, 5)):
        prns = [s.prn for s in sats if s.sig == sig]
        if not prns:
            continue
        N = int(round(fs * T))
        groups.append(Group(sig, prns, fs, fi, T, N, 2 * N, N, n_sum, dop_bins(T, 0.0, 5000.0), 0))
    return RefineWorkload("refine_12mhz", fs, fi, False, buf, sats, groups, Nb, K, 0)


def periodic_code_ffts(g: Group) -> np.ndarray:
    """Conjugated DFTs of the code repeated over the group's N samples
    (nearest-chip resampling wraps modulo the code length), zero padded to L."""
    out = np.empty((len(g.prns), g.L), np.complex64)
    for i, p in enumerate(g.prns):
        out[i] = codes.gen_code_fft(codes.gen_code(g.sig, p), codes.code_cyc(g.sig), 0.0,
                                    g.fs, g.N, g.L - g.N)
    return out


def long_code_ffts(g: Group) -> np.ndarray:
    out = np.empty((len(g.prns), g.L), np.complex64)
    for i, p in enumerate(g.prns):
        out[i] = long_replica_fft(g.sig, p, g.fs, g.T, g.L)
    return out


@dataclass
class TrackChannel:
    sig: str
    prn: int
    ant: int              # antenna (IF buffer)
    fd0: float            # Doppler at t = 0 (Hz)
    rate: float           # Doppler rate (Hz/s)
    coff0: float          # code offset at t = 0 (s)
    N: int                # samples per code period
    T: float              # code period (s)


@dataclass
class TrackWorkload:
    """Tracking-correlator batch: n_ant antenna streams, channels with their
    own code bank, open-loop carrier / code trajectories."""
    fs: float
    fi: float
    bufs: list
    channels: list
    pos: dict             # per signal: tap positions (samples)

    def jobs_at(self, t: float, banks_ptr: list) -> list:
        """Job specs for every channel whose code period starts at time t
        (multiple of its period), following src/sdr_ch.c:692-733: carrier at
        fi + fd(t), phase = integral of the carrier, code offset drifting with
        the carrier-aided rate."""
        out = []
        for c, ptr in zip(self.channels, banks_ptr):
            k = int(round(t / c.T))
            if abs(k * c.T - t) > 1e-9:
                continue
            fd = c.fd0 + c.rate * t
            fc = self.fi + fd
            phi = self.fi * t + c.fd0 * t + 0.5 * c.rate * t * t
            coff = c.coff0 - (c.fd0 * t + 0.5 * c.rate * t * t) / CARRIER[c.sig]
            L = len(self.bufs[c.ant])
            ix = int(round(t * self.fs)) % L
            out.append(dict(buf=c.ant, ix=ix, N=c.N, fs=self.fs, fc=fc, phi=phi - np.floor(phi),
                            coff=(coff % c.T) * self.fs, cpx_code=False, pos=self.pos[c.sig],
                            code_ptr=ptr))
        return out


TRACK_SIGS = (("L1CA", 0.375), ("E1B", 0.25), ("L5I", 0.375))


def track_24mhz(seed: int = 5, n_ch: int = 256, n_ant: int = 8, t_buf: float = 0.1) -> TrackWorkload:
    """24 MHz complex IQ, 3-bit, n_ant antenna streams of t_buf seconds
    (replayed cyclically for longer runs); n_ch channels mixing L1 C/A, E1-B
    and L5-I with Doppler rates U[0, 2] Hz/s; taps P/E/L at +-0.5 chip, the
    noise tap at -120 samples and 40 taps at 0.05-chip spacing (44 taps)."""
    fs, fi, bits = 24e6, 3.0e6, 3
    rng = np.random.default_rng(seed)
    chans = []
    counts = [int(round(f * n_ch)) for _, f in TRACK_SIGS]
    counts[-1] = n_ch - sum(counts[:-1])
    for (sig, _), cnt in zip(TRACK_SIGS, counts):
        prns = list(codes.PRN_SETS[sig])
        T = codes.code_cyc(sig)
        for i in range(cnt):
            chans.append(TrackChannel(sig, prns[i % len(prns)], i % n_ant,
                                      float(rng.uniform(-4000, 4000)), float(rng.uniform(0, 2)),
                                      float(rng.uniform(0, T)), int(round(fs * T)), T))
    pos = {}
    for sig, _ in TRACK_SIGS:
        L, T = codes.SIGNALS[sig]
        sc = T / (L if sig != "E1B" else L // 2) * fs      # samples per chip
        pos[sig] = np.concatenate([[0.0, -0.5 * sc, 0.5 * sc, -120.0],
                                   np.arange(-20, 20) * 0.05 * sc])
    n = int(round(t_buf * fs))
    bufs = []
    for a in range(n_ant):
        sats = [Sat(c.sig, c.prn, (1 - c.coff0 / c.T) * codes.SIGNALS[c.sig][0], c.fd0, 0.0, 45.0, a)
                for c in chans if c.ant == a][:12]
        bufs.append(gen_if(n, fs, {s: fi for s, _ in TRACK_SIGS}, sats, iq=True, bits=bits,
                           seed=seed * 100 + a))
    return TrackWorkload(fs, fi, bufs, chans, pos)


def track_banks(wl: TrackWorkload) -> list:
    """Per channel code bank (int8 [10 N, 2]) as the receiver builds it."""
    from .track import code_bank
    cache = {}
    out = []
    for c in wl.channels:
        key = (c.sig, c.prn)
        if key not in cache:
            cache[key] = code_bank(codes.gen_code(c.sig, c.prn), c.T, wl.fs, c.N)
        out.append(cache[key])
    return out


def group_code_ffts(g: Group) -> np.ndarray:
    """[n_prn, L] complex64 conjugated code DFTs of a group."""
    out = np.empty((len(g.prns), g.L), np.complex64)
    for i, p in enumerate(g.prns):
        out[i] = tiled_code_fft(g.sig, p, g.fs, g.tile, g.N, g.L - g.N)
    return out
