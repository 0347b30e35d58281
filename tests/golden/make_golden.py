"""Generates the golden fixtures in this folder from the reference itself.

Run with POCKETSDR_REF naming the reference source tree (it builds
oracle/_ref first):

    POCKETSDR_REF=<tree> python tests/golden/make_golden.py

Every output is produced by the reference's own C functions
(src/sdr_func.c, src/sdr_code.c), compiled from source by oracle/Makefile, on
seeded inputs. The fixtures are what the GPU parity tests compare against on
machines where the reference is absent.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from pocketsdr_b200 import codes, synth  # noqa: E402


def mix_cases(rng, nbuf):
    cases = [(0, 64, 4.0, 0.0, 0.0), (nbuf - 40, 100, 4e6, 1.25e6, 0.3)]
    for _ in range(30):
        N = int(rng.integers(1, 1500))
        ix = int(rng.integers(0, nbuf))
        fs = float(rng.uniform(1e6, 40e6))
        fc = float(rng.uniform(-0.45 * fs, 0.45 * fs))
        phi = float(rng.uniform(-2, 2))
        cases.append((ix, N, fs, fc, phi))
    return cases


def main() -> int:
    oracle.build()          # the reference tree from POCKETSDR_REF
    R = oracle.Reference()
    rng = np.random.default_rng(20240601)

    # ---- carrier wipe-off -------------------------------------------------
    nbuf = 5000
    buf = rng.integers(0, 256, nbuf, dtype=np.uint8)
    cases = mix_cases(rng, nbuf)
    outs = [R.mix_carr(buf, ix, N, fs, fc, phi) for ix, N, fs, fc, phi in cases]
    np.savez_compressed(os.path.join(HERE, "mix.npz"), buf=buf,
                        cases=np.array(cases, np.float64),
                        out=np.concatenate(outs), lens=np.array([len(o) for o in outs]))
    # full 64K table through the reference (byte b at phase index i)
    tb = np.repeat(np.arange(256, dtype=np.uint8), 256)
    tab = R.mix_carr(tb, 0, 65536, 256.0, 1.0, 0.0)
    meta = {"mix_table_sha256": hashlib.sha256(tab.tobytes()).hexdigest()}

    # ---- standard correlators --------------------------------------------
    N = 3000
    IQ = rng.integers(-128, 128, (N, 2), dtype=np.int8)
    code_r = np.repeat(rng.choice(np.array([-1, 1], np.int8), (10 * N, 1)), 2, axis=1)
    code_c = rng.choice(np.array([-1, 0, 1], np.int8), (10 * N, 2))
    ccases = []
    for k in range(6):
        n = int(rng.integers(3, 40))
        sp = float(rng.uniform(0.2, 6.0))
        pos = np.concatenate([[0.0, -sp, sp], rng.uniform(-40, 40, n - 3)])
        coff = float(rng.uniform(-N, 2 * N)) if k else 1234.56
        ccases.append((coff, pos))
    corr_out = {}
    for name, code, cpx in (("real", code_r, False), ("cpx", code_c, True)):
        cs, Cs = [], []
        for coff, pos in ccases:
            c, Cb = R.corr_std(IQ, code, coff, pos, cpx)
            cs.append(c)
            Cs.append(Cb)
        corr_out[f"corr_{name}"] = np.concatenate(cs)
        corr_out[f"C_{name}"] = np.stack(Cs)
    np.savez_compressed(os.path.join(HERE, "corr_std.npz"), IQ=IQ, code_real=code_r,
                        code_cpx=code_c, coffs=np.array([c for c, _ in ccases]),
                        pos=np.concatenate([p for _, p in ccases]),
                        npos=np.array([len(p) for _, p in ccases]), **corr_out)

    # ---- complex-buffer (python-facing) variants --------------------------
    nb = 2500
    cbuf = (rng.integers(-7, 8, nb) + 1j * rng.integers(-7, 8, nb)).astype(np.complex64)
    code_f = rng.choice(np.array([-1.0, 1.0], np.float32), 2000)
    pos_i = np.array([0.0, -3.0, 3.0, -1.0, 1.0, 7.0, -120.0])
    cstd = R.corr_std_cpx(cbuf, 1700, 2000, 4e6, 1.1e6, 0.25, code_f, pos_i)
    cf_py = rng.standard_normal(2000).astype(np.float32) + 1j * rng.standard_normal(2000).astype(np.float32)
    cfft = R.corr_fft_cpx(cbuf, 900, 2000, 4e6, -0.7e6, 0.6, cf_py.astype(np.complex64))
    np.savez_compressed(os.path.join(HERE, "cpx_buffer.npz"), buff=cbuf, code=code_f, pos=pos_i,
                        corr_std=cstd, code_fft=cf_py.astype(np.complex64), corr_fft=cfft)

    # ---- FFT correlator and search ------------------------------------------
    fs, fi, T = 2e6, 0.5e6, 1e-3
    Ns = int(fs * T)
    sats = [synth.Sat("L1CA", 3, 100.3, 1200.0, 0.1, 50.0),
            synth.Sat("L1CA", 17, 800.7, -2300.0, 0.7, 46.0),
            synth.Sat("L1CA", 25, 420.0, 300.0, 0.4, 44.0)]
    ifbuf = synth.gen_if(7 * Ns, fs, {"L1CA": fi}, sats, iq=False, bits=2, seed=77)
    code_fft = codes.gen_code_fft(codes.gen_code("L1CA", 3), T, 0.0, fs, Ns, Ns)
    code_fft_ref = R.gen_code_fft(codes.gen_code("L1CA", 3), None, T, 0.0, fs, Ns, Ns)
    fds = synth.dop_bins(T, 0.0, 2500.0)
    P = np.zeros((len(fds), 2 * Ns), np.float32)
    ix_list = [0, 6 * Ns - 700]          # the second window wraps the buffer
    for ix in ix_list:
        R.search_code(code_fft_ref, ifbuf, ix, 2 * Ns, fs, fi, fds, P, T)
    cn0, pk = R.corr_max(P, 2 * Ns, Ns, len(fds), T)
    fd = R.fine_dop(P, 2 * Ns, fds, pk)
    IQm = R.mix_carr(ifbuf, 0, 2 * Ns, fs, fi + 1000.0, 0.0)
    corr = R.corr_fft(IQm, code_fft_ref)
    np.savez_compressed(os.path.join(HERE, "search.npz"), ifbuf=ifbuf, code_fft=code_fft_ref,
                        fds=fds, ix=np.array(ix_list), P=P, cn0=np.float32(cn0),
                        peak=np.array(pk), fd=np.float64(fd), IQm=IQm, corr=corr,
                        params=np.array([fs, fi, T]))
    meta["code_fft_numpy_vs_ref_rel"] = float(np.abs(code_fft - code_fft_ref).max() /
                                              np.abs(code_fft_ref).max())
    # ---- real front-end data: the reference's own L1 sample -----------------
    # sample/L1_20211125_004000_12MHz_I.bin (12 MHz, IF 3 MHz, INT8 real, 2-bit
    # values). 20 ms of it, packed as the reference's sdr_read_data does
    # (src/sdr_func.c:451-505: SDR_CPX8(raw, 0)), searched for GPS L1 C/A
    # PRN 1-32 with 4 ms coherent x 5 sums (48 000-point circular correlation
    # of the code tiled x4), +-5 kHz in 250 Hz bins, by the reference's
    # sdr_search_code / sdr_corr_max / sdr_fine_dop.
    src = os.path.join(oracle.REF_ROOT, "sample", "L1_20211125_004000_12MHz_I.bin")
    raw = np.fromfile(src, np.int8)[:5 * 48000]
    real_buf = (raw.astype(np.uint8) & 0x0F).astype(np.uint8)
    fs, fi, T, N = 12e6, 3e6, 4e-3, 48000
    fds = np.arange(-5000, 5001, 250, dtype=np.float32)
    res = []
    for prn in range(1, 33):
        cf = R.gen_code_fft(np.tile(codes.gen_code("L1CA", prn), 4), None, T, 0.0, fs, N, 0)
        P = np.zeros((len(fds), N), np.float32)
        for s in range(5):
            R.search_code(cf, real_buf, s * N, N, fs, fi, fds, P, T)
        cn0, pk = R.corr_max(P, N, N, len(fds), T)
        res.append((prn, pk[0], pk[1], cn0, float(P[pk[0], pk[1]]), R.fine_dop(P, N, fds, pk)))
    res = np.array(res, dtype=[("prn", np.int32), ("bin", np.int32), ("offset", np.int32),
                               ("cn0", np.float32), ("pmax", np.float32), ("fd", np.float64)])
    np.savez_compressed(os.path.join(HERE, "real_l1ca.npz"), buf=real_buf, fds=fds, res=res,
                        params=np.array([fs, fi, T, N, 5]))
    meta["real_l1ca_detected_38dbhz"] = [int(r["prn"]) for r in res if r["cn0"] >= 38.0]

    # Doppler bins: exact floats
    meta["dop_bins"] = {f"{T}_{d}_{m}": R.dop_bins(T, d, m).tolist()
                        for T, d, m in ((1e-3, 0.0, 5000.0), (4e-3, 0.0, 5000.0),
                                        (1e-3, 123.4, 1000.0), (2e-3, -77.7, 3333.0),
                                        (10e-3, 0.0, 10000.0))}
    with open(os.path.join(HERE, "meta.json"), "w") as f:
        json.dump(meta, f, indent=1)
    for fn in sorted(os.listdir(HERE)):
        if fn.endswith((".npz", ".json")):
            print(fn, os.path.getsize(os.path.join(HERE, fn)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
