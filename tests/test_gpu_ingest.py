"""IF ingest on the GPU (sdrg_ingest_*, sdr_lpf_*) against the reference's
own receiver code (src/sdr_rcv.c write_buff + src/sdr_func.c LPF +
src/sdr_array.c combine, through oracle/rcv_shim.c; the restatement when that
build is absent): every output byte identical, over consecutive blocks (the
LPF history and the fs/4 phase carry across them)."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import ingest_cases  # noqa: E402


@pytest.fixture(scope="module")
def chk():
    from oracle import oracle
    return oracle.Ingest()


def _gpu_ingest(torch, cfg, raws, ix0, n_slots=3):
    from pocketsdr_b200 import ingest
    ing = ingest.Ingest(cfg["fmt"], cfg["N"], cfg["fs"], IQ=cfg["IQ"], bits=cfg["bits"],
                        lut_off=cfg["off"], lut_scale=cfg["scale"], lpf_fc=cfg["lpf_fc"],
                        w=cfg["w"], arch_on=cfg["arch_on"])
    N = cfg["N"]
    nb = ing.n_rf + ing.narch
    bufs = [torch.zeros(N * n_slots, dtype=torch.uint8, device="cuda") for _ in range(nb)]
    outs = []
    for j, raw in enumerate(raws):
        ix = ix0 + j
        base = N * (ix % n_slots)
        ing.run(torch.from_numpy(raw).cuda(), ix, bufs, base)
        torch.cuda.synchronize()
        outs.append(np.stack([b[base:base + N].cpu().numpy() for b in bufs]))
    ing.close()
    return outs


@pytest.mark.parametrize("N", [3000, 5, 4096, 24000])
def test_ingest_matches_reference(chk, gpu, N):
    torch = pytest.importorskip("torch")
    for name, cfg in ingest_cases.cases(N=N, seed=N):
        raws = ingest_cases.raw_blocks(cfg, 5, seed=N + 1)
        ref = chk.receiver(**cfg)
        want = [ref.write(r, 7 + j) for j, r in enumerate(raws)]
        got = _gpu_ingest(torch, cfg, raws, 7)
        for j, (g, w) in enumerate(zip(got, want)):
            assert np.array_equal(g, w), (name, N, j, np.argwhere(g != w)[:5].tolist())


def test_drop_in_lpf_matches_reference(chk, gpu):
    from pocketsdr_b200._lib import lib, ptr
    rng = np.random.default_rng(21)
    for fc, fs in ((4e6, 16e6), (5.4e6, 24e6), (0.9e6, 2.4e6)):
        ref = chk.lpf(fc, fs)
        h = lib.sdr_lpf_new(fc, fs)
        assert h
        try:
            for n in (3, 1000, 2048, 7, 1, 50000):
                d = rng.integers(0, 256, n, dtype=np.uint8)
                want = ref.apply(d)
                got = d.copy()
                lib.sdr_lpf_apply(h, ptr(got), n)
                assert np.array_equal(got, want), (fc, n)
        finally:
            lib.sdr_lpf_free(h)
    assert not lib.sdr_lpf_new(13e6, 24e6)      # cutoff above fs/2: no filter, as the reference


def test_ingest_feeds_search(ref, chk, gpu):
    """Raw RAW16 front-end data (two 3-bit real L1 channels with fs/4 mixing
    and LPF) -> device IF buffer -> batched search, against the reference's
    ingest and search on the same bytes: same peaks."""
    torch = pytest.importorskip("torch")
    from pocketsdr_b200 import acquire, synth
    fs, T = 12e6, 1e-3
    N = int(fs * T)
    rng = np.random.default_rng(4)
    # a 3-bit real L1 C/A signal at IF fs/4 in RF channel 0's nibble codes
    sats = [synth.Sat("L1CA", 7, 211.25, 1250.0, 0.3, 52.0)]
    x = synth.gen_if(8 * N, fs, {"L1CA": fs / 4}, sats, iq=False, bits=3, seed=2)
    I = ((x << 4).astype(np.int8) >> 4).astype(np.int32)            # odd levels -7..7
    # the front end's 3-bit code of each level: invert RF channel 0's table
    lut = chk.gen_lutc(4, 0, 1, 3, 1)[:16]                          # phase 0, low nibble
    lvl = ((lut << 4).astype(np.int8) >> 4).astype(np.int32)
    code3 = {int(v): c for c, v in enumerate(lvl)}
    nib = np.array([code3[int(v)] for v in I], np.uint8)
    raw = np.zeros((8 * N, 2), np.uint8)
    raw[:, 0] = nib | (rng.integers(0, 16, 8 * N, dtype=np.uint8) << 4)
    raw[:, 1] = rng.integers(0, 256, 8 * N, dtype=np.uint8)
    cfg = dict(fmt=4, N=N, IQ=[1, 1, 2, 2], bits=[3, 3, 2, 2], off=(0.0, 0.0), scale=(1.0, 1.0),
               lpf_fc=[0.45 * fs / 2, 0.0, 0.0, 0.0], fs=fs, w=None, arch_on=None)
    blocks = [raw[j * N:(j + 1) * N].reshape(-1) for j in range(8)]
    rcv = chk.receiver(**cfg)
    ref_buf = np.concatenate([rcv.write(b, j)[0] for j, b in enumerate(blocks)])
    got = _gpu_ingest(torch, cfg, blocks, 0, n_slots=8)
    gpu_buf = np.concatenate([g[0] for g in got])
    assert np.array_equal(gpu_buf, ref_buf)
    fds = synth.dop_bins(T, 0.0, 5000.0)
    g = synth.Group("L1CA", [5, 7, 9], fs, 0.0, T, N, 2 * N, N, 4, fds, 0)
    cf = synth.group_code_ffts(g)
    plan = acquire.AcqPlan([g], [cf])
    res = plan.run_host([gpu_buf], [0])
    for i, p in enumerate(g.prns):
        P = np.zeros((len(fds), 2 * N), np.float32)
        for s in range(4):
            ref.search_code(cf[i], ref_buf, s * N, 2 * N, fs, 0.0, fds, P, T)
        cn0, pk = ref.corr_max(P, 2 * N, N, len(fds), T)
        if p == 7:
            assert (res["bin"][i], res["offset"][i]) == pk and abs(res["cn0"][i] - cn0) < 0.1
