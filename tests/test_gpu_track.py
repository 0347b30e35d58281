"""Batched tracking correlators (sdrg_corr_batch) against the oracle:
carrier wipe-off + multi-tap correlation bit-exact per job, including
circular-buffer wraps, complex codes and the full 107-tap limit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run_batch(torch, bufs, specs, banks):
    from pocketsdr_b200 import track
    from pocketsdr_b200._lib import torch_stream
    d_bufs = [torch.from_numpy(b).cuda() for b in bufs]
    d_banks = [torch.from_numpy(np.ascontiguousarray(bk)).cuda() for bk in banks]
    for s, db in zip(specs, d_banks):
        s["code_ptr"] = db.data_ptr()
    jobs = track.make_jobs(specs)
    n = len(specs)
    corr = torch.zeros(n * track.SDR_MAX_CORR * 2, dtype=torch.float32, device="cuda")
    Cb = torch.zeros(n * 4, dtype=torch.float32, device="cuda")
    track.corr_batch(jobs, [b.data_ptr() for b in d_bufs], [len(b) for b in bufs],
                     corr.data_ptr(), Cb.data_ptr(), torch_stream())
    torch.cuda.synchronize()
    corr = corr.cpu().numpy().view(np.complex64).reshape(n, track.SDR_MAX_CORR)
    Cb = Cb.cpu().numpy().view(np.complex64).reshape(n, 2)
    return corr, Cb


def test_corr_batch_random_jobs_bit_exact(orc):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(33)
    bufs = [rng.integers(0, 256, 70001, dtype=np.uint8), rng.integers(0, 256, 50000, dtype=np.uint8)]
    specs, banks = [], []
    for j in range(24):
        b = int(rng.integers(0, 2))
        N = int(rng.integers(16, 30000))
        cpx = bool(j % 3 == 2)
        bank = (rng.choice(np.array([-1, 0, 1], np.int8), (10 * N, 2)) if cpx else
                np.repeat(rng.choice(np.array([-1, 1], np.int8), (10 * N, 1)), 2, 1))
        n = 107 if j == 0 else int(rng.integers(1, 60))
        pos = np.concatenate([[0.0, -5.5, 5.5], rng.uniform(-N, N, max(n - 3, 0))])[:n]
        ix = len(bufs[b]) - int(rng.integers(1, N)) if j % 4 == 1 else int(rng.integers(0, len(bufs[b])))
        fs = float(rng.uniform(2e6, 48e6))
        specs.append(dict(buf=b, ix=ix, N=N, fs=fs, fc=float(rng.uniform(-0.45, 0.45) * fs),
                          phi=float(rng.uniform(-3, 3)), coff=float(rng.uniform(0, N)),
                          cpx_code=cpx, pos=pos))
        banks.append(bank)
    corr, Cb = _run_batch(torch, bufs, specs, banks)
    for j, (s, bank) in enumerate(zip(specs, banks)):
        IQ = orc.mix_carr(bufs[s["buf"]], s["ix"], s["N"], s["fs"], s["fc"], s["phi"])
        ref, refC = orc.corr_std(IQ, bank, s["coff"], s["pos"], s["cpx_code"])
        n = len(s["pos"])
        assert np.array_equal(corr[j, :n].view(np.uint32), ref.view(np.uint32)), j
        assert np.array_equal(Cb[j].view(np.uint32), refC.view(np.uint32)), j


def test_corr_batch_l1ca_tracking_taps(orc):
    """Receiver-shaped jobs: 24 MHz IQ, L1 C/A banks built like trk_new
    (src/sdr_ch.c:265-272), P/E/L at +-0.5 chip, 40 taps at 0.05 chip and the
    noise tap at -120 samples."""
    torch = pytest.importorskip("torch")
    from pocketsdr_b200 import codes, synth, track
    fs, T = 24e6, 1e-3
    N = int(fs * T)
    sats = [synth.Sat("L1CA", p, 100.0 * p, 300.0 * p - 2000, 0.1 * p, 45.0) for p in (3, 7, 11)]
    buf = synth.gen_if(6 * N, fs, {"L1CA": 4.0e6}, sats, iq=True, bits=3, seed=9)
    sc = T / 1023 * fs
    pos = np.concatenate([[0.0, -0.5 * sc, 0.5 * sc, -120.0],
                          np.arange(-20, 20) * 0.05 * sc])
    specs, banks = [], []
    for k, s in enumerate(sats):
        bank = track.code_bank(codes.gen_code("L1CA", s.prn), T, fs, N)
        coff = (1023 - s.code_phase) / 1023 * N + 0.37
        specs.append(dict(buf=0, ix=(2 + k) * N, N=N, fs=fs, fc=4.0e6 + s.doppler, phi=0.25,
                          coff=coff, cpx_code=False, pos=pos))
        banks.append(bank)
    corr, Cb = _run_batch(torch, [buf], specs, banks)
    for j, (s, bank) in enumerate(zip(specs, banks)):
        IQ = orc.mix_carr(buf, s["ix"], N, fs, s["fc"], s["phi"])
        ref, refC = orc.corr_std(IQ, bank, s["coff"], pos, False)
        assert np.array_equal(corr[j, :len(pos)].view(np.uint32), ref.view(np.uint32)), j
        assert np.array_equal(Cb[j].view(np.uint32), refC.view(np.uint32)), j


def test_corr_batch_arbitrary_code_bytes_and_alignment(orc):
    """Real-code banks holding any int8 value (-128, 0, independent I and Q
    bytes), half of them at a 2-byte offset (no 4-byte alignment: the
    byte-wise path), odd lengths and tap offsets: bit-exact. The packed path's
    one special case, a mixed sample of -128 against a negative code byte,
    is checked to occur."""
    torch = pytest.importorskip("torch")
    from pocketsdr_b200 import track
    from pocketsdr_b200._lib import torch_stream
    rng = np.random.default_rng(71)
    buf = rng.integers(0, 256, 90001, dtype=np.uint8)
    specs, banks, keep = [], [], []
    n_special = 0
    for j in range(10):
        N = int(rng.integers(1000, 20000)) | (j & 1)          # odd and even lengths
        bank = rng.integers(-128, 128, (10 * N, 2), dtype=np.int8)
        bank[rng.random(10 * N) < 0.1] = 0
        bank[rng.random(10 * N) < 0.05, 0] = -128
        n = int(rng.integers(3, 40))
        pos = np.concatenate([[0.0, -1.5, 2.5], rng.uniform(-N, N, n - 3)])
        spec = dict(buf=0, ix=int(rng.integers(0, len(buf))), N=N, fs=12e6,
                    fc=float(rng.uniform(-5e6, 5e6)), phi=float(rng.uniform(-1, 1)),
                    coff=float(rng.uniform(0, N)), cpx_code=False, pos=pos)
        # device copy, at a 2-byte offset for odd j
        off = j & 1
        dev = torch.zeros((10 * N + 1) * 2, dtype=torch.int8, device="cuda")
        dev[2 * off:2 * off + 20 * N] = torch.from_numpy(bank.reshape(-1)).cuda()
        keep.append(dev)
        spec["code_ptr"] = dev.data_ptr() + 2 * off
        specs.append(spec)
        banks.append(bank)
        IQ = orc.mix_carr(buf, spec["ix"], N, spec["fs"], spec["fc"], spec["phi"])
        n_special += int(np.sum((IQ.view(np.int8).reshape(-1, 2) == -128).any(1)))
    assert n_special > 0
    d_buf = torch.from_numpy(buf).cuda()
    jobs = track.make_jobs(specs)
    n = len(specs)
    corr = torch.zeros(n * track.SDR_MAX_CORR * 2, dtype=torch.float32, device="cuda")
    Cb = torch.zeros(n * 4, dtype=torch.float32, device="cuda")
    track.corr_batch(jobs, [d_buf.data_ptr()], [len(buf)], corr.data_ptr(), Cb.data_ptr(),
                     torch_stream())
    torch.cuda.synchronize()
    corr = corr.cpu().numpy().view(np.complex64).reshape(n, track.SDR_MAX_CORR)
    Cb = Cb.cpu().numpy().view(np.complex64).reshape(n, 2)
    for j, (s, bank) in enumerate(zip(specs, banks)):
        IQ = orc.mix_carr(buf, s["ix"], s["N"], s["fs"], s["fc"], s["phi"])
        ref, refC = orc.corr_std(IQ, bank, s["coff"], s["pos"], False)
        k = len(s["pos"])
        assert np.array_equal(corr[j, :k].view(np.uint32), ref.view(np.uint32)), j
        assert np.array_equal(Cb[j].view(np.uint32), refC.view(np.uint32)), j
