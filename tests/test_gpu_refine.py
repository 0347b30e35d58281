"""GPU refinement (sdrg_refine_*): FP32 block sums against the FP64 oracle,
the hand-written adjoint against the FP64 gradient and against central
differences of the GPU forward, the autograd Function, and Gauss-Newton
refinement against the FP64 oracle's (0.01 chip, 5 Hz) - from perturbed
truth and from the GPU acquisition grid's peak."""
import numpy as np
import pytest

from pocketsdr_b200 import codes, synth

pytestmark = pytest.mark.gpu


def _specs(wl):
    from pocketsdr_b200.refine import RefineSpec
    return [RefineSpec(codes.gen_code(s.sig, s.prn), synth.code_rate(s.sig), wl.fi,
                       synth.CARRIER[s.sig]) for s in wl.sats]


def _setup(wl, th):
    import torch
    from pocketsdr_b200.refine import RefinePlan
    plan = RefinePlan(_specs(wl), wl.fs, wl.iq, wl.Nb, wl.K)
    buf = torch.from_numpy(wl.buf).cuda()
    theta = torch.tensor(np.asarray(th, np.float64), device="cuda")
    rate = plan.carrier_aided_rate(theta)
    return plan, buf, theta, rate


def _perturbed(wl, rng, dtau_chip=0.04, dfd=6.0, lo=0.0):
    """Truth offset by +-[lo, 1] x (dtau_chip chips, dfd Hz), random phase."""
    th = []
    for s in wl.sats:
        rn = synth.code_rate(s.sig)
        div = 2 if s.sig == "E1B" else 1
        a, b = rng.uniform(lo, 1.0, 2) * rng.choice([-1.0, 1.0], 2)
        th.append([s.tau + a * dtau_chip * div / rn, s.doppler + b * dfd, rng.uniform(0, 1)])
    return np.array(th)


def _noise_scales(wl, ref):
    """Per (signal, block) noise-level magnitudes of C, D and E:
    sqrt(E[x^2] sum w^2) with w = c, dc, t' c (from the FP64 Q, P, Qtt)."""
    b = wl.buf[wl.ix0: wl.ix0 + wl.K * wl.Nb]
    xr = ((b << 4).astype(np.int8) >> 4).astype(np.float64)
    xi = (b.astype(np.int8) >> 4).astype(np.float64) if wl.iq else 0.0 * xr
    ex2 = float(np.mean(xr ** 2 + xi ** 2))
    return (np.sqrt(ex2 * ref[:, :, 6]), np.sqrt(ex2 * ref[:, :, 10]),
            np.sqrt(ex2 * ref[:, :, 8]))


def _tau_err_chips(s, tau):
    T = codes.code_cyc(s.sig)
    div = 2 if s.sig == "E1B" else 1
    return ((tau - s.tau + T / 2) % T - T / 2) * synth.code_rate(s.sig) / div


def _oracle_sums(orc, wl, th, rate):
    out = []
    for s, t, r in zip(wl.sats, th, rate):
        out.append(orc.refine_sums(codes.gen_code(s.sig, s.prn), synth.code_rate(s.sig), r,
                                   wl.fi, t, wl.buf, wl.iq, wl.fs, wl.ix0, wl.Nb, wl.K))
    return np.stack(out)


@pytest.fixture(scope="module")
def wl():
    return synth.refine_12mhz(seed=31, n_l1ca=3, n_e1b=3)


def test_refine_sums_match_fp64_oracle(orc, wl):
    rng = np.random.default_rng(1)
    th = _perturbed(wl, rng, 0.2, 20.0)
    plan, buf, theta, rate = _setup(wl, th)
    S = plan.sums(buf, wl.ix0, theta, rate, mode=1).cpu().numpy().astype(np.float64)
    C0 = plan.sums(buf, wl.ix0, theta, rate, mode=0).cpu().numpy()
    ref = _oracle_sums(orc, wl, th, rate.cpu().numpy())
    # FP32 accumulation against FP64, each quantity within 1e-4 of its natural
    # magnitude: the noise level sqrt(sum of squared terms) for the signed
    # sums (C, D, E, Qt, R), the value itself for the positive ones (Q, Qtt, P)
    sC, sD, sE = _noise_scales(wl, ref)
    scale = [sC, sC, sD, sD, sE, sE, ref[:, :, 6], np.sqrt(ref[:, :, 8]), ref[:, :, 8],
             np.sqrt(ref[:, :, 10]), ref[:, :, 10]]
    for col in range(11):
        err = np.abs(S[:, :, col] - ref[:, :, col]) / scale[col]
        assert err.max() < 1e-4, (col, err.max())
    np.testing.assert_allclose(C0, S[:, :, :2], rtol=0, atol=1e-6 * np.abs(S[:, :, :2]).max())


def test_refine_vjp_matches_fp64_gradient(orc, wl):
    import torch
    rng = np.random.default_rng(2)
    th = _perturbed(wl, rng, 0.15, 10.0)
    plan, buf, theta, rate = _setup(wl, th)
    g = rng.standard_normal((plan.n, plan.K, 2)).astype(np.float32)
    S = plan.sums(buf, wl.ix0, theta, rate, mode=1)
    grad = plan.vjp(S, torch.from_numpy(g).cuda()).cpu().numpy()
    ref = _oracle_sums(orc, wl, th, rate.cpu().numpy())
    sC, sD, sE = _noise_scales(wl, ref)
    dt = (np.arange(wl.K) + 0.5 - 0.5 * wl.K) * wl.Nb / wl.fs
    for i, s in enumerate(wl.sats):
        gc = g[i, :, 0].astype(np.float64) + 1j * g[i, :, 1]
        rn = synth.code_rate(s.sig)
        gr = orc.refine_vjp(ref[i], gc, rn, wl.Nb, wl.fs)
        # per component: 1e-4 of the gradient's noise-level magnitude
        tol = 1e-4 * np.array([rn * np.sum(np.abs(gc) * sD[i]),
                               2 * np.pi * np.sum(np.abs(gc) * (sE[i] + np.abs(dt) * sC[i])),
                               2 * np.pi * np.sum(np.abs(gc) * sC[i])])
        assert np.all(np.abs(grad[i] - gr) <= tol), (grad[i], gr, tol)


def _central(f, theta, j, h):
    import torch
    st = torch.zeros_like(theta)
    st[:, j] = torch.from_numpy(np.asarray(h, np.float64)).cuda()
    return ((f(theta + st) - f(theta - st)) / (2 * st[:, j])).cpu().numpy()


def test_autograd_backward_matches_gpu_central_differences():
    """torch.autograd through CorrBlocks against central differences of the
    GPU forward itself: the correlation-power loss for delay and Doppler, a
    random linear functional of the C_k for Doppler and carrier phase (the
    power loss has no phase gradient). The delay step is small against the
    chip (the model is piecewise linear in tau) and the signals strong, so
    that chip-centre crossings inside the step stay far below 2 %."""
    import torch
    from pocketsdr_b200.refine import corr_blocks, corr_power
    w1 = synth.refine_12mhz(seed=32, n_l1ca=2, n_e1b=2, cn0=(44.0, 45.0))
    rng = np.random.default_rng(3)
    th = _perturbed(w1, rng, 0.3, 15.0, lo=0.4)
    plan, buf, theta, rate = _setup(w1, th)
    rn = np.array([synth.code_rate(s.sig) for s in w1.sats])

    x = theta.clone().requires_grad_(True)
    corr_power(plan, buf, w1.ix0, x, rate).sum().backward()
    grad = x.grad.cpu().numpy()

    def power(t):
        with torch.no_grad():
            return corr_power(plan, buf, w1.ix0, t, rate).double()

    np.testing.assert_allclose(grad[:, 0], _central(power, theta, 0, 5e-5 / rn), rtol=0.02)
    np.testing.assert_allclose(grad[:, 1], _central(power, theta, 1, [0.05] * plan.n), rtol=0.01)

    g = torch.from_numpy(rng.standard_normal((plan.n, plan.K, 2)).astype(np.float32)).cuda()
    x = theta.clone().requires_grad_(True)
    (corr_blocks(plan, buf, w1.ix0, x, rate) * g).sum().backward()
    grad = x.grad.cpu().numpy()

    def lin(t):
        with torch.no_grad():
            return (corr_blocks(plan, buf, w1.ix0, t, rate).double() * g.double()).sum(dim=(1, 2))

    np.testing.assert_allclose(grad[:, 1], _central(lin, theta, 1, [0.05] * plan.n), rtol=0.01)
    np.testing.assert_allclose(grad[:, 2], _central(lin, theta, 2, [1e-3] * plan.n), rtol=0.01)


def test_power_loss_phase_gradient_is_zero(wl):
    import torch
    from pocketsdr_b200.refine import corr_power
    rng = np.random.default_rng(4)
    plan, buf, theta, rate = _setup(wl, _perturbed(wl, rng))
    x = theta.clone().requires_grad_(True)
    corr_power(plan, buf, wl.ix0, x, rate).sum().backward()
    g = x.grad.cpu().numpy()
    assert np.all(g[:, 2] == 0.0)
    assert np.all(np.abs(g[:, :2]).max(axis=1) > 0)


def test_gauss_newton_matches_fp64_oracle(orc, wl):
    rng = np.random.default_rng(5)
    th0 = _perturbed(wl, rng)
    plan, buf, theta, rate = _setup(wl, th0)
    info = plan.gn(buf, wl.ix0, theta, rate, models=(1,) * 5).cpu().numpy()
    th = theta.cpu().numpy()
    for i, s in enumerate(wl.sats):
        tr, _, infos = orc.refine_gn(codes.gen_code(s.sig, s.prn), synth.code_rate(s.sig),
                                     synth.CARRIER[s.sig], wl.fi, th0[i], wl.buf, wl.iq, wl.fs,
                                     wl.ix0, wl.Nb, wl.K, [1] * 5)
        div = 2 if s.sig == "E1B" else 1
        assert abs(th[i, 0] - tr[0]) * synth.code_rate(s.sig) / div < 0.01
        assert abs(th[i, 1] - tr[1]) < 5.0
        assert abs(_tau_err_chips(s, th[i, 0])) < 0.1
        assert abs(th[i, 1] - s.doppler) < 5.0
        assert np.all(info[:, i, 4] == 1.0)
        assert info[0, i, 0] == pytest.approx(infos[0][0], rel=1e-4)


def test_gauss_newton_in_a_cuda_graph(wl):
    """sdrg_refine_gn allocates nothing and never synchronises: five steps
    captured once and replayed give the eager result."""
    import torch
    rng = np.random.default_rng(6)
    th0 = _perturbed(wl, rng)
    plan, buf, theta, rate = _setup(wl, th0)
    plan.gn(buf, wl.ix0, theta, rate)                  # eager reference
    eager = theta.clone()
    t_g = torch.tensor(th0, device="cuda")
    r_g = plan.carrier_aided_rate(t_g)
    start_t, start_r = t_g.clone(), r_g.clone()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        plan.gn(buf, wl.ix0, t_g, r_g, info=False)     # warm-up on the capture stream
    torch.cuda.current_stream().wait_stream(s)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        plan.gn(buf, wl.ix0, t_g, r_g, info=False)
    t_g.copy_(start_t)
    r_g.copy_(start_r)
    graph.replay()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(t_g.cpu().numpy(), eager.cpu().numpy())


def test_refine_from_acquisition_peak(orc, wl):
    """The full path on a small case: the GPU grid search (10 ms / 8 ms
    coherent) gives the peaks; Gauss-Newton from there on the GPU and in the
    FP64 oracle agree within 0.01 chip and 5 Hz; both land near the truth."""
    import torch
    from pocketsdr_b200.acquire import AcqPlan
    from pocketsdr_b200.refine import theta_from_peaks
    acq = AcqPlan(wl.groups, [synth.periodic_code_ffts(g) for g in wl.groups])
    res = acq.run_host([wl.buf], [0])
    fc = [synth.CARRIER[s.sig] for s in wl.sats]
    th0 = theta_from_peaks(res["offset"], res["fd"], 0, wl.fs, fc, wl.t_ref)
    plan, buf, theta, rate = _setup(wl, th0)
    plan.gn(buf, wl.ix0, theta, rate, models=(1,) * 5)
    th = theta.cpu().numpy()
    for i, s in enumerate(wl.sats):
        tr, _, _ = orc.refine_gn(codes.gen_code(s.sig, s.prn), synth.code_rate(s.sig), fc[i],
                                 wl.fi, th0[i], wl.buf, wl.iq, wl.fs, wl.ix0, wl.Nb, wl.K, [1] * 5)
        div = 2 if s.sig == "E1B" else 1
        assert abs(th[i, 0] - tr[0]) * synth.code_rate(s.sig) / div < 0.01
        assert abs(th[i, 1] - tr[1]) < 5.0
        assert abs(_tau_err_chips(s, th[i, 0])) < 0.1
        assert abs(th[i, 1] - s.doppler) < 5.0, (s, th[i], res[i])
