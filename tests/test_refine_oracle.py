"""FP64 refinement oracle on the CPU: the analytic derivatives of the block
correlations against central finite differences of the model itself, the
zero carrier-phase gradient of the power loss, and Gauss-Newton convergence.
The refinement model has no reference counterpart, so these tests are what
pins the oracle the GPU refinement is checked against."""
import numpy as np
import pytest

from pocketsdr_b200 import codes, synth


@pytest.fixture(scope="module")
def wl():
    return synth.refine_12mhz(seed=21, n_l1ca=1, n_e1b=1, cn0=(44.0, 45.0))


def _sig(wl, i):
    s = wl.sats[i]
    return s, codes.gen_code(s.sig, s.prn), synth.code_rate(s.sig), synth.CARRIER[s.sig]


def _f(orc, wl, chips, rn, rate, th, g):
    """sum_k Re(conj(g_k) C_k(theta)) in FP64."""
    S = orc.refine_sums(chips, rn, rate, wl.fi, th, wl.buf, wl.iq, wl.fs, wl.ix0, wl.Nb, wl.K)
    return float(np.sum(np.real(np.conj(g) * orc.refine_corr(S))))


def _knot_samples(wl, chips, rn, rate, th, eps):
    """Samples whose code phase lies within eps chip of a chip centre (the
    model's derivative in tau jumps there)."""
    n = np.arange(wl.ix0, wl.ix0 + wl.K * wl.Nb, dtype=np.float64)
    t = n / wl.fs
    u = rate * (t - wl.t_ref) + rn * (wl.t_ref - th[0]) - 0.5
    return int(np.sum(np.abs(u - np.round(u)) < eps))


@pytest.mark.parametrize("i", [0, 1], ids=["L1CA", "E1B"])
def test_fp64_vjp_matches_central_differences(orc, wl, i):
    s, chips, rn, fc = _sig(wl, i)
    rng = np.random.default_rng(5 + i)
    th = np.array([s.tau + 0.15 / rn, s.doppler + 7.0, s.phase + 0.2])
    rate = rn * (1 + th[1] / fc)
    g = rng.standard_normal(wl.K) + 1j * rng.standard_normal(wl.K)
    S = orc.refine_sums(chips, rn, rate, wl.fi, th, wl.buf, wl.iq, wl.fs, wl.ix0, wl.Nb, wl.K)
    grad = orc.refine_vjp(S, g, rn, wl.Nb, wl.fs)
    # tau: the model is piecewise linear in tau; a sample whose code phase
    # crosses a chip centre inside +-h changes the slope by at most
    # 4 |x| |g| rate_nom, allowed for explicitly (h is large against the
    # double rounding of the code phase, ~1e-11 chip)
    h_chip = 1e-5
    h = h_chip / rn
    fd_tau = (_f(orc, wl, chips, rn, rate, th + [h, 0, 0], g)
              - _f(orc, wl, chips, rn, rate, th - [h, 0, 0], g)) / (2 * h)
    n_knot = _knot_samples(wl, chips, rn, rate, th, h_chip)
    tol = 1e-6 * abs(grad[0]) + n_knot * 4 * 3 * np.abs(g).max() * rn
    assert abs(fd_tau - grad[0]) <= tol, (fd_tau, grad[0], n_knot)
    for j, h in ((1, 1e-2), (2, 1e-6)):
        e = np.zeros(3)
        e[j] = h
        fd = (_f(orc, wl, chips, rn, rate, th + e, g) - _f(orc, wl, chips, rn, rate, th - e, g)) / (2 * h)
        assert fd == pytest.approx(grad[j], rel=1e-6, abs=1e-6 * np.abs(grad).max())


def test_fp64_power_loss_has_no_phase_gradient(orc, wl):
    s, chips, rn, fc = _sig(wl, 0)
    th = np.array([s.tau + 0.1 / rn, s.doppler - 4.0, 0.37])
    rate = rn * (1 + th[1] / fc)
    S = orc.refine_sums(chips, rn, rate, wl.fi, th, wl.buf, wl.iq, wl.fs, wl.ix0, wl.Nb, wl.K)
    Cb = orc.refine_corr(S)
    grad = orc.refine_vjp(S, 2 * Cb, rn, wl.Nb, wl.fs)        # d sum |C_k|^2
    assert abs(grad[2]) <= 1e-9 * np.abs(grad[:2]).max()

    def power(phi):
        S2 = orc.refine_sums(chips, rn, rate, wl.fi, [th[0], th[1], phi], wl.buf, wl.iq, wl.fs,
                             wl.ix0, wl.Nb, wl.K)
        return float(np.sum(np.abs(orc.refine_corr(S2)) ** 2))

    assert power(0.37) == pytest.approx(power(0.81), rel=1e-12)


@pytest.mark.parametrize("model", [1, 2])
def test_fp64_gauss_newton_converges_on_strong_signals(orc, wl, model):
    for i in range(len(wl.sats)):
        s, chips, rn, fc = _sig(wl, i)
        chip_div = 2 if s.sig == "E1B" else 1          # BOC half-chips per chip
        th0 = [s.tau - 0.04 * chip_div / rn, s.doppler + 6.0, 0.0]
        th, rate, infos = orc.refine_gn(chips, rn, fc, wl.fi, th0, wl.buf, wl.iq, wl.fs, wl.ix0,
                                        wl.Nb, wl.K, [model] * 5)
        T = codes.code_cyc(s.sig)
        dtau = ((th[0] - s.tau + T / 2) % T - T / 2) * rn / chip_div
        assert abs(dtau) < 0.01, (s.sig, dtau)
        assert abs(th[1] - s.doppler) < 1.0
        dphi = (th[2] - s.phase + 0.25) % 0.5 - 0.25    # sign of the amplitude is free
        assert abs(dphi) < 0.02
        assert all(inf[4] == 1 for inf in infos)
        assert infos[-1][0] >= infos[0][0]              # correlation power grew
        assert rate == pytest.approx(rn * (1 + th[1] / fc), rel=1e-15)


def test_fp64_power_model_moves_only_delay_and_doppler(orc, wl):
    s, chips, rn, fc = _sig(wl, 0)
    th0 = [s.tau - 0.05 / rn, s.doppler - 8.0, 0.0]
    th, _, infos = orc.refine_gn(chips, rn, fc, wl.fi, th0, wl.buf, wl.iq, wl.fs, wl.ix0,
                                 wl.Nb, wl.K, [0] * 4)
    assert all(inf[3] == 0.0 for inf in infos)           # no phase step of its own
    T = codes.code_cyc(s.sig)
    assert abs(((th[0] - s.tau + T / 2) % T - T / 2) * rn) < 0.02
    assert abs(th[1] - s.doppler) < 3.0
