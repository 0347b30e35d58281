/*
 * refine_oracle.c - test-only FP64 CPU statement of the refinement model:
 * per-block correlation sums, their derivatives with respect to code delay,
 * Doppler and carrier phase, and one Gauss-Newton step. Test
 * infrastructure: the shipped library never links or calls it.
 *
 * The reference has no counterpart (its finest estimate is the three-bin
 * quadratic of src/sdr_func.c:709-744 and the tracking loops of
 * src/sdr_ch.c); the model below is this project's own, so these functions
 * are pinned by central finite differences in the tests, not by reference
 * output.
 *
 * Model for one signal, samples n of the packed IF buffer, t = n / fs:
 *   psi(t) / 2 pi = fi t + fd (t - t_ref) + phi
 *   u(t) = rate (t - t_ref) + rate_nom (t_ref - tau) - 1/2      (chips)
 *   c(u) = chip[i] (1 - a) + chip[i + 1] a,  i = floor(u) mod Lc, a = frac(u)
 * i.e. the code linearly interpolated through the chip centres, so that the
 * correlation of rectangular received chips with c peaks at the true delay.
 * Blocks k = 0..K-1 cover samples [ix0 + k Nb, ix0 + (k+1) Nb); t_ref is the
 * middle of the span, (ix0 + K Nb / 2) / fs, and t' is the time from the
 * block centre.
 */
#include <math.h>
#include <string.h>
#include "sdr_oracle.h"

#define ORC_PI 3.1415926535897932

static inline int nibI(uint8_t b) { return (int)(int8_t)(uint8_t)(b << 4) >> 4; }
static inline int nibQ(uint8_t b) { return (int)(int8_t)b >> 4; }

void orc_refine_sums(const int8_t *chips, int Lc, double rate_nom, double rate,
                     double fi, const double *theta, const uint8_t *buf, int iq,
                     double fs, int ix0, int Nb, int K, double *out)
{
    const double tau = theta[0], fd = theta[1], phi = theta[2];
    const double t_ref = (ix0 + 0.5 * K * (double)Nb) / fs;
    for (int k = 0; k < K; k++) {
        double s[ORC_REFINE_W];
        memset(s, 0, sizeof(s));
        for (int n = 0; n < Nb; n++) {
            const long m = (long)ix0 + (long)k * Nb + n;
            const double t = m / fs;
            const double tp = (n - 0.5 * Nb) / fs;
            const double xr = nibI(buf[m]), xi = iq ? nibQ(buf[m]) : 0.0;
            double cyc = fi * t + fd * (t - t_ref) + phi;
            cyc -= floor(cyc);
            const double cs = cos(2.0 * ORC_PI * cyc), sn = sin(2.0 * ORC_PI * cyc);
            const double yr = xr * cs + xi * sn, yi = xi * cs - xr * sn;   /* x e^{-j psi} */
            double u = rate * (t - t_ref) + rate_nom * (t_ref - tau) - 0.5;
            u -= floor(u / Lc) * Lc;
            const double fl = floor(u);
            int i = (int)fl;
            if (i >= Lc) i -= Lc;
            const int j = i + 1 == Lc ? 0 : i + 1;
            const double a = u - fl;
            const double c = chips[i] + a * (chips[j] - chips[i]);
            const double dc = (double)chips[j] - chips[i];
            s[0] += yr * c;       s[1] += yi * c;
            s[2] += yr * dc;      s[3] += yi * dc;
            s[4] += tp * yr * c;  s[5] += tp * yi * c;
            s[6] += c * c;
            s[7] += tp * c * c;
            s[8] += tp * tp * c * c;
            s[9] += c * dc;
            s[10] += dc * dc;
        }
        memcpy(out + (size_t)k * ORC_REFINE_W, s, sizeof(s));
    }
}

/* Cholesky solve of the symmetric 3x3 system H x = b; 0 when H is not
 * positive definite. */
static int chol3(const double H[3][3], const double *b, double *x)
{
    double L[3][3] = {{0}};
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j <= i; j++) {
            double s = H[i][j];
            for (int k = 0; k < j; k++) s -= L[i][k] * L[j][k];
            if (i == j) {
                if (!(s > 0.0)) return 0;
                L[i][i] = sqrt(s);
            } else {
                L[i][j] = s / L[j][j];
            }
        }
    }
    double y[3];
    for (int i = 0; i < 3; i++) {
        double s = b[i];
        for (int k = 0; k < i; k++) s -= L[i][k] * y[k];
        y[i] = s / L[i][i];
    }
    for (int i = 2; i >= 0; i--) {
        double s = y[i];
        for (int k = i + 1; k < 3; k++) s -= L[k][i] * x[k];
        x[i] = s / L[i][i];
    }
    return 1;
}

/*
 * One Gauss-Newton step. Models (x ~ amplitude * s(theta) + noise):
 *  REFINE_POWER (0): a complex amplitude A_k per block - Gauss-Newton on the
 *     correlation-power loss sum_k |C_k|^2 / Q_k. The carrier phase is not
 *     observable (its row vanishes once A_k is eliminated): only (tau, fd)
 *     move, and fd is pinned only by the phase slope inside each block.
 *  REFINE_COHERENT (1): one real amplitude a and a common carrier phase over
 *     all blocks (fully coherent over the span; no data-bit flips).
 *  REFINE_BLOCKS (2): a real amplitude a_k per block (data-bit signs between
 *     blocks allowed) and a common carrier phase.
 * Every model first folds the closed-form phase into phi (arg sum_k C_k for
 * model 1, arg(sum_k C_k^2) / 2 otherwise; C, D and E rotate with it), takes
 * the least-squares amplitudes at that phase, eliminates them (Schur
 * complement), solves the 3x3 normal equations for (tau, fd, phi) in FP64
 * (phi row = identity for model 0), clamps the step to +-0.5 chip and
 * +-fs / (4 Nb) Hz, and makes the code rate follow the carrier
 * (rate_nom (1 + fd / fc)) if fc > 0.
 * info = {sum_k |C_k|^2 before the step, d tau (chips), d fd (Hz),
 *         d phi (cycles, after the phase fold), status (1 = solved)}.
 */
void orc_refine_step(const double *sums, int K, int Nb, double fs, double rate_nom,
                     double fc, int model, double *theta, double *rate, double *info)
{
    const double tp2 = 2.0 * ORC_PI, fp2 = 4.0 * ORC_PI * ORC_PI;
    double zr = 0, zi = 0, wr = 0, wi = 0, power = 0;
    for (int k = 0; k < K; k++) {
        const double *s = sums + (size_t)k * ORC_REFINE_W;
        zr += s[0] * s[0] - s[1] * s[1];
        zi += 2.0 * s[0] * s[1];
        wr += s[0];
        wi += s[1];
        power += s[0] * s[0] + s[1] * s[1];
    }
    double alpha;
    if (model == 1) alpha = (wr == 0.0 && wi == 0.0) ? 0.0 : atan2(wi, wr);
    else alpha = (zr == 0.0 && zi == 0.0) ? 0.0 : 0.5 * atan2(zi, zr);
    const double ca = cos(alpha), sa = -sin(alpha);   /* e^{-j alpha} */
    /* rotated per-block terms */
    double H[3][3] = {{0}}, b[3] = {0};
    double sCr = 0, sQ = 0, sR = 0;
    for (int k = 0; k < K; k++) {
        const double *s = sums + (size_t)k * ORC_REFINE_W;
        sCr += s[0] * ca - s[1] * sa;
        sQ += s[6];
        sR += -rate_nom * s[9];
    }
    const double a1 = sQ > 0.0 ? sCr / sQ : 0.0;     /* model 1 amplitude */
    for (int k = 0; k < K; k++) {
        const double *s = sums + (size_t)k * ORC_REFINE_W;
        const double dt = (k + 0.5 - 0.5 * K) * Nb / fs;   /* block centre - t_ref */
        const double Q = s[6];
        if (!(Q > 0.0)) continue;
        const double Qt = s[7] + dt * Q;
        const double Qtt = s[8] + 2.0 * dt * s[7] + dt * dt * Q;
        const double Rt = -rate_nom * s[9];                /* sum c dc/dtau */
        const double Pt = rate_nom * rate_nom * s[10];      /* sum (dc/dtau)^2 */
        const double Cr = s[0] * ca - s[1] * sa, Ci = s[0] * sa + s[1] * ca;
        const double Dr = -rate_nom * (s[2] * ca - s[3] * sa);
        const double Di = -rate_nom * (s[2] * sa + s[3] * ca);
        const double Er = (s[4] + dt * s[0]) * ca - (s[5] + dt * s[1]) * sa;
        const double Ei = (s[4] + dt * s[0]) * sa + (s[5] + dt * s[1]) * ca;
        if (model == 0) {
            const double Ar = Cr / Q, Ai = Ci / Q, A2 = Ar * Ar + Ai * Ai;
            H[0][0] += A2 * (Pt - Rt * Rt / Q);
            H[1][1] += fp2 * A2 * (Qtt - Qt * Qt / Q);
            b[0] += Ar * Dr + Ai * Di - A2 * Rt;            /* Re(conj(A) D) - |A|^2 R */
            b[1] += tp2 * (Ar * Ei - Ai * Er);              /* 2 pi Im(conj(A) E) */
        } else {
            const double a = model == 1 ? a1 : Cr / Q, a2 = a * a;
            H[0][0] += a2 * (model == 1 ? Pt : Pt - Rt * Rt / Q);
            H[1][1] += fp2 * a2 * Qtt;
            H[1][2] += fp2 * a2 * Qt;
            H[2][2] += fp2 * a2 * Q;
            b[0] += a * (Dr - a * Rt);
            b[1] += tp2 * a * Ei;
            b[2] += tp2 * a * Ci;
        }
    }
    if (model == 1 && sQ > 0.0) H[0][0] -= a1 * a1 * sR * sR / sQ;
    if (model == 0) H[2][2] = 1.0;
    H[2][1] = H[1][2];
    double x[3] = {0, 0, 0};
    const int ok = chol3((const double (*)[3])H, b, x);
    if (!ok) x[0] = x[1] = x[2] = 0.0;
    const double lim_t = 0.5 / rate_nom, lim_f = 0.25 * fs / Nb;
    if (x[0] > lim_t) x[0] = lim_t;
    if (x[0] < -lim_t) x[0] = -lim_t;
    if (x[1] > lim_f) x[1] = lim_f;
    if (x[1] < -lim_f) x[1] = -lim_f;
    theta[0] += x[0];
    theta[1] += x[1];
    double ph = theta[2] + alpha / tp2 + x[2];
    theta[2] = ph - floor(ph);
    *rate = fc > 0.0 ? rate_nom * (1.0 + theta[1] / fc) : rate_nom;
    info[0] = power;
    info[1] = x[0] * rate_nom;
    info[2] = x[1];
    info[3] = x[2];
    info[4] = ok;
}
