/*
 * sdr_oracle.c - test-only CPU restatement of Pocket SDR's signal-search and
 * correlation hot path. See sdr_oracle.h. This file is test infrastructure:
 * the shipped library (pocketsdr_b200) never links or calls it.
 *
 * The refinement model (no reference counterpart) lives in refine_oracle.c.
 *
 * Built with -ffp-contract=off so that every fused multiply-add below is an
 * explicit fma() call, written where the reference build (gcc -O3 -mfma,
 * GNU C default -ffp-contract=fast) contracts the same expression.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "sdr_oracle.h"

#define ORC_PI 3.1415926535897932
#define ORC_CSCALE (1 / 11.2f)          /* src/pocket_sdr.h:61 */

static int8_t carr_I[256], carr_Q[256]; /* quantised carrier, 8-bit phase */
static int8_t mixtab[65536 * 2];        /* (byte << 8 | phase) -> (I, Q) */
static int inited = 0;

/* sign-extended nibbles of a packed sample (src/pocket_sdr.h:104-105) */
static inline int nib_I(uint8_t b) { return (int)(int8_t)(uint8_t)(b << 4) >> 4; }
static inline int nib_Q(uint8_t b) { return (int)(int8_t)b >> 4; }

/* src/sdr_func.c:113-134: carrier amplitude ROUND(cos|sin(-2 pi i/256)/CSCALE),
 * products wrapped to int8 exactly as the reference's int8_t stores. */
void orc_init(void)
{
    if (inited) return;
    for (int ph = 0; ph < 256; ph++) {
        double ang = -2.0 * ORC_PI * ph / 256;
        carr_I[ph] = (int8_t)floor(cos(ang) / ORC_CSCALE + 0.5);
        carr_Q[ph] = (int8_t)floor(sin(ang) / ORC_CSCALE + 0.5);
    }
    for (int b = 0; b < 256; b++) {
        int I = nib_I((uint8_t)b), Q = nib_Q((uint8_t)b);
        for (int ph = 0; ph < 256; ph++) {
            int e = (b << 8) | ph;
            mixtab[2 * e]     = (int8_t)(I * carr_I[ph] - Q * carr_Q[ph]);
            mixtab[2 * e + 1] = (int8_t)(I * carr_Q[ph] + Q * carr_I[ph]);
        }
    }
    inited = 1;
}

const int8_t *orc_mix_table(void) { orc_init(); return mixtab; }

/* src/sdr_func.c:772-807: uint32 phase accumulator, scale 2^32, the top 8 bits
 * select the carrier phase. p_i = p0 + i*s (mod 2^32). */
static void mix_seg(const uint8_t *data, int N, double phi, double step,
                    int8_t *IQ)
{
    const double scale = 4294967296.0;
    uint32_t p = (uint32_t)((phi - floor(phi)) * scale);
    uint32_t s = (uint32_t)(int)(step * scale);
    for (int i = 0; i < N; i++, p += s) {
        int e = ((int)data[i] << 8) + (int)(p >> 24);
        IQ[2 * i] = mixtab[2 * e];
        IQ[2 * i + 1] = mixtab[2 * e + 1];
    }
}

/* src/sdr_func.c:824-836: a window crossing the end of the circular buffer
 * is mixed as two segments; the second restarts the phase from
 * phi + step * n. */
void orc_mix_carr(const uint8_t *buff, int len_buff, int ix, int N, double fs,
                  double fc, double phi, int8_t *IQ)
{
    orc_init();
    double step = fc / fs;
    if (ix + N <= len_buff) {
        mix_seg(buff + ix, N, phi, step, IQ);
    } else {
        int n = len_buff - ix;
        mix_seg(buff + ix, n, phi, step, IQ);
        mix_seg(buff, N - n, phi + step * n, step, IQ + 2 * n);
    }
}

/* float -> int8 as C's (int8_t) cast on x86 (truncate toward zero, then keep
 * the low byte), then pack 4+4 (src/pocket_sdr.h:103). */
static uint8_t pack_f(float re, float im)
{
    int8_t r = (int8_t)(int)re, q = (int8_t)(int)im;
    return (uint8_t)(((uint8_t)q << 4) | ((uint8_t)r & 0x0F));
}

/* src/sdr_func.c:839-848 */
void orc_mix_carr_cpx(const float *buff, int len_buff, int ix, int N,
                      double fs, double fc, double phi, int8_t *IQ)
{
    orc_init();
    uint8_t *tmp = (uint8_t *)malloc(N > 0 ? N : 1);
    for (int i = 0, j = ix; i < N; i++, j = (j + 1) % len_buff) {
        tmp[i] = pack_f(buff[2 * j], buff[2 * j + 1]);
    }
    mix_seg(tmp, N, phi, fc / fs, IQ);
    free(tmp);
}

/* int8 "sign" product of the AVX2 path (_mm256_sign_epi8): x, -x or 0 by the
 * sign of c, where negating -128 wraps back to -128. */
static inline int sgn_mul(int x, int c)
{
    if (c == 0) return 0;
    if (c > 0) return x;
    return x == -128 ? -128 : -x;
}

/* src/sdr_func.c:861-912 (real code) and :915-956 (complex code), AVX2 build:
 * the first 16*floor(len/16) terms are sign products (see sgn_mul) summed
 * exactly in int32, and the sum is converted to float once; the remaining
 * (len mod 16) terms are exact int products added one by one in float; the
 * result is scaled by CSCALE. */
static void dot_code(const int8_t *IQ, const int8_t *code, int len, int cpx,
                     float *c)
{
    int main_len = len >= 16 ? (len / 16) * 16 : 0;
    int32_t sr = 0, si = 0;
    int i = 0;
    for (; i < main_len; i++) {
        int I = IQ[2 * i], Q = IQ[2 * i + 1], cI = code[2 * i], cQ = code[2 * i + 1];
        if (cpx) {
            sr += sgn_mul(I, cI) + sgn_mul(Q, cQ);
            /* the AVX2 path negates the code byte with int8 wrap too */
            si += sgn_mul(Q, cI) + sgn_mul(I, cQ == -128 ? -128 : -cQ);
        } else {
            sr += sgn_mul(I, cI);
            si += sgn_mul(Q, cQ);
        }
    }
    float fr = (float)sr, fi = (float)si;
    for (; i < len; i++) {
        int I = IQ[2 * i], Q = IQ[2 * i + 1], cI = code[2 * i], cQ = code[2 * i + 1];
        if (cpx) { fr += (float)(I * cI + Q * cQ); fi += (float)(Q * cI - I * cQ); }
        else     { fr += (float)(I * cI);          fi += (float)(Q * cQ); }
    }
    float sc = 1.0f * ORC_CSCALE;
    c[0] = fr * sc;
    c[1] = fi * sc;
}

/* src/sdr_func.c:981-1008 / :1029-1057. Tap i at p = coff + pos[i] samples:
 * integer shift j = floor(p), bank k = (int)((p - j) * 10); j wrapped once
 * into [0, N). corr1 = IQ[0:j] . code_k[N-j:N], corr2 = IQ[j:N] . code_k[0:N-j].
 * The sign of the E/P/L polarity test is taken from
 * sum_i fma(c1.re, c2.re, c1.im * c2.im), the contraction gcc -mfma emits. */
void orc_corr_std(const int8_t *IQ, const int8_t *code, int N, double coff,
                  const double *pos, int n, int cpx_code, float *corr,
                  float *C)
{
    float c1[ORC_MAX_CORR][2], c2[ORC_MAX_CORR][2];
    for (int i = 0; i < n; i++) {
        double p = coff + pos[i];
        int j = (int)floor(p), k = (int)((p - j) * ORC_N_CODES);
        if (j < 0) j += N; else if (j >= N) j -= N;
        const int8_t *bank = code + 2 * (size_t)k * N;
        dot_code(IQ, bank + 2 * (N - j), j, cpx_code, c1[i]);
        dot_code(IQ + 2 * j, bank, N - j, cpx_code, c2[i]);
    }
    float dot = 0.0f;
    for (int i = 0; i < 3 && i < n; i++) {
        dot = dot + fmaf(c1[i][0], c2[i][0], c1[i][1] * c2[i][1]);
    }
    float sign = dot < 0.0f ? -1.0f : 1.0f;
    for (int i = 0; i < n; i++) {
        corr[2 * i]     = (c1[i][0] + sign * c2[i][0]) / N;
        corr[2 * i + 1] = (c1[i][1] + sign * c2[i][1]) / N;
    }
    if (C && n > 0) {
        C[0] = c1[0][0]; C[1] = c1[0][1];
        C[2] = c2[0][0]; C[3] = c2[0][1];
    }
}

/* src/sdr_func.c:1060-1072: the code is cast to int8 (I = Q) as one bank. */
void orc_corr_std_cpx(const float *buff, int len_buff, int ix, int N,
                      double fs, double fc, double phi, const float *code,
                      const double *pos, int n, float *corr)
{
    int8_t *IQ = (int8_t *)malloc(4 * (size_t)N + 2);
    float C[4];
    orc_mix_carr_cpx(buff, len_buff, ix, N, fs, fc, phi, IQ);
    for (int i = 0; i < N; i++) {
        IQ[2 * (N + i)] = IQ[2 * (N + i) + 1] = (int8_t)(int)code[i];
    }
    orc_corr_std(IQ, IQ + 2 * N, N, 0.0, pos, n, 0, corr, C);
    free(IQ);
}

/* ---- double-precision mixed-radix FFT (own implementation) --------------- */

static int small_factor(int n)
{
    if (n % 4 == 0) return 4;
    if (n % 2 == 0) return 2;
    for (int p = 3; p * p <= n; p += 2) if (n % p == 0) return p;
    return n;
}

void orc_fft(const double *in, int N, int dir, double *out)
{
    if (N <= 0) return;
    int lvl_n[40], lvl_p[40], L = 0;
    for (int n = N; n > 1; ) {
        int p = small_factor(n);
        lvl_n[L] = n; lvl_p[L] = p; L++; n /= p;
    }
    double *tw = (double *)malloc(sizeof(double) * 2 * N);
    double *cur = (double *)malloc(sizeof(double) * 2 * N);
    double *nxt = (double *)malloc(sizeof(double) * 2 * N);
    double sgn = dir ? 1.0 : -1.0;
    for (int e = 0; e < N; e++) {
        double a = 2.0 * ORC_PI * e / N;
        tw[2 * e] = cos(a);
        tw[2 * e + 1] = sgn * sin(a);
    }
    /* Decimation in time, iterative. Leaf t = r0*(N/p0) + r1*(N/(p0 p1)) + ...
     * holds input r0 + p0*(r1 + p1*(r2 + ...)), so that every level-l block
     * of length n holds its p sub-transforms of length n/p back to back. */
    for (int t = 0; t < N; t++) {
        int rem = t, src = 0, mul = 1, blk = N;
        for (int l = 0; l < L; l++) {
            blk /= lvl_p[l];
            int r = rem / blk;
            rem %= blk;
            src += r * mul;
            mul *= lvl_p[l];
        }
        cur[2 * t] = in[2 * src];
        cur[2 * t + 1] = in[2 * src + 1];
    }
    /* combine: X[k + q m] = sum_r w_n^(r (k + q m)) F_r[k] */
    for (int l = L - 1; l >= 0; l--) {
        int n = lvl_n[l], p = lvl_p[l], m = n / p, ts = N / n;
        for (int base = 0; base < N; base += n) {
            for (int kk = 0; kk < n; kk++) {
                int k = kk % m;
                double re = 0.0, im = 0.0;
                for (int r = 0; r < p; r++) {
                    long e = ((long)r * kk % n) * ts;
                    const double *f = cur + 2 * ((size_t)base + (size_t)r * m + k);
                    re += f[0] * tw[2 * e] - f[1] * tw[2 * e + 1];
                    im += f[0] * tw[2 * e + 1] + f[1] * tw[2 * e];
                }
                nxt[2 * ((size_t)base + kk)] = re;
                nxt[2 * ((size_t)base + kk) + 1] = im;
            }
        }
        double *t = cur; cur = nxt; nxt = t;
    }
    memcpy(out, cur, sizeof(double) * 2 * N);
    free(tw); free(cur); free(nxt);
}

/* src/sdr_func.c:1088-1102: x = IQ * CSCALE (float), X = FFT(x),
 * Z = X * code_fft * (1/N/N) (scale computed in float), corr = IFFT(Z). */
void orc_corr_fft(const int8_t *IQ, const float *code_fft, int N, float *corr)
{
    if (N <= 0) return;
    double *a = (double *)malloc(sizeof(double) * 2 * N);
    double *b = (double *)malloc(sizeof(double) * 2 * N);
    float s = 1.0f / N / N;
    for (int i = 0; i < N; i++) {
        a[2 * i] = (double)(IQ[2 * i] * ORC_CSCALE);
        a[2 * i + 1] = (double)(IQ[2 * i + 1] * ORC_CSCALE);
    }
    orc_fft(a, N, 0, b);
    for (int i = 0; i < N; i++) {
        double xr = b[2 * i], xi = b[2 * i + 1];
        double cr = code_fft[2 * i], ci = code_fft[2 * i + 1];
        a[2 * i] = (xr * cr - xi * ci) * s;
        a[2 * i + 1] = (xr * ci + xi * cr) * s;
    }
    orc_fft(a, N, 1, b);
    for (int i = 0; i < 2 * N; i++) corr[i] = (float)b[i];
    free(a); free(b);
}

void orc_corr_fft_cpx(const float *buff, int len_buff, int ix, int N,
                      double fs, double fc, double phi, const float *code_fft,
                      float *corr)
{
    int8_t *IQ = (int8_t *)malloc(2 * (size_t)N);
    orc_mix_carr_cpx(buff, len_buff, ix, N, fs, fc, phi, IQ);
    orc_corr_fft(IQ, code_fft, N, corr);
    free(IQ);
}

/* src/sdr_func.c:664-687: per bin, mix at fi + fds[i] with phase 0, FFT
 * correlate, P[i*N+j] += fma(re, re, im*im) (gcc -mfma contraction). */
void orc_search_code(const float *code_fft, const uint8_t *buff, int len_buff,
                     int ix, int N, double fs, double fi, const float *fds,
                     int len_fds, float *P)
{
    int8_t *IQ = (int8_t *)malloc(2 * (size_t)N);
    float *C = (float *)malloc(sizeof(float) * 2 * N);
    for (int i = 0; i < len_fds; i++) {
        orc_mix_carr(buff, len_buff, ix, N, fs, fi + fds[i], 0.0, IQ);
        orc_corr_fft(IQ, code_fft, N, C);
        for (int j = 0; j < N; j++) {
            P[(size_t)i * N + j] += fmaf(C[2 * j], C[2 * j], C[2 * j + 1] * C[2 * j + 1]);
        }
    }
    free(IQ); free(C);
}

/* src/sdr_func.c:690-706: first strict maximum in row-major order, running
 * mean in double, C/N0 = 10 log10((Pmax - Pave) / Pave / T). */
float orc_corr_max(const float *P, int N, int Nmax, int M, double T, int *ix)
{
    double pmax = 0.0, pave = 0.0;
    int n = 0;
    for (int i = 0; i < M; i++) {
        for (int j = 0; j < Nmax; j++) {
            double v = P[(size_t)i * N + j];
            pave += (v - pave) / ++n;
            if (v <= pmax) continue;
            pmax = v; ix[0] = i; ix[1] = j;
        }
    }
    return pave > 0.0 ? (float)(10.0 * log10((pmax - pave) / pave / T)) : 0.0f;
}

/* src/sdr_func.c:709-744: vertex of the parabola through the three bins
 * around the peak (the reference solves the same 3x3 system by least
 * squares); edges return the bin itself. */
double orc_fine_dop(const float *P, int N, const float *fds, int len_fds,
                    const int *ix)
{
    if (ix[0] == 0 || ix[0] == len_fds - 1) return fds[ix[0]];
    double x0 = fds[ix[0] - 1], x1 = fds[ix[0]], x2 = fds[ix[0] + 1];
    double y0 = P[(size_t)(ix[0] - 1) * N + ix[1]];
    double y1 = P[(size_t)ix[0] * N + ix[1]];
    double y2 = P[(size_t)(ix[0] + 1) * N + ix[1]];
    /* Newton divided differences: y = a + b (x-x0) + c (x-x0)(x-x1) */
    double d01 = (y1 - y0) / (x1 - x0), d12 = (y2 - y1) / (x2 - x1);
    double c = (d12 - d01) / (x2 - x0);
    if (c == 0.0) return fds[ix[0]];
    double b = d01 - c * (x0 + x1);   /* coefficient of x in c x^2 + b x + a */
    return -b / (2.0 * c);
}

/* src/sdr_func.c:757-769 */
int orc_dop_bins(double T, float dop, float max_dop, float *fds)
{
    float step = (float)(0.5 / T);
    int len = (int)(2.0 * max_dop / step) + 1;
    if (fds) for (int i = 0; i < len; i++) fds[i] = dop - max_dop + i * step;
    return len;
}

/* src/sdr_code.c:2556-2568: chip index (int)((coff*fs + i) * dx) % len_code
 * with dx = len_code / T / fs. */
void orc_res_code(const int8_t *code_I, const int8_t *code_Q, int len_code,
                  double T, double coff, double fs, int N, int Nz,
                  int8_t *code_res)
{
    double dx = len_code / T / fs;
    memset(code_res, 0, 2 * (size_t)(N + Nz));
    for (int i = 0; i < N; i++) {
        int j = (int)((coff * fs + i) * dx) % len_code;
        code_res[2 * i] = code_I[j];
        code_res[2 * i + 1] = code_Q ? code_Q[j] : code_I[j];
    }
}

/* src/sdr_code.c:2589-2608 */
void orc_gen_code_fft(const int8_t *code_I, const int8_t *code_Q,
                      int len_code, double T, double coff, double fs, int N,
                      int Nz, float *code_fft)
{
    int L = N + Nz;
    double dx = len_code / T / fs;
    double *a = (double *)calloc(2 * (size_t)L, sizeof(double));
    double *b = (double *)malloc(sizeof(double) * 2 * L);
    for (int i = 0; i < N; i++) {
        int j = (int)((coff * fs + i) * dx) % len_code;
        a[2 * i] = code_I[j];
        a[2 * i + 1] = code_Q ? code_Q[j] : 0;
    }
    orc_fft(a, L, 0, b);
    for (int i = 0; i < L; i++) {
        code_fft[2 * i] = (float)b[2 * i];
        code_fft[2 * i + 1] = (float)-b[2 * i + 1];
    }
    free(a); free(b);
}

/* src/sdr_func.c:1116-1182 (hann_window, sdr_psd_cpx): Welch PSD without
 * overlap, Hann window (float taps, float sum of squares), |X|^2 summed in
 * float over the M = len / N segments in order, matplotlib.psd scale, dB;
 * real data keeps N/2 bins, complex data is rotated to start at -fs/2. The
 * transform is the oracle's double FFT of the float-windowed segment. */
void orc_psd_cpx(const float *buff, int len_buff, int N, double fs, int IQ, float *psd)
{
    float *w = (float *)malloc(sizeof(float) * N), *p = (float *)calloc(N, sizeof(float));
    double *a = (double *)malloc(sizeof(double) * 2 * N), *b = (double *)malloc(sizeof(double) * 2 * N);
    float wss = 0.0f;
    for (int i = 0; i < N; i++) {
        w[i] = (float)(0.5 + 0.5 * cos(2.0 * 3.1415926535897932 * (i - 0.5 * (N - 1)) / (N - 1)));
        wss += w[i] * w[i];
    }
    int M = len_buff / N;
    for (int i = 0; i < M; i++) {
        for (int j = 0; j < N; j++) {
            a[2 * j] = (float)(buff[2 * ((size_t)N * i + j)] * w[j]);
            a[2 * j + 1] = (float)(buff[2 * ((size_t)N * i + j) + 1] * w[j]);
        }
        orc_fft(a, N, 0, b);
        for (int j = 0; j < N; j++) {
            float re = (float)b[2 * j], im = (float)b[2 * j + 1];
            p[j] += re * re + im * im;
        }
    }
    float scale = (float)(1.0 / M / wss / fs * (IQ == 1 ? 2.0 : 1.0));
    if (IQ == 1) {
        for (int i = 0; i < N / 2; i++) psd[i] = 10.0f * log10f(p[i] * scale);
    } else {
        for (int i = 0; i < N / 2; i++) psd[i] = 10.0f * log10f(p[N / 2 + i] * scale);
        for (int i = N / 2; i < N; i++) psd[i] = 10.0f * log10f(p[i - N / 2] * scale);
    }
    free(w); free(p); free(a); free(b);
}

/* src/sdr_ch.c:626-664 (interp_corr, CSK): the correlation, rotated so the
 * zero lag sits at n = (int)(280 R) (R = N / (len_code / 2) samples per
 * chip), linearly interpolated in double at n + i R for i = -255..255 (the
 * reference build forms n + i R as one fused multiply-add); the
 * first strict maximum of |c| (float) gives ix (0 when all are 0), the symbol
 * (uint8)(255 - ix % 256) and the taps interpolated at n + ix R + pos[k]. */
static void orc_interp(const float *C, double x, float *c)
{
    int i = (int)x;
    double a1 = x - i, a0 = 1.0 - a1;
    c[0] = (float)(a0 * C[2 * i] + a1 * C[2 * i + 2]);
    c[1] = (float)(a0 * C[2 * i + 1] + a1 * C[2 * i + 3]);
}

void orc_csk(const float *corr, int N, int len_code, const double *pos, int npos, uint8_t *sym,
             float *Cout)
{
    double R = (double)N / (len_code / 2);
    int n = (int)(280 * R);
    float *C = (float *)malloc(sizeof(float) * 4 * n);
    memcpy(C, corr + 2 * (N - n), sizeof(float) * 2 * n);
    memcpy(C + 2 * n, corr, sizeof(float) * 2 * n);
    double P_max = 0.0;
    int ix = 0;
    for (int i = -255; i <= 255; i++) {
        float c[2];
        orc_interp(C, fma((double)i, R, (double)n), c);   /* gcc -mfma contracts n + i*R */
        double P = sqrtf(c[0] * c[0] + c[1] * c[1]);
        if (P <= P_max) continue;
        P_max = P;
        ix = i;
    }
    *sym = (uint8_t)(255 - ix % 256);
    for (int k = 0; k < npos; k++) orc_interp(C, fma((double)ix, R, (double)n) + pos[k], Cout + 2 * k);
    free(C);
}
