/*
 * ingest_oracle.c - TEST INFRASTRUCTURE: plain-C restatement of Pocket SDR's
 * IF ingest (raw front-end data -> packed sdr_cpx8_t IF buffers), the
 * checker for the GPU ingest kernel. Pinned in tests/test_oracle.py against
 * the reference's own code (oracle/rcv_shim.c) where that is built.
 *
 * Follows, per block of N samples:
 *   raw -> int8 / cpx8 tables        src/sdr_rcv.c:773-829 (gen_LUTC,
 *                                    gen_LUT8, gen_LUTC_rtoc)
 *   raw -> buffers per format        src/sdr_rcv.c:840-921 (write_buff)
 *   9-tap LPF, in place, history     src/sdr_func.c:311-405 (sdr_lpf_new,
 *                                    sdr_lpf_apply)
 *   array combine                    src/sdr_array.c:487-498, 553-578
 *                                    (build_lut, sdr_arch_combine)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "sdr_oracle.h"

enum { F_INT8 = 1, F_INT8X2, F_RAW8, F_RAW16, F_RAW16I, F_RAW32, F_CS8, F_CS16 };

static int clipi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

/* SDR_CPX8 (src/pocket_sdr.h:105): I in the low nibble, Q in the high one */
static uint8_t cpx8(int I, int Q) { return (uint8_t)(((Q & 0xF) << 4) | (I & 0xF)); }
static int cpx8_i(uint8_t b) { return (int)(int8_t)(uint8_t)(b << 4) >> 4; }
static int cpx8_q(uint8_t b) { return (int)(int8_t)b >> 4; }

static int n_rfch(int fmt)
{
    return fmt == F_RAW8 ? 2 : fmt == F_RAW16 ? 4 : (fmt == F_RAW16I || fmt == F_RAW32) ? 8 : 1;
}

/* src/sdr_rcv.c:801-813: round((raw - off) / scale), clipped to +-7 */
void orc_gen_lut8(int fmt, double off, double scale, int8_t *out)
{
    int n = fmt == F_CS16 ? 65536 : 256;
    if (scale <= 0.0) scale = 1.0;
    for (int i = -n / 2; i < n / 2; i++) {
        int v = (int)floor((i - off) / scale + 0.5);
        int j = fmt == F_CS16 ? (uint16_t)i : (uint8_t)i;
        out[j] = (int8_t)clipi(v, -7, 7);
    }
}

/* src/sdr_rcv.c:773-797 and :816-829: the front end's 2-bit / 3-bit sample
 * codes per RF channel; rtoc: 4 x 256 entries, one per fs/4 phase
 * (x e^{-i pi/2 phase}) */
void orc_gen_lutc(int fmt, int rfch, int IQ, int bits, int rtoc, uint8_t *out)
{
    static const int v2i[4] = {1, 3, -1, -3}, v2q[4] = {-1, -3, 1, 3};
    static const int v3[8] = {1, 3, 5, 7, -1, -3, -5, -7};
    for (int i = 0; i < 256; i++) {
        if (rtoc) {
            int val = (i >> (rfch % 2 ? 4 : 0)) & 0xF;
            int I = v3[((val << 1) & 6) + ((val >> 3) & 1)];
            out[i] = cpx8(I, 0);
            out[256 + i] = cpx8(0, -I);
            out[512 + i] = cpx8(-I, 0);
            out[768 + i] = cpx8(0, I);
            continue;
        }
        int I, Q = 0;
        if (fmt == F_RAW16I) {
            I = v2i[(i >> ((rfch % 4) * 2)) & 3];
        } else if (IQ == 1 && bits == 2) {
            I = v2i[(i >> (rfch % 2 ? 4 : 0)) & 3];
        } else if (IQ == 1 && bits == 3) {
            int val = (i >> (rfch % 2 ? 4 : 0)) & 0xF;
            I = v3[((val << 1) & 6) + ((val >> 3) & 1)];
        } else {
            I = v2i[(i >> (rfch % 2 ? 4 : 0)) & 3];
            Q = v2q[(i >> (rfch % 2 ? 6 : 2)) & 3];
        }
        out[i] = cpx8(I, Q);
    }
}

/* src/sdr_func.c:311-332: windowed-sinc (Hamming) taps in Q13 */
int orc_lpf_taps(double fc, double fs, int *h)
{
    if (fc <= 0.0 || fs <= 0.0 || fc >= fs * 0.5) return 0;
    const double PI = 3.1415926535897932;
    double fn = fc / fs, hd[9], sum = 0.0;
    for (int i = 0; i < 9; i++) {
        double t = i - 4.0;
        double s = (t == 0.0) ? 2.0 * fn : sin(2.0 * PI * fn * t) / (PI * t);
        hd[i] = s * (0.54 - 0.46 * cos(2.0 * PI * i / 8));
        sum += hd[i];
    }
    for (int i = 0; i < 9; i++) {
        int v = (int)floor((1 << 13) * hd[i] / sum + 0.5);
        h[i] = (int16_t)clipi(v, -32768, 32767);
    }
    return 1;
}

/* src/sdr_func.c:361-405: out[n] = clip((h4 x[n-4] + sum_k h_k (x[n-8+k] +
 * x[n-k]) + 2^12) >> 13, +-7) per component, x[-8..-1] = the previous
 * call's last 8 inputs (zeros at first) */
struct orc_ingest {
    int fmt, N, nrfch, narch;
    int rtoc[8];
    int8_t lut8[2][65536];
    uint8_t lutc[8][1024];
    int lpf[8], h[8][9];
    int8_t hist[8][8][2];
    int16_t w[8][8][2];
    int arch_on[8];
};

static void lpf_block(const int *h, int8_t hist[8][2], uint8_t *d, int N)
{
    int8_t *x = (int8_t *)malloc(2 * (size_t)(N + 8));
    memcpy(x, hist, 16);
    for (int i = 0; i < N; i++) { x[2 * (8 + i)] = (int8_t)cpx8_i(d[i]); x[2 * (8 + i) + 1] = (int8_t)cpx8_q(d[i]); }
    for (int i = 0; i < N; i++) {
        int a[2];
        for (int c = 0; c < 2; c++) {
            const int8_t *p = x + 2 * i + c;
            int acc = h[4] * p[2 * 4];
            for (int k = 0; k < 4; k++) acc += h[k] * (p[2 * k] + p[2 * (8 - k)]);
            a[c] = clipi((acc + (1 << 12)) >> 13, -7, 7);
        }
        d[i] = cpx8(a[0], a[1]);
    }
    memcpy(hist, x + 2 * N, 16);
    free(x);
}

void *orc_ingest_new(int fmt, int N, const int *IQ, const int *bits, const double *off,
                     const double *scale, const double *lpf_fc, double fs, int narch,
                     const int16_t *w, const int *arch_on)
{
    struct orc_ingest *g = (struct orc_ingest *)calloc(1, sizeof(*g));
    g->fmt = fmt; g->N = N; g->nrfch = n_rfch(fmt); g->narch = narch;
    int int8fmt = fmt == F_INT8 || fmt == F_INT8X2 || fmt == F_CS8 || fmt == F_CS16;
    for (int k = 0; k < g->nrfch; k++) g->rtoc[k] = IQ[k] == 1;
    if (int8fmt) {
        orc_gen_lut8(fmt, off[0], scale[0], g->lut8[0]);
        if (fmt == F_CS16) orc_gen_lut8(fmt, off[1], scale[1], g->lut8[1]);
    } else {
        for (int k = 0; k < g->nrfch; k++)
            orc_gen_lutc(fmt, k, IQ[k], bits[k], g->rtoc[k], g->lutc[k]);
    }
    for (int k = 0; k < g->nrfch; k++) g->lpf[k] = orc_lpf_taps(lpf_fc[k], fs, g->h[k]);
    for (int m = 0; m < narch; m++) {
        g->arch_on[m] = arch_on[m];
        for (int j = 0; j < g->nrfch; j++) {
            g->w[m][j][0] = w[(m * g->nrfch + j) * 2];
            g->w[m][j][1] = w[(m * g->nrfch + j) * 2 + 1];
        }
    }
    return g;
}

/* One block of raw data at block counter ix into out[(nrfch + narch) * N]
 * (RF channels, then array channels; an array channel that is off leaves
 * its row as it was). */
void orc_ingest_write(void *p, const uint8_t *raw, int64_t ix, uint8_t *out)
{
    struct orc_ingest *g = (struct orc_ingest *)p;
    const int N = g->N, ph0 = (int)((ix * N) & 3);
    for (int i = 0; i < N; i++) {
        const int ph = (ph0 + i) & 3;
        switch (g->fmt) {
        case F_INT8: {
            int I = g->lut8[0][raw[i]];
            out[i] = !g->rtoc[0] ? cpx8(I, 0) : ph == 0 ? cpx8(I, 0) : ph == 1 ? cpx8(0, -I) :
                     ph == 2 ? cpx8(-I, 0) : cpx8(0, I);
            break;
        }
        case F_INT8X2: out[i] = cpx8(g->lut8[0][raw[2 * i]], -g->lut8[0][raw[2 * i + 1]]); break;
        case F_CS8: out[i] = cpx8(g->lut8[0][raw[2 * i]], g->lut8[0][raw[2 * i + 1]]); break;
        case F_CS16: {
            uint16_t a = (uint16_t)(raw[4 * i] | (raw[4 * i + 1] << 8));
            uint16_t b = (uint16_t)(raw[4 * i + 2] | (raw[4 * i + 3] << 8));
            out[i] = cpx8(g->lut8[0][a], g->lut8[1][b]);
            break;
        }
        case F_RAW16I:
            for (int k = 0; k < 8; k++) out[(size_t)k * N + i] = g->lutc[k][raw[2 * i + k / 4]];
            break;
        default: {   /* RAW8 / RAW16 / RAW32: two RF channels per byte */
            const int bpr = g->nrfch / 2;
            for (int k = 0; k < g->nrfch; k++) {
                const uint8_t byte = raw[(size_t)bpr * i + k / 2];
                out[(size_t)k * N + i] = g->rtoc[k] ? g->lutc[k][(ph << 8) | byte] : g->lutc[k][byte];
            }
        }
        }
    }
    const int nlpf = (g->fmt == F_RAW8 || g->fmt == F_RAW16 || g->fmt == F_RAW32) ? g->nrfch : 1;
    for (int k = 0; k < nlpf; k++)
        if (g->lpf[k]) lpf_block(g->h[k], g->hist[k], out + (size_t)k * N, N);
    const int multi = g->fmt == F_RAW8 || g->fmt == F_RAW16 || g->fmt == F_RAW16I || g->fmt == F_RAW32;
    if (!multi || g->nrfch < 2) return;
    for (int m = 0; m < g->narch; m++) {
        if (!g->arch_on[m]) continue;
        uint8_t *o = out + (size_t)(g->nrfch + m) * N;
        for (int i = 0; i < N; i++) {
            int32_t I = 0, Q = 0;
            for (int j = 0; j < g->nrfch; j++) {
                const uint8_t b = out[(size_t)j * N + i];
                const int32_t x = cpx8_i(b), y = cpx8_q(b);
                const int32_t wr = g->w[m][j][0], wi = g->w[m][j][1];
                I += x * wr - y * wi;
                Q += x * wi + y * wr;
            }
            I += I >= 0 ? 128 : -128;
            Q += Q >= 0 ? 128 : -128;
            I /= 256;
            Q /= 256;
            o[i] = cpx8(clipi(I, -8, 7), clipi(Q, -8, 7));
        }
    }
}

void orc_ingest_free(void *p) { free(p); }

/* sdr_lpf_apply on a caller buffer with a persistent 8-sample history */
struct orc_lpf { int h[9]; int8_t hist[8][2]; };
void *orc_lpf_new(double fc, double fs)
{
    struct orc_lpf *f = (struct orc_lpf *)calloc(1, sizeof(*f));
    if (!orc_lpf_taps(fc, fs, f->h)) { free(f); return NULL; }
    return f;
}
void orc_lpf_apply(void *p, uint8_t *data, int N)
{
    struct orc_lpf *f = (struct orc_lpf *)p;
    if (f && N > 0) lpf_block(f->h, f->hist, data, N);
}
void orc_lpf_free(void *p) { free(p); }
