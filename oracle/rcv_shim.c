/*
 * rcv_shim.c - TEST INFRASTRUCTURE (the checker): exposes the reference
 * receiver's IF-ingest path to the parity tests.
 *
 * Pocket SDR builds its IF buffers in src/sdr_rcv.c: raw front-end data ->
 * lookup tables (gen_LUT8 :801-813, gen_LUTC :773-797, gen_LUTC_rtoc
 * :816-829) -> packed sdr_cpx8_t buffers (write_buff :840-936), with the
 * per-channel LPF (sdr_lpf_new / sdr_lpf_apply, src/sdr_func.c:311-405) and
 * the array beam-forming combine (sdr_arch_combine, src/sdr_array.c:553-578)
 * applied in the same call. Those builders and write_buff are file-local
 * (static), so this file compiles src/sdr_rcv.c in its own translation unit:
 * the #include below reads it from the reference tree at build time
 * (oracle/Makefile); nothing of it is copied into this repository. The shim
 * only assembles a receiver state (sdr_rcv_t) around buffers, tables, LPFs
 * and array weights the way sdr_rcv_start (src/sdr_rcv.c:1368-1381) and
 * sdr_arch_set_beam (src/sdr_array.c:501-542) do, then calls write_buff.
 *
 * The Pocket SDR front-end USB driver (src/sdr_dev.c, src/sdr_usb.c) needs
 * libusb, which this machine lacks; sdr_rcv.c refers to it, the ingest path
 * never opens a device, so those entry points are stubs that fail.
 */
#include "sdr_rcv.c"

/* ---- libusb front-end driver stubs (never called by write_buff) --------- */
int sdr_usb_req(sdr_usb_t *usb, int mode, uint8_t req, uint16_t val, uint8_t *data, int size)
{
    (void)usb; (void)mode; (void)req; (void)val; (void)data; (void)size;
    return 0;
}
sdr_dev_t *sdr_dev_open(int bus, int port) { (void)bus; (void)port; return NULL; }
void sdr_dev_close(sdr_dev_t *dev) { (void)dev; }
int sdr_dev_start(sdr_dev_t *dev) { (void)dev; return 0; }
int sdr_dev_stop(sdr_dev_t *dev) { (void)dev; return 0; }
int sdr_dev_read(sdr_dev_t *dev, uint8_t *buff, int size)
{
    (void)dev; (void)buff; (void)size;
    return 0;
}
int sdr_dev_get_info(sdr_dev_t *dev, int *fmt, double *fs, double *fo, int *IQ, int *bits)
{
    (void)dev; (void)fmt; (void)fs; (void)fo; (void)IQ; (void)bits;
    return 0;
}
int sdr_dev_get_gain(sdr_dev_t *dev, int ch) { (void)dev; (void)ch; return 0; }
int sdr_dev_set_gain(sdr_dev_t *dev, int ch, int gain) { (void)dev; (void)ch; (void)gain; return 0; }
int sdr_dev_get_filt(sdr_dev_t *dev, int ch, double *bw, double *freq, int *order)
{
    (void)dev; (void)ch; (void)bw; (void)freq; (void)order;
    return 0;
}
int sdr_dev_set_filt(sdr_dev_t *dev, int ch, double bw, double freq, int order)
{
    (void)dev; (void)ch; (void)bw; (void)freq; (void)order;
    return 0;
}

/* ---- checker entry points ------------------------------------------------ */

/* The reference's raw -> int8 table (gen_LUT8): 256 entries, 65536 for CS16. */
void orr_gen_lut8(int fmt, double off, double scale, int8_t *out)
{
    int n = fmt == SDR_FMT_CS16 ? 65536 : 256;
    int8_t *t = gen_LUT8(fmt, off, scale);
    memcpy(out, t, (size_t)n);
    sdr_free(t);
}

/* The reference's raw byte -> sdr_cpx8_t table of one RF channel: 1024
 * entries (4 fs/4 phases x 256) when rtoc, else 256 (gen_LUTC_rtoc,
 * gen_LUTC). */
void orr_gen_lutc(int fmt, int rfch, int IQ, int bits, int rtoc, uint8_t *out)
{
    sdr_cpx8_t *t = rtoc ? gen_LUTC_rtoc(rfch) : gen_LUTC(fmt, rfch, IQ, bits);
    memcpy(out, t, rtoc ? 1024 : 256);
    sdr_free(t);
}

/* The taps sdr_lpf_new computes (the first LPF_N_TAP ints of its private
 * state struct, src/sdr_func.c:70-74). Returns 0 when no filter is made. */
int orr_lpf_taps(double fc, double fs, int *h)
{
    sdr_lpf_t *lpf = sdr_lpf_new(fc, fs);
    if (!lpf) return 0;
    memcpy(h, lpf, 9 * sizeof(int));
    sdr_lpf_free(lpf);
    return 1;
}

/* A receiver state for write_buff: fmt, N samples per block, per RF channel
 * sampling type / bits / LPF cutoff (<= 0: none), the int8 table offsets
 * and scales ([1]: CS16 Q), and narch array channels with Q8 weights
 * w[(m * nrfch + j) * 2 + {0,1}] (enabled when arch_on[m]). Buffers hold
 * N * MAX_BUFF samples like the receiver's (sdr_rcv.c:698). */
void *orr_rcv_new(int fmt, int N, const int *IQ, const int *bits, const double *off,
                  const double *scale, const double *lpf_fc, double fs, int narch,
                  const int16_t *w, const int *arch_on)
{
    sdr_rcv_t *rcv = (sdr_rcv_t *)sdr_malloc(sizeof(sdr_rcv_t));
    rcv->fmt = fmt;
    rcv->N = N;
    rcv->fs = fs;
    rcv->nrfch = num_rfch(fmt);
    rcv->narch = narch;
    for (int k = 0; k < rcv->nrfch; k++) {
        rcv->rfch[k].IQ = IQ[k];
        rcv->rfch[k].bits = bits[k];
    }
    if (fmt == SDR_FMT_INT8 || fmt == SDR_FMT_INT8X2 || fmt == SDR_FMT_CS8 ||
        fmt == SDR_FMT_CS16) {
        rcv->rfch[0].LUT = (void *)gen_LUT8(fmt, off[0], scale[0]);
        if (fmt == SDR_FMT_CS16) rcv->rfch[1].LUT = (void *)gen_LUT8(fmt, off[1], scale[1]);
    } else {
        for (int k = 0; k < rcv->nrfch; k++) {
            rcv->rfch[k].LUT = rtoc_of(rcv, k) ? (void *)gen_LUTC_rtoc(k) :
                (void *)gen_LUTC(fmt, k, IQ[k], bits[k]);
        }
    }
    for (int k = 0; k < rcv->nrfch; k++) {
        if (lpf_fc[k] > 0.0) rcv->rfch[k].lpf = sdr_lpf_new(lpf_fc[k], fs);
    }
    for (int m = 0; m < narch; m++) {
        sdr_arch_t *a = rcv->arch + m;
        a->scale = arch_on[m] ? 1.0 : 0.0;
        for (int j = 0; j < rcv->nrfch; j++) {
            int32_t wr = w[(m * rcv->nrfch + j) * 2], wi = w[(m * rcv->nrfch + j) * 2 + 1];
            a->w[j * 2] = (int16_t)wr;
            a->w[j * 2 + 1] = (int16_t)wi;
            for (int b = 0; b < 256; b++) {   /* as build_lut, src/sdr_array.c:487-498 */
                int32_t I = SDR_CPX8_I((sdr_cpx8_t)b), Q = SDR_CPX8_Q((sdr_cpx8_t)b);
                a->LUT[j][b].I = I * wr - Q * wi;
                a->LUT[j][b].Q = I * wi + Q * wr;
            }
        }
    }
    for (int b = 0; b < rcv->nrfch + narch; b++) rcv->buff[b] = sdr_buff_new(N * MAX_BUFF, 2);
    return rcv;
}

/* One block: write_buff(rcv, raw, ix); then block ix of every buffer (RF
 * channels, then array channels) is at out + b * N. */
void orr_write_buff(void *p, const uint8_t *raw, int64_t ix, uint8_t *out)
{
    sdr_rcv_t *rcv = (sdr_rcv_t *)p;
    write_buff(rcv, raw, ix);
    int base = rcv->N * (int)(ix % MAX_BUFF);
    for (int b = 0; b < rcv->nrfch + rcv->narch; b++) {
        memcpy(out + (size_t)b * rcv->N, rcv->buff[b]->data + base, (size_t)rcv->N);
    }
}

void orr_rcv_free(void *p)
{
    sdr_rcv_t *rcv = (sdr_rcv_t *)p;
    if (!rcv) return;
    for (int k = 0; k < rcv->nrfch; k++) {
        sdr_free(rcv->rfch[k].LUT);
        sdr_lpf_free(rcv->rfch[k].lpf);
    }
    for (int b = 0; b < rcv->nrfch + rcv->narch; b++) sdr_buff_free(rcv->buff[b]);
    sdr_free(rcv);
}

/* Plain sdr_lpf_apply on a caller buffer with a persistent filter. */
void *orr_lpf_new(double fc, double fs) { return sdr_lpf_new(fc, fs); }
void orr_lpf_apply(void *lpf, uint8_t *data, int N) { sdr_lpf_apply((sdr_lpf_t *)lpf, data, N); }
void orr_lpf_free(void *lpf) { sdr_lpf_free((sdr_lpf_t *)lpf); }
