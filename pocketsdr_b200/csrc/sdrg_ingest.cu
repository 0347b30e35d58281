// sdrg_ingest.cu - IF ingest on the device: raw front-end data -> packed
// sdr_cpx8_t IF buffers, per-channel low-pass filter, array beam-forming.
//
// Reference: the receiver's write_buff (src/sdr_rcv.c:840-936) turns one block
// of raw samples into the IF buffers through lookup tables built by gen_LUT8
// (:801-813), gen_LUTC (:773-797) and gen_LUTC_rtoc (:816-829), filters
// channels in place with sdr_lpf_apply (src/sdr_func.c:361-405, taps from
// sdr_lpf_new :311-332) and, for the multi-channel RAW formats, combines the
// RF channels into array channels (sdr_arch_combine, src/sdr_array.c:553-578,
// table of build_lut :487-498). On the CPU that is a serial pass per block
// ahead of every search and correlator; here one kernel does all of it, so
// raw bytes uploaded once become search-ready buffers without a host pass.
//
// Kernel: one CTA per tile of 1024 samples. It unpacks the tile and the 8
// samples before it (the filter's reach; the previous block's last 8
// unfiltered samples for the first tile) of every RF channel into shared
// memory, then each thread filters, packs and combines its samples. The
// filter is the reference's integer FIR, so every output byte is exact.
// Reads 1-4 raw bytes and writes one byte per channel per sample: HBM bound.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "sdrg_internal.h"

namespace sdrg {

enum { F_CPX8 = 0, F_INT8 = 1, F_INT8X2, F_RAW8, F_RAW16, F_RAW16I, F_RAW32, F_CS8, F_CS16 };

constexpr int kTile = 1024;
constexpr int kIngThreads = 256;
constexpr int kMaxRf = 8, kMaxArch = 8;

static int n_rfch(int fmt)
{
    return fmt == F_RAW8 ? 2 : fmt == F_RAW16 ? 4 : (fmt == F_RAW16I || fmt == F_RAW32) ? 8 : 1;
}

__host__ __device__ __forceinline__ uint8_t pack8(int I, int Q)
{
    return (uint8_t)(((Q & 0xF) << 4) | (I & 0xF));
}

struct IngestArgs {
    const uint8_t *raw;
    int fmt, N, nrfch, ph0;
    int rtoc_mask, lpf_mask;
    const int8_t *lut8;       // [2][65536] (INT8 formats; CS16 uses both)
    const uint8_t *lutc;      // [8][1024] (RAW formats)
    const char2 *hist_in;     // [8][8] unfiltered samples before the block
    char2 *hist_out;          // [8][8]
    uint8_t *out[kMaxRf];
    int narch;
    uint8_t *aout[kMaxArch];
    int h[kMaxRf][9];
    short2 w[kMaxArch][kMaxRf];
};

// sample n of RF channel k, as write_buff stores it (before the LPF)
__device__ __forceinline__ char2 unpack(const IngestArgs &a, int k, int n)
{
    uint8_t b;
    switch (a.fmt) {
    case F_CPX8:
        b = a.raw[n];
        break;
    case F_INT8: {
        const int I = __ldg(a.lut8 + a.raw[n]);
        if (!(a.rtoc_mask & 1)) { b = pack8(I, 0); break; }
        const int ph = (a.ph0 + n) & 3;
        b = ph == 0 ? pack8(I, 0) : ph == 1 ? pack8(0, -I) : ph == 2 ? pack8(-I, 0) : pack8(0, I);
        break;
    }
    case F_INT8X2:
        b = pack8(__ldg(a.lut8 + a.raw[2 * n]), -__ldg(a.lut8 + a.raw[2 * n + 1]));
        break;
    case F_CS8:
        b = pack8(__ldg(a.lut8 + a.raw[2 * n]), __ldg(a.lut8 + a.raw[2 * n + 1]));
        break;
    case F_CS16: {
        const uint16_t u = (uint16_t)(a.raw[4 * n] | (a.raw[4 * n + 1] << 8));
        const uint16_t v = (uint16_t)(a.raw[4 * n + 2] | (a.raw[4 * n + 3] << 8));
        b = pack8(__ldg(a.lut8 + u), __ldg(a.lut8 + 65536 + v));
        break;
    }
    case F_RAW16I:
        b = __ldg(a.lutc + k * 1024 + a.raw[2 * n + k / 4]);
        break;
    default: {   // RAW8 / RAW16 / RAW32: RF channels 2j and 2j+1 share byte j
        const int bpr = a.nrfch / 2;
        const uint8_t byte = a.raw[(size_t)bpr * n + k / 2];
        const int ph = ((a.rtoc_mask >> k) & 1) ? ((a.ph0 + n) & 3) : 0;
        b = __ldg(a.lutc + k * 1024 + (ph << 8) + byte);
    }
    }
    return make_char2((signed char)((int8_t)(uint8_t)(b << 4) >> 4), (signed char)((int8_t)b >> 4));
}

__global__ void __launch_bounds__(kIngThreads) ingest_kernel(IngestArgs a)
{
    __shared__ char2 xs[kMaxRf][kTile + 8];
    const int t0 = blockIdx.x * kTile;
    const int nk = a.nrfch;
    for (int idx = threadIdx.x; idx < kTile + 8; idx += kIngThreads) {
        const int n = t0 - 8 + idx;
        if (n >= a.N) continue;
        for (int k = 0; k < nk; ++k)
            xs[k][idx] = n < 0 ? a.hist_in[k * 8 + 8 + n] : unpack(a, k, n);
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < kTile; idx += kIngThreads) {
        const int n = t0 + idx;
        if (n >= a.N) continue;
        int yi[kMaxRf], yq[kMaxRf];
#pragma unroll
        for (int k = 0; k < kMaxRf; ++k) {
            if (k >= nk) break;
            const char2 *x = xs[k] + idx;      // x[0..8] = samples n-8 .. n
            int I = x[8].x, Q = x[8].y;
            if ((a.lpf_mask >> k) & 1) {
                const int *h = a.h[k];
                int ai = h[4] * x[4].x, aq = h[4] * x[4].y;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    ai += h[j] * (x[j].x + x[8 - j].x);
                    aq += h[j] * (x[j].y + x[8 - j].y);
                }
                I = min(7, max(-7, (ai + (1 << 12)) >> 13));
                Q = min(7, max(-7, (aq + (1 << 12)) >> 13));
            }
            yi[k] = I;
            yq[k] = Q;
            a.out[k][n] = pack8(I, Q);
        }
        for (int m = 0; m < a.narch; ++m) {
            int I = 0, Q = 0;
            for (int k = 0; k < nk; ++k) {
                const short2 w = a.w[m][k];
                I += yi[k] * w.x - yq[k] * w.y;
                Q += yi[k] * w.y + yq[k] * w.x;
            }
            I += I >= 0 ? 128 : -128;
            Q += Q >= 0 ? 128 : -128;
            I /= 256;
            Q /= 256;
            a.aout[m][n] = pack8(min(7, max(-8, I)), min(7, max(-8, Q)));
        }
    }
    // the tile holding sample N-1 keeps the block's last 8 unfiltered samples
    if (t0 <= a.N - 1 && a.N - 1 < t0 + kTile && threadIdx.x < 8 * nk) {
        const int k = threadIdx.x / 8, j = threadIdx.x % 8;
        a.hist_out[k * 8 + j] = xs[k][a.N - t0 + j];
    }
}

// ---- host tables (restating the reference's builders) -----------------------
// src/sdr_rcv.c:801-813
static void host_lut8(int fmt, double off, double scale, int8_t *out)
{
    const int n = fmt == F_CS16 ? 65536 : 256;
    if (scale <= 0.0) scale = 1.0;
    for (int i = -n / 2; i < n / 2; i++) {
        int v = (int)floor((i - off) / scale + 0.5);
        int j = fmt == F_CS16 ? (uint16_t)i : (uint8_t)i;
        out[j] = (int8_t)(v < -7 ? -7 : v > 7 ? 7 : v);
    }
}

// src/sdr_rcv.c:773-797 (gen_LUTC) and :816-829 (gen_LUTC_rtoc): the front
// end's 2-bit and 3-bit sample codes; rtoc: the 4 fs/4 phases
static void host_lutc(int fmt, int rfch, int IQ, int bits, int rtoc, uint8_t *out)
{
    static const int v2i[4] = {1, 3, -1, -3}, v2q[4] = {-1, -3, 1, 3};
    static const int v3[8] = {1, 3, 5, 7, -1, -3, -5, -7};
    for (int i = 0; i < 256; i++) {
        if (rtoc) {
            const int val = (i >> (rfch % 2 ? 4 : 0)) & 0xF;
            const int I = v3[((val << 1) & 6) + ((val >> 3) & 1)];
            out[i] = pack8(I, 0);
            out[256 + i] = pack8(0, -I);
            out[512 + i] = pack8(-I, 0);
            out[768 + i] = pack8(0, I);
            continue;
        }
        int I, Q = 0;
        if (fmt == F_RAW16I) {
            I = v2i[(i >> ((rfch % 4) * 2)) & 3];
        } else if (IQ == 1 && bits == 2) {
            I = v2i[(i >> (rfch % 2 ? 4 : 0)) & 3];
        } else if (IQ == 1 && bits == 3) {
            const int val = (i >> (rfch % 2 ? 4 : 0)) & 0xF;
            I = v3[((val << 1) & 6) + ((val >> 3) & 1)];
        } else {
            I = v2i[(i >> (rfch % 2 ? 4 : 0)) & 3];
            Q = v2q[(i >> (rfch % 2 ? 6 : 2)) & 3];
        }
        for (int p = 0; p < 4; ++p) out[p * 256 + i] = pack8(I, Q);
    }
}

// src/sdr_func.c:311-332: Hamming-windowed sinc, 9 taps, Q13
static int host_lpf_taps(double fc, double fs, int *h)
{
    if (fc <= 0.0 || fs <= 0.0 || fc >= fs * 0.5) return 0;
    const double PI = 3.1415926535897932;
    double fn = fc / fs, hd[9], sum = 0.0;
    for (int i = 0; i < 9; i++) {
        const double t = i - 4.0;
        const double s = (t == 0.0) ? 2.0 * fn : sin(2.0 * PI * fn * t) / (PI * t);
        hd[i] = s * (0.54 - 0.46 * cos(2.0 * PI * i / 8));
        sum += hd[i];
    }
    for (int i = 0; i < 9; i++) {
        int v = (int)floor((1 << 13) * hd[i] / sum + 0.5);
        v = v < -32768 ? -32768 : v > 32767 ? 32767 : v;
        h[i] = (int16_t)v;
    }
    return 1;
}

static int launch_ingest(IngestArgs &a, cudaStream_t st)
{
    if (a.N <= 0) return SDRG_OK;
    const int grid = (a.N + kTile - 1) / kTile;
    ingest_kernel<<<grid, kIngThreads, 0, st>>>(a);
    SDRG_CUDA(cudaGetLastError());
    return SDRG_OK;
}

} // namespace sdrg

using namespace sdrg;

struct sdrg_ingest {
    sdrg_ingest_cfg_t cfg;
    int nrfch = 1;
    int rtoc_mask = 0, lpf_mask = 0;
    int h[kMaxRf][9] = {};
    int8_t *lut8_dev = nullptr;     // [2][65536]
    uint8_t *lutc_dev = nullptr;    // [8][1024]
    char2 *hist_dev = nullptr;      // [2][8][8] double-buffered history
    int parity = 0;
};

// sdr_lpf_t of the drop-in calls (opaque to callers, as in the reference)
struct sdr_lpf_tag {
    int h[9];
    char2 hist[8];     // last 8 unfiltered samples of the previous call
};

extern "C" {

int sdrg_lpf_taps(double fc, double fs, int *h)
{
    int t[9];
    if (!host_lpf_taps(fc, fs, t)) return 0;
    if (h) memcpy(h, t, sizeof(t));
    return 1;
}

sdrg_ingest_t *sdrg_ingest_new(const sdrg_ingest_cfg_t *cfg)
{
    if (!cfg || cfg->fmt < F_INT8 || cfg->fmt > F_CS16 || cfg->N <= 0 || cfg->narch < 0 ||
        cfg->narch > kMaxArch) {
        set_error(SDRG_ERR_ARG, "sdrg_ingest_new: bad format %d, N %d or narch %d",
                  cfg ? cfg->fmt : -1, cfg ? cfg->N : 0, cfg ? cfg->narch : 0);
        return nullptr;
    }
    const int fmt = cfg->fmt;
    const int multi = fmt == F_RAW8 || fmt == F_RAW16 || fmt == F_RAW16I || fmt == F_RAW32;
    if (cfg->narch > 0 && !multi) {
        set_error(SDRG_ERR_ARG, "sdrg_ingest_new: array channels need a multi-channel RAW format");
        return nullptr;
    }
    Device *dev;
    cudaStream_t st;
    if (ensure_device(&dev) || thread_stream(&st)) return nullptr;
    sdrg_ingest_t *g = new sdrg_ingest_t();
    g->cfg = *cfg;
    g->nrfch = n_rfch(fmt);
    const int int8fmt = fmt == F_INT8 || fmt == F_INT8X2 || fmt == F_CS8 || fmt == F_CS16;
    std::vector<int8_t> lut8(2 * 65536, 0);
    std::vector<uint8_t> lutc(kMaxRf * 1024, 0);
    for (int k = 0; k < g->nrfch; ++k) {
        // real sampling selects the fs/4 real-to-complex tables
        // (rtoc_of, src/sdr_rcv.c:51-54)
        if (cfg->IQ[k] == 1) g->rtoc_mask |= 1 << k;
    }
    if (int8fmt) {
        host_lut8(fmt, cfg->lut_off[0], cfg->lut_scale[0], lut8.data());
        if (fmt == F_CS16) host_lut8(fmt, cfg->lut_off[1], cfg->lut_scale[1], lut8.data() + 65536);
    } else {
        for (int k = 0; k < g->nrfch; ++k)
            host_lutc(fmt, k, cfg->IQ[k], cfg->bits[k], (g->rtoc_mask >> k) & 1,
                      lutc.data() + k * 1024);
    }
    // channels the reference filters in write_buff: all RF channels of
    // RAW8 / RAW16 / RAW32, channel 0 otherwise (src/sdr_rcv.c:872-924)
    const int nlpf = (fmt == F_RAW8 || fmt == F_RAW16 || fmt == F_RAW32) ? g->nrfch : 1;
    for (int k = 0; k < nlpf; ++k)
        if (host_lpf_taps(cfg->lpf_fc[k], cfg->fs, g->h[k])) g->lpf_mask |= 1 << k;
    bool ok = cudaMalloc(&g->lut8_dev, lut8.size()) == cudaSuccess &&
              cudaMalloc(&g->lutc_dev, lutc.size()) == cudaSuccess &&
              cudaMalloc(&g->hist_dev, 2 * kMaxRf * 8 * sizeof(char2)) == cudaSuccess &&
              cudaMemcpyAsync(g->lut8_dev, lut8.data(), lut8.size(), cudaMemcpyHostToDevice, st) ==
                  cudaSuccess &&
              cudaMemcpyAsync(g->lutc_dev, lutc.data(), lutc.size(), cudaMemcpyHostToDevice, st) ==
                  cudaSuccess &&
              cudaMemsetAsync(g->hist_dev, 0, 2 * kMaxRf * 8 * sizeof(char2), st) == cudaSuccess &&
              cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) {
        cuda_error(cudaGetLastError(), "sdrg_ingest_new");
        sdrg_ingest_free(g);
        return nullptr;
    }
    return g;
}

void sdrg_ingest_free(sdrg_ingest_t *g)
{
    if (!g) return;
    if (g->lut8_dev) cudaFree(g->lut8_dev);
    if (g->lutc_dev) cudaFree(g->lutc_dev);
    if (g->hist_dev) cudaFree(g->hist_dev);
    delete g;
}

int sdrg_ingest_run(sdrg_ingest_t *g, const uint8_t *raw_dev, int64_t ix, uint8_t *const *buf_dev,
                    int base, void *stream)
{
    if (!g || !raw_dev || !buf_dev || base < 0 || ix < 0)
        return set_error(SDRG_ERR_ARG, "sdrg_ingest_run: null argument or negative base / ix");
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    IngestArgs a = {};
    a.raw = raw_dev;
    a.fmt = g->cfg.fmt;
    a.N = g->cfg.N;
    a.nrfch = g->nrfch;
    a.ph0 = (int)((ix * (int64_t)g->cfg.N) & 3);    // src/sdr_rcv.c:846
    a.rtoc_mask = g->rtoc_mask;
    a.lpf_mask = g->lpf_mask;
    a.lut8 = g->lut8_dev;
    a.lutc = g->lutc_dev;
    a.hist_in = g->hist_dev + g->parity * kMaxRf * 8;
    a.hist_out = g->hist_dev + (g->parity ^ 1) * kMaxRf * 8;
    for (int k = 0; k < g->nrfch; ++k) {
        if (!buf_dev[k]) return set_error(SDRG_ERR_ARG, "sdrg_ingest_run: no buffer %d", k);
        a.out[k] = buf_dev[k] + base;
        memcpy(a.h[k], g->h[k], sizeof(a.h[k]));
    }
    a.narch = 0;
    for (int m = 0; m < g->cfg.narch; ++m) {
        if (!g->cfg.arch_on[m]) continue;   // sdr_arch_combine returns for scale <= 0
        uint8_t *o = buf_dev[g->nrfch + m];
        if (!o) return set_error(SDRG_ERR_ARG, "sdrg_ingest_run: no buffer %d", g->nrfch + m);
        a.aout[a.narch] = o + base;
        for (int k = 0; k < g->nrfch; ++k)
            a.w[a.narch][k] = make_short2(g->cfg.w[m][k][0], g->cfg.w[m][k][1]);
        a.narch++;
    }
    if ((e = launch_ingest(a, (cudaStream_t)stream))) return e;
    g->parity ^= 1;
    return SDRG_OK;
}

// ---- drop-in LPF -----------------------------------------------------------------
sdr_lpf_t *sdr_lpf_new(double fc, double fs)
{
    int h[9];
    if (!host_lpf_taps(fc, fs, h)) return nullptr;   // as the reference: NULL for a bad cutoff
    sdr_lpf_t *f = new sdr_lpf_t();
    memcpy(f->h, h, sizeof(h));
    memset(f->hist, 0, sizeof(f->hist));
    return f;
}

void sdr_lpf_free(sdr_lpf_t *lpf)
{
    delete lpf;
}

void sdr_lpf_apply(sdr_lpf_t *lpf, sdr_cpx8_t *data, int N)
{
    if (!lpf || !data || N <= 0) return;
    Device *dev;
    cudaStream_t st;
    int e;
    ThreadCtx &c = tctx();
    c.host[0].pinned = true;
    const size_t nb = ((size_t)N + 255) / 256 * 256;
    if ((e = ensure_device(&dev)) || (e = thread_stream(&st)) || (e = c.host[0].reserve(2 * nb)) ||
        (e = c.dev[0].reserve(2 * nb + 2 * kMaxRf * 8 * sizeof(char2))))
        return;   // error recorded; data left unfiltered
    uint8_t *h_in = (uint8_t *)c.host[0].ptr, *h_out = h_in + nb;
    uint8_t *d_in = (uint8_t *)c.dev[0].ptr, *d_out = d_in + nb;
    char2 *d_hist = (char2 *)(d_in + 2 * nb);
    memcpy(h_in, data, (size_t)N);
    IngestArgs a = {};
    a.raw = d_in;
    a.fmt = F_CPX8;
    a.N = N;
    a.nrfch = 1;
    a.lpf_mask = 1;
    a.hist_in = d_hist;
    a.hist_out = d_hist + kMaxRf * 8;
    a.out[0] = d_out;
    memcpy(a.h[0], lpf->h, sizeof(a.h[0]));
    if (cudaMemcpyAsync(d_in, h_in, (size_t)N, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(d_hist, lpf->hist, sizeof(lpf->hist), cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        launch_ingest(a, st) ||
        cudaMemcpyAsync(h_out, d_out, (size_t)N, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cuda_error(cudaGetLastError(), "sdr_lpf_apply");
        return;
    }
    // next history: the last 8 of (history, this call's unfiltered input)
    char2 nh[8];
    for (int j = 0; j < 8; ++j) {
        const int n = N - 8 + j;
        if (n < 0) {
            nh[j] = lpf->hist[8 + n];
        } else {
            const uint8_t b = h_in[n];
            nh[j] = make_char2((signed char)((int8_t)(uint8_t)(b << 4) >> 4),
                               (signed char)((int8_t)b >> 4));
        }
    }
    memcpy(lpf->hist, nh, sizeof(nh));
    memcpy(data, h_out, (size_t)N);
}

} // extern "C"
