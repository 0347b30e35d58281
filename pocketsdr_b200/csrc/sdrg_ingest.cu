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
// Kernel (one instantiation per format): one CTA per tile of 1024 samples,
// 4 consecutive samples per thread. It unpacks the tile and the 8 samples
// before it (the filter's reach; the previous block's last 8 unfiltered
// samples for the first tile) of every RF channel into shared memory as
// packed bytes (tables staged in shared memory, raw bytes read with one
// vector load per 4 samples), then each thread filters (the reference's
// integer FIR on nibbles extracted with bfe), packs and stores 4 samples per
// channel as one 32-bit word and forms the array channels. Every output byte
// is exact. Reads 1-4 raw bytes and writes one byte per channel per sample.
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
    int N, ph0;
    int rtoc_mask, lpf_mask;
    int vec;                  // raw 16-byte aligned and outputs 4-byte aligned
    const int8_t *lut8;       // [2][65536] (INT8 formats; CS16 uses both)
    const uint8_t *lutc;      // [8][1024] (RAW formats)
    const uint8_t *hist_in;   // [8][8] packed samples before the block (unfiltered)
    uint8_t *hist_out;        // [8][8]
    uint8_t *out[kMaxRf];
    int narch;
    uint8_t *aout[kMaxArch];
    int amask[kMaxArch];      // RF channels with a non-zero weight per array channel
    int h[kMaxRf][9];
    short2 w[kMaxArch][kMaxRf];
};

__host__ __device__ constexpr int bps_of(int f)
{
    return (f == F_CPX8 || f == F_INT8 || f == F_RAW8) ? 1
         : (f == F_INT8X2 || f == F_CS8 || f == F_RAW16 || f == F_RAW16I) ? 2 : 4;
}
__host__ __device__ constexpr int nrf_of(int f)
{
    return f == F_RAW8 ? 2 : f == F_RAW16 ? 4 : (f == F_RAW16I || f == F_RAW32) ? 8 : 1;
}

// sign-extended 4-bit field at bit `pos` (the I or Q nibble of a packed sample)
__device__ __forceinline__ int nib(uint32_t w, int pos)
{
    int r;
    asm("bfe.s32 %0, %1, %2, 4;" : "=r"(r) : "r"(w), "r"(pos));
    return r;
}

// Packed byte (as write_buff stores it, before the LPF) of RF channel k for
// one sample whose raw bytes are `b` (little-endian, bps_of(FMT) bytes), at
// fs/4 phase ph.
template <int FMT>
__device__ __forceinline__ uint32_t unpack1(uint32_t b, int k, int ph, const IngestArgs &a,
                                            const uint8_t *lutc, const int8_t *lut8)
{
    if constexpr (FMT == F_CPX8) {
        return b & 0xFF;
    } else if constexpr (FMT == F_INT8) {
        const int I = lut8[b & 0xFF];
        if (!(a.rtoc_mask & 1)) return pack8(I, 0);
        return ph == 0 ? pack8(I, 0) : ph == 1 ? pack8(0, -I) : ph == 2 ? pack8(-I, 0) : pack8(0, I);
    } else if constexpr (FMT == F_INT8X2) {
        return pack8(lut8[b & 0xFF], -lut8[(b >> 8) & 0xFF]);
    } else if constexpr (FMT == F_CS8) {
        return pack8(lut8[b & 0xFF], lut8[(b >> 8) & 0xFF]);
    } else if constexpr (FMT == F_CS16) {
        return pack8(__ldg(a.lut8 + (b & 0xFFFF)), __ldg(a.lut8 + 65536 + (b >> 16)));
    } else if constexpr (FMT == F_RAW16I) {
        return lutc[k * 1024 + ((b >> (8 * (k / 4))) & 0xFF)];
    } else {   // RAW8 / RAW16 / RAW32: RF channels 2j and 2j+1 share byte j
        const int p = ((a.rtoc_mask >> k) & 1) ? ph : 0;
        return lutc[k * 1024 + (p << 8) + ((b >> (8 * (k / 2))) & 0xFF)];
    }
}

// raw bytes of sample s of a loaded quad (4 samples)
template <int BPS>
__device__ __forceinline__ uint32_t sample_bytes(const uint32_t *rw, int s)
{
    if constexpr (BPS == 1) return (rw[0] >> (8 * s)) & 0xFF;
    else if constexpr (BPS == 2) return (rw[s >> 1] >> (16 * (s & 1))) & 0xFFFF;
    else return rw[s];
}

// One CTA per tile of kTile samples (256 threads x 4 samples): unpack the
// tile and the 8 samples before it into shared memory (packed bytes, one
// 32-bit word per 4 samples and channel), then filter, pack, store and
// combine 4 samples per thread.
template <int FMT>
__global__ void __launch_bounds__(kIngThreads) ingest_kernel(IngestArgs a)
{
    constexpr int NRF = nrf_of(FMT), BPS = bps_of(FMT), QW = (kTile + 8) / 4;
    __shared__ uint32_t xs[NRF][QW];
    __shared__ uint8_t lutc[(FMT >= F_RAW8 && FMT <= F_RAW32) ? NRF * 1024 : 4];
    __shared__ int8_t lut8[(FMT == F_INT8 || FMT == F_INT8X2 || FMT == F_CS8) ? 256 : 4];
    if constexpr (FMT >= F_RAW8 && FMT <= F_RAW32) {
        for (int i = threadIdx.x; i < NRF * 256; i += kIngThreads)
            ((uint32_t *)lutc)[i] = __ldg((const uint32_t *)a.lutc + i);
    }
    if constexpr (FMT == F_INT8 || FMT == F_INT8X2 || FMT == F_CS8) {
        if (threadIdx.x < 64) ((uint32_t *)lut8)[threadIdx.x] = __ldg((const uint32_t *)a.lut8 + threadIdx.x);
    }
    __syncthreads();
    const int t0 = blockIdx.x * kTile;
    for (int qd = threadIdx.x; qd < QW; qd += kIngThreads) {
        const int n0 = t0 - 8 + 4 * qd;             // first sample of the quad
        uint32_t wq[NRF];
#pragma unroll
        for (int k = 0; k < NRF; ++k) wq[k] = 0u;
        if (n0 < 0) {                               // before the block: history
#pragma unroll
            for (int k = 0; k < NRF; ++k)
                wq[k] = *(const uint32_t *)(a.hist_in + k * 8 + 8 + n0);
        } else if (n0 < a.N) {
            uint32_t rw[BPS];
            const bool full = n0 + 4 <= a.N;
            if (full && a.vec) {
                const uint8_t *src = a.raw + (size_t)n0 * BPS;
                if constexpr (BPS == 1) rw[0] = __ldg((const uint32_t *)src);
                else if constexpr (BPS == 2) { const uint2 v = __ldg((const uint2 *)src); rw[0] = v.x; rw[1] = v.y; }
                else { const uint4 v = __ldg((const uint4 *)src); rw[0] = v.x; rw[1] = v.y; rw[2] = v.z; rw[3] = v.w; }
            } else {
#pragma unroll
                for (int i = 0; i < BPS; ++i) rw[i] = 0u;
                const int ns = full ? 4 : a.N - n0;
                for (int i = 0; i < ns * BPS; ++i)
                    rw[i >> 2] |= (uint32_t)a.raw[(size_t)n0 * BPS + i] << (8 * (i & 3));
            }
            const int ns = full ? 4 : a.N - n0;
#pragma unroll
            for (int sm = 0; sm < 4; ++sm) {
                if (sm < ns) {
                    const uint32_t b = sample_bytes<BPS>(rw, sm);
                    const int ph = (a.ph0 + n0 + sm) & 3;
#pragma unroll
                    for (int k = 0; k < NRF; ++k)
                        wq[k] |= unpack1<FMT>(b, k, ph, a, lutc, lut8) << (8 * sm);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < NRF; ++k) xs[k][qd] = wq[k];
    }
    __syncthreads();

    const int n0 = t0 + 4 * threadIdx.x;           // this thread's 4 outputs
    if (n0 < a.N) {
        const int ns = n0 + 4 <= a.N ? 4 : a.N - n0;
        uint32_t yw[NRF];
#pragma unroll
        for (int k = 0; k < NRF; ++k) {
            const uint32_t w2 = xs[k][threadIdx.x + 2];   // samples n0 .. n0+3
            uint32_t y = w2;
            if ((a.lpf_mask >> k) & 1) {
                const uint32_t w0 = xs[k][threadIdx.x], w1 = xs[k][threadIdx.x + 1];
                int xi[12], xq[12];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    xi[j] = nib(w0, 8 * j); xq[j] = nib(w0, 8 * j + 4);
                    xi[4 + j] = nib(w1, 8 * j); xq[4 + j] = nib(w1, 8 * j + 4);
                    xi[8 + j] = nib(w2, 8 * j); xq[8 + j] = nib(w2, 8 * j + 4);
                }
                const int *h = a.h[k];
                y = 0u;
#pragma unroll
                for (int j = 0; j < 4; ++j) {       // output n0 + j: inputs n0+j-8 .. n0+j
                    int ai = h[4] * xi[j + 4], aq = h[4] * xq[j + 4];
#pragma unroll
                    for (int m = 0; m < 4; ++m) {
                        ai += h[m] * (xi[j + m] + xi[j + 8 - m]);
                        aq += h[m] * (xq[j + m] + xq[j + 8 - m]);
                    }
                    const int I = min(7, max(-7, (ai + (1 << 12)) >> 13));
                    const int Q = min(7, max(-7, (aq + (1 << 12)) >> 13));
                    y |= (uint32_t)pack8(I, Q) << (8 * j);
                }
            }
            yw[k] = y;
            uint8_t *dst = a.out[k] + n0;
            if (ns == 4 && a.vec) *(uint32_t *)dst = y;
            else for (int j = 0; j < ns; ++j) dst[j] = (uint8_t)(y >> (8 * j));
        }
        for (int m = 0; m < a.narch; ++m) {
            int I[4] = {0, 0, 0, 0}, Q[4] = {0, 0, 0, 0};
#pragma unroll
            for (int k = 0; k < NRF; ++k) {
                if (!((a.amask[m] >> k) & 1)) continue;
                const int wr = a.w[m][k].x, wi = a.w[m][k].y;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int xi = nib(yw[k], 8 * j), xq = nib(yw[k], 8 * j + 4);
                    I[j] += xi * wr - xq * wi;
                    Q[j] += xi * wi + xq * wr;
                }
            }
            uint32_t o = 0u;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int ii = (I[j] + (I[j] >= 0 ? 128 : -128)) / 256;
                const int qq = (Q[j] + (Q[j] >= 0 ? 128 : -128)) / 256;
                o |= (uint32_t)pack8(min(7, max(-8, ii)), min(7, max(-8, qq))) << (8 * j);
            }
            uint8_t *dst = a.aout[m] + n0;
            if (ns == 4 && a.vec) *(uint32_t *)dst = o;
            else for (int j = 0; j < ns; ++j) dst[j] = (uint8_t)(o >> (8 * j));
        }
    }
    // the tile holding sample N-1 keeps the block's last 8 unfiltered samples
    if (t0 <= a.N - 1 && a.N - 1 < t0 + kTile && threadIdx.x < 8 * NRF) {
        const int k = threadIdx.x / 8, j = threadIdx.x % 8;
        const int p = a.N - t0 + j;                 // buffer position of sample N-8+j
        a.hist_out[k * 8 + j] = (uint8_t)(xs[k][p >> 2] >> (8 * (p & 3)));
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

static int launch_ingest(IngestArgs &a, int fmt, cudaStream_t st)
{
    if (a.N <= 0) return SDRG_OK;
    const int grid = (a.N + kTile - 1) / kTile;
    switch (fmt) {
    case F_CPX8: ingest_kernel<F_CPX8><<<grid, kIngThreads, 0, st>>>(a); break;
    case F_INT8: ingest_kernel<F_INT8><<<grid, kIngThreads, 0, st>>>(a); break;
    case F_INT8X2: ingest_kernel<F_INT8X2><<<grid, kIngThreads, 0, st>>>(a); break;
    case F_RAW8: ingest_kernel<F_RAW8><<<grid, kIngThreads, 0, st>>>(a); break;
    case F_RAW16: ingest_kernel<F_RAW16><<<grid, kIngThreads, 0, st>>>(a); break;
    case F_RAW16I: ingest_kernel<F_RAW16I><<<grid, kIngThreads, 0, st>>>(a); break;
    case F_RAW32: ingest_kernel<F_RAW32><<<grid, kIngThreads, 0, st>>>(a); break;
    case F_CS8: ingest_kernel<F_CS8><<<grid, kIngThreads, 0, st>>>(a); break;
    case F_CS16: ingest_kernel<F_CS16><<<grid, kIngThreads, 0, st>>>(a); break;
    default: return set_error(SDRG_ERR_ARG, "ingest: bad format %d", fmt);
    }
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
    uint8_t *hist_dev = nullptr;    // [2][8][8] double-buffered history (packed samples)
    int parity = 0;
};

// sdr_lpf_t of the drop-in calls (opaque to callers, as in the reference)
struct sdr_lpf_tag {
    int h[9];
    uint8_t hist[8];   // last 8 unfiltered (packed) samples of the previous call
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
              cudaMalloc(&g->hist_dev, 2 * kMaxRf * 8) == cudaSuccess &&
              cudaMemcpyAsync(g->lut8_dev, lut8.data(), lut8.size(), cudaMemcpyHostToDevice, st) ==
                  cudaSuccess &&
              cudaMemcpyAsync(g->lutc_dev, lutc.data(), lutc.size(), cudaMemcpyHostToDevice, st) ==
                  cudaSuccess &&
              cudaMemsetAsync(g->hist_dev, 0, 2 * kMaxRf * 8, st) == cudaSuccess &&
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
    a.N = g->cfg.N;
    a.ph0 = (int)((ix * (int64_t)g->cfg.N) & 3);    // src/sdr_rcv.c:846
    a.rtoc_mask = g->rtoc_mask;
    a.lpf_mask = g->lpf_mask;
    a.lut8 = g->lut8_dev;
    a.lutc = g->lutc_dev;
    a.hist_in = g->hist_dev + g->parity * kMaxRf * 8;
    a.hist_out = g->hist_dev + (g->parity ^ 1) * kMaxRf * 8;
    // vector loads / stores when the raw block is 16-byte and every output
    // 4-byte aligned (else the same kernel moves bytes)
    bool vec = ((uintptr_t)raw_dev & 15) == 0;
    for (int k = 0; k < g->nrfch; ++k) {
        if (!buf_dev[k]) return set_error(SDRG_ERR_ARG, "sdrg_ingest_run: no buffer %d", k);
        a.out[k] = buf_dev[k] + base;
        vec = vec && ((uintptr_t)a.out[k] & 3) == 0;
        memcpy(a.h[k], g->h[k], sizeof(a.h[k]));
    }
    a.narch = 0;
    for (int m = 0; m < g->cfg.narch; ++m) {
        if (!g->cfg.arch_on[m]) continue;   // sdr_arch_combine returns for scale <= 0
        uint8_t *o = buf_dev[g->nrfch + m];
        if (!o) return set_error(SDRG_ERR_ARG, "sdrg_ingest_run: no buffer %d", g->nrfch + m);
        a.aout[a.narch] = o + base;
        vec = vec && ((uintptr_t)a.aout[a.narch] & 3) == 0;
        a.amask[a.narch] = 0;
        for (int k = 0; k < g->nrfch; ++k) {
            a.w[a.narch][k] = make_short2(g->cfg.w[m][k][0], g->cfg.w[m][k][1]);
            // zero weights add nothing to the sums: skip those channels
            if (g->cfg.w[m][k][0] || g->cfg.w[m][k][1]) a.amask[a.narch] |= 1 << k;
        }
        a.narch++;
    }
    a.vec = vec;
    if ((e = launch_ingest(a, g->cfg.fmt, (cudaStream_t)stream))) return e;
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
    ThreadCtx &c = tctx();
    c.host[0].pinned = true;
    const size_t nb = ((size_t)N + 255) / 256 * 256;
    if (ensure_device(&dev) || thread_stream(&st) || c.host[0].reserve(2 * nb) ||
        c.dev[0].reserve(2 * nb + 2 * kMaxRf * 8))
        return;   // error recorded; data left unfiltered
    uint8_t *h_in = (uint8_t *)c.host[0].ptr, *h_out = h_in + nb;
    uint8_t *d_in = (uint8_t *)c.dev[0].ptr, *d_out = d_in + nb;
    uint8_t *d_hist = d_in + 2 * nb;
    memcpy(h_in, data, (size_t)N);
    IngestArgs a = {};
    a.raw = d_in;
    a.N = N;
    a.lpf_mask = 1;
    a.vec = 1;           // scratch slots are 256-byte aligned
    a.hist_in = d_hist;
    a.hist_out = d_hist + kMaxRf * 8;
    a.out[0] = d_out;
    memcpy(a.h[0], lpf->h, sizeof(a.h[0]));
    if (cudaMemcpyAsync(d_in, h_in, (size_t)N, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(d_hist, lpf->hist, sizeof(lpf->hist), cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        launch_ingest(a, F_CPX8, st) ||
        cudaMemcpyAsync(h_out, d_out, (size_t)N, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cuda_error(cudaGetLastError(), "sdr_lpf_apply");
        return;
    }
    // next history: the last 8 of (history, this call's unfiltered input)
    uint8_t nh[8];
    for (int j = 0; j < 8; ++j) {
        const int n = N - 8 + j;
        nh[j] = n < 0 ? lpf->hist[8 + n] : h_in[n];
    }
    memcpy(lpf->hist, nh, sizeof(nh));
    memcpy(data, h_out, (size_t)N);
}

} // extern "C"
