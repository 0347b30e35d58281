// sdrg_psd.cu - power spectral density of IF data on the device.
//
// Reference: sdr_psd_cpx (src/sdr_func.c:1141-1182): Welch's method without
// overlap - M = len / N segments, each multiplied by a Hann window
// (hann_window, :1116-1125), forward FFT, |X|^2 summed over the segments in
// order, scaled as matplotlib.psd (1 / M / sum w^2 / fs, x2 for real
// sampling) and converted to dB; real (IQ = 1) data keeps the N/2 positive
// bins, complex data is rotated so the output runs from -fs/2. The receiver
// feeds it a window of a packed IF buffer (sdr_rcv_rfch_psd,
// src/sdr_rcv.c:395-412), which sdrg_psd_if reads directly.
//
// Kernels: psd_fwd_kernel (one CTA per (segment, r): windowed sub-transform
// F_r = FFT_M(w x)[R m + r] of the split L = N = R M), psd_pow_kernel (split
// combine to X[k], |X|^2 per segment at natural k), psd_sum_kernel (per bin,
// the sum over segments in the reference's order, scale, dB, rotation).
#include <cmath>
#include <cstring>
#include <vector>

#include "sdrg_internal.h"

namespace sdrg {

struct LoadSeg {
    const float2 *x;        // float IQ (mode 0) or null
    const uint8_t *buf;     // packed cpx8 circular buffer (mode 1)
    int len, ix0;           // buffer length, first sample of the segment
    const float *w;
    int R, r;
    __device__ __forceinline__ float2 operator()(int m) const
    {
        const int n = R * m + r;
        const float wn = __ldg(w + n);
        float2 v;
        if (x) {
            v = __ldg(x + (size_t)ix0 + n);
        } else {
            int p = ix0 + n;
            if (p >= len) p -= len;
            const uint8_t b = __ldg(buf + p);
            v = make_float2((float)((int8_t)(uint8_t)(b << 4) >> 4), (float)((int8_t)b >> 4));
        }
        return make_float2(__fmul_rn(v.x, wn), __fmul_rn(v.y, wn));
    }
};

struct PsdArgs {
    FftPlanK pl;
    const float2 *tw;
    int R, N;
    const float2 *x;
    const uint8_t *buf;
    int len, ix;
    const float *w;
    float2 *F;              // [n_seg][R][M]
};

__global__ void __launch_bounds__(512, 1) psd_fwd_kernel(PsdArgs a)
{
    extern __shared__ float2 smem[];
    float2 *sm = smem;
    float2 *tw = smem + a.pl.M;
    const int r = (int)(blockIdx.x % a.R);
    const int seg = (int)(blockIdx.x / a.R);
    load_twiddles(tw, a.tw, a.pl.twtot);
    __syncthreads();
    int ix0;
    if (a.x) {
        ix0 = seg * a.N;
    } else {
        const long long s0 = (long long)a.ix + (long long)seg * a.N;
        ix0 = (int)(s0 % a.len);
    }
    LoadSeg ld{a.x, a.buf, a.len, ix0, a.w, a.R, r};
    fft_forward(sm, tw, a.pl, ld);
    float2 *dst = a.F + ((size_t)seg * a.R + r) * a.pl.M;
    for (int i = threadIdx.x; i < a.pl.M; i += blockDim.x) dst[i] = sm[i];
}

template <int R>
__global__ void __launch_bounds__(256) psd_pow_kernel(const float2 *F, const float2 *split,
                                                      const int *kperm, int M, int n_seg,
                                                      float *pw)
{
    const size_t total = (size_t)n_seg * M;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t s = i / M;
        const int q = (int)(i - s * M);
        float2 g[R];
#pragma unroll
        for (int r = 0; r < R; ++r) g[r] = F[(s * R + r) * (size_t)M + q];
        split_combine_fwd<R>(g, R > 1 ? __ldg(split + q) : make_float2(1.0f, 0.0f));
        const int k = __ldg(kperm + q);
#pragma unroll
        for (int j = 0; j < R; ++j)
            pw[s * (size_t)R * M + (size_t)j * M + k] =
                __fadd_rn(__fmul_rn(g[j].x, g[j].x), __fmul_rn(g[j].y, g[j].y));
    }
}

// out[i] for i < n_out: bin k = i (real) or (i + N/2) mod N (complex)
__global__ void psd_sum_kernel(const float *pw, int n_seg, int N, int IQ, float scale, float *out)
{
    const int n_out = IQ == 1 ? N / 2 : N;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_out; i += gridDim.x * blockDim.x) {
        const int k = IQ == 1 ? i : (i < N / 2 ? N / 2 + i : i - N / 2);
        float p = 0.0f;
        for (int s = 0; s < n_seg; ++s) p = __fadd_rn(p, pw[(size_t)s * N + k]);
        out[i] = 10.0f * log10f(__fmul_rn(p, scale));
    }
}

static int psd_device(const float2 *x, const uint8_t *buf, int len, int ix, int n, int N,
                      double fs, int IQ, float *out, cudaStream_t st)
{
    if (N <= 1 || n < 0 || (IQ != 1 && IQ != 2) || !out || !(fs > 0.0) || (!x && !buf) ||
        (buf && (len <= 0 || ix < 0 || ix >= len || n > len)))
        return set_error(SDRG_ERR_ARG, "psd: bad arguments (N=%d n=%d IQ=%d)", N, n, IQ);
    const FftPlan *pl = get_plan(N);
    if (!pl) return tctx().error ? tctx().error : SDRG_ERR_ARG;
    // hann_window (src/sdr_func.c:1116-1125): taps rounded to float, the
    // squares summed in float in index order
    std::vector<float> w(N);
    float wss = 0.0f;
    for (int i = 0; i < N; i++) {
        w[i] = (float)(0.5 + 0.5 * cos(2.0 * 3.1415926535897932 * (i - 0.5 * (N - 1)) / (N - 1)));
        wss += w[i] * w[i];
    }
    const int n_seg = n / N;
    const float scale = (float)(1.0 / n_seg / wss / fs * (IQ == 1 ? 2.0 : 1.0));
    static bool attr_set = false;
    if (!attr_set) {
        SDRG_CUDA(cudaFuncSetAttribute(psd_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)g_smem_limit()));
        attr_set = true;
    }
    float *w_dev = nullptr, *pw = nullptr;
    float2 *F = nullptr;
    const size_t segs = n_seg > 0 ? (size_t)n_seg : 1;
    cudaError_t ce = stream_alloc((void **)&w_dev, (size_t)N * sizeof(float), st);
    if (ce == cudaSuccess) ce = stream_alloc((void **)&F, segs * N * sizeof(float2), st);
    if (ce == cudaSuccess) ce = stream_alloc((void **)&pw, segs * N * sizeof(float), st);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(w_dev, w.data(), (size_t)N * sizeof(float), cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess && n_seg > 0) {
        PsdArgs a = {};
        a.pl = pl->k; a.tw = pl->tw_dev; a.R = pl->R; a.N = N; a.x = x; a.buf = buf;
        a.len = len; a.ix = ix; a.w = w_dev; a.F = F;
        psd_fwd_kernel<<<(unsigned)(n_seg * pl->R), pl->threads, pl->smem, st>>>(a);
        const int M = pl->M;
        size_t units = (size_t)n_seg * M;
        const int gb = (int)((units + 255) / 256 > 8192 ? 8192 : (units + 255) / 256);
        switch (pl->R) {
#define SDRG_PSD_POW(RR) \
        case RR: psd_pow_kernel<RR><<<gb, 256, 0, st>>>(F, pl->split_dev, pl->kperm_dev, M, n_seg, pw); break;
        SDRG_PSD_POW(1) SDRG_PSD_POW(2) SDRG_PSD_POW(3) SDRG_PSD_POW(4) SDRG_PSD_POW(5)
        SDRG_PSD_POW(6) SDRG_PSD_POW(8) SDRG_PSD_POW(10) SDRG_PSD_POW(12) SDRG_PSD_POW(15)
        SDRG_PSD_POW(16) SDRG_PSD_POW(20)
#undef SDRG_PSD_POW
        default: break;
        }
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) {
        const int n_out = IQ == 1 ? N / 2 : N;
        psd_sum_kernel<<<(n_out + 255) / 256, 256, 0, st>>>(pw, n_seg, N, IQ, scale, out);
        ce = cudaGetLastError();
    }
    if (w_dev) cudaFreeAsync(w_dev, st);
    if (F) cudaFreeAsync(F, st);
    if (pw) cudaFreeAsync(pw, st);
    if (ce != cudaSuccess) return cuda_error(ce, "psd");
    return SDRG_OK;
}

} // namespace sdrg

using namespace sdrg;

extern "C" {

int sdrg_psd(const sdr_cpx_t *buff_dev, int len_buff, int N, double fs, int IQ, float *psd_dev,
             void *stream)
{
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    if (!buff_dev) return set_error(SDRG_ERR_ARG, "sdrg_psd: null buffer");
    return psd_device((const float2 *)buff_dev, nullptr, 0, 0, len_buff, N, fs, IQ, psd_dev,
                      (cudaStream_t)stream);
}

int sdrg_psd_if(const uint8_t *if_dev, int len_if, int ix, int n, int N, double fs, int IQ,
                float *psd_dev, void *stream)
{
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    if (!if_dev) return set_error(SDRG_ERR_ARG, "sdrg_psd_if: null buffer");
    return psd_device(nullptr, if_dev, len_if, ix, n, N, fs, IQ, psd_dev, (cudaStream_t)stream);
}

void sdr_psd_cpx(const sdr_cpx_t *buff, int len_buff, int N, double fs, int IQ, float *psd)
{
    if (!psd || N <= 1) return;
    const int n_out = IQ == 1 ? N / 2 : N;
    Device *dev;
    cudaStream_t st;
    ThreadCtx &c = tctx();
    c.host[0].pinned = true;
    const size_t nin = (size_t)(len_buff > 0 ? len_buff : 0) * sizeof(float2);
    const size_t nout = (size_t)n_out * sizeof(float);
    if (!buff || len_buff < 0 || (IQ != 1 && IQ != 2)) {
        set_error(SDRG_ERR_ARG, "sdr_psd_cpx: bad arguments");
        memset(psd, 0, nout);
        return;
    }
    if (ensure_device(&dev) || thread_stream(&st) ||
        c.host[0].reserve(nin > nout ? nin : nout) || c.dev[0].reserve(nin + nout + 256)) {
        memset(psd, 0, nout);
        return;
    }
    float2 *x_d = (float2 *)c.dev[0].ptr;
    float *o_d = (float *)((uint8_t *)c.dev[0].ptr + (nin + 255) / 256 * 256);
    memcpy(c.host[0].ptr, buff, nin);
    if (cudaMemcpyAsync(x_d, c.host[0].ptr, nin, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        psd_device(x_d, nullptr, 0, 0, len_buff, N, fs, IQ, o_d, st) ||
        cudaMemcpyAsync(c.host[0].ptr, o_d, nout, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        if (!tctx().error) cuda_error(cudaGetLastError(), "sdr_psd_cpx");
        memset(psd, 0, nout);
        return;
    }
    memcpy(psd, c.host[0].ptr, nout);
}

} // extern "C"
