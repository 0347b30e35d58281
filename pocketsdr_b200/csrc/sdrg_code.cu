// sdrg_code.cu - spreading-code replicas on the device.
//
// Reference: src/sdr_code.c:2556-2568 (sdr_res_code: nearest-chip resampling
// into sdr_cpx16_t, zero padded), src/sdr_code.c:2589-2608 (sdr_gen_code_fft:
// the resampled, zero-padded replica, forward DFT, conjugate) and
// src/sdr_ch.c:265-272 (a tracking channel's SDR_N_CODES fractional-phase
// banks, bank k resampled with code offset -k / fs / SDR_N_CODES).
// The receiver builds these on the CPU, one PRN at a time (one FFT per PRN in
// acq_new, src/sdr_ch.c:192-201). Here every PRN of a signal group is
// resampled and transformed in one launch sequence, and the code DFTs can be
// written straight into an acquisition plan's permuted layout.
//
// Chip index of replica sample n (both functions):
//   j = (int)((coff * fs + n) * dx) % len_code,   dx = len_code / T / fs,
// every double operation rounded once, in the reference's order. The index
// arithmetic is therefore bit-identical; the DFT is this library's FP32
// mixed-radix FFT (sdrg_fft.cuh), split L = R * M like the search transforms.
#include <cmath>
#include <cstdio>
#include <cstring>

#include "sdrg_internal.h"

namespace sdrg {

__device__ __forceinline__ int chip_at(double cf, double dx, int n, int len)
{
    return (int)__dmul_rn(__dadd_rn(cf, (double)n), dx) % len;
}

// ---- resampled code banks (sdr_res_code) --------------------------------------
constexpr int kMaxBanks = 32;

struct ResArgs {
    const int8_t *ci, *cq;     // [n_code][len] chips (cq may be null)
    int len, n_code, n_bank;
    int N, L;                  // replica samples, N + Nz
    int vec;                   // samples stored per thread (8 or 1)
    double dx;
    double cf[kMaxBanks];      // coff_b * fs per bank
    char2 *out;                // [n_code][n_bank][L]
};

// 8 output samples (16 bytes) per thread when rows are multiples of 8 samples
// and the output is 16-byte aligned (a.vec = 8), else one; the code rows are
// read through the read-only cache (a code is a few KB).
__global__ void __launch_bounds__(256) res_code_kernel(ResArgs a)
{
    const int per = a.L;                          // samples per bank row
    const int vec = a.vec;
    const int upr = per / vec;                    // units per row
    const size_t units = (size_t)a.n_code * a.n_bank * upr;
    for (size_t u = blockIdx.x * (size_t)blockDim.x + threadIdx.x; u < units;
         u += (size_t)gridDim.x * blockDim.x) {
        const size_t row = u / (size_t)upr;
        const int n0 = (int)(u - row * (size_t)upr) * vec;
        const int b = (int)(row % a.n_bank);
        const size_t p = row / a.n_bank;
        const int8_t *ci = a.ci + p * a.len;
        const int8_t *cq = a.cq ? a.cq + p * a.len : nullptr;
        const double cf = a.cf[b];
        uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int n = n0 + k;
            if (k < vec && n < a.N) {
                const int j = chip_at(cf, a.dx, n, a.len);
                const uint32_t I = (uint8_t)__ldg(ci + j);
                const uint32_t Q = cq ? (uint32_t)(uint8_t)__ldg(cq + j) : I;
                w[k >> 1] |= (I | (Q << 8)) << (16 * (k & 1));
            }
        }
        char2 *dst = a.out + row * (size_t)per + n0;
        if (vec == 8) {
            *(int4 *)dst = make_int4((int)w[0], (int)w[1], (int)w[2], (int)w[3]);
        } else {
            dst[0] = make_char2((signed char)(w[0] & 0xff), (signed char)((w[0] >> 8) & 0xff));
        }
    }
}

// ---- code DFTs (sdr_gen_code_fft) ---------------------------------------------
// Element m of sub-sequence r: replica sample n = R m + r, zero past N.
struct LoadChips {
    const int8_t *ci, *cq;
    int len, N, R, r;
    double cf, dx;
    __device__ __forceinline__ float2 operator()(int m) const
    {
        const int n = R * m + r;
        if (n >= N) return make_float2(0.0f, 0.0f);
        const int j = chip_at(cf, dx, n, len);
        return make_float2((float)__ldg(ci + j), cq ? (float)__ldg(cq + j) : 0.0f);
    }
};

struct CodeFwdArgs {
    FftPlanK pl;
    const float2 *tw;
    int R;
    const int8_t *ci, *cq;
    int len, N;
    double cf, dx;
    float2 *F;                 // [n_code][R][M] sub-spectra (digit-reversed)
};

// one CTA per (code, r): F_r = FFT_M(x[R m + r])
__global__ void __launch_bounds__(512, 1) code_fwd_kernel(CodeFwdArgs a)
{
    extern __shared__ float2 smem[];
    float2 *sm = smem;
    float2 *tw = smem + a.pl.M;
    const int r = (int)(blockIdx.x % a.R);
    const size_t p = blockIdx.x / a.R;
    load_twiddles(tw, a.tw, a.pl.twtot);
    __syncthreads();
    LoadChips ld{a.ci + p * a.len, a.cq ? a.cq + p * a.len : nullptr, a.len, a.N, a.R, r,
                 a.cf, a.dx};
    fft_forward(sm, tw, a.pl, ld);
    float2 *dst = a.F + (p * a.R + r) * (size_t)a.pl.M;
    for (int i = threadIdx.x; i < a.pl.M; i += blockDim.x) dst[i] = sm[i];
}

// X[k + j M] = sum_r e^{-2 pi i r (k + j M) / L} F_r[k] at k = k(q), then the
// conjugate, stored at natural index k(q) + j M (natural) or at [code][j][q]
// (the acquisition plan's permuted layout).
template <int R>
__global__ void __launch_bounds__(256) code_combine_kernel(const float2 *F, const float2 *split,
                                                           const int *kperm, int M, int n_code,
                                                           int natural, float2 *out)
{
    const size_t total = (size_t)n_code * M;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t p = i / M;
        const int q = (int)(i - p * M);
        float2 g[R];
#pragma unroll
        for (int r = 0; r < R; ++r) g[r] = F[(p * R + r) * (size_t)M + q];
        split_combine_fwd<R>(g, R > 1 ? __ldg(split + q) : make_float2(1.0f, 0.0f));
        const int k = natural ? __ldg(kperm + q) : q;
#pragma unroll
        for (int j = 0; j < R; ++j) out[(p * R + j) * (size_t)M + k] = cconj(g[j]);
    }
}

static int grid_for(size_t units, int threads)
{
    size_t b = (units + threads - 1) / threads;
    return (int)(b > 8192 ? 8192 : (b < 1 ? 1 : b));
}

// Validates the chip-index range of samples 0..N-1: the reference reads
// code_I[j] with j from (int)((coff*fs + n)*dx) % len_code, which is negative
// (before the array) when (coff*fs)*dx <= -1 and overflows int past 2^31.
static int check_index_range(double cf, double dx, int N, const char *what)
{
    const double lo = cf * dx, hi = (cf + (double)N) * dx;
    if (!(lo > -1.0) || !(hi < 2147483647.0))
        return set_error(SDRG_ERR_ARG, "%s: code offset out of range (chip index %.6g .. %.6g)",
                         what, lo, hi);
    return SDRG_OK;
}

int res_code_device(const int8_t *ci, const int8_t *cq, int len_code, int n_code, double T,
                    double coff, double fs, int N, int Nz, int n_bank, char2 *out,
                    cudaStream_t st)
{
    if (!ci || !out || len_code <= 0 || n_code <= 0 || N <= 0 || Nz < 0 || !(T > 0) ||
        !(fs > 0) || n_bank <= 0 || n_bank > kMaxBanks || (long)N + Nz > (1L << 30))
        return set_error(SDRG_ERR_ARG, "res_code: bad arguments (len_code=%d n_code=%d N=%d "
                         "Nz=%d n_bank=%d, at most %d banks)", len_code, n_code, N, Nz, n_bank,
                         kMaxBanks);
    ResArgs a = {};
    a.ci = ci; a.cq = cq; a.len = len_code; a.n_code = n_code; a.n_bank = n_bank;
    a.N = N; a.L = N + Nz; a.out = out;
    a.dx = (double)len_code / T / fs;
    int e;
    for (int b = 0; b < n_bank; ++b) {
        // bank b: offset coff - b / fs / n_bank (b = 0: coff itself; with
        // coff = 0 and n_bank = SDR_N_CODES the reference's -k / fs / 10)
        const double cb = coff - (double)b / fs / (double)n_bank;
        a.cf[b] = cb * fs;
        if ((e = check_index_range(a.cf[b], a.dx, N, "res_code"))) return e;
    }
    a.vec = (a.L % 8 == 0 && ((uintptr_t)out & 15) == 0) ? 8 : 1;
    const size_t units = (size_t)n_code * n_bank * (size_t)(a.L / a.vec);
    res_code_kernel<<<grid_for(units, 256), 256, 0, st>>>(a);
    SDRG_CUDA(cudaGetLastError());
    return SDRG_OK;
}

int code_fft_device(const int8_t *ci, const int8_t *cq, int len_code, int n_code, double T,
                    double coff, double fs, int N, int L, int natural, float2 *out,
                    cudaStream_t st, const FftPlan *pl_in)
{
    if (!ci || !out || len_code <= 0 || n_code <= 0 || N <= 0 || L < N || !(T > 0) ||
        !(fs > 0))
        return set_error(SDRG_ERR_ARG, "gen_code_fft: bad arguments (len_code=%d n_code=%d "
                         "N=%d L=%d)", len_code, n_code, N, L);
    const FftPlan *pl = pl_in ? pl_in : get_plan(L);
    if (!pl) return tctx().error ? tctx().error : SDRG_ERR_ARG;
    if (pl->L != L) return set_error(SDRG_ERR_ARG, "gen_code_fft: plan length %d != L=%d", pl->L, L);
    const double dx = (double)len_code / T / fs;
    const double cf = coff * fs;
    int e;
    if ((e = check_index_range(cf, dx, N, "gen_code_fft"))) return e;

    static bool attr_set = false;
    if (!attr_set) {
        SDRG_CUDA(cudaFuncSetAttribute(code_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)g_smem_limit()));
        attr_set = true;
    }
    // sub-spectra scratch, stream-ordered so concurrent calls on other
    // streams never share it
    float2 *F = nullptr;
    SDRG_CUDA(stream_alloc((void **)&F, (size_t)n_code * L * sizeof(float2), st));
    CodeFwdArgs fa = {};
    fa.pl = pl->k; fa.tw = pl->tw_dev; fa.R = pl->R; fa.ci = ci; fa.cq = cq;
    fa.len = len_code; fa.N = N; fa.cf = cf; fa.dx = dx; fa.F = F;
    code_fwd_kernel<<<(unsigned)(n_code * pl->R), pl->threads, pl->smem, st>>>(fa);
    cudaError_t le = cudaGetLastError();
    if (le == cudaSuccess) {
        const int M = pl->M;
        const int gb = grid_for((size_t)n_code * M, 256);
        switch (pl->R) {
#define SDRG_COMBINE(RR) \
        case RR: code_combine_kernel<RR><<<gb, 256, 0, st>>>(F, pl->split_dev, pl->kperm_dev, M, \
                                                             n_code, natural, out); break;
        SDRG_COMBINE(1) SDRG_COMBINE(2) SDRG_COMBINE(3) SDRG_COMBINE(4) SDRG_COMBINE(5)
        SDRG_COMBINE(6) SDRG_COMBINE(8) SDRG_COMBINE(10) SDRG_COMBINE(12) SDRG_COMBINE(15)
        SDRG_COMBINE(16) SDRG_COMBINE(20)
#undef SDRG_COMBINE
        default:
            cudaFreeAsync(F, st);
            return set_error(SDRG_ERR_ARG, "gen_code_fft: unsupported split %d", pl->R);
        }
        le = cudaGetLastError();
    }
    cudaError_t fe = cudaFreeAsync(F, st);
    if (le != cudaSuccess) return cuda_error(le, "gen_code_fft launch");
    if (fe != cudaSuccess) return cuda_error(fe, "cudaFreeAsync");
    return SDRG_OK;
}

} // namespace sdrg

using namespace sdrg;

// Host-pointer body shared by the two drop-in calls: stages the chips on the
// thread's stream, runs `body` and copies `out_bytes` back.
template <class Body>
static int code_host_call(const int8_t *code_I, const int8_t *code_Q, int len_code,
                          size_t out_bytes, void *out_host, Body body)
{
    Device *dev;
    cudaStream_t st;
    int e;
    if ((e = ensure_device(&dev)) || (e = thread_stream(&st))) return e;
    ThreadCtx &c = tctx();
    const size_t cb = ((size_t)len_code * 2 + 255) / 256 * 256;
    c.host[0].pinned = true;
    if ((e = c.dev[0].reserve(cb)) || (e = c.dev[1].reserve(out_bytes)) ||
        (e = c.host[0].reserve(cb > out_bytes ? cb : out_bytes)))
        return e;
    int8_t *h = (int8_t *)c.host[0].ptr;
    memcpy(h, code_I, (size_t)len_code);
    if (code_Q) memcpy(h + len_code, code_Q, (size_t)len_code);
    int8_t *ci = (int8_t *)c.dev[0].ptr;
    SDRG_CUDA(cudaMemcpyAsync(ci, h, (size_t)len_code * (code_Q ? 2 : 1), cudaMemcpyHostToDevice, st));
    if ((e = body(ci, code_Q ? ci + len_code : nullptr, c.dev[1].ptr, st))) {
        cudaStreamSynchronize(st);
        return e;
    }
    SDRG_CUDA(cudaMemcpyAsync(c.host[0].ptr, c.dev[1].ptr, out_bytes, cudaMemcpyDeviceToHost, st));
    SDRG_CUDA(cudaStreamSynchronize(st));
    memcpy(out_host, c.host[0].ptr, out_bytes);
    return SDRG_OK;
}

extern "C" {

void sdr_res_code(const int8_t *code_I, const int8_t *code_Q, int len_code, double T,
                  double coff, double fs, int N, int Nz, sdr_cpx16_t *code_res)
{
    if (!code_res || N + Nz <= 0) return;
    const size_t ob = (size_t)(N + Nz) * sizeof(sdr_cpx16_t);
    if (N == 0 && Nz > 0) {            // the reference: all padding, zeros
        memset(code_res, 0, ob);
        return;
    }
    int e = SDRG_ERR_ARG;
    if (!code_I || len_code <= 0 || N <= 0 || Nz < 0) {
        set_error(SDRG_ERR_ARG, "sdr_res_code: bad arguments (len_code=%d N=%d Nz=%d)",
                  len_code, N, Nz);
    } else {
        e = code_host_call(code_I, code_Q, len_code, ob, code_res,
            [&](const int8_t *ci, const int8_t *cq, void *out, cudaStream_t st) {
                return res_code_device(ci, cq, len_code, 1, T, coff, fs, N, Nz, 1, (char2 *)out,
                                       st);
            });
    }
    if (e) memset(code_res, 0, ob);
}

void sdr_gen_code_fft(const int8_t *code_I, const int8_t *code_Q, int len_code, double T,
                      double coff, double fs, int N, int Nz, sdr_cpx_t *code_fft)
{
    if (!code_fft || N + Nz <= 0) return;
    const size_t ob = (size_t)(N + Nz) * sizeof(sdr_cpx_t);
    if (N == 0 && Nz > 0) {            // the DFT of all-zero padding
        memset(code_fft, 0, ob);
        return;
    }
    int e = SDRG_ERR_ARG;
    if (!code_I || len_code <= 0 || N <= 0 || Nz < 0) {
        set_error(SDRG_ERR_ARG, "sdr_gen_code_fft: bad arguments (len_code=%d N=%d Nz=%d)",
                  len_code, N, Nz);
    } else {
        e = code_host_call(code_I, code_Q, len_code, ob, code_fft,
            [&](const int8_t *ci, const int8_t *cq, void *out, cudaStream_t st) {
                return code_fft_device(ci, cq, len_code, 1, T, coff, fs, N, N + Nz, 1,
                                       (float2 *)out, st);
            });
    }
    if (e) memset(code_fft, 0, ob);
}

int sdrg_res_code(const int8_t *code_I_dev, const int8_t *code_Q_dev, int len_code, int n_code,
                  double T, double coff, double fs, int N, int Nz, int n_bank,
                  sdr_cpx16_t *code_res_dev, void *stream)
{
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    return res_code_device(code_I_dev, code_Q_dev, len_code, n_code, T, coff, fs, N, Nz, n_bank,
                           (char2 *)code_res_dev, (cudaStream_t)stream);
}

int sdrg_gen_code_fft(const int8_t *code_I_dev, const int8_t *code_Q_dev, int len_code,
                      int n_code, double T, double coff, double fs, int N, int Nz,
                      sdr_cpx_t *code_fft_dev, void *stream)
{
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    if (Nz < 0) return set_error(SDRG_ERR_ARG, "sdrg_gen_code_fft: Nz=%d", Nz);
    return code_fft_device(code_I_dev, code_Q_dev, len_code, n_code, T, coff, fs, N, N + Nz, 1,
                           (float2 *)code_fft_dev, (cudaStream_t)stream);
}

} // extern "C"
