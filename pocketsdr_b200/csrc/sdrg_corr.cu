// sdrg_corr.cu - standard multi-tap correlators (reference: src/sdr_func.c:
// 851-1072). Bit-exact with the reference's AVX2 build:
//  * tap i at p = coff + pos[i]: shift j = floor(p), code bank k =
//    (int)((p - j) * 10), j wrapped once into [0, N) (host, in double);
//  * corr1 = IQ[0:j] . code_k[N-j:N], corr2 = IQ[j:N] . code_k[0:N-j];
//  * each dot: the first 16*floor(len/16) terms are int8 "sign products"
//    (x, -x or 0 by the sign of the code, negating -128 gives -128, as
//    _mm256_sign_epi8) summed in int32 and converted to float once; the
//    remaining len mod 16 exact integer products are added one at a time in
//    float; then the sum is scaled by CSCALE;
//  * polarity: dot = sum_{i<3} fma(c1.re, c2.re, c1.im*c2.im) (the
//    contraction the reference's gcc -mfma build emits), sign = dot < 0 ? -1:1;
//  * corr = (c1 + sign*c2) / N, C = {c1[0], c2[0]}.
#include <cmath>
#include <cstring>
#include <vector>

#include "sdrg_internal.h"

namespace sdrg {

__device__ __forceinline__ int sgn_mul8(int x, int c)
{
    return c > 0 ? x : (c < 0 ? (x == -128 ? -128 : -x) : 0);
}
__device__ __forceinline__ int neg8(int c) { return c == -128 ? -128 : -c; }

// one block per (tap, half); blockDim.x = 256
template <int CPX>
__global__ void __launch_bounds__(256) corr_half_kernel(
    const char2 *__restrict__ IQ, const char2 *__restrict__ code, int N,
    const int2 *__restrict__ jk, float cs, float2 *__restrict__ c12)
{
    const int tap = blockIdx.x, h = blockIdx.y;
    const int j = jk[tap].x, k = jk[tap].y;
    const int len = h == 0 ? j : N - j;
    const char2 *x = IQ + (h == 0 ? 0 : j);
    const char2 *y = code + (size_t)k * N + (h == 0 ? N - j : 0);
    const int main_len = (len / 16) * 16;
    int sr = 0, si = 0;
    for (int i = threadIdx.x; i < main_len; i += blockDim.x) {
        const char2 a = x[i], c = y[i];
        if (CPX) {
            sr += sgn_mul8(a.x, c.x) + sgn_mul8(a.y, c.y);
            si += sgn_mul8(a.y, c.x) + sgn_mul8(a.x, neg8(c.y));
        } else {
            sr += sgn_mul8(a.x, c.x);
            si += sgn_mul8(a.y, c.y);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    __shared__ int red[2][8];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { red[0][w] = sr; red[1][w] = si; }
    __syncthreads();
    if (threadIdx.x == 0) {
        int tr = 0, ti = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { tr += red[0][i]; ti += red[1][i]; }
        float fr = (float)tr, fi = (float)ti;
        for (int i = main_len; i < len; ++i) {
            const char2 a = x[i], c = y[i];
            if (CPX) {
                fr = __fadd_rn(fr, (float)(a.x * c.x + a.y * c.y));
                fi = __fadd_rn(fi, (float)(a.y * c.x - a.x * c.y));
            } else {
                fr = __fadd_rn(fr, (float)(a.x * c.x));
                fi = __fadd_rn(fi, (float)(a.y * c.y));
            }
        }
        c12[2 * tap + h] = make_float2(__fmul_rn(fr, cs), __fmul_rn(fi, cs));
    }
}

__global__ void corr_finish_kernel(const float2 *__restrict__ c12, int n, int N,
                                   float2 *__restrict__ corr, float2 *__restrict__ C)
{
    __shared__ float sign;
    if (threadIdx.x == 0) {
        float dot = 0.0f;
        for (int i = 0; i < 3 && i < n; ++i) {
            const float2 a = c12[2 * i], b = c12[2 * i + 1];
            dot = __fadd_rn(dot, __fmaf_rn(a.x, b.x, __fmul_rn(a.y, b.y)));
        }
        sign = dot < 0.0f ? -1.0f : 1.0f;
        if (C && n > 0) { C[0] = c12[0]; C[1] = c12[1]; }
    }
    __syncthreads();
    const float fN = (float)N;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float2 a = c12[2 * i], b = c12[2 * i + 1];
        corr[i] = make_float2(__fdiv_rn(__fadd_rn(a.x, __fmul_rn(sign, b.x)), fN),
                              __fdiv_rn(__fadd_rn(a.y, __fmul_rn(sign, b.y)), fN));
    }
}

// float code -> (int8) as one bank with I = Q (src/sdr_func.c:1066-1068)
__global__ void code_from_float_kernel(const float *__restrict__ in, int N, char2 *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) {
        const signed char v = (signed char)(int8_t)__float2int_rz(in[i]);
        out[i] = make_char2(v, v);
    }
}

// Shift/bank of each tap, evaluated on the host in double exactly as the
// reference (src/sdr_func.c:988-990). Returns false when a shift falls
// outside one wrap (the reference reads outside its arrays there).
static bool tap_params(int N, double coff, const double *pos, int n, int nbank, int2 *jk)
{
    for (int i = 0; i < n; ++i) {
        double p = coff + pos[i];
        int j = (int)floor(p), k = (int)((p - j) * SDR_N_CODES);
        if (j < 0) j += N; else if (j >= N) j -= N;
        if (j < 0 || j > N || k < 0 || k >= nbank) return false;
        jk[i] = make_int2(j, k);
    }
    return true;
}

// IQ_dev / code_dev already on the device; results to host corr / C.
static int corr_std_device(const char2 *IQ_dev, const char2 *code_dev, int N, int nbank,
                           double coff, const double *pos, int n, int cpx,
                           sdr_cpx_t *corr, sdr_cpx_t *C, cudaStream_t st)
{
    if (n <= 0) return SDRG_OK;
    if (n > SDR_MAX_CORR) return set_error(SDRG_ERR_ARG, "corr_std: n=%d > %d", n, SDR_MAX_CORR);
    ThreadCtx &c = tctx();
    int e;
    c.host[2].pinned = true;
    const size_t jkb = sizeof(int2) * n, outb = sizeof(float2) * (n + 2);
    if ((e = c.host[2].reserve(jkb + outb + 64)) || (e = c.dev[5].reserve(jkb + sizeof(float2) * 2 * n + outb + 64)))
        return e;
    int2 *jk_h = (int2 *)c.host[2].ptr;
    if (!tap_params(N, coff, pos, n, nbank, jk_h))
        return set_error(SDRG_ERR_ARG, "corr_std: a tap shift leaves [-N, 2N) or the code bank");
    int2 *jk_d = (int2 *)c.dev[5].ptr;
    float2 *c12 = (float2 *)(jk_d + n);
    float2 *out_d = c12 + 2 * n;     // corr[n], C[2]
    float2 *out_h = (float2 *)(jk_h + n);
    SDRG_CUDA(cudaMemcpyAsync(jk_d, jk_h, jkb, cudaMemcpyHostToDevice, st));
    if (cpx) corr_half_kernel<1><<<dim3(n, 2), 256, 0, st>>>(IQ_dev, code_dev, N, jk_d, kCScale, c12);
    else     corr_half_kernel<0><<<dim3(n, 2), 256, 0, st>>>(IQ_dev, code_dev, N, jk_d, kCScale, c12);
    SDRG_CUDA(cudaGetLastError());
    corr_finish_kernel<<<1, 128, 0, st>>>(c12, n, N, out_d, out_d + n);
    SDRG_CUDA(cudaGetLastError());
    SDRG_CUDA(cudaMemcpyAsync(out_h, out_d, outb, cudaMemcpyDeviceToHost, st));
    SDRG_CUDA(cudaStreamSynchronize(st));
    memcpy(corr, out_h, sizeof(float2) * n);
    if (C) memcpy(C, out_h + n, sizeof(float2) * 2);
    return SDRG_OK;
}

static void corr_std_host(const sdr_cpx16_t *IQ, const sdr_cpx16_t *code, int N, double coff,
                          const double *pos, int n, sdr_cpx_t *corr, sdr_cpx_t *C, int cpx)
{
    if (N <= 0 || n <= 0) return;
    cudaStream_t st;
    int e;
    ThreadCtx &c = tctx();
    const size_t iqb = (size_t)N * 2, cb = (size_t)N * 2 * SDR_N_CODES;
    c.host[0].pinned = true;
    if ((e = ensure_device(nullptr)) || (e = thread_stream(&st)) ||
        (e = c.host[0].reserve(iqb + cb + 16)) || (e = c.dev[0].reserve(iqb + cb + 16)))
        goto fail;
    {
        uint8_t *h = (uint8_t *)c.host[0].ptr;
        memcpy(h, IQ, iqb);
        memcpy(h + iqb, code, cb);
        uint8_t *d = (uint8_t *)c.dev[0].ptr;
        if (cudaMemcpyAsync(d, h, iqb + cb, cudaMemcpyHostToDevice, st) != cudaSuccess) {
            cuda_error(cudaGetLastError(), "corr_std H2D");
            goto fail;
        }
        if (corr_std_device((const char2 *)d, (const char2 *)(d + iqb), N, SDR_N_CODES, coff,
                            pos, n, cpx, corr, C, st))
            goto fail;
    }
    return;
fail:
    memset(corr, 0, sizeof(sdr_cpx_t) * n);
    if (C) memset(C, 0, sizeof(sdr_cpx_t) * 2);
}

} // namespace sdrg

using namespace sdrg;

extern "C" {

void sdr_corr_std(const sdr_cpx16_t *IQ, const sdr_cpx16_t *code, int N, double coff,
                  const double *pos, int n, sdr_cpx_t *corr, sdr_cpx_t *C)
{
    corr_std_host(IQ, code, N, coff, pos, n, corr, C, 0);
}

void sdr_corr_std_cpx_code(const sdr_cpx16_t *IQ, const sdr_cpx16_t *code, int N, double coff,
                           const double *pos, int n, sdr_cpx_t *corr, sdr_cpx_t *C)
{
    corr_std_host(IQ, code, N, coff, pos, n, corr, C, 1);
}

void sdr_corr_std_cpx(const sdr_cpx_t *buff, int len_buff, int ix, int N, double fs,
                      double fc, double phi, const float *code, const double *pos, int n,
                      sdr_cpx_t *corr)
{
    if (N <= 0 || n <= 0) return;
    cudaStream_t st;
    int e;
    ThreadCtx &c = tctx();
    c.host[0].pinned = true;
    if ((e = ensure_device(nullptr)) || (e = thread_stream(&st)) ||
        (e = c.dev[0].reserve((size_t)N * 4 + (size_t)N * 4 + 64)) ||
        (e = c.host[0].reserve((size_t)N * 4 + 16))) {
        memset(corr, 0, sizeof(sdr_cpx_t) * n);
        return;
    }
    char2 *iq_d = (char2 *)c.dev[0].ptr;
    char2 *code_d = iq_d + N;
    float *codef_d = (float *)(code_d + N + 8);
    if (mix_cpx_device(buff, len_buff, ix, N, fs, fc, phi, iq_d, st)) {
        memset(corr, 0, sizeof(sdr_cpx_t) * n);
        return;
    }
    memcpy(c.host[0].ptr, code, (size_t)N * 4);
    if (cudaMemcpyAsync(codef_d, c.host[0].ptr, (size_t)N * 4, cudaMemcpyHostToDevice, st) !=
        cudaSuccess) {
        cuda_error(cudaGetLastError(), "corr_std_cpx H2D");
        memset(corr, 0, sizeof(sdr_cpx_t) * n);
        return;
    }
    code_from_float_kernel<<<(N + 255) / 256, 256, 0, st>>>(codef_d, N, code_d);
    sdr_cpx_t Cb[2];
    // the reference passes a single bank (src/sdr_func.c:1070); a tap whose
    // fractional shift selects another bank reads past it there and is
    // rejected here
    if (corr_std_device(iq_d, code_d, N, 1, 0.0, pos, n, 0, corr, Cb, st)) {
        memset(corr, 0, sizeof(sdr_cpx_t) * n);
    }
}

} // extern "C"
