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

// Shift and code bank of every tap, passed by value (at most SDR_MAX_CORR).
struct TapArgs {
    int n;
    int2 jk[SDR_MAX_CORR];
};

// Samples of one half-dot product summed by one block (256 threads x 4).
constexpr int kCorrChunk = 1024;

// Grid (tap, half, chunk), blockDim.x = 256: block (tap, h, ch) sums the
// sign products of samples [ch kCorrChunk, (ch + 1) kCorrChunk) of the 16-
// aligned part of the tap's half-dot into acc[2 tap + h] (int32 atomics: the
// integer sum is exact whatever the order). The last block to finish (ticket)
// adds each half's float tail in the reference's order, scales, applies the
// polarity test and writes corr[n], C[2]; it leaves acc and the ticket at 0.
template <int CPX>
__global__ void __launch_bounds__(256) corr_std_kernel(
    const char2 *__restrict__ IQ, const char2 *__restrict__ code, int N, TapArgs ta, float cs,
    int2 *acc, unsigned *ticket, float2 *corr, float2 *C)
{
    const int tap = blockIdx.x, h = blockIdx.y;
    const int j = ta.jk[tap].x, k = ta.jk[tap].y;
    const int len = h == 0 ? j : N - j;
    const char2 *x = IQ + (h == 0 ? 0 : j);
    const char2 *y = code + (size_t)k * N + (h == 0 ? N - j : 0);
    const int main_len = (len / 16) * 16;
    const int c0 = blockIdx.z * kCorrChunk;
    int sr = 0, si = 0;
    if (c0 < main_len) {
        const int c1 = min(main_len, c0 + kCorrChunk);
        char2 a[4], c[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = c0 + threadIdx.x + u * 256;
            a[u] = i < c1 ? x[i] : make_char2(0, 0);
            c[u] = i < c1 ? y[i] : make_char2(0, 0);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (CPX) {
                sr += sgn_mul8(a[u].x, c[u].x) + sgn_mul8(a[u].y, c[u].y);
                si += sgn_mul8(a[u].y, c[u].x) + sgn_mul8(a[u].x, neg8(c[u].y));
            } else {
                sr += sgn_mul8(a[u].x, c[u].x);
                si += sgn_mul8(a[u].y, c[u].y);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sr += __shfl_xor_sync(0xffffffffu, sr, o);
            si += __shfl_xor_sync(0xffffffffu, si, o);
        }
        if ((threadIdx.x & 31) == 0 && (sr || si)) {
            atomicAdd(&acc[2 * tap + h].x, sr);
            atomicAdd(&acc[2 * tap + h].y, si);
        }
    }
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x * gridDim.y * gridDim.z - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // every half: its integer sum, then its tail in float one product at a
    // time in the reference's order, scaled
    __shared__ float2 c12[2 * SDR_MAX_CORR];
    const int n = ta.n;
    for (int q = threadIdx.x; q < 2 * n; q += blockDim.x) {
        const int tq = q >> 1, hq = q & 1;
        const int jq = ta.jk[tq].x, kq = ta.jk[tq].y;
        const int lq = hq == 0 ? jq : N - jq;
        const char2 *xq = IQ + (hq == 0 ? 0 : jq);
        const char2 *yq = code + (size_t)kq * N + (hq == 0 ? N - jq : 0);
        float fr = (float)atomicExch(&acc[q].x, 0), fi = (float)atomicExch(&acc[q].y, 0);
        for (int i = (lq / 16) * 16; i < lq; ++i) {
            const char2 av = xq[i], cv = yq[i];
            if (CPX) {
                fr = __fadd_rn(fr, (float)(av.x * cv.x + av.y * cv.y));
                fi = __fadd_rn(fi, (float)(av.y * cv.x - av.x * cv.y));
            } else {
                fr = __fadd_rn(fr, (float)(av.x * cv.x));
                fi = __fadd_rn(fi, (float)(av.y * cv.y));
            }
        }
        c12[q] = make_float2(__fmul_rn(fr, cs), __fmul_rn(fi, cs));
    }
    __syncthreads();
    __shared__ float sign;
    if (threadIdx.x == 0) {
        float dot = 0.0f;
        for (int i = 0; i < 3 && i < n; ++i) {
            const float2 a = c12[2 * i], b = c12[2 * i + 1];
            dot = __fadd_rn(dot, __fmaf_rn(a.x, b.x, __fmul_rn(a.y, b.y)));
        }
        sign = dot < 0.0f ? -1.0f : 1.0f;
        if (n > 0) { C[0] = c12[0]; C[1] = c12[1]; }
        *ticket = 0u;
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

// The thread's device scratch of the synchronous correlators: integer
// partial sums (2 SDR_MAX_CORR int2), outputs (SDR_MAX_CORR + 2) and the
// finishing ticket, zeroed once (the finishing block leaves them 0).
static int corr_scratch(int2 **acc, float2 **out, unsigned **ticket, cudaStream_t st)
{
    ThreadCtx &c = tctx();
    const size_t bytes = sizeof(int2) * 2 * SDR_MAX_CORR + sizeof(float2) * (SDR_MAX_CORR + 2) + 16;
    const bool fresh = c.corr_dev.size < bytes;
    int e;
    if ((e = c.corr_dev.reserve(bytes))) return e;
    *acc = (int2 *)c.corr_dev.ptr;
    *out = (float2 *)(*acc + 2 * SDR_MAX_CORR);
    *ticket = (unsigned *)(*out + SDR_MAX_CORR + 2);
    if (fresh) SDRG_CUDA(cudaMemsetAsync(c.corr_dev.ptr, 0, bytes, st));
    return SDRG_OK;
}

// IQ_dev / code_dev on the device, tap shifts in ta; results to host corr / C
// through the pinned staging `out_h` (n + 2 values). One launch.
static int corr_std_run(const char2 *IQ_dev, const char2 *code_dev, int N, const TapArgs &ta,
                        int cpx, float2 *out_h, sdr_cpx_t *corr, sdr_cpx_t *C, cudaStream_t st)
{
    const int n = ta.n;
    int2 *acc;
    float2 *out_d;
    unsigned *ticket;
    int e;
    if ((e = corr_scratch(&acc, &out_d, &ticket, st))) return e;
    const dim3 grid((unsigned)n, 2, (unsigned)((N + kCorrChunk - 1) / kCorrChunk));
    if (cpx) corr_std_kernel<1><<<grid, 256, 0, st>>>(IQ_dev, code_dev, N, ta, kCScale, acc,
                                                     ticket, out_d, out_d + n);
    else     corr_std_kernel<0><<<grid, 256, 0, st>>>(IQ_dev, code_dev, N, ta, kCScale, acc,
                                                     ticket, out_d, out_d + n);
    SDRG_CUDA(cudaGetLastError());
    SDRG_CUDA(cudaMemcpyAsync(out_h, out_d, sizeof(float2) * (n + 2), cudaMemcpyDeviceToHost, st));
    SDRG_CUDA(cudaStreamSynchronize(st));
    memcpy(corr, out_h, sizeof(float2) * n);
    if (C) memcpy(C, out_h + n, sizeof(float2) * 2);
    return SDRG_OK;
}

constexpr int kBankCacheMax = 16;

// The device copy of the caller's code bank (pointer, N): every bank a tap
// selects (mask) is on the device and equal, byte for byte, to the caller's
// bank once the uploads queued on st (staged through `stage`, SDR_N_CODES x
// 2N bytes of pinned memory) have run.
static int bank_on_device(const sdr_cpx16_t *code, int N, uint32_t mask, uint8_t *stage,
                          cudaStream_t st, const char2 **dev_out)
{
    ThreadCtx &c = tctx();
    const size_t bb = (size_t)N * 2;                 // bytes per bank
    BankCache *bc = nullptr;
    for (BankCache *b : c.banks)
        if (b->key == code && b->N == N) { bc = b; break; }
    if (!bc) {
        if ((int)c.banks.size() >= kBankCacheMax) {   // evict the least recently used
            size_t lru = 0;
            for (size_t i = 1; i < c.banks.size(); ++i)
                if (c.banks[i]->used < c.banks[lru]->used) lru = i;
            SDRG_CUDA(cudaStreamSynchronize(st));
            delete c.banks[lru];
            c.banks.erase(c.banks.begin() + (long)lru);
        }
        int fe;
        if ((fe = alloc_fault("cudaMalloc"))) return fe;
        void *d = nullptr;
        SDRG_CUDA(cudaMalloc(&d, bb * SDR_N_CODES));
        bc = new BankCache();
        bc->key = code;
        bc->N = N;
        bc->dev = d;
        bc->host.resize(bb * SDR_N_CODES);
        c.banks.push_back(bc);
    }
    bc->used = ++c.bank_clock;
    const uint8_t *src = (const uint8_t *)code;
    for (int k = 0; k < SDR_N_CODES; ++k) {
        if (!((mask >> k) & 1u)) continue;
        const size_t off = (size_t)k * bb;
        if (((bc->valid >> k) & 1u) && memcmp(bc->host.data() + off, src + off, bb) == 0) continue;
        memcpy(bc->host.data() + off, src + off, bb);
        memcpy(stage + off, src + off, bb);
        bc->valid |= 1u << k;
        SDRG_CUDA(cudaMemcpyAsync((uint8_t *)bc->dev + off, stage + off, bb,
                                  cudaMemcpyHostToDevice, st));
    }
    *dev_out = (const char2 *)bc->dev;
    return SDRG_OK;
}

// sdr_corr_std / sdr_corr_std_cpx_code: IQ staged and uploaded, the selected
// code banks resident on the device (uploaded when their bytes change), one
// launch, results back.
static void corr_std_host(const sdr_cpx16_t *IQ, const sdr_cpx16_t *code, int N, double coff,
                          const double *pos, int n, sdr_cpx_t *corr, sdr_cpx_t *C, int cpx)
{
    if (N <= 0 || n <= 0) return;
    cudaStream_t st;
    ThreadCtx &c = tctx();
    TapArgs ta;
    uint32_t mask = 0;
    const size_t iqb = (size_t)N * 2, cb = (size_t)N * 2 * SDR_N_CODES;
    c.host[0].pinned = true;
    c.host[2].pinned = true;
    if (n > SDR_MAX_CORR) {
        set_error(SDRG_ERR_ARG, "corr_std: n=%d > %d", n, SDR_MAX_CORR);
        goto fail;
    }
    ta.n = n;
    if (!tap_params(N, coff, pos, n, SDR_N_CODES, ta.jk)) {
        set_error(SDRG_ERR_ARG, "corr_std: a tap shift leaves [-N, 2N) or the code bank");
        goto fail;
    }
    for (int i = 0; i < n; ++i) mask |= 1u << ta.jk[i].y;
    // a failing step has recorded its error in the thread's last-error state
    if (ensure_device(nullptr) || thread_stream(&st) || c.host[0].reserve(iqb + cb + 16) ||
        c.dev[0].reserve(iqb + 16) || c.host[2].reserve(sizeof(float2) * (SDR_MAX_CORR + 2)))
        goto fail;
    {
        // the IQ window goes first, so that its copy overlaps the comparison
        // of the code banks on the host
        uint8_t *h = (uint8_t *)c.host[0].ptr;
        const char2 *code_d = nullptr;
        memcpy(h, IQ, iqb);
        if (cudaMemcpyAsync(c.dev[0].ptr, h, iqb, cudaMemcpyHostToDevice, st) != cudaSuccess) {
            cuda_error(cudaGetLastError(), "corr_std H2D");
            goto fail;
        }
        if (bank_on_device(code, N, mask, h + iqb, st, &code_d)) goto fail;
        if (corr_std_run((const char2 *)c.dev[0].ptr, code_d, N, ta, cpx, (float2 *)c.host[2].ptr,
                         corr, C, st))
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
    ThreadCtx &c = tctx();
    c.host[0].pinned = true;
    if (ensure_device(nullptr) || thread_stream(&st) ||
        c.dev[0].reserve((size_t)N * 4 + (size_t)N * 4 + 64) ||
        c.host[0].reserve((size_t)N * 4 + 16)) {
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
    TapArgs ta;
    ta.n = n;
    c.host[2].pinned = true;
    if (n > SDR_MAX_CORR) {
        set_error(SDRG_ERR_ARG, "corr_std: n=%d > %d", n, SDR_MAX_CORR);
        memset(corr, 0, sizeof(sdr_cpx_t) * n);
        return;
    }
    if (!tap_params(N, 0.0, pos, n, 1, ta.jk)) {
        set_error(SDRG_ERR_ARG, "corr_std: a tap shift leaves [-N, 2N) or the code bank");
        memset(corr, 0, sizeof(sdr_cpx_t) * n);
        return;
    }
    if (c.host[2].reserve(sizeof(float2) * (SDR_MAX_CORR + 2)) ||
        corr_std_run(iq_d, code_d, N, ta, 0, (float2 *)c.host[2].ptr, corr, Cb, st)) {
        memset(corr, 0, sizeof(sdr_cpx_t) * n);
    }
}

} // extern "C"

// ---------------------------------------------------------------------------
// batched tracking correlators (sdrg_corr_batch)
// ---------------------------------------------------------------------------
namespace sdrg {

struct CorrJobDev {
    const uint8_t *buf;
    int len, ix, N, nsplit;
    uint32_t p0a, p0b, step;
    int cpx, tap0, n;
    size_t iq_off;              // first sample of this job in the IQ scratch
    const char2 *code;          // bank [SDR_N_CODES][N]
    int vec;                    // real code, 4-byte aligned bank: packed dot products
    int has128;                 // set by mixb_kernel: the window holds a -128 byte
};

struct TapDev { int job, j, k, pad; };

__device__ __forceinline__ char2 mix_byte_b(uint8_t byte, uint32_t phase, const char2 *ctab)
{
    const int I = (int)(int8_t)(uint8_t)(byte << 4) >> 4;
    const int Q = (int)(int8_t)byte >> 4;
    const char2 c = ctab[phase >> 24];
    char2 o;
    o.x = (signed char)(I * c.x - Q * c.y);
    o.y = (signed char)(I * c.y + Q * c.x);
    return o;
}

// grid (chunks, jobs): carrier wipe-off of every job's window into the IQ
// scratch, with the reference's phase restart at the buffer wrap
__global__ void mixb_kernel(CorrJobDev *__restrict__ jobs, const char2 *__restrict__ ctab_g,
                            char2 *__restrict__ iq)
{
    __shared__ char2 ctab[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) ctab[i] = ctab_g[i];
    __syncthreads();
    const CorrJobDev J = jobs[blockIdx.y];
    char2 *out = iq + J.iq_off;
    bool m128 = false;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < J.N; n += gridDim.x * blockDim.x) {
        int pos = J.ix + n;
        if (pos >= J.len) pos -= J.len;
        const uint32_t ph = n < J.nsplit ? J.p0a + J.step * (uint32_t)n
                                         : J.p0b + J.step * (uint32_t)(n - J.nsplit);
        const char2 o = mix_byte_b(__ldg(J.buf + pos), ph, ctab);
        out[n] = o;
        m128 |= (o.x == -128) | (o.y == -128);
    }
    if (m128) atomicOr(&jobs[blockIdx.y].has128, 1);
}

// sign-product partial sums of one half-dot over [0, main_len) (integer)
template <bool CPX>
__device__ __forceinline__ void half_main(const char2 *__restrict__ x, const char2 *__restrict__ y,
                                          int main_len, int &sr, int &si)
{
    for (int i = threadIdx.x; i < main_len; i += blockDim.x) {
        const char2 a = x[i], c = __ldg(y + i);
        if (CPX) {
            sr += sgn_mul8(a.x, c.x) + sgn_mul8(a.y, c.y);
            si += sgn_mul8(a.y, c.x) + sgn_mul8(a.x, neg8(c.y));
        } else {
            sr += sgn_mul8(a.x, c.x);
            si += sgn_mul8(a.y, c.y);
        }
    }
}

// Packed form of half_main<false>, four samples per dp4a. sgn_mul8(x, c)
// equals x * sgn(c) except for x = -128 with c < 0, where the reference's
// byte negation wraps to -128 (x * sgn(c) = +128): with FIX those lanes are
// counted and 256 taken off each, so the integer sums are identical. Windows
// without a -128 sample (flagged by mixb_kernel) skip the count.
template <bool FIX>
__device__ __forceinline__ void sgn_dot4(int &s, uint32_t x, uint32_t c)
{
    const uint32_t u = (c & 0x7f7f7f7fu) + 0x7f7f7f7fu;        // bit 7: c's low 7 bits != 0
    const uint32_t pos = ((u & ~c) & 0x80808080u) >> 7;        // 1 in lanes with c > 0
    uint32_t negm;                                              // -1 in lanes with c < 0
    asm("prmt.b32 %0, %1, 0, 0xBA98;" : "=r"(negm) : "r"(c));  // each byte's sign replicated
    s = __dp4a((int)x, (int)(pos | negm), s);                   // x * sgn(c), four lanes
    if (FIX) {
        const uint32_t t = x ^ 0x80808080u;                    // 0 in lanes with x = -128
        const uint32_t v = (t & 0x7f7f7f7fu) + 0x7f7f7f7fu;
        const uint32_t m = (~(v | t) & 0x80808080u) >> 7;      // 1 in lanes with x = -128
        s += 256 * __dp4a((int)m, (int)negm, 0);               // minus 256 per such lane
    }
}

// The main part of one half-dot with a real code: H pairs of 32-bit words
// (p, p + H), each word two char2 samples. xp / yp point at the aligned word
// holding a stream's first sample; XO / YO: the stream starts at its second
// sample, so each word is joined from two loads (the second one's first
// sample is in the stream, so the load stays inside the array).
template <int XO, int YO, bool FIX>
__device__ __forceinline__ void half_vec(const uint32_t *__restrict__ xp,
                                         const uint32_t *__restrict__ yp, int H, int &sr, int &si)
{
    for (int p = threadIdx.x; p < H; p += blockDim.x) {
        uint32_t x0 = __ldg(xp + p), x1 = __ldg(xp + p + H);
        uint32_t y0 = __ldg(yp + p), y1 = __ldg(yp + p + H);
        if (XO) {
            x0 = __funnelshift_r(x0, __ldg(xp + p + 1), 16);
            x1 = __funnelshift_r(x1, __ldg(xp + p + H + 1), 16);
        }
        if (YO) {
            y0 = __funnelshift_r(y0, __ldg(yp + p + 1), 16);
            y1 = __funnelshift_r(y1, __ldg(yp + p + H + 1), 16);
        }
        sgn_dot4<FIX>(sr, __byte_perm(x0, x1, 0x6420), __byte_perm(y0, y1, 0x6420));   // I lanes
        sgn_dot4<FIX>(si, __byte_perm(x0, x1, 0x7531), __byte_perm(y0, y1, 0x7531));   // Q lanes
    }
}

// x at sample xoff of xb, code at sample yoff of yb (both 4-byte aligned
// arrays); main_len a multiple of 16 samples
__device__ __forceinline__ void half_main_vec(const uint32_t *xb, size_t xoff,
                                              const uint32_t *yb, size_t yoff, int main_len,
                                              bool fix, int &sr, int &si)
{
    const uint32_t *xp = xb + (xoff >> 1), *yp = yb + (yoff >> 1);
    const int H = main_len >> 2;
    switch ((int)(xoff & 1) | ((int)(yoff & 1) << 1) | (fix ? 4 : 0)) {
    case 0: half_vec<0, 0, false>(xp, yp, H, sr, si); break;
    case 1: half_vec<1, 0, false>(xp, yp, H, sr, si); break;
    case 2: half_vec<0, 1, false>(xp, yp, H, sr, si); break;
    case 3: half_vec<1, 1, false>(xp, yp, H, sr, si); break;
    case 4: half_vec<0, 0, true>(xp, yp, H, sr, si); break;
    case 5: half_vec<1, 0, true>(xp, yp, H, sr, si); break;
    case 6: half_vec<0, 1, true>(xp, yp, H, sr, si); break;
    default: half_vec<1, 1, true>(xp, yp, H, sr, si); break;
    }
}

// one block (128 threads) per tap: both half-dots of src/sdr_func.c:990-991
__global__ void __launch_bounds__(128) tapb_kernel(const TapDev *__restrict__ taps,
                                                   const CorrJobDev *__restrict__ jobs,
                                                   const char2 *__restrict__ iq, float cs,
                                                   float2 *__restrict__ c12)
{
    const TapDev T = taps[blockIdx.x];
    const CorrJobDev J = jobs[T.job];
    const int N = J.N, j = T.j;
    const char2 *IQ = iq + J.iq_off;
    const char2 *bank = J.code + (size_t)T.k * N;
    __shared__ int red[2][2][4];
    int sum[2][2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int len = h == 0 ? j : N - j;
        const char2 *x = IQ + (h == 0 ? 0 : j);
        const char2 *y = bank + (h == 0 ? N - j : 0);
        int sr = 0, si = 0;
        if (J.vec)
            half_main_vec((const uint32_t *)iq, J.iq_off + (h == 0 ? 0 : j),
                          (const uint32_t *)J.code, (size_t)T.k * N + (h == 0 ? N - j : 0),
                          (len / 16) * 16, J.has128 != 0, sr, si);
        else if (J.cpx) half_main<true>(x, y, (len / 16) * 16, sr, si);
        else half_main<false>(x, y, (len / 16) * 16, sr, si);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sr += __shfl_xor_sync(0xffffffffu, sr, o);
            si += __shfl_xor_sync(0xffffffffu, si, o);
        }
        sum[h][0] = sr;
        sum[h][1] = si;
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[0][0][w] = sum[0][0]; red[0][1][w] = sum[0][1];
        red[1][0][w] = sum[1][0]; red[1][1][w] = sum[1][1];
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        const int h = threadIdx.x;
        const int len = h == 0 ? j : N - j;
        const char2 *x = IQ + (h == 0 ? 0 : j);
        const char2 *y = bank + (h == 0 ? N - j : 0);
        int tr = 0, ti = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { tr += red[h][0][i]; ti += red[h][1][i]; }
        float fr = (float)tr, fi = (float)ti;
        for (int i = (len / 16) * 16; i < len; ++i) {
            const char2 a = x[i], c = y[i];
            if (J.cpx) {
                fr = __fadd_rn(fr, (float)(a.x * c.x + a.y * c.y));
                fi = __fadd_rn(fi, (float)(a.y * c.x - a.x * c.y));
            } else {
                fr = __fadd_rn(fr, (float)(a.x * c.x));
                fi = __fadd_rn(fi, (float)(a.y * c.y));
            }
        }
        c12[2 * blockIdx.x + h] = make_float2(__fmul_rn(fr, cs), __fmul_rn(fi, cs));
    }
}

// one warp per job: polarity test and outputs (src/sdr_func.c:993-1007)
__global__ void finb_kernel(const CorrJobDev *__restrict__ jobs, const float2 *__restrict__ c12,
                            float2 *__restrict__ corr, float2 *__restrict__ C)
{
    const CorrJobDev J = jobs[blockIdx.x];
    const float2 *cc = c12 + 2 * (size_t)J.tap0;
    float dot = 0.0f;
    for (int i = 0; i < 3 && i < J.n; ++i) {
        const float2 a = cc[2 * i], b = cc[2 * i + 1];
        dot = __fadd_rn(dot, __fmaf_rn(a.x, b.x, __fmul_rn(a.y, b.y)));
    }
    const float sign = dot < 0.0f ? -1.0f : 1.0f;
    const float fN = (float)J.N;
    float2 *out = corr + (size_t)blockIdx.x * SDR_MAX_CORR;
    for (int i = threadIdx.x; i < J.n; i += blockDim.x) {
        const float2 a = cc[2 * i], b = cc[2 * i + 1];
        out[i] = make_float2(__fdiv_rn(__fadd_rn(a.x, __fmul_rn(sign, b.x)), fN),
                             __fdiv_rn(__fadd_rn(a.y, __fmul_rn(sign, b.y)), fN));
    }
    if (C && threadIdx.x == 0 && J.n > 0) {
        C[2 * (size_t)blockIdx.x] = cc[0];
        C[2 * (size_t)blockIdx.x + 1] = cc[1];
    }
}

static inline uint32_t phase_b(double phi) { return (uint32_t)((phi - floor(phi)) * 4294967296.0); }
static inline uint32_t step_b(double step) { return (uint32_t)(int)(step * 4294967296.0); }

} // namespace sdrg

extern "C" int sdrg_corr_batch(const sdrg_corr_job_t *jobs, int n_job, const uint8_t *const *if_dev,
                               const int *len_if, sdr_cpx_t *corr_dev, sdr_cpx_t *C_dev, void *stream)
{
    if (n_job <= 0) return SDRG_OK;
    if (!jobs || !if_dev || !len_if || !corr_dev)
        return set_error(SDRG_ERR_ARG, "sdrg_corr_batch: null argument");
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    cudaStream_t st = (cudaStream_t)stream;
    if (!st && (e = thread_stream(&st))) return e;
    ThreadCtx &c = tctx();
    // table sizes
    size_t n_tap = 0, n_iq = 0;
    for (int i = 0; i < n_job; ++i) {
        const sdrg_corr_job_t &J = jobs[i];
        if (J.N <= 0 || J.n <= 0 || J.n > SDR_MAX_CORR || !J.code || !J.pos || J.buf < 0 ||
            J.ix < 0 || J.ix >= len_if[J.buf] || J.N > len_if[J.buf] || J.fs <= 0)
            return set_error(SDRG_ERR_ARG, "sdrg_corr_batch: bad job %d", i);
        n_tap += J.n;
        n_iq += ((size_t)J.N + 15) / 16 * 16;
    }
    const size_t jb = sizeof(CorrJobDev) * n_job, tb = sizeof(TapDev) * n_tap;
    const size_t tab_bytes = (jb + tb + 255) / 256 * 256;
    const size_t dev_bytes = tab_bytes + n_iq * sizeof(char2) + 2 * n_tap * sizeof(float2) + 512;
    if (!c.cb_ev) {
        SDRG_CUDA(cudaEventCreateWithFlags(&c.cb_ev, cudaEventDisableTiming));
        SDRG_CUDA(cudaEventCreateWithFlags(&c.cb_done, cudaEventDisableTiming));
    }
    // the previous call's upload from the host staging has finished, and this
    // call's device work follows the previous call's (which may be on another
    // stream) because both use this thread's scratch
    SDRG_CUDA(cudaEventSynchronize(c.cb_ev));
    SDRG_CUDA(cudaStreamWaitEvent(st, c.cb_done, 0));
    c.cb_host.pinned = true;
    if (dev_bytes > c.cb_dev.size) SDRG_CUDA(cudaStreamSynchronize(st));
    if ((e = c.cb_host.reserve(tab_bytes)) || (e = c.cb_dev.reserve(dev_bytes))) return e;
    CorrJobDev *jh = (CorrJobDev *)c.cb_host.ptr;
    TapDev *th = (TapDev *)((char *)c.cb_host.ptr + jb);
    size_t tap = 0, iq_off = 0;
    std::vector<int2> jk(SDR_MAX_CORR);
    for (int i = 0; i < n_job; ++i) {
        const sdrg_corr_job_t &J = jobs[i];
        const int len = len_if[J.buf];
        // the reference's tap arithmetic (src/sdr_func.c:988-990), in double
        if (!tap_params(J.N, J.coff, J.pos, J.n, SDR_N_CODES, jk.data()))
            return set_error(SDRG_ERR_ARG, "sdrg_corr_batch: job %d tap outside one wrap", i);
        // sdr_mix_carr's phase arithmetic and wrap split (src/sdr_func.c:772-836)
        const double step = J.fc / J.fs;
        const int n1 = (J.ix + J.N <= len) ? J.N : len - J.ix;
        CorrJobDev d;
        d.buf = if_dev[J.buf]; d.len = len; d.ix = J.ix; d.N = J.N; d.nsplit = n1;
        d.p0a = phase_b(J.phi);
        d.p0b = n1 < J.N ? phase_b(J.phi + step * n1) : 0;
        d.step = step_b(step);
        d.cpx = J.cpx_code ? 1 : 0; d.tap0 = (int)tap; d.n = J.n;
        d.iq_off = iq_off;
        d.code = (const char2 *)J.code;
        d.vec = !J.cpx_code && ((uintptr_t)J.code & 3) == 0;
        d.has128 = 0;
        jh[i] = d;
        for (int t = 0; t < J.n; ++t) th[tap + t] = TapDev{i, jk[t].x, jk[t].y, 0};
        tap += J.n;
        iq_off += ((size_t)J.N + 15) / 16 * 16;
    }
    char *db = (char *)c.cb_dev.ptr;
    CorrJobDev *jd = (CorrJobDev *)db;
    TapDev *td = (TapDev *)(db + jb);
    char2 *iq = (char2 *)(db + tab_bytes);
    float2 *c12 = (float2 *)(db + tab_bytes + ((n_iq * sizeof(char2) + 255) / 256) * 256);
    SDRG_CUDA(cudaMemcpyAsync(db, c.cb_host.ptr, jb + tb, cudaMemcpyHostToDevice, st));
    SDRG_CUDA(cudaEventRecord(c.cb_ev, st));
    int maxN = 0;
    for (int i = 0; i < n_job; ++i) maxN = jobs[i].N > maxN ? jobs[i].N : maxN;
    dim3 mg((unsigned)((maxN + 255) / 256 < 64 ? (maxN + 255) / 256 : 64), (unsigned)n_job);
    mixb_kernel<<<mg, 256, 0, st>>>(jd, dev->ctab_dev, iq);
    SDRG_CUDA(cudaGetLastError());
    tapb_kernel<<<(unsigned)n_tap, 128, 0, st>>>(td, jd, iq, kCScale, c12);
    SDRG_CUDA(cudaGetLastError());
    finb_kernel<<<(unsigned)n_job, 32, 0, st>>>(jd, c12, (float2 *)corr_dev, (float2 *)C_dev);
    SDRG_CUDA(cudaGetLastError());
    SDRG_CUDA(cudaEventRecord(c.cb_done, st));
    return SDRG_OK;
}
