// sdrg_mix.cu - carrier wipe-off (reference: src/sdr_func.c:772-848).
//
// A packed sample (I in the low nibble, Q in the high nibble, each sign-
// extended) is rotated by the quantised carrier of its 8-bit phase:
//   I' = (int8)(I*cI - Q*cQ),  Q' = (int8)(I*cQ + Q*cI)
// which is exactly the reference's 64K-entry table entry (src/sdr_func.c:
// 113-134); the phase of sample n is p0 + n*step (uint32, wrapping), and a
// window that crosses the end of the circular buffer restarts the phase at
// the wrap from phi + step*n (src/sdr_func.c:829-835).
#include <cmath>
#include <cstring>
#include <vector>

#include "sdrg_internal.h"

namespace sdrg {

__device__ __forceinline__ char2 mix_byte(uint8_t byte, uint32_t phase, const char2 *ctab)
{
    const int I = (int)(int8_t)(uint8_t)(byte << 4) >> 4;
    const int Q = (int)(int8_t)byte >> 4;
    const char2 c = ctab[phase >> 24];
    char2 o;
    o.x = (signed char)(I * c.x - Q * c.y);
    o.y = (signed char)(I * c.y + Q * c.x);
    return o;
}

// Window sample n is buf[(ix + n) mod len], its carrier phase
// n < nsplit ? p0a + n step : p0b + (n - nsplit) step (the restart at the
// buffer wrap). 16 samples per thread: where its 16 samples lie contiguous in
// the buffer (inside one segment of the window) and the output is 16-byte
// aligned, the one or two aligned 16-byte blocks that hold them, realigned
// with funnel shifts (any window start), the nibbles of four samples
// sign-extended at once, each rotation as two dp2a of the sample bytes with
// the carrier's 16-bit coefficient pairs, and two 16-byte stores; otherwise
// sample by sample (mix_byte). HBM bound by design: 1 byte read and 2 bytes
// written per sample.
// 16-byte loads per thread (two measured slower: 1.09 against 1.45 T
// samples/s)
constexpr int kMixVec = 1;
constexpr int kMixPer = 16 * kMixVec;

// Sign-extended nibbles of four packed samples: the low (I) or high (Q)
// nibble of each byte of w as a signed byte (a nibble n >= 8 becomes n | 0xF0:
// the multiply sets the upper four bits of exactly those bytes, no carries).
__device__ __forceinline__ uint32_t nibbles_i(uint32_t w)
{
    const uint32_t lo = w & 0x0F0F0F0Fu;
    return lo | ((lo & 0x08080808u) * 0x1Eu);
}
__device__ __forceinline__ uint32_t nibbles_q(uint32_t w)
{
    return nibbles_i(w >> 4);
}

// bytes s .. s + 15 of the 32 bytes lo:hi (s in 0..15)
__device__ __forceinline__ uint4 realign16(uint4 lo, uint4 hi, int s)
{
    const uint32_t sh = 8u * (uint32_t)(s & 3);
    const uint32_t w[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
    uint4 r;
    switch (s >> 2) {
    case 0:
        r = make_uint4(__funnelshift_r(w[0], w[1], sh), __funnelshift_r(w[1], w[2], sh),
                       __funnelshift_r(w[2], w[3], sh), __funnelshift_r(w[3], w[4], sh));
        break;
    case 1:
        r = make_uint4(__funnelshift_r(w[1], w[2], sh), __funnelshift_r(w[2], w[3], sh),
                       __funnelshift_r(w[3], w[4], sh), __funnelshift_r(w[4], w[5], sh));
        break;
    case 2:
        r = make_uint4(__funnelshift_r(w[2], w[3], sh), __funnelshift_r(w[3], w[4], sh),
                       __funnelshift_r(w[4], w[5], sh), __funnelshift_r(w[5], w[6], sh));
        break;
    default:
        r = make_uint4(__funnelshift_r(w[3], w[4], sh), __funnelshift_r(w[4], w[5], sh),
                       __funnelshift_r(w[5], w[6], sh), __funnelshift_r(w[6], w[7], sh));
        break;
    }
    return r;
}

__global__ void __launch_bounds__(256) mix_kernel(
    const uint8_t *__restrict__ buf, int len, int ix, int N, int nsplit, uint32_t p0a,
    uint32_t p0b, uint32_t step, const char2 *__restrict__ ctab_g, char2 *__restrict__ out)
{
    __shared__ char2 ctab[256];
    // the same carrier as 16-bit coefficient pairs for dp2a: I' = (cI, -cQ) . (I, Q),
    // Q' = (cQ, cI) . (I, Q) - the exact integer products and sums of mix_byte
    __shared__ uint2 cdp[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        const char2 c = ctab_g[i];
        ctab[i] = c;
        cdp[i] = make_uint2((uint32_t)(uint16_t)(int16_t)c.x | ((uint32_t)(uint16_t)(int16_t)(-c.y) << 16),
                            (uint32_t)(uint16_t)(int16_t)c.y | ((uint32_t)(uint16_t)(int16_t)c.x << 16));
    }
    __syncthreads();
    const long long n0l = (long long)kMixPer * (blockIdx.x * (long long)blockDim.x + threadIdx.x);
    if (n0l >= N) return;
    const int n0 = (int)n0l;
    int pos0 = ix + n0;
    if (pos0 >= len) pos0 -= len;
    // the aligned block holding the first sample's byte starts s bytes before
    // it; the second block is needed when s > 0
    const int s = (int)(((uintptr_t)buf + (uintptr_t)pos0) & 15u), a0 = pos0 - s;
    const bool fast = n0 + kMixPer <= N && pos0 + kMixPer <= len && a0 >= 0 &&
                      (s == 0 || a0 + 16 * kMixVec + 16 <= len) &&
                      (n0 + kMixPer <= nsplit || n0 >= nsplit) &&
                      (((uintptr_t)(out + n0)) & 15u) == 0;
    if (fast) {
        uint4 w[kMixVec];
        if (s == 0) {
#pragma unroll
            for (int v = 0; v < kMixVec; ++v) w[v] = *(const uint4 *)(buf + a0 + 16 * v);
        } else {
            uint4 b[kMixVec + 1];
#pragma unroll
            for (int v = 0; v <= kMixVec; ++v) b[v] = *(const uint4 *)(buf + a0 + 16 * v);
#pragma unroll
            for (int v = 0; v < kMixVec; ++v) w[v] = realign16(b[v], b[v + 1], s);
        }
        uint32_t ph = n0 < nsplit ? p0a + step * (uint32_t)n0 : p0b + step * (uint32_t)(n0 - nsplit);
#pragma unroll
        for (int v = 0; v < kMixVec; ++v) {
            const uint32_t wd[4] = {w[v].x, w[v].y, w[v].z, w[v].w};
            uint32_t o[8];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t I4 = nibbles_i(wd[q]), Q4 = nibbles_q(wd[q]);
                uint32_t t[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    // sample k of the word: bytes (I, Q) for dp2a
                    const uint32_t sv = __byte_perm(I4, Q4, (uint32_t)(k | ((4 + k) << 4)));
                    const uint2 cf = cdp[ph >> 24];
                    ph += step;
                    const int ii = __dp2a_lo((int)cf.x, (int)sv, 0);
                    const int qq = __dp2a_lo((int)cf.y, (int)sv, 0);
                    t[k] = __byte_perm((uint32_t)ii, (uint32_t)qq, 0x0040u);   // (I', Q') bytes
                }
                o[2 * q] = __byte_perm(t[0], t[1], 0x5410u);
                o[2 * q + 1] = __byte_perm(t[2], t[3], 0x5410u);
            }
            uint4 *d = (uint4 *)(out + n0 + 16 * v);
            d[0] = make_uint4(o[0], o[1], o[2], o[3]);
            d[1] = make_uint4(o[4], o[5], o[6], o[7]);
        }
    } else {
        for (int n = n0; n < N && n < n0 + kMixPer; ++n) {
            int pos = ix + n;
            if (pos >= len) pos -= len;
            const uint32_t ph = n < nsplit ? p0a + step * (uint32_t)n
                                           : p0b + step * (uint32_t)(n - nsplit);
            out[n] = mix_byte(buf[pos], ph, ctab);
        }
    }
}

// float I/Q -> (int8) -> 4+4-bit pack (src/sdr_func.c:842-844, SDR_CPX8 of
// src/pocket_sdr.h:103): C's float->int8 conversion truncates toward zero.
__global__ void pack_cpx_kernel(const float2 *__restrict__ in, int N, uint8_t *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float2 v = in[i];
    const int8_t re = (int8_t)__float2int_rz(v.x);
    const int8_t im = (int8_t)__float2int_rz(v.y);
    out[i] = (uint8_t)(((uint8_t)im << 4) | ((uint8_t)re & 0x0F));
}

static inline uint32_t phase_of(double phi)
{
    return (uint32_t)((phi - floor(phi)) * 4294967296.0);
}
static inline uint32_t step_of(double step)
{
    return (uint32_t)(int)(step * 4294967296.0);
}

int launch_mix(const uint8_t *buf_dev, int len, int ix, int N, int nsplit, uint32_t p0a,
               uint32_t p0b, uint32_t step, const char2 *ctab_dev, char2 *out_dev,
               cudaStream_t st)
{
    const int threads = 256;
    const long long units = ((long long)N + kMixPer - 1) / kMixPer;
    const unsigned blocks = (unsigned)((units + threads - 1) / threads);
    mix_kernel<<<blocks, threads, 0, st>>>(buf_dev, len, ix, N, nsplit, p0a, p0b, step, ctab_dev,
                                           out_dev);
    SDRG_CUDA(cudaGetLastError());
    return SDRG_OK;
}

// Mixes the float buffer as sdr_corr_*_cpx do (src/sdr_func.c:839-848) into
// iq_dev (device, N samples) on stream st. The phase runs continuously over
// the N samples (the float buffer is repacked first, so no phase restart).
int mix_cpx_device(const sdr_cpx_t *buff, int len_buff, int ix, int N, double fs,
                        double fc, double phi, char2 *iq_dev, cudaStream_t st)
{
    if (!buff || len_buff <= 0 || N <= 0)
        return set_error(SDRG_ERR_ARG, "mix_carr_cpx: bad buffer (len=%d N=%d)", len_buff, N);
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    ThreadCtx &c = tctx();
    c.host[1].pinned = true;
    if ((e = c.host[1].reserve((size_t)N * 8)) || (e = c.dev[4].reserve((size_t)N * 9 + 64)))
        return e;
    // gather the window j = ix, ix+1, ... (mod len_buff)
    float2 *h = (float2 *)c.host[1].ptr;
    int j = ((ix % len_buff) + len_buff) % len_buff;
    for (int i = 0; i < N;) {
        int n = len_buff - j < N - i ? len_buff - j : N - i;
        memcpy(h + i, buff + j, (size_t)n * 8);
        i += n;
        j = 0;
    }
    float2 *fin = (float2 *)c.dev[4].ptr;
    uint8_t *packed = (uint8_t *)(fin + N);
    SDRG_CUDA(cudaMemcpyAsync(fin, h, (size_t)N * 8, cudaMemcpyHostToDevice, st));
    pack_cpx_kernel<<<(N + 255) / 256, 256, 0, st>>>(fin, N, packed);
    SDRG_CUDA(cudaGetLastError());
    if ((e = launch_mix(packed, N, 0, N, N, phase_of(phi), 0, step_of(fc / fs), dev->ctab_dev,
                        iq_dev, st)))
        return e;
    // the staging buffer is reused by the next call: finish the copy first
    SDRG_CUDA(cudaStreamSynchronize(st));
    return SDRG_OK;
}

} // namespace sdrg

using namespace sdrg;

extern "C" {

void sdr_mix_carr(const sdr_buff_t *buff, int ix, int N, double fs, double fc, double phi,
                  sdr_cpx16_t *IQ)
{
    if (N <= 0) return;
    if (!buff || !buff->data || ix < 0 || ix >= buff->N || N > buff->N) {
        set_error(SDRG_ERR_ARG, "sdr_mix_carr: bad window ix=%d N=%d len=%d", ix, N,
                  buff ? buff->N : 0);
        memset(IQ, 0, (size_t)N * 2);
        return;
    }
    Device *dev;
    cudaStream_t st;
    ThreadCtx &c = tctx();
    c.host[0].pinned = true;
    // a failing step has recorded its error in the thread's last-error state
    if (ensure_device(&dev) || thread_stream(&st) ||
        c.host[0].reserve((size_t)N * 3 + 16) || c.dev[0].reserve((size_t)N * 3 + 64)) {
        memset(IQ, 0, (size_t)N * 2);
        return;
    }
    const double step = fc / fs;
    const int n1 = (ix + N <= buff->N) ? N : buff->N - ix;
    uint8_t *h = (uint8_t *)c.host[0].ptr;
    memcpy(h, buff->data + ix, (size_t)n1);
    if (n1 < N) memcpy(h + n1, buff->data, (size_t)(N - n1));
    const uint32_t p0a = phase_of(phi);
    const uint32_t p0b = n1 < N ? phase_of(phi + step * n1) : 0;
    uint8_t *win_d = (uint8_t *)c.dev[0].ptr;
    const size_t off = ((size_t)N + 15) / 16 * 16;
    char2 *out_d = (char2 *)(win_d + off);
    char2 *out_h = (char2 *)(h + off);
    if (cudaMemcpyAsync(win_d, h, (size_t)N, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        launch_mix(win_d, N, 0, N, n1, p0a, p0b, step_of(step), dev->ctab_dev, out_d, st) ||
        cudaMemcpyAsync(out_h, out_d, (size_t)N * 2, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cuda_error(cudaGetLastError(), "sdr_mix_carr");
        memset(IQ, 0, (size_t)N * 2);
        return;
    }
    memcpy(IQ, out_h, (size_t)N * 2);
}

int sdrg_mix_carr(const uint8_t *buf_dev, int len, int ix, int N, double fs, double fc,
                  double phi, sdr_cpx16_t *IQ_dev, void *stream)
{
    if (N <= 0) return SDRG_OK;
    if (!buf_dev || !IQ_dev || len <= 0 || ix < 0 || ix >= len || N > len)
        return set_error(SDRG_ERR_ARG, "sdrg_mix_carr: bad window ix=%d N=%d len=%d", ix, N, len);
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    // the phases of sdr_mix_carr (src/sdr_func.c:824-836): restart at the wrap
    const double step = fc / fs;
    const int n1 = (ix + N <= len) ? N : len - ix;
    return launch_mix(buf_dev, len, ix, N, n1, phase_of(phi), n1 < N ? phase_of(phi + step * n1) : 0,
                      step_of(step), dev->ctab_dev, (char2 *)IQ_dev, (cudaStream_t)stream);
}

} // extern "C"
