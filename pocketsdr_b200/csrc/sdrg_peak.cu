// sdrg_peak.cu - grid peak / C/N0 / fine Doppler (reference:
// src/sdr_func.c:690-769).
//
// Per PRN grid [M rows][Nmax cols] (row stride `row_stride`), split over up
// to kPeakChunksMax CTAs (partial maxima and sums) and combined in order by a
// second small kernel:
//  * peak: the first strict maximum in row-major order that exceeds 0
//    (src/sdr_func.c:695-702: P_max starts at 0 and only P > P_max updates),
//    i.e. the largest value with ties broken toward the lower linear index;
//  * mean: sum of all cells in double / cell count (the reference keeps a
//    running mean in double);
//  * C/N0 = 10 log10((Pmax - Pave) / Pave / T), 0 when Pave <= 0;
//  * fine Doppler: vertex of the parabola through the peak bin and its two
//    neighbours at the peak offset (src/sdr_func.c:728-744), the bin itself
//    at the edges.
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "sdrg_internal.h"

namespace sdrg {

constexpr int kPeakThreads = 1024;
constexpr int kPeakChunksMax = 64;

__device__ __forceinline__ void better(float &v, long long &i, float v2, long long i2)
{
    if (v2 > v || (v2 == v && i2 >= 0 && (i < 0 || i2 < i))) { v = v2; i = i2; }
}

__device__ __forceinline__ double fine_dop_dev(const float *P, size_t row_stride, const float *fds,
                                               int M, int bin, int off)
{
    if (bin == 0 || bin == M - 1) return fds[bin];
    const double x0 = fds[bin - 1], x1 = fds[bin], x2 = fds[bin + 1];
    const double y0 = P[(size_t)(bin - 1) * row_stride + off];
    const double y1 = P[(size_t)bin * row_stride + off];
    const double y2 = P[(size_t)(bin + 1) * row_stride + off];
    const double d01 = (y1 - y0) / (x1 - x0), d12 = (y2 - y1) / (x2 - x1);
    const double c = (d12 - d01) / (x2 - x0);
    const double b = d01 - c * (x0 + x1);
    return -b / (2.0 * c);
}

// Partial reduction of one contiguous range of a PRN grid: (largest value
// > 0 with its lowest linear index, double sum) per (chunk, PRN).
struct PeakPart {
    float v;
    long long i;
    double s;
};

__global__ void __launch_bounds__(kPeakThreads) peak_part_kernel(
    const float *__restrict__ P, int M, int Nmax, size_t row_stride, size_t prn_stride,
    int n_chunks, PeakPart *__restrict__ parts)
{
    const float *G = P + (size_t)blockIdx.y * prn_stride;
    float vmax = 0.0f;        // only values > 0 can become the peak
    long long imax = -1;
    double sum = 0.0;
    const bool vec = (Nmax % 4 == 0) && (row_stride % 4 == 0) &&
                     (((uintptr_t)G & 15) == 0);
    const int w4 = vec ? 4 : 1;               // cells per unit
    const int nu = Nmax / w4;                 // units per row
    const long long units = (long long)M * nu;
    const long long per = (units + n_chunks - 1) / n_chunks;
    const long long u0 = (long long)blockIdx.x * per;
    const long long u1 = u0 + per < units ? u0 + per : units;
    if (vec) {
        for (long long t = u0 + threadIdx.x; t < u1; t += blockDim.x) {
            const int r = (int)(t / nu), q = (int)(t - (long long)r * nu);
            const float4 v = *(const float4 *)(G + (size_t)r * row_stride + 4 * q);
            const long long base = (long long)r * Nmax + 4 * q;
            sum += (double)v.x + (double)v.y + (double)v.z + (double)v.w;
            if (v.x > vmax) { vmax = v.x; imax = base; }
            if (v.y > vmax) { vmax = v.y; imax = base + 1; }
            if (v.z > vmax) { vmax = v.z; imax = base + 2; }
            if (v.w > vmax) { vmax = v.w; imax = base + 3; }
        }
    } else {
        for (long long t = u0 + threadIdx.x; t < u1; t += blockDim.x) {
            const int r = (int)(t / Nmax), q = (int)(t - (long long)r * Nmax);
            const float v = G[(size_t)r * row_stride + q];
            sum += (double)v;
            if (v > vmax) { vmax = v; imax = t; }
        }
    }
    // block reduction: (max value, lowest index) and the sum
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float v2 = __shfl_xor_sync(0xffffffffu, vmax, o);
        const long long i2 = __shfl_xor_sync(0xffffffffu, imax, o);
        better(vmax, imax, v2, i2);
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
    }
    __shared__ float sv[32];
    __shared__ long long si[32];
    __shared__ double ss[32];
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) { sv[w] = vmax; si[w] = imax; ss[w] = sum; }
    __syncthreads();
    if (threadIdx.x == 0) {
        float v = 0.0f;
        long long i = -1;
        double s = 0.0;
        for (int k = 0; k < nw; ++k) { better(v, i, sv[k], si[k]); s += ss[k]; }
        PeakPart pp;
        pp.v = v; pp.i = i; pp.s = s;
        parts[(size_t)blockIdx.y * n_chunks + blockIdx.x] = pp;
    }
}

// Combines the chunks of one PRN in order; C/N0 and fine Doppler.
__global__ void peak_final_kernel(const float *__restrict__ P, int M, int Nmax,
                                  size_t row_stride, size_t prn_stride, double T,
                                  const float *__restrict__ fds, int n_chunks,
                                  const PeakPart *__restrict__ parts,
                                  sdrg_acq_result_t *__restrict__ res)
{
    if (threadIdx.x != 0) return;
    const float *G = P + (size_t)blockIdx.x * prn_stride;
    float v = 0.0f;
    long long i = -1;
    double s = 0.0;
    for (int k = 0; k < n_chunks; ++k) {
        const PeakPart pp = parts[(size_t)blockIdx.x * n_chunks + k];
        better(v, i, pp.v, pp.i);
        s += pp.s;
    }
    const long long cells = (long long)M * Nmax;
    const double pave = cells > 0 ? s / (double)cells : 0.0;
    sdrg_acq_result_t out;
    out.bin = i >= 0 ? (int)(i / Nmax) : -1;
    out.offset = i >= 0 ? (int)(i % Nmax) : -1;
    out.pmax = v;
    out.pave = pave;
    out.cn0 = pave > 0.0 ? (float)(10.0 * log10(((double)v - pave) / pave / T)) : 0.0f;
    out.fd = (i >= 0 && fds) ? fine_dop_dev(G, row_stride, fds, M, out.bin, out.offset) : 0.0;
    res[blockIdx.x] = out;
}

size_t peak_scratch_bytes(int n_prn)
{
    return (size_t)n_prn * kPeakChunksMax * sizeof(PeakPart);
}

// chunks per PRN: about 4 CTAs per SM in all, at least 64 K cells each
static int peak_chunks(int n_prn, long long cells)
{
    Device *dev = nullptr;
    const int sms = (ensure_device(&dev) == SDRG_OK && dev->sm_count > 0) ? dev->sm_count : 148;
    long long c = (4LL * sms + n_prn - 1) / n_prn;
    const long long cap = cells / 65536 > 0 ? cells / 65536 : 1;
    c = c < cap ? c : cap;
    c = c < kPeakChunksMax ? c : kPeakChunksMax;
    return (int)(c > 0 ? c : 1);
}

int launch_peaks(const float *P, int n_prn, int M_rows, int Nmax, size_t row_stride,
                 size_t prn_stride, double T, const float *fds_dev, sdrg_acq_result_t *res,
                 void *scratch, cudaStream_t st)
{
    const int nc = peak_chunks(n_prn, (long long)M_rows * Nmax);
    PeakPart *parts = (PeakPart *)scratch;
    peak_part_kernel<<<dim3((unsigned)nc, (unsigned)n_prn), kPeakThreads, 0, st>>>(
        P, M_rows, Nmax, row_stride, prn_stride, nc, parts);
    SDRG_CUDA(cudaGetLastError());
    peak_final_kernel<<<n_prn, 32, 0, st>>>(P, M_rows, Nmax, row_stride, prn_stride, T, fds_dev,
                                             nc, parts, res);
    SDRG_CUDA(cudaGetLastError());
    return SDRG_OK;
}

} // namespace sdrg

using namespace sdrg;

extern "C" {

float sdr_corr_max(const float *P, int N, int Nmax, int M, double T, int *ix)
{
    if (M <= 0 || Nmax <= 0 || N < Nmax) return 0.0f;
    cudaStream_t st;
    ThreadCtx &c = tctx();
    const size_t pb = (size_t)M * N * sizeof(float);
    c.host[2].pinned = true;
    // a failing step has recorded its error in the thread's last-error state
    if (ensure_device(nullptr) || thread_stream(&st) ||
        c.dev[3].reserve(pb + 256 + peak_scratch_bytes(1)) || c.host[2].reserve(pb + 256))
        return 0.0f;
    memcpy(c.host[2].ptr, P, pb);
    float *P_d = (float *)c.dev[3].ptr;
    sdrg_acq_result_t *r_d = (sdrg_acq_result_t *)((char *)c.dev[3].ptr + ((pb + 127) / 128) * 128);
    sdrg_acq_result_t *r_h = (sdrg_acq_result_t *)((char *)c.host[2].ptr + ((pb + 127) / 128) * 128);
    if (cudaMemcpyAsync(P_d, c.host[2].ptr, pb, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        launch_peaks(P_d, 1, M, Nmax, (size_t)N, 0, T, nullptr, r_d,
                     (char *)c.dev[3].ptr + ((pb + 127) / 128) * 128 + 128, st) ||
        cudaMemcpyAsync(r_h, r_d, sizeof(sdrg_acq_result_t), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cuda_error(cudaGetLastError(), "sdr_corr_max");
        return 0.0f;
    }
    if (r_h->bin >= 0) {   // the reference leaves ix untouched when no cell > 0
        ix[0] = r_h->bin;
        ix[1] = r_h->offset;
    }
    return r_h->cn0;
}

double sdr_fine_dop(const float *P, int N, const float *fds, int len_fds, const int *ix)
{
    if (ix[0] == 0 || ix[0] == len_fds - 1) return fds[ix[0]];
    const double x0 = fds[ix[0] - 1], x1 = fds[ix[0]], x2 = fds[ix[0] + 1];
    const double y0 = P[(size_t)(ix[0] - 1) * N + ix[1]];
    const double y1 = P[(size_t)ix[0] * N + ix[1]];
    const double y2 = P[(size_t)(ix[0] + 1) * N + ix[1]];
    const double d01 = (y1 - y0) / (x1 - x0), d12 = (y2 - y1) / (x2 - x1);
    const double cc = (d12 - d01) / (x2 - x0);
    const double b = d01 - cc * (x0 + x1);
    return -b / (2.0 * cc);
}

float *sdr_dop_bins(double T, float dop, float max_dop, int *len_fds)
{
    // src/sdr_func.c:757-769; the reference build (gcc -O3 -mfma) evaluates
    // dop - max_dop + i * step as one fused multiply-add
    const float step = (float)(0.5 / T);
    *len_fds = (int)(2.0 * max_dop / step) + 1;
    float *fds = (float *)malloc(sizeof(float) * (*len_fds > 0 ? *len_fds : 1));
    if (!fds) {
        set_error(SDRG_ERR_NOMEM, "sdr_dop_bins: malloc");
        *len_fds = 0;
        return nullptr;
    }
    for (int i = 0; i < *len_fds; ++i) fds[i] = fmaf((float)i, step, dop - max_dop);
    return fds;
}

} // extern "C"
