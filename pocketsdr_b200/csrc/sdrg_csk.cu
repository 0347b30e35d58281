// sdrg_csk.cu - QZSS L6 CSK tracking correlators on the device.
//
// Reference: a tracking L6D / L6E channel (src/sdr_ch.c:705-720) mixes one
// code period (sdr_mix_carr), correlates it against the code bank of its
// fractional code phase with an FFT (sdr_corr_fft) and decodes the code-shift
// keying with CSK (src/sdr_ch.c:636-664): the correlation, rotated so that
// lag 0 sits at n = (int)(280 R) (R = N / (len_code / 2) samples per chip), is
// linearly interpolated (interp_corr, :626-632) at n + i R for the 511 chip
// shifts i = -255..255; the first strict maximum of |c| is the symbol
// (uint8)(255 - i % 256) and the channel's correlator outputs are
// interpolated at n + i R + pos[k]. Here every L6 channel of an epoch runs in
// one call: the mixing + FFT correlation of each job (the same kernels as the
// search, sdrg_search.cu) and one CSK-decode CTA per job.
//
// Bit-exactness of the decode: positions n + i R are formed with one fused
// multiply-add, as the reference build (gcc -O3 -mfma) compiles them; the
// interpolation and |c| are plain double / float operations in the reference's
// order (__dmul_rn / __dadd_rn, __fmul_rn / __fadd_rn, IEEE sqrtf).
#include <cstring>
#include <vector>

#include "sdrg_internal.h"

namespace sdrg {

constexpr int kCskThreads = 512;

struct CskArgs {
    const float2 *corr;       // [n_job][stride] FFT correlations
    size_t stride;
    const int *N;             // [n_job] samples per code period
    const int *len_code;      // [n_job]
    const int *npos;          // [n_job]
    const double *pos;        // [n_job][SDR_MAX_CORR]
    uint8_t *sym;             // [n_job]
    float2 *C;                // [n_job][SDR_MAX_CORR]
};

// C[t] of the rotated correlation: corr[N - n + t] for t < n, corr[t - n] after
__device__ __forceinline__ float2 rot(const float2 *corr, int N, int n, int t)
{
    return t < n ? __ldg(corr + (N - n + t)) : __ldg(corr + (t - n));
}

// interp_corr (src/sdr_ch.c:626-632): i = (int)x, weights in double, result
// rounded to float
__device__ __forceinline__ float2 interp(const float2 *corr, int N, int n, double x)
{
    const int i = (int)x;
    const double a1 = __dsub_rn(x, (double)i), a0 = __dsub_rn(1.0, a1);
    const float2 u = rot(corr, N, n, i), v = rot(corr, N, n, i + 1);
    return make_float2(
        (float)__dadd_rn(__dmul_rn(a0, (double)u.x), __dmul_rn(a1, (double)v.x)),
        (float)__dadd_rn(__dmul_rn(a0, (double)u.y), __dmul_rn(a1, (double)v.y)));
}

__global__ void __launch_bounds__(kCskThreads) csk_kernel(CskArgs a)
{
    __shared__ float sp[kCskThreads];
    __shared__ int si[kCskThreads];
    const int j = blockIdx.x;
    const int N = a.N[j];
    const float2 *corr = a.corr + (size_t)j * a.stride;
    const double R = (double)N / (double)(a.len_code[j] / 2);
    const int n = (int)(280.0 * R);
    // candidate shift i = threadIdx.x - 255 (511 of the 512 threads)
    const int i = (int)threadIdx.x - 255;
    float P = -1.0f;
    if (i <= 255) {
        const float2 c = interp(corr, N, n, __fma_rn((double)i, R, (double)n));
        P = sqrtf(__fadd_rn(__fmul_rn(c.x, c.x), __fmul_rn(c.y, c.y)));
    }
    sp[threadIdx.x] = P;
    si[threadIdx.x] = i;
    __syncthreads();
    // maximum, lowest shift on ties (the reference keeps the first strict max)
    for (int s = kCskThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            const float p2 = sp[threadIdx.x + s];
            const int i2 = si[threadIdx.x + s];
            if (p2 > sp[threadIdx.x] || (p2 == sp[threadIdx.x] && i2 < si[threadIdx.x])) {
                sp[threadIdx.x] = p2;
                si[threadIdx.x] = i2;
            }
        }
        __syncthreads();
    }
    // the reference starts from P_max = 0, ix = 0: no positive power keeps 0
    const int ix = sp[0] > 0.0f ? si[0] : 0;
    if (threadIdx.x == 0) a.sym[j] = (uint8_t)(255 - ix % 256);
    const double x0 = __fma_rn((double)ix, R, (double)n);
    for (int k = threadIdx.x; k < a.npos[j]; k += kCskThreads)
        a.C[(size_t)j * SDR_MAX_CORR + k] =
            interp(corr, N, n, __dadd_rn(x0, a.pos[(size_t)j * SDR_MAX_CORR + k]));
}

// Gathers n code DFTs of N complex values: row r of dst from src[r].
__global__ void gather_codes_kernel(const float2 *const *src, float2 *dst, int N, int n)
{
    const int r = blockIdx.y;
    if (r >= n) return;
    const float4 *s = (const float4 *)src[r];
    float4 *d = (float4 *)(dst + (size_t)r * N);
    const bool v = (N % 2 == 0) && (((uintptr_t)s & 15) == 0);
    if (v) {
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N / 2; i += gridDim.x * blockDim.x)
            d[i] = __ldg(s + i);
    } else {
        const float2 *s2 = src[r];
        float2 *d2 = dst + (size_t)r * N;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
            d2[i] = s2[i];
    }
}

static int launch_csk(const CskArgs &a, int n_job, cudaStream_t st)
{
    csk_kernel<<<n_job, kCskThreads, 0, st>>>(a);
    SDRG_CUDA(cudaGetLastError());
    return SDRG_OK;
}

// job tables on the device: N | len_code | npos (ints), pos (doubles)
struct CskTables {
    std::vector<int> ints;
    std::vector<double> pos;
};

static int csk_check(int N, int len_code, int npos, const double *pos, int j)
{
    if (N <= 0 || len_code < 2 || npos < 0 || npos > SDR_MAX_CORR || (npos && !pos))
        return set_error(SDRG_ERR_ARG, "L6 CSK job %d: bad N %d, len_code %d or taps %d", j, N,
                         len_code, npos);
    // every interpolation stays inside the 2 n rotated points
    const double R = (double)N / (len_code / 2);
    const int n = (int)(280 * R);
    if (n > N || n < 2)
        return set_error(SDRG_ERR_ARG, "L6 CSK job %d: N %d too short for 280 chips", j, N);
    double lo = n - 255 * R, hi = n + 255 * R + 1.0;
    for (int k = 0; k < npos; ++k) {
        const double a = n - 255 * R + pos[k], b = n + 255 * R + pos[k] + 1.0;
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    if (lo < 0.0 || hi >= 2.0 * n)
        return set_error(SDRG_ERR_ARG, "L6 CSK job %d: a tap lies outside +-280 chips", j);
    return SDRG_OK;
}

static int csk_upload(const CskTables &t, int n_job, void **dev, cudaStream_t st, CskArgs &a)
{
    const size_t ib = t.ints.size() * sizeof(int), db = t.pos.size() * sizeof(double);
    char *d = nullptr;
    SDRG_CUDA(stream_alloc((void **)&d, ib + db + 16, st));
    *dev = d;
    double *pos_d = (double *)(d + (ib + 15) / 16 * 16);
    if (cudaMemcpyAsync(d, t.ints.data(), ib, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(pos_d, t.pos.data(), db, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return cuda_error(cudaGetLastError(), "L6 CSK tables");
    const int *ip = (const int *)d;
    a.N = ip;
    a.len_code = ip + n_job;
    a.npos = ip + 2 * n_job;
    a.pos = pos_d;
    return SDRG_OK;
}

} // namespace sdrg

using namespace sdrg;

extern "C" {

int sdrg_csk_decode(const sdr_cpx_t *corr_dev, int n_job, int N, int len_code,
                    const double *pos, int npos, uint8_t *sym_dev, sdr_cpx_t *C_dev,
                    void *stream)
{
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    if (!corr_dev || !sym_dev || !C_dev || n_job <= 0)
        return set_error(SDRG_ERR_ARG, "sdrg_csk_decode: null argument or no jobs");
    if ((e = csk_check(N, len_code, npos, pos, 0))) return e;
    cudaStream_t st = (cudaStream_t)stream;
    CskTables t;
    t.ints.assign(3 * (size_t)n_job, 0);
    t.pos.assign((size_t)n_job * SDR_MAX_CORR, 0.0);
    for (int j = 0; j < n_job; ++j) {
        t.ints[j] = N;
        t.ints[n_job + j] = len_code;
        t.ints[2 * n_job + j] = npos;
        for (int k = 0; k < npos; ++k) t.pos[(size_t)j * SDR_MAX_CORR + k] = pos[k];
    }
    CskArgs a = {};
    a.corr = (const float2 *)corr_dev;
    a.stride = (size_t)N;
    a.sym = sym_dev;
    a.C = (float2 *)C_dev;
    void *td = nullptr;
    e = csk_upload(t, n_job, &td, st, a);
    if (!e) e = launch_csk(a, n_job, st);
    if (td) cudaFreeAsync(td, st);
    return e;
}

int sdrg_l6_csk_batch(const sdrg_l6_job_t *jobs, int n_job, const uint8_t *const *if_dev,
                      const int *len_if, uint8_t *sym_dev, sdr_cpx_t *C_dev,
                      sdr_cpx_t *corr_dev, void *stream)
{
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    if (!jobs || n_job <= 0 || !if_dev || !len_if || !sym_dev || !C_dev)
        return set_error(SDRG_ERR_ARG, "sdrg_l6_csk_batch: null argument or no jobs");
    cudaStream_t st = (cudaStream_t)stream;
    int Nmax = 0;
    size_t scr = 0;
    for (int j = 0; j < n_job; ++j) {
        const sdrg_l6_job_t &b = jobs[j];
        if (b.buf < 0 || !if_dev[b.buf] || b.ix < 0 || b.ix >= len_if[b.buf] ||
            b.N > len_if[b.buf] || !b.code_fft)
            return set_error(SDRG_ERR_ARG, "sdrg_l6_csk_batch: job %d: bad window or code", j);
        if ((e = csk_check(b.N, b.len_code, b.n, b.pos, j))) return e;
        const size_t s = corr_job_scratch(b.N);
        if (!s) return tctx().error ? tctx().error : SDRG_ERR_ARG;
        scr = s > scr ? s : scr;
        Nmax = b.N > Nmax ? b.N : Nmax;
    }
    // one batch (one code permutation, one forward and one consumer launch for
    // all jobs) when every job reads the same buffer with the same length and
    // that length splits over one cluster; job by job otherwise
    bool same = true;
    for (int j = 1; j < n_job; ++j)
        same = same && jobs[j].buf == jobs[0].buf && jobs[j].N == jobs[0].N;
    const FftPlan *pl0 = get_plan(jobs[0].N);
    const bool batched = same && pl0 && pl0->R <= 8;

    // staging: mixing words (5 per job; transposed for the batch) | CSK ints
    // (3 per job) | tap positions (SDR_MAX_CORR doubles per job), one upload
    const size_t mb = 5 * (size_t)n_job * sizeof(uint32_t), ib = 3 * (size_t)n_job * sizeof(int);
    const size_t pb = (size_t)n_job * SDR_MAX_CORR * sizeof(double);
    const size_t cpb = (size_t)n_job * sizeof(float2 *);
    const size_t o_i = (mb + 15) / 16 * 16, o_p = (o_i + ib + 15) / 16 * 16;
    const size_t o_c = (o_p + pb + 15) / 16 * 16;
    const size_t tab_bytes = (o_c + cpb + 255) / 256 * 256;
    const size_t cb = corr_dev ? 0 : ((size_t)n_job * Nmax * sizeof(float2) + 255) / 256 * 256;
    const size_t wb = batched ? 3 * (size_t)n_job * Nmax * sizeof(float2) : scr;
    const size_t dev_bytes = tab_bytes + cb + wb + 256;
    ThreadCtx &c = tctx();
    if (!c.l6_ev) {
        SDRG_CUDA(cudaEventCreateWithFlags(&c.l6_ev, cudaEventDisableTiming));
        SDRG_CUDA(cudaEventCreateWithFlags(&c.l6_done, cudaEventDisableTiming));
    }
    // the previous call's upload from the staging has landed, and this call's
    // device work follows the previous call's (both use this thread's scratch)
    SDRG_CUDA(cudaEventSynchronize(c.l6_ev));
    SDRG_CUDA(cudaStreamWaitEvent(st, c.l6_done, 0));
    c.l6_host.pinned = true;
    if (dev_bytes > c.l6_dev.size) SDRG_CUDA(cudaStreamSynchronize(st));
    if ((e = c.l6_host.reserve(tab_bytes)) || (e = c.l6_dev.reserve(dev_bytes))) return e;
    char *hb = (char *)c.l6_host.ptr;
    uint32_t *mix = (uint32_t *)hb;
    int *ints = (int *)(hb + o_i);
    double *posh = (double *)(hb + o_p);
    const float2 **codes_h = (const float2 **)(hb + o_c);
    memset(posh, 0, pb);
    for (int j = 0; j < n_job; ++j) {
        const sdrg_l6_job_t &b = jobs[j];
        ints[j] = b.N;
        ints[n_job + j] = b.len_code;
        ints[2 * n_job + j] = b.n;
        for (int k = 0; k < b.n; ++k) posh[(size_t)j * SDR_MAX_CORR + k] = b.pos[k];
        codes_h[j] = (const float2 *)b.code_fft;
        uint32_t w[5];
        corr_job_tables(len_if[b.buf], b.ix, b.N, b.fs, b.fc, b.phi, w);
        for (int k = 0; k < 5; ++k) {
            if (batched) mix[(size_t)k * n_job + j] = w[k];
            else mix[5 * (size_t)j + k] = w[k];
        }
    }
    char *db = (char *)c.l6_dev.ptr;
    SDRG_CUDA(cudaMemcpyAsync(db, hb, o_c + cpb, cudaMemcpyHostToDevice, st));
    SDRG_CUDA(cudaEventRecord(c.l6_ev, st));
    const uint32_t *mix_d = (const uint32_t *)db;
    float2 *corr = corr_dev ? (float2 *)corr_dev : (float2 *)(db + tab_bytes);
    char *work = db + tab_bytes + cb;
    e = SDRG_OK;
    if (batched) {
        float2 *codes = (float2 *)work;       // the jobs' code DFTs back to back
        const dim3 gg((unsigned)((Nmax / 2 + 255) / 256 < 64 ? (Nmax / 2 + 255) / 256 : 64),
                      (unsigned)n_job);
        gather_codes_kernel<<<gg, 256, 0, st>>>((const float2 *const *)(db + o_c), codes, Nmax,
                                                n_job);
        const cudaError_t ge = cudaGetLastError();
        if (ge != cudaSuccess) e = cuda_error(ge, "sdrg_l6_csk_batch codes");
        if (!e)
            e = corr_jobs_device(if_dev[jobs[0].buf], len_if[jobs[0].buf], mix_d, n_job, Nmax,
                                 codes, corr, codes + (size_t)n_job * Nmax, st);
    } else {
        // each job: mixing + FFT correlation (src/sdr_ch.c:710-713)
        for (int j = 0; j < n_job && !e; ++j) {
            const sdrg_l6_job_t &b = jobs[j];
            e = corr_job_device(if_dev[b.buf], len_if[b.buf], mix_d + 5 * j, b.N,
                                (const float2 *)b.code_fft, corr + (size_t)j * Nmax, work, st);
        }
    }
    if (!e) {
        CskArgs a = {};
        a.corr = corr;
        a.stride = (size_t)Nmax;
        a.N = (const int *)(db + o_i);
        a.len_code = a.N + n_job;
        a.npos = a.N + 2 * n_job;
        a.pos = (const double *)(db + o_p);
        a.sym = sym_dev;
        a.C = (float2 *)C_dev;
        e = launch_csk(a, n_job, st);
    }
    cudaError_t re = cudaEventRecord(c.l6_done, st);
    if (!e && re != cudaSuccess) e = cuda_error(re, "sdrg_l6_csk_batch");
    return e;
}

} // extern "C"
