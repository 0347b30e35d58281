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
    SDRG_CUDA(cudaMallocAsync((void **)&d, ib + db + 16, st));
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
    // correlations: the caller's buffer ([n_job][Nmax]) or scratch
    CskTables t;
    t.ints.assign(3 * (size_t)n_job, 0);
    t.pos.assign((size_t)n_job * SDR_MAX_CORR, 0.0);
    std::vector<uint32_t> mix(5 * (size_t)n_job);
    for (int j = 0; j < n_job; ++j) {
        const sdrg_l6_job_t &b = jobs[j];
        t.ints[j] = b.N;
        t.ints[n_job + j] = b.len_code;
        t.ints[2 * n_job + j] = b.n;
        for (int k = 0; k < b.n; ++k) t.pos[(size_t)j * SDR_MAX_CORR + k] = b.pos[k];
        corr_job_tables(len_if[b.buf], b.ix, b.N, b.fs, b.fc, b.phi, mix.data() + 5 * j);
    }
    float2 *corr = (float2 *)corr_dev;
    char *work = nullptr;
    const size_t cb = corr ? 0 : (size_t)n_job * Nmax * sizeof(float2);
    const size_t mb = mix.size() * sizeof(uint32_t);
    if (cudaMallocAsync((void **)&work, cb + mb + scr + 512, st) != cudaSuccess)
        return cuda_error(cudaGetLastError(), "sdrg_l6_csk_batch scratch");
    if (!corr) corr = (float2 *)work;
    uint32_t *mix_d = (uint32_t *)(work + (cb + 255) / 256 * 256);
    void *scratch = (char *)mix_d + (mb + 255) / 256 * 256;
    e = SDRG_OK;
    if (cudaMemcpyAsync(mix_d, mix.data(), mb, cudaMemcpyHostToDevice, st) != cudaSuccess)
        e = cuda_error(cudaGetLastError(), "sdrg_l6_csk_batch tables");
    // each job: mixing + FFT correlation (src/sdr_ch.c:710-713)
    for (int j = 0; j < n_job && !e; ++j) {
        const sdrg_l6_job_t &b = jobs[j];
        e = corr_job_device(if_dev[b.buf], len_if[b.buf], mix_d + 5 * j, b.N,
                            (const float2 *)b.code_fft, corr + (size_t)j * Nmax, scratch, st);
    }
    CskArgs a = {};
    a.corr = corr;
    a.stride = (size_t)Nmax;
    a.sym = sym_dev;
    a.C = (float2 *)C_dev;
    void *td = nullptr;
    if (!e) e = csk_upload(t, n_job, &td, st, a);
    if (!e) e = launch_csk(a, n_job, st);
    if (td) cudaFreeAsync(td, st);
    cudaFreeAsync(work, st);
    return e;
}

} // extern "C"
