// sdrg_refine.cu - differentiable refinement of code delay, Doppler and
// carrier phase: per-block correlation sums with their derivatives, the
// vector-Jacobian product of the block correlations, and Gauss-Newton steps.
//
// No counterpart in the reference: its finest estimates are the three-bin
// Doppler quadratic of src/sdr_func.c:709-744 and the tracking loops of
// src/sdr_ch.c. Model for one signal (t = n / fs, n = sample index of the
// packed IF buffer):
//   psi(t) / 2 pi = fi t + fd (t - t_ref) + phi
//   u(t) = rate (t - t_ref) + rate_nom (t_ref - tau) - 1/2          (chips)
//   c(u) = chip[i] (1 - a) + chip[i+1] a,  i = floor(u) mod Lc,  a = frac(u)
// - the code linearly interpolated through the chip centres, so that d/dtau
// exists and the correlation with rectangular received chips peaks at the
// true delay. theta = (tau [s], fd [Hz], phi [cycles at t_ref]); `rate` is
// the code rate the model uses (the Gauss-Newton driver keeps it at
// rate_nom (1 + fd / fc)) and is not differentiated.
// Block k covers samples [ix0 + k Nb, ix0 + (k+1) Nb); t_ref is the middle of
// the span, (ix0 + K Nb / 2) / fs; t' is the time from the block centre.
// Per (signal, block) the sums kernel forms, in FP32,
//   C = sum x c e^{-j psi}   D = sum x dc e^{-j psi}   E = sum t' x c e^{-j psi}
//   Q = sum c^2   Qt = sum t' c^2   Qtt = sum t'^2 c^2   R = sum c dc
//   P = sum dc^2                       (dc = chip[i+1] - chip[i])
// from which dC/dtau = -rate_nom D, dC/dfd = -2 pi j (E + (t_k - t_ref) C)
// and dC/dphi = -2 pi j C. The carrier and code phases advance as exact
// 64-bit fixed-point recurrences (2^64 per carrier cycle, 2^44 per chip)
// from starting values computed in double per CTA, so they stay within
// 1e-9 cycle / chip of the double-precision model over a whole block.
// Backward passes recompute these sums from the IF samples rather than
// storing per-sample terms.
#include <cooperative_groups.h>
#include <cmath>
#include <vector>

#include "sdrg_internal.h"

namespace cg = cooperative_groups;

namespace sdrg {

constexpr int kRfThreads = 256;
constexpr int kRfW = 12;          // floats per (signal, block), mode 1
constexpr int kRfMaxLc = 65536;   // chips held in shared memory

constexpr int kCodeFrac = 44;                         // code phase fraction bits
constexpr long long kCodeMask = (1LL << kCodeFrac) - 1;
constexpr float kCodeScale = 5.684341886080802e-14f;  // 2^-44

// fraction of a cycle in [0, 1) -> 64-bit phase (2^64 per cycle)
__device__ inline unsigned long long cycles_to_u64(double f)
{
    const double v = ldexp(f, 64);
    return v >= 18446744073709551616.0 ? 0ull : __double2ull_rn(v);
}

struct RefineSigDev {
    const int8_t *chips;
    int Lc;
    double rate_nom, fi, fc;
};

struct RfArgs {
    const RefineSigDev *sigs;
    const double *theta;   // [n][3]
    const double *rate;    // [n]
    const uint8_t *buf;
    int ix0, Nb, K, S, iq;
    double fs;
    float *out;            // [n][K][W]
};

template <int MODE>
__global__ void __launch_bounds__(kRfThreads) refine_sums_kernel(RfArgs a)
{
    constexpr int W = MODE ? 11 : 2;     // accumulators
    constexpr int OW = MODE ? kRfW : 2;  // output stride
    extern __shared__ int8_t sh_chips[];
    __shared__ float red[kRfThreads / 32][W];
    __shared__ float tot[W];
    __shared__ unsigned long long sh_p, sh_dp;
    __shared__ long long sh_u, sh_du;

    const int sig = blockIdx.y;
    const int k = blockIdx.x / a.S, slice = blockIdx.x % a.S;
    const RefineSigDev S = a.sigs[sig];
    const int per = (a.Nb + a.S - 1) / a.S;
    const int n_lo = slice * per, n_hi = min(a.Nb, n_lo + per);   // offsets in the block
    const long long Lfx = (long long)S.Lc << kCodeFrac;

    for (int i = threadIdx.x; i < S.Lc; i += blockDim.x) sh_chips[i] = S.chips[i];
    if (threadIdx.x == 0) {
        const double tau = a.theta[3 * sig], fd = a.theta[3 * sig + 1], phi = a.theta[3 * sig + 2];
        const double rate = a.rate[sig];
        const double t_ref = (a.ix0 + 0.5 * a.K * (double)a.Nb) / a.fs;
        const double t0 = (double)((long long)a.ix0 + (long long)k * a.Nb + n_lo) / a.fs;
        double cyc = S.fi * t0 + fd * (t0 - t_ref) + phi;
        cyc -= floor(cyc);
        double stp = (S.fi + fd) / a.fs;
        stp -= floor(stp);
        sh_p = cycles_to_u64(cyc);
        sh_dp = cycles_to_u64(stp);
        double u = rate * (t0 - t_ref) + S.rate_nom * (t_ref - tau) - 0.5;
        u -= floor(u / S.Lc) * S.Lc;
        // the modulo keeps the chip index inside the table even for
        // non-finite theta or rate (garbage results, no stray reads)
        long long U = llrint(ldexp(u, kCodeFrac)) % Lfx;
        if (U < 0) U += Lfx;
        sh_u = U;
        long long du = llrint(ldexp(rate / a.fs, kCodeFrac));
        if (!(du >= 0 && du < Lfx / kRfThreads)) du = 0;
        sh_du = du;
    }
    __syncthreads();

    // carrier: 64-bit phase (2^64 per cycle); code: 64-bit chips with
    // kCodeFrac fractional bits - both exact integer recurrences, so the
    // phases drift from the double model by < 1e-9 cycle / chip per slice
    const unsigned long long dp_step = sh_dp * (unsigned long long)kRfThreads;
    unsigned long long ph = sh_p + sh_dp * (unsigned long long)threadIdx.x;
    const long long du = sh_du;
    const long long du_step = du * kRfThreads;           // < Lfx by the clamp above
    long long u = (sh_u + du * threadIdx.x) % Lfx;
    const float dt = (float)(1.0 / a.fs), half = 0.5f * (float)a.Nb;
    const uint8_t *x = a.buf + (long long)a.ix0 + (long long)k * a.Nb;

    float acc[W];
#pragma unroll
    for (int i = 0; i < W; ++i) acc[i] = 0.0f;

    for (int n = n_lo + threadIdx.x; n < n_hi; n += kRfThreads) {
        const uint8_t b = __ldg(x + n);
        const float xr = (float)((int)(int8_t)(uint8_t)(b << 4) >> 4);
        const float xi = a.iq ? (float)((int)(int8_t)b >> 4) : 0.0f;
        float sn, cs;
        // angle 2 pi ph / 2^64, from the top 32 bits
        sincospif((float)(uint32_t)(ph >> 32) * 4.656612873077393e-10f, &sn, &cs);
        const float yr = xr * cs + xi * sn, yi = xi * cs - xr * sn;  // x e^{-j psi}
        const int ci = (int)(u >> kCodeFrac);
        const int cj = ci + 1 == S.Lc ? 0 : ci + 1;
        const float fa = (float)(u & kCodeMask) * kCodeScale;
        const float c0 = (float)sh_chips[ci], c1 = (float)sh_chips[cj];
        const float dc = c1 - c0;
        const float c = fmaf(fa, dc, c0);
        acc[0] = fmaf(yr, c, acc[0]);
        acc[1] = fmaf(yi, c, acc[1]);
        if constexpr (MODE) {
            const float tp = ((float)n - half) * dt;
            const float cc = c * c, tcc = tp * cc;
            acc[2] = fmaf(yr, dc, acc[2]);
            acc[3] = fmaf(yi, dc, acc[3]);
            acc[4] = fmaf(tp * yr, c, acc[4]);
            acc[5] = fmaf(tp * yi, c, acc[5]);
            acc[6] += cc;
            acc[7] += tcc;
            acc[8] = fmaf(tp, tcc, acc[8]);
            acc[9] = fmaf(c, dc, acc[9]);
            acc[10] = fmaf(dc, dc, acc[10]);
        }
        ph += dp_step;
        u += du_step;
        if (u >= Lfx) u -= Lfx;
    }
    // warp, CTA, then cluster (the S slices of one block), in a fixed order
#pragma unroll
    for (int i = 0; i < W; ++i) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
#pragma unroll
        for (int i = 0; i < W; ++i) red[w][i] = acc[i];
    }
    __syncthreads();
    if (threadIdx.x < W) {
        float s = 0.0f;
#pragma unroll
        for (int j = 0; j < kRfThreads / 32; ++j) s += red[j][threadIdx.x];
        tot[threadIdx.x] = s;
    }
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    if (slice == 0 && threadIdx.x < OW) {
        float s = 0.0f;
        if (threadIdx.x < W) {
            for (int r = 0; r < a.S; ++r) s += cl.map_shared_rank(tot, r)[threadIdx.x];
        }
        a.out[((size_t)sig * a.K + k) * OW + threadIdx.x] = s;
    }
    cl.sync();   // peers keep their shared memory until rank 0 has read it
}

// ---- per-signal kernels (one thread per signal) ------------------------------

struct BlockTerms {
    double Cr, Ci, Dr, Di, Er, Ei, Q, Qt, Qtt, R, P;
};

// block k's sums, with E, Qt, Qtt moved to t - t_ref and D, R, P to d/dtau
__device__ inline BlockTerms block_terms(const float *s, int k, int K, int Nb, double fs,
                                         double rn)
{
    const double dt = (k + 0.5 - 0.5 * K) * Nb / fs;
    BlockTerms b;
    b.Cr = s[0]; b.Ci = s[1];
    b.Dr = -rn * s[2]; b.Di = -rn * s[3];
    b.Er = s[4] + dt * s[0]; b.Ei = s[5] + dt * s[1];
    b.Q = s[6];
    b.Qt = s[7] + dt * s[6];
    b.Qtt = s[8] + 2.0 * dt * s[7] + dt * dt * s[6];
    b.R = -rn * s[9];
    b.P = rn * rn * s[10];
    return b;
}

__global__ void refine_vjp_kernel(const RefineSigDev *sigs, int n, int K, int Nb, double fs,
                                  const float *sums, const float *g, double *grad)
{
    const int sig = blockIdx.x * blockDim.x + threadIdx.x;
    if (sig >= n) return;
    const double rn = sigs[sig].rate_nom, tp2 = 6.283185307179586;
    double gt = 0, gf = 0, gp = 0;
    for (int k = 0; k < K; ++k) {
        const BlockTerms b = block_terms(sums + ((size_t)sig * K + k) * kRfW, k, K, Nb, fs, rn);
        const double gr = g[((size_t)sig * K + k) * 2], gi = g[((size_t)sig * K + k) * 2 + 1];
        gt += gr * b.Dr + gi * b.Di;                 // Re(conj(g) dC/dtau)
        gf += tp2 * (gr * b.Ei - gi * b.Er);         // Re(conj(g) (-2 pi j) E)
        gp += tp2 * (gr * b.Ci - gi * b.Cr);         // Re(conj(g) (-2 pi j) C)
    }
    grad[3 * sig] = gt;
    grad[3 * sig + 1] = gf;
    grad[3 * sig + 2] = gp;
}

// Cholesky solve of a symmetric 3x3 system; false if not positive definite
__device__ inline bool chol3(const double H[3][3], const double b[3], double x[3])
{
    double L[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j <= i; ++j) {
            double s = H[i][j];
            for (int q = 0; q < j; ++q) s -= L[i][q] * L[j][q];
            if (i == j) {
                if (!(s > 0.0)) return false;
                L[i][i] = sqrt(s);
            } else {
                L[i][j] = s / L[j][j];
            }
        }
    }
    double y[3];
    for (int i = 0; i < 3; ++i) {
        double s = b[i];
        for (int q = 0; q < i; ++q) s -= L[i][q] * y[q];
        y[i] = s / L[i][i];
    }
    for (int i = 2; i >= 0; --i) {
        double s = y[i];
        for (int q = i + 1; q < 3; ++q) s -= L[q][i] * x[q];
        x[i] = s / L[i][i];
    }
    return true;
}

// One Gauss-Newton step per signal (models as in sdrg_refine_gn).
__global__ void refine_step_kernel(const RefineSigDev *sigs, int n, int K, int Nb, double fs,
                                   int model, const float *sums, double *theta, double *rate,
                                   double *info)
{
    const int sig = blockIdx.x * blockDim.x + threadIdx.x;
    if (sig >= n) return;
    const RefineSigDev S = sigs[sig];
    const double rn = S.rate_nom, tp2 = 6.283185307179586, fp2 = tp2 * tp2;
    const float *s0 = sums + (size_t)sig * K * kRfW;
    double zr = 0, zi = 0, wr = 0, wi = 0, power = 0, sQ = 0, sR = 0;
    for (int k = 0; k < K; ++k) {
        const float *s = s0 + k * kRfW;
        const double cr = s[0], ci = s[1];
        zr += cr * cr - ci * ci;
        zi += 2.0 * cr * ci;
        wr += cr;
        wi += ci;
        power += cr * cr + ci * ci;
        sQ += s[6];
        sR += -rn * s[9];
    }
    double alpha;
    if (model == 1) alpha = (wr == 0.0 && wi == 0.0) ? 0.0 : atan2(wi, wr);
    else alpha = (zr == 0.0 && zi == 0.0) ? 0.0 : 0.5 * atan2(zi, zr);
    double sa, ca;
    sincos(alpha, &sa, &ca);
    sa = -sa;                                         // e^{-j alpha}
    double sCr = 0;
    for (int k = 0; k < K; ++k) sCr += s0[k * kRfW] * ca - s0[k * kRfW + 1] * sa;
    const double a1 = sQ > 0.0 ? sCr / sQ : 0.0;
    double H[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, bv[3] = {0, 0, 0};
    for (int k = 0; k < K; ++k) {
        const BlockTerms t = block_terms(s0 + k * kRfW, k, K, Nb, fs, rn);
        if (!(t.Q > 0.0)) continue;
        const double Cr = t.Cr * ca - t.Ci * sa, Ci = t.Cr * sa + t.Ci * ca;
        const double Dr = t.Dr * ca - t.Di * sa, Di = t.Dr * sa + t.Di * ca;
        const double Er = t.Er * ca - t.Ei * sa, Ei = t.Er * sa + t.Ei * ca;
        if (model == 0) {
            const double Ar = Cr / t.Q, Ai = Ci / t.Q, A2 = Ar * Ar + Ai * Ai;
            H[0][0] += A2 * (t.P - t.R * t.R / t.Q);
            H[1][1] += fp2 * A2 * (t.Qtt - t.Qt * t.Qt / t.Q);
            bv[0] += Ar * Dr + Ai * Di - A2 * t.R;
            bv[1] += tp2 * (Ar * Ei - Ai * Er);
        } else {
            const double a = model == 1 ? a1 : Cr / t.Q, a2 = a * a;
            H[0][0] += a2 * (model == 1 ? t.P : t.P - t.R * t.R / t.Q);
            H[1][1] += fp2 * a2 * t.Qtt;
            H[1][2] += fp2 * a2 * t.Qt;
            H[2][2] += fp2 * a2 * t.Q;
            bv[0] += a * (Dr - a * t.R);
            bv[1] += tp2 * a * Ei;
            bv[2] += tp2 * a * Ci;
        }
    }
    if (model == 1 && sQ > 0.0) H[0][0] -= a1 * a1 * sR * sR / sQ;
    if (model == 0) H[2][2] = 1.0;
    H[2][1] = H[1][2];
    double x[3] = {0, 0, 0};
    const bool ok = chol3(H, bv, x);
    if (!ok) x[0] = x[1] = x[2] = 0.0;
    const double lim_t = 0.5 / rn, lim_f = 0.25 * fs / Nb;
    x[0] = fmin(fmax(x[0], -lim_t), lim_t);
    x[1] = fmin(fmax(x[1], -lim_f), lim_f);
    double *th = theta + 3 * sig;
    th[0] += x[0];
    th[1] += x[1];
    const double ph = th[2] + alpha / tp2 + x[2];
    th[2] = ph - floor(ph);
    rate[sig] = S.fc > 0.0 ? rn * (1.0 + th[1] / S.fc) : rn;
    if (info) {
        double *o = info + 5 * (size_t)sig;
        o[0] = power;
        o[1] = x[0] * rn;
        o[2] = x[1];
        o[3] = x[2];
        o[4] = ok ? 1.0 : 0.0;
    }
}

} // namespace sdrg

using namespace sdrg;

struct sdrg_refine_plan {
    int n = 0, Nb = 0, K = 0, S = 1, iq = 0, max_lc = 0;
    double fs = 0;
    RefineSigDev *sigs_dev = nullptr;
    int8_t *chips_dev = nullptr;
    float *sums_dev = nullptr;    // [n][K][12], Gauss-Newton scratch
};

extern "C" void sdrg_refine_plan_free(sdrg_refine_plan *p)
{
    if (!p) return;
    cudaFree(p->sigs_dev);
    cudaFree(p->chips_dev);
    cudaFree(p->sums_dev);
    delete p;
}

extern "C" sdrg_refine_plan *sdrg_refine_plan_new(const sdrg_refine_sig_t *sigs, int n_sig,
                                                  double fs, int iq, int Nb, int K)
{
    if (!sigs || n_sig <= 0 || n_sig > 65535 || Nb <= 0 || K <= 0 || !(fs > 0.0) ||
        (long long)Nb * K > (1LL << 30)) {
        set_error(SDRG_ERR_ARG, "sdrg_refine_plan_new: bad arguments");
        return nullptr;
    }
    Device *d = nullptr;
    if (ensure_device(&d)) return nullptr;
    size_t total = 0;
    int max_lc = 0;
    for (int i = 0; i < n_sig; ++i) {
        const sdrg_refine_sig_t &s = sigs[i];
        // the per-iteration code advance (256 samples) must stay below one
        // code period, with room for the carrier-aided rate change
        if (!s.chips || s.Lc < 2 || s.Lc > kRfMaxLc || !(s.rate > 0.0) ||
            s.rate * kRfThreads / fs * 1.01 >= s.Lc) {
            set_error(SDRG_ERR_ARG, "sdrg_refine_plan_new: bad signal %d", i);
            return nullptr;
        }
        total += (size_t)(s.Lc + 15) / 16 * 16;
        max_lc = s.Lc > max_lc ? s.Lc : max_lc;
    }
    sdrg_refine_plan *p = new sdrg_refine_plan();
    p->n = n_sig; p->Nb = Nb; p->K = K; p->iq = iq ? 1 : 0; p->fs = fs; p->max_lc = max_lc;
    // slices per block: enough CTAs for a few waves over the SMs, cluster <= 8
    int S = 1;
    while (S < 8 && (long long)n_sig * K * S < 4LL * d->sm_count && Nb / (2 * S) >= kRfThreads) S *= 2;
    p->S = S;
    std::vector<int8_t> chips(total, 0);
    std::vector<RefineSigDev> hs(n_sig);
    auto fail = [&](cudaError_t e, const char *what) {
        cuda_error(e, what);
        sdrg_refine_plan_free(p);
        return (sdrg_refine_plan *)nullptr;
    };
    cudaError_t e;
    if ((e = cudaMalloc(&p->chips_dev, total)) != cudaSuccess) return fail(e, "cudaMalloc chips");
    if ((e = cudaMalloc(&p->sigs_dev, sizeof(RefineSigDev) * n_sig)) != cudaSuccess)
        return fail(e, "cudaMalloc sigs");
    if ((e = cudaMalloc(&p->sums_dev, sizeof(float) * kRfW * n_sig * K)) != cudaSuccess)
        return fail(e, "cudaMalloc sums");
    size_t off = 0;
    for (int i = 0; i < n_sig; ++i) {
        std::copy(sigs[i].chips, sigs[i].chips + sigs[i].Lc, chips.begin() + off);
        hs[i] = RefineSigDev{p->chips_dev + off, sigs[i].Lc, sigs[i].rate, sigs[i].fi, sigs[i].fc};
        off += (size_t)(sigs[i].Lc + 15) / 16 * 16;
    }
    cudaStream_t st;
    if (thread_stream(&st)) { sdrg_refine_plan_free(p); return nullptr; }
    if ((e = cudaMemcpyAsync(p->chips_dev, chips.data(), total, cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(p->sigs_dev, hs.data(), sizeof(RefineSigDev) * n_sig,
                             cudaMemcpyHostToDevice, st)) ||
        (e = cudaStreamSynchronize(st)))
        return fail(e, "refine plan upload");
    return p;
}

static int refine_check_span(const sdrg_refine_plan *p, const uint8_t *if_dev, int len_if, int ix0)
{
    if (!p || !if_dev || ix0 < 0 || (long long)ix0 + (long long)p->K * p->Nb > len_if)
        return set_error(SDRG_ERR_ARG, "sdrg_refine: span [ix0, ix0 + K Nb) outside the buffer");
    return SDRG_OK;
}

template <int MODE>
static int launch_refine_sums(const sdrg_refine_plan *p, const RfArgs &a, cudaStream_t st)
{
    static bool attr_set = false;
    const size_t smem = (size_t)(p->max_lc + 15) / 16 * 16;
    if (!attr_set) {
        SDRG_CUDA(cudaFuncSetAttribute(refine_sums_kernel<MODE>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kRfMaxLc));
        attr_set = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(p->K * p->S), (unsigned)p->n);
    cfg.blockDim = dim3(kRfThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = p->S;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    SDRG_CUDA(cudaLaunchKernelEx(&cfg, refine_sums_kernel<MODE>, a));
    return SDRG_OK;
}

static int refine_sums(const sdrg_refine_plan *p, const uint8_t *if_dev, int ix0,
                       const double *theta, const double *rate, int mode, float *out,
                       cudaStream_t st)
{
    RfArgs a{p->sigs_dev, theta, rate, if_dev, ix0, p->Nb, p->K, p->S, p->iq, p->fs, out};
    return mode ? launch_refine_sums<1>(p, a, st) : launch_refine_sums<0>(p, a, st);
}

extern "C" int sdrg_refine_sums(sdrg_refine_plan *p, const uint8_t *if_dev, int len_if, int ix0,
                                const double *theta_dev, const double *rate_dev, int mode,
                                float *out_dev, void *stream)
{
    int e;
    if ((e = refine_check_span(p, if_dev, len_if, ix0))) return e;
    if (!theta_dev || !rate_dev || !out_dev || (mode != 0 && mode != 1))
        return set_error(SDRG_ERR_ARG, "sdrg_refine_sums: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;   // NULL: the legacy default stream
    return refine_sums(p, if_dev, ix0, theta_dev, rate_dev, mode, out_dev, st);
}

extern "C" int sdrg_refine_vjp(sdrg_refine_plan *p, const float *sums_dev, const float *g_dev,
                               double *grad_dev, void *stream)
{
    if (!p || !sums_dev || !g_dev || !grad_dev)
        return set_error(SDRG_ERR_ARG, "sdrg_refine_vjp: null argument");
    cudaStream_t st = (cudaStream_t)stream;   // NULL: the legacy default stream
    refine_vjp_kernel<<<(p->n + 127) / 128, 128, 0, st>>>(p->sigs_dev, p->n, p->K, p->Nb, p->fs,
                                                          sums_dev, g_dev, grad_dev);
    SDRG_CUDA(cudaGetLastError());
    return SDRG_OK;
}

extern "C" int sdrg_refine_gn(sdrg_refine_plan *p, const uint8_t *if_dev, int len_if, int ix0,
                              double *theta_dev, double *rate_dev, const int *models, int n_step,
                              double *info_dev, void *stream)
{
    int e;
    if ((e = refine_check_span(p, if_dev, len_if, ix0))) return e;
    if (!theta_dev || !rate_dev || n_step < 0 || (n_step && !models))
        return set_error(SDRG_ERR_ARG, "sdrg_refine_gn: bad arguments");
    for (int i = 0; i < n_step; ++i)
        if (models[i] < 0 || models[i] > 2)
            return set_error(SDRG_ERR_ARG, "sdrg_refine_gn: model %d", models[i]);
    cudaStream_t st = (cudaStream_t)stream;   // NULL: the legacy default stream
    for (int i = 0; i < n_step; ++i) {
        if ((e = refine_sums(p, if_dev, ix0, theta_dev, rate_dev, 1, p->sums_dev, st))) return e;
        refine_step_kernel<<<(p->n + 127) / 128, 128, 0, st>>>(
            p->sigs_dev, p->n, p->K, p->Nb, p->fs, models[i], p->sums_dev, theta_dev, rate_dev,
            info_dev ? info_dev + (size_t)i * 5 * p->n : nullptr);
        SDRG_CUDA(cudaGetLastError());
    }
    return SDRG_OK;
}

namespace sdrg {
// theta / rate from acquisition peaks: code phase 0 at sample ix_grid + offset
// (a sdr_search_code lag), fd = the fine Doppler, phase 0
__global__ void refine_from_peaks_kernel(const RefineSigDev *sigs, int n,
                                         const sdrg_acq_result_t *res, int ix_grid, double fs,
                                         double t_ref, double *theta, double *rate)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double t0 = (double)((long long)ix_grid + res[i].offset) / fs;
    const double fd = res[i].fd, fc = sigs[i].fc;
    const double sc = fc > 0.0 ? fd / fc : 0.0;
    theta[3 * i] = t0 + sc * (t0 - t_ref);      // carrier-aided code rate over t0 .. t_ref
    theta[3 * i + 1] = fd;
    theta[3 * i + 2] = 0.0;
    rate[i] = sigs[i].rate_nom * (1.0 + sc);
}
} // namespace sdrg

extern "C" int sdrg_refine_from_peaks(sdrg_refine_plan *p, const sdrg_acq_result_t *res_dev,
                                      int ix_grid, int ix0, double *theta_dev, double *rate_dev,
                                      void *stream)
{
    if (!p || !res_dev || !theta_dev || !rate_dev)
        return set_error(SDRG_ERR_ARG, "sdrg_refine_from_peaks: null argument");
    cudaStream_t st = (cudaStream_t)stream;   // NULL: the legacy default stream
    const double t_ref = (ix0 + 0.5 * p->K * (double)p->Nb) / p->fs;
    refine_from_peaks_kernel<<<(p->n + 127) / 128, 128, 0, st>>>(p->sigs_dev, p->n, res_dev,
                                                                 ix_grid, p->fs, t_ref,
                                                                 theta_dev, rate_dev);
    SDRG_CUDA(cudaGetLastError());
    return SDRG_OK;
}

extern "C" int sdrg_refine_plan_info(const sdrg_refine_plan *p, int *out4)
{
    if (!p || !out4) return set_error(SDRG_ERR_ARG, "sdrg_refine_plan_info: null argument");
    out4[0] = p->n;
    out4[1] = p->K;
    out4[2] = p->Nb;
    out4[3] = p->S;
    return SDRG_OK;
}
