// sdrg_search.cu - FFT correlator and parallel-code-phase search on sm_100a.
//
// Reference path: src/sdr_func.c:664-687 (sdr_search_code), :1088-1113
// (sdr_corr_fft, sdr_corr_fft_cpx). A length-L correlation is computed as
//   X   = FFT_L(mix(IF) * CSCALE)                         (fwd_kernel)
//   Z   = X * code_fft * (1/L^2)
//   y   = IFFT_L(Z);  P += |y|^2   or  corr = y           (cons_kernel)
// with L = R*M split over R CTAs:
//   forward  (decimation in time):  F_r = FFT_M(x[R m + r]),  r < R, one
//            independent CTA each;
//   inverse  (decimation in frequency): CTA c of an R-CTA cluster produces
//            y[R m + c] = IFFT_M(w_c)[m] with
//            w_c[k] = e^{+2 pi i c k / L} sum_j Z[k + j M] e^{+2 pi i c j / R}
//            and Z[k + j M] = code[k + j M] * sum_r e^{-2 pi i r (k + j M)/L} F_r[k].
// Each cluster CTA forms w_0..w_{R-1} for 1/R of the k range and stores them
// into the owners' shared memory (distributed shared memory), so X and the
// code are read from L2/HBM exactly once per (PRN, bin, sum).
// The forward transform of a (bin, sum) block does not depend on the PRN: it
// is computed once per signal group and reused by every PRN's consumer task.
#include <cooperative_groups.h>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "sdrg_internal.h"

namespace cg = cooperative_groups;

namespace sdrg {

// ---------------------------------------------------------------------------
// mixing of one packed sample (bit-exact with the reference's 64K table,
// src/sdr_func.c:113-134 and :772-807)
// ---------------------------------------------------------------------------
__device__ __forceinline__ char2 mix_one(uint8_t byte, uint32_t phase,
                                         const char2 *ctab)
{
    const int I = (int)(int8_t)(uint8_t)(byte << 4) >> 4;
    const int Q = (int)(int8_t)byte >> 4;
    const char2 c = ctab[phase >> 24];
    char2 o;
    o.x = (signed char)(I * c.x - Q * c.y);
    o.y = (signed char)(I * c.y + Q * c.x);
    return o;
}

// ---------------------------------------------------------------------------
// forward kernel
// ---------------------------------------------------------------------------
struct FwdArgs {
    FftPlanK pl;
    const float2 *tw;      // per-pass twiddles (global)
    const char2 *ctab;     // carrier table (global)
    int R;                 // split factor
    int n_bin, n_sum;
    float cscale;
    // mode 0: packed IF + mixing
    const uint8_t *buf;    // circular IF buffer
    int buf_len;
    const int *ix;         // [n_sum] first sample of each sum
    const uint32_t *phstep;   // [n_bin] phase step per sample
    const uint32_t *ph0a;     // [n_bin] phase at sample 0
    const uint32_t *ph0b;     // [n_bin * n_sum] phase restart after the wrap
    const int *nsplit;        // [n_sum] samples before the buffer wrap
    // mode 1: already mixed samples (sdr_cpx16_t), one block
    const char2 *iq;
    float2 *X;             // out: [n_bin][n_sum][R][M]
    int ix_per_bin;        // 1: ix / nsplit indexed by bin (independent windows per bin)
};

struct LoadIF {
    const uint8_t *buf;
    int len, ix0, nsplit, R, r;
    uint32_t step, p0a, p0b;
    const char2 *ctab;
    float cs;
    __device__ __forceinline__ float2 operator()(int m) const
    {
        const int n = R * m + r;
        int pos = ix0 + n;
        if (pos >= len) pos -= len;
        const uint32_t ph = n < nsplit ? p0a + step * (uint32_t)n
                                       : p0b + step * (uint32_t)(n - nsplit);
        const char2 v = mix_one(__ldg(buf + pos), ph, ctab);
        return make_float2(__fmul_rn((float)v.x, cs), __fmul_rn((float)v.y, cs));
    }
};

struct LoadIQ {
    const char2 *iq;
    int R, r;
    float cs;
    __device__ __forceinline__ float2 operator()(int m) const
    {
        const char2 v = iq[R * m + r];
        return make_float2(__fmul_rn((float)v.x, cs), __fmul_rn((float)v.y, cs));
    }
};

// One forward block: (bin, sum, r) = blk of the group described by a; sm
// (M points), tw (the plan's twiddles) and ctab (256 carrier values) in
// shared memory. Ends after its spectrum is stored.
template <int MODE, int SP>
__device__ __forceinline__ void fwd_block(const FwdArgs &a, int blk, float2 *sm, float2 *tw,
                                          char2 *ctab)
{
    const int r = blk % a.R;
    const int bs = blk / a.R;            // b * n_sum + s
    const int s = bs % a.n_sum, b = bs / a.n_sum;

    load_twiddles(tw, a.tw, a.pl.twtot);
    if (MODE == 0) {
        for (int i = threadIdx.x; i < 256; i += blockDim.x) ctab[i] = a.ctab[i];
    }
    __syncthreads();

    if (MODE == 0) {
        const int w = a.ix_per_bin ? b : s;
        LoadIF ld{a.buf, a.buf_len, a.ix[w], a.nsplit[w], a.R, r, a.phstep[b],
                  a.ph0a[b], a.ph0b[bs], ctab, a.cscale};
        if constexpr (SP == 1) fft_forward_static<Plan24000>(sm, tw, ld);
        else fft_forward(sm, tw, a.pl, ld);
    } else {
        LoadIQ ld{a.iq, a.R, r, a.cscale};
        if constexpr (SP == 1) fft_forward_static<Plan24000>(sm, tw, ld);
        else fft_forward(sm, tw, a.pl, ld);
    }
    // store F_r (digit-reversed order) contiguously
    float2 *dst = a.X + ((size_t)bs * a.R + r) * a.pl.M;
    const int M = a.pl.M;
    if ((M & 1) == 0) {
        float4 *d4 = (float4 *)dst;
        const float4 *s4 = (const float4 *)sm;
        for (int i = threadIdx.x; i < M / 2; i += blockDim.x) d4[i] = s4[i];
    } else {
        for (int i = threadIdx.x; i < M; i += blockDim.x) dst[i] = sm[i];
    }
}

template <int MODE, int SP>
__global__ void __launch_bounds__(512, 1) fwd_kernel(FwdArgs a)
{
    extern __shared__ float2 smem[];
    float2 *tw = smem + a.pl.M;
    fwd_block<MODE, SP>(a, blockIdx.x, smem, tw, (char2 *)(tw + a.pl.twtot));
}

// Forward blocks of every signal group of a plan in one launch (groups on the
// compile-time 24 000-point plan): block i belongs to the group g with
// blk0[g] <= i < blk0[g + 1].
constexpr int kMaxWorkGroups = 8;
struct FwdMulti {
    int n_group;
    int blk0[kMaxWorkGroups + 1];
    FwdArgs g[kMaxWorkGroups];
};

__global__ void __launch_bounds__(512, 1) fwd_multi_kernel(FwdMulti m)
{
    extern __shared__ float2 smem[];
    int g = 0;
    while (g + 1 < m.n_group && (int)blockIdx.x >= m.blk0[g + 1]) ++g;
    const FwdArgs &a = m.g[g];
    float2 *tw = smem + Plan24000::M;
    fwd_block<0, 1>(a, (int)blockIdx.x - m.blk0[g], smem, tw, (char2 *)(tw + Plan24000::TWTOT));
}

// In-place split combine of a group's forward sub-spectra: for every (bin,
// sum) bs and position q, X[bs][r][q] = F_r[q] (r < R) becomes
// X[bs][j][q] = X(k(q) + j M) (j < R), the spectrum the consumers multiply by
// each PRN's code. The same arithmetic as the consumer's own combine
// (split_combine_fwd), done once per bin and sum instead of once per PRN.
template <int R>
__global__ void __launch_bounds__(256) xcomb_kernel(float2 *X, const float2 *__restrict__ split,
                                                    int M)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= M) return;
    float2 *x = X + (size_t)blockIdx.y * R * M + q;
    float2 g[R];
#pragma unroll
    for (int r = 0; r < R; ++r) g[r] = x[(size_t)r * M];
    split_combine_fwd<R>(g, __ldg(split + q));
#pragma unroll
    for (int j = 0; j < R; ++j) x[(size_t)j * M] = g[j];
}

// ---------------------------------------------------------------------------
// consumer kernel
// ---------------------------------------------------------------------------
struct ConsArgs {
    FftPlanK pl;
    const float2 *tw;       // per-pass twiddles
    const float2 *split;    // [M] exp(+2 pi i k(q) / L)
    const float2 *X;        // [n_bin][n_sum][R][M]
    const float2 *code;     // [n_prn][R][M] permuted conj code DFT
    int n_prn, n_bin, n_sum;
    int prn0;               // first PRN of this launch (tasks are bin-major)
    float scale;            // 1/L^2 as the reference computes it in float
    int Nmax;               // grid columns kept
    size_t prn_stride;      // P stride between PRNs (elements)
    size_t bin_stride;      // P stride between bins (elements)
    int accumulate;         // 1: P += |y|^2 from the first sum on (IN/OUT P)
    int code_per_bin;       // 1: bin b correlates with code b (independent jobs)
    float *P;               // mode 0
    float2 *Y;              // mode 1: [n_bin][L]
    // mode 0 with a split (R > 1) and several sums: the power of output
    // n = R m + c is summed in Q[task][c][m] (Mq = ceil(Nmax / R) per row),
    // where each CTA's accesses are consecutive; the last sum writes P
    float *Q;               // or null: every sum reads and writes P
    int Mq;
    int q_by_sm;            // 1: Q row of the SM the CTA runs on (one consumer CTA
                            // per SM; the row is the CTA's alone for the task's
                            // sums), 0: Q row of the task and CTA
    int *stage_err;         // staged splits: error word (a bulk-copy wait ran out)
    int x_comb;             // 1: X holds the combined spectrum, X[bs][j][q] = X(k(q) + j M)
                            // (xcomb_kernel ran); 0: the sub-spectra F_r
};

// Power store of one sum. kDirect: P = (add ? P : 0) + |y|^2. With the
// accumulator Q: kQFirst Q = (add ? P : 0) + |y|^2, kQMid Q += |y|^2,
// kQLast P = Q + |y|^2 - the same additions in the same order.
enum { kDirect = 0, kQFirst = 1, kQMid = 2, kQLast = 3 };

template <int R>
struct StorePower {
    typedef float Old;
    float *row;       // P for this (prn, bin)
    float *q;         // Q row of this (task, c), or null
    int c, Nmax;
    bool add;
    int mode;
    __device__ __forceinline__ float pre(int m) const
    {
        const int n = R * m + c;
        if (n >= Nmax) return 0.0f;
        if (mode == kQMid || mode == kQLast) return q[m];
        return add ? row[n] : 0.0f;
    }
    __device__ __forceinline__ void operator()(int m, float2 y, float old) const
    {
        const int n = R * m + c;
        if (n < Nmax) {
            const float pw = y.x * y.x + y.y * y.y;
            const float v = (add || mode >= kQMid) ? old + pw : pw;
            if (mode == kQFirst || mode == kQMid) q[m] = v;
            else row[n] = v;
        }
    }
};

template <int R>
struct StoreComplex {
    typedef int Old;
    float2 *row;
    int c;
    __device__ __forceinline__ int pre(int) const { return 0; }
    __device__ __forceinline__ void operator()(int m, float2 y, int) const { row[R * m + c] = y; }
};

// Hint to bring [p, p + n) into L2 (cp.async.bulk.prefetch.L2): only the
// 16-byte-aligned interior of the range is named, so nothing outside it is
// touched; there is no completion to wait for.
__device__ __forceinline__ void prefetch_l2(const float2 *p, int n)
{
    uintptr_t a0 = ((uintptr_t)p + 15) & ~(uintptr_t)15;
    const uintptr_t e = ((uintptr_t)(p + n)) & ~(uintptr_t)15;
    while (a0 < e) {
        const uint32_t sz = (uint32_t)min((uintptr_t)32768, e - a0);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a0), "r"(sz) : "memory");
        a0 += sz;
    }
}

// Bound of every wait of a kernel on an mbarrier (bulk copies into shared
// memory, partner CTAs; never reached in normal operation). Past it the CTA
// sets the launch's error word, which the synchronous entry points report and
// clear, and goes on.
constexpr long long kBulkWaitCycles = 4000000000LL;     // about 2 s at 1.97 GHz

// The compile-time plan of a consumer instantiation: SP 1 the 24 000-point
// plan, SP 2 the 12 000-point one (two CTAs per SM), SP 0 none (runtime plan).
template <int SP> struct PlanOf { using P = Plan24000; };
template <> struct PlanOf<2> { using P = Plan12000; };

// ---- synchronisation of the CTAs that share a task --------------------------
// A Sync type is a barrier over the CTAs of a task, called whole, or split
// into arrive() (by every thread, at the same point) and wait() (by every
// thread, anywhere before it touches what the barrier protects).
struct CtaSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
    __device__ __forceinline__ void arrive() const { __syncthreads(); }
    __device__ __forceinline__ void wait() const {}
};
struct ClusterSync {
    __device__ __forceinline__ void operator()() const { cg::this_cluster().sync(); }
    // split cluster barrier; the unaligned forms, since threads reach wait()
    // at different points of the combine loop
    __device__ __forceinline__ void arrive() const
    {
        asm volatile("barrier.cluster.arrive.release;" ::: "memory");
    }
    __device__ __forceinline__ void wait() const
    {
        asm volatile("barrier.cluster.wait.acquire;" ::: "memory");
    }
};

// The two CTAs of a 2-way task inside a larger cluster (the work list's
// narrow tasks in 8-CTA clusters), without holding up the other pairs. Each
// CTA has two mbarriers (one expected arrival each), used by alternate
// barrier calls; a call arrives remotely on the partner's barrier of that
// turn (release at cluster scope, after the CTA's own barrier, so the CTA's
// writes into the partner's shared memory and its reads of its own come
// before) and passes when its own barrier of that turn has completed the
// phase (acquire). With two barriers in turn, a barrier cannot complete a
// second phase before its owner has seen the first: the partner's next
// arrival on it needs the owner's arrival of the turn in between. Thread 0
// keeps the turn and the parities in shared memory (state[0]: turn,
// state[1 + turn]: parity).
struct PairSync {
    uint32_t bar;        // this CTA's two mbarriers (shared::cta address of the first)
    uint32_t remote;     // the partner's two mbarriers (shared::cluster address)
    uint32_t *state;     // turn and parities (shared, thread 0)
    int *err;            // error word: a wait reached kBulkWaitCycles
    __device__ __forceinline__ void operator()() const
    {
        __syncthreads();
        if (threadIdx.x == 0) {
            const uint32_t turn = state[0], par = state[1 + turn];
            asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];"
                         ::"r"(remote + 8u * turn) : "memory");
            const long long t0 = clock64();
            for (;;) {
                if (clock64() - t0 >= kBulkWaitCycles) { atomicOr(err, 1); break; }
                uint32_t done;
                asm volatile("{\n\t.reg .pred p;\n\t"
                             "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
                             "selp.u32 %0, 1, 0, p;\n\t}"
                             : "=r"(done) : "r"(bar + 8u * turn), "r"(par) : "memory");
                if (done) break;
            }
            state[1 + turn] = par ^ 1u;
            state[0] = turn ^ 1u;
        }
        __syncthreads();
    }
    __device__ __forceinline__ void arrive() const { (*this)(); }
    __device__ __forceinline__ void wait() const {}
};

// One position of the consumer's combine: g[r] = the sub-spectra F_r(k)
// (x_comb 0) or the spectrum X(k + r M) (x_comb 1), cs[j] the code at
// k + j M, t = exp(+2 pi i k / L); leaves g[j] = the input of CTA j's
// inverse transform at this position.
template <int R>
__device__ __forceinline__ void combine_point(float2 *g, const float2 *cs, float2 t, int x_comb,
                                              float scale)
{
    if (!x_comb) split_combine_fwd<R>(g, t);   // X[k + jM]
#pragma unroll
    for (int j = 0; j < R; ++j) {
        const float2 z = cmul(g[j], cs[j]);
        g[j] = make_float2(z.x * scale, z.y * scale);
    }
    Dft<R, 1>::run(g);                         // sum_j Z e^{+2 pi i c j/R}
    float2 w = t;
#pragma unroll
    for (int j = 1; j < R; ++j) {
        g[j] = cmul(g[j], w);
        if (j + 1 < R) w = cmul(w, t);
    }
}

// The sums of one consumer task (PRN prn, bin b; this CTA's share c of its
// R-way split): per sum, combine + code product into the split's shared
// memory (dst[j]: CTA j of the task), barrier, inverse transform and power
// (or complex) store. ns_run iterations, each with its two barriers
// (sync(): over the CTA, the cluster or the pair of CTAs that share the task),
// so that CTAs whose tasks have fewer sums - or none (active false) - keep
// step with the others; the twiddles are in tw.
template <int R, int MODE, int SP, class Sync>
__device__ __forceinline__ void cons_task(const ConsArgs &a, float2 *sm, const float2 *tw,
                                          float2 *const *dst, int c, int task, int prn, int b,
                                          int ns_run, bool active, const Sync &sync)
{
    const int M = SP ? PlanOf<SP>::P::M : a.pl.M;   // SP: compile-time plan
    const int Mc = (M + R - 1) / R;
    const int q0 = c * Mc, q1 = min(M, q0 + Mc);
    const float2 *code = a.code + (size_t)(a.code_per_bin ? b : prn) * R * M;
    for (int s = 0; s < ns_run; ++s) {
        // all CTAs of the cluster are done with their shared memory: arrive
        // here, wait after this thread's first global loads of the combine
        // are in flight (before its first store into shared memory)
        sync.arrive();
        bool waited = false;
        const bool run = active && s < a.n_sum;
        const float2 *Xs = a.X + ((size_t)b * a.n_sum + s) * R * M;
        // U positions per iteration: all their global loads are issued
        // before any arithmetic or (remote) shared-memory store (more loads
        // in flight per thread: 1 CTA of 16 warps per SM). At R = 8 one
        // position already issues 17 loads, which the L2 prefetch serves:
        // a second one only fills the load queue (measured 2 % slower).
        constexpr int U = R <= 2 ? 4 : (R <= 6 ? 2 : 1);
        const int qstep = U * blockDim.x;
        for (int q = q0 + threadIdx.x; run && q < q1; q += qstep) {
            float2 xs[U][R], cs[U][R], ts[U];
            bool ok[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int qq = q + u * blockDim.x;
                ok[u] = qq < q1;
                const int ql = ok[u] ? qq : q;
                ts[u] = R > 1 ? __ldg(a.split + ql) : make_float2(1.0f, 0.0f);
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    xs[u][r] = __ldg(Xs + (size_t)r * M + ql);
                    cs[u][r] = __ldg(code + (size_t)r * M + ql);
                }
            }
            if (!waited) {
                sync.wait();
                waited = true;
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (!ok[u]) continue;
                const int qq = q + u * blockDim.x;
                float2 *g = xs[u];
                if constexpr (R == 1) {
                    const float2 z = cmul(g[0], cs[u][0]);
                    dst[0][qq] = make_float2(z.x * a.scale, z.y * a.scale);
                } else {
                    combine_point<R>(g, cs[u], ts[u], a.x_comb, a.scale);
#pragma unroll
                    for (int j = 0; j < R; ++j) dst[j][qq] = g[j];
                }
            }
        }
        if (!waited) sync.wait();
        sync();
        if (!run) continue;
        // the next sum's spectra head for L2 during this sum's transform
        if (s + 1 < a.n_sum && threadIdx.x < R && q1 > q0)
            prefetch_l2(Xs + (size_t)R * M + (size_t)threadIdx.x * M + q0, q1 - q0);

        if (MODE == 0) {
            float *row = a.P + (size_t)(prn) * a.prn_stride + (size_t)b * a.bin_stride;
            const bool useq = R > 1 && a.Q && a.n_sum > 1;
            const int mode = !useq ? kDirect
                : (s == 0 ? kQFirst : (s == a.n_sum - 1 ? kQLast : kQMid));
            float *qrow = nullptr;
            if (useq) {
                uint32_t sm = 0;
                if (a.q_by_sm) asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
                qrow = a.Q + (a.q_by_sm ? (size_t)sm : (size_t)task * R + c) * a.Mq;
            }
            StorePower<R> st{row, qrow, c, a.Nmax, mode == kDirect ? (a.accumulate || s > 0)
                                                                  : (a.accumulate != 0), mode};
            if constexpr (SP != 0) fft_inverse_static<typename PlanOf<SP>::P>(sm, tw, st);
            else fft_inverse(sm, tw, a.pl, st);
        } else {
            float2 *row = a.Y + (size_t)b * (size_t)R * M;
            StoreComplex<R> st{row, c};
            if constexpr (SP != 0) fft_inverse_static<typename PlanOf<SP>::P>(sm, tw, st);
            else fft_inverse(sm, tw, a.pl, st);
        }
    }
}

template <int R, int MODE, int SP>
__global__ void __launch_bounds__(512, 1) cons_kernel(ConsArgs a)
{
    extern __shared__ float2 smem[];
    float2 *sm = smem;
    float2 *tw = smem + a.pl.M;
    const int M = SP ? PlanOf<SP>::P::M : a.pl.M;   // SP: compile-time plan
    const int c = (R > 1) ? (int)(blockIdx.x % R) : 0;
    // bin-major tasks: the PRNs of one Doppler bin run side by side, so the
    // bin's forward spectra are fetched from HBM once and then hit in L2
    const int task = blockIdx.x / R;
    const int n_prn_l = a.n_prn - a.prn0;
    const int prn = a.prn0 + task % n_prn_l;
    const int b = task / n_prn_l;
    if (b >= a.n_bin) return;     // uniform across the cluster
    const int Mc = (M + R - 1) / R;
    const int q0 = c * Mc, q1 = min(M, q0 + Mc);
    const float2 *code = a.code + (size_t)(a.code_per_bin ? b : prn) * R * M;
    // this CTA's ranges of the first sum's spectra and of the code head for
    // L2 while the twiddles load
    if (threadIdx.x < R && q1 > q0 && a.n_sum > 0) {
        prefetch_l2(a.X + (size_t)b * a.n_sum * R * M + (size_t)threadIdx.x * M + q0, q1 - q0);
        prefetch_l2(code + (size_t)threadIdx.x * M + q0, q1 - q0);
    }

    if constexpr (SP != 0) load_twiddles_static<typename PlanOf<SP>::P>(tw, a.tw);
    else load_twiddles(tw, a.tw, a.pl.twtot);

    float2 *dst[R];
    if constexpr (R > 1) {
        cg::cluster_group cl = cg::this_cluster();
#pragma unroll
        for (int j = 0; j < R; ++j) dst[j] = cl.map_shared_rank(sm, j);
    } else {
        dst[0] = sm;
    }
    if constexpr (R > 1) cons_task<R, MODE, SP>(a, sm, tw, dst, c, task, prn, b, a.n_sum, true, ClusterSync{});
    else cons_task<R, MODE, SP>(a, sm, tw, dst, c, task, prn, b, a.n_sum, true, CtaSync{});
    // keep remote shared memory alive until every CTA has finished reading
    if constexpr (R > 1) cg::this_cluster().sync();
}

// ---------------------------------------------------------------------------
// work-list consumer: every (PRN, bin) task of every signal group of a plan
// in one persistent launch. Groups on the compile-time 24 000-point plan with
// split R = 8 (e.g. 192 000 points) form the wide queue, R = 2 (48 000) the
// narrow one. The launch asks for clusters of 8 CTAs and accepts clusters of 2
// where 8 do not fit (a preferred cluster dimension; 8-CTA clusters fit 120
// of the 148 SMs): an 8-CTA cluster takes wide tasks while there are any,
// then four narrow tasks at a time; a 2-CTA cluster takes one narrow task at
// a time. Tasks are claimed with one atomic per unit, in bin-major order
// within each group (the PRNs of a bin share its spectra in L2).
// ---------------------------------------------------------------------------
struct WorkGroup {
    const float2 *split, *X, *code;
    float *P, *Q;
    int R, n_prn, n_bin, n_sum, Nmax, Mq, q_by_sm;
    size_t prn_stride, bin_stride;
    float scale;
    int task0;              // first task of the group in its queue
    int x_comb;             // X holds the combined spectrum (ConsArgs::x_comb)
};

struct WorkArgs {
    FftPlanK pl;            // the 24 000-point plan
    const float2 *tw;       // its twiddles
    int n_group;
    int n_task[2];          // tasks of the wide (R = 8) and narrow (R = 2) queues
    int *next;              // [2] next unclaimed task of each queue, 0 at launch
    int *err;               // error word: a pair wait reached its bound
    WorkGroup g[kMaxWorkGroups];
};

__device__ __forceinline__ int work_group_of(const WorkArgs &a, int q, int t)
{
    for (int g = 0; g < a.n_group; ++g) {
        const WorkGroup &G = a.g[g];
        if ((G.R == 8) == (q == 0) && t >= G.task0 && t < G.task0 + G.n_prn * G.n_bin) return g;
    }
    return -1;
}

__device__ __forceinline__ ConsArgs work_cons_args(const WorkArgs &a, const WorkGroup &G)
{
    ConsArgs ca = {};
    ca.pl = a.pl; ca.tw = a.tw; ca.split = G.split; ca.X = G.X; ca.code = G.code;
    ca.n_prn = G.n_prn; ca.n_bin = G.n_bin; ca.n_sum = G.n_sum; ca.prn0 = 0;
    ca.scale = G.scale; ca.Nmax = G.Nmax; ca.prn_stride = G.prn_stride;
    ca.bin_stride = G.bin_stride; ca.accumulate = 0; ca.P = G.P; ca.Q = G.Q; ca.Mq = G.Mq;
    ca.q_by_sm = G.q_by_sm; ca.x_comb = G.x_comb;
    return ca;
}

__global__ void __launch_bounds__(512, 1) work_cons_kernel(WorkArgs a)
{
    extern __shared__ float2 smem[];
    float2 *sm = smem;
    float2 *tw = smem + Plan24000::M;
    __shared__ int unit[3];           // queue (0 wide, 1 narrow, -1 none), first task, tasks
    __shared__ __align__(8) uint64_t pair_bar[2];
    __shared__ uint32_t pair_state[3];
    cg::cluster_group cl = cg::this_cluster();
    const int csize = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const uint32_t bar0 = (uint32_t)__cvta_generic_to_shared(pair_bar);
    uint32_t remote0;                 // the partner CTA (rank ^ 1) of narrow tasks
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote0) : "r"(bar0), "r"(rank ^ 1));
    if (threadIdx.x == 0) {
        for (int k = 0; k < 2; ++k)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0 + 8u * k) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        pair_state[0] = pair_state[1] = pair_state[2] = 0u;
    }
    const PairSync pair{bar0, remote0, pair_state, a.err};
    load_twiddles(tw, a.tw, Plan24000::TWTOT);
    for (;;) {
        if (rank == 0 && threadIdx.x == 0) {
            int q = -1, t = 0, n = 0;
            if (csize >= 8) {
                t = atomicAdd(&a.next[0], 1);
                if (t < a.n_task[0]) { q = 0; n = 1; }
            }
            if (q < 0) {
                const int per = csize / 2;
                t = atomicAdd(&a.next[1], per);
                if (t < a.n_task[1]) { q = 1; n = min(per, a.n_task[1] - t); }
            }
            unit[0] = q; unit[1] = t; unit[2] = n;
        }
        cl.sync();                    // the unit (and, at first, the twiddles and
                                      // every CTA's pair barriers) visible
        const int *lu = cl.map_shared_rank(unit, 0);
        const int q = lu[0], t0 = lu[1], n = lu[2];
        if (q < 0) break;             // uniform across the cluster
        const int R = q == 0 ? 8 : 2;
        const int slot = rank / R, c = rank % R;
        const bool active = slot < n;
        const int gi = active ? work_group_of(a, q, t0 + slot) : -1;
        const WorkGroup &G = a.g[gi >= 0 ? gi : 0];
        const int local = t0 + slot - G.task0;
        const int prn = local % G.n_prn, b = local / G.n_prn;
        const ConsArgs ca = work_cons_args(a, G);
        const bool run = gi >= 0;
        if (run && threadIdx.x < R && G.n_sum > 0) {
            const int Mc = (Plan24000::M + R - 1) / R, q0 = c * Mc;
            const int q1 = min(Plan24000::M, q0 + Mc);
            prefetch_l2(G.X + (size_t)b * G.n_sum * R * Plan24000::M +
                        (size_t)threadIdx.x * Plan24000::M + q0, q1 - q0);
            prefetch_l2(G.code + (size_t)prn * R * Plan24000::M +
                        (size_t)threadIdx.x * Plan24000::M + q0, q1 - q0);
        }
        if (R == 8) {
            float2 *dst[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) dst[j] = cl.map_shared_rank(sm, j);
            cons_task<8, 0, 1>(ca, sm, tw, dst, c, local, prn, b, run ? G.n_sum : 0, run,
                               ClusterSync{});
        } else {
            float2 *dst[2];
#pragma unroll
            for (int j = 0; j < 2; ++j) dst[j] = cl.map_shared_rank(sm, 2 * slot + j);
            // both CTAs of the pair run the same task (or none): the pair's
            // barriers alone keep them in step
            cons_task<2, 0, 1>(ca, sm, tw, dst, c, local, prn, b, run ? G.n_sum : 0, run, pair);
        }
    }
    // the leader's unit word and every CTA's shared memory stay alive until
    // the whole cluster is done
    cl.sync();
}

// ---------------------------------------------------------------------------
// staged consumer for splits R > 8 (L up to 20 * M, e.g. 480 000 = 20 x 24 000):
// the combine writes the R sub-spectra w_c of a chunk of tasks to a scratch W
// in global memory (about 256 MB per chunk: it passes through HBM, the L2
// holding what is in flight), then R independent CTAs per task run the
// length-M inverse transforms. Same arithmetic as cons_kernel's cluster
// exchange.
// ---------------------------------------------------------------------------
struct StageArgs {
    const float2 *split, *X, *code;
    int R, M, n_prn, n_bin, n_sum;
    int task0, s;            // first task of the chunk, sum index
    float scale;
    float2 *W;               // [chunk][R][M]
    float *Q;                // power grids: [chunk][R][M] |y|^2 summed over the sums
    long long wait_cycles;   // bound of the first wait for each bulk copy
};

template <int R>
__global__ void __launch_bounds__(256) stage_combine_kernel(StageArgs a)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.M) return;
    const int tl = blockIdx.y, task = a.task0 + tl;
    const int prn = task % a.n_prn, b = task / a.n_prn;
    const size_t M = a.M;
    const float2 *Xs = a.X + ((size_t)b * a.n_sum + a.s) * R * M;
    const float2 *code = a.code + (size_t)prn * R * M;
    const float2 t = __ldg(a.split + q), tc = cconj(t);
    float2 g[R];
    g[0] = __ldg(Xs + q);
    float2 w = tc;
#pragma unroll
    for (int r = 1; r < R; ++r) {
        g[r] = cmul(__ldg(Xs + r * M + q), w);
        if (r + 1 < R) w = cmul(w, tc);
    }
    Dft<R, -1>::run(g);                     // X[k + jM]
#pragma unroll
    for (int j = 0; j < R; ++j) {
        const float2 z = cmul(g[j], __ldg(code + j * M + q));
        g[j] = make_float2(z.x * a.scale, z.y * a.scale);
    }
    Dft<R, 1>::run(g);                      // sum_j Z e^{+2 pi i c j / R}
    w = t;
#pragma unroll
    for (int j = 1; j < R; ++j) {
        g[j] = cmul(g[j], w);
        if (j + 1 < R) w = cmul(w, t);
    }
    float2 *Wt = a.W + (size_t)tl * R * M;
#pragma unroll
    for (int j = 0; j < R; ++j) Wt[j * M + q] = g[j];
}

// Power of output n = R m + c accumulated over the sums in Q[c][m], so that
// each CTA reads and writes consecutive addresses (the grid row itself holds
// a CTA's outputs R floats apart). The first sum stores |y|^2, or adds it to
// the caller's grid value when accumulating (the reference's order); later
// sums add to Q. stage_power_kernel moves Q into the grid after the last sum.
struct StorePowerQ {
    typedef float Old;
    float *q;            // Q row of this (task, c)
    const float *p;      // grid row of the task (seed of the first sum)
    int c, R, Nmax;
    int mode;            // 0: store, 1: add to Q, 2: add to the grid value
    const int *skip;     // shared flag: the CTA's input never arrived
    __device__ __forceinline__ float pre(int m) const
    {
        const int n = R * m + c;
        if (n >= Nmax || mode == 0 || *skip) return 0.0f;
        return mode == 1 ? q[m] : p[n];
    }
    __device__ __forceinline__ void operator()(int m, float2 y, float old) const
    {
        const int n = R * m + c;
        if (n < Nmax && !*skip) {
            const float pw = y.x * y.x + y.y * y.y;
            q[m] = mode ? old + pw : pw;
        }
    }
};

struct StoreComplexRt {
    typedef int Old;
    float2 *row;
    int c, R;
    const int *skip;     // shared flag: the CTA's input never arrived
    __device__ __forceinline__ int pre(int) const { return 0; }
    __device__ __forceinline__ void operator()(int m, float2 y, int) const
    {
        if (!*skip) row[R * m + c] = y;
    }
};

// ---- bulk copies through the TMA engine (cp.async.bulk, mbarrier) ----------

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;"
                 ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// bytes (a multiple of 16) from global src to shared dst, both 16-byte
// aligned, completing on bar
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes,
                                              uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                 "[%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
// waits for phase `parity` of bar to complete; false once `limit` clock
// cycles have passed (checked before each try: a limit of 0 gives up at once)
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit)
{
    const long long t0 = clock64();
    for (;;) {
        if (clock64() - t0 >= limit) return false;
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
        if (done) return true;
    }
}

// W exceeds L2: UL loads per thread in flight before the shared-memory stores,
// so the copy runs at HBM bandwidth rather than latency
__device__ __forceinline__ void load_plain(float2 *sm, const float2 *src, int M)
{
    constexpr int UL = 8;
    if ((M & 1) == 0) {
        const float4 *s4 = (const float4 *)src;
        float4 *d4 = (float4 *)sm;
        const int n4 = M / 2;
        for (int i0 = threadIdx.x; i0 < n4; i0 += UL * blockDim.x) {
            float4 v[UL];
#pragma unroll
            for (int u = 0; u < UL; ++u) {
                const int i = i0 + u * blockDim.x;
                if (i < n4) v[u] = __ldg(s4 + i);
            }
#pragma unroll
            for (int u = 0; u < UL; ++u) {
                const int i = i0 + u * blockDim.x;
                if (i < n4) d4[i] = v[u];
            }
        }
    } else {
        for (int i = threadIdx.x; i < M; i += blockDim.x) sm[i] = __ldg(src + i);
    }
}

// grid (R, chunk tasks): CTA c of a task inverts w_c
template <int MODE, int SP>
__global__ void __launch_bounds__(512, 1) stage_ifft_kernel(ConsArgs ca, StageArgs a)
{
    extern __shared__ float2 smem[];
    float2 *sm = smem;
    float2 *tw = smem + ca.pl.M;
    const int M = SP ? Plan24000::M : ca.pl.M;
    const int c = blockIdx.x, tl = blockIdx.y, task = a.task0 + tl;
    const int prn = task % a.n_prn, b = task / a.n_prn;
    const float2 *src = a.W + ((size_t)tl * a.R + c) * M;
    bool copied = false;
    __shared__ int skip;     // set when a region's copy never completed
    if (threadIdx.x == 0) skip = 0;
    if constexpr (SP == 1) {
        // compile-time plan: passes 3..1 run warp by warp on REG points each,
        // so each warp's region is brought in by its own bulk copy and the warp
        // starts as soon as that region has landed (the twiddles load meanwhile)
        constexpr int NW = Plan24000::R0, REG = Plan24000::M / NW;
        constexpr uint32_t RB = REG * sizeof(float2);
        static_assert(RB % 16 == 0, "bulk copies move multiples of 16 bytes");
        __shared__ __align__(8) uint64_t bar[NW];
        if (((smem_u32(sm) | (uint32_t)(uintptr_t)src) & 15u) == 0) {
            const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
            if (threadIdx.x == 0) {
                for (int k = 0; k < NW; ++k) mbar_init(&bar[k], 1);
                mbar_init_fence();
            }
            __syncthreads();
            if (lane == 0) {
                mbar_expect_tx(&bar[w], RB);
                bulk_copy_g2s(sm + w * REG, src + w * REG, RB, &bar[w]);
            }
            load_twiddles(tw, ca.tw, ca.pl.twtot);
            __syncthreads();
            if (!mbar_wait(&bar[w], 0, a.wait_cycles)) {
                // give up on the bound: record it and wait (bounded) for the
                // copy in flight before the region is touched; if even that
                // runs out, the CTA stores nothing (the flag is read after
                // the barrier before the last pass)
                if (lane == 0) atomicOr(ca.stage_err, 1);
                if (!mbar_wait(&bar[w], 0, kBulkWaitCycles) && lane == 0) skip = 1;
            }
            copied = true;
        }
    }
    if (!copied) {
        load_twiddles(tw, ca.tw, ca.pl.twtot);
        load_plain(sm, src, M);
        __syncthreads();
    }
    if (MODE == 0) {
        const float *row = ca.P + (size_t)prn * ca.prn_stride + (size_t)b * ca.bin_stride;
        StorePowerQ st{a.Q + ((size_t)tl * a.R + c) * M, row, c, a.R, ca.Nmax,
                       a.s > 0 ? 1 : (ca.accumulate ? 2 : 0), &skip};
        if constexpr (SP == 1) fft_inverse_static<Plan24000>(sm, tw, st);
        else fft_inverse(sm, tw, ca.pl, st);
    } else {
        StoreComplexRt st{ca.Y + (size_t)b * a.R * M, c, a.R, &skip};
        if constexpr (SP == 1) fft_inverse_static<Plan24000>(sm, tw, st);
        else fft_inverse(sm, tw, ca.pl, st);
    }
}

// Grid rows of a chunk from Q: P[n] = Q[n % R][n / R] for n < Nmax, through a
// shared-memory tile of kStageTm positions x R sub-transforms, so that both
// the Q reads and the grid writes are consecutive.
constexpr int kStageTm = 64;

__global__ void __launch_bounds__(256) stage_power_kernel(ConsArgs ca, StageArgs a)
{
    __shared__ float tile[kStageTm * 20];
    const int R = a.R, M = a.M;
    const int m0 = blockIdx.x * kStageTm, tl = blockIdx.y, task = a.task0 + tl;
    const int prn = task % a.n_prn, b = task / a.n_prn;
    const float *Qt = a.Q + (size_t)tl * R * M;
    for (int i = threadIdx.x; i < R * kStageTm; i += blockDim.x) {
        const int c = i / kStageTm, mm = i - c * kStageTm, m = m0 + mm;
        tile[mm * R + c] = (m < M) ? Qt[(size_t)c * M + m] : 0.0f;
    }
    __syncthreads();
    float *row = ca.P + (size_t)prn * ca.prn_stride + (size_t)b * ca.bin_stride;
    const long n0 = (long)R * m0;
    for (int i = threadIdx.x; i < R * kStageTm; i += blockDim.x) {
        const long n = n0 + i;
        if (n < ca.Nmax) row[n] = tile[i];
    }
}

// out[p][j][q] = code_nat[p][k(q) + j M] (permuted order of the DIF output)
__global__ void perm_code_kernel(const float2 *code_nat, const int *kperm, int M,
                                 int R, int n_prn, float2 *out)
{
    const size_t total = (size_t)n_prn * R * M;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const int q = (int)(i % M);
        const size_t pj = i / M;           // p * R + j
        const int j = (int)(pj % R);
        const size_t p = pj / R;
        out[i] = code_nat[p * (size_t)R * M + (size_t)j * M + kperm[q]];
    }
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
template <int MODE>
static int launch_fwd(const FftPlan *pl, const FwdArgs &a, int n_blocks, cudaStream_t st)
{
    static bool attr_set[2][2] = {{false, false}, {false, false}};
    // the compile-time 24 000-point plan where it applies
    const int sp = Plan24000::matches(pl->k, pl->threads) ? 1 : 0;
    if (!attr_set[MODE][sp]) {
        SDRG_CUDA(cudaFuncSetAttribute(sp ? fwd_kernel<MODE, 1> : fwd_kernel<MODE, 0>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(g_smem_limit())));
        attr_set[MODE][sp] = true;
    }
    if (sp) fwd_kernel<MODE, 1><<<n_blocks, pl->threads, pl->smem, st>>>(a);
    else fwd_kernel<MODE, 0><<<n_blocks, pl->threads, pl->smem, st>>>(a);
    SDRG_CUDA(cudaGetLastError());
    return SDRG_OK;
}

// Dynamic shared memory of a consumer launch: the transform and its twiddles
// (the compact twiddles of the 12 000-point compile-time plan, whose CTAs
// then fit two per SM).
static size_t cons_smem(const FftPlan *pl)
{
    if (pl->R == 4 && Plan12000::matches(pl->k, pl->threads))
        return (size_t)(Plan12000::M + Plan12000::TWS) * sizeof(float2);
    return pl->smem;
}

// Combines the sub-spectra of n_bs (bin, sum) blocks in place; returns 1 in
// *done when it ran (splits 2..8), 0 otherwise (no split, or a staged one).
static int launch_xcomb(const FftPlan *pl, float2 *X, int n_bs, cudaStream_t st, int *done)
{
    *done = 0;
    if (pl->R < 2 || pl->R > 8 || n_bs <= 0) return SDRG_OK;
    const dim3 g((unsigned)((pl->M + 255) / 256), (unsigned)n_bs);
    switch (pl->R) {
    case 2: xcomb_kernel<2><<<g, 256, 0, st>>>(X, pl->split_dev, pl->M); break;
    case 3: xcomb_kernel<3><<<g, 256, 0, st>>>(X, pl->split_dev, pl->M); break;
    case 4: xcomb_kernel<4><<<g, 256, 0, st>>>(X, pl->split_dev, pl->M); break;
    case 5: xcomb_kernel<5><<<g, 256, 0, st>>>(X, pl->split_dev, pl->M); break;
    case 6: xcomb_kernel<6><<<g, 256, 0, st>>>(X, pl->split_dev, pl->M); break;
    case 8: xcomb_kernel<8><<<g, 256, 0, st>>>(X, pl->split_dev, pl->M); break;
    default: return SDRG_OK;
    }
    SDRG_CUDA(cudaGetLastError());
    *done = 1;
    return SDRG_OK;
}

template <int R, int MODE, int SP>
static int launch_cons_RS(const FftPlan *pl, const ConsArgs &a, int n_tasks, cudaStream_t st)
{
    static bool attr_set = false;
    if (!attr_set) {
        SDRG_CUDA(cudaFuncSetAttribute(cons_kernel<R, MODE, SP>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(g_smem_limit())));
        if (R > 1) {
            SDRG_CUDA(cudaFuncSetAttribute(cons_kernel<R, MODE, SP>,
                                           cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        }
        attr_set = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(n_tasks * R));
    cfg.blockDim = dim3(pl->threads);
    cfg.dynamicSmemBytes = cons_smem(pl);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = R;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = R > 1 ? 1 : 0;
    SDRG_CUDA(cudaLaunchKernelEx(&cfg, cons_kernel<R, MODE, SP>, a));
    return SDRG_OK;
}

// the compile-time 24 000-point plan where it applies (R = 1, 2, 8), the
// 12 000-point one for 4-way splits, the runtime plan otherwise
template <int R, int MODE>
static int launch_cons_R(const FftPlan *pl, const ConsArgs &a, int n_tasks, cudaStream_t st)
{
    if constexpr (R == 1 || R == 2 || R == 8) {
        if (Plan24000::matches(pl->k, pl->threads))
            return launch_cons_RS<R, MODE, 1>(pl, a, n_tasks, st);
    }
    if constexpr (R == 4) {
        if (Plan12000::matches(pl->k, pl->threads))
            return launch_cons_RS<R, MODE, 2>(pl, a, n_tasks, st);
    }
    return launch_cons_RS<R, MODE, 0>(pl, a, n_tasks, st);
}

template <int MODE>
static int launch_cons(const FftPlan *pl, const ConsArgs &a, int n_tasks, cudaStream_t st)
{
    switch (pl->R) {
    case 1: return launch_cons_R<1, MODE>(pl, a, n_tasks, st);
    case 2: return launch_cons_R<2, MODE>(pl, a, n_tasks, st);
    case 3: return launch_cons_R<3, MODE>(pl, a, n_tasks, st);
    case 4: return launch_cons_R<4, MODE>(pl, a, n_tasks, st);
    case 5: return launch_cons_R<5, MODE>(pl, a, n_tasks, st);
    case 6: return launch_cons_R<6, MODE>(pl, a, n_tasks, st);
    case 8: return launch_cons_R<8, MODE>(pl, a, n_tasks, st);
    default: return set_error(SDRG_ERR_ARG, "unsupported split %d", pl->R);
    }
}

template <int MODE, int SP>
static int set_stage_attr()
{
    static bool done = false;
    if (!done) {
        // the per-block limit covers the kernel's static shared memory too
        // (its bulk-copy barriers)
        cudaFuncAttributes fa;
        SDRG_CUDA(cudaFuncGetAttributes(&fa, stage_ifft_kernel<MODE, SP>));
        SDRG_CUDA(cudaFuncSetAttribute(stage_ifft_kernel<MODE, SP>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(g_smem_limit() - fa.sharedSizeBytes)));
        done = true;
    }
    return SDRG_OK;
}

// Tasks of a staged split (R > 8) in chunks of w_tasks, each chunk through
// the scratch W (w_tasks * L complex), sum by sum.
// Staged inverse launches still to run with a first bulk-copy wait bound of 0
// (sdrg_inject_stage_timeout): their waits give up at once and report, the
// copies themselves land and are waited for with the full bound.
static std::atomic<int> g_stage_timeouts{0};

static long long stage_wait_bound()
{
    int n = g_stage_timeouts.load();
    while (n > 0 && !g_stage_timeouts.compare_exchange_weak(n, n - 1)) {
    }
    return n > 0 ? 0 : kBulkWaitCycles;
}

template <int MODE>
static int launch_staged(const FftPlan *pl, const ConsArgs &ca, int n_tasks, cudaStream_t st,
                         float2 *W, int w_tasks)
{
    if (!W || w_tasks <= 0) return set_error(SDRG_ERR_ARG, "staged FFT split without scratch");
    if (!ca.stage_err) return set_error(SDRG_ERR_ARG, "staged FFT split without an error word");
    const bool sp = Plan24000::matches(pl->k, pl->threads);
    int e;
    if ((e = sp ? set_stage_attr<MODE, 1>() : set_stage_attr<MODE, 0>())) return e;
    if (pl->R > 20) return set_error(SDRG_ERR_ARG, "unsupported staged split %d", pl->R);
    StageArgs sa = {};
    sa.split = pl->split_dev; sa.X = ca.X; sa.code = ca.code;
    sa.R = pl->R; sa.M = pl->M; sa.n_prn = ca.n_prn - ca.prn0; sa.n_bin = ca.n_bin;
    sa.n_sum = ca.n_sum; sa.scale = ca.scale; sa.W = W;
    // power grids: Q follows the w_tasks sub-spectra in the same scratch
    sa.Q = MODE == 0 ? (float *)(W + (size_t)w_tasks * pl->L) : nullptr;
    for (int t0 = 0; t0 < n_tasks; t0 += w_tasks) {
        const int n = n_tasks - t0 < w_tasks ? n_tasks - t0 : w_tasks;
        for (int s = 0; s < ca.n_sum; ++s) {
            sa.task0 = t0;
            sa.s = s;
            const dim3 gc((unsigned)((pl->M + 255) / 256), (unsigned)n);
            switch (pl->R) {
            case 10: stage_combine_kernel<10><<<gc, 256, 0, st>>>(sa); break;
            case 12: stage_combine_kernel<12><<<gc, 256, 0, st>>>(sa); break;
            case 15: stage_combine_kernel<15><<<gc, 256, 0, st>>>(sa); break;
            case 16: stage_combine_kernel<16><<<gc, 256, 0, st>>>(sa); break;
            case 20: stage_combine_kernel<20><<<gc, 256, 0, st>>>(sa); break;
            default: return set_error(SDRG_ERR_ARG, "unsupported staged split %d", pl->R);
            }
            SDRG_CUDA(cudaGetLastError());
            const dim3 gi((unsigned)pl->R, (unsigned)n);
            sa.wait_cycles = stage_wait_bound();
            if (sp) stage_ifft_kernel<MODE, 1><<<gi, pl->threads, pl->smem, st>>>(ca, sa);
            else stage_ifft_kernel<MODE, 0><<<gi, pl->threads, pl->smem, st>>>(ca, sa);
            SDRG_CUDA(cudaGetLastError());
        }
        if (MODE == 0) {
            sa.task0 = t0;
            const int mn = (ca.Nmax + pl->R - 1) / pl->R;    // positions holding n < Nmax
            const dim3 gp((unsigned)((mn + kStageTm - 1) / kStageTm), (unsigned)n);
            stage_power_kernel<<<gp, 256, 0, st>>>(ca, sa);
            SDRG_CUDA(cudaGetLastError());
        }
    }
    return SDRG_OK;
}

// the consumer for any plan: cluster exchange for R <= 8, staged otherwise
template <int MODE>
static int launch_consumer(const FftPlan *pl, const ConsArgs &ca, int n_tasks, cudaStream_t st,
                           float2 *W, int w_tasks)
{
    if (pl->R <= 8) return launch_cons<MODE>(pl, ca, n_tasks, st);
    return launch_staged<MODE>(pl, ca, n_tasks, st, W, w_tasks);
}

// bytes of a staged split's scratch for w_tasks tasks: the sub-spectra W and,
// for power grids (MODE 0), the power accumulator Q behind them
static size_t staged_bytes(const FftPlan *pl, int w_tasks, int mode)
{
    return (size_t)w_tasks * pl->L * (sizeof(float2) + (mode == 0 ? sizeof(float) : 0));
}

// scratch tasks for a staged split: about 256 MB of sub-spectra per chunk
static int staged_chunk(const FftPlan *pl, int n_tasks)
{
    if (pl->R <= 8) return 0;
    long c = (256L << 20) / ((long)pl->L * (long)sizeof(float2));
    if (c < 1) c = 1;
    return (int)(c < n_tasks ? c : n_tasks);
}

static int perm_code(const FftPlan *pl, const float2 *nat, int n_prn, float2 *out,
                     cudaStream_t st)
{
    size_t total = (size_t)n_prn * pl->L;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    perm_code_kernel<<<blocks, 256, 0, st>>>(nat, pl->kperm_dev, pl->M, pl->R, n_prn, out);
    SDRG_CUDA(cudaGetLastError());
    return SDRG_OK;
}

// reference phase arithmetic (src/sdr_func.c:776-778)
static inline uint32_t phase_of(double phi)
{
    return (uint32_t)((phi - floor(phi)) * 4294967296.0);
}
static inline uint32_t step_of(double step)
{
    return (uint32_t)(int)(step * 4294967296.0);
}

// The calling thread's error word for staged launches (device, zeroed once).
static int thread_stage_err(int **out, cudaStream_t st)
{
    ThreadCtx &c = tctx();
    if (!c.stage_err.ptr) {
        int e;
        if ((e = c.stage_err.reserve(sizeof(int)))) return e;
        SDRG_CUDA(cudaMemsetAsync(c.stage_err.ptr, 0, sizeof(int), st));
    }
    *out = (int *)c.stage_err.ptr;
    return SDRG_OK;
}

// After a synchronous call that ran a staged split (its work on st has
// completed): reports, and clears, a bulk-copy wait of stage_ifft_kernel that
// reached its bound, recorded in the error word err.
static int stage_wait_check(const FftPlan *pl, int *err, cudaStream_t st, bool always = false)
{
    if (!always && (!pl || pl->R <= 8)) return SDRG_OK;
    if (!err) return SDRG_OK;
    int v = 0;
    SDRG_CUDA(cudaMemcpyAsync(&v, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    SDRG_CUDA(cudaStreamSynchronize(st));
    if (!v) return SDRG_OK;
    SDRG_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    SDRG_CUDA(cudaStreamSynchronize(st));
    return set_error(SDRG_ERR_CUDA, "FFT consumer: a wait for a bulk copy into shared memory "
                     "or for a partner CTA reached its bound; results of that call are not valid");
}

// Plan for a batch of n transforms of length N. The default split puts one
// CTA of each of its R sub-transforms on an SM; a batch that would leave more
// than half of the SMs idle (n R < SMs / 2) takes the largest finer cluster
// split (up to 8) that keeps n R within two waves, so that the same work is
// spread over more SMs (10 L6 channels of 96 000 points: 4 -> 8 ways, 110 K ->
// 145 K channel-epochs/s). A schedule set for N is kept as it is.
static const FftPlan *plan_for_jobs(int N, int n)
{
    const FftPlan *pl = get_plan(N);
    if (!pl || pl->R > 8 || sdrg_fft_schedule_get(N, nullptr, nullptr)) return pl;
    Device *dev;
    if (ensure_device(&dev)) return pl;
    const long sms = dev->sm_count;
    if (2L * n * pl->R >= sms) return pl;
    for (int R : {8, 6, 5, 4, 3, 2}) {
        if (R <= pl->R) break;
        if ((long)n * R > 2 * sms || !shape_ok(N, R)) continue;
        if (const FftPlan *p2 = get_plan_shaped(N, R, 0)) return p2;
    }
    return pl;
}

// Common body of the drop-in FFT correlator calls. iq_dev holds N mixed
// samples on the device; code_host is the natural-order conjugated code DFT.
static int corr_fft_device(const char2 *iq_dev, const sdr_cpx_t *code_host, int N,
                           sdr_cpx_t *corr_host)
{
    const FftPlan *pl = plan_for_jobs(N, 1);
    if (!pl) return tctx().error;
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    cudaStream_t st;
    if ((e = thread_stream(&st))) return e;
    ThreadCtx &c = tctx();
    const size_t cb = (size_t)N * sizeof(float2);
    if ((e = c.dev[1].reserve(2 * cb)) || (e = c.dev[2].reserve(cb)) ||
        (e = c.dev[3].reserve(cb)))
        return e;
    c.host[0].pinned = true;
    if ((e = c.host[0].reserve(cb))) return e;
    float2 *code_nat = (float2 *)c.dev[1].ptr;
    float2 *code_perm = code_nat + N;
    float2 *X = (float2 *)c.dev[2].ptr;
    float2 *Y = (float2 *)c.dev[3].ptr;
    memcpy(c.host[0].ptr, code_host, cb);
    SDRG_CUDA(cudaMemcpyAsync(code_nat, c.host[0].ptr, cb, cudaMemcpyHostToDevice, st));
    if ((e = perm_code(pl, code_nat, 1, code_perm, st))) return e;

    FwdArgs fa = {};
    fa.pl = pl->k; fa.tw = pl->tw_dev; fa.ctab = dev->ctab_dev; fa.R = pl->R;
    fa.n_bin = 1; fa.n_sum = 1; fa.cscale = kCScale; fa.iq = iq_dev; fa.X = X;
    if ((e = launch_fwd<1>(pl, fa, pl->R, st))) return e;

    ConsArgs ca = {};
    ca.pl = pl->k; ca.tw = pl->tw_dev; ca.split = pl->split_dev; ca.X = X;
    ca.code = code_perm; ca.n_prn = 1; ca.n_bin = 1; ca.n_sum = 1; ca.prn0 = 0;
    ca.scale = 1.0f / N / N; ca.Nmax = N; ca.Y = Y;
    if ((e = thread_stage_err(&ca.stage_err, st))) return e;
    const int wt = staged_chunk(pl, 1);
    if (wt && (e = c.dev[5].reserve((size_t)wt * cb))) return e;
    if ((e = launch_consumer<1>(pl, ca, 1, st, wt ? (float2 *)c.dev[5].ptr : nullptr, wt)))
        return e;
    SDRG_CUDA(cudaMemcpyAsync(c.host[0].ptr, Y, cb, cudaMemcpyDeviceToHost, st));
    SDRG_CUDA(cudaStreamSynchronize(st));
    if ((e = stage_wait_check(pl, ca.stage_err, st))) return e;
    memcpy(corr_host, c.host[0].ptr, cb);
    return SDRG_OK;
}

// ---------------------------------------------------------------------------
// one correlation job on device data: sdr_mix_carr(buf, ix, N, fs, fc, phi)
// then sdr_corr_fft with a natural-order conjugated code DFT
// ---------------------------------------------------------------------------
void corr_job_tables(int len, int ix, int N, double fs, double fc, double phi, uint32_t *tab)
{
    // mixing phases as sdr_mix_carr (src/sdr_func.c:824-836): restart at the
    // buffer wrap with phi + step * n
    const double step = fc / fs;
    const int n1 = (ix + N <= len) ? N : len - ix;
    tab[0] = step_of(step);
    tab[1] = phase_of(phi);
    tab[2] = n1 < N ? phase_of(phi + step * n1) : 0;
    tab[3] = (uint32_t)ix;
    tab[4] = (uint32_t)n1;
}

size_t corr_job_scratch(int N)
{
    const FftPlan *pl = get_plan(N);
    if (!pl) return 0;
    const int wt = staged_chunk(pl, 1);
    return (size_t)N * sizeof(float2) * (2 + (size_t)wt);
}

int corr_job_device(const uint8_t *buf, int len, const uint32_t *tab_dev, int N,
                    const float2 *code_nat, float2 *corr, void *scratch, cudaStream_t st)
{
    const FftPlan *pl = plan_for_jobs(N, 1);
    if (!pl) return tctx().error ? tctx().error : SDRG_ERR_ARG;
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    float2 *code_perm = (float2 *)scratch, *X = code_perm + N, *W = X + N;
    if ((e = perm_code(pl, code_nat, 1, code_perm, st))) return e;
    FwdArgs fa = {};
    fa.pl = pl->k; fa.tw = pl->tw_dev; fa.ctab = dev->ctab_dev; fa.R = pl->R;
    fa.n_bin = 1; fa.n_sum = 1; fa.cscale = kCScale;
    fa.buf = buf; fa.buf_len = len;
    fa.phstep = tab_dev; fa.ph0a = tab_dev + 1; fa.ph0b = tab_dev + 2;
    fa.ix = (const int *)(tab_dev + 3); fa.nsplit = (const int *)(tab_dev + 4);
    fa.X = X;
    if ((e = launch_fwd<0>(pl, fa, pl->R, st))) return e;
    ConsArgs ca = {};
    ca.pl = pl->k; ca.tw = pl->tw_dev; ca.split = pl->split_dev; ca.X = X; ca.code = code_perm;
    ca.n_prn = 1; ca.n_bin = 1; ca.n_sum = 1; ca.prn0 = 0;
    ca.scale = 1.0f / N / N; ca.Nmax = N; ca.Y = corr;
    if ((e = thread_stage_err(&ca.stage_err, st))) return e;
    const int wt = staged_chunk(pl, 1);
    return launch_consumer<1>(pl, ca, 1, st, wt ? W : nullptr, wt);
}

// n jobs of the same length N on one buffer in one launch each (splits of a
// thread-block cluster, R <= 8): tab_dev = phstep[n] | ph0a[n] | ph0b[n] |
// ix[n] | nsplit[n]; code_nat [n][N]; corr [n][N]; scratch 2 n N complex.
int corr_jobs_device(const uint8_t *buf, int len, const uint32_t *tab_dev, int n, int N,
                     const float2 *code_nat, float2 *corr, void *scratch, cudaStream_t st)
{
    const FftPlan *pl = plan_for_jobs(N, n);
    if (!pl) return tctx().error ? tctx().error : SDRG_ERR_ARG;
    if (pl->R > 8) return set_error(SDRG_ERR_ARG, "batched jobs need a cluster split (N=%d)", N);
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    float2 *code_perm = (float2 *)scratch, *X = code_perm + (size_t)n * N;
    if ((e = perm_code(pl, code_nat, n, code_perm, st))) return e;
    FwdArgs fa = {};
    fa.pl = pl->k; fa.tw = pl->tw_dev; fa.ctab = dev->ctab_dev; fa.R = pl->R;
    fa.n_bin = n; fa.n_sum = 1; fa.cscale = kCScale;
    fa.buf = buf; fa.buf_len = len;
    fa.phstep = tab_dev; fa.ph0a = tab_dev + n; fa.ph0b = tab_dev + 2 * n;
    fa.ix = (const int *)(tab_dev + 3 * n); fa.nsplit = (const int *)(tab_dev + 4 * n);
    fa.ix_per_bin = 1;
    fa.X = X;
    if ((e = launch_fwd<0>(pl, fa, n * pl->R, st))) return e;
    ConsArgs ca = {};
    ca.pl = pl->k; ca.tw = pl->tw_dev; ca.split = pl->split_dev; ca.X = X; ca.code = code_perm;
    ca.n_prn = 1; ca.n_bin = n; ca.n_sum = 1; ca.prn0 = 0; ca.code_per_bin = 1;
    ca.scale = 1.0f / N / N; ca.Nmax = N; ca.Y = corr;
    return launch_cons<1>(pl, ca, n, st);
}

// ---------------------------------------------------------------------------
// batched plan
// ---------------------------------------------------------------------------
struct GroupState {
    sdrg_acq_sig_t sig;
    const FftPlan *pl;
    std::vector<float> fds;
    std::vector<uint32_t> phstep;       // per bin
    float2 *code = nullptr;             // [n_prn][R][M]
    float2 *X = nullptr;                // [n_bin][n_sum][R][M]
    float *P = nullptr;                 // [n_prn][n_bin][Nmax]
    float2 *W = nullptr;                // staged splits: [w_tasks][R][M] sub-spectra
    float *Q = nullptr;                 // cluster splits, several sums: power accumulator
    int Mq = 0;                         // its row length, ceil(Nmax / R)
    int q_by_sm = 0;                    // Q holds one row per SM (see ConsArgs)
    void *peak_parts = nullptr;         // partial peak reductions
    int w_tasks = 0;
    uint32_t *tab_dev = nullptr;        // phstep | ph0a | ph0b | (int) ix | nsplit
    uint32_t *tab_host = nullptr;       // pinned mirror
    size_t tab_words = 0;
    cudaEvent_t tab_ev = nullptr;       // last upload of tab_host
    int last_len = -1, last_ix = -1;
    int res_off = 0;
};

} // namespace sdrg

struct sdrg_acq_plan {
    std::vector<sdrg::GroupState> g;
    int n_res = 0;
    int *stage_err = nullptr;   // device error word of the staged launches
    int64_t cells = 0;
    // Signal groups run concurrently on internal streams forked from and
    // joined back to the caller's stream: a group whose clusters cannot use
    // every SM (8-CTA clusters fit 120 of 148) leaves room for the others.
    std::vector<cudaStream_t> streams;
    cudaEvent_t ev_fork = nullptr;
    std::vector<cudaEvent_t> ev_join;
    // kernel timing (sdrg_acq_profile): event pairs recorded around launches
    struct Rec { int kind, run; cudaEvent_t a, b; int n; };   // n: kernel launches inside
    bool prof = false;
    int run = 0;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<Rec> ev_used;
    // sdrg_acq_run_graph: the captured launch sequence and the buffers it
    // was captured for
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    std::vector<intptr_t> graph_key;
    int graph_captures = 0;
    // work-list consumer (sdrg_acq_set_worklist): eligible when every group
    // is on the 24 000-point compile-time plan with split 2 or 8
    bool wl_ok = false;
    int wl_mode = 0;            // 0 per-group launches, 1 work list (-1: the work list
                                // where allowed)
    int *wl_next = nullptr;     // [2] device queue heads
};

static void drop_graph(sdrg_acq_plan_t *plan)
{
    if (plan->graph_exec) cudaGraphExecDestroy(plan->graph_exec);
    if (plan->graph) cudaGraphDestroy(plan->graph);
    plan->graph_exec = nullptr;
    plan->graph = nullptr;
    plan->graph_key.clear();
}

namespace sdrg {

// device reduction for (group, PRN) peaks, defined in sdrg_peak.cu
int launch_peaks(const float *P, int n_prn, int M_rows, int Nmax, size_t row_stride,
                 size_t prn_stride, double T, const float *fds_dev,
                 sdrg_acq_result_t *res, void *scratch, cudaStream_t st);
size_t peak_scratch_bytes(int n_prn);

static int group_tables(GroupState &G, const int *len_if, const int *ix)
{
    const sdrg_acq_sig_t &s = G.sig;
    const int nb = s.len_fds, ns = s.n_sum;
    uint32_t *t = G.tab_host;
    uint32_t *phstep = t, *ph0a = t + nb, *ph0b = t + 2 * nb;
    int *ixs = (int *)(t + 2 * nb + (size_t)nb * ns);
    int *nsplit = ixs + ns;
    const int len = len_if[s.buf];
    for (int b = 0; b < nb; ++b) {
        phstep[b] = G.phstep[b];
        ph0a[b] = 0;   // sdr_search_code mixes with phi = 0 (src/sdr_func.c:673)
    }
    for (int k = 0; k < ns; ++k) {
        long long pos = ((long long)ix[s.buf] + (long long)k * s.N) % len;
        if (pos < 0) pos += len;
        ixs[k] = (int)pos;
        nsplit[k] = (pos + s.L > len) ? (int)(len - pos) : s.L;
        for (int b = 0; b < nb; ++b) {
            const double step = (s.fi + (double)G.fds[b]) / s.fs;
            ph0b[(size_t)b * ns + k] = nsplit[k] < s.L ? phase_of(0.0 + step * nsplit[k]) : 0;
        }
    }
    return SDRG_OK;
}

static int prof_begin(sdrg_acq_plan *plan, cudaStream_t st, cudaEvent_t *ev)
{
    if (!plan->prof) return SDRG_OK;
    for (int i = 0; i < 2; ++i) {
        if (plan->ev_pool.empty()) {
            cudaEvent_t e;
            SDRG_CUDA(cudaEventCreate(&e));
            plan->ev_pool.push_back(e);
        }
        ev[i] = plan->ev_pool.back();
        plan->ev_pool.pop_back();
    }
    SDRG_CUDA(cudaEventRecord(ev[0], st));
    return SDRG_OK;
}

static int prof_end(sdrg_acq_plan *plan, cudaStream_t st, cudaEvent_t *ev, int kind,
                    int n_launch = 1)
{
    if (!plan->prof) return SDRG_OK;
    SDRG_CUDA(cudaEventRecord(ev[1], st));
    plan->ev_used.push_back({kind, plan->run, ev[0], ev[1], n_launch});
    return SDRG_OK;
}

} // namespace sdrg

using namespace sdrg;

extern "C" {

int sdrg_inject_stage_timeout(int n)
{
    if (n < 0) return set_error(SDRG_ERR_ARG, "sdrg_inject_stage_timeout: n=%d", n);
    g_stage_timeouts.store(n);
    return SDRG_OK;
}

int sdrg_acq_profile(sdrg_acq_plan_t *plan, int enable)
{
    if (!plan) return set_error(SDRG_ERR_ARG, "sdrg_acq_profile: null plan");
    plan->prof = enable != 0;
    return SDRG_OK;
}

int sdrg_acq_profile_get(sdrg_acq_plan_t *plan, double *ms, int64_t *launches)
{
    if (!plan || !ms || !launches) return set_error(SDRG_ERR_ARG, "sdrg_acq_profile_get: null");
    const int ng = (int)plan->g.size(), nk = 3 * ng;
    for (int k = 0; k < nk + 3; ++k) { ms[k] = 0.0; launches[k] = 0; }
    // per-run union span of each kernel kind (launches of different groups
    // overlap on the internal streams): [earliest start, latest end]
    std::vector<double> lo(3), hi(3);
    int cur = -1;
    cudaEvent_t ref = nullptr;
    auto flush = [&]() {
        for (int k = 0; k < 3; ++k)
            if (hi[k] > lo[k]) { ms[nk + k] += hi[k] - lo[k]; launches[nk + k] += 1; }
    };
    for (auto &u : plan->ev_used) {
        SDRG_CUDA(cudaEventSynchronize(u.b));
        if (u.kind < 0) {   // reference event of a run, recorded before the fork
            if (cur >= 0) flush();
            cur = u.run;
            ref = u.a;
            for (int k = 0; k < 3; ++k) { lo[k] = 1e300; hi[k] = -1e300; }
            continue;
        }
        float t = 0.0f, t0 = 0.0f, t1 = 0.0f;
        SDRG_CUDA(cudaEventElapsedTime(&t, u.a, u.b));
        ms[u.kind] += t;
        launches[u.kind] += u.n;
        if (!ref) continue;
        SDRG_CUDA(cudaEventElapsedTime(&t0, ref, u.a));
        SDRG_CUDA(cudaEventElapsedTime(&t1, ref, u.b));
        const int k = u.kind % 3;
        lo[k] = t0 < lo[k] ? t0 : lo[k];
        hi[k] = t1 > hi[k] ? t1 : hi[k];
    }
    if (cur >= 0) flush();
    for (auto &u : plan->ev_used) {
        plan->ev_pool.push_back(u.a);
        if (u.b != u.a) plan->ev_pool.push_back(u.b);
    }
    plan->ev_used.clear();
    return SDRG_OK;
}

void sdr_corr_fft(const sdr_cpx16_t *IQ, const sdr_cpx_t *code_fft, int N,
                  sdr_cpx_t *corr)
{
    if (N <= 0) return;
    Device *dev;
    if (ensure_device(&dev)) { memset(corr, 0, sizeof(sdr_cpx_t) * N); return; }
    cudaStream_t st;
    ThreadCtx &c = tctx();
    if (thread_stream(&st) || c.dev[0].reserve((size_t)N * 2) ||
        ((c.host[1].pinned = true), c.host[1].reserve((size_t)N * 2))) {
        memset(corr, 0, sizeof(sdr_cpx_t) * N);
        return;
    }
    memcpy(c.host[1].ptr, IQ, (size_t)N * 2);
    if (cudaMemcpyAsync(c.dev[0].ptr, c.host[1].ptr, (size_t)N * 2,
                        cudaMemcpyHostToDevice, st) != cudaSuccess ||
        corr_fft_device((const char2 *)c.dev[0].ptr, code_fft, N, corr)) {
        memset(corr, 0, sizeof(sdr_cpx_t) * N);
    }
}

void sdr_corr_fft_cpx(const sdr_cpx_t *buff, int len_buff, int ix, int N, double fs,
                      double fc, double phi, const sdr_cpx_t *code_fft, sdr_cpx_t *corr)
{
    if (N <= 0) return;
    cudaStream_t st;
    ThreadCtx &c = tctx();
    if (ensure_device(nullptr) || thread_stream(&st) ||
        c.dev[0].reserve((size_t)N * 2) ||
        mix_cpx_device(buff, len_buff, ix, N, fs, fc, phi, (char2 *)c.dev[0].ptr, st) ||
        corr_fft_device((const char2 *)c.dev[0].ptr, code_fft, N, corr)) {
        memset(corr, 0, sizeof(sdr_cpx_t) * N);
    }
}

void sdr_search_code(const sdr_cpx_t *code_fft, double T, const sdr_buff_t *buff,
                     int ix, int N, double fs, double fi, const float *fds, int len_fds,
                     float *P)
{
    (void)T;
    if (N <= 0 || len_fds <= 0) return;
    if (!buff || !buff->data || ix < 0 || ix >= buff->N || N > buff->N) {
        set_error(SDRG_ERR_ARG, "sdr_search_code: bad buffer window ix=%d N=%d len=%d", ix, N,
                  buff ? buff->N : 0);
        return;
    }
    const FftPlan *pl = plan_for_jobs(N, len_fds);
    if (!pl) return;
    Device *dev;
    cudaStream_t st;
    if (ensure_device(&dev) || thread_stream(&st)) return;
    ThreadCtx &c = tctx();
    const size_t cb = (size_t)N * sizeof(float2);
    const size_t pb = (size_t)len_fds * N * sizeof(float);
    const size_t xb = (size_t)len_fds * cb;
    const size_t tabw = 3 * (size_t)len_fds + 2;
    for (int i = 0; i < 3; ++i) c.host[i].pinned = true;
    if (c.dev[0].reserve((size_t)N + 64) || c.dev[1].reserve(2 * cb) ||
        c.dev[2].reserve(xb) || c.dev[3].reserve(pb) ||
        c.dev[4].reserve(tabw * 4) || c.host[0].reserve(cb) ||
        c.host[1].reserve((size_t)N + 16 + tabw * 4) || c.host[2].reserve(pb))
        return;
    uint8_t *win_h = (uint8_t *)c.host[1].ptr;
    uint32_t *tab_h = (uint32_t *)(win_h + ((N + 15) / 16) * 16);
    // window copy with the circular wrap (src/sdr_func.c:829-835)
    const int n1 = (ix + N <= buff->N) ? N : buff->N - ix;
    memcpy(win_h, buff->data + ix, (size_t)n1);
    if (n1 < N) memcpy(win_h + n1, buff->data, (size_t)(N - n1));
    // tables: phstep[len_fds] | ph0a[len_fds] | ph0b[len_fds] | ix | nsplit
    uint32_t *phstep = tab_h, *ph0a = tab_h + len_fds, *ph0b = tab_h + 2 * len_fds;
    int *ixs = (int *)(tab_h + 3 * len_fds), *nsplit = ixs + 1;
    for (int b = 0; b < len_fds; ++b) {
        const double step = (fi + (double)fds[b]) / fs;
        phstep[b] = step_of(step);
        ph0a[b] = phase_of(0.0);
        ph0b[b] = n1 < N ? phase_of(0.0 + step * n1) : 0;
    }
    ixs[0] = 0;
    nsplit[0] = n1;
    uint8_t *win_d = (uint8_t *)c.dev[0].ptr;
    float2 *code_nat = (float2 *)c.dev[1].ptr, *code_perm = code_nat + N;
    float2 *X = (float2 *)c.dev[2].ptr;
    float *P_d = (float *)c.dev[3].ptr;
    uint32_t *tab_d = (uint32_t *)c.dev[4].ptr;
    memcpy(c.host[0].ptr, code_fft, cb);
    memcpy(c.host[2].ptr, P, pb);
    if (cudaMemcpyAsync(win_d, win_h, (size_t)N, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(tab_d, tab_h, tabw * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(code_nat, c.host[0].ptr, cb, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(P_d, c.host[2].ptr, pb, cudaMemcpyHostToDevice, st) != cudaSuccess) {
        cuda_error(cudaGetLastError(), "sdr_search_code H2D");
        return;
    }
    if (perm_code(pl, code_nat, 1, code_perm, st)) return;
    FwdArgs fa = {};
    fa.pl = pl->k; fa.tw = pl->tw_dev; fa.ctab = dev->ctab_dev; fa.R = pl->R;
    fa.n_bin = len_fds; fa.n_sum = 1; fa.cscale = kCScale;
    fa.buf = win_d; fa.buf_len = N;
    fa.phstep = tab_d; fa.ph0a = tab_d + len_fds; fa.ph0b = tab_d + 2 * len_fds;
    fa.ix = (const int *)(tab_d + 3 * len_fds);
    fa.nsplit = fa.ix + 1;
    fa.X = X;
    if (launch_fwd<0>(pl, fa, len_fds * pl->R, st)) return;
    ConsArgs ca = {};
    ca.pl = pl->k; ca.tw = pl->tw_dev; ca.split = pl->split_dev; ca.X = X; ca.code = code_perm;
    ca.n_prn = 1; ca.n_bin = len_fds; ca.n_sum = 1; ca.prn0 = 0;
    ca.scale = 1.0f / N / N; ca.Nmax = N; ca.prn_stride = 0; ca.bin_stride = N;
    ca.accumulate = 1; ca.P = P_d;
    if (thread_stage_err(&ca.stage_err, st)) return;
    const int wt = staged_chunk(pl, len_fds);
    if (wt && c.dev[5].reserve(staged_bytes(pl, wt, 0))) return;
    if (launch_consumer<0>(pl, ca, len_fds, st, wt ? (float2 *)c.dev[5].ptr : nullptr, wt))
        return;
    if (cudaMemcpyAsync(c.host[2].ptr, P_d, pb, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cuda_error(cudaGetLastError(), "sdr_search_code D2H");
        return;
    }
    if (stage_wait_check(pl, ca.stage_err, st)) return;   // P unchanged, error recorded
    memcpy(P, c.host[2].ptr, pb);
}

// ---- batched --------------------------------------------------------------
sdrg_acq_plan_t *sdrg_acq_plan_new(const sdrg_acq_sig_t *sigs, int n_sig)
{
    if (!sigs || n_sig <= 0) {
        set_error(SDRG_ERR_ARG, "sdrg_acq_plan_new: no signal groups");
        return nullptr;
    }
    Device *dev;
    cudaStream_t st;
    if (ensure_device(&dev) || thread_stream(&st)) return nullptr;
    sdrg_acq_plan_t *plan = new sdrg_acq_plan_t();
    plan->g.resize(n_sig);
    const int n_streams = n_sig < 4 ? n_sig : 4;
    plan->streams.resize(n_streams, nullptr);
    plan->ev_join.resize(n_streams, nullptr);
    bool sok = cudaEventCreateWithFlags(&plan->ev_fork, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; i < n_streams && sok; ++i) {
        sok = cudaStreamCreateWithFlags(&plan->streams[i], cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&plan->ev_join[i], cudaEventDisableTiming) == cudaSuccess;
    }
    sok = sok && cudaMalloc(&plan->stage_err, sizeof(int)) == cudaSuccess &&
          cudaMemsetAsync(plan->stage_err, 0, sizeof(int), st) == cudaSuccess;
    if (!sok) {
        cuda_error(cudaGetLastError(), "sdrg_acq_plan_new streams");
        sdrg_acq_plan_free(plan);
        return nullptr;
    }
    int res_off = 0;
    for (int gi = 0; gi < n_sig; ++gi) {
        GroupState &G = plan->g[gi];
        G.sig = sigs[gi];
        const sdrg_acq_sig_t &s = G.sig;
        if (s.L <= 0 || s.N <= 0 || s.Nmax <= 0 || s.Nmax > s.L || s.n_sum <= 0 ||
            s.n_prn <= 0 || s.len_fds <= 0 || !s.fds || s.fs <= 0) {
            set_error(SDRG_ERR_ARG, "sdrg_acq_plan_new: bad parameters for group %d", gi);
            sdrg_acq_plan_free(plan);
            return nullptr;
        }
        G.pl = plan_for_jobs(s.L, s.n_prn * s.len_fds);
        if (!G.pl) { sdrg_acq_plan_free(plan); return nullptr; }
        G.fds.assign(s.fds, s.fds + s.len_fds);
        G.sig.fds = nullptr;
        G.sig.code_fft = nullptr;
        G.phstep.resize(s.len_fds);
        for (int b = 0; b < s.len_fds; ++b) G.phstep[b] = step_of((s.fi + (double)G.fds[b]) / s.fs);
        const size_t L = (size_t)s.L;
        float2 *nat = nullptr;
        if (alloc_fault("sdrg_acq_plan_new")) {
            sdrg_acq_plan_free(plan);
            return nullptr;
        }
        bool ok = cudaMalloc(&G.code, (size_t)s.n_prn * L * sizeof(float2)) == cudaSuccess &&
                  cudaMalloc(&nat, (size_t)s.n_prn * L * sizeof(float2)) == cudaSuccess &&
                  cudaMalloc(&G.X, (size_t)s.len_fds * s.n_sum * L * sizeof(float2)) == cudaSuccess &&
                  cudaMalloc(&G.P, (size_t)s.n_prn * s.len_fds * s.Nmax * sizeof(float)) == cudaSuccess;
        G.w_tasks = staged_chunk(G.pl, s.n_prn * s.len_fds);
        ok = ok && (!G.w_tasks ||
                    cudaMalloc(&G.W, staged_bytes(G.pl, G.w_tasks, 0)) == cudaSuccess);
        if (G.pl->R > 1 && G.pl->R <= 8 && s.n_sum > 1) {
            G.Mq = (s.Nmax + G.pl->R - 1) / G.pl->R;
            // a consumer CTA needs more than half of an SM's shared memory, so
            // at most one runs on an SM at a time: the power accumulator can
            // be one row per SM (a few MB that stay in L2) instead of one per
            // task and CTA (1.1 GB for the E1-B group, whose dirty lines were
            // written back to HBM after every run)
            G.q_by_sm = 2 * (cons_smem(G.pl) + 1024) > dev->smem_per_sm;
            const size_t rows = G.q_by_sm ? (size_t)dev->nsmid
                                          : (size_t)s.n_prn * s.len_fds * G.pl->R;
            ok = ok && cudaMalloc(&G.Q, rows * G.Mq * sizeof(float)) == cudaSuccess;
        }
        ok = ok && cudaMalloc(&G.peak_parts, peak_scratch_bytes(s.n_prn)) == cudaSuccess;
        G.tab_words = 2 * (size_t)s.len_fds + (size_t)s.len_fds * s.n_sum + 2 * (size_t)s.n_sum + s.len_fds;
        ok = ok && cudaMalloc(&G.tab_dev, G.tab_words * 4) == cudaSuccess &&
             cudaMallocHost(&G.tab_host, G.tab_words * 4) == cudaSuccess &&
             cudaEventCreateWithFlags(&G.tab_ev, cudaEventDisableTiming) == cudaSuccess;
        // Uploads are ordered on the thread's (non-blocking) stream: a plain
        // cudaMemcpy from pageable memory may return before its DMA lands and
        // runs on the legacy stream, which kernels on `st` do not wait for.
        if (sigs[gi].code_fft) {
            ok = ok && cudaMemcpyAsync(nat, sigs[gi].code_fft, (size_t)s.n_prn * L * sizeof(float2),
                                       cudaMemcpyHostToDevice, st) == cudaSuccess;
            ok = ok && perm_code(G.pl, nat, s.n_prn, G.code, st) == SDRG_OK;
        } else {
            // codes come later from sdrg_acq_set_codes; zero until then
            ok = ok && cudaMemsetAsync(G.code, 0, (size_t)s.n_prn * L * sizeof(float2), st) ==
                           cudaSuccess;
        }
        // Doppler bins as float on the device for the fine-Doppler fit
        if (ok) {
            float *fd_dev = (float *)(G.tab_dev + G.tab_words - s.len_fds);
            ok = cudaMemcpyAsync(fd_dev, G.fds.data(), s.len_fds * sizeof(float),
                                 cudaMemcpyHostToDevice, st) == cudaSuccess;
        }
        ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
        if (nat) cudaFree(nat);
        if (!ok) {
            cuda_error(cudaGetLastError(), "sdrg_acq_plan_new allocation");
            sdrg_acq_plan_free(plan);
            return nullptr;
        }
        G.res_off = res_off;
        res_off += s.n_prn;
        plan->cells += (int64_t)s.n_prn * s.len_fds * s.Nmax;
    }
    plan->n_res = res_off;
    // the work-list consumer: all groups on the 24 000-point compile-time
    // plan, splits 2 (narrow queue) or 8 (wide queue), at most kMaxWorkGroups
    bool wl = n_sig <= kMaxWorkGroups;
    for (auto &G : plan->g)
        wl = wl && (G.pl->R == 2 || G.pl->R == 8) && Plan24000::matches(G.pl->k, G.pl->threads);
    if (wl && cudaMalloc(&plan->wl_next, 2 * sizeof(int)) != cudaSuccess) {
        cuda_error(cudaGetLastError(), "sdrg_acq_plan_new work list");
        sdrg_acq_plan_free(plan);
        return nullptr;
    }
    plan->wl_ok = wl;
    return plan;
}

void sdrg_acq_plan_free(sdrg_acq_plan_t *plan)
{
    if (!plan) return;
    drop_graph(plan);
    if (plan->cap_stream) {
        cudaStreamSynchronize(plan->cap_stream);
        cudaStreamDestroy(plan->cap_stream);
    }
    for (cudaStream_t s : plan->streams) {
        if (!s) continue;
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    for (auto ev : plan->ev_join) if (ev) cudaEventDestroy(ev);
    if (plan->stage_err) cudaFree(plan->stage_err);
    if (plan->wl_next) cudaFree(plan->wl_next);
    if (plan->ev_fork) cudaEventDestroy(plan->ev_fork);
    for (auto ev : plan->ev_pool) cudaEventDestroy(ev);
    for (auto &u : plan->ev_used) {
        cudaEventDestroy(u.a);
        if (u.b != u.a) cudaEventDestroy(u.b);
    }
    for (auto &G : plan->g) {
        if (G.code) cudaFree(G.code);
        if (G.X) cudaFree(G.X);
        if (G.P) cudaFree(G.P);
        if (G.W) cudaFree(G.W);
        if (G.Q) cudaFree(G.Q);
        if (G.peak_parts) cudaFree(G.peak_parts);
        if (G.tab_dev) cudaFree(G.tab_dev);
        if (G.tab_host) cudaFreeHost(G.tab_host);
        if (G.tab_ev) cudaEventDestroy(G.tab_ev);
    }
    delete plan;
}

int64_t sdrg_acq_plan_cells(const sdrg_acq_plan_t *plan) { return plan ? plan->cells : 0; }

const float *sdrg_acq_grid(const sdrg_acq_plan_t *plan, int g)
{
    if (!plan || g < 0 || g >= (int)plan->g.size()) return nullptr;
    return plan->g[g].P;
}

int sdrg_acq_grid_host(const sdrg_acq_plan_t *plan, int g, float *dst)
{
    if (!plan || g < 0 || g >= (int)plan->g.size() || !dst)
        return set_error(SDRG_ERR_ARG, "sdrg_acq_grid_host: bad argument");
    int e;
    if ((e = ensure_device(nullptr))) return e;
    const sdrg_acq_sig_t &s = plan->g[g].sig;
    SDRG_CUDA(cudaDeviceSynchronize());
    SDRG_CUDA(cudaMemcpy(dst, plan->g[g].P, (size_t)s.n_prn * s.len_fds * s.Nmax * sizeof(float),
                         cudaMemcpyDeviceToHost));
    return SDRG_OK;
}

int sdrg_acq_set_codes(sdrg_acq_plan_t *plan, int g, const int8_t *code_I_dev,
                       const int8_t *code_Q_dev, int len_code, double T, double coff, int N,
                       void *stream)
{
    if (!plan || g < 0 || g >= (int)plan->g.size())
        return set_error(SDRG_ERR_ARG, "sdrg_acq_set_codes: no group %d", g);
    GroupState &G = plan->g[g];
    if (N <= 0 || N > G.sig.L)
        return set_error(SDRG_ERR_ARG, "sdrg_acq_set_codes: replica length %d outside 1..L=%d",
                         N, G.sig.L);
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    cudaStream_t st = (cudaStream_t)stream;
    if (!st && (e = thread_stream(&st))) return e;
    return code_fft_device(code_I_dev, code_Q_dev, len_code, G.sig.n_prn, T, coff, G.sig.fs, N,
                           G.sig.L, 0, G.code, st, G.pl);
}

// Times the consumer (code product + inverse FFT + power accumulation) of a
// synthetic search - 4 PRNs x 8 bins x 4 sums of length L, L/2 offsets kept -
// for every cluster split of L with 256- and 512-thread CTAs (a staged split
// only when L has no cluster split), best of 3 runs after one warm-up, and
// sets L's schedule to the fastest.
int sdrg_fft_autotune(int L, int *R_out, int *threads_out, double *ms_out)
{
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    if (L <= 1) return set_error(SDRG_ERR_ARG, "autotune: bad length %d", L);
    cudaStream_t st;
    if ((e = thread_stream(&st))) return e;
    const int n_prn = 4, n_bin = 8, n_sum = 4, Nmax = L / 2 > 0 ? L / 2 : 1;
    struct Cand { int R, t; };
    std::vector<Cand> cands;
    static const int Rc[] = {1, 2, 3, 4, 5, 6, 8};
    for (int R : Rc)
        if (shape_ok(L, R))
            for (int t : {256, 512}) cands.push_back({R, t});
    float2 *X = nullptr, *code = nullptr, *W = nullptr;
    float *P = nullptr, *Q = nullptr;
    const size_t xb = (size_t)n_bin * n_sum * L * sizeof(float2);
    const size_t cb = (size_t)n_prn * L * sizeof(float2);
    const size_t pb = (size_t)n_prn * n_bin * Nmax * sizeof(float);
    // the cluster splits' power accumulator, for the largest row set (R = 8)
    const size_t qb = (size_t)n_prn * n_bin * (Nmax + 8) * sizeof(float);
    if ((e = alloc_fault("autotune"))) return e;
    if (cudaMalloc(&X, xb) != cudaSuccess || cudaMalloc(&code, cb) != cudaSuccess ||
        cudaMalloc(&P, pb) != cudaSuccess || cudaMalloc(&Q, qb) != cudaSuccess) {
        e = cuda_error(cudaGetLastError(), "autotune buffers");
        cudaFree(X); cudaFree(code); cudaFree(P); cudaFree(Q);
        return e;
    }
    cudaMemsetAsync(X, 0, xb, st);
    cudaMemsetAsync(code, 0, cb, st);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    int bestR = 0, bestT = 0;
    double best = 1e30;
    std::vector<Cand> tried = cands;
    if (tried.empty()) {           // no cluster split: the default (staged) shape
        int R, M;
        FftPlanK k;
        if (plan_shape(L, &R, &M, &k)) tried.push_back({R, 0});
    }
    for (const Cand &cd : tried) {
        const FftPlan *pl = cd.t ? get_plan_shaped(L, cd.R, cd.t) : get_plan(L);
        if (!pl) { sdr_gpu_clear_error(); continue; }
        if (pl->threads > 512) continue;
        ConsArgs ca = {};
        ca.pl = pl->k; ca.tw = pl->tw_dev; ca.split = pl->split_dev; ca.X = X; ca.code = code;
        ca.n_prn = n_prn; ca.n_bin = n_bin; ca.n_sum = n_sum; ca.prn0 = 0;
        ca.scale = 1.0f / L / L; ca.Nmax = Nmax;
        ca.prn_stride = (size_t)n_bin * Nmax; ca.bin_stride = Nmax; ca.accumulate = 0; ca.P = P;
        if ((e = thread_stage_err(&ca.stage_err, st))) break;
        if (pl->R > 1 && pl->R <= 8) {
            ca.Q = Q;
            ca.Mq = (Nmax + pl->R - 1) / pl->R;
        }
        const int wt = staged_chunk(pl, n_prn * n_bin);
        if (wt && !W && cudaMalloc(&W, staged_bytes(pl, wt, 0)) != cudaSuccess) {
            e = cuda_error(cudaGetLastError(), "autotune scratch");
            break;
        }
        double tbest = 1e30;
        bool ok = true;
        for (int rep = 0; rep < 4 && ok; ++rep) {
            cudaEventRecord(a, st);
            ok = launch_consumer<0>(pl, ca, n_prn * n_bin, st, W, wt) == SDRG_OK;
            cudaEventRecord(b, st);
            if (ok && cudaEventSynchronize(b) == cudaSuccess && rep > 0) {
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, a, b);
                tbest = ms < tbest ? ms : tbest;
            }
        }
        if (!ok) { sdr_gpu_clear_error(); continue; }
        if (tbest < best) { best = tbest; bestR = pl->R; bestT = pl->threads; }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaStreamSynchronize(st);
    cudaFree(X); cudaFree(code); cudaFree(P); cudaFree(Q);
    if (W) cudaFree(W);
    if (e) return e;
    if (!bestR) return set_error(SDRG_ERR_ARG, "autotune: no runnable shape for length %d", L);
    if ((e = set_schedule(L, bestR, bestT, best))) return e;
    if (R_out) *R_out = bestR;
    if (threads_out) *threads_out = bestT;
    if (ms_out) *ms_out = best;
    return SDRG_OK;
}

// Start-sample tables of group gi when the read position or length of its
// buffer changed since the last upload: written into the pinned staging
// buffer once the previous upload from it has completed, then copied on st.
static int upload_tables(GroupState &G, const int *len_if, const int *ix, cudaStream_t st)
{
    const sdrg_acq_sig_t &s = G.sig;
    if (G.last_len == len_if[s.buf] && G.last_ix == ix[s.buf]) return SDRG_OK;
    SDRG_CUDA(cudaEventSynchronize(G.tab_ev));   // previous upload done
    group_tables(G, len_if, ix);
    SDRG_CUDA(cudaMemcpyAsync(G.tab_dev, G.tab_host, (G.tab_words - s.len_fds) * 4,
                              cudaMemcpyHostToDevice, st));
    SDRG_CUDA(cudaEventRecord(G.tab_ev, st));
    G.last_len = len_if[s.buf];
    G.last_ix = ix[s.buf];
    return SDRG_OK;
}

static int check_run(const sdrg_acq_plan_t *plan, const int *len_if)
{
    for (size_t gi = 0; gi < plan->g.size(); ++gi) {
        const sdrg_acq_sig_t &s = plan->g[gi].sig;
        if (len_if[s.buf] < s.L)
            return set_error(SDRG_ERR_ARG, "IF buffer %d shorter than L=%d", s.buf, s.L);
    }
    return SDRG_OK;
}

// The launch sequence of one run: fork the internal streams from `caller`,
// every group's forward / consumer / peak kernels on its stream, join back.
// With `ix` the tables are uploaded on the group streams as needed; without
// (graph capture) the caller has uploaded them and no profiling events are
// recorded.
static bool use_worklist(const sdrg_acq_plan_t *plan)
{
    return plan->wl_ok && plan->wl_mode != 0;
}

// The forward arguments of group G on IF buffer if_dev[G.sig.buf].
static FwdArgs group_fwd_args(const GroupState &G, const Device *dev,
                              const uint8_t *const *if_dev, const int *len_if)
{
    const sdrg_acq_sig_t &s = G.sig;
    const int nb = s.len_fds, ns = s.n_sum;
    FwdArgs fa = {};
    fa.pl = G.pl->k; fa.tw = G.pl->tw_dev; fa.ctab = dev->ctab_dev; fa.R = G.pl->R;
    fa.n_bin = nb; fa.n_sum = ns; fa.cscale = kCScale;
    fa.buf = if_dev[s.buf]; fa.buf_len = len_if[s.buf];
    fa.phstep = G.tab_dev; fa.ph0a = G.tab_dev + nb; fa.ph0b = G.tab_dev + 2 * nb;
    fa.ix = (const int *)(G.tab_dev + 2 * nb + (size_t)nb * ns);
    fa.nsplit = fa.ix + ns;
    fa.X = G.X;
    return fa;
}

// The run as a work list, on the caller's stream: one forward launch for
// every group, the persistent consumer over every group's tasks (plus a
// drain launch of regular 8-CTA clusters, which finds the queues empty
// unless no 8-CTA cluster formed in the first), then each group's peaks.
// Kernel timing (profiling) goes to group 0's forward and consumer entries.
static int launch_run_worklist(sdrg_acq_plan_t *plan, Device *dev, const uint8_t *const *if_dev,
                               const int *len_if, const int *ix, sdrg_acq_result_t *res_dev,
                               cudaStream_t caller)
{
    int e;
    const int ng = (int)plan->g.size();
    const FftPlan *pl0 = plan->g[0].pl;
    static bool attr_set = false;
    if (!attr_set) {
        SDRG_CUDA(cudaFuncSetAttribute(fwd_multi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)g_smem_limit()));
        cudaFuncAttributes fa;
        SDRG_CUDA(cudaFuncGetAttributes(&fa, work_cons_kernel));
        SDRG_CUDA(cudaFuncSetAttribute(work_cons_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(g_smem_limit() - fa.sharedSizeBytes)));
        attr_set = true;
    }
    FwdMulti fm = {};
    fm.n_group = ng;
    WorkArgs wa = {};
    wa.pl = pl0->k; wa.tw = pl0->tw_dev; wa.n_group = ng; wa.next = plan->wl_next;
    wa.err = plan->stage_err;
    for (int gi = 0; gi < ng; ++gi) {
        GroupState &G = plan->g[gi];
        const sdrg_acq_sig_t &s = G.sig;
        if (ix && (e = upload_tables(G, len_if, ix, caller))) return e;
        fm.g[gi] = group_fwd_args(G, dev, if_dev, len_if);
        fm.blk0[gi + 1] = fm.blk0[gi] + s.len_fds * s.n_sum * G.pl->R;
        WorkGroup &W = wa.g[gi];
        W.split = G.pl->split_dev; W.X = G.X; W.code = G.code; W.P = G.P; W.Q = G.Q;
        W.R = G.pl->R; W.n_prn = s.n_prn; W.n_bin = s.len_fds; W.n_sum = s.n_sum;
        W.Nmax = s.Nmax; W.Mq = G.Mq; W.q_by_sm = G.q_by_sm;
        W.prn_stride = (size_t)s.len_fds * s.Nmax;
        W.bin_stride = s.Nmax; W.scale = 1.0f / s.L / s.L;
        const int q = W.R == 8 ? 0 : 1;
        W.task0 = wa.n_task[q];
        wa.n_task[q] += s.n_prn * s.len_fds;
    }
    cudaEvent_t ev[2];
    if ((e = prof_begin(plan, caller, ev))) return e;
    fwd_multi_kernel<<<fm.blk0[ng], pl0->threads, pl0->smem, caller>>>(fm);
    SDRG_CUDA(cudaGetLastError());
    int n_fwd = 1;
    for (int gi = 0; gi < ng; ++gi) {
        GroupState &G = plan->g[gi];
        if ((e = launch_xcomb(G.pl, G.X, G.sig.len_fds * G.sig.n_sum, caller, &wa.g[gi].x_comb)))
            return e;
        n_fwd += wa.g[gi].x_comb;
    }
    if ((e = prof_end(plan, caller, ev, 0, n_fwd))) return e;

    if ((e = prof_begin(plan, caller, ev))) return e;
    SDRG_CUDA(cudaMemsetAsync(plan->wl_next, 0, 2 * sizeof(int), caller));
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(pl0->threads);
    cfg.dynamicSmemBytes = pl0->smem;
    cfg.stream = caller;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2; attr[0].val.clusterDim.y = 1; attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributePreferredClusterDimension;
    attr[1].val.preferredClusterDim.x = 8; attr[1].val.preferredClusterDim.y = 1;
    attr[1].val.preferredClusterDim.z = 1;
    cfg.attrs = attr;
    // one CTA per SM (shared memory), a whole number of 8-CTA clusters
    cfg.gridDim = dim3((unsigned)((dev->sm_count + 7) / 8 * 8));
    cfg.numAttrs = 2;
    SDRG_CUDA(cudaLaunchKernelEx(&cfg, work_cons_kernel, wa));
    // drain: regular 8-CTA clusters take whatever is left (normally nothing)
    attr[0].val.clusterDim.x = 8;
    cfg.gridDim = dim3((unsigned)(dev->sm_count / 8 * 8 > 0 ? dev->sm_count / 8 * 8 : 8));
    cfg.numAttrs = 1;
    SDRG_CUDA(cudaLaunchKernelEx(&cfg, work_cons_kernel, wa));
    if ((e = prof_end(plan, caller, ev, 1, 2))) return e;

    for (int gi = 0; gi < ng; ++gi) {
        GroupState &G = plan->g[gi];
        const sdrg_acq_sig_t &s = G.sig;
        const int nb = s.len_fds;
        const float *fd_dev = (const float *)(G.tab_dev + G.tab_words - nb);
        if ((e = prof_begin(plan, caller, ev))) return e;
        if ((e = launch_peaks(G.P, s.n_prn, nb, s.Nmax, s.Nmax, (size_t)nb * s.Nmax, s.T,
                              fd_dev, res_dev + G.res_off, G.peak_parts, caller)))
            return e;
        if ((e = prof_end(plan, caller, ev, 3 * gi + 2, 2))) return e;
    }
    return SDRG_OK;
}

static int launch_run(sdrg_acq_plan_t *plan, Device *dev, const uint8_t *const *if_dev,
                      const int *len_if, const int *ix, sdrg_acq_result_t *res_dev,
                      cudaStream_t caller)
{
    int e;
    const bool prof = plan->prof && ix;
    if (prof) {
        cudaEvent_t r[2];
        if ((e = prof_begin(plan, caller, r))) return e;   // records r[0]
        plan->ev_pool.push_back(r[1]);
        plan->ev_used.push_back({-1, plan->run, r[0], r[0]});
    }
    const bool saved = plan->prof;
    plan->prof = prof;
    struct Restore { sdrg_acq_plan_t *p; bool v; ~Restore() { p->prof = v; } } restore{plan, saved};
    if (use_worklist(plan)) return launch_run_worklist(plan, dev, if_dev, len_if, ix, res_dev, caller);
    // fork: every internal stream starts after the caller's prior work
    SDRG_CUDA(cudaEventRecord(plan->ev_fork, caller));
    for (cudaStream_t s2 : plan->streams) SDRG_CUDA(cudaStreamWaitEvent(s2, plan->ev_fork, 0));
    for (size_t gi = 0; gi < plan->g.size(); ++gi) {
        GroupState &G = plan->g[gi];
        const sdrg_acq_sig_t &s = G.sig;
        cudaStream_t st = plan->streams[gi % plan->streams.size()];
        if (ix && (e = upload_tables(G, len_if, ix, st))) return e;
        const int nb = s.len_fds, ns = s.n_sum;
        FwdArgs fa = {};
        fa.pl = G.pl->k; fa.tw = G.pl->tw_dev; fa.ctab = dev->ctab_dev; fa.R = G.pl->R;
        fa.n_bin = nb; fa.n_sum = ns; fa.cscale = kCScale;
        fa.buf = if_dev[s.buf]; fa.buf_len = len_if[s.buf];
        fa.phstep = G.tab_dev; fa.ph0a = G.tab_dev + nb; fa.ph0b = G.tab_dev + 2 * nb;
        fa.ix = (const int *)(G.tab_dev + 2 * nb + (size_t)nb * ns);
        fa.nsplit = fa.ix + ns;
        fa.X = G.X;
        cudaEvent_t ev[2];
        if ((e = prof_begin(plan, st, ev))) return e;
        if ((e = launch_fwd<0>(G.pl, fa, nb * ns * G.pl->R, st))) return e;
        int xc = 0;
        if ((e = launch_xcomb(G.pl, G.X, nb * ns, st, &xc))) return e;
        if ((e = prof_end(plan, st, ev, 3 * (int)gi + 0, 1 + xc))) return e;
        ConsArgs ca = {};
        ca.x_comb = xc;
        ca.pl = G.pl->k; ca.tw = G.pl->tw_dev; ca.split = G.pl->split_dev; ca.X = G.X;
        ca.code = G.code; ca.n_prn = s.n_prn; ca.n_bin = nb; ca.n_sum = ns; ca.prn0 = 0;
        ca.scale = 1.0f / s.L / s.L; ca.Nmax = s.Nmax;
        ca.prn_stride = (size_t)nb * s.Nmax; ca.bin_stride = s.Nmax;
        ca.accumulate = 0; ca.P = G.P; ca.Q = G.Q; ca.Mq = G.Mq; ca.q_by_sm = G.q_by_sm;
        ca.stage_err = plan->stage_err;
        if ((e = prof_begin(plan, st, ev))) return e;
        if ((e = launch_consumer<0>(G.pl, ca, s.n_prn * nb, st, G.W, G.w_tasks))) return e;
        // a staged split launches a combine and an inverse pass per chunk and sum
        const int n_cons = G.pl->R <= 8 ? 1
            : 2 * ns * ((s.n_prn * nb + G.w_tasks - 1) / G.w_tasks);
        if ((e = prof_end(plan, st, ev, 3 * (int)gi + 1, n_cons))) return e;
        const float *fd_dev = (const float *)(G.tab_dev + G.tab_words - nb);
        if ((e = prof_begin(plan, st, ev))) return e;
        if ((e = launch_peaks(G.P, s.n_prn, nb, s.Nmax, s.Nmax, (size_t)nb * s.Nmax, s.T,
                              fd_dev, res_dev + G.res_off, G.peak_parts, st)))
            return e;
        if ((e = prof_end(plan, st, ev, 3 * (int)gi + 2, 2))) return e;
    }
    // join: the caller's stream continues after every group
    for (size_t i = 0; i < plan->streams.size(); ++i) {
        SDRG_CUDA(cudaEventRecord(plan->ev_join[i], plan->streams[i]));
        SDRG_CUDA(cudaStreamWaitEvent(caller, plan->ev_join[i], 0));
    }
    return SDRG_OK;
}

int sdrg_acq_run(sdrg_acq_plan_t *plan, const uint8_t *const *if_dev, const int *len_if,
                 const int *ix, sdrg_acq_result_t *res_dev, void *stream)
{
    if (!plan || !if_dev || !len_if || !ix || !res_dev)
        return set_error(SDRG_ERR_ARG, "sdrg_acq_run: null argument");
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    cudaStream_t caller = (cudaStream_t)stream;
    if (!caller && (e = thread_stream(&caller))) return e;
    if ((e = check_run(plan, len_if))) return e;
    if ((e = launch_run(plan, dev, if_dev, len_if, ix, res_dev, caller))) return e;
    plan->run++;
    return SDRG_OK;
}

// The buffers a captured graph was made for: kernel arguments hold the IF
// pointers and lengths and the result pointer, the tables hold the rest.
static std::vector<intptr_t> graph_key(const sdrg_acq_plan_t *plan, const uint8_t *const *if_dev,
                                       const int *len_if, const sdrg_acq_result_t *res_dev)
{
    int nbuf = 0;
    for (auto &G : plan->g) nbuf = G.sig.buf + 1 > nbuf ? G.sig.buf + 1 : nbuf;
    std::vector<intptr_t> k;
    k.push_back((intptr_t)res_dev);
    for (int b = 0; b < nbuf; ++b) {
        k.push_back((intptr_t)if_dev[b]);
        k.push_back((intptr_t)len_if[b]);
    }
    return k;
}

static int capture_graph(sdrg_acq_plan_t *plan, Device *dev, const uint8_t *const *if_dev,
                         const int *len_if, sdrg_acq_result_t *res_dev)
{
    drop_graph(plan);
    if (!plan->cap_stream)
        SDRG_CUDA(cudaStreamCreateWithFlags(&plan->cap_stream, cudaStreamNonBlocking));
    SDRG_CUDA(cudaStreamBeginCapture(plan->cap_stream, cudaStreamCaptureModeRelaxed));
    int e = launch_run(plan, dev, if_dev, len_if, nullptr, res_dev, plan->cap_stream);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(plan->cap_stream, &graph);
    if (e) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return e;
    }
    if (ce != cudaSuccess) return cuda_error(ce, "sdrg_acq_run_graph: capture");
    const cudaError_t ie = cudaGraphInstantiate(&plan->graph_exec, graph, 0);
    if (ie != cudaSuccess) {
        cudaGraphDestroy(graph);
        plan->graph_exec = nullptr;
        return cuda_error(ie, "sdrg_acq_run_graph: instantiate");
    }
    plan->graph = graph;
    plan->graph_key = graph_key(plan, if_dev, len_if, res_dev);
    return SDRG_OK;
}

int sdrg_acq_run_graph(sdrg_acq_plan_t *plan, const uint8_t *const *if_dev, const int *len_if,
                       const int *ix, sdrg_acq_result_t *res_dev, void *stream)
{
    if (!plan || !if_dev || !len_if || !ix || !res_dev)
        return set_error(SDRG_ERR_ARG, "sdrg_acq_run_graph: null argument");
    Device *dev;
    int e;
    if ((e = ensure_device(&dev))) return e;
    cudaStream_t caller = (cudaStream_t)stream;
    if (!caller && (e = thread_stream(&caller))) return e;
    if ((e = check_run(plan, len_if))) return e;
    if (!plan->graph_exec || plan->graph_key != graph_key(plan, if_dev, len_if, res_dev)) {
        if ((e = capture_graph(plan, dev, if_dev, len_if, res_dev))) return e;
        ++plan->graph_captures;
    }
    // tables first, on the caller's stream, ordered before the replay
    for (auto &G : plan->g)
        if ((e = upload_tables(G, len_if, ix, caller))) return e;
    SDRG_CUDA(cudaGraphLaunch(plan->graph_exec, caller));
    plan->run++;
    return SDRG_OK;
}

int sdrg_acq_set_worklist(sdrg_acq_plan_t *plan, int mode)
{
    if (!plan || mode < -1 || mode > 1)
        return set_error(SDRG_ERR_ARG, "sdrg_acq_set_worklist: bad argument");
    if (mode == 1 && !plan->wl_ok)
        return set_error(SDRG_ERR_ARG, "sdrg_acq_set_worklist: the plan's groups are not all on "
                         "the 24 000-point plan with split 2 or 8");
    if (mode != plan->wl_mode) drop_graph(plan);
    plan->wl_mode = mode;
    return use_worklist(plan) ? 1 : 0;
}

int sdrg_acq_graph_captures(const sdrg_acq_plan_t *plan)
{
    return plan ? plan->graph_captures : 0;
}

int sdrg_acq_run_host(sdrg_acq_plan_t *plan, const uint8_t *const *if_host, const int *len_if,
                      const int *ix, sdrg_acq_result_t *res_host)
{
    if (!plan || !if_host || !len_if || !ix || !res_host)
        return set_error(SDRG_ERR_ARG, "sdrg_acq_run_host: null argument");
    int e;
    if ((e = ensure_device(nullptr))) return e;
    cudaStream_t st;
    if ((e = thread_stream(&st))) return e;
    int nbuf = 0;
    for (auto &G : plan->g) nbuf = G.sig.buf + 1 > nbuf ? G.sig.buf + 1 : nbuf;
    std::vector<uint8_t *> bufs(nbuf, nullptr);
    sdrg_acq_result_t *res_dev = nullptr;
    e = SDRG_OK;
    for (int b = 0; b < nbuf && !e; ++b) {
        if (cudaMalloc(&bufs[b], len_if[b]) != cudaSuccess ||
            cudaMemcpyAsync(bufs[b], if_host[b], len_if[b], cudaMemcpyHostToDevice, st) != cudaSuccess)
            e = cuda_error(cudaGetLastError(), "sdrg_acq_run_host IF upload");
    }
    if (!e && cudaMalloc(&res_dev, plan->n_res * sizeof(sdrg_acq_result_t)) != cudaSuccess)
        e = cuda_error(cudaGetLastError(), "sdrg_acq_run_host result alloc");
    if (!e) e = sdrg_acq_run(plan, (const uint8_t *const *)bufs.data(), len_if, ix, res_dev, st);
    if (!e && (cudaMemcpyAsync(res_host, res_dev, plan->n_res * sizeof(sdrg_acq_result_t),
                               cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess))
        e = cuda_error(cudaGetLastError(), "sdrg_acq_run_host D2H");
    cudaStreamSynchronize(st);
    if (!e && use_worklist(plan)) e = stage_wait_check(nullptr, plan->stage_err, st, true);
    for (size_t gi = 0; gi < plan->g.size() && !e; ++gi)
        e = stage_wait_check(plan->g[gi].pl, plan->stage_err, st);
    for (auto p : bufs) if (p) cudaFree(p);
    if (res_dev) cudaFree(res_dev);
    return e;
}

} // extern "C"

// ---------------------------------------------------------------------------
// FFT correlator that allocates nothing (sdrg_corr_fft_noalloc)
// ---------------------------------------------------------------------------
namespace sdrg {

// Largest sub-transform held by one CTA, and the fixed scratch layout:
// permuted code DFT (N) | forward spectrum (N) | twiddles (2 * kNaMaxM) |
// digit-reversal map (kNaMaxM ints) | split twiddles (kNaMaxM).
constexpr int kNaMaxN = SDRG_NOALLOC_MAX_N;
constexpr int kNaMaxM = 28672;
constexpr size_t kNaCode = 0;
constexpr size_t kNaX = kNaCode + (size_t)kNaMaxN * sizeof(float2);
constexpr size_t kNaTw = kNaX + (size_t)kNaMaxN * sizeof(float2);
constexpr size_t kNaKperm = kNaTw + (size_t)2 * kNaMaxM * sizeof(float2);
constexpr size_t kNaSplit = kNaKperm + (size_t)kNaMaxM * sizeof(int);
constexpr size_t kNaBytes = kNaSplit + (size_t)kNaMaxM * sizeof(float2);

// Every GPU that loads the library holds this array until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

// Device address of g_noalloc_scratch per device, looked up once with that
// device current (the host-side symbol is not a device address).
static std::mutex g_na_mtx;
static unsigned char *g_na_base[64];

// The FFT tables of a length-N plan with pass structure k, written into the
// fixed array by every call (so a call, or a CUDA-graph replay of one, never
// meets another length's tables): the same values get_plan builds on the
// host - per-pass twiddles exp(-2 pi i (i j mod Ls) / Ls), the digit-reversed
// frequency index k(q) of each DIF output position and the split twiddles
// exp(+2 pi i k(q) / N) - from double sincospi, rounded to float.
__global__ void __launch_bounds__(256) na_tables_kernel(FftPlanK k, int N, float2 *tw,
                                                        int *kperm, float2 *split)
{
    const int total = k.twtot + k.M;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        if (t < k.twtot) {
            int p = 0;
            while (p + 1 < k.npass && t >= k.twoff[p + 1]) ++p;
            const int Ls = k.Ls[p], S = Ls / k.radix[p], loc = t - k.twoff[p];
            const int j = loc / S + 1, i = loc - (j - 1) * S;
            const long e = (long)i * j % Ls;
            double sn, cs;
            sincospi(-2.0 * (double)e / Ls, &sn, &cs);
            tw[t] = make_float2((float)cs, (float)sn);
        } else {
            const int q = t - k.twtot;
            int rem = q, blk = k.M, kk = 0, mul = 1;
            for (int p = 0; p < k.npass; ++p) {
                blk /= k.radix[p];
                const int j = rem / blk;
                rem -= j * blk;
                kk += j * mul;
                mul *= k.radix[p];
            }
            kperm[q] = kk;
            double sn, cs;
            sincospi(2.0 * (double)kk / N, &sn, &cs);
            split[q] = make_float2((float)cs, (float)sn);
        }
    }
}

} // namespace sdrg

extern "C" int sdrg_corr_fft_noalloc(const sdr_cpx16_t *IQ_dev, const sdr_cpx_t *code_fft_dev,
                                     int N, sdr_cpx_t *corr_dev, void *stream)
{
    if (N <= 0 || N > kNaMaxN)
        return set_error(SDRG_ERR_ARG, "sdrg_corr_fft_noalloc: N=%d outside 1..%d", N, kNaMaxN);
    if (!IQ_dev || !code_fft_dev || !corr_dev)
        return set_error(SDRG_ERR_ARG, "sdrg_corr_fft_noalloc: null pointer");
    // the default cluster split of N (schedules do not apply here)
    FftPlan pl;
    int R, M;
    FftPlanK k;
    if (!cluster_shape(N, &R, &M, &k) || M > kNaMaxM || k.twtot > 2 * kNaMaxM)
        return set_error(SDRG_ERR_ARG, "sdrg_corr_fft_noalloc: length %d has no plan "
                         "within the fixed scratch", N);
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    SDRG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(SDRG_ERR_ARG, "device %d out of range", dev);
    unsigned char *base;
    {
        std::lock_guard<std::mutex> lk(g_na_mtx);
        if (!g_na_base[dev]) {
            // set-up, once per device, with that device current
            void *p = nullptr;
            SDRG_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
            g_na_base[dev] = (unsigned char *)p;
        }
        base = g_na_base[dev];
    }
    pl.L = N; pl.R = R; pl.M = M; pl.k = k;
    int t = 32;
    while (t < 512 && t * 8 < M) t *= 2;
    pl.threads = t;
    pl.smem = (size_t)M * sizeof(float2) + (size_t)k.twtot * sizeof(float2) + 512;
    pl.tw_dev = (float2 *)(base + kNaTw);
    pl.kperm_dev = (int *)(base + kNaKperm);
    pl.split_dev = (float2 *)(base + kNaSplit);
    const int nt = k.twtot + M;
    na_tables_kernel<<<(nt + 255) / 256, 256, 0, st>>>(k, N, pl.tw_dev, pl.kperm_dev, pl.split_dev);
    SDRG_CUDA(cudaGetLastError());
    float2 *code_perm = (float2 *)(base + kNaCode);
    float2 *X = (float2 *)(base + kNaX);
    int e;
    if ((e = perm_code(&pl, (const float2 *)code_fft_dev, 1, code_perm, st))) return e;
    FwdArgs fa = {};
    fa.pl = pl.k; fa.tw = pl.tw_dev; fa.ctab = nullptr; fa.R = pl.R;
    fa.n_bin = 1; fa.n_sum = 1; fa.cscale = kCScale; fa.iq = (const char2 *)IQ_dev; fa.X = X;
    if ((e = launch_fwd<1>(&pl, fa, pl.R, st))) return e;
    ConsArgs ca = {};
    ca.pl = pl.k; ca.tw = pl.tw_dev; ca.split = pl.split_dev; ca.X = X;
    ca.code = code_perm; ca.n_prn = 1; ca.n_bin = 1; ca.n_sum = 1; ca.prn0 = 0;
    ca.scale = 1.0f / N / N; ca.Nmax = N; ca.Y = (float2 *)corr_dev;
    return launch_cons<1>(&pl, ca, 1, st);
}
