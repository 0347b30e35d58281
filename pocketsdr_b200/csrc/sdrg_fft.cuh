// sdrg_fft.cuh - shared-memory mixed-radix FFT for one CTA (sm_100a).
//
// One CTA transforms M <= ~27K complex floats held in shared memory.
//   forward : decimation in frequency (DIF), natural-order input, output in
//             mixed-radix digit-reversed positions;
//   inverse : decimation in time (DIT), input in those digit-reversed
//             positions, natural-order output, unnormalised (exp(+i)).
// A forward DIF followed by the inverse DIT therefore needs no reordering:
// the frequency-domain product is formed directly in the permuted order,
// with the code DFT stored permuted once at plan time.
//
// Pass p works on sub-sequences of length Ls_p = M / (r_0 ... r_{p-1}); a
// butterfly reads r_p elements at stride S_p = Ls_p / r_p, so butterflies
// never overlap and each pass runs in place with one barrier after it.
// Twiddles: pass 0 uses w = exp(-2 pi i * i / Ls_0) from a table of S_0
// entries and forms w^j by repeated products; every later pass reads all of
// its twiddles from a table of S_p * (r_p - 1) entries.
// Butterfly kernels are compile-time DFTs of size 2,3,4,5 and Cooley-Tukey
// composites of them (6,8,10,12,15,16) with constant twiddles.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sdrg {

constexpr int kMaxPass = 8;

// ---- compile-time trigonometry (Taylor series, double) --------------------
__host__ __device__ constexpr double cx_pi() { return 3.14159265358979323846; }

__host__ __device__ constexpr double cx_sin(double x)
{
    double term = x, sum = x;
    for (int n = 1; n < 24; ++n) {
        term *= -x * x / ((2.0 * n) * (2.0 * n + 1.0));
        sum += term;
    }
    return sum;
}

__host__ __device__ constexpr double cx_cos(double x)
{
    double term = 1.0, sum = 1.0;
    for (int n = 1; n < 24; ++n) {
        term *= -x * x / ((2.0 * n - 1.0) * (2.0 * n));
        sum += term;
    }
    return sum;
}

// exp(dir * 2 pi i * e / n) with the angle folded into [-pi, pi]
template <int N, int DIR>
struct TwConst {
    float c[N], s[N];
    __host__ __device__ constexpr TwConst() : c(), s()
    {
        for (int e = 0; e < N; ++e) {
            int ee = (e <= N / 2) ? e : e - N;
            double a = DIR * 2.0 * cx_pi() * ee / N;
            c[e] = (float)cx_cos(a);
            s[e] = (float)cx_sin(a);
        }
    }
};

// ---- complex helpers --------------------------------------------------------
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// multiply by dir*i (dir=+1: i, dir=-1: -i)
template <int DIR>
__device__ __forceinline__ float2 cmul_i(float2 a)
{
    return DIR > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// ---- in-register DFTs, natural order in and out ---------------------------
// DIR = -1: forward (exp(-i)), DIR = +1: backward (exp(+i)).
template <int N, int DIR> struct Dft;

template <int DIR> struct Dft<1, DIR> {
    __device__ __forceinline__ static void run(float2 *) {}
};

template <int DIR> struct Dft<2, DIR> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <int DIR> struct Dft<3, DIR> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        const float c = 0.86602540378443864676f; // sqrt(3)/2
        float2 s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
        float2 a = make_float2(v[0].x - 0.5f * s.x, v[0].y - 0.5f * s.y);
        float2 t = cmul_i<DIR>(make_float2(c * d.x, c * d.y));
        v[0] = cadd(v[0], s);
        v[1] = cadd(a, t);
        v[2] = csub(a, t);
    }
};

template <int DIR> struct Dft<4, DIR> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        float2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        float2 c = cadd(v[1], v[3]), d = cmul_i<DIR>(csub(v[1], v[3]));
        v[0] = cadd(a, c);
        v[2] = csub(a, c);
        v[1] = cadd(b, d);
        v[3] = csub(b, d);
    }
};

template <int DIR> struct Dft<5, DIR> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        const float c1 = 0.30901699437494742410f;  // cos(2pi/5)
        const float c2 = -0.80901699437494742410f; // cos(4pi/5)
        const float s1 = 0.95105651629515357212f;  // sin(2pi/5)
        const float s2 = 0.58778525229247312917f;  // sin(4pi/5)
        float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        float2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        float2 x0 = v[0];
        float2 a1 = make_float2(x0.x + c1 * t1.x + c2 * t2.x, x0.y + c1 * t1.y + c2 * t2.y);
        float2 a2 = make_float2(x0.x + c2 * t1.x + c1 * t2.x, x0.y + c2 * t1.y + c1 * t2.y);
        float2 b1 = make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
        float2 b2 = make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
        b1 = cmul_i<DIR>(b1);
        b2 = cmul_i<DIR>(b2);
        v[0] = cadd(x0, cadd(t1, t2));
        v[1] = cadd(a1, b1);
        v[4] = csub(a1, b1);
        v[2] = cadd(a2, b2);
        v[3] = csub(a2, b2);
    }
};

// Cooley-Tukey composite N = A*B: n = B*n1 + n2, k = k1 + A*k2.
template <int A, int B, int DIR>
struct DftCT {
    static constexpr int N = A * B;
    __device__ __forceinline__ static void run(float2 *v)
    {
        constexpr TwConst<N, DIR> tw{};
        float2 y[N];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) {
            float2 t[A];
#pragma unroll
            for (int n1 = 0; n1 < A; ++n1) t[n1] = v[B * n1 + n2];
            Dft<A, DIR>::run(t);
#pragma unroll
            for (int k1 = 0; k1 < A; ++k1) {
                const int e = (n2 * k1) % N;
                // quarter turns are exact rotations (no multiplication)
                if (e == 0) {
                    y[n2 * A + k1] = t[k1];
                } else if (4 * e == N) {
                    y[n2 * A + k1] = cmul_i<DIR>(t[k1]);
                } else if (2 * e == N) {
                    y[n2 * A + k1] = make_float2(-t[k1].x, -t[k1].y);
                } else if (4 * e == 3 * N) {
                    y[n2 * A + k1] = cmul_i<-DIR>(t[k1]);
                } else {
                    y[n2 * A + k1] = cmul(t[k1], make_float2(tw.c[e], tw.s[e]));
                }
            }
        }
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) {
            float2 t[B];
#pragma unroll
            for (int n2 = 0; n2 < B; ++n2) t[n2] = y[n2 * A + k1];
            Dft<B, DIR>::run(t);
#pragma unroll
            for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = t[k2];
        }
    }
};

template <int DIR> struct Dft<6, DIR>  : DftCT<2, 3, DIR> {};
template <int DIR> struct Dft<8, DIR>  : DftCT<2, 4, DIR> {};
template <int DIR> struct Dft<10, DIR> : DftCT<2, 5, DIR> {};
template <int DIR> struct Dft<12, DIR> : DftCT<4, 3, DIR> {};
template <int DIR> struct Dft<15, DIR> : DftCT<3, 5, DIR> {};
template <int DIR> struct Dft<16, DIR> : DftCT<4, 4, DIR> {};
template <int DIR> struct Dft<20, DIR> : DftCT<4, 5, DIR> {};   // staged splits only

// ---- kernel-side plan --------------------------------------------------------
struct FftPlanK {
    int M;                  // transform length held by one CTA
    int npass;
    int radix[kMaxPass];    // DIF order
    int Ls[kMaxPass];       // sub-sequence length at pass p
    int twoff[kMaxPass];    // offset of pass p's table in the twiddle array
    int twtot;              // total twiddle entries (sum of S_p)
};

// Runs fn<R>() for the runtime radix r (instantiates every supported radix).
#define SDRG_RADIX_DISPATCH(r, CALL)            \
    switch (r) {                                \
    case 1:  { constexpr int R_ = 1;  CALL; } break;  \
    case 2:  { constexpr int R_ = 2;  CALL; } break;  \
    case 3:  { constexpr int R_ = 3;  CALL; } break;  \
    case 4:  { constexpr int R_ = 4;  CALL; } break;  \
    case 5:  { constexpr int R_ = 5;  CALL; } break;  \
    case 6:  { constexpr int R_ = 6;  CALL; } break;  \
    case 8:  { constexpr int R_ = 8;  CALL; } break;  \
    case 10: { constexpr int R_ = 10; CALL; } break;  \
    case 12: { constexpr int R_ = 12; CALL; } break;  \
    case 15: { constexpr int R_ = 15; CALL; } break;  \
    case 16: { constexpr int R_ = 16; CALL; } break;  \
    default: break;                             \
    }

// Twiddle powers w^1..w^(R-1) applied to v[1..R-1]
template <int R>
__device__ __forceinline__ void apply_tw(float2 *v, float2 w1)
{
    float2 w = w1;
#pragma unroll
    for (int j = 1; j < R; ++j) {
        v[j] = cmul(v[j], w);
        if (j + 1 < R) w = cmul(w, w1);
    }
}

// Per-thread walk over the butterflies of a pass without a division per
// butterfly: butterfly b = blk*S + i; the thread starts at b = tid and
// advances by nthr = dblk*S + di.
struct BflyWalk {
    int blk, i, dblk, di, S;
    __device__ __forceinline__ BflyWalk(int tid, int nthr, int S_) : S(S_)
    {
        blk = tid / S; i = tid - blk * S;
        dblk = nthr / S; di = nthr - dblk * S;
    }
    __device__ __forceinline__ void next()
    {
        blk += dblk; i += di;
        if (i >= S) { i -= S; ++blk; }
    }
};

// Pass tables for p >= 1 hold every twiddle: twp[(j-1)*S + i] =
// exp(-2 pi i * i*j / Ls), j = 1..R-1, so consecutive threads read
// consecutive entries.
template <int R, bool CONJ>
__device__ __forceinline__ void apply_tw_table(float2 *v, const float2 *twp, int S, int i)
{
#pragma unroll
    for (int j = 1; j < R; ++j) {
        const float2 w = twp[(j - 1) * S + i];
        v[j] = cmul(v[j], CONJ ? cconj(w) : w);
    }
}

// One in-place inner pass (p >= 1): DIF forward (FWD: DFT, then twiddles) or
// DIT inverse (conjugate twiddles, then backward DFT). Radices up to 10 take
// two butterflies per iteration (loads of both issued before either DFT) for
// instruction-level parallelism; a pass with stride 1 has unit twiddles.
template <int R, bool FWD>
__device__ __forceinline__ void bfly_inner(float2 *v, const float2 *twp, int S, int i)
{
    if (FWD) {
        Dft<R, -1>::run(v);
        if (S > 1) apply_tw_table<R, false>(v, twp, S, i);
    } else {
        if (S > 1) apply_tw_table<R, true>(v, twp, S, i);
        Dft<R, 1>::run(v);
    }
}

template <int R, bool FWD>
__device__ __forceinline__ void inner_pass(float2 *sm, int M, int Ls, const float2 *twp,
                                           int tid, int nthr)
{
    constexpr int U = R <= 10 ? 2 : 1;
    const int S = Ls / R, nb = M / R;
    BflyWalk w(tid, nthr, S);
    int b = tid;
    for (; b + (U - 1) * nthr < nb; b += U * nthr) {
        float2 v[U][R];
        float2 *p[U];
        int ii[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            p[u] = sm + w.blk * Ls + w.i;
            ii[u] = w.i;
            w.next();
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int j = 0; j < R; ++j) v[u][j] = p[u][j * S];
#pragma unroll
        for (int u = 0; u < U; ++u) bfly_inner<R, FWD>(v[u], twp, S, ii[u]);
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int j = 0; j < R; ++j) p[u][j * S] = v[u][j];
    }
    for (; b < nb; b += nthr, w.next()) {
        float2 v[R];
        float2 *p = sm + w.blk * Ls + w.i;
#pragma unroll
        for (int j = 0; j < R; ++j) v[j] = p[j * S];
        bfly_inner<R, FWD>(v, twp, S, w.i);
#pragma unroll
        for (int j = 0; j < R; ++j) p[j * S] = v[j];
    }
}

template <int R>
__device__ __forceinline__ void dif_pass(float2 *sm, int M, int Ls, const float2 *twp,
                                         int tid, int nthr)
{
    inner_pass<R, true>(sm, M, Ls, twp, tid, nthr);
}

template <int R>
__device__ __forceinline__ void dit_pass(float2 *sm, int M, int Ls, const float2 *twp,
                                         int tid, int nthr)
{
    inner_pass<R, false>(sm, M, Ls, twp, tid, nthr);
}

// First DIF pass fused with the input: element m comes from load(m).
template <int R, class Load>
__device__ __forceinline__ void dif_pass0_load(float2 *sm, int M,
                                               const float2 *twp, Load &load,
                                               int tid, int nthr)
{
    const int S = M / R;
    for (int i = tid; i < S; i += nthr) {
        float2 v[R];
#pragma unroll
        for (int j = 0; j < R; ++j) v[j] = load(i + j * S);
        Dft<R, -1>::run(v);
        if (i) apply_tw<R>(v, twp[i]);
#pragma unroll
        for (int j = 0; j < R; ++j) sm[i + j * S] = v[j];
    }
}

// Last DIT pass fused with the output: store(m, y_m, old_m) for natural
// index m, where old_m = store.pre(m) is fetched before the butterfly so a
// global read-modify-write overlaps the shared-memory work.
template <int R, class Store>
__device__ __forceinline__ void dit_pass0_store(const float2 *sm, int M,
                                                const float2 *twp, Store &store,
                                                int tid, int nthr)
{
    const int S = M / R;
    for (int i = tid; i < S; i += nthr) {
        typename Store::Old old[R];
#pragma unroll
        for (int j = 0; j < R; ++j) old[j] = store.pre(i + j * S);
        float2 v[R];
#pragma unroll
        for (int j = 0; j < R; ++j) v[j] = sm[i + j * S];
        if (i) apply_tw<R>(v, cconj(twp[i]));
        Dft<R, 1>::run(v);
#pragma unroll
        for (int j = 0; j < R; ++j) store(i + j * S, v[j], old[j]);
    }
}

// Full forward transform: pass 0 fused with load(), result left in sm
// (digit-reversed order). Ends with a barrier.
template <class Load>
__device__ void fft_forward(float2 *sm, const float2 *tw, const FftPlanK &pl,
                            Load &load)
{
    const int tid = threadIdx.x, nthr = blockDim.x;
    {
        const int r = pl.radix[0];
        const float2 *twp = tw + pl.twoff[0];
        SDRG_RADIX_DISPATCH(r, (dif_pass0_load<R_>(sm, pl.M, twp, load, tid, nthr)));
    }
    __syncthreads();
    for (int p = 1; p < pl.npass; ++p) {
        const int r = pl.radix[p], Ls = pl.Ls[p];
        const float2 *twp = tw + pl.twoff[p];
        SDRG_RADIX_DISPATCH(r, (dif_pass<R_>(sm, pl.M, Ls, twp, tid, nthr)));
        __syncthreads();
    }
}

// Full inverse transform of sm (digit-reversed input); the last pass hands
// every natural-order output to store(). Starts after the caller's barrier;
// no barrier at the end.
template <class Store>
__device__ void fft_inverse(float2 *sm, const float2 *tw, const FftPlanK &pl,
                            Store &store)
{
    const int tid = threadIdx.x, nthr = blockDim.x;
    for (int p = pl.npass - 1; p >= 1; --p) {
        const int r = pl.radix[p], Ls = pl.Ls[p];
        const float2 *twp = tw + pl.twoff[p];
        SDRG_RADIX_DISPATCH(r, (dit_pass<R_>(sm, pl.M, Ls, twp, tid, nthr)));
        __syncthreads();
    }
    {
        const int r = pl.radix[0];
        const float2 *twp = tw + pl.twoff[0];
        SDRG_RADIX_DISPATCH(r, (dit_pass0_store<R_>(sm, pl.M, twp, store, tid, nthr)));
    }
}

// ---- compile-time plans -------------------------------------------------------
// A 4-pass plan fixed at compile time: every stride, table offset, loop trip
// count and divisor is a constant, so shared-memory addresses take immediate
// offsets and the butterfly loops unroll. The global table layout is the
// runtime plan's (pass 0: S0 entries; pass p >= 1: S_p * (r_p - 1) entries),
// so a matching runtime plan's tables serve it unchanged. Its passes read one
// twiddle per butterfly (the first S_p entries of each pass's table) and form
// the powers in registers, so with COMPACT the shared-memory copy holds only
// those (T_p: offsets in shared memory, TWS entries; load_twiddles_static):
// S0 + S1 + S2 entries instead of TWTOT, which lets two 12 000-point CTAs
// share an SM.
template <int M_, int NT_, int R0_, int R1_, int R2_, int R3_, bool COMPACT = false>
struct StaticPlan4 {
    static constexpr int M = M_, NT = NT_;
    static constexpr int R0 = R0_, R1 = R1_, R2 = R2_, R3 = R3_;
    static constexpr int S0 = M / R0, S1 = S0 / R1, S2 = S1 / R2, S3 = S2 / R3;
    static constexpr int O0 = 0, O1 = S0, O2 = O1 + S1 * (R1 - 1), O3 = O2 + S2 * (R2 - 1);
    static constexpr int TWTOT = O3 + S3 * (R3 - 1);
    static constexpr int T0 = 0, T1 = COMPACT ? S0 : O1, T2 = COMPACT ? S0 + S1 : O2,
                         T3 = COMPACT ? S0 + S1 + S2 : O3;
    static constexpr int TWS = COMPACT ? S0 + S1 + S2 : TWTOT;
    static_assert(S3 == 1 && R0 * R1 * R2 * R3 == M, "plan must cover M");
    static bool matches(const FftPlanK &k, int threads)
    {
        return k.M == M && k.npass == 4 && k.radix[0] == R0 && k.radix[1] == R1 &&
               k.radix[2] == R2 && k.radix[3] == R3 && k.twtot == TWTOT && threads == NT;
    }
};

// The plan of every 24 000-point sub-transform (L = 24 000 x {1, 2, 8}: the
// 12 and 24 MHz searches of 1 ms and 4 ms codes).
using Plan24000 = StaticPlan4<24000, 512, 16, 10, 10, 15>;
// 12 000-point sub-transforms of a 4-way split (L = 48 000), two CTAs of 8
// warps per SM: the same 1500-point warp blocks (10 x 10 x 15) after a first
// radix of 8, compact twiddles.
using Plan12000 = StaticPlan4<12000, 256, 8, 10, 10, 15, true>;

// inner pass with compile-time radix R, stride S (sub-length R*S)
template <int R, int S, int M, int NT, bool FWD>
__device__ __forceinline__ void s_inner(float2 *sm, const float2 *twp)
{
    constexpr int NB = M / R, LS = R * S, IT = (NB + NT - 1) / NT;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int b = threadIdx.x + it * NT;
        if (b < NB) {
            const int blk = b / S, i = b - blk * S;
            float2 *p = sm + blk * LS + i;
            float2 v[R];
#pragma unroll
            for (int j = 0; j < R; ++j) v[j] = p[j * S];
            if (FWD) {
                Dft<R, -1>::run(v);
                if (S > 1) {
#pragma unroll
                    for (int j = 1; j < R; ++j) v[j] = cmul(v[j], twp[(j - 1) * S + i]);
                }
            } else {
                if (S > 1) {
#pragma unroll
                    for (int j = 1; j < R; ++j) v[j] = cmul(v[j], cconj(twp[(j - 1) * S + i]));
                }
                Dft<R, 1>::run(v);
            }
#pragma unroll
            for (int j = 0; j < R; ++j) p[j * S] = v[j];
        }
    }
}

// last inverse pass (radix R, stride S = M / R) handing outputs to store()
// Largest radix whose warp-private passes take butterflies in pairs (radix
// 15 in pairs and an unrolled last pass measured slower: 9.64 and 9.73 against
// 9.84 G cells/s on the multi-GNSS search).
constexpr int kPairMax = 10;
template <int R, int S, int NT, class Store>
__device__ __forceinline__ void s_pass0_store(const float2 *sm, const float2 *twp, Store &store)
{
    constexpr int IT = (S + NT - 1) / NT;
#pragma unroll 1
    for (int it = 0; it < IT; ++it) {
        const int i = threadIdx.x + it * NT;
        if (i < S) {
            typename Store::Old old[R];
#pragma unroll
            for (int j = 0; j < R; ++j) old[j] = store.pre(i + j * S);
            float2 v[R];
#pragma unroll
            for (int j = 0; j < R; ++j) v[j] = sm[i + j * S];
            if (i) apply_tw<R>(v, cconj(twp[i]));
            Dft<R, 1>::run(v);
#pragma unroll
            for (int j = 0; j < R; ++j) store(i + j * S, v[j], old[j]);
        }
    }
}

// inner inverse pass (radix R, stride S) restricted to one warp's region of
// M / W consecutive elements (W warps): the passes after the first DIF pass
// (the last DIT passes) never reach outside a block of Ls_1 = M / R0 points,
// so when R0 equals the warp count each warp owns one such block.
// one butterfly of an inner pass at p (stride S, index i in its block):
// forward DIF (DFT, then twiddles) or inverse DIT (conjugate twiddles, then
// backward DFT)
template <int R, int S, bool FWD>
__device__ __forceinline__ void s_bfly(float2 *p, const float2 *twp, int i)
{
    float2 v[R];
#pragma unroll
    for (int j = 0; j < R; ++j) v[j] = p[j * S];
    // powers of the first twiddle by repeated products: one table load
    // instead of R - 1
    if (FWD) {
        Dft<R, -1>::run(v);
        if (S > 1) apply_tw<R>(v, twp[i]);
    } else {
        if (S > 1) apply_tw<R>(v, cconj(twp[i]));
        Dft<R, 1>::run(v);
    }
#pragma unroll
    for (int j = 0; j < R; ++j) p[j * S] = v[j];
}

// two butterflies of a warp-private pass at once (p0 always, p1 when ok1):
// both loads before either butterfly's arithmetic, both stores after (more
// independent work per warp between shared-memory round trips; radices up to
// 10, where the registers allow: multi-GNSS search +1.4 % on per-group
// launches, +4.5 % as a work list)
template <int R, int S, bool FWD>
__device__ __forceinline__ void s_bfly2(float2 *p0, int i0, float2 *p1, int i1, bool ok1,
                                        const float2 *twp)
{
    float2 v0[R], v1[R];
#pragma unroll
    for (int j = 0; j < R; ++j) v0[j] = p0[j * S];
    if (ok1) {
#pragma unroll
        for (int j = 0; j < R; ++j) v1[j] = p1[j * S];
    }
    if (FWD) {
        Dft<R, -1>::run(v0);
        if (S > 1) apply_tw<R>(v0, twp[i0]);
        if (ok1) {
            Dft<R, -1>::run(v1);
            if (S > 1) apply_tw<R>(v1, twp[i1]);
        }
    } else {
        if (S > 1) apply_tw<R>(v0, cconj(twp[i0]));
        Dft<R, 1>::run(v0);
        if (ok1) {
            if (S > 1) apply_tw<R>(v1, cconj(twp[i1]));
            Dft<R, 1>::run(v1);
        }
    }
#pragma unroll
    for (int j = 0; j < R; ++j) p0[j * S] = v0[j];
    if (ok1) {
#pragma unroll
        for (int j = 0; j < R; ++j) p1[j * S] = v1[j];
    }
}

template <int R, int S, int REG, bool FWD = false>
__device__ __forceinline__ void s_inner_warp(float2 *sm, const float2 *twp)
{
    constexpr int NB = REG / R, LS = R * S, IT = (NB + 31) / 32;
    static_assert(REG % LS == 0, "a warp's region holds whole blocks");
    const int lane = threadIdx.x & 31;
    float2 *base = sm + (threadIdx.x >> 5) * REG;
    if constexpr (S >= 8 && S <= 16) {
        // one block per half-warp, lane i < S: the half-warp's R accesses
        // are S consecutive elements, in distinct banks (lanes taken in order
        // put two blocks LS apart into one half-warp, whose elements collided
        // in the banks: 1.9x the wavefronts at R = 10, S = 15). Strides of 8
        // to 16 keep at least half of the lanes busy.
        constexpr int NBLK = REG / LS, IH = (NBLK + 1) / 2;
        const int i = lane & 15;
        if constexpr (R <= kPairMax) {
#pragma unroll
            for (int it = 0; it < IH; it += 2) {
                const int b0 = 2 * it + (lane >> 4), b1 = b0 + 2;
                if (b0 < NBLK && i < S)
                    s_bfly2<R, S, FWD>(base + b0 * LS + i, i, base + b1 * LS + i, i,
                                       it + 1 < IH && b1 < NBLK, twp);
            }
        } else {
#pragma unroll
            for (int it = 0; it < IH; ++it) {
                const int blk = 2 * it + (lane >> 4);
                if (blk < NBLK && i < S) s_bfly<R, S, FWD>(base + blk * LS + i, twp, i);
            }
        }
    } else {
        if constexpr (R <= kPairMax) {
#pragma unroll
            for (int it = 0; it < IT; it += 2) {
                const int b0 = lane + it * 32, b1 = b0 + 32;
                if (b0 < NB) {
                    const int k0 = b0 / S, i0 = b0 - k0 * S, k1 = b1 / S, i1 = b1 - k1 * S;
                    s_bfly2<R, S, FWD>(base + k0 * LS + i0, i0, base + k1 * LS + i1, i1,
                                       it + 1 < IT && b1 < NB, twp);
                }
            }
        } else {
#pragma unroll
            for (int it = 0; it < IT; ++it) {
                const int b = lane + it * 32;
                if (b < NB) {
                    const int blk = b / S, i = b - blk * S;
                    s_bfly<R, S, FWD>(base + blk * LS + i, twp, i);
                }
            }
        }
    }
}

// Forward transform with a compile-time plan (same contract as fft_forward):
// pass 0 over the CTA fused with load(), then, with R0 = warps per CTA, passes
// 1..3 warp by warp on the independent blocks of M / R0 points. Ends with a
// barrier.
template <class P, class Load>
__device__ __forceinline__ void fft_forward_static(float2 *sm, const float2 *tw, Load &load)
{
    static_assert(P::R0 * 32 == P::NT, "one warp per block after the first pass");
    constexpr int REG = P::M / P::R0;
    dif_pass0_load<P::R0>(sm, P::M, tw + P::T0, load, threadIdx.x, P::NT);
    __syncthreads();
    s_inner_warp<P::R1, P::S1, REG, true>(sm, tw + P::T1);
    __syncwarp();
    s_inner_warp<P::R2, P::S2, REG, true>(sm, tw + P::T2);
    __syncwarp();
    s_inner_warp<P::R3, P::S3, REG, true>(sm, tw + P::T3);
    __syncthreads();
}

// Inverse transform with a compile-time plan (same contract as fft_inverse).
// With R0 = warps per CTA, passes 3..1 run warp by warp (warp barriers only)
// and one CTA barrier precedes the last pass.
template <class P, class Store>
__device__ __forceinline__ void fft_inverse_static(float2 *sm, const float2 *tw, Store &store)
{
    if constexpr (P::R0 * 32 == P::NT) {
        constexpr int REG = P::M / P::R0;
        s_inner_warp<P::R3, P::S3, REG>(sm, tw + P::T3);
        __syncwarp();
        s_inner_warp<P::R2, P::S2, REG>(sm, tw + P::T2);
        __syncwarp();
        s_inner_warp<P::R1, P::S1, REG>(sm, tw + P::T1);
        __syncthreads();
    } else {
        static_assert(P::TWS == P::TWTOT, "CTA-wide passes read the full tables");
        s_inner<P::R3, P::S3, P::M, P::NT, false>(sm, tw + P::O3);
        __syncthreads();
        s_inner<P::R2, P::S2, P::M, P::NT, false>(sm, tw + P::O2);
        __syncthreads();
        s_inner<P::R1, P::S1, P::M, P::NT, false>(sm, tw + P::O1);
        __syncthreads();
    }
    s_pass0_store<P::R0, P::S0, P::NT>(sm, tw + P::T0, store);
}

// Split combine of a length-L = R*M forward transform computed as R
// decimated sub-transforms F_r = FFT_M(x[R m + r]): given g[r] = F_r[k] at
// k = k(q) and t = exp(+2 pi i k / L), leaves g[j] = X[k + j M]
// = sum_r e^{-2 pi i r (k + j M) / L} F_r[k].
template <int R>
__device__ __forceinline__ void split_combine_fwd(float2 *g, float2 t)
{
    if constexpr (R > 1) {
        const float2 tc = cconj(t);
        float2 w = tc;
#pragma unroll
        for (int r = 1; r < R; ++r) {
            g[r] = cmul(g[r], w);
            if (r + 1 < R) w = cmul(w, tc);
        }
        Dft<R, -1>::run(g);
    }
}

// Copies the per-pass twiddle tables from global to shared memory, with up
// to 8 loads per thread in flight (a 24 000-point plan holds ~3 000 entries,
// about 6 per thread of a 512-thread CTA).
__device__ __forceinline__ void load_twiddles(float2 *tw_sm, const float2 *tw_g,
                                              int n)
{
    constexpr int UL = 8;
    for (int i0 = threadIdx.x; i0 < n; i0 += UL * blockDim.x) {
        float2 v[UL];
#pragma unroll
        for (int u = 0; u < UL; ++u) {
            const int i = i0 + u * blockDim.x;
            if (i < n) v[u] = __ldg(tw_g + i);
        }
#pragma unroll
        for (int u = 0; u < UL; ++u) {
            const int i = i0 + u * blockDim.x;
            if (i < n) tw_sm[i] = v[u];
        }
    }
}

// The shared-memory twiddles of a compile-time plan: the whole table, or
// with P's COMPACT layout the first S_p entries of passes 0..2 (pass 3 has
// stride 1 and no twiddles).
template <class P>
__device__ __forceinline__ void load_twiddles_static(float2 *tw_sm, const float2 *tw_g)
{
    if constexpr (P::TWS == P::TWTOT) {
        load_twiddles(tw_sm, tw_g, P::TWTOT);
    } else {
        for (int i = threadIdx.x; i < P::TWS; i += blockDim.x) {
            const int g = i < P::T1 ? P::O0 + i : (i < P::T2 ? P::O1 + (i - P::T1)
                                                             : P::O2 + (i - P::T2));
            tw_sm[i] = __ldg(tw_g + g);
        }
    }
}

} // namespace sdrg
