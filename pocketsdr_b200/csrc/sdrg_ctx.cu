// sdrg_ctx.cu - device context, per-thread streams and scratch, error state,
// FFT plan construction and the library's version/init entry points.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <map>

#include "sdrg_internal.h"

namespace sdrg {

const float kCScale = 1 / 11.2f;

// ---- errors --------------------------------------------------------------------
ThreadCtx &tctx()
{
    static thread_local ThreadCtx ctx;
    return ctx;
}

int set_error(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ThreadCtx &c = tctx();
    c.error = code;
    c.msg = buf;
    fprintf(stderr, "pocketsdr_b200: %s\n", buf);
    return code;
}

int cuda_error(cudaError_t e, const char *what)
{
    return set_error(e == cudaErrorMemoryAllocation ? SDRG_ERR_NOMEM : SDRG_ERR_CUDA,
                     "%s: %s", what, cudaGetErrorString(e));
}

// ---- simulated allocation failures ---------------------------------------------
// Error paths are tested without touching the device allocator's real limits:
// sdrg_inject_alloc_failure(n) (or SDRG_FAIL_ALLOC=n in the environment, read
// once) makes the n-th following device or pinned allocation attempt of the
// library fail as cudaMalloc would with cudaErrorMemoryAllocation.
static std::mutex g_fail_mtx;
static long g_fail_after = -2;   // -2: environment not read yet, -1: off

int alloc_fault(const char *what)
{
    std::lock_guard<std::mutex> lk(g_fail_mtx);
    if (g_fail_after == -2) {
        const char *e = getenv("SDRG_FAIL_ALLOC");
        g_fail_after = e ? atol(e) : -1;
    }
    if (g_fail_after < 0) return SDRG_OK;
    if (g_fail_after-- > 0) return SDRG_OK;
    g_fail_after = -1;
    return set_error(SDRG_ERR_NOMEM, "%s: simulated allocation failure", what);
}

// ---- device ------------------------------------------------------------------
static std::mutex g_dev_mtx;
static Device g_dev;
static int g_dev_wanted = -1;

static void build_ctab(int8_t *ctab)
{
    // src/sdr_func.c:115-118: ROUND(cos|sin(-2 pi i / 256) / SDR_CSCALE),
    // ROUND(x) = floor(x + 0.5), PI = 3.1415926535897932, in double.
    const double pi = 3.1415926535897932;
    for (int i = 0; i < 256; ++i) {
        ctab[2 * i] = (int8_t)floor(cos(-2.0 * pi * i / 256) / (double)kCScale + 0.5);
        ctab[2 * i + 1] = (int8_t)floor(sin(-2.0 * pi * i / 256) / (double)kCScale + 0.5);
    }
}

// The upper bound of the SM identifiers (%nsmid; identifiers need not be
// contiguous), for buffers indexed by the SM a CTA runs on.
__global__ void nsmid_kernel(int *out)
{
    unsigned n;
    asm volatile("mov.u32 %0, %%nsmid;" : "=r"(n));
    *out = (int)n;
}

int ensure_device(Device **out)
{
    std::lock_guard<std::mutex> lk(g_dev_mtx);
    if (g_dev.id < 0) {
        int id = g_dev_wanted;
        if (id < 0) {
            const char *env = getenv("SDRG_DEVICE");
            id = env ? atoi(env) : 0;
        }
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess || n <= id) {
            return set_error(SDRG_ERR_NODEV, "no CUDA device %d available (%s)", id,
                             e != cudaSuccess ? cudaGetErrorString(e) : "count too small");
        }
        SDRG_CUDA(cudaSetDevice(id));
        cudaDeviceProp prop;
        SDRG_CUDA(cudaGetDeviceProperties(&prop, id));
        if (prop.major < 10) {
            return set_error(SDRG_ERR_NODEV, "device %d (%s, sm_%d%d) is not sm_100", id,
                             prop.name, prop.major, prop.minor);
        }
        g_dev.sm_count = prop.multiProcessorCount;
        g_dev.smem_optin = prop.sharedMemPerBlockOptin;
        g_dev.smem_per_sm = prop.sharedMemPerMultiprocessor;
        {
            int *d = nullptr, h = 0;
            SDRG_CUDA(cudaMalloc(&d, sizeof(int)));
            nsmid_kernel<<<1, 1>>>(d);
            SDRG_CUDA(cudaGetLastError());
            SDRG_CUDA(cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost));
            SDRG_CUDA(cudaFree(d));
            g_dev.nsmid = h > 0 ? h : prop.multiProcessorCount;
        }
        build_ctab(g_dev.ctab);
        SDRG_CUDA(cudaMalloc(&g_dev.ctab_dev, 512));
        SDRG_CUDA(cudaMemcpy(g_dev.ctab_dev, g_dev.ctab, 512, cudaMemcpyHostToDevice));
        // a pageable cudaMemcpy may return before its DMA completes, and the
        // library's kernels run on non-blocking streams: settle it here
        SDRG_CUDA(cudaDeviceSynchronize());
        cudaMemPoolProps pp = {};
        pp.allocType = cudaMemAllocationTypePinned;
        pp.location.type = cudaMemLocationTypeDevice;
        pp.location.id = id;
        SDRG_CUDA(cudaMemPoolCreate(&g_dev.pool, &pp));
        uint64_t keep = UINT64_MAX;
        SDRG_CUDA(cudaMemPoolSetAttribute(g_dev.pool, cudaMemPoolAttrReleaseThreshold, &keep));
        g_dev.id = id;
    }
    SDRG_CUDA(cudaSetDevice(g_dev.id));
    if (out) *out = &g_dev;
    return SDRG_OK;
}

size_t g_smem_limit() { return g_dev.id >= 0 ? g_dev.smem_optin : 232448; }

cudaError_t stream_alloc(void **p, size_t bytes, cudaStream_t st)
{
    if (!g_dev.pool) return cudaErrorInitializationError;
    return cudaMallocFromPoolAsync(p, bytes, g_dev.pool, st);
}

int thread_stream(cudaStream_t *s)
{
    ThreadCtx &c = tctx();
    if (!c.stream) {
        SDRG_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    }
    *s = c.stream;
    return SDRG_OK;
}

BankCache::~BankCache()
{
    if (dev) cudaFree(dev);      // at thread exit; errors ignored
}

ThreadCtx::~ThreadCtx()
{
    for (BankCache *b : banks) delete b;
}

Scratch::~Scratch()
{
    // Released at thread exit; errors are ignored (the context may be gone).
    if (ptr) {
        if (pinned) cudaFreeHost(ptr); else cudaFree(ptr);
    }
}

int Scratch::reserve(size_t bytes)
{
    if (bytes <= size) return SDRG_OK;
    size_t want = bytes + bytes / 4 + 256;
    if (ptr) {
        if (pinned) cudaFreeHost(ptr); else cudaFree(ptr);
        ptr = nullptr;
        size = 0;
    }
    int fe;
    if ((fe = alloc_fault(pinned ? "cudaMallocHost" : "cudaMalloc"))) return fe;
    cudaError_t e = pinned ? cudaMallocHost(&ptr, want) : cudaMalloc(&ptr, want);
    if (e != cudaSuccess) {
        ptr = nullptr;
        return cuda_error(e, pinned ? "cudaMallocHost" : "cudaMalloc");
    }
    size = want;
    return SDRG_OK;
}

// ---- FFT plans -----------------------------------------------------------------
static const int kRadices[] = {16, 15, 12, 10, 8, 6, 5, 4, 3, 2};

struct Fact { int a, b, c; };  // 2^a 3^b 5^c

static bool factor235(int n, Fact *f)
{
    f->a = f->b = f->c = 0;
    if (n <= 0) return false;
    while (n % 2 == 0) { n /= 2; f->a++; }
    while (n % 3 == 0) { n /= 3; f->b++; }
    while (n % 5 == 0) { n /= 5; f->c++; }
    return n == 1;
}

// Best radix sequence for 2^a 3^b 5^c: fewest passes, then the largest
// smallest radix (balanced passes). Exhaustive over the small exponent space;
// fixed arrays (no heap use: the no-allocation correlator shapes its plans
// with this too).
struct Radices {
    int r[kMaxPass + 1];
    int n = 0;
    int min_r() const
    {
        int m = 1 << 30;
        for (int i = 0; i < n; ++i) m = r[i] < m ? r[i] : m;
        return m;
    }
};

static void best_radices(int n, Radices &cur, Radices &best)
{
    if (n == 1) {
        if (best.n == 0 || cur.n < best.n || (cur.n == best.n && cur.min_r() > best.min_r()))
            best = cur;
        return;
    }
    if ((best.n && cur.n + 1 > best.n) || cur.n >= kMaxPass + 1) return;
    int last = cur.n == 0 ? 1 << 30 : cur.r[cur.n - 1];
    for (int r : kRadices) {
        if (r > last || n % r) continue;  // non-increasing order avoids repeats
        cur.r[cur.n++] = r;
        best_radices(n / r, cur, best);
        cur.n--;
    }
}

static size_t plan_smem(int M, const FftPlanK &k)
{
    return (size_t)M * sizeof(float2) + (size_t)k.twtot * sizeof(float2) + 512;
}

// Max dynamic shared memory per CTA assumed when no device is present.
static const size_t kSmemDefault = 232448;

// Pass structure of a length-L transform split R ways (M = L / R): false
// when M is not 2-3-5-smooth, needs too many passes or does not fit one CTA.
static bool shape_for_R(int L, int R, int *Mout, FftPlanK *kout)
{
    if (R <= 0 || L % R) return false;
    size_t smax = g_dev.id >= 0 ? g_dev.smem_optin : kSmemDefault;
    int M = L / R;
    Fact f;
    if (!factor235(M, &f)) return false;
    Radices cur, best;
    if (M == 1) best.r[best.n++] = 1;
    else best_radices(M, cur, best);
    if (best.n == 0 || best.n > kMaxPass) return false;
    // Even radices first (largest first), odd radices last: the last
    // passes have the smallest strides, and an odd stride of 8-byte
    // elements spreads a half-warp over all 16 bank pairs (stable insertion
    // sort)
    auto before = [](int a, int b) {
        if ((a & 1) != (b & 1)) return (a & 1) == 0;
        return a > b;
    };
    for (int i = 1; i < best.n; ++i)
        for (int j = i; j > 0 && before(best.r[j], best.r[j - 1]); --j) {
            const int t = best.r[j];
            best.r[j] = best.r[j - 1];
            best.r[j - 1] = t;
        }
    if (M == Plan12000::M) {
        // the compile-time 12 000-point plan's passes (first radix = its 8
        // warps, then the 1500-point warp blocks of 10 x 10 x 15), so that
        // its tables serve that plan
        best.n = 4;
        best.r[0] = Plan12000::R0; best.r[1] = Plan12000::R1;
        best.r[2] = Plan12000::R2; best.r[3] = Plan12000::R3;
    }
    FftPlanK k{};
    k.M = M;
    k.npass = best.n;
    int Ls = M, off = 0;
    for (int p = 0; p < k.npass; ++p) {
        k.radix[p] = best.r[p];
        k.Ls[p] = Ls;
        k.twoff[p] = off;
        // pass 0: S entries (powers formed in registers); later passes:
        // S * (r - 1) entries, every twiddle of the pass
        off += (p == 0) ? Ls / best.r[p] : (Ls / best.r[p]) * (best.r[p] - 1);
        Ls /= best.r[p];
    }
    k.twtot = off;   // M == 1: one radix-1 pass, one unit twiddle
    if (plan_smem(M, k) > smax) return false;
    *Mout = M;
    *kout = k;
    return true;
}

// The default rule restricted to cluster splits (R <= 8), schedules not
// consulted; no heap use.
bool cluster_shape(int L, int *Rout, int *Mout, FftPlanK *kout)
{
    for (int R : {1, 2, 3, 4, 5, 6, 8}) {
        if (shape_for_R(L, R, Mout, kout)) {
            *Rout = R;
            return true;
        }
    }
    return false;
}

bool shape_ok(int L, int R)
{
    int M;
    FftPlanK k;
    return shape_for_R(L, R, &M, &k);
}

// R <= 8: one thread-block cluster per transform; R in 10..20: staged
// through a scratch buffer in global memory (a cluster cannot exceed 8
// portably)
static const int kSplits[] = {1, 2, 3, 4, 5, 6, 8, 10, 12, 15, 16, 20};

static bool split_allowed(int R)
{
    for (int r : kSplits)
        if (r == R) return true;
    return false;
}

// ---- schedules (autotuned or loaded; per length: split and CTA size) -------
struct Sched {
    int R, threads;
    double ms;
};
static std::mutex g_sched_mtx;
static std::map<int, Sched> g_sched;

static bool sched_of(int L, Sched *out)
{
    std::lock_guard<std::mutex> lk(g_sched_mtx);
    auto it = g_sched.find(L);
    if (it == g_sched.end()) return false;
    *out = it->second;
    return true;
}

bool plan_shape(int L, int *Rout, int *Mout, FftPlanK *kout)
{
    Sched sc;
    if (sched_of(L, &sc) && shape_for_R(L, sc.R, Mout, kout)) {
        *Rout = sc.R;
        return true;
    }
    for (int R : kSplits) {
        if (shape_for_R(L, R, Mout, kout)) {
            *Rout = R;
            return true;
        }
    }
    return false;
}

static std::mutex g_plan_mtx;
static std::map<int, FftPlan *> g_plans;
static std::map<long long, FftPlan *> g_shaped;   // (L, R, threads) -> plan
static std::vector<FftPlan *> g_retired;          // replaced by a new schedule

// default CTA size: up to 512 threads, at least 8 points per thread
static int default_threads(int M)
{
    int t = 32;
    while (t < 512 && t * 8 < M) t *= 2;
    return t;
}

// R_force / t_force > 0 impose the split and CTA size; otherwise the length's
// schedule, else the default rule.
static int build_plan(int L, FftPlan *pl, int R_force = 0, int t_force = 0)
{
    int R = 0, M;
    FftPlanK k;
    Sched sc = {0, 0, 0.0};
    const bool have = !R_force && sched_of(L, &sc);
    if (R_force) {
        if (!shape_for_R(L, R_force, &M, &k))
            return set_error(SDRG_ERR_ARG, "FFT length %d cannot be split %d ways", L, R_force);
        R = R_force;
    } else if (!plan_shape(L, &R, &M, &k)) {
        return set_error(SDRG_ERR_ARG,
                         "FFT length %d unsupported (needs L = R*M, R in {1..6,8,10,12,15,16,20}, "
                         "M 2-3-5-smooth and fitting one CTA)", L);
    }
    pl->L = L; pl->R = R; pl->M = M; pl->k = k;
    int t = default_threads(M);
    if (t_force > 0) t = t_force;
    else if (have && sc.R == R && sc.threads > 0) t = sc.threads;
    pl->threads = t;
    pl->smem = plan_smem(M, k);
    // per-pass twiddles: pass 0 exp(-2 pi i * i / Ls_0), i < S_0; pass p >= 1
    // exp(-2 pi i * i*j / Ls_p) at (j-1)*S_p + i, j = 1..r_p-1 (double, rounded)
    std::vector<float2> tw(k.twtot > 0 ? k.twtot : 1);
    for (int p = 0; p < k.npass; ++p) {
        int Ls = k.Ls[p], r = k.radix[p], S = Ls / r;
        int jmax = (p == 0) ? 1 : r - 1;
        for (int j = 1; j <= jmax; ++j) {
            for (int i = 0; i < S; ++i) {
                double a = -2.0 * M_PI * (double)((long)i * j % Ls) / Ls;
                tw[k.twoff[p] + (j - 1) * S + i] = make_float2((float)cos(a), (float)sin(a));
            }
        }
    }
    // digit-reversed frequency index of each DIF output position
    pl->kperm.resize(M);
    for (int q = 0; q < M; ++q) {
        int rem = q, blk = M, kk = 0, mul = 1;
        for (int p = 0; p < k.npass; ++p) {
            blk /= k.radix[p];
            int j = rem / blk;
            rem %= blk;
            kk += j * mul;
            mul *= k.radix[p];
        }
        pl->kperm[q] = kk;
    }
    std::vector<float2> split(M);
    for (int q = 0; q < M; ++q) {
        double a = 2.0 * M_PI * (double)pl->kperm[q] / L;
        split[q] = make_float2((float)cos(a), (float)sin(a));
    }
    SDRG_CUDA(cudaMalloc(&pl->tw_dev, tw.size() * sizeof(float2)));
    SDRG_CUDA(cudaMemcpy(pl->tw_dev, tw.data(), tw.size() * sizeof(float2),
                         cudaMemcpyHostToDevice));
    SDRG_CUDA(cudaMalloc(&pl->kperm_dev, M * sizeof(int)));
    SDRG_CUDA(cudaMemcpy(pl->kperm_dev, pl->kperm.data(), M * sizeof(int),
                         cudaMemcpyHostToDevice));
    SDRG_CUDA(cudaMalloc(&pl->split_dev, M * sizeof(float2)));
    SDRG_CUDA(cudaMemcpy(pl->split_dev, split.data(), M * sizeof(float2),
                         cudaMemcpyHostToDevice));
    // the plan is used at once by kernels on non-blocking streams, which do
    // not order after these legacy-stream copies
    SDRG_CUDA(cudaDeviceSynchronize());
    return SDRG_OK;
}

const FftPlan *get_plan(int L)
{
    std::lock_guard<std::mutex> lk(g_plan_mtx);
    auto it = g_plans.find(L);
    if (it != g_plans.end()) return it->second;
    FftPlan *pl = new FftPlan();
    if (build_plan(L, pl) != SDRG_OK) {
        delete pl;
        return nullptr;
    }
    g_plans[L] = pl;
    return pl;
}

const FftPlan *get_plan_shaped(int L, int R, int threads)
{
    std::lock_guard<std::mutex> lk(g_plan_mtx);
    const long long key = ((long long)L << 24) | ((long long)R << 12) | threads;
    auto it = g_shaped.find(key);
    if (it != g_shaped.end()) return it->second;
    FftPlan *pl = new FftPlan();
    if (build_plan(L, pl, R, threads) != SDRG_OK) {
        delete pl;
        return nullptr;
    }
    g_shaped[key] = pl;
    return pl;
}

int set_schedule(int L, int R, int threads, double ms)
{
    if (L <= 0) return set_error(SDRG_ERR_ARG, "schedule: bad length %d", L);
    if (R == 0) {                      // back to the default rule
        std::lock_guard<std::mutex> lk(g_sched_mtx);
        g_sched.erase(L);
    } else {
        int M;
        FftPlanK k;
        if (!split_allowed(R) || !shape_for_R(L, R, &M, &k))
            return set_error(SDRG_ERR_ARG, "schedule: length %d cannot be split %d ways", L, R);
        if (threads != 128 && threads != 256 && threads != 512)
            return set_error(SDRG_ERR_ARG, "schedule: CTA size %d not 128, 256 or 512", threads);
        std::lock_guard<std::mutex> lk(g_sched_mtx);
        g_sched[L] = Sched{R, threads, ms};
    }
    // plans built from now on follow the schedule; a cached one is retired
    // (kept alive: acquisition plans may still point to it)
    std::lock_guard<std::mutex> lk(g_plan_mtx);
    auto it = g_plans.find(L);
    if (it != g_plans.end()) {
        g_retired.push_back(it->second);
        g_plans.erase(it);
    }
    return SDRG_OK;
}

} // namespace sdrg

using namespace sdrg;

extern "C" {

int sdr_gpu_last_error(char *buff, int size)
{
    ThreadCtx &c = tctx();
    if (buff && size > 0) {
        snprintf(buff, (size_t)size, "%s", c.msg.c_str());
    }
    return c.error;
}

void sdr_gpu_clear_error(void)
{
    ThreadCtx &c = tctx();
    c.error = 0;
    c.msg.clear();
}

int sdrg_init(int device)
{
    {
        std::lock_guard<std::mutex> lk(g_dev_mtx);
        if (g_dev.id >= 0 && device >= 0 && device != g_dev.id) {
            return set_error(SDRG_ERR_ARG, "already initialised on device %d", g_dev.id);
        }
        g_dev_wanted = device;
    }
    return ensure_device(nullptr);
}

int sdrg_fft_supported(int N)
{
    int R, M;
    FftPlanK k;
    return N > 0 && plan_shape(N, &R, &M, &k) ? 1 : 0;
}

const char *sdrg_version(void) { return "pocketsdr_b200 0.1 (sm_100a)"; }

void sdrg_inject_alloc_failure(int after)
{
    std::lock_guard<std::mutex> lk(g_fail_mtx);
    g_fail_after = after < 0 ? -1 : after;
}

// When the reference's sdr_func.o is linked with its hot symbols renamed to
// *_cpu (the integration recipe), its initialiser still sets up the log
// streams and CPU tables; call it if present.
void sdr_func_init_cpu(const char *file) __attribute__((weak));

int sdrg_fft_schedule_set(int L, int R, int threads)
{
    return set_schedule(L, R, threads, 0.0);
}

int sdrg_fft_schedule_get(int L, int *R, int *threads)
{
    Sched sc;
    if (!sched_of(L, &sc)) return 0;
    if (R) *R = sc.R;
    if (threads) *threads = sc.threads;
    return 1;
}

// File lines "sdrg_fft <L> <R> <threads> <ms>"; other lines are ignored, so
// the reference's FFTW wisdom file given to sdr_func_init loads nothing.
int sdrg_fft_schedule_save(const char *path)
{
    if (!path) return set_error(SDRG_ERR_ARG, "schedule save: no path");
    FILE *f = fopen(path, "w");
    if (!f) return set_error(SDRG_ERR_ARG, "schedule save: cannot open %s", path);
    fprintf(f, "# pocketsdr_b200 FFT schedules: sdrg_fft <length> <split> <threads> <ms>\n");
    {
        std::lock_guard<std::mutex> lk(g_sched_mtx);
        for (const auto &kv : g_sched)
            fprintf(f, "sdrg_fft %d %d %d %.6f\n", kv.first, kv.second.R, kv.second.threads,
                    kv.second.ms);
    }
    fclose(f);
    return SDRG_OK;
}

int sdrg_fft_schedule_load(const char *path)
{
    if (!path) return set_error(SDRG_ERR_ARG, "schedule load: no path");
    FILE *f = fopen(path, "r");
    if (!f) return set_error(SDRG_ERR_ARG, "schedule load: cannot open %s", path);
    char line[256];
    int n = 0, bad = 0;
    while (fgets(line, sizeof(line), f)) {
        int L, R, t;
        double ms = 0.0;
        if (sscanf(line, "sdrg_fft %d %d %d %lf", &L, &R, &t, &ms) < 3) continue;
        if (set_schedule(L, R, t, ms) == SDRG_OK) ++n;
        else ++bad;
    }
    fclose(f);
    if (bad) return set_error(SDRG_ERR_ARG, "schedule load: %d invalid entries in %s", bad, path);
    return n;
}

void sdr_func_init(const char *file)
{
    if (sdr_func_init_cpu) sdr_func_init_cpu(file ? file : "");
    // the reference imports FFTW wisdom from `file` (src/sdr_func.c:118-121);
    // its counterpart here is a schedule file, read when present
    if (file && *file) {
        FILE *f = fopen(file, "r");
        if (f) {
            fclose(f);
            sdrg_fft_schedule_load(file);
        }
    }
    ensure_device(nullptr);
}

} // extern "C"
