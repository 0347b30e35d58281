// sdrg_internal.h - host-side internals shared by the library's .cu files.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include <mutex>
#include <string>
#include <vector>

#include "pocket_sdr_gpu.h"
#include "sdrg_fft.cuh"

namespace sdrg {

// SDR_CSCALE of src/pocket_sdr.h:61, evaluated in float on the host
// (1 / 11.2f) and handed to kernels as an argument.
extern const float kCScale;

// ---- error state (per host thread) ----------------------------------------
int set_error(int code, const char *fmt, ...);
// SDRG_OK, or SDRG_ERR_NOMEM (error set) when a simulated allocation failure
// is due (sdrg_inject_alloc_failure); called before each library allocation.
int alloc_fault(const char *what);
int cuda_error(cudaError_t e, const char *what);
#define SDRG_CUDA(call)                                            \
    do {                                                           \
        cudaError_t e__ = (call);                                  \
        if (e__ != cudaSuccess) return ::sdrg::cuda_error(e__, #call); \
    } while (0)

// ---- device context ----------------------------------------------------------
struct Device {
    int id = -1;
    int sm_count = 0;
    int nsmid = 0;              // upper bound of the SM identifiers (%nsmid)
    size_t smem_optin = 0;      // max dynamic shared memory per block
    size_t smem_per_sm = 0;     // shared memory of one SM
    int8_t ctab[512];           // quantised carrier (I,Q) for 256 phases
    char2 *ctab_dev = nullptr;  // same table on the device
    cudaMemPool_t pool = nullptr;   // the library's stream-ordered scratch pool
};
int ensure_device(Device **out);   // lazy init of the selected device
// Stream-ordered scratch from the library's own memory pool, which keeps
// freed memory mapped (no release threshold): repeated calls of the same
// size reuse it instead of mapping new pages after every synchronisation, as
// the process's default pool would. Free with cudaFreeAsync.
cudaError_t stream_alloc(void **p, size_t bytes, cudaStream_t st);
size_t g_smem_limit();             // max dynamic shared memory per CTA

// Grow-only device / pinned buffers owned by one host thread.
struct Scratch {
    void *ptr = nullptr;
    size_t size = 0;
    bool pinned = false;
    ~Scratch();
    int reserve(size_t bytes);
};

// A tracking channel's code bank ([SDR_N_CODES][N] sdr_cpx16_t, host memory
// of the caller) kept on the device by the synchronous correlators of one
// host thread: `host` holds the bytes each uploaded bank had, so a later call
// uploads a bank only when the caller's bytes differ.
struct BankCache {
    const void *key = nullptr;   // the caller's bank pointer
    int N = 0;
    void *dev = nullptr;         // [SDR_N_CODES][N] char2 on the device
    std::vector<uint8_t> host;   // [SDR_N_CODES][N] char2: what dev holds
    uint32_t valid = 0;          // bit k: bank k is on the device
    uint64_t used = 0;           // last use (for eviction)
    BankCache() = default;
    BankCache(const BankCache &) = delete;
    BankCache &operator=(const BankCache &) = delete;
    ~BankCache();
};

struct ThreadCtx {
    cudaStream_t stream = nullptr;
    std::vector<BankCache *> banks;   // sdr_corr_std* code banks (bounded, LRU)
    uint64_t bank_clock = 0;
    Scratch dev[6];      // device scratch slots
    Scratch host[3];     // pinned host staging slots
    // batched correlators (asynchronous): their own slots and the event of
    // the last upload from cb_host
    Scratch stage_err;   // device error word of staged FFT launches
    Scratch corr_dev;    // synchronous correlators: partials, outputs, ticket
    Scratch cb_dev, cb_host;
    cudaEvent_t cb_ev = nullptr, cb_done = nullptr;
    // batched L6 CSK tracking (asynchronous): the same scheme
    Scratch l6_dev, l6_host;
    cudaEvent_t l6_ev = nullptr, l6_done = nullptr;
    int error = 0;
    std::string msg;
    ~ThreadCtx();
};
ThreadCtx &tctx();
int thread_stream(cudaStream_t *s);  // creates the thread's stream lazily

// ---- FFT plans -------------------------------------------------------------
// A length-L transform is split as L = R * M: R CTAs (a thread-block cluster
// when R > 1) each hold one length-M sub-transform in shared memory.
struct FftPlan {
    int L = 0, R = 0, M = 0;
    FftPlanK k{};              // pass structure for the length-M transform
    int threads = 0;           // CTA size
    size_t smem = 0;           // dynamic shared memory bytes per CTA
    float2 *tw_dev = nullptr;  // per-pass twiddles (k.twtot entries)
    int *kperm_dev = nullptr;  // k(q): natural frequency index at position q
    float2 *split_dev = nullptr; // exp(+2 pi i k(q) / L) at position q (R > 1)
    std::vector<int> kperm;    // host copy of k(q)
};
// Returns a cached plan for length L (thread-safe), or nullptr with the
// error set when L has no supported decomposition.
const FftPlan *get_plan(int L);
// A plan with an imposed split and CTA size (cached per shape; autotuning).
const FftPlan *get_plan_shaped(int L, int R, int threads);
// Sets length L's schedule (R = 0: back to the default rule); later plans
// for L use it.
int set_schedule(int L, int R, int threads, double ms);
bool plan_shape(int L, int *R, int *M, FftPlanK *k);
bool shape_ok(int L, int R);       // L splits R ways into a fitting length
// The default split rule over cluster splits only (R <= 8), ignoring any
// schedule; allocates nothing.
bool cluster_shape(int L, int *R, int *M, FftPlanK *k);

// ---- kernel launch helpers (defined in the .cu files) -----------------------
// Packed IF source of one coherent block for the forward transform.
struct IfWindow {
    const uint8_t *buf;   // device circular buffer
    int len;              // buffer length (samples)
    int ix;               // first sample
};

// Packs a float I/Q window as the reference's python-facing calls do
// (src/sdr_func.c:839-848) and mixes it into iq_dev (device, N samples).
int mix_cpx_device(const sdr_cpx_t *buff, int len_buff, int ix, int N, double fs,
                   double fc, double phi, char2 *iq_dev, cudaStream_t st);

// Replica generation (sdrg_code.cu), asynchronous on st, DEVICE pointers.
// res_code_device: out[c][b][N+Nz] = sdr_res_code(code c, coff - b/fs/n_bank);
// code_fft_device: conjugated DFT of each code's N-sample replica zero padded
// to L, natural order ([c][L]) or the acquisition layout ([c][R][M] at the
// forward transform's digit-reversed positions).
int res_code_device(const int8_t *ci, const int8_t *cq, int len_code, int n_code, double T,
                    double coff, double fs, int N, int Nz, int n_bank, char2 *out,
                    cudaStream_t st);
// natural = 0 writes the permuted layout of plan pl (null: the length's
// default plan), the one a consumer using pl reads
int code_fft_device(const int8_t *ci, const int8_t *cq, int len_code, int n_code, double T,
                    double coff, double fs, int N, int L, int natural, float2 *out,
                    cudaStream_t st, const FftPlan *pl = nullptr);

// One correlation job on device data (sdrg_search.cu): sdr_mix_carr of the
// window [ix, ix + N) of circular buffer buf (len samples) at (fs, fc, phi)
// followed by sdr_corr_fft with the natural-order conjugated code DFT
// code_nat, into corr[N]. tab_dev holds the 5 words corr_job_tables fills;
// scratch must hold corr_job_scratch(N) bytes. Asynchronous on st.
void corr_job_tables(int len, int ix, int N, double fs, double fc, double phi, uint32_t *tab);
size_t corr_job_scratch(int N);
int corr_job_device(const uint8_t *buf, int len, const uint32_t *tab_dev, int N,
                    const float2 *code_nat, float2 *corr, void *scratch, cudaStream_t st);

// n such jobs of one length N on one buffer, batched (cluster splits only):
// tab_dev = phstep[n] | ph0a[n] | ph0b[n] | ix[n] | nsplit[n] (the words of
// corr_job_tables, transposed), code_nat and corr [n][N], scratch 2 n N
// complex values.
int corr_jobs_device(const uint8_t *buf, int len, const uint32_t *tab_dev, int n, int N,
                     const float2 *code_nat, float2 *corr, void *scratch, cudaStream_t st);

} // namespace sdrg
