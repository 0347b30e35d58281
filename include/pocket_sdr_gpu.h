/*
 * pocket_sdr_gpu.h - B200 (sm_100a) implementation of Pocket SDR's
 * signal-search and correlation hot path behind a C ABI.
 *
 * Part 1 ("drop-in") declares the reference's own entry points with the same
 * names, argument types and meaning (Pocket SDR src/pocket_sdr.h), so a C
 * program or the python/sdr_func.py ctypes layer can bind this library in
 * place of the reference's src/sdr_func.c for these functions. All buffers are
 * caller-owned HOST memory, exactly as in the reference; each call copies its
 * window to the GPU, runs the kernels and copies the result back.
 *
 * Part 2 ("batched", prefix sdrg_) is additive: device-resident IF buffers,
 * many signals x PRNs x Doppler bins x non-coherent sums in one launch
 * sequence, device pointers, an explicit stream, and an int status.
 *
 * Errors: the reference functions return void and exit(-1) on allocation
 * failure (src/sdr_func.c:150-153). Here nothing exits: a failing call leaves
 * its outputs zero-filled (P is left unchanged), prints one line to stderr
 * and records a message readable with sdr_gpu_last_error() on the calling
 * thread.
 *
 * Threading: every entry point may be called concurrently from several host
 * threads (the reference calls them from one thread per receiver channel,
 * src/sdr_rcv.c:495-520); each host thread gets its own CUDA stream and
 * staging buffers.
 */
#ifndef POCKET_SDR_GPU_H
#define POCKET_SDR_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- types: same layout as src/pocket_sdr.h:105-113 and :242-245 -------- */
#ifndef POCKET_SDR_H
typedef uint8_t sdr_cpx8_t;                 /* 4+4-bit I/Q, I in low nibble */
typedef struct { int8_t I, Q; } sdr_cpx16_t; /* mixed sample */
typedef float sdr_cpx_t[2];                  /* single precision complex */
typedef struct {                             /* IF data buffer */
    sdr_cpx8_t *data;
    int IQ, N;
} sdr_buff_t;
#define SDR_N_CODES  10                      /* src/pocket_sdr.h:60 */
#define SDR_MAX_CORR 107                     /* src/pocket_sdr.h:58 */
#define SDR_MAX_RFCH 8                       /* src/pocket_sdr.h:47 */
#define SDR_MAX_ARCH 8                       /* src/pocket_sdr.h:48 */
#define SDR_FMT_INT8   1                     /* IF data formats, src/pocket_sdr.h:85-92 */
#define SDR_FMT_INT8X2 2
#define SDR_FMT_RAW8   3
#define SDR_FMT_RAW16  4
#define SDR_FMT_RAW16I 5
#define SDR_FMT_RAW32  6
#define SDR_FMT_CS8    7
#define SDR_FMT_CS16   8
typedef struct sdr_lpf_tag sdr_lpf_t;        /* LPF state (opaque) */
#endif

/* =========================================================================
 * Part 1: drop-in entry points (same signatures as the reference)
 * ========================================================================= */

/* Replaces src/sdr_func.c:113-134 (sdr_func_init, src/pocket_sdr.h:392).
 * Initialises the GPU context and the quantised carrier table. `file` (an FFT
 * wisdom path in the reference) is accepted and ignored. May be called more
 * than once. */
void sdr_func_init(const char *file);

/* Replaces src/sdr_func.c:824-836 (sdr_mix_carr, src/pocket_sdr.h:429).
 * Bit-exact carrier wipe-off, including the circular-buffer wrap. */
void sdr_mix_carr(const sdr_buff_t *buff, int ix, int N, double fs, double fc,
    double phi, sdr_cpx16_t *IQ);

/* Replaces src/sdr_func.c:981-1008 (sdr_corr_std, src/pocket_sdr.h:415).
 * Bit-exact integer correlation and FP32 scaling. `code` is the
 * SDR_N_CODES x N bank. */
void sdr_corr_std(const sdr_cpx16_t *IQ, const sdr_cpx16_t *code, int N,
    double coff, const double *pos, int n, sdr_cpx_t *corr, sdr_cpx_t *C);

/* Replaces src/sdr_func.c:1029-1057 (sdr_corr_std_cpx_code,
 * src/pocket_sdr.h:417). Complex-code (E5 AltBOC) correlator. */
void sdr_corr_std_cpx_code(const sdr_cpx16_t *IQ, const sdr_cpx16_t *code,
    int N, double coff, const double *pos, int n, sdr_cpx_t *corr,
    sdr_cpx_t *C);

/* Replaces src/sdr_func.c:1060-1072 (sdr_corr_std_cpx, src/pocket_sdr.h:420),
 * the python/sdr_func.py corr_std() binding (python/sdr_func.py:156-171). */
void sdr_corr_std_cpx(const sdr_cpx_t *buff, int len_buff, int ix, int N,
    double fs, double fc, double phi, const float *code, const double *pos,
    int n, sdr_cpx_t *corr);

/* Replaces src/sdr_func.c:1088-1102 (sdr_corr_fft, src/pocket_sdr.h:423).
 * corr = IFFT(FFT(IQ * CSCALE) * code_fft / N^2), FP32, any N whose FFT plan
 * is supported (see sdrg_fft_supported). */
void sdr_corr_fft(const sdr_cpx16_t *IQ, const sdr_cpx_t *code_fft, int N,
    sdr_cpx_t *corr);

/* Replaces src/sdr_func.c:1105-1113 (sdr_corr_fft_cpx, src/pocket_sdr.h:425),
 * the python/sdr_func.py corr_fft() binding (python/sdr_func.py:174-183). */
void sdr_corr_fft_cpx(const sdr_cpx_t *buff, int len_buff, int ix, int N,
    double fs, double fc, double phi, const sdr_cpx_t *code_fft,
    sdr_cpx_t *corr);

/* Replaces src/sdr_func.c:664-687 (sdr_search_code, src/pocket_sdr.h:404).
 * P[i*N+j] += |corr_i[j]|^2 for every Doppler bin i (P is read, accumulated
 * and written back). T is unused, as in the reference. The reference's 1 ms
 * CPU-release sleep every 22 bins is not reproduced. */
void sdr_search_code(const sdr_cpx_t *code_fft, double T,
    const sdr_buff_t *buff, int ix, int N, double fs, double fi,
    const float *fds, int len_fds, float *P);

/* Replaces src/sdr_func.c:690-706 (sdr_corr_max, src/pocket_sdr.h:407).
 * First strict maximum in row-major order and C/N0 from the grid mean. */
float sdr_corr_max(const float *P, int N, int Nmax, int M, double T, int *ix);

/* Replaces src/sdr_func.c:709-744 (sdr_fine_dop, src/pocket_sdr.h:408).
 * Vertex of the parabola through the peak bin and its two neighbours. */
double sdr_fine_dop(const float *P, int N, const float *fds, int len_fds,
    const int *ix);

/* Replaces src/sdr_func.c:757-769 (sdr_dop_bins, src/pocket_sdr.h:411).
 * Returns a malloc'ed array; release it with free() (the reference's
 * sdr_free is free()). */
float *sdr_dop_bins(double T, float dop, float max_dop, int *len_fds);

/* Replaces src/sdr_code.c:2556-2568 (sdr_res_code, src/pocket_sdr.h:462-463).
 * Nearest-chip resampling: sample i < N takes chip
 * (int)((coff*fs + i) * (len_code/T/fs)) % len_code (Q = code_Q's chip, or
 * code_I's for a real code), samples N..N+Nz-1 are 0. Bit-identical to the
 * reference. A code offset that would index before the code (the reference
 * reads out of bounds there) is rejected. */
void sdr_res_code(const int8_t *code_I, const int8_t *code_Q, int len_code,
    double T, double coff, double fs, int N, int Nz, sdr_cpx16_t *code_res);

/* Replaces src/sdr_code.c:2589-2608 (sdr_gen_code_fft, src/pocket_sdr.h:464-465).
 * Conjugated DFT (natural order, N+Nz points) of the resampled replica
 * zero padded by Nz (replica Q = code_Q's chips, or 0 for a real code). FP32
 * mixed-radix FFT on the GPU: N+Nz must be supported (sdrg_fft_supported). */
void sdr_gen_code_fft(const int8_t *code_I, const int8_t *code_Q, int len_code,
    double T, double coff, double fs, int N, int Nz, sdr_cpx_t *code_fft);

/* Replace src/sdr_func.c:311-405 (sdr_lpf_new / sdr_lpf_free / sdr_lpf_apply,
 * src/pocket_sdr.h:449-451): the 9-tap symmetric integer FIR (Hamming-windowed
 * sinc, Q13 taps) applied in place to packed samples, each output clipped to
 * +-7, with the last 8 inputs carried to the next call. sdr_lpf_new returns
 * NULL for a cutoff outside (0, fs/2), as the reference. Bit-identical. */
sdr_lpf_t *sdr_lpf_new(double fc, double fs);
void sdr_lpf_free(sdr_lpf_t *lpf);
void sdr_lpf_apply(sdr_lpf_t *lpf, sdr_cpx8_t *data, int N);

/* Replaces src/sdr_func.c:1141-1182 (sdr_psd_cpx, src/pocket_sdr.h:430-431).
 * Welch PSD without overlap (Hann window, len_buff / N segments), dB/Hz:
 * N/2 bins for IQ = 1, N bins from -fs/2 for IQ = 2. FP32 on the GPU; N must
 * be supported (sdrg_fft_supported). */
void sdr_psd_cpx(const sdr_cpx_t *buff, int len_buff, int N, double fs, int IQ,
    float *psd);

/* =========================================================================
 * Part 2: additive entry points (no reference counterpart)
 * ========================================================================= */

#define SDRG_OK          0
#define SDRG_ERR_ARG    -1   /* invalid argument / unsupported size */
#define SDRG_ERR_CUDA   -2   /* CUDA runtime or launch error */
#define SDRG_ERR_NOMEM  -3   /* device or pinned allocation failed */
#define SDRG_ERR_NODEV  -4   /* no usable CUDA device */

/* Message of the last failed call on this host thread ("" if none); copies
 * at most size-1 bytes into buff and returns the last status code. */
int sdr_gpu_last_error(char *buff, int size);

/* Clears the calling thread's error state. */
void sdr_gpu_clear_error(void);

/* Selects and initialises a device (default: device 0, or $SDRG_DEVICE).
 * Optional; every entry point initialises lazily. */
int sdrg_init(int device);

/* 1 when an FFT of length N has a GPU plan (N = R*M with R in
 * {1,2,3,4,5,6,8} (one thread-block cluster) or {10,12,15,16,20} (staged
 * through a scratch buffer in device memory), M 2-3-5-smooth and small enough for one
 * CTA's shared memory (<= ~27 000)), else 0. */
int sdrg_fft_supported(int N);

/* Library version string. */
const char *sdrg_version(void);

/* Error-path testing: the after-th following device or pinned allocation
 * attempt of the library (0: the next one) fails as an out-of-memory
 * cudaMalloc would (SDRG_ERR_NOMEM); -1 cancels. SDRG_FAIL_ALLOC=n in the
 * environment sets it once at start-up. Nothing is allocated or faulted on
 * the device. */
void sdrg_inject_alloc_failure(int after);

/* Error-path testing of the staged splits (lengths split more than 8 ways,
 * e.g. 480 000 points): the next n staged inverse-FFT launches give up their
 * first wait for each bulk copy into shared memory at once, as if its bound
 * (about 2 s) had run out. Each copy is still issued in full, lands and is
 * waited for with the full bound before its data is used; the launch records
 * the failure in its error word, and the synchronous call that ran it
 * (sdr_search_code, sdr_corr_fft, sdrg_acq_run_host) returns / records
 * SDRG_ERR_CUDA and clears the word, so the next call runs normally. Nothing
 * is faulted or left waiting on the device. 0 cancels. */
int sdrg_inject_stage_timeout(int n);

/* ---- FFT schedules --------------------------------------------------------
 * The reference keeps FFTW planning wisdom in a file (sdr_func_init(file),
 * src/sdr_func.c:118-121). Here a transform length's schedule - how it is
 * split over CTAs (R) and the CTA size - can be chosen by timing the
 * candidates on the device (sdrg_fft_autotune) and kept in a schedule file;
 * sdr_func_init(file) loads that file when it exists (lines
 * "sdrg_fft <L> <R> <threads> <ms>"; anything else in the file is ignored).
 * Plans built after a schedule is set use it; without one the library's
 * default rule applies (smallest split that fits one CTA). R = 0 in
 * sdrg_fft_schedule_set removes a schedule. Results do not depend on the
 * schedule beyond FP32 rounding. */
int sdrg_fft_autotune(int L, int *R, int *threads, double *ms);
int sdrg_fft_schedule_set(int L, int R, int threads);
int sdrg_fft_schedule_get(int L, int *R, int *threads);   /* 1: set, 0: none */
int sdrg_fft_schedule_save(const char *path);
int sdrg_fft_schedule_load(const char *path);             /* entries loaded, or < 0 */

/* ---- FFT correlator that allocates nothing --------------------------------
 * No counterpart in the reference (an addition of this library).
 * Same result as sdr_corr_fft (corr = IFFT(FFT(IQ * CSCALE) * code_fft / N^2),
 * within FP32 rounding) for callers that cannot call cudaMalloc: a real-time
 * receiver channel thread that must not stall on the device-wide
 * synchronisation an allocation may bring, or a host application whose
 * device memory all comes from its own pool or budget. Inputs and output
 * are DEVICE pointers owned by the caller (IQ_dev: N mixed samples,
 * code_fft_dev: N conjugated code-DFT values in natural order, corr_dev: N
 * outputs); `stream` is a cudaStream_t (NULL = the legacy default stream);
 * the call is asynchronous on it and allocates nothing.
 * All intermediate data (permuted code DFT, forward spectrum, FFT tables)
 * live in one fixed device array of about 1.8 MB that every GPU loading the
 * library holds until the process exits; N above SDRG_NOALLOC_MAX_N (65536),
 * or a length whose cluster split does not fit that array, is rejected with
 * SDRG_ERR_ARG. FFT schedules (sdrg_fft_schedule_set, autotuning) do not
 * apply: this entry always takes the default split of N. The first call on
 * a device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current; make that first call before any stream capture.
 * Every call shares the array and leaves its contents behind; each call
 * first rewrites every table it reads, so no call depends on an earlier
 * one, but calls that overlap on the GPU (other streams, other host threads)
 * race on the array and must be serialised by the caller. Returns SDRG_OK or
 * a negative status. */
#define SDRG_NOALLOC_MAX_N 65536
int sdrg_corr_fft_noalloc(const sdr_cpx16_t *IQ_dev, const sdr_cpx_t *code_fft_dev,
    int N, sdr_cpx_t *corr_dev, void *stream);

/* ---- batched parallel-code-phase acquisition ----------------------------
 * One signal group = one code family at one sampling setup: all its PRNs
 * share L, fs, fi, Doppler bins and sums, so the forward FFT of every
 * (Doppler bin, sum) is computed once and reused by every PRN. */
typedef struct {
    int L;                 /* FFT length (samples mixed per coherent block) */
    int N;                 /* sample advance between non-coherent sums */
    int Nmax;              /* code offsets kept per Doppler bin (grid cols) */
    int n_sum;             /* non-coherent sums */
    int n_prn;             /* PRNs (code FFTs) in this group */
    int len_fds;           /* Doppler bins */
    double fs, fi, T;      /* sampling rate, IF (Hz), coherent time (s) */
    const float *fds;      /* [len_fds] Doppler bins (Hz), HOST */
    const sdr_cpx_t *code_fft; /* [n_prn][L] conjugated code DFTs, HOST, or
                              NULL (zeros until sdrg_acq_set_codes) */
    int buf;               /* index of the IF buffer this group reads */
} sdrg_acq_sig_t;

/* Per (group, PRN) result of one sdrg_acq_run. */
typedef struct {
    int bin, offset;       /* peak Doppler bin and code offset (samples) */
    float cn0;             /* C/N0 (dB-Hz), as sdr_corr_max */
    float pmax;            /* peak power */
    double pave;           /* grid mean power */
    double fd;             /* fine Doppler (Hz), as sdr_fine_dop */
} sdrg_acq_result_t;

typedef struct sdrg_acq_plan sdrg_acq_plan_t;

/* Builds a plan: uploads the code FFTs (permuted for the kernels), FFT
 * tables, Doppler phase steps and allocates the grid and work buffers.
 * Returns NULL on error (see sdr_gpu_last_error). */
sdrg_acq_plan_t *sdrg_acq_plan_new(const sdrg_acq_sig_t *sigs, int n_sig);
void sdrg_acq_plan_free(sdrg_acq_plan_t *plan);

/* Total grid cells (sum over groups of n_prn * len_fds * Nmax). */
int64_t sdrg_acq_plan_cells(const sdrg_acq_plan_t *plan);

/* Runs the whole search on `stream` (a cudaStream_t, NULL = the calling
 * thread's stream). if_dev[b] is a DEVICE pointer to packed IF buffer b of
 * len_if[b] samples (circular); ix[b] is the first sample of sum 0. Results
 * for group g, PRN p are written to res_dev[offset_g + p] (DEVICE pointer;
 * offset_g = sum of n_prn of the groups before g). Asynchronous. */
int sdrg_acq_run(sdrg_acq_plan_t *plan, const uint8_t *const *if_dev,
    const int *len_if, const int *ix, sdrg_acq_result_t *res_dev,
    void *stream);

/* sdrg_acq_run through a CUDA graph. The first call, and a call whose IF
 * buffer pointers, lengths or result pointer differ from the ones captured,
 * captures the plan's launch sequence (fork to the internal streams, every
 * group's forward / consumer / peak kernels, join) into a graph; every call
 * then uploads the start-sample tables on `stream` when ix changed and
 * replays the graph there: one launch per run. Same results as
 * sdrg_acq_run; kernel timing (sdrg_acq_profile) does not see graph runs.
 * The graph is released with the plan. */
int sdrg_acq_run_graph(sdrg_acq_plan_t *plan, const uint8_t *const *if_dev,
    const int *len_if, const int *ix, sdrg_acq_result_t *res_dev,
    void *stream);

/* Number of graph captures sdrg_acq_run_graph has made for the plan. */
int sdrg_acq_graph_captures(const sdrg_acq_plan_t *plan);

/* How a run issues its consumer work (the per-PRN loop of
 * app/pocket_acq/pocket_acq.c:152-192 and search_sig, src/sdr_ch.c:398-450,
 * done as one work list). mode 1: every group's (PRN, Doppler bin) tasks are
 * one work list consumed by a single persistent launch (clusters of 8 CTAs
 * where they fit, of 2 elsewhere; tasks claimed dynamically, the 8-way
 * splits first), after one forward-transform launch for all groups, all on
 * the caller's stream; needs every group on the 24 000-point sub-transform
 * with split 2 or 8 (48 000 / 192 000 points), else SDRG_ERR_ARG. mode 0
 * (default, the faster on the multi-GNSS benchmark): each group's forward /
 * consumer / peak launches on concurrent internal streams. mode -1: the work
 * list where the plan allows it, else per-group launches. The
 * arithmetic is the same either way (grids agree within FP32 rounding, the
 * kernels being compiled apart; same peaks). Returns 1 when runs use the work
 * list, 0 when not, or a negative status. A captured graph is re-captured
 * on the next sdrg_acq_run_graph after a change. */
int sdrg_acq_set_worklist(sdrg_acq_plan_t *plan, int mode);

/* Device pointer to the accumulated grid of group g, laid out
 * [n_prn][len_fds][Nmax] (float), valid after sdrg_acq_run completes. */
const float *sdrg_acq_grid(const sdrg_acq_plan_t *plan, int g);

/* Copies the grid of group g to HOST memory dst (n_prn*len_fds*Nmax floats),
 * after the plan's last run on its stream has completed (synchronous). */
int sdrg_acq_grid_host(const sdrg_acq_plan_t *plan, int g, float *dst);

/* Kernel timing: when enabled, every sdrg_acq_run records CUDA events on its
 * stream around each kernel launch. sdrg_acq_profile_get waits for them and
 * returns, since the last get, the summed milliseconds and launch counts per
 * group g and kernel: index 3*g + 0 forward FFT, 3*g + 1 consumer (code
 * multiply + inverse FFT + power), 3*g + 2 peak reduction; then, at
 * 3*n_sig + k, the per-run span of kernel kind k over all groups (earliest
 * start to latest end; groups run concurrently on internal streams) summed
 * over runs, with the number of runs. Arrays hold 3*n_sig + 3 entries.
 * Resets after reading. */
int sdrg_acq_profile(sdrg_acq_plan_t *plan, int enable);
int sdrg_acq_profile_get(sdrg_acq_plan_t *plan, double *ms, int64_t *launches);

/* ---- batched tracking correlators ------------------------------------------
 * One job = what src/sdr_ch.c:725-733 does for one channel and one code
 * period: sdr_mix_carr(buff[buf], ix, N, fs, fc, phi, IQ) followed by
 * sdr_corr_std (or sdr_corr_std_cpx_code when cpx_code) on that IQ with the
 * channel's SDR_N_CODES x N code bank, code offset coff (samples) and n tap
 * positions pos (samples). Results are bit-identical to those two calls. */
typedef struct {
    int buf;                    /* IF buffer index */
    int ix;                     /* first sample in the circular buffer */
    int N;                      /* samples (one code period) */
    double fs, fc, phi;         /* sdr_mix_carr arguments */
    double coff;                /* sdr_corr_std code offset (samples) */
    const sdr_cpx16_t *code;    /* DEVICE pointer: code bank [SDR_N_CODES][N] */
    int cpx_code;               /* 1: complex-code correlator */
    int n;                      /* taps (1..SDR_MAX_CORR) */
    const double *pos;          /* HOST pointer: n tap positions (samples) */
} sdrg_corr_job_t;

/* Runs n_job jobs on `stream` (NULL = the calling thread's stream); if_dev /
 * len_if describe the device IF buffers. corr_dev receives
 * [n_job][SDR_MAX_CORR] correlations, C_dev (may be NULL) [n_job][2] boundary
 * partials, both DEVICE pointers. Asynchronous. */
int sdrg_corr_batch(const sdrg_corr_job_t *jobs, int n_job, const uint8_t *const *if_dev,
    const int *len_if, sdr_cpx_t *corr_dev, sdr_cpx_t *C_dev, void *stream);

/* ---- carrier wipe-off on the device -----------------------------------------
 * sdr_mix_carr (src/sdr_func.c:824-836) on a device-resident circular IF
 * buffer: IQ_dev[n] = the window sample (ix + n) mod len of buf_dev (len
 * packed sdr_cpx8_t samples) mixed with the carrier of frequency fc and phase
 * phi (cycles) at sample ix, the phase restarting at the buffer wrap as in the
 * reference. Bit-identical to sdr_mix_carr. DEVICE pointers; asynchronous on
 * `stream` (NULL = the legacy default stream). */
int sdrg_mix_carr(const uint8_t *buf_dev, int len, int ix, int N, double fs,
    double fc, double phi, sdr_cpx16_t *IQ_dev, void *stream);

/* ---- spreading-code chips (host) -------------------------------------------
 * The reference's sdr_gen_code / sdr_sec_code (src/sdr_code.c:2173-2182,
 * :2274-2283; src/pocket_sdr.h:454-455) for the signals of the search and
 * tracking paths: "L1CA" (PRN 1-210), "L5I" / "L5Q" (1-210), "L6D" (193-202),
 * "L6E" (203-212), "E1B" (1-50, BOC(1,1) sub-carrier applied: 8184 values)
 * and "B1I" (1-63); case-insensitive. Same chips as the reference: +1 / -1,
 * 0 in the off slots of time-multiplexed codes (L6D / L6E). Secondary codes:
 * NH10 (L5I), NH20 (L5Q, B1I PRN 6-58), the Manchester overlay of SBAS L5
 * (PRN 120-158), otherwise the one-chip code {1}. Host only, no device work.
 * Returns the code length and, if `chips` is not NULL, writes the chips there
 * (`cap` values available; fewer than the length is SDRG_ERR_ARG). An
 * unknown signal or PRN returns SDRG_ERR_ARG (the reference returns NULL). */
int sdrg_gen_code(const char *sig, int prn, int8_t *chips, int cap);
int sdrg_sec_code(const char *sig, int prn, int8_t *chips, int cap);

/* ---- replicas on the device ------------------------------------------------
 * Batched forms of sdr_res_code / sdr_gen_code_fft (src/sdr_code.c:2556-2608)
 * for n_code codes of len_code chips each, stored back to back
 * (code_I_dev[c * len_code + i]; code_Q_dev likewise, or NULL for real
 * codes). All pointers are DEVICE pointers; `stream` is a cudaStream_t
 * (NULL = the legacy default stream); asynchronous.
 *
 * sdrg_res_code writes code_res_dev[(c * n_bank + b) * (N + Nz) + i] =
 * sdr_res_code(code c, coff - b / fs / n_bank)[i] for b < n_bank <= 32; with
 * coff = 0 and n_bank = SDR_N_CODES these are a tracking channel's
 * fractional-phase code banks (src/sdr_ch.c:265-272), bit-identical.
 *
 * sdrg_gen_code_fft writes code_fft_dev[c * (N + Nz) + k] =
 * sdr_gen_code_fft(code c, coff)[k]; its sub-spectra scratch is
 * stream-ordered (cudaMallocAsync / cudaFreeAsync on `stream`). */
int sdrg_res_code(const int8_t *code_I_dev, const int8_t *code_Q_dev, int len_code,
    int n_code, double T, double coff, double fs, int N, int Nz, int n_bank,
    sdr_cpx16_t *code_res_dev, void *stream);
int sdrg_gen_code_fft(const int8_t *code_I_dev, const int8_t *code_Q_dev, int len_code,
    int n_code, double T, double coff, double fs, int N, int Nz,
    sdr_cpx_t *code_fft_dev, void *stream);

/* Sets the code DFTs of plan group g on the device from chips, replacing
 * what sdrg_acq_plan_new uploaded (a plan may also be created with
 * code_fft = NULL for a group and get its codes only from here): PRN p of
 * the group takes code_I_dev[p * len_code ...] (n_prn codes, DEVICE), code
 * period T, offset coff, an N-sample replica zero padded to the group's L
 * (the receiver's acquisition uses N = L / 2, src/sdr_ch.c:197). Same values
 * as sdr_gen_code_fft, written directly in the plan's internal layout.
 * `stream` NULL = the calling thread's stream; asynchronous; a later
 * sdrg_acq_run on the same stream sees the new codes. */
int sdrg_acq_set_codes(sdrg_acq_plan_t *plan, int g, const int8_t *code_I_dev,
    const int8_t *code_Q_dev, int len_code, double T, double coff, int N, void *stream);

/* ---- PSD on the device ----------------------------------------------------
 * sdr_psd_cpx on DEVICE data (buff_dev: len_buff complex floats; psd_dev:
 * N/2 or N floats), and straight from a packed IF buffer: n samples of the
 * circular cpx8 buffer if_dev (len_if samples) from sample ix - the window the
 * receiver's sdr_rcv_rfch_psd (src/sdr_rcv.c:395-412) unpacks to floats
 * first. Asynchronous on `stream` (NULL = the legacy default stream);
 * scratch is stream-ordered (cudaMallocAsync). */
int sdrg_psd(const sdr_cpx_t *buff_dev, int len_buff, int N, double fs, int IQ,
    float *psd_dev, void *stream);
int sdrg_psd_if(const uint8_t *if_dev, int len_if, int ix, int n, int N, double fs,
    int IQ, float *psd_dev, void *stream);

/* ---- batched signal search ---------------------------------------------------
 * The receiver searches one channel at a time: update_srch_ch
 * (src/sdr_rcv.c:1222-1257) gives the search to the next IDLE channel, whose
 * search_sig (src/sdr_ch.c:398-450) accumulates sdr_search_code over one code
 * period per update until n_sum * T >= sdr_t_acq and then decides with
 * sdr_corr_max / sdr_fine_dop. sdrg_search_batch runs that whole search for
 * every channel the caller submits (the caller keeps the receiver's choice of
 * which channels are ready: re-acquisition, assisted or short-code ones) in
 * one batched acquisition on the device: unaided channels of one code setup
 * share a signal group with sdr_dop_bins(T, 0, max_dop) bins; a channel with an
 * external Doppler aid gets its own fd_ext_n (default 3) bins of 0.5 / T around
 * fd_ext. Sum s uses samples [ix + s N, ix + s N + 2 N) of its IF buffer, the
 * windows of consecutive code periods from ix. */
typedef struct {
    const int8_t *code_dev; /* [n_prn][len_code] code chips, DEVICE */
    int len_code, n_prn;
    double T;              /* code period (s) */
    double fs, fi;         /* sampling rate, IF (Hz) */
    int N;                 /* samples per code period (FFTs of 2 N) */
    double max_dop;        /* Doppler range (Hz), the receiver's sdr_max_dop */
    int buf;               /* IF buffer index */
} sdrg_srch_setup_t;

typedef struct {
    int setup;             /* setup index */
    int prn;               /* code row within the setup */
    float fd_ext;          /* external Doppler aid (Hz), 0: none (sdr_acq_t) */
    int fd_ext_n;          /* aided bins, 0: 3 */
} sdrg_srch_req_t;

typedef struct {
    int found;             /* C/N0 >= thres_cn0: start tracking */
    int bin, offset;       /* peak Doppler bin (of the request's bins), offset */
    float cn0;             /* C/N0 (dB-Hz), as sdr_corr_max */
    double fd;             /* fine Doppler (Hz), as sdr_fine_dop */
    double coff;           /* code offset (s) = offset / fs, as start_track gets */
    int n_sum;             /* code periods accumulated */
} sdrg_srch_res_t;

/* Runs every request's search (res[i] for req[i]); if_dev / len_if: DEVICE
 * IF buffers; t_acq: the receiver's sdr_t_acq (s); thres_cn0: its
 * sdr_thres_cn0_l. Synchronous (returns with the results on the host);
 * work is issued on `stream` (NULL = the calling thread's stream). The
 * acquisition plan of the last call is kept per host thread and reused by
 * the next call with the same group structure (same setups, request counts
 * and bins); sdrg_search_release frees it (it is also freed at thread exit). */
int sdrg_search_batch(const sdrg_srch_setup_t *setups, int n_setup,
    const sdrg_srch_req_t *req, int n_req, const uint8_t *const *if_dev,
    const int *len_if, int ix, double t_acq, double thres_cn0, sdrg_srch_res_t *res,
    void *stream);

/* The grouping sdrg_search_batch uses (host only, no device work): returns
 * the number of signal groups (or a negative status) and, if non-NULL, each
 * request's group and each group's sums and Doppler bins. */
void sdrg_search_release(void);

int sdrg_srch_groups(const sdrg_srch_setup_t *setups, int n_setup,
    const sdrg_srch_req_t *req, int n_req, double t_acq, int *group_of_req,
    int *n_sum, int *len_fds);

/* ---- IF ingest ----------------------------------------------------------------
 * One block of raw front-end data into the IF buffers on the device: what the
 * receiver's write_buff (src/sdr_rcv.c:840-936) does per block - raw samples
 * through the format's tables (gen_LUT8 / gen_LUTC / gen_LUTC_rtoc,
 * src/sdr_rcv.c:773-829; real-sampled channels of INT8 and RAW8/16/32 get the
 * fs/4 real-to-complex mix), the LPF of the filtered channels
 * (src/sdr_func.c:361-405: every RF channel of RAW8/16/32, channel 0
 * otherwise) and, for the multi-channel RAW formats, the array channels
 * (sdr_arch_combine, src/sdr_array.c:553-578). Bit-identical bytes. */
typedef struct {
    int fmt;                     /* SDR_FMT_INT8 .. SDR_FMT_CS16 */
    int N;                       /* samples per RF channel per block */
    double fs;                   /* sampling rate (Hz), for the LPF taps */
    int IQ[SDR_MAX_RFCH];        /* per RF channel: 1 real (I), 2 complex (IQ) */
    int bits[SDR_MAX_RFCH];      /* per RF channel: bits per component */
    double lut_off[2];           /* INT8/INT8X2/CS8/CS16: raw -> int8 table */
    double lut_scale[2];         /*   round((raw - off) / scale), clipped to +-7;
                                    [1] is CS16's Q table (src/sdr_rcv.c:801-813) */
    double lpf_fc[SDR_MAX_RFCH]; /* LPF cutoff per RF channel (Hz), <= 0: none */
    int narch;                   /* array channels (RAW8/16/16I/32 only) */
    int arch_on[SDR_MAX_ARCH];   /* 0: not written (sdr_arch_t.scale <= 0) */
    int16_t w[SDR_MAX_ARCH][SDR_MAX_RFCH][2]; /* Q8 weights (re, im), sdr_arch_t.w */
} sdrg_ingest_cfg_t;

typedef struct sdrg_ingest sdrg_ingest_t;

/* Builds the tables and LPF taps on the device; NULL on error. */
sdrg_ingest_t *sdrg_ingest_new(const sdrg_ingest_cfg_t *cfg);
void sdrg_ingest_free(sdrg_ingest_t *ing);

/* raw_dev: one block (N samples, the format's bytes per sample), DEVICE.
 * buf_dev[b] (HOST array of DEVICE pointers): RF channel buffers b < n_rf
 * (2, 4, 8 or 8 for RAW8/16/16I/32, else 1) then the narch array channel
 * buffers; the block lands at [base, base + N) of each. ix: the block
 * counter (the fs/4 phase of its first sample is (ix * N) & 3, as the
 * receiver's, src/sdr_rcv.c:846). Asynchronous on `stream` (a cudaStream_t,
 * NULL = the legacy default stream); the LPF history passes from one call to
 * the next, so calls on one ingest object must be ordered (one stream). */
int sdrg_ingest_run(sdrg_ingest_t *ing, const uint8_t *raw_dev, int64_t ix,
    uint8_t *const *buf_dev, int base, void *stream);

/* The LPF taps sdr_lpf_new computes for (fc, fs) into h[9]; returns 1, or 0
 * (h untouched) when the cutoff is outside (0, fs/2). */
int sdrg_lpf_taps(double fc, double fs, int *h);

/* ---- QZSS L6 CSK tracking ---------------------------------------------------
 * What a tracking L6D / L6E channel does per code period (src/sdr_ch.c:705-720):
 * sdr_mix_carr of its window, sdr_corr_fft with the code bank of its
 * fractional code phase, and the CSK decode (src/sdr_ch.c:636-664) giving the
 * code-shift symbol and the correlator outputs around it - for every L6
 * channel of an epoch in one call. The decode is bit-identical to the
 * reference's CSK on the same correlation; the correlation itself is the FP32
 * FFT correlator of sdr_corr_fft. */
typedef struct {
    int buf;                   /* IF buffer index */
    int ix;                    /* first sample of the window (the reference's ix + i) */
    int N;                     /* samples per code period */
    double fs, fc, phi;        /* sdr_mix_carr arguments (phi at sample ix) */
    const sdr_cpx_t *code_fft; /* DEVICE: conjugated code DFT of the bank (N values) */
    int len_code;              /* code length incl. TDM zeros (sdr_ch_t.len_code) */
    int n;                     /* correlator taps (<= SDR_MAX_CORR) */
    const double *pos;         /* HOST: tap positions (samples) */
} sdrg_l6_job_t;

/* sym_dev[j]: symbol of job j; C_dev: [n_job][SDR_MAX_CORR] correlator
 * outputs; corr_dev (may be NULL): [n_job][max N] the FFT correlations. All
 * DEVICE pointers; asynchronous on `stream` (NULL = the legacy default
 * stream); scratch is stream-ordered. */
int sdrg_l6_csk_batch(const sdrg_l6_job_t *jobs, int n_job, const uint8_t *const *if_dev,
    const int *len_if, uint8_t *sym_dev, sdr_cpx_t *C_dev, sdr_cpx_t *corr_dev,
    void *stream);

/* The CSK decode alone on n_job given correlations corr_dev [n_job][N] (DEVICE)
 * with common code length and taps (pos: HOST); outputs as above. */
int sdrg_csk_decode(const sdr_cpx_t *corr_dev, int n_job, int N, int len_code,
    const double *pos, int npos, uint8_t *sym_dev, sdr_cpx_t *C_dev, void *stream);

/* Host convenience: copies IF buffers to the device, runs, and copies the
 * n_prn-total results back (synchronous). if_host[b] are HOST pointers. */
int sdrg_acq_run_host(sdrg_acq_plan_t *plan, const uint8_t *const *if_host,
    const int *len_if, const int *ix, sdrg_acq_result_t *res_host);

/* ---- differentiable refinement (no reference counterpart) ------------------
 * The reference stops at the acquisition grid (peak, C/N0 and the three-bin
 * Doppler quadratic of src/sdr_func.c:709-744). These calls refine code
 * delay, Doppler and carrier phase of many signals at once from that peak.
 * Model of one signal over samples n of a packed IF buffer, t = n / fs:
 *   psi(t) / 2 pi = fi t + fd (t - t_ref) + phi
 *   u(t) = rate (t - t_ref) + rate_nom (t_ref - tau) - 1/2   (chips)
 *   replica = chips linearly interpolated at u (through the chip centres)
 * theta = {tau (s), fd (Hz), phi (cycles at t_ref)} per signal, in double;
 * `rate` (chips/s) per signal is the code rate the model uses and is not
 * differentiated. The span is K blocks of Nb samples from ix0; t_ref =
 * (ix0 + K Nb / 2) / fs. Per (signal, block k) the FP32 sums are
 *   {Re C, Im C, Re D, Im D, Re E, Im E, Q, Qt, Qtt, R, P, 0}
 *   C = sum x c e^{-j psi}, D = sum x dc e^{-j psi}, E = sum t' x c e^{-j psi},
 *   Q = sum c^2, Qt = sum t' c^2, Qtt = sum t'^2 c^2, R = sum c dc,
 *   P = sum dc^2, with dc = chip[i+1] - chip[i] and t' the time from the
 *   block centre; so dC/dtau = -rate_nom D, dC/dphi = -2 pi j C and
 *   dC/dfd = -2 pi j (E + (t_k - t_ref) C), t_k = block centre. */
typedef struct {
    const int8_t *chips;   /* HOST: Lc chip values (+-1 or 0), copied */
    int Lc;                /* chips per code period (2..65536) */
    double rate;           /* nominal chip rate (chips/s) */
    double fi;             /* IF (Hz) */
    double fc;             /* RF carrier (Hz) for a carrier-aided code rate; 0: none */
} sdrg_refine_sig_t;

typedef struct sdrg_refine_plan sdrg_refine_plan_t;

/* Uploads the signals' chips; iq: 1 complex samples, 0 real (Q nibble
 * ignored). Returns NULL on error (see sdr_gpu_last_error). */
sdrg_refine_plan_t *sdrg_refine_plan_new(const sdrg_refine_sig_t *sigs, int n_sig,
    double fs, int iq, int Nb, int K);
void sdrg_refine_plan_free(sdrg_refine_plan_t *plan);

/* out4 = {n_sig, K, Nb, CTAs per block}. */
int sdrg_refine_plan_info(const sdrg_refine_plan_t *plan, int *out4);

/* Block sums on `stream` (a cudaStream_t; NULL = the legacy default stream,
 * for every sdrg_refine_* call), all DEVICE
 * pointers: if_dev (len_if samples; the span must lie inside, no wrap),
 * theta_dev [n_sig][3] and rate_dev [n_sig] doubles; mode 0 writes C only
 * (out_dev [n_sig][K][2] floats), mode 1 all twelve ([n_sig][K][12]).
 * Asynchronous; allocates nothing. */
int sdrg_refine_sums(sdrg_refine_plan_t *plan, const uint8_t *if_dev, int len_if, int ix0,
    const double *theta_dev, const double *rate_dev, int mode, float *out_dev, void *stream);

/* Vector-Jacobian product of the block correlations: grad_dev[n_sig][3]
 * (double) = d/dtheta sum_k Re(conj(g_k) C_k), from mode-1 sums and g_dev
 * [n_sig][K][2] floats (the upstream gradient of (Re C_k, Im C_k)). */
int sdrg_refine_vjp(sdrg_refine_plan_t *plan, const float *sums_dev, const float *g_dev,
    double *grad_dev, void *stream);

/* Starting theta / rate from acquisition results (DEVICE array of n_sig
 * sdrg_acq_result_t in the plan's signal order, e.g. written by
 * sdrg_acq_run): code phase 0 at sample ix_grid + offset, fd = the fine
 * Doppler, phi = 0, carrier-aided code rate; t_ref from ix0. */
int sdrg_refine_from_peaks(sdrg_refine_plan_t *plan, const sdrg_acq_result_t *res_dev,
    int ix_grid, int ix0, double *theta_dev, double *rate_dev, void *stream);

/* n_step Gauss-Newton steps, step i in model models[i] (HOST array):
 *   0  correlation-power loss: complex amplitude per block (carrier phase
 *      not observable; only tau and fd move);
 *   1  coherent: one real amplitude and a common carrier phase;
 *   2  coherent with a real amplitude per block (data-bit signs).
 * Each step recomputes the mode-1 sums, folds the closed-form carrier phase
 * into phi, eliminates the least-squares amplitudes, solves the 3x3 normal
 * equations of (tau, fd, phi) in FP64, clamps the step to +-0.5 chip and
 * +-fs / (4 Nb) Hz, and sets rate = rate_nom (1 + fd / fc) when fc > 0.
 * theta_dev and rate_dev are updated in place; info_dev (may be NULL)
 * receives [n_step][n_sig][5] doubles {power sum_k |C_k|^2 before the step,
 * d tau (chips), d fd (Hz), d phi (cycles), 1 if the system was solved}.
 * Asynchronous, two kernel launches per step, no allocation and no host
 * synchronisation (capturable in a CUDA graph). */
int sdrg_refine_gn(sdrg_refine_plan_t *plan, const uint8_t *if_dev, int len_if, int ix0,
    double *theta_dev, double *rate_dev, const int *models, int n_step, double *info_dev,
    void *stream);

#ifdef __cplusplus
}
#endif
#endif /* POCKET_SDR_GPU_H */
