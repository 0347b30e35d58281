/*
 * track_bench.c - test infrastructure (the CPU baseline of the tracking
 * benchmark): runs the reference's own sdr_mix_carr + sdr_corr_std
 * (src/sdr_func.c:824-836, :981-1008; the sequence of a tracking channel's
 * epoch, src/sdr_ch.c:725-733) for a list of correlator jobs over a pool of
 * pthreads, each thread a contiguous share of the jobs, with no Python between
 * calls. Linked against the reference build (oracle/_ref/libsdr_ref.so).
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>

typedef struct { uint8_t *data; int IQ, N; } ref_buff_t;       /* sdr_buff_t */
typedef struct { int8_t I, Q; } ref_cpx16_t;                   /* sdr_cpx16_t */
typedef float ref_cpx_t[2];                                    /* sdr_cpx_t */

void sdr_func_init(const char *file);
void sdr_mix_carr(const ref_buff_t *buff, int ix, int N, double fs, double fc, double phi,
                  ref_cpx16_t *IQ);
void sdr_corr_std(const ref_cpx16_t *IQ, const ref_cpx16_t *code, int N, double coff,
                  const double *pos, int n, ref_cpx_t *corr, ref_cpx_t *C);

typedef struct {
    int buf, ix, N, npos;
    double fs, fc, phi, coff;
    const double *pos;            /* npos tap positions (samples) */
    const ref_cpx16_t *code;      /* SDR_N_CODES x N bank */
    float *corr;                  /* npos x 2 outputs */
} orc_track_job_t;

typedef struct {
    const ref_buff_t *bufs;
    const orc_track_job_t *jobs;
    int j0, j1;
} slice_t;

static void *run_slice(void *arg)
{
    const slice_t *s = (const slice_t *)arg;
    int nmax = 0;
    for (int j = s->j0; j < s->j1; ++j) nmax = s->jobs[j].N > nmax ? s->jobs[j].N : nmax;
    ref_cpx16_t *IQ = (ref_cpx16_t *)malloc(sizeof(ref_cpx16_t) * (nmax > 0 ? nmax : 1));
    if (!IQ) return NULL;
    for (int j = s->j0; j < s->j1; ++j) {
        const orc_track_job_t *b = &s->jobs[j];
        ref_cpx_t C[2];
        sdr_mix_carr(&s->bufs[b->buf], b->ix, b->N, b->fs, b->fc, b->phi, IQ);
        sdr_corr_std(IQ, b->code, b->N, b->coff, b->pos, b->npos, (ref_cpx_t *)b->corr, C);
    }
    free(IQ);
    return NULL;
}

static pthread_once_t init_once = PTHREAD_ONCE_INIT;
static void init_tables(void) { sdr_func_init(""); }   /* the mixing table */

/* Runs every job once over `threads` threads; returns 0, or -1 when a thread
 * cannot start. */
int orc_track_run(const ref_buff_t *bufs, const orc_track_job_t *jobs, int n, int threads)
{
    pthread_once(&init_once, init_tables);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    slice_t sl[256];
    int started = 0, rc = 0;
    for (int t = 0; t < threads; ++t) {
        sl[t].bufs = bufs;
        sl[t].jobs = jobs;
        sl[t].j0 = (int)((long long)n * t / threads);
        sl[t].j1 = (int)((long long)n * (t + 1) / threads);
        if (pthread_create(&th[t], NULL, run_slice, &sl[t]) != 0) { rc = -1; break; }
        started++;
    }
    for (int t = 0; t < started; ++t) pthread_join(th[t], NULL);
    return rc;
}
