/*
 * sdr_oracle.h - CPU restatement of Pocket SDR's signal-search / correlation
 * hot path, used ONLY as a test checker (tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg). The product library never links this code.
 *
 * Every function states the reference lines it restates
 * (paths relative to the Pocket SDR source tree).
 *
 * Types are plain C arrays so the file builds without the reference headers:
 *   packed IF sample  : uint8_t, I in low nibble, Q in high nibble
 *   mixed sample      : int8_t[2] (I, Q)
 *   complex float     : float[2]
 */
#ifndef SDR_ORACLE_H
#define SDR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_N_CODES 10     /* code banks per code (src/pocket_sdr.h:60) */
#define ORC_MAX_CORR 107   /* max correlators (src/pocket_sdr.h:58) */

/* Build the 256-entry carrier table and the 64K mixed-sample table
 * (src/sdr_func.c:113-134). Idempotent. */
void orc_init(void);

/* Raw access to the 64K x (I,Q) table, for table-equivalence tests. */
const int8_t *orc_mix_table(void);

/* Carrier wipe-off over a circular buffer (src/sdr_func.c:772-836). */
void orc_mix_carr(const uint8_t *buff, int len_buff, int ix, int N, double fs,
                  double fc, double phi, int8_t *IQ);

/* Float buffer -> packed 4+4 -> mix (src/sdr_func.c:839-848). */
void orc_mix_carr_cpx(const float *buff, int len_buff, int ix, int N,
                      double fs, double fc, double phi, int8_t *IQ);

/* Standard correlator (src/sdr_func.c:981-1008) and its complex-code form
 * (src/sdr_func.c:1029-1057). cpx_code selects the latter. */
void orc_corr_std(const int8_t *IQ, const int8_t *code, int N, double coff,
                  const double *pos, int n, int cpx_code, float *corr,
                  float *C);

/* Python-facing mix + correlate (src/sdr_func.c:1060-1072). */
void orc_corr_std_cpx(const float *buff, int len_buff, int ix, int N,
                      double fs, double fc, double phi, const float *code,
                      const double *pos, int n, float *corr);

/* In-place-free complex FFT in double precision, any length (mixed radix with
 * a direct DFT for prime factors). dir = 0 forward (exp(-i)), 1 backward
 * (exp(+i)), unnormalised, as the reference's FFT shim
 * (lib/pocketfft/pocketfft_wrap.cpp, src/sdr_func.c:236-264). */
void orc_fft(const double *in, int N, int dir, double *out);

/* FFT correlator (src/sdr_func.c:1088-1102), FFT in double. */
void orc_corr_fft(const int8_t *IQ, const float *code_fft, int N, float *corr);

/* Python-facing mix + FFT correlate (src/sdr_func.c:1105-1113). */
void orc_corr_fft_cpx(const float *buff, int len_buff, int ix, int N,
                      double fs, double fc, double phi, const float *code_fft,
                      float *corr);

/* Parallel code phase search, accumulating into P (src/sdr_func.c:664-687),
 * without the reference's 1 ms CPU-release sleep. */
void orc_search_code(const float *code_fft, const uint8_t *buff, int len_buff,
                     int ix, int N, double fs, double fi, const float *fds,
                     int len_fds, float *P);

/* Peak and C/N0 (src/sdr_func.c:690-706). */
float orc_corr_max(const float *P, int N, int Nmax, int M, double T, int *ix);

/* Fine Doppler by a 3-point quadratic (src/sdr_func.c:709-744). */
double orc_fine_dop(const float *P, int N, const float *fds, int len_fds,
                    const int *ix);

/* Doppler bins (src/sdr_func.c:757-769); returns the count, fills fds when
 * non-NULL. */
int orc_dop_bins(double T, float dop, float max_dop, float *fds);

/* Nearest-chip resampling (src/sdr_code.c:2556-2568); code_Q may be NULL. */
void orc_res_code(const int8_t *code_I, const int8_t *code_Q, int len_code,
                  double T, double coff, double fs, int N, int Nz,
                  int8_t *code_res);

/* Conjugated code DFT (src/sdr_code.c:2589-2608), FFT in double. */
void orc_gen_code_fft(const int8_t *code_I, const int8_t *code_Q,
                      int len_code, double T, double coff, double fs, int N,
                      int Nz, float *code_fft);

/* ---- refinement model (refine_oracle.c; no reference counterpart) ------- */
#define ORC_REFINE_W 12    /* sums per block */

/* FP64 per-block sums for one signal: out[k * 12 + i] =
 * {Re C, Im C, Re D, Im D, Re E, Im E, Q, Qt, Qtt, R, P, 0} with
 * C = sum x c e^{-j psi}, D = sum x dc e^{-j psi}, E = sum t' x c e^{-j psi},
 * Q = sum c^2, Qt = sum t' c^2, Qtt = sum t'^2 c^2, R = sum c dc,
 * P = sum dc^2; dc = chip[i+1] - chip[i]; theta = {tau (s), fd (Hz),
 * phi (cycles at t_ref)}. */
void orc_refine_sums(const int8_t *chips, int Lc, double rate_nom, double rate,
                     double fi, const double *theta, const uint8_t *buf, int iq,
                     double fs, int ix0, int Nb, int K, double *out);

/* One Gauss-Newton step from the block sums (model 0: power loss with
 * complex block amplitudes; 1: one real amplitude and a common carrier phase;
 * 2: real block amplitudes and a common carrier phase); updates theta and
 * rate, info[5] = {power, d tau (chips), d fd (Hz), d phi (cycles), solved}. */
void orc_refine_step(const double *sums, int K, int Nb, double fs, double rate_nom,
                     double fc, int model, double *theta, double *rate, double *info);

/* Welch PSD of float IQ data (src/sdr_func.c:1141-1182). */
void orc_psd_cpx(const float *buff, int len_buff, int N, double fs, int IQ, float *psd);

/* L6 CSK decode of an N-point FFT correlation (src/sdr_ch.c:626-664). */
void orc_csk(const float *corr, int N, int len_code, const double *pos, int npos, uint8_t *sym,
             float *C);

/* IF ingest (ingest_oracle.c): raw front-end blocks -> packed cpx8 buffers,
 * per-channel LPF and array combine, as src/sdr_rcv.c:773-936,
 * src/sdr_func.c:311-405 and src/sdr_array.c:487-578. */
void orc_gen_lut8(int fmt, double off, double scale, int8_t *out);
void orc_gen_lutc(int fmt, int rfch, int IQ, int bits, int rtoc, uint8_t *out);
int orc_lpf_taps(double fc, double fs, int *h);
void *orc_ingest_new(int fmt, int N, const int *IQ, const int *bits, const double *off,
                     const double *scale, const double *lpf_fc, double fs, int narch,
                     const int16_t *w, const int *arch_on);
void orc_ingest_write(void *g, const uint8_t *raw, int64_t ix, uint8_t *out);
void orc_ingest_free(void *g);
void *orc_lpf_new(double fc, double fs);
void orc_lpf_apply(void *f, uint8_t *data, int N);
void orc_lpf_free(void *f);

#ifdef __cplusplus
}
#endif
#endif
