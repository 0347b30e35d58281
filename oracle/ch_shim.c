/*
 * ch_shim.c - TEST INFRASTRUCTURE (the checker): exposes the reference
 * channel's QZSS L6 CSK decoder to the parity tests.
 *
 * A tracking L6D / L6E channel correlates each code period with an FFT
 * (sdr_mix_carr + sdr_corr_fft, src/sdr_ch.c:705-716) and then runs CSK
 * (src/sdr_ch.c:636-664): the correlation is linearly interpolated
 * (interp_corr, :626-632) at 511 chip shifts, the strongest one gives the
 * symbol, and the tap outputs are interpolated around it. CSK and interp_corr
 * are file-local (static), so this file compiles src/sdr_ch.c in its own
 * translation unit: the #include below reads it from the reference tree at
 * build time (oracle/Makefile); nothing of it is copied here. The shim sets
 * up only the channel fields CSK reads (N, len_code, tap positions, symbol
 * buffer) and returns what CSK leaves behind.
 */
#include "sdr_ch.c"

/* CSK on corr[N] (complex float): *sym = the symbol CSK appends to the
 * channel's symbol buffer, C[npos] = its correlator outputs. */
void orr_csk(const float *corr, int N, int len_code, const double *pos, int npos, uint8_t *sym,
             float *C)
{
    sdr_ch_t ch;
    memset(&ch, 0, sizeof(ch));
    ch.trk = (sdr_trk_t *)sdr_malloc(sizeof(sdr_trk_t));
    ch.nav = (sdr_nav_t *)sdr_malloc(sizeof(sdr_nav_t));
    ch.N = N;
    ch.len_code = len_code;
    ch.trk->npos = npos;
    ch.trk->nposx = 0;
    for (int i = 0; i < npos; i++) ch.trk->pos[i] = pos[i];
    CSK(&ch, (const sdr_cpx_t *)corr);
    *sym = ch.nav->syms[SDR_MAX_NSYM - 1];
    memcpy(C, ch.trk->C, sizeof(sdr_cpx_t) * npos);
    sdr_free(ch.trk);
    sdr_free(ch.nav);
}
