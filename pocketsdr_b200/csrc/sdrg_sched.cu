// sdrg_sched.cu - batched signal-search scheduling (host code).
//
// Reference: the receiver searches ONE channel at a time. update_srch_ch
// (src/sdr_rcv.c:1222-1257) hands the search to the next IDLE channel in
// round-robin order; that channel's search_sig (src/sdr_ch.c:398-450) runs
// sdr_search_code over one code period per receiver update, accumulating
// until n_sum * T >= sdr_t_acq, then sdr_corr_max decides (C/N0 >=
// sdr_thres_cn0_l) and sdr_fine_dop / the peak offset seed tracking
// (start_track, src/sdr_ch.c:377-395). A channel with an external Doppler
// aid (acq->fd_ext, from re-acquisition or another band) searches only
// fd_ext_n (default 3) bins of 0.5 / T around it.
//
// Here every channel that is ready to search is submitted at once: the
// requests are grouped into signal groups (one per code setup for unaided
// searches, one per aided request with its own bins), the whole accumulation
// (n_sum code periods from ix) runs as one batched acquisition plan on the
// device, and every channel gets the reference's decision and tracking seed.
#include <cstdlib>
#include <cstring>
#include <vector>

#include "sdrg_internal.h"

namespace {

struct SrchGroup {
    int setup = 0;
    bool aided = false;
    std::vector<int> reqs;       // request indices (rows of the group)
    std::vector<float> fds;      // Doppler bins
    int n_sum = 0;
};

// search_sig ends after the update where n_sum * T >= sdr_t_acq
int sums_for(double T, double t_acq)
{
    int n = 1;
    while (n * T < t_acq && n < (1 << 20)) ++n;
    return n;
}

int make_groups(const sdrg_srch_setup_t *su, int n_su, const sdrg_srch_req_t *rq, int n_rq,
                double t_acq, std::vector<SrchGroup> &out)
{
    using namespace sdrg;
    out.clear();
    if (!su || n_su <= 0 || !rq || n_rq <= 0 || !(t_acq > 0.0))
        return set_error(SDRG_ERR_ARG, "search batch: no setups, no requests or t_acq <= 0");
    for (int s = 0; s < n_su; ++s) {
        const sdrg_srch_setup_t &u = su[s];
        if (!(u.T > 0.0) || !(u.fs > 0.0) || u.N <= 0 || u.n_prn <= 0 || u.len_code <= 0 ||
            u.buf < 0 || !(u.max_dop > 0.0))
            return set_error(SDRG_ERR_ARG, "search batch: bad setup %d", s);
    }
    std::vector<int> unaided(n_su, -1);
    for (int i = 0; i < n_rq; ++i) {
        const sdrg_srch_req_t &r = rq[i];
        if (r.setup < 0 || r.setup >= n_su || r.prn < 0 || r.prn >= su[r.setup].n_prn)
            return set_error(SDRG_ERR_ARG, "search batch: request %d: bad setup %d / code %d", i,
                             r.setup, r.prn);
        const sdrg_srch_setup_t &u = su[r.setup];
        if (r.fd_ext != 0.0f) {
            // aided: nw bins of 0.5 / T around fd_ext (src/sdr_ch.c:405-413)
            SrchGroup g;
            g.setup = r.setup;
            g.aided = true;
            g.reqs.push_back(i);
            const int nw = r.fd_ext_n > 0 ? r.fd_ext_n : 3;
            for (int k = 0; k < nw; ++k)
                g.fds.push_back((float)(r.fd_ext + (k - nw / 2) * 0.5 / u.T));
            g.n_sum = sums_for(u.T, t_acq);
            out.push_back(g);
            continue;
        }
        if (unaided[r.setup] < 0) {
            // acq_new's bins: sdr_dop_bins(T, 0, max_dop) (src/sdr_ch.c:204)
            SrchGroup g;
            g.setup = r.setup;
            int n = 0;
            float *f = sdr_dop_bins(u.T, 0.0f, (float)u.max_dop, &n);
            if (!f || n <= 0) {
                free(f);
                return set_error(SDRG_ERR_ARG, "search batch: no Doppler bins for setup %d",
                                 r.setup);
            }
            g.fds.assign(f, f + n);
            free(f);
            g.n_sum = sums_for(u.T, t_acq);
            unaided[r.setup] = (int)out.size();
            out.push_back(g);
        }
        out[unaided[r.setup]].reqs.push_back(i);
    }
    return SDRG_OK;
}

// The last call's plan of this host thread, reused by a call with the same
// group structure (a receiver submits the same kind of batch again and
// again); freed when the structure changes, by sdrg_search_release or at
// thread exit.
struct PlanCache {
    std::vector<double> key;
    sdrg_acq_plan_t *plan = nullptr;
    ~PlanCache() { if (plan) sdrg_acq_plan_free(plan); }
};

PlanCache &plan_cache()
{
    static thread_local PlanCache c;
    return c;
}

std::vector<double> plan_key(const std::vector<sdrg_acq_sig_t> &sigs,
                             const std::vector<SrchGroup> &gs)
{
    std::vector<double> k;
    for (size_t g = 0; g < sigs.size(); ++g) {
        const sdrg_acq_sig_t &s = sigs[g];
        k.insert(k.end(), {(double)s.L, (double)s.N, (double)s.Nmax, (double)s.n_sum,
                           (double)s.n_prn, (double)s.len_fds, s.fs, s.fi, s.T, (double)s.buf});
        k.insert(k.end(), gs[g].fds.begin(), gs[g].fds.end());
    }
    return k;
}

// Gathers n code rows of len bytes: row r of dst is copied from src[r].
__global__ void gather_rows_kernel(const int8_t *const *src, int8_t *dst, int len, int n)
{
    const int r = blockIdx.y;
    if (r >= n) return;
    const int8_t *s = src[r];
    int8_t *d = dst + (size_t)r * len;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x)
        d[i] = s[i];
}

} // namespace

using namespace sdrg;

extern "C" {

void sdrg_search_release(void)
{
    PlanCache &pc = plan_cache();
    if (pc.plan) sdrg_acq_plan_free(pc.plan);
    pc.plan = nullptr;
    pc.key.clear();
}

int sdrg_srch_groups(const sdrg_srch_setup_t *setups, int n_setup, const sdrg_srch_req_t *req,
                     int n_req, double t_acq, int *group_of_req, int *n_sum, int *len_fds)
{
    std::vector<SrchGroup> gs;
    int e;
    if ((e = make_groups(setups, n_setup, req, n_req, t_acq, gs))) return e;
    for (size_t g = 0; g < gs.size(); ++g) {
        for (int i : gs[g].reqs)
            if (group_of_req) group_of_req[i] = (int)g;
        if (n_sum) n_sum[g] = gs[g].n_sum;
        if (len_fds) len_fds[g] = (int)gs[g].fds.size();
    }
    return (int)gs.size();
}

int sdrg_search_batch(const sdrg_srch_setup_t *setups, int n_setup, const sdrg_srch_req_t *req,
                      int n_req, const uint8_t *const *if_dev, const int *len_if, int ix,
                      double t_acq, double thres_cn0, sdrg_srch_res_t *res, void *stream)
{
    if (!if_dev || !len_if || !res || ix < 0)
        return set_error(SDRG_ERR_ARG, "sdrg_search_batch: null argument or ix < 0");
    std::vector<SrchGroup> gs;
    int e;
    if ((e = make_groups(setups, n_setup, req, n_req, t_acq, gs))) return e;
    Device *dev;
    if ((e = ensure_device(&dev))) return e;
    cudaStream_t st = (cudaStream_t)stream;
    if (!st && (e = thread_stream(&st))) return e;

    // one plan group per search group: 2N-point FFTs of an N-sample replica
    // zero padded (acq_new, src/sdr_ch.c:197), N offsets kept
    int n_buf = 0;
    std::vector<sdrg_acq_sig_t> sigs(gs.size());
    for (size_t g = 0; g < gs.size(); ++g) {
        const sdrg_srch_setup_t &u = setups[gs[g].setup];
        sdrg_acq_sig_t &s = sigs[g];
        memset(&s, 0, sizeof(s));
        s.L = 2 * u.N; s.N = u.N; s.Nmax = u.N; s.n_sum = gs[g].n_sum;
        s.n_prn = (int)gs[g].reqs.size(); s.len_fds = (int)gs[g].fds.size();
        s.fs = u.fs; s.fi = u.fi; s.T = u.T; s.fds = gs[g].fds.data(); s.code_fft = nullptr;
        s.buf = u.buf;
        n_buf = u.buf + 1 > n_buf ? u.buf + 1 : n_buf;
    }
    PlanCache &pc = plan_cache();
    std::vector<double> key = plan_key(sigs, gs);
    if (pc.plan && pc.key != key) {
        cudaStreamSynchronize(st);
        sdrg_acq_plan_free(pc.plan);
        pc.plan = nullptr;
    }
    if (!pc.plan) {
        pc.plan = sdrg_acq_plan_new(sigs.data(), (int)sigs.size());
        if (!pc.plan) return tctx().error ? tctx().error : SDRG_ERR_CUDA;
        pc.key = key;
    }
    sdrg_acq_plan_t *plan = pc.plan;

    size_t rows = 0, maxlen = 0;
    for (const SrchGroup &g : gs) {
        rows += g.reqs.size();
        const size_t lc = (size_t)setups[g.setup].len_code;
        maxlen = lc > maxlen ? lc : maxlen;
    }
    int8_t *chips = nullptr;
    sdrg_acq_result_t *rdev = nullptr;
    std::vector<sdrg_acq_result_t> rhost(rows);
    std::vector<int> ixs(n_buf, ix);
    e = SDRG_OK;
    if (stream_alloc((void **)&chips, rows * maxlen, st) != cudaSuccess ||
        stream_alloc((void **)&rdev, rows * sizeof(sdrg_acq_result_t), st) != cudaSuccess) {
        e = cuda_error(cudaGetLastError(), "sdrg_search_batch scratch");
    }
    // each group's codes gathered per request (one kernel over a table of
    // source rows), then the code DFTs on the device
    std::vector<const int8_t *> srcs(rows);
    {
        size_t r = 0;
        for (const SrchGroup &g : gs)
            for (int i : g.reqs) {
                const sdrg_srch_setup_t &u = setups[g.setup];
                srcs[r++] = u.code_dev + (size_t)req[i].prn * u.len_code;
            }
    }
    const int8_t **src_d = nullptr;
    if (!e && (stream_alloc((void **)&src_d, rows * sizeof(int8_t *), st) != cudaSuccess ||
               cudaMemcpyAsync(src_d, srcs.data(), rows * sizeof(int8_t *), cudaMemcpyHostToDevice,
                               st) != cudaSuccess))
        e = cuda_error(cudaGetLastError(), "sdrg_search_batch code table");
    size_t row = 0;
    for (size_t g = 0; g < gs.size() && !e; ++g) {
        const sdrg_srch_setup_t &u = setups[gs[g].setup];
        int8_t *dst = chips + row * maxlen;
        const int n = (int)gs[g].reqs.size();
        gather_rows_kernel<<<dim3((unsigned)((u.len_code + 255) / 256 < 16 ? (u.len_code + 255) / 256 : 16),
                                  (unsigned)n), 256, 0, st>>>(src_d + row, dst, u.len_code, n);
        const cudaError_t ge = cudaGetLastError();
        if (ge != cudaSuccess) e = cuda_error(ge, "code gather");
        if (!e) e = sdrg_acq_set_codes(plan, (int)g, dst, nullptr, u.len_code, u.T, 0.0, u.N, st);
        row += gs[g].reqs.size();
    }
    if (src_d) cudaFreeAsync(src_d, st);
    if (!e) e = sdrg_acq_run(plan, if_dev, len_if, ixs.data(), rdev, st);
    if (!e && (cudaMemcpyAsync(rhost.data(), rdev, rows * sizeof(sdrg_acq_result_t),
                               cudaMemcpyDeviceToHost, st) != cudaSuccess ||
               cudaStreamSynchronize(st) != cudaSuccess))
        e = cuda_error(cudaGetLastError(), "sdrg_search_batch results");
    if (chips) cudaFreeAsync(chips, st);
    if (rdev) cudaFreeAsync(rdev, st);
    cudaStreamSynchronize(st);
    if (e) {                          // a failed plan is not kept
        sdrg_acq_plan_free(plan);
        pc.plan = nullptr;
        return e;
    }

    // search_sig's decision per channel (src/sdr_ch.c:424-447)
    row = 0;
    for (const SrchGroup &g : gs) {
        const sdrg_srch_setup_t &u = setups[g.setup];
        for (size_t j = 0; j < g.reqs.size(); ++j, ++row) {
            const sdrg_acq_result_t &r = rhost[row];
            sdrg_srch_res_t &o = res[g.reqs[j]];
            o.found = r.cn0 >= thres_cn0;
            o.bin = r.bin;
            o.offset = r.offset;
            o.cn0 = r.cn0;
            o.fd = r.fd;
            o.coff = r.offset / u.fs;
            o.n_sum = g.n_sum;
        }
    }
    return SDRG_OK;
}

} // extern "C"
