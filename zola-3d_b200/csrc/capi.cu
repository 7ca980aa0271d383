// C-ABI entry points (include/zola_b200.h).  Host wrappers copy in/out; the
// _dev forms take device pointers and a stream.  Every call validates its
// arguments and reports failures through the return code and zola_last_error.
#include <cuda_runtime.h>

#include <algorithm>

#include <cstring>
#include <new>

#include "zola_internal.h"

using namespace zola;

namespace zola {

int ensure_scratch(zola_ctx* ctx, size_t bytes, std::string& err) {
    if (bytes <= ctx->scratch_bytes) return 0;
    if (ctx->scratch) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->scratch);
        ctx->scratch = nullptr;
        ctx->scratch_bytes = 0;
    }
    cudaError_t e = cudaMalloc(&ctx->scratch, bytes);
    if (e != cudaSuccess) {
        err = std::string("scratch cudaMalloc: ") + cudaGetErrorString(e);
        return ZOLA_E_CUDA;
    }
    ctx->scratch_bytes = bytes;
    return 0;
}

// Staging area of the host-buffer calls: grows in 64 MiB steps, never shrinks,
// so repeated calls of similar size allocate nothing.
int ensure_io(zola_ctx* ctx, size_t bytes) {
    if (bytes <= ctx->io_bytes) return 0;
    const size_t step = (size_t)64 << 20;
    bytes = (bytes + step - 1) / step * step;
    if (ctx->io) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->io);
        ctx->io = nullptr;
        ctx->io_bytes = 0;
    }
    cudaError_t e = cudaMalloc(&ctx->io, bytes);
    if (e != cudaSuccess) {
        ctx->err = std::string("staging cudaMalloc: ") + cudaGetErrorString(e);
        return ZOLA_E_CUDA;
    }
    ctx->io_bytes = bytes;
    return 0;
}

void prof_begin(zola_ctx* ctx, int stage, cudaStream_t st) {
    if (!ctx->profile) return;
    if ((size_t)ctx->ev_used + 2 > ctx->ev_pool.size()) {
        for (int k = 0; k < 64; ++k) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            ctx->ev_pool.push_back(e);
        }
        ctx->ev_stage.resize(ctx->ev_pool.size() / 2);
    }
    ctx->ev_stage[ctx->ev_used / 2] = stage;
    cudaEventRecord(ctx->ev_pool[ctx->ev_used++], st);
}

void prof_end(zola_ctx* ctx, cudaStream_t st) {
    if (!ctx->profile) return;
    cudaEventRecord(ctx->ev_pool[ctx->ev_used++], st);
}

void prof_collect(zola_ctx* ctx) {
    if (!ctx->profile) return;
    for (int k = 0; k + 1 < ctx->ev_used; k += 2) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ctx->ev_pool[k], ctx->ev_pool[k + 1]) == cudaSuccess) {
            int sidx = ctx->ev_stage[k / 2];
            ctx->stage_ms[sidx] += ms;
            ctx->stage_launches[sidx] += 1;
        }
    }
    ctx->ev_used = 0;
}

}  // namespace zola

namespace {

int set_err(zola_ctx* ctx, int code, const char* msg) {
    if (ctx) ctx->err = msg;
    return code;
}

bool check_fit_params(zola_ctx* ctx, const zola_fit_params* prm) {
    if (!prm) { ctx->err = "fit params is null"; return false; }
    if (prm->max_iter < 1 || prm->max_iter > 1000) { ctx->err = "max_iter must be in [1, 1000]"; return false; }
    if (!(prm->zmax >= prm->zmin) || !(prm->xymax > 0) || !(prm->step_xy > 0) || !(prm->step_z > 0) ||
        !(prm->tol_xyz >= 0)) {
        ctx->err = "fit params: need zmax >= zmin, xymax > 0, step_xy > 0, step_z > 0, tol_xyz >= 0";
        return false;
    }
    if (prm->precision != ZOLA_PREC_FP64 && prm->precision != ZOLA_PREC_SPLIT) {
        ctx->err = "unknown precision";
        return false;
    }
    return true;
}

}  // namespace

extern "C" {

int zola_ctx_create(int device, zola_ctx** out) {
    if (!out) return ZOLA_E_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) return ZOLA_E_NODEV;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return ZOLA_E_NODEV;
    if (prop.major != 10) return ZOLA_E_NODEV;  // built for sm_100a only
    if (cudaSetDevice(device) != cudaSuccess) return ZOLA_E_CUDA;
    zola_ctx* c = new (std::nothrow) zola_ctx();
    if (!c) return ZOLA_E_ARG;
    c->device = device;
    c->num_sms = prop.multiProcessorCount;
    // The context's stream is a blocking stream: CUDA orders it with the legacy
    // default stream, so device buffers that default-stream work (torch's
    // default stream, plain cudaMemcpy) wrote before a call are complete when the
    // call reads them.  The copy stream only carries host-to-device copies of
    // the host-buffer calls and stays non-blocking.
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamDefault) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->feed_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&c->d_counter, 64 * sizeof(int)) != cudaSuccess) {
        delete c;
        return ZOLA_E_CUDA;
    }
    c->d_status_word = c->d_counter + 32;
    cudaMemset(c->d_counter, 0, 64 * sizeof(int));
    *out = c;
    return ZOLA_OK;
}

int zola_ctx_destroy(zola_ctx* ctx) {
    if (!ctx) return ZOLA_E_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->io) cudaFree(ctx->io);
    if (ctx->calib_area) cudaFree(ctx->calib_area);
    if (ctx->calib_fit_area) cudaFree(ctx->calib_fit_area);
    if (ctx->d_counter) cudaFree(ctx->d_counter);
    if (ctx->h_flags) cudaFreeHost(ctx->h_flags);
    if (ctx->h_feed) cudaFreeHost(ctx->h_feed);
    if (ctx->h_tune) cudaFreeHost(ctx->h_tune);
    if (ctx->h_mix) cudaFreeHost(ctx->h_mix);
    for (cudaEvent_t e : ctx->mix_ev)
        if (e) cudaEventDestroy(e);
    for (cudaStream_t x : ctx->mix_stream)
        if (x) {
            cudaStreamSynchronize(x);
            cudaStreamDestroy(x);
        }
    for (cudaEvent_t e : ctx->tune_ev)
        if (e) cudaEventDestroy(e);
    if (ctx->ev_init) cudaEventDestroy(ctx->ev_init);
    cudaStreamSynchronize(ctx->feed_stream);
    cudaStreamDestroy(ctx->feed_stream);
    for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->feed_ev) cudaEventDestroy(e);
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamDestroy(ctx->copy_stream);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return ZOLA_OK;
}

const char* zola_last_error(const zola_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void* zola_ctx_stream(zola_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

long long zola_ctx_launches(const zola_ctx* ctx) { return ctx ? ctx->launches : -1; }

int zola_ctx_profile(zola_ctx* ctx, int enable) {
    if (!ctx) return ZOLA_E_ARG;
    cudaStreamSynchronize(ctx->stream);
    prof_collect(ctx);
    ctx->profile = enable ? 1 : 0;
    return ZOLA_OK;
}

int zola_ctx_stage_stats(zola_ctx* ctx, double* ms, long long* launches, int reset) {
    if (!ctx) return ZOLA_E_ARG;
    cudaStreamSynchronize(ctx->stream);
    prof_collect(ctx);
    for (int k = 0; k < ZOLA_NSTAGES; ++k) {
        if (ms) ms[k] = ctx->stage_ms[k];
        if (launches) launches[k] = ctx->stage_launches[k];
        if (reset) { ctx->stage_ms[k] = 0; ctx->stage_launches[k] = 0; }
    }
    return ZOLA_OK;
}

int zola_psf_load(zola_ctx* ctx, const zola_optics* optics, const double* zernike, int nz, zola_psf** out) {
    if (!ctx || !optics || !out) return set_err(ctx, ZOLA_E_ARG, "zola_psf_load: null argument");
    *out = nullptr;
    cudaSetDevice(ctx->device);
    zola_psf* p = new (std::nothrow) zola_psf();
    if (!p) return set_err(ctx, ZOLA_E_ARG, "out of host memory");
    p->ctx = ctx;
    int rc = build_psf_tables(p, optics, zernike, nz, ctx->err);
    if (rc) {
        if (p->d_tables) cudaFree(p->d_tables);
        delete p;
        return rc;
    }
    *out = p;
    return ZOLA_OK;
}

int zola_psf_free(zola_psf* psf) {
    if (!psf) return ZOLA_E_ARG;
    cudaSetDevice(psf->ctx->device);
    cudaStreamSynchronize(psf->ctx->stream);
    for (auto& kv : psf->win) {
        if (kv.second.d_C) cudaFree(kv.second.d_C);
        if (kv.second.d_G) cudaFree(kv.second.d_G);
        if (kv.second.d_split) free_split_plan(kv.second.d_split);
    }
    if (psf->d_tables) cudaFree(psf->d_tables);
    delete psf;
    return ZOLA_OK;
}

int zola_psf_info(const zola_psf* psf, int* N, int* K) {
    if (!psf || !N || !K) return ZOLA_E_ARG;
    *N = psf->N;
    *K = psf->K;
    return ZOLA_OK;
}

int zola_psf_model_prec_dev(zola_psf* psf, int R, const double* d_xyz, int n, double* d_out, double* d_dout,
                            int precision, void* stream) {
    if (!psf) return ZOLA_E_ARG;
    zola_ctx* ctx = psf->ctx;
    if (n < 0 || (n > 0 && (!d_xyz || !d_out))) return set_err(ctx, ZOLA_E_ARG, "zola_psf_model: bad n or null buffer");
    if (precision != ZOLA_PREC_FP64 && precision != ZOLA_PREC_SPLIT) return set_err(ctx, ZOLA_E_ARG, "unknown precision");
    WindowTables* w = get_window(psf, R, ctx->err);
    if (!w) return ZOLA_E_ARG;
    if (n == 0) return ZOLA_OK;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    if (precision == ZOLA_PREC_SPLIT) {
        if (psf->o.kz_reset) return set_err(ctx, ZOLA_E_ARG, "split model needs kz_reset = 0 tables");
        return launch_model_split(ctx, psf, w, d_xyz, n, d_out, d_dout, st);
    }
    return launch_model_f64(ctx, psf, w, d_xyz, n, d_out, d_dout, st);
}

int zola_psf_model_dev(zola_psf* psf, int R, const double* d_xyz, int n, double* d_out, double* d_dout,
                       void* stream) {
    if (!psf) return ZOLA_E_ARG;
    zola_ctx* ctx = psf->ctx;
    if (n < 0 || (n > 0 && (!d_xyz || !d_out))) return set_err(ctx, ZOLA_E_ARG, "zola_psf_model: bad n or null buffer");
    WindowTables* w = get_window(psf, R, ctx->err);
    if (!w) return ZOLA_E_ARG;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    return launch_model_f64(ctx, psf, w, d_xyz, n, d_out, d_dout, st);
}

int zola_psf_model_prec(zola_psf* psf, int R, const double* xyz, int n, double* out, double* dout, int precision) {
    if (!psf) return ZOLA_E_ARG;
    zola_ctx* ctx = psf->ctx;
    if (n < 0 || (n > 0 && (!xyz || !out))) return set_err(ctx, ZOLA_E_ARG, "zola_psf_model: bad n or null buffer");
    if (R < 4 || R % 2 || R > psf->N) return set_err(ctx, ZOLA_E_ARG, "ROI side must be even, >= 4 and <= the pupil grid");
    if (n == 0) return ZOLA_OK;
    cudaSetDevice(ctx->device);
    DevBuf<double> dx, dout_, ddout;
    size_t rr = (size_t)R * R;
    ZOLA_CUDA_CHECK(dx.alloc(3 * (size_t)n), ctx);
    ZOLA_CUDA_CHECK(dout_.alloc(rr * n), ctx);
    if (dout) ZOLA_CUDA_CHECK(ddout.alloc(3 * rr * n), ctx);
    ZOLA_CUDA_CHECK(cudaMemcpyAsync(dx.p, xyz, 3 * sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream), ctx);
    int rc = zola_psf_model_prec_dev(psf, R, dx.p, n, dout_.p, dout ? ddout.p : nullptr, precision, ctx->stream);
    if (rc) return rc;
    ZOLA_CUDA_CHECK(cudaMemcpyAsync(out, dout_.p, rr * n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), ctx);
    if (dout)
        ZOLA_CUDA_CHECK(cudaMemcpyAsync(dout, ddout.p, 3 * rr * n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), ctx);
    ZOLA_CUDA_CHECK(cudaStreamSynchronize(ctx->stream), ctx);
    return ZOLA_OK;
}

int zola_psf_model(zola_psf* psf, int R, const double* xyz, int n, double* out, double* dout) {
    return zola_psf_model_prec(psf, R, xyz, n, out, dout, ZOLA_PREC_FP64);
}

int zola_ctx_set_pool(zola_ctx* ctx, int max_slots) {
    if (!ctx || max_slots < 0) return ZOLA_E_ARG;
    ctx->split_pool_max = max_slots;
    return ZOLA_OK;
}

int zola_ctx_set_split_mode(zola_ctx* ctx, int mode) {
    if (!ctx || (mode != ZOLA_SPLIT_STAGED && mode != ZOLA_SPLIT_FUSED && mode != ZOLA_SPLIT_FLOW)) return ZOLA_E_ARG;
    ctx->split_mode = mode;
    return ZOLA_OK;
}

int zola_ctx_set_flow(zola_ctx* ctx, int units, const int* ctas) {
    if (!ctx || units < 0) return ZOLA_E_ARG;
    int sum = 0, zeros = 0;
    if (ctas) {
        for (int s = 0; s < zola::FLOW_STAGES; ++s) {
            if (ctas[s] < 0) return set_err(ctx, ZOLA_E_ARG, "zola_ctx_set_flow: negative CTA count");
            zeros += ctas[s] == 0;
            sum += ctas[s];
        }
        if (sum != 0 && (zeros || sum != ctx->num_sms))
            return set_err(ctx, ZOLA_E_ARG,
                           "zola_ctx_set_flow: every stage needs a CTA, and the counts must add up to the SM count");
    }
    ctx->flow_units = units;
    for (int s = 0; s < zola::FLOW_STAGES; ++s) ctx->flow_ctas[s] = ctas ? ctas[s] : 0;
    return ZOLA_OK;
}

int zola_ctx_set_tuning(zola_ctx* ctx, int enable, const char* cache_path) {
    if (!ctx) return ZOLA_E_ARG;
    ctx->tune = enable ? 1 : 0;
    ctx->tune_path = cache_path ? cache_path : "";
    tune_load(ctx);
    return ZOLA_OK;
}

int zola_fit_flow_shape(zola_psf* psf, int R, int* units, int* ctas, double* ns_per_eval) {
    if (!psf) return ZOLA_E_ARG;
    zola_ctx* ctx = psf->ctx;
    WindowTables* w = get_window(psf, R, ctx->err);
    if (!w) return ZOLA_E_ARG;
    FlowShape f;
    const bool tuned = flow_shape(ctx, psf, w, &f, ns_per_eval);
    if (units) *units = f.units;
    if (ctas)
        for (int s = 0; s < zola::FLOW_STAGES; ++s) ctas[s] = f.ctas[s];
    return tuned ? 1 : 0;
}

int zola_ctx_set_round_graphs(zola_ctx* ctx, int enable) {
    if (!ctx) return ZOLA_E_ARG;
    ctx->round_graphs = enable != 0;
    return ZOLA_OK;
}

int zola_fit_split_pool(zola_psf* psf, int R, int* pool, double* ns_per_eval) {
    if (!psf) return ZOLA_E_ARG;
    WindowTables* w = get_window(psf, R, psf->ctx->err);
    if (!w) return ZOLA_E_ARG;
    return split_pool_choice(psf, w, pool, ns_per_eval);
}

int zola_ctx_flow_stats(zola_ctx* ctx, double* busy, double* clocks_per_unit, double* evaluations) {
    if (!ctx) return ZOLA_E_ARG;
    for (int s = 0; s < zola::FLOW_STAGES; ++s) {
        if (busy) busy[s] = ctx->flow_busy[s];
        if (clocks_per_unit) clocks_per_unit[s] = ctx->flow_clk_per_unit[s];
    }
    if (evaluations) *evaluations = ctx->flow_evals;
    return ZOLA_OK;
}

int zola_ctx_set_wait_limit(zola_ctx* ctx, long long clocks) {
    if (!ctx || clocks < 0) return ZOLA_E_ARG;
    ctx->wait_limit = clocks;
    return ZOLA_OK;
}

}  // extern "C"

namespace {

int fit_dev_impl(zola_ctx* ctx, zola_psf* psf, int R, const float* d_rois, const float* d_scmos,
                 const double* d_init5, int n, const zola_fit_params* prm, double* d_out5, double* d_crlb5,
                 double* d_nll, int* d_status, int* d_iters, void* stream, const zola::RoiFeed* feed = nullptr,
                 const int* d_avail = nullptr) {
    if (!ctx || !psf) return ZOLA_E_ARG;
    if (psf->ctx != ctx) return set_err(ctx, ZOLA_E_ARG, "psf belongs to another context");
    if (!check_fit_params(ctx, prm)) return ZOLA_E_ARG;
    if (n < 0 || (n > 0 && (!d_rois || !d_init5 || !d_out5))) return set_err(ctx, ZOLA_E_ARG, "zola_fit_batch: bad n or null buffer");
    if (psf->o.kz_reset) return set_err(ctx, ZOLA_E_ARG, "fit needs a PSF built with kz_reset = 0 (the fit model tables)");
    WindowTables* w = get_window(psf, R, ctx->err);
    if (!w) return ZOLA_E_ARG;
    if (n == 0) return ZOLA_OK;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    if (d_avail && prm->precision != ZOLA_PREC_SPLIT)
        return set_err(ctx, ZOLA_E_ARG, "zola_fit_batch_stream_dev: streaming inputs need split precision");
    if (prm->precision == ZOLA_PREC_SPLIT)
        return launch_fit_split(ctx, psf, w, d_rois, d_scmos, d_init5, n, prm, d_out5, d_crlb5, d_nll, d_status, d_iters,
                                st, feed, d_avail);
    if (feed && feed->n_chunks > 0)  // the FP64 form needs every input before it starts
        ZOLA_CUDA_CHECK(cudaStreamWaitEvent(st, feed->ev[feed->n_chunks - 1], 0), ctx);
    return launch_fit_f64(ctx, psf, w, d_rois, d_scmos, d_init5, n, prm, d_out5, d_crlb5, d_nll, d_status, d_iters, st);
}

int mixed_dev_impl(zola_ctx* ctx, const zola_fit_class* classes, int nclass, cudaStream_t st,
                   const zola::RoiFeed* feeds);

int fit_host_impl(zola_ctx* ctx, zola_psf* psf, int R, const float* rois, const float* scmos, const double* init5,
                  int n, const zola_fit_params* prm, double* out5, double* crlb5, double* nll, int* status,
                  int* iters) {
    if (!ctx || !psf) return ZOLA_E_ARG;
    if (n < 0 || (n > 0 && (!rois || !init5 || !out5))) return set_err(ctx, ZOLA_E_ARG, "zola_fit_batch: bad n or null buffer");
    if (n == 0) return ZOLA_OK;
    cudaSetDevice(ctx->device);
    const size_t rr = (size_t)R * R, nn = (size_t)n;
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    // staging layout: rois | init | out | crlb | nll | status | iters | scmos
    const size_t off_i = al(rr * nn * sizeof(float)), off_o = off_i + al(5 * nn * sizeof(double));
    const size_t off_c = off_o + al(5 * nn * sizeof(double)), off_n = off_c + al(5 * nn * sizeof(double));
    const size_t off_s = off_n + al(nn * sizeof(double)), off_t = off_s + al(nn * sizeof(int));
    const size_t off_v = off_t + al(nn * sizeof(int));
    const size_t total = off_v + (scmos ? al(rr * nn * sizeof(float)) : 0);
    if (ensure_io(ctx, total)) return ZOLA_E_CUDA;
    char* base = (char*)ctx->io;
    float* dr = (float*)base;
    double* di = (double*)(base + off_i);
    double* dout = (double*)(base + off_o);
    double* dcr = crlb5 ? (double*)(base + off_c) : nullptr;
    double* dnll = nll ? (double*)(base + off_n) : nullptr;
    int* dst = status ? (int*)(base + off_s) : nullptr;
    int* dit = iters ? (int*)(base + off_t) : nullptr;
    float* dv = scmos ? (float*)(base + off_v) : nullptr;
    // Inputs go up in chunks of about 32 MB on the copy stream (at most 64 chunks); the
    // split fit starts on the first chunk and takes the others as they land.
    constexpr int MAX_CHUNKS = 64;
    while ((int)ctx->feed_ev.size() < MAX_CHUNKS) {
        cudaEvent_t e;
        ZOLA_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), ctx);
        ctx->feed_ev.push_back(e);
    }
    size_t per = std::max<size_t>(1024, ((size_t)32 << 20) / (rr * sizeof(float) * (scmos ? 2 : 1)));
    per = std::max(per, (nn + MAX_CHUNKS - 1) / MAX_CHUNKS);
    int chunk_end[MAX_CHUNKS];
    int nch = 0;
    cudaStream_t cs = ctx->copy_stream;
    ZOLA_CUDA_CHECK(cudaMemcpyAsync(di, init5, 5 * nn * sizeof(double), cudaMemcpyHostToDevice, cs), ctx);
    for (size_t a = 0; a < nn; a += per, ++nch) {
        const size_t b = std::min(nn, a + per);
        ZOLA_CUDA_CHECK(cudaMemcpyAsync(dr + a * rr, rois + a * rr, (b - a) * rr * sizeof(float), cudaMemcpyHostToDevice,
                                        cs), ctx);
        if (scmos)
            ZOLA_CUDA_CHECK(cudaMemcpyAsync(dv + a * rr, scmos + a * rr, (b - a) * rr * sizeof(float),
                                            cudaMemcpyHostToDevice, cs), ctx);
        ZOLA_CUDA_CHECK(cudaEventRecord(ctx->feed_ev[nch], cs), ctx);
        chunk_end[nch] = (int)b;
    }
    zola::RoiFeed feed;
    feed.n_chunks = nch;
    feed.chunk_end = chunk_end;
    feed.ev = ctx->feed_ev.data();
    int rc = fit_dev_impl(ctx, psf, R, dr, dv, di, n, prm, dout, dcr, dnll, dst, dit, ctx->stream, &feed);
    if (rc) {
        cudaStreamSynchronize(cs);  // no copy may still write the staging area
        return rc;
    }
    if (rc) return rc;
    ZOLA_CUDA_CHECK(cudaMemcpyAsync(out5, dout, 5 * nn * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), ctx);
    if (crlb5) ZOLA_CUDA_CHECK(cudaMemcpyAsync(crlb5, dcr, 5 * nn * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), ctx);
    if (nll) ZOLA_CUDA_CHECK(cudaMemcpyAsync(nll, dnll, nn * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), ctx);
    if (status) ZOLA_CUDA_CHECK(cudaMemcpyAsync(status, dst, nn * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), ctx);
    if (iters) ZOLA_CUDA_CHECK(cudaMemcpyAsync(iters, dit, nn * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), ctx);
    ZOLA_CUDA_CHECK(cudaStreamSynchronize(ctx->stream), ctx);
    return ZOLA_OK;
}

}  // namespace

extern "C" {

int zola_fit_batch_dev(zola_ctx* ctx, zola_psf* psf, int R, const float* d_rois, const double* d_init5, int n,
                       const zola_fit_params* prm, double* d_out5, double* d_crlb5, double* d_nll, int* d_status,
                       int* d_iters, void* stream) {
    return fit_dev_impl(ctx, psf, R, d_rois, nullptr, d_init5, n, prm, d_out5, d_crlb5, d_nll, d_status, d_iters, stream);
}

int zola_fit_batch_stream_dev(zola_ctx* ctx, zola_psf* psf, int R, const float* d_rois, const double* d_init5,
                              const int* d_avail, int n, const zola_fit_params* prm, double* d_out5, double* d_crlb5,
                              double* d_nll, int* d_status, int* d_iters, void* stream) {
    if (ctx && n > 0 && !d_avail) return set_err(ctx, ZOLA_E_ARG, "zola_fit_batch_stream_dev: null ROI count");
    return fit_dev_impl(ctx, psf, R, d_rois, nullptr, d_init5, n, prm, d_out5, d_crlb5, d_nll, d_status, d_iters, stream,
                        nullptr, d_avail);
}

int zola_fit_batch_mixed_dev(zola_ctx* ctx, const zola_fit_class* classes, int nclass, void* stream) {
    if (!ctx || nclass < 0 || nclass > ZOLA_MAX_CLASSES || (nclass > 0 && !classes)) return ZOLA_E_ARG;
    cudaSetDevice(ctx->device);
    return mixed_dev_impl(ctx, classes, nclass, stream ? (cudaStream_t)stream : ctx->stream, nullptr);
}

}  // extern "C"

namespace {

// One class of a mixed batch: its PSF, parameters and buffers, and the window
// tables of its ROI size (built here when missing).
int check_mixed_class(zola_ctx* ctx, const zola_fit_class& k, WindowTables** w) {
    if (!k.psf || k.psf->ctx != ctx) return set_err(ctx, ZOLA_E_ARG, "zola_fit_batch_mixed: bad PSF");
    if (!check_fit_params(ctx, &k.prm)) return ZOLA_E_ARG;
    if (k.prm.precision != ZOLA_PREC_SPLIT)
        return set_err(ctx, ZOLA_E_ARG, "zola_fit_batch_mixed: every class needs split precision");
    if (k.n < 0 || (k.n > 0 && (!k.d_rois || !k.d_init5 || !k.d_out5)))
        return set_err(ctx, ZOLA_E_ARG, "zola_fit_batch_mixed: bad n or null buffer");
    if (k.psf->o.kz_reset)
        return set_err(ctx, ZOLA_E_ARG, "fit needs a PSF built with kz_reset = 0 (the fit model tables)");
    *w = get_window(k.psf, k.R, ctx->err);
    return *w ? ZOLA_OK : ZOLA_E_ARG;
}

// feeds (nullable): per class, its input chunks still arriving on the copy stream
int mixed_dev_impl(zola_ctx* ctx, const zola_fit_class* classes, int nclass, cudaStream_t st,
                   const zola::RoiFeed* feeds) {
    zola::MixedClass mc[ZOLA_MAX_CLASSES];
    zola::RoiFeed fd[ZOLA_MAX_CLASSES];
    int m = 0;
    for (int c = 0; c < nclass; ++c) {
        const zola_fit_class& k = classes[c];
        WindowTables* w = nullptr;
        if (int rc = check_mixed_class(ctx, k, &w)) return rc;
        if (k.n == 0) continue;
        const zola_fit_params& pr = k.prm;
        zola::FitParamsDev fp{pr.zmin, pr.zmax, pr.xymax, pr.tol_xyz, pr.step_xy, pr.step_z, pr.max_iter, 1e-3};
        if (feeds) fd[m] = feeds[c];
        mc[m++] = zola::MixedClass{k.psf, w,
                                   zola::FitIO{k.d_rois, nullptr, k.d_init5, k.n, fp, k.d_out5, k.d_crlb5, k.d_nll,
                                               k.d_status, k.d_iters}};
    }
    if (m == 0) return ZOLA_OK;
    return zola::launch_fit_split_mixed(ctx, m, mc, st, feeds ? fd : nullptr);
}

}  // namespace

extern "C" {

int zola_fit_batch_mixed(zola_ctx* ctx, const zola_fit_class* classes, int nclass) {
    if (!ctx || nclass < 0 || nclass > ZOLA_MAX_CLASSES || (nclass > 0 && !classes)) return ZOLA_E_ARG;
    cudaSetDevice(ctx->device);
    // staging layout per class: rois | init | out | crlb | nll | status | iters
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    size_t off[ZOLA_MAX_CLASSES][8] = {};
    size_t total = 0;
    for (int c = 0; c < nclass; ++c) {
        const zola_fit_class& k = classes[c];
        WindowTables* w = nullptr;  // every class is checked before the first copy reads a host buffer
        if (int rc = check_mixed_class(ctx, k, &w)) return rc;
        const size_t n = (size_t)k.n, rr = (size_t)k.R * k.R;
        const size_t sz[7] = {rr * n * 4, n * 40, n * 40, k.d_crlb5 ? n * 40 : 0, k.d_nll ? n * 8 : 0,
                              k.d_status ? n * 4 : 0, k.d_iters ? n * 4 : 0};
        for (int q = 0; q < 7; ++q) {
            off[c][q] = total;
            total += al(sz[q]);
        }
    }
    if (total == 0) return ZOLA_OK;
    if (ensure_io(ctx, total)) return ZOLA_E_CUDA;
    char* base = (char*)ctx->io;
    // Inputs go up on the copy stream in chunks of about 32 MB (at most 64 a class),
    // the classes' chunks interleaved, so that every class starts fitting on its
    // first chunk while the rest are still crossing the host link.
    constexpr int MAX_CHUNKS = 64;
    while ((int)ctx->feed_ev.size() < MAX_CHUNKS * ZOLA_MAX_CLASSES) {
        cudaEvent_t e;
        ZOLA_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), ctx);
        ctx->feed_ev.push_back(e);
    }
    int chunk_end[ZOLA_MAX_CLASSES][MAX_CHUNKS];
    size_t per[ZOLA_MAX_CLASSES];
    zola::RoiFeed feeds[ZOLA_MAX_CLASSES];
    cudaStream_t cs = ctx->copy_stream;
    int most = 0;
    for (int c = 0; c < nclass; ++c) {
        const zola_fit_class& k = classes[c];
        const size_t n = (size_t)k.n, rr = (size_t)k.R * k.R;
        per[c] = std::max<size_t>(1024, ((size_t)32 << 20) / (rr * sizeof(float)));
        per[c] = std::max(per[c], (n + MAX_CHUNKS - 1) / MAX_CHUNKS);
        feeds[c].n_chunks = (int)((n + per[c] - 1) / per[c]);
        feeds[c].chunk_end = chunk_end[c];
        feeds[c].ev = ctx->feed_ev.data() + (size_t)c * MAX_CHUNKS;
        most = std::max(most, feeds[c].n_chunks);
        if (n > 0)
            ZOLA_CUDA_CHECK(cudaMemcpyAsync(base + off[c][1], k.d_init5, n * 40, cudaMemcpyHostToDevice, cs), ctx);
    }
    for (int j = 0; j < most; ++j)
        for (int c = 0; c < nclass; ++c) {
            if (j >= feeds[c].n_chunks) continue;
            const zola_fit_class& k = classes[c];
            const size_t rr = (size_t)k.R * k.R, a = (size_t)j * per[c], b = std::min((size_t)k.n, a + per[c]);
            ZOLA_CUDA_CHECK(cudaMemcpyAsync(base + off[c][0] + a * rr * 4, k.d_rois + a * rr, (b - a) * rr * 4,
                                            cudaMemcpyHostToDevice, cs), ctx);
            ZOLA_CUDA_CHECK(cudaEventRecord(feeds[c].ev[j], cs), ctx);
            chunk_end[c][j] = (int)b;
        }
    zola_fit_class dev[ZOLA_MAX_CLASSES];
    for (int c = 0; c < nclass; ++c) {
        dev[c] = classes[c];
        dev[c].d_rois = (const float*)(base + off[c][0]);
        dev[c].d_init5 = (const double*)(base + off[c][1]);
        dev[c].d_out5 = (double*)(base + off[c][2]);
        dev[c].d_crlb5 = classes[c].d_crlb5 ? (double*)(base + off[c][3]) : nullptr;
        dev[c].d_nll = classes[c].d_nll ? (double*)(base + off[c][4]) : nullptr;
        dev[c].d_status = classes[c].d_status ? (int*)(base + off[c][5]) : nullptr;
        dev[c].d_iters = classes[c].d_iters ? (int*)(base + off[c][6]) : nullptr;
    }
    int rc = mixed_dev_impl(ctx, dev, nclass, ctx->stream, feeds);
    if (rc) {
        cudaStreamSynchronize(cs);  // no copy may still write the staging area
        return rc;
    }
    cudaStream_t st = ctx->stream;
    for (int c = 0; c < nclass; ++c) {
        const zola_fit_class& k = classes[c];
        const size_t n = (size_t)k.n;
        if (n == 0) continue;
        ZOLA_CUDA_CHECK(cudaMemcpyAsync(k.d_out5, dev[c].d_out5, n * 40, cudaMemcpyDeviceToHost, st), ctx);
        if (k.d_crlb5) ZOLA_CUDA_CHECK(cudaMemcpyAsync(k.d_crlb5, dev[c].d_crlb5, n * 40, cudaMemcpyDeviceToHost, st), ctx);
        if (k.d_nll) ZOLA_CUDA_CHECK(cudaMemcpyAsync(k.d_nll, dev[c].d_nll, n * 8, cudaMemcpyDeviceToHost, st), ctx);
        if (k.d_status) ZOLA_CUDA_CHECK(cudaMemcpyAsync(k.d_status, dev[c].d_status, n * 4, cudaMemcpyDeviceToHost, st), ctx);
        if (k.d_iters) ZOLA_CUDA_CHECK(cudaMemcpyAsync(k.d_iters, dev[c].d_iters, n * 4, cudaMemcpyDeviceToHost, st), ctx);
    }
    ZOLA_CUDA_CHECK(cudaStreamSynchronize(st), ctx);
    return ZOLA_OK;
}

int zola_fit_batch(zola_ctx* ctx, zola_psf* psf, int R, const float* rois, const double* init5, int n,
                   const zola_fit_params* prm, double* out5, double* crlb5, double* nll, int* status, int* iters) {
    return fit_host_impl(ctx, psf, R, rois, nullptr, init5, n, prm, out5, crlb5, nll, status, iters);
}

int zola_fit_batch_scmos_dev(zola_ctx* ctx, zola_psf* psf, int R, const float* d_rois, const float* d_scmos,
                             const double* d_init5, int n, const zola_fit_params* prm, double* d_out5, double* d_crlb5,
                             double* d_nll, int* d_status, int* d_iters, void* stream) {
    if (ctx && n > 0 && !d_scmos) return set_err(ctx, ZOLA_E_ARG, "zola_fit_batch_scmos: null sCMOS map");
    return fit_dev_impl(ctx, psf, R, d_rois, d_scmos, d_init5, n, prm, d_out5, d_crlb5, d_nll, d_status, d_iters,
                        stream);
}

int zola_fit_batch_scmos(zola_ctx* ctx, zola_psf* psf, int R, const float* rois, const float* scmos,
                         const double* init5, int n, const zola_fit_params* prm, double* out5, double* crlb5,
                         double* nll, int* status, int* iters) {
    if (ctx && n > 0 && !scmos) return set_err(ctx, ZOLA_E_ARG, "zola_fit_batch_scmos: null sCMOS map");
    return fit_host_impl(ctx, psf, R, rois, scmos, init5, n, prm, out5, crlb5, nll, status, iters);
}

}  // extern "C"
