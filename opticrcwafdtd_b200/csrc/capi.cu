// capi.cu -- the extern "C" entry points of liborf_fdtd.so (include/orf_fdtd.h).
#include "engine.cuh"
#include "job2d.cuh"
#include "job3d.cuh"

using namespace orf;

namespace orf {

orf_ctx* default_ctx(int* status) {
    static thread_local orf_ctx* ctxs[64] = {nullptr};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("no CUDA device: %s", cudaGetErrorString(e));
        *status = ORF_ENODEV;
        return nullptr;
    }
    if (dev >= 64) { *status = ORF_ENODEV; return nullptr; }
    if (!ctxs[dev]) {
        orf_ctx* c = nullptr;
        int st = orf_ctx_create(dev, nullptr, &c);
        if (st != ORF_OK) { *status = st; return nullptr; }
        ctxs[dev] = c;
    }
    *status = ORF_OK;
    return ctxs[dev];
}

void ctx_retain(orf_ctx* c) { c->refs.fetch_add(1); }

void ctx_release(orf_ctx* c) {
    if (c->refs.fetch_sub(1) != 1) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    dev_trim(c->device);   // the device blocks cached for reuse go back to the driver
    delete c;
}

}  // namespace orf

extern "C" {

int32_t orf_abi_version(void) { return ORF_ABI_VERSION; }

const char* orf_status_string(int32_t s) {
    switch (s) {
        case ORF_OK: return "ORF_OK";
        case ORF_EINVAL: return "ORF_EINVAL";
        case ORF_ENOMEM_DEVICE: return "ORF_ENOMEM_DEVICE";
        case ORF_ECANCELLED: return "ORF_ECANCELLED";
        case ORF_ETIMEOUT_DEVICE: return "ORF_ETIMEOUT_DEVICE";
        case ORF_ECUDA: return "ORF_ECUDA";
        case ORF_ENODEV: return "ORF_ENODEV";
        case ORF_EBUSY: return "ORF_EBUSY";
        case ORF_ETOOLARGE: return "ORF_ETOOLARGE";
    }
    return "ORF_UNKNOWN";
}

int32_t orf_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return ORF_EINVAL;
    std::snprintf(buf, len, "%s", last_error());
    return ORF_OK;
}

int32_t orf_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int32_t orf_ctx_create(int32_t device, void* stream, orf_ctx** out) {
    if (!out) return ORF_EINVAL;
    *out = nullptr;
    int n = orf_device_count();
    if (n <= 0) { set_error("no CUDA device available"); return ORF_ENODEV; }
    if (device < 0 || device >= n) { set_error("device %d outside 0..%d", device, n - 1); return ORF_EINVAL; }
    ORF_ON_DEVICE(device);
    auto c = new orf_ctx();
    c->device = device;
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (stream) {
        c->stream = static_cast<cudaStream_t>(stream);
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) { delete c; set_error("stream: %s", cudaGetErrorString(e)); return ORF_ECUDA; }
        c->own_stream = true;
    }
    c->tuning.use_graph = 1;
    *out = c;
    return ORF_OK;
}

int32_t orf_ctx_destroy(orf_ctx* c) {
    if (!c) return ORF_EINVAL;
    ctx_release(c);
    return ORF_OK;
}

int32_t orf_ctx_set_tuning(orf_ctx* c, const orf_tuning* t) {
    if (!c || !t) return ORF_EINVAL;
    if (t->tsteps < 0 || t->tsteps > kMaxSub) { set_error("tsteps must be 0..%d", kMaxSub); return ORF_EINVAL; }
    c->tuning = *t;
    return ORF_OK;
}

int32_t orf_ctx_set_timing(orf_ctx* c, int32_t on) {
    if (!c) return ORF_EINVAL;
    c->timing = on != 0;
    return ORF_OK;
}

int32_t orf_ctx_set_wait_injection(orf_ctx* c, int32_t stall_plane, int64_t wait_ns) {
    if (!c) return ORF_EINVAL;
    if (wait_ns < 0) { set_error("wait_ns must be >= 0"); return ORF_EINVAL; }
    c->stall_plane = stall_plane < 0 ? -1 : stall_plane;
    c->wait_ns = (unsigned long long)wait_ns;
    return ORF_OK;
}

int32_t orf_ctx_get_stats(orf_ctx* c, orf_kernel_stats* st) {
    if (!c || !st) return ORF_EINVAL;
    *st = c->stats;
    return ORF_OK;
}

int32_t orf_ctx_reset_stats(orf_ctx* c) {
    if (!c) return ORF_EINVAL;
    c->stats = orf_kernel_stats{};
    return ORF_OK;
}

int32_t orf_out2d_sizes(const orf_sim2d* s, int64_t* n_flux, int64_t* n_flux_z, int64_t* n_P, int64_t* n_PZ) {
    if (!s) return ORF_EINVAL;
    if (n_flux) *n_flux = (int64_t)s->n_mon * s->n_lambda;
    if (n_flux_z) *n_flux_z = (int64_t)s->n_monz * s->n_lambda;
    if (n_P) *n_P = (int64_t)s->nz * s->n_lambda * s->n_mon;
    if (n_PZ) *n_PZ = (int64_t)s->nx * s->n_lambda * s->n_monz;
    return ORF_OK;
}

namespace {
// scanned: the caller validated the sim with its permittivity scan already
int run2d_ctx(orf_ctx* ctx, const orf_sim2d* sim, orf_out2d* out, orf_progress_fn progress, void* user,
              bool scanned) {
    if (!ctx || !sim || !out) { set_error("NULL argument"); return ORF_EINVAL; }
    ORF_ON_DEVICE(ctx->device);
    // host phases into the context's counters: set-up (tables, device
    // block, uploads), the time loop, results and release
    const double t0 = now_s();
    orf_job* job = nullptr;
    ORF_TRY(make_job2d(ctx, sim, &job, !scanned));
    std::unique_ptr<orf_job> guard(job);
    const double t1 = now_s();
    ORF_TRY(job->advance(job->step_budget(), progress, user));
    const double t2 = now_s();
    ORF_TRY(job->finish2d(out));
    guard.reset();
    const double t3 = now_s();
    ctx->stats.setup_ms += 1e3 * (t1 - t0);
    ctx->stats.loop_ms += 1e3 * (t2 - t1);
    ctx->stats.finish_ms += 1e3 * (t3 - t2);
    out->wall_time = t3 - t0;
    return ORF_OK;
}
}  // namespace

int32_t orf_fdtd2d_run_ctx(orf_ctx* ctx, const orf_sim2d* sim, orf_out2d* out, orf_progress_fn progress,
                           void* user) {
    return run2d_ctx(ctx, sim, out, progress, user, false);
}

int32_t orf_fdtd2d_run(const orf_sim2d* sim, orf_out2d* out, orf_progress_fn progress, void* user) {
    if (!out) { set_error("out is NULL"); return ORF_EINVAL; }
    ORF_TRY(validate2d(sim));   // before any device work; the job does not scan again
    int st = ORF_OK;
    orf_ctx* c = default_ctx(&st);
    if (!c) return st;
    return run2d_ctx(c, sim, out, progress, user, true);
}

int32_t orf_job2d_create(orf_ctx* ctx, const orf_sim2d* sim, orf_job** job) {
    if (!ctx || !job) return ORF_EINVAL;
    ORF_ON_DEVICE(ctx->device);
    const int st = make_job2d(ctx, sim, job);
    if (st == ORF_OK) ctx_retain(ctx);
    return st;
}

int32_t orf_job3d_create(orf_ctx* ctx, const orf_sim3d* sim, orf_job** job) {
    if (!ctx || !job) return ORF_EINVAL;
    ORF_ON_DEVICE(ctx->device);
    const int st = make_job3d(ctx, sim, job);
    if (st == ORF_OK) ctx_retain(ctx);
    return st;
}

int32_t orf_job3d_create_slab(orf_ctx* ctx, const orf_sim3d* slab, int32_t z_offset, int32_t nz_global,
                              orf_job** job) {
    if (!ctx || !job || !slab) return ORF_EINVAL;
    ORF_ON_DEVICE(ctx->device);
    const int st = make_job3d_slab(ctx, slab, z_offset, nz_global, job);
    if (st == ORF_OK) ctx_retain(ctx);
    return st;
}

int32_t orf_job3d_step(orf_job* job, int64_t nsteps) {
    if (!job) return ORF_EINVAL;
    if (job->dims != 3) {
        set_error("orf_job3d_step takes a 3D job");
        return ORF_EINVAL;
    }
    ORF_ON_DEVICE(job->ctx->device);
    return job->step_async(nsteps);
}

int32_t orf_job3d_plane(orf_job* job, int32_t buffer, int32_t field, int32_t k, void** dev, size_t* bytes) {
    if (!job || job->dims != 3) return ORF_EINVAL;
    return job->plane_ptr(buffer, field, k, dev, bytes);
}

int32_t orf_job_advance(orf_job* job, int64_t nsteps) {
    if (!job || nsteps < 0) return ORF_EINVAL;
    ORF_ON_DEVICE(job->ctx->device);
    return job->advance(nsteps, nullptr, nullptr);
}

int32_t orf_job_sync(orf_job* job) {
    if (!job) return ORF_EINVAL;
    ORF_ON_DEVICE(job->ctx->device);
    ORF_CUDA(cudaStreamSynchronize(job->ctx->stream));
    return ORF_OK;
}

int32_t orf_job_reset(orf_job* job) {
    if (!job) return ORF_EINVAL;
    ORF_ON_DEVICE(job->ctx->device);
    return job->reset();
}
int64_t orf_job_steps_done(orf_job* job) { return job ? job->steps_done() : -1; }
int64_t orf_job_cells(orf_job* job) { return job ? job->cells() : -1; }
int32_t orf_job2d_finish(orf_job* job, orf_out2d* out) {
    if (!job || !out) return ORF_EINVAL;
    ORF_ON_DEVICE(job->ctx->device);
    return job->finish2d(out);
}
int32_t orf_job3d_finish(orf_job* job, orf_out3d* out) {
    if (!job || !out) return ORF_EINVAL;
    ORF_ON_DEVICE(job->ctx->device);
    return job->finish3d(out);
}
int32_t orf_job_get_fields(orf_job* job, double* const* f, int32_t nf) {
    if (!job || !f) return ORF_EINVAL;
    ORF_ON_DEVICE(job->ctx->device);
    return job->get_fields(f, nf);
}
int32_t orf_job_destroy(orf_job* job) {
    if (!job) return ORF_OK;
    orf_ctx* c = job->ctx;
    {
        ORF_ON_DEVICE(c->device);
        delete job;
        ctx_release(c);
    }
    return ORF_OK;
}

int32_t orf_out3d_sizes(const orf_sim3d* s, int32_t* na, int32_t* nb) {
    if (!s) return ORF_EINVAL;
    const int n[3] = {s->nx, s->ny, s->nz};
    for (int m = 0; m < s->n_mon; ++m) {
        const int q = s->mon_axis[m];
        if (q < 0 || q > 2) { set_error("monitors(%d).axis must be 1..3", m + 1); return ORF_EINVAL; }
        if (na) na[m] = n[(q + 1) % 3];
        if (nb) nb[m] = n[(q + 2) % 3];
    }
    return ORF_OK;
}

namespace {
int run3d_ctx(orf_ctx* ctx, const orf_sim3d* sim, orf_out3d* out, orf_progress_fn progress, void* user,
              bool scanned) {
    if (!ctx || !sim || !out) { set_error("NULL argument"); return ORF_EINVAL; }
    ORF_ON_DEVICE(ctx->device);
    // host phases into the context's counters: set-up (tables, device
    // block, uploads), the time loop, results and release
    const double t0 = now_s();
    orf_job* job = nullptr;
    ORF_TRY(make_job3d(ctx, sim, &job, !scanned));
    std::unique_ptr<orf_job> guard(job);
    const double t1 = now_s();
    ORF_TRY(job->advance(job->step_budget(), progress, user));
    const double t2 = now_s();
    ORF_TRY(job->finish3d(out));
    guard.reset();
    const double t3 = now_s();
    ctx->stats.setup_ms += 1e3 * (t1 - t0);
    ctx->stats.loop_ms += 1e3 * (t2 - t1);
    ctx->stats.finish_ms += 1e3 * (t3 - t2);
    out->wall_time = t3 - t0;
    return ORF_OK;
}
}  // namespace

int32_t orf_fdtd3d_run_ctx(orf_ctx* ctx, const orf_sim3d* sim, orf_out3d* out, orf_progress_fn progress,
                           void* user) {
    return run3d_ctx(ctx, sim, out, progress, user, false);
}

int32_t orf_fdtd3d_run(const orf_sim3d* sim, orf_out3d* out, orf_progress_fn progress, void* user) {
    if (!out) { set_error("out is NULL"); return ORF_EINVAL; }
    ORF_TRY(validate3d(sim));   // before any device work; the job does not scan again
    int st = ORF_OK;
    orf_ctx* c = default_ctx(&st);
    if (!c) return st;
    return run3d_ctx(c, sim, out, progress, user, true);
}

int32_t orf_plan2d(const orf_sim2d* sim, const orf_tuning* tuning, orf_tile2d* tiles, int32_t cap,
                   int32_t* n_interior, int32_t* n_frame, int32_t* tsteps, int32_t* variant) {
    ORF_TRY(validate2d(sim));
    orf_tuning tu{};
    if (tuning) tu = *tuning;
    if (tu.tsteps < 0 || tu.tsteps > kMaxSub) { set_error("tsteps must be 0..%d", kMaxSub); return ORF_EINVAL; }
    Plan2D p;
    ORF_TRY(plan2d(sim, tu, &p));
    if (n_interior) *n_interior = p.nfast;
    if (n_frame) *n_frame = p.nframe;
    if (tsteps) *tsteps = p.T;
    if (variant) *variant = p.fvariant;
    const int n = p.nfast + p.nframe;
    if (!tiles) return ORF_OK;
    if (cap < n) {
        set_error("orf_plan2d: %d tiles, room for %d", n, cap);
        return cap > 0 ? ORF_ETOOLARGE : ORF_OK;
    }
    for (int q = 0; q < n; ++q) {
        const FastTile2D& t = p.tiles[q];
        const bool fr = q >= p.nfast;
        tiles[q] = orf_tile2d{fr ? 1 : 0, t.li0, t.lk0, fr ? p.lx_pml : p.lx_int,
                              fr ? p.lz_pml : 0, t.oi0, t.ok0, t.ow, t.oh, t.flags};
        if (!fr) {
            Variant2D v;
            fast2d_info(p.fvariant, sim->precision == ORF_DOUBLE, false, &v);
            tiles[q].lz = v.lz();
        }
    }
    return ORF_OK;
}

int32_t orf_plan3d(const orf_sim3d* sim, orf_tile3d* tiles, int32_t cap, int32_t* n_interior, int32_t* n_cpml) {
    ORF_TRY(validate3d(sim));
    std::vector<Tile3D> ti, tp;
    plan3d(sim, ti, tp);
    if (n_interior) *n_interior = (int32_t)ti.size();
    if (n_cpml) *n_cpml = (int32_t)tp.size();
    const size_t n = ti.size() + tp.size();
    if (!tiles) return ORF_OK;
    if ((size_t)cap < n) {
        set_error("orf_plan3d: %zu tiles, room for %d", n, cap);
        return cap > 0 ? ORF_ETOOLARGE : ORF_OK;
    }
    const bool px = sim->periodic[0] != 0, py = sim->periodic[1] != 0;
    for (size_t q = 0; q < n; ++q) {
        const bool pml = q >= ti.size();
        const Tile3D& t = pml ? tp[q - ti.size()] : ti[q];
        // the kernel's choice (step3d_fused.cu): TMA unless the halo wraps
        const bool wrapx = px && (t.i0 == 0 || t.i0 + kTile3X >= sim->nx);
        const bool wrapy = py && (t.j0 == 0 || t.j0 + kTile3Y >= sim->ny);
        tiles[q] = orf_tile3d{pml ? 1 : 0, t.i0, t.j0, t.tw, t.th, t.k0, t.k1, (wrapx || wrapy) ? 0 : 1,
                              t.i0 - 4, t.i0};
    }
    return ORF_OK;
}

int32_t orf_check_violations(uint64_t* count, int32_t reset) {
    if (!count) return ORF_EINVAL;
    *count = 0;
#ifdef ORF_CHECK
    unsigned long long a = 0, b = 0;
    const int s1 = fast2d_violations_f32(&a, reset), s2 = fast2d_violations_f64(&b, reset);
    if (s1 != ORF_OK || s2 != ORF_OK) {
        set_error("reading the checked build's violation counters failed");
        return ORF_ECUDA;
    }
    *count = a + b;
    return ORF_OK;
#else
    (void)reset;
    set_error("this library is the normal build; the checked one is lib/liborf_fdtd_check.so");
    return ORF_EINVAL;
#endif
}

int32_t orf_batch2d_run(orf_ctx* ctx, int32_t n, const orf_sim2d* sims, orf_out2d* outs, orf_progress_fn progress,
                        void* user) {
    if (!ctx || n < 0 || (n > 0 && (!sims || !outs))) { set_error("NULL argument"); return ORF_EINVAL; }
    ORF_ON_DEVICE(ctx->device);
    return batch2d_run(ctx, n, sims, outs, progress, user);
}

}  // extern "C"
