// batch.cu -- many independent 2D runs advanced together (orf_batch2d_run).
//
// The reference runs its sweeps (examples/cpo_box_scan.m:23-31,
// optimizeGratingCoupler.m:1-12, the app's period sweep) as sequential
// orf.fdtd2D calls.  Here every instance is set up as a device-resident job,
// and their tile descriptors (self-contained, FastTile2D), DFT streams and
// state pointers are concatenated: one persistent interior launch and one
// frame launch advance all instances per fused step block, one flush and one
// check launch close each chunk, and the chunk sequence is captured as a
// CUDA graph.  Instances of uneven size and step budget coexist: a finished
// instance's tiles turn into no-ops.
#include <algorithm>

#include "job2d.cuh"

namespace orf {
namespace {

template <class R>
int run_batch(orf_ctx* ctx, int n, const orf_sim2d* sims, orf_out2d* outs, orf_progress_fn progress, void* user) {
    std::vector<std::unique_ptr<Job2D<R>>> jobs;
    jobs.reserve(n);
    for (int q = 0; q < n; ++q) {
        auto j = std::make_unique<Job2D<R>>();
        j->ctx = ctx;
        const int st = j->create(&sims[q]);
        if (st != ORF_OK) {
            char buf[600];
            std::snprintf(buf, sizeof buf, "instance %d: %s", q + 1, last_error());
            set_error("%s", buf);
            return st;
        }
        jobs.push_back(std::move(j));
    }
    // all instances share the kernel variant and the fused step count T
    const int T = jobs[0]->T, fv = jobs[0]->fvariant;
    const bool te = jobs[0]->te;
    bool idx16 = false;
    for (auto& j : jobs) {
        if (j->T != T || j->fvariant != fv) {
            set_error("batch instances picked different tilings");
            return ORF_EINVAL;
        }
        idx16 = idx16 || j->idx16;
    }
    if (idx16) {
        for (auto& j : jobs)
            if (!j->idx16) {
                set_error("mixing instances with <= 256 and > 256 distinct permittivities is not supported");
                return ORF_EINVAL;
            }
    }
    std::vector<FastTile2D> inner, frame;
    std::vector<DftStream> streams;
    std::vector<FlushItem> items;
    std::vector<JobState*> states;
    int64_t interior_cells = 0, cells = 0, nmax = 0;
    for (auto& j : jobs) {
        inner.insert(inner.end(), j->ftiles_host.begin(), j->ftiles_host.begin() + j->nfast);
        frame.insert(frame.end(), j->ftiles_host.begin() + j->nfast, j->ftiles_host.end());
        for (int q = 0; q < j->nfast; ++q) interior_cells += (int64_t)j->ftiles_host[q].ow * j->ftiles_host[q].oh;
        cells += j->cells();
        const int s0 = (int)streams.size();
        streams.insert(streams.end(), j->host_streams.begin(), j->host_streams.end());
        for (int q = 0; q < j->nstreams; ++q)
            for (int e0 = 0; e0 < j->host_streams[q].len; e0 += 128)
                for (int l0 = 0; l0 < j->nL; l0 += 8) items.push_back({s0 + q, e0, l0, 0});
        states.push_back(j->d_st);
        nmax = std::max<int64_t>(nmax, j->nmax);
    }
    Arena ar;
    FastTile2D *d_inner = nullptr, *d_frame = nullptr;
    DftStream* d_streams = nullptr;
    FlushItem* d_items = nullptr;
    JobState** d_states = nullptr;
    ar.add(&d_inner, inner.size() + 1);
    ar.add(&d_frame, frame.size() + 1);
    ar.add(&d_streams, streams.size() + 1);
    ar.add(&d_items, items.size() + 1);
    ar.add(&d_states, states.size() + 1);
    ORF_TRY(ar.alloc());
    struct Guard {
        Arena* a;
        ~Guard() { a->release(); }
    } guard{&ar};
    cudaStream_t st = ctx->stream;
    auto up = [&](void* d, const void* h, size_t b) -> int {
        if (!b) return ORF_OK;
        ORF_CUDA(cudaMemcpyAsync(d, h, b, cudaMemcpyHostToDevice, st));
        ctx->stats.h2d_bytes += (int64_t)b;
        return ORF_OK;
    };
    ORF_TRY(up(d_inner, inner.data(), inner.size() * sizeof(FastTile2D)));
    ORF_TRY(up(d_frame, frame.data(), frame.size() * sizeof(FastTile2D)));
    ORF_TRY(up(d_streams, streams.data(), streams.size() * sizeof(DftStream)));
    ORF_TRY(up(d_items, items.data(), items.size() * sizeof(FlushItem)));
    ORF_TRY(up(d_states, states.data(), states.size() * sizeof(JobState*)));
    ORF_CUDA(cudaStreamSynchronize(st));

    const bool f64 = sizeof(R) == 8;
    const int bps_f = fast2d_blocks_per_sm(f64, te, idx16, false, fv);
    const int bps_p = fast2d_blocks_per_sm(f64, te, idx16, true, 0);
    const int grid_f = (int)std::min<size_t>(inner.size(), (size_t)ctx->sm_count * std::max(1, bps_f));
    const int grid_p = (int)std::min<size_t>(frame.size(), (size_t)ctx->sm_count * std::max(1, bps_p));
    const int ni = (int)inner.size(), nf = (int)frame.size();
    ChunkEngine eng;
    eng.ctx = ctx;
    eng.fp64 = f64;
    eng.T = T;
    eng.par = 0;
    eng.d_streams = d_streams;
    eng.d_items = d_items;
    eng.nitems = (int)items.size();
    eng.d_states = d_states;
    eng.nstates = n;
    eng.step = [&](int off, int nsub, int par, int we, cudaStream_t s, KernelTimer* tm) -> cudaError_t {
        cudaError_t e = cudaSuccess;
        cudaEvent_t a = nullptr;
        if (ni) {
            if (tm && tm->begin(s, &a) != ORF_OK) return cudaErrorUnknown;
            e = launch_fast2d(f64, te, idx16, false, fv, d_inner, ni, off, nsub, par, we, grid_f, s);
            if (e != cudaSuccess) return e;
            if (tm && tm->end(s, 0, interior_cells * nsub, a) != ORF_OK) return cudaErrorUnknown;
        }
        if (nf) {
            if (tm && tm->begin(s, &a) != ORF_OK) return cudaErrorUnknown;
            e = launch_fast2d(f64, te, idx16, true, 0, d_frame, nf, off, nsub, par, we, grid_p, s);
            if (e != cudaSuccess) return e;
            if (tm && tm->end(s, 1, (cells - interior_cells) * nsub, a) != ORF_OK) return cudaErrorUnknown;
        }
        return e;
    };

    // time loop: graph replays in batches; every instance's status ring is
    // read after each batch (progress = mean fraction, stop when all are done)
    const int64_t chunks = (nmax + kChunk - 1) / kChunk;
    constexpr int kBatch = 8, kInFlight = 4;
    std::vector<cudaEvent_t> evs;
    int64_t enq = 0;
    size_t head = 0;
    int rc = ORF_OK;
    auto all_done = [&]() {
        for (auto& j : jobs)
            if (!j->pl.done) return false;
        return true;
    };
    auto poll = [&]() -> int {
        double frac = 0.0;
        bool fresh = false;
        for (auto& j : jobs) {
            const long long before = j->pl.seen;
            j->pl.poll(nullptr, nullptr);
            fresh = fresh || j->pl.seen != before;
            const double t = j->pl.last_step * j->S;
            frac += j->pl.done ? 1.0 : progress_fraction(t, j->src_end, 1.0, j->shutoff);
        }
        if (progress && fresh) {
            char msg[96];
            std::snprintf(msg, sizeof msg, "batch of %d runs", n);
            if (progress(frac / n, msg, user)) {
                for (auto& j : jobs) *j->cancel_h = 1;
                return ORF_ECANCELLED;
            }
        }
        return ORF_OK;
    };
    while (!all_done()) {
        while (enq < chunks && evs.size() - head < (size_t)kInFlight) {
            const int nb = (int)std::min<int64_t>(kBatch, chunks - enq);
            ORF_TRY(eng.enqueue(nb, st));
            enq += nb;
            cudaEvent_t e;
            ORF_CUDA(cudaEventCreateWithFlags(&e, cudaEventBlockingSync | cudaEventDisableTiming));
            ORF_CUDA(cudaEventRecord(e, st));
            evs.push_back(e);
        }
        if (head < evs.size()) {
            ORF_CUDA(cudaEventSynchronize(evs[head]));
            ++head;
        }
        rc = poll();
        if (rc != ORF_OK) break;
        if (head == evs.size() && enq >= chunks) break;
    }
    cudaError_t se = cudaStreamSynchronize(st);
    for (auto e : evs) cudaEventDestroy(e);
    ORF_CUDA(se);
    eng.collect_timing();
    if (rc != ORF_OK) return rc;
    for (int q = 0; q < n; ++q) {
        ctx->stats.cell_updates += jobs[q]->pl.last_step * jobs[q]->cells();
        ORF_TRY(jobs[q]->finish2d(&outs[q]));
    }
    return ORF_OK;
}

}  // namespace

int batch2d_run(orf_ctx* ctx, int n, const orf_sim2d* sims, orf_out2d* outs, orf_progress_fn progress, void* user) {
    if (n == 0) return ORF_OK;
    const double t0 = now_s();
    for (int q = 0; q < n; ++q) {
        const int st = validate2d(&sims[q]);
        if (st != ORF_OK) {
            char buf[600];
            std::snprintf(buf, sizeof buf, "instance %d: %s", q + 1, last_error());
            set_error("%s", buf);
            return st;
        }
        if (sims[q].pol != sims[0].pol || sims[q].precision != sims[0].precision) {
            set_error("all instances of a batch share pol and precision (instance %d differs)", q + 1);
            return ORF_EINVAL;
        }
    }
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != ctx->device) ORF_CUDA(cudaSetDevice(ctx->device));
    const int rc = sims[0].precision == ORF_SINGLE ? run_batch<float>(ctx, n, sims, outs, progress, user)
                                                   : run_batch<double>(ctx, n, sims, outs, progress, user);
    const double wall = now_s() - t0;
    if (rc == ORF_OK)
        for (int q = 0; q < n; ++q) outs[q].wall_time = wall;
    return rc;
}

}  // namespace orf
