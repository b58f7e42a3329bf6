// batch.cu -- many independent 2D runs advanced together (orf_batch2d_run).
//
// The reference runs its sweeps (examples/cpo_box_scan.m:23-31,
// optimizeGratingCoupler.m:1-12, the app's period sweep) as sequential
// orf.fdtd2D calls.  Here every instance is set up as a device-resident job,
// and instances of one kernel configuration form a group (group.cuh): their
// tile descriptors (self-contained, FastTile2D), DFT streams and state
// pointers are concatenated, so one persistent interior launch and one frame
// launch advance all of them per fused step block, one flush and one check
// launch close each chunk, and the chunk sequence is captured as a CUDA
// graph.  Instances of uneven size and step budget coexist: a finished
// instance's tiles turn into no-ops.  Instances of both polarisations, or
// with more than 256 distinct permittivities, fall into further groups.
#include <algorithm>
#include <string>
#include <thread>

#include "group.cuh"

namespace orf {
namespace {

template <class R>
int run_batch(orf_ctx* ctx, int n, const orf_sim2d* sims, orf_out2d* outs, orf_progress_fn progress, void* user) {
    double t0 = now_s();
    // instance set-up (host tables, tile plans, device blocks, uploads) on
    // several host threads: create() is safe to run concurrently (its errors
    // are per thread, the block cache and the byte counter take locks)
    std::vector<std::unique_ptr<Job2D<R>>> jobs(n);
    std::vector<int> status(n, ORF_OK);
    std::vector<std::string> why(n);
    const int nthreads = (int)std::max(1u, std::min<unsigned>({16u, std::thread::hardware_concurrency(), (unsigned)n}));
    auto work = [&](int tid) {
        for (int q = tid; q < n; q += nthreads) {
            auto j = std::make_unique<Job2D<R>>();
            j->ctx = ctx;
            status[q] = j->create(&sims[q]);
            if (status[q] != ORF_OK) {
                why[q] = last_error();
                continue;
            }
            jobs[q] = std::move(j);
        }
    };
    if (nthreads == 1) {
        work(0);
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < nthreads; ++t) pool.emplace_back(work, t);
        for (auto& t : pool) t.join();
    }
    for (int q = 0; q < n; ++q)
        if (status[q] != ORF_OK) {
            set_error("instance %d: %s", q + 1, why[q].c_str());
            return status[q];
        }
    // instances sharing a kernel configuration (precision, index width,
    // fused step count, interior variant) form one group: one launch per
    // kernel advances all of its members
    std::vector<std::unique_ptr<Group2D<R>>> groups;
    int64_t nmax = 0;
    for (auto& j : jobs) {
        Group2D<R>* g = nullptr;
        for (auto& c : groups)
            if (Group2D<R>::compatible(c->jobs[0], j.get())) g = c.get();
        if (!g) {
            groups.push_back(std::make_unique<Group2D<R>>());
            g = groups.back().get();
            g->ctx = ctx;
        }
        g->add(j.get());
        nmax = std::max<int64_t>(nmax, j->nmax);
    }
    cudaStream_t st = ctx->stream;
    for (auto& g : groups) ORF_TRY(g->build(st));
    double t1 = now_s();
    ctx->stats.setup_ms += 1e3 * (t1 - t0);

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
            for (auto& g : groups) ORF_TRY(g->enqueue(nb, st));
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
    for (auto& g : groups) g->eng.collect_timing();
    if (rc != ORF_OK) return rc;
    t0 = now_s();
    ctx->stats.loop_ms += 1e3 * (t0 - t1);
    for (int q = 0; q < n; ++q) ctx->stats.cell_updates += jobs[q]->pl.last_step * jobs[q]->cells();
    // results of the instances on host threads, each with a stream of its own
    // (the loop has ended: the instances' sums are final and independent)
    auto fin = [&](int tid) {
        cudaSetDevice(ctx->device);
        cudaStream_t fs = nullptr;
        if (cudaStreamCreateWithFlags(&fs, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            for (int q = tid; q < n; q += nthreads) {
                status[q] = ORF_ECUDA;
                why[q] = "cannot create a stream for the results";
            }
            return;
        }
        for (int q = tid; q < n; q += nthreads) {
            status[q] = jobs[q]->finish2d_on(&outs[q], fs);
            if (status[q] != ORF_OK) why[q] = last_error();
        }
        cudaStreamDestroy(fs);
    };
    if (nthreads == 1) {
        fin(0);
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < nthreads; ++t) pool.emplace_back(fin, t);
        for (auto& t : pool) t.join();
    }
    for (int q = 0; q < n; ++q)
        if (status[q] != ORF_OK) {
            set_error("instance %d: %s", q + 1, why[q].c_str());
            return status[q];
        }
    groups.clear();
    jobs.clear();
    ctx->stats.finish_ms += 1e3 * (now_s() - t0);
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
        if (sims[q].precision != sims[0].precision) {
            set_error("all instances of a batch share the precision (instance %d differs)", q + 1);
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
