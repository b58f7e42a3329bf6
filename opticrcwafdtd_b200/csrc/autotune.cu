// autotune.cu -- orf_autotune2d: pick the 2D kernel variant and fused step
// depth for one problem shape by timing them on the device.
//
// The reference has no tuning knobs (its time loop is fixed MATLAB code).
// Here the interior tile geometry (variant) and the number of time steps
// fused per launch (T) trade halo recomputation against launches and
// register pressure, and the best pair depends on the grid shape, the
// polarisation and the precision.  Every candidate performs the same
// arithmetic cell by cell, so the choice changes speed only, never results.
#include <algorithm>
#include <cstring>

#include "job2d.cuh"

namespace orf {
namespace {

int time_candidate(orf_ctx* ctx, const orf_sim2d* sim, int steps, double* ms) {
    orf_job* j = nullptr;
    ORF_TRY(make_job2d(ctx, sim, &j));
    std::unique_ptr<orf_job> job(j);
    ORF_TRY(job->advance(kChunk, nullptr, nullptr));   // warm: graph capture, first-touch
    cudaEvent_t a = nullptr, b = nullptr;
    ORF_CUDA(cudaEventCreate(&a));
    ORF_CUDA(cudaEventCreate(&b));
    cudaEventRecord(a, ctx->stream);
    const int st = job->advance(steps, nullptr, nullptr);
    cudaEventRecord(b, ctx->stream);
    const cudaError_t e = cudaEventSynchronize(b);
    float t = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    ORF_TRY(st);
    ORF_CUDA(e);
    *ms = t;
    return ORF_OK;
}

// a batch candidate: the time loop of the batched call (its set-up and
// results are the same for every candidate), outputs discarded; the faster
// of two calls, so that one disturbed call does not decide the pick
int time_batch(orf_ctx* ctx, int n, const orf_sim2d* sims, double* ms) {
    std::vector<orf_out2d> outs(n);
    *ms = 1e300;
    for (int rep = 0; rep < 2; ++rep) {
        std::memset(outs.data(), 0, sizeof(orf_out2d) * n);
        const double l0 = ctx->stats.loop_ms;
        ORF_TRY(batch2d_run(ctx, n, sims, outs.data(), nullptr, nullptr));
        *ms = std::min(*ms, ctx->stats.loop_ms - l0);
    }
    return ORF_OK;
}

}  // namespace
}  // namespace orf

using namespace orf;

extern "C" int32_t orf_autotune2d(orf_ctx* ctx, int32_t n, const orf_sim2d* sims, int32_t steps, orf_tuning* best) {
    if (!ctx || !sims || n < 1) {
        set_error("ctx and at least one sim are required");
        return ORF_EINVAL;
    }
    for (int q = 0; q < n; ++q) ORF_TRY(validate2d(&sims[q]));
    ORF_ON_DEVICE(ctx->device);
    if (steps <= 0) steps = 4 * kChunk;
    // time a bounded piece of each run: no candidate may stop early on the
    // shutoff or the step budget
    std::vector<orf_sim2d> s(sims, sims + n);
    for (auto& q : s) {
        q.shutoff = 0.0;
        q.max_time = (double)(steps + (n == 1 ? 3 * kChunk : 0)) * q.courant * q.dx;
    }
    const orf_tuning saved = ctx->tuning;
    const bool timing = ctx->timing;
    ctx->timing = false;
    orf_tuning pick = saved;
    double best_ms = 1e300;
    static const int kDepths[] = {4, 6, 8, 10};
    int rc = ORF_OK;
    for (int v = 1; v <= variant2d_count() && rc == ORF_OK; ++v)
        for (int T : kDepths) {
            ctx->tuning.tsteps = T;
            ctx->tuning.variant = v;
            ctx->tuning.use_graph = 1;
            double ms = 0;
            rc = n == 1 ? time_candidate(ctx, s.data(), steps, &ms) : time_batch(ctx, n, s.data(), &ms);
            if (rc != ORF_OK) break;
            if (ms < best_ms) {
                best_ms = ms;
                pick = ctx->tuning;
            }
        }
    ctx->timing = timing;
    if (rc != ORF_OK) {
        ctx->tuning = saved;
        return rc;
    }
    ctx->tuning = pick;
    if (best) *best = pick;
    return ORF_OK;
}
