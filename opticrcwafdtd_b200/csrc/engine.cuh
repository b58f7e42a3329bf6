// engine.cuh -- the chunked time loop shared by 2D, 3D and batched runs.
//
// One chunk = kChunk time steps = ceil(kChunk / T) step-kernel launches
// (each fusing up to T steps), one DFT flush launch and one check launch.
// All per-step state (step counter, done flag, energy) lives in device
// memory, so a captured chunk sequence replays unchanged: the time loop runs
// as CUDA graph launches of G chunks, and the host only polls the status ring
// the check kernel writes into mapped pinned memory (no per-chunk sync).
#pragma once
#include <functional>

#include "runtime.cuh"

namespace orf {

// CUDA events around individual launches (orf_ctx_set_timing).
struct KernelTimer {
    struct Rec {
        int kind;                 // 0 interior, 1 frame, 2 flush/check
        int64_t cells;            // cell updates of the launch
        cudaEvent_t a, b;
    };
    std::vector<cudaEvent_t> pool;
    std::vector<Rec> recs;
    size_t used = 0;
    ~KernelTimer();
    int begin(cudaStream_t s, cudaEvent_t* a);
    int end(cudaStream_t s, int kind, int64_t cells, cudaEvent_t a);
    void collect(orf_kernel_stats* st);
};

struct ChunkEngine {
    orf_ctx* ctx = nullptr;
    bool fp64 = false;
    int T = 1;                        // time steps fused per step launch
    int par = 0;                      // field buffer holding the current state
    // launches the step kernels of all instances for steps [off, off+nsub) of
    // the chunk, reading buffer par; want_energy on the chunk's last launch
    // timer (may be null) records per-kernel events in timing mode
    std::function<cudaError_t(int off, int nsub, int par, int want_energy, cudaStream_t, KernelTimer* timer)> step;
    DftStream* d_streams = nullptr;
    FlushItem* d_items = nullptr;
    int nitems = 0;
    JobState** d_states = nullptr;
    int nstates = 0;

    // graph cache
    cudaGraphExec_t gexec = nullptr;
    int gchunks = 0;
    int gpar = -1;

    KernelTimer timer;

    ~ChunkEngine();
    int launches_per_chunk() const { return (kChunk + T - 1) / T; }
    int enqueue_chunk(cudaStream_t s, bool timed);
    // enqueue n chunks (graph replays where possible)
    int enqueue(int nchunks, cudaStream_t s);
    void drop_graph();
    // fold the recorded events into ctx->stats (after a sync)
    void collect_timing();
};

// A second stream for running a job's CPML-frame launch next to its
// interior launch: both read buffer par and write disjoint cells of par^1,
// so they may overlap (small grids fill only part of the GPU with either).
// fork() records the fork on s, returns the side stream waiting on it;
// join() makes s wait for the side stream.  Captured as parallel graph
// branches when s is being captured.
struct SideStream {
    cudaStream_t s2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool ok() const { return s2 != nullptr; }
    int init() {
        if (s2) return ORF_OK;
        ORF_CUDA(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
        ORF_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        ORF_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        return ORF_OK;
    }
    cudaError_t fork(cudaStream_t s) {
        cudaError_t e = cudaEventRecord(ev_fork, s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s2, ev_fork, 0);
        return e;
    }
    cudaError_t join(cudaStream_t s) {
        cudaError_t e = cudaEventRecord(ev_join, s2);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ev_join, 0);
        return e;
    }
    ~SideStream() {
        if (s2) {
            cudaStreamSynchronize(s2);
            cudaStreamDestroy(s2);
        }
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
    }
};

// Host-side progress loop over one job's status ring.
struct ProgressLoop {
    const ChunkStatus* ring = nullptr;   // mapped host ring of the job
    volatile int* cancel = nullptr;      // mapped host cancel flag read by the check kernel
    long long seen = 0;                  // ring entries consumed
    double S = 0, src_end = 0, shutoff = 0;
    bool done = false;
    bool cancelled = false;
    long long last_step = 0;
    // consume finished entries; returns ORF_ECANCELLED if the callback asks
    int poll(orf_progress_fn progress, void* user);
};

// Enqueue `chunks` chunks of one engine in batches, at most kInFlight
// batches ahead of the GPU, reading the status ring after each batch: the
// progress callback fires every chunk and enqueueing stops as soon as the
// device reports the run done (shutoff) or the callback cancels.
int run_chunks(ChunkEngine& eng, ProgressLoop& pl, orf_ctx* ctx, int64_t chunks, orf_progress_fn progress,
               void* user);

}  // namespace orf
