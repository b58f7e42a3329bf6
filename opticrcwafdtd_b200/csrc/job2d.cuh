// job2d.cuh -- device-resident 2D run (orf.fdtd2D).
#pragma once
#include <algorithm>

#include "engine.cuh"

namespace orf {

// Host-only tile plan of a 2D run (job2d.cu, plan2d): tiles are
// [interior | frame] with loaded windows, output rectangles and flags.
struct Plan2D {
    int fvariant = 1, T = 1;
    int nfast = 0, nframe = 0;
    int lx_int = 0, lx_pml = 0, lz_pml = 0;
    std::vector<FastTile2D> tiles;
};
int plan2d(const orf_sim2d* s, const orf_tuning& tuning, Plan2D* plan);

// Frame tiles in runs of one CPML specialisation (flags 8 / 16): the
// persistent frame launch then keeps the CTAs of an SM in the same code
// (mixed, they miss in the instruction cache); the order changes no value.
template <class It>
void sort_frame_tiles(It first, It last) {
    std::stable_sort(first, last, [](const FastTile2D& a, const FastTile2D& b) {
        return (a.flags & 24) > (b.flags & 24);
    });
}

template <class R>
struct Job2D : orf_job {
    // geometry / options
    bool te = true, per = false, idx16 = false;
    int nx = 0, nz = 0, nzA = 0, nxB = 0, pitch = 0;
    int nM = 0, nMZ = 0, nL = 0, nlut = 0;
    double dx = 0, Cc = 0, S = 0, src_end = 0, shutoff = 0;
    int64_t nmax = 0, nsrc = 0;
    int64_t enq_steps = 0;     // steps enqueued since the last reset
    // device
    Arena arena;
    Inst2D<R> h{};
    Inst2D<R>* d_inst = nullptr;
    JobState* d_st = nullptr;
    JobState** d_states = nullptr;
    // interior tiles (pipelined kernel without CPML) and frame tiles (CPML /
    // boundary instantiation), one descriptor array: [interior | frame]
    std::vector<FastTile2D> ftiles_host;
    int nfast = 0, nframe = 0;
    FastTile2D* d_ftiles = nullptr;
    int fvariant = 1, T = 1, grid_fast = 0, grid_frame = 0;
    DftStream* d_streams = nullptr;
    std::vector<DftStream> host_streams;
    FlushItem* d_items = nullptr;
    FluxPair* d_pairs = nullptr;
    int nstreams = 0, nitems = 0, npairs = 0;
    void* d_acc = nullptr;
    double* d_omega = nullptr;
    double* d_flux = nullptr;
    double2* d_stage = nullptr;
    // mapped host memory
    ChunkStatus* ring_h = nullptr;
    ChunkStatus* ring_d = nullptr;
    volatile int* cancel_h = nullptr;
    int* cancel_d = nullptr;
    ChunkEngine eng;
    ProgressLoop pl;
    SideStream side;   // CPML frame launches next to the interior ones
    // no-allocation mode: device state carved from ext_base (see noalloc.cu),
    // no mapped status ring, no graphs, no events
    void* ext_base = nullptr;
    size_t ext_cap = 0;

    Job2D() { dims = 2; }
    ~Job2D() override;
    int create(const orf_sim2d* s);
    int pick_tiling(const orf_sim2d* s);
    int init_state();
    int advance(int64_t nsteps, orf_progress_fn progress, void* user) override;
    int64_t steps_done() override;
    int64_t cells() const override { return (int64_t)nx * nz; }
    int64_t step_budget() const override { return nmax; }
    int reset() override;
    int get_fields(double* const* f, int nf) override;
    int finish2d(orf_out2d* o) override;
    int finish2d_on(orf_out2d* o, cudaStream_t st);
    // enqueue every remaining chunk with direct launches, then synchronize
    int advance_all_direct();
    void state_regions(int b, std::vector<std::pair<void*, size_t>>& out) override;
    uint64_t state_key() const override;
    JobState* state_dev() const override { return d_st; }
    int64_t nmax_steps() const override { return nmax; }
    void resume_host(const JobState& js) override;
};

}  // namespace orf
