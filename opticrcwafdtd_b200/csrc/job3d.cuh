// job3d.cuh -- device-resident 3D run (orf.fdtd3D).
#pragma once
#include <cuda.h>

#include "engine.cuh"

namespace orf {

// Host-only tile plan of a 3D run (job3d.cu): interior tiles and CPML tiles.
// zlo / zhi: the low / high z end has its CPML layer (false: the end of a z
// slab that borders another slab, whose planes run as interior tiles)
void plan3d(const orf_sim3d* s, std::vector<Tile3D>& tiles, std::vector<Tile3D>& tiles_pml, bool zlo = true,
            bool zhi = true);

template <class R>
struct Job3D : orf_job {
    int n[3] = {0, 0, 0};
    bool per[3] = {false, false, false};
    int pitch = 0, nM = 0, nL = 0, idxw = 1, zc = 4;
    double d = 0, Cc = 0, S = 0, src_end = 0, shutoff = 0;
    int64_t nmax = 0, nsrc = 0, enq_steps = 0;
    // z slab of a larger grid (orf_job3d_create_slab): global index of local
    // plane 0 and the global plane count (the z CPML profile is the global one)
    bool slab = false;
    int z_off = 0, nz_glob = 0;
    // step-by-step enqueueing (orf_job3d_step): steps enqueued and the
    // sample slot of the next step in its chunk
    int64_t sdone = 0;
    int soff = 0;
    Arena arena;
    Inst3D<R> h{};
    Inst3D<R>* d_inst = nullptr;
    JobState* d_st = nullptr;
    JobState** d_states = nullptr;
    std::vector<Tile3D> tiles, tiles_pml;   // interior / CPML tiles
    Tile3D* d_tiles = nullptr;
    Tile3D* d_tiles_pml = nullptr;
    DftStream* d_streams = nullptr;
    std::vector<DftStream> host_streams;
    FlushItem* d_items = nullptr;
    FluxPair* d_pairs = nullptr;
    int nstreams = 0, nitems = 0, npairs = 0;
    void* d_acc = nullptr;
    double* d_omega = nullptr;
    double* d_flux = nullptr;
    double2* d_stage = nullptr;
    size_t stage_elems = 0;
    std::vector<std::pair<int, int>> planes;   // (Na, Nb) per monitor
    ChunkStatus* ring_h = nullptr;
    ChunkStatus* ring_d = nullptr;
    volatile int* cancel_h = nullptr;
    int* cancel_d = nullptr;
    ChunkEngine eng;
    ProgressLoop pl;
    SideStream side;   // CPML tiles next to the interior tiles

    Job3D() { dims = 3; }
    ~Job3D() override {
        if (arena.base) {
            cudaStreamSynchronize(ctx->stream);
            arena.release();
        }
        host_mapped_free(ring_h);
        host_mapped_free((void*)cancel_h);
    }
    size_t N() const { return (size_t)n[0] * n[1] * n[2]; }
    size_t NP() const { return (size_t)pitch * n[1] * n[2]; }
    int64_t cells() const override { return (int64_t)N(); }
    int64_t step_budget() const override { return nmax; }

    int create(const orf_sim3d* s);
    int step_async(int64_t nsteps) override;
    int plane_ptr(int buffer, int field, int k, void** dev, size_t* bytes) override;
    static constexpr int kTmaps3 = 23;   // E[2][3], H[2][3], index[3], z psi H[2][2], z psi E[2][2]
    // rows_pitch / nplanes: row length and plane count of the array (the
    // field pitch and nz unless given)
    int encode_tmap3(CUtensorMap* m, CUtensorMapDataType t, const void* base, size_t esz, int bx, int by,
                     int rows_pitch = 0, int nplanes = 0);
    int init_state();
    int advance(int64_t nsteps, orf_progress_fn progress, void* user) override;
    int64_t steps_done() override;
    int reset() override;
    int get_fields(double* const* f, int nf) override;
    int finish3d(orf_out3d* o) override;
    void state_regions(int b, std::vector<std::pair<void*, size_t>>& out) override;
    uint64_t state_key() const override;
    JobState* state_dev() const override { return d_st; }
    int64_t nmax_steps() const override { return nmax; }
    void resume_host(const JobState& js) override;
};


}  // namespace orf
