// group.cuh -- a set of resident jobs advanced by shared launches.
//
// The reference runs every sweep point as its own orf.fdtd2D / orf.fdtd3D
// call (examples/cpo_box_scan.m:23-31, optimizeGratingCoupler.m:1-12).  A
// group concatenates the self-contained work descriptors of several jobs of
// one kernel configuration -- 2D: FastTile2D tiles; 3D: Inst3D records plus
// Tile3D columns re-indexed into them -- together with their DFT streams,
// flush items and JobState pointers, so that one launch per kernel advances
// every member, one flush and one check launch close each chunk for all of
// them, and the chunk sequence replays as a CUDA graph.  Membership may
// change between chunks (serving): a new member starts from zeroed fields in
// both ping-pong buffers, so it can join at either buffer parity, and a
// finished member's tiles become no-ops until it is removed.  Every member's
// arithmetic is the same as when it runs alone.
#pragma once
#include "job2d.cuh"
#include "job3d.cuh"

namespace orf {

struct Group {
    orf_ctx* ctx = nullptr;
    bool dirty = true;            // membership changed since the last build
    virtual ~Group() { arena.release(); }
    virtual int build(cudaStream_t upload) = 0;   // rebuild device descriptor arrays
    virtual int size() const = 0;
    virtual void remove(orf_job* j) = 0;
    virtual int64_t cells() const = 0;
    // enqueue n chunks of every member on stream s (graph replays)
    int enqueue(int nchunks, cudaStream_t s) { return eng.enqueue(nchunks, s); }

    Arena arena;
    DftStream* d_streams = nullptr;
    FlushItem* d_items = nullptr;
    JobState** d_states = nullptr;
    std::vector<DftStream> streams;
    std::vector<FlushItem> items;
    std::vector<JobState*> states;
    ChunkEngine eng;

  protected:
    // append one member's DFT streams, flush items and state pointer
    void add_streams(const std::vector<DftStream>& hs, int nL, JobState* st) {
        const int s0 = (int)streams.size();
        streams.insert(streams.end(), hs.begin(), hs.end());
        for (int q = 0; q < (int)hs.size(); ++q)
            for (int e0 = 0; e0 < hs[q].len; e0 += 128)
                for (int l0 = 0; l0 < nL; l0 += 8) items.push_back({s0 + q, e0, l0, 0});
        states.push_back(st);
    }
    int upload(cudaStream_t st, void* d, const void* h, size_t b) {
        if (!b) return ORF_OK;
        ORF_CUDA(cudaMemcpyAsync(d, h, b, cudaMemcpyHostToDevice, st));
        ctx->stats.h2d_bytes += (int64_t)b;
        return ORF_OK;
    }
    void wire_engine(bool fp64, int T) {
        eng.ctx = ctx;
        eng.fp64 = fp64;
        eng.T = T;
        eng.d_streams = d_streams;
        eng.d_items = d_items;
        eng.nitems = (int)items.size();
        eng.d_states = d_states;
        eng.nstates = (int)states.size();
        eng.drop_graph();   // descriptor addresses changed; eng.par carries over
    }
};

// 2D members share precision, polarisation, index width, fused step count T
// and the interior kernel variant.
template <class R>
struct Group2D : Group {
    std::vector<Job2D<R>*> jobs;
    bool te = true, idx16 = false;
    int T = 1, fv = 1;
    FastTile2D *d_inner = nullptr, *d_frame = nullptr;
    int ni = 0, nf = 0, grid_f = 0, grid_p = 0;
    SideStream side;   // CPML frame launches next to the interior ones
    int64_t interior_cells = 0, all_cells = 0;

    static bool compatible(const Job2D<R>* a, const Job2D<R>* b) {
        return a->te == b->te && a->idx16 == b->idx16 && a->T == b->T && a->fvariant == b->fvariant;
    }
    void add(Job2D<R>* j) {
        if (jobs.empty()) {
            te = j->te;
            idx16 = j->idx16;
            T = j->T;
            fv = j->fvariant;
        }
        jobs.push_back(j);
        dirty = true;
    }
    void remove(orf_job* j) override {
        for (size_t q = 0; q < jobs.size(); ++q)
            if (jobs[q] == j) {
                jobs.erase(jobs.begin() + q);
                dirty = true;
                return;
            }
    }
    int size() const override { return (int)jobs.size(); }
    int64_t cells() const override { return all_cells; }

    int build(cudaStream_t st) override {
        std::vector<FastTile2D> inner, frame;
        streams.clear();
        items.clear();
        states.clear();
        interior_cells = all_cells = 0;
        for (auto* j : jobs) {
            inner.insert(inner.end(), j->ftiles_host.begin(), j->ftiles_host.begin() + j->nfast);
            frame.insert(frame.end(), j->ftiles_host.begin() + j->nfast, j->ftiles_host.end());
            for (int q = 0; q < j->nfast; ++q)
                interior_cells += (int64_t)j->ftiles_host[q].ow * j->ftiles_host[q].oh;
            all_cells += j->cells();
            add_streams(j->host_streams, j->nL, j->d_st);
        }
        sort_frame_tiles(frame.begin(), frame.end());   // members' frames, by CPML specialisation
        cudaStreamSynchronize(st);   // descriptors of the previous build may still be read
        arena.release();
        Arena ar;
        ar.add(&d_inner, inner.size() + 1);
        ar.add(&d_frame, frame.size() + 1);
        ar.add(&d_streams, streams.size() + 1);
        ar.add(&d_items, items.size() + 1);
        ar.add(&d_states, states.size() + 1);
        ORF_TRY(ar.alloc());
        arena = ar;
        ORF_TRY(upload(st, d_inner, inner.data(), inner.size() * sizeof(FastTile2D)));
        ORF_TRY(upload(st, d_frame, frame.data(), frame.size() * sizeof(FastTile2D)));
        ORF_TRY(upload(st, d_streams, streams.data(), streams.size() * sizeof(DftStream)));
        ORF_TRY(upload(st, d_items, items.data(), items.size() * sizeof(FlushItem)));
        ORF_TRY(upload(st, d_states, states.data(), states.size() * sizeof(JobState*)));
        ORF_CUDA(cudaStreamSynchronize(st));
        const bool f64 = sizeof(R) == 8;
        ni = (int)inner.size();
        nf = (int)frame.size();
        const int bps_f = fast2d_blocks_per_sm(f64, te, idx16, false, fv);
        const int bps_p = fast2d_blocks_per_sm(f64, te, idx16, true, 0);
        grid_f = (int)std::min<int64_t>(ni, (int64_t)ctx->sm_count * std::max(1, bps_f));
        grid_p = (int)std::min<int64_t>(nf, (int64_t)ctx->sm_count * std::max(1, bps_p));
        wire_engine(f64, T);
        if (ni && nf) ORF_TRY(side.init());
        eng.step = [this, f64](int off, int nsub, int par, int we, cudaStream_t s, KernelTimer* tm) -> cudaError_t {
            cudaError_t e = cudaSuccess;
            cudaEvent_t a = nullptr;
            const bool overlap = !tm && side.ok() && ni && nf;
            cudaStream_t fs = s;
            if (overlap) {
                e = side.fork(s);
                if (e != cudaSuccess) return e;
                fs = side.s2;
            }
            if (ni) {
                if (tm && tm->begin(s, &a) != ORF_OK) return cudaErrorUnknown;
                e = launch_fast2d(f64, te, idx16, false, fv, d_inner, ni, off, nsub, par, we, grid_f, s);
                if (e != cudaSuccess) return e;
                if (tm && tm->end(s, 0, interior_cells * nsub, a) != ORF_OK) return cudaErrorUnknown;
            }
            if (nf) {
                if (tm && tm->begin(fs, &a) != ORF_OK) return cudaErrorUnknown;
                e = launch_fast2d(f64, te, idx16, true, 0, d_frame, nf, off, nsub, par, we, grid_p, fs);
                if (e != cudaSuccess) return e;
                if (tm && tm->end(fs, 1, (all_cells - interior_cells) * nsub, a) != ORF_OK) return cudaErrorUnknown;
            }
            if (overlap) e = side.join(s);
            return e;
        };
        dirty = false;
        return ORF_OK;
    }
};

// 3D members share precision and index width (zc is the z-segment length,
// the same for every job).
template <class R>
struct Group3D : Group {
    std::vector<Job3D<R>*> jobs;
    int zc = 4, idxw = 1;
    Inst3D<R>* d_insts = nullptr;
    Tile3D *d_tiles = nullptr, *d_tiles_pml = nullptr;
    int nt = 0, ntp = 0;
    SideStream side;   // CPML tiles next to the interior tiles
    int64_t all_cells = 0;

    static bool compatible(const Job3D<R>* a, const Job3D<R>* b) { return a->zc == b->zc && a->idxw == b->idxw; }
    void add(Job3D<R>* j) {
        if (jobs.empty()) {
            zc = j->zc;
            idxw = j->idxw;
        }
        jobs.push_back(j);
        dirty = true;
    }
    void remove(orf_job* j) override {
        for (size_t q = 0; q < jobs.size(); ++q)
            if (jobs[q] == j) {
                jobs.erase(jobs.begin() + q);
                dirty = true;
                return;
            }
    }
    int size() const override { return (int)jobs.size(); }
    int64_t cells() const override { return all_cells; }

    int build(cudaStream_t st) override {
        std::vector<Inst3D<R>> insts;
        std::vector<Tile3D> tl, tp;
        streams.clear();
        items.clear();
        states.clear();
        all_cells = 0;
        for (auto* j : jobs) {
            const int id = (int)insts.size();
            insts.push_back(j->h);
            for (Tile3D t : j->tiles) {
                t.inst = id;
                tl.push_back(t);
            }
            for (Tile3D t : j->tiles_pml) {
                t.inst = id;
                tp.push_back(t);
            }
            all_cells += j->cells();
            add_streams(j->host_streams, j->nL, j->d_st);
        }
        cudaStreamSynchronize(st);
        arena.release();
        Arena ar;
        ar.add(&d_insts, insts.size() + 1);
        ar.add(&d_tiles, tl.size() + 1);
        ar.add(&d_tiles_pml, tp.size() + 1);
        ar.add(&d_streams, streams.size() + 1);
        ar.add(&d_items, items.size() + 1);
        ar.add(&d_states, states.size() + 1);
        ORF_TRY(ar.alloc());
        arena = ar;
        ORF_TRY(upload(st, d_insts, insts.data(), insts.size() * sizeof(Inst3D<R>)));
        ORF_TRY(upload(st, d_tiles, tl.data(), tl.size() * sizeof(Tile3D)));
        ORF_TRY(upload(st, d_tiles_pml, tp.data(), tp.size() * sizeof(Tile3D)));
        ORF_TRY(upload(st, d_streams, streams.data(), streams.size() * sizeof(DftStream)));
        ORF_TRY(upload(st, d_items, items.data(), items.size() * sizeof(FlushItem)));
        ORF_TRY(upload(st, d_states, states.data(), states.size() * sizeof(JobState*)));
        ORF_CUDA(cudaStreamSynchronize(st));
        nt = (int)tl.size();
        ntp = (int)tp.size();
        const bool f64 = sizeof(R) == 8;
        wire_engine(f64, 1);
        if (nt && ntp) ORF_TRY(side.init());
        eng.step = [this, f64](int off, int nsub, int par, int we, cudaStream_t s, KernelTimer* tm) -> cudaError_t {
            (void)nsub;
            cudaEvent_t a = nullptr;
            if (tm && tm->begin(s, &a) != ORF_OK) return cudaErrorUnknown;
            const bool overlap = !tm && side.ok() && nt && ntp;
            cudaError_t e = overlap ? side.fork(s) : cudaSuccess;
            if (e == cudaSuccess) e = launch_step3d(f64, false, idxw, d_insts, d_tiles, nt, par, off, we, wait_ctl(ctx), s);
            if (e == cudaSuccess)
                e = launch_step3d(f64, true, idxw, d_insts, d_tiles_pml, ntp, par, off, we, wait_ctl(ctx),
                                  overlap ? side.s2 : s);
            if (e == cudaSuccess && overlap) e = side.join(s);
            if (e != cudaSuccess) return e;
            if (tm && tm->end(s, 0, all_cells, a) != ORF_OK) return cudaErrorUnknown;
            return e;
        };
        dirty = false;
        return ORF_OK;
    }
};

}  // namespace orf
