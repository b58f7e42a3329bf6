// serve.cu -- continuous-batching server for streams of FDTD jobs (orf_serve_*).
//
// The reference serves nothing: every sweep point, optimiser evaluation or
// app request is one blocking orf.fdtd2D / orf.fdtd3D call
// (examples/cpo_box_scan.m:23-31, optimizeGratingCoupler.m:1-12,
// toolbox/+orf/fdtd2D.m:1-29).  The server accepts 2D and 3D jobs at any
// time and keeps as many resident on the GPU as its device-memory budget and
// slot count allow:
//
//   submit  copies the sim (all arrays) into a FIFO queue and returns a ticket;
//   step    (one scheduling round) admits queued jobs in FIFO order while
//           their device arenas fit the budget, adds each to the group of
//           resident jobs sharing its kernel configuration and size class
//           (group.cuh; a class spans a factor of 4 in cells), runs chunks of
//           every group -- each group on its own stream, so groups overlap --
//           and retires the jobs whose device state reports done (shutoff or
//           step budget): their results go to the caller's out struct, their
//           memory back to the budget.  The group whose chunk costs most runs
//           macro_steps time steps per round; a group of smaller jobs runs
//           proportionally more chunks (at most half the status ring), so
//           small jobs are not held to the pace of the largest ones;
//   poll    reports a finished ticket with its submit/admit/done times.
//
// A job is admitted only between chunks and starts from zeroed fields, so its
// arithmetic is the same as a run of that sim alone; the alone-vs-mix
// identity is a test.  FIFO admission means a large job at the head waits
// for memory rather than being overtaken.  A job whose arena exceeds the
// whole budget fails with ORF_ETOOLARGE when nothing else is resident.
#include <deque>
#include <mutex>
#include <unordered_map>

#include "group.cuh"

namespace orf {
namespace {

template <class T>
const T* keep(std::vector<T>& v, const T* p, size_t n) {
    if (!p) return nullptr;
    v.assign(p, p + n);
    return v.data();
}

struct SrvJob {
    int64_t ticket = 0;
    int dims = 2;
    orf_sim2d s2{};
    orf_sim3d s3{};
    std::vector<double> a0, a1, a2, a3, lam;
    std::vector<int32_t> i0, i1;
    orf_out2d* o2 = nullptr;   // caller's out structs, written at retirement
    orf_out3d* o3 = nullptr;
    std::unique_ptr<orf_job> job;
    ProgressLoop* pl = nullptr;   // the job's status-ring reader
    Group* group = nullptr;
    size_t need = 0;    // device arena bytes, known after the first admission attempt
    std::vector<unsigned char> snapshot;   // checkpoint of a preempted job, restored at re-admission
    orf_serve_job_info info{};

    void copy2d(const orf_sim2d* s, orf_out2d* o) {
        dims = 2;
        s2 = *s;
        const size_t nx = s->nx, nz = s->nz, nzA = s->periodic_z ? nz : nz - 1;
        s2.eps = keep(a0, s->eps, nx * nz);
        s2.eps_x = keep(a1, s->eps_x, nx * nzA);
        s2.eps_z = keep(a2, s->eps_z, (nx - 1) * nz);
        s2.src_profile = keep(a3, s->src_profile, nz);
        s2.monitors = keep(i0, s->monitors, (size_t)s->n_mon);
        s2.monitors_z = keep(i1, s->monitors_z, (size_t)s->n_monz);
        s2.lambdas = keep(lam, s->lambdas, (size_t)s->n_lambda);
        o2 = o;
    }
    void copy3d(const orf_sim3d* s, orf_out3d* o) {
        dims = 3;
        s3 = *s;
        const int n[3] = {s->nx, s->ny, s->nz};
        const size_t N = (size_t)n[0] * n[1] * n[2];
        const int a = s->src_axis;
        const size_t nab = (size_t)n[(a + 1) % 3] * n[(a + 2) % 3];
        // the three permittivity arrays and four source profiles share storage
        a0.resize(3 * N);
        std::copy(s->eps_x, s->eps_x + N, a0.begin());
        std::copy(s->eps_y, s->eps_y + N, a0.begin() + N);
        std::copy(s->eps_z, s->eps_z + N, a0.begin() + 2 * N);
        s3.eps_x = a0.data();
        s3.eps_y = a0.data() + N;
        s3.eps_z = a0.data() + 2 * N;
        a1.resize(4 * nab);
        std::copy(s->src_Ea, s->src_Ea + nab, a1.begin());
        std::copy(s->src_Eb, s->src_Eb + nab, a1.begin() + nab);
        std::copy(s->src_Ha, s->src_Ha + nab, a1.begin() + 2 * nab);
        std::copy(s->src_Hb, s->src_Hb + nab, a1.begin() + 3 * nab);
        s3.src_Ea = a1.data();
        s3.src_Eb = a1.data() + nab;
        s3.src_Ha = a1.data() + 2 * nab;
        s3.src_Hb = a1.data() + 3 * nab;
        s3.mon_axis = keep(i0, s->mon_axis, (size_t)s->n_mon);
        s3.mon_index = keep(i1, s->mon_index, (size_t)s->n_mon);
        s3.lambdas = keep(lam, s->lambdas, (size_t)s->n_lambda);
        o3 = o;
    }
    int precision() const { return dims == 2 ? s2.precision : s3.precision; }
};

struct GroupSlot {
    int64_t key = 0;
    std::unique_ptr<Group> g;
    cudaStream_t stream = nullptr;
};

}  // namespace
}  // namespace orf

using namespace orf;

struct orf_server {
    orf_ctx* ctx = nullptr;
    size_t budget = 0, used = 0;
    int max_jobs = 1024;
    int chunks_per_step = 4;
    double t0 = 0;
    std::mutex mu;   // guards queue, finished and next (submit/poll may come from other threads)
    int64_t next = 1;
    std::deque<std::unique_ptr<SrvJob>> queue;
    std::unordered_map<int64_t, orf_serve_job_info> finished;
    std::vector<std::unique_ptr<SrvJob>> resident;
    std::vector<GroupSlot> groups;

    double clock() const { return now_s() - t0; }

    ~orf_server() {
        for (auto& s : groups)
            if (s.stream) cudaStreamSynchronize(s.stream);
        resident.clear();
        for (auto& s : groups) {
            s.g.reset();
            if (s.stream) cudaStreamDestroy(s.stream);
        }
    }

    // size class of a job: floor(log4(cells))
    static int64_t size_class(int64_t cells) {
        int64_t c = 0;
        while (cells >= 4) {
            cells >>= 2;
            ++c;
        }
        return c;
    }

    // chunks of each group in this round: the group whose chunk costs most
    // (cells x the rough cost of a cell update of its kind; only the ratios
    // matter) runs chunks_per_step, cheaper ones proportionally more, up to
    // half the status ring read between rounds
    void plan_round(std::vector<int>& nch) const {
        nch.assign(groups.size(), chunks_per_step);
        std::vector<double> cost(groups.size());
        double top = 0.0;
        for (size_t q = 0; q < groups.size(); ++q) {
            const bool is3d = (groups[q].key & 3) == 3;
            cost[q] = (double)groups[q].g->cells() * (is3d ? 2.0 : 1.0);
            top = std::max(top, cost[q]);
        }
        for (size_t q = 0; q < groups.size(); ++q) {
            const double r = cost[q] > 0 ? top / cost[q] : 1.0;
            nch[q] = (int)std::min<double>(kStatusRing / 2, std::max<double>(chunks_per_step,
                                                                              std::floor(chunks_per_step * r)));
        }
    }

    Group* group_for(int64_t key) {
        for (auto& s : groups)
            if (s.key == key) return s.g.get();
        return nullptr;
    }

    int new_group(int64_t key, std::unique_ptr<Group> g) {
        GroupSlot s;
        s.key = key;
        g->ctx = ctx;
        s.g = std::move(g);
        ORF_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
        groups.push_back(std::move(s));
        return ORF_OK;
    }

    // Create the job's device state within the budget and place it in its
    // group.  Returns ORF_OK, or an error with *fits = false when the job
    // waits for memory.
    template <class R>
    int admit2d(SrvJob* J, size_t left, bool* fits) {
        auto j = std::make_unique<Job2D<R>>();
        j->ctx = ctx;
        j->budget = left;
        const int st = j->create(&J->s2);
        J->need = j->need;
        if (st != ORF_OK) {
            *fits = !((st == ORF_ETOOLARGE && j->need > left) || st == ORF_ENOMEM_DEVICE);
            return st;
        }
        const int64_t key = 2 | (int64_t)(sizeof(R) == 8) << 2 | (int64_t)j->te << 3 | (int64_t)j->idx16 << 4 |
                            (int64_t)j->T << 8 | (int64_t)j->fvariant << 16 | size_class(j->cells()) << 24;
        Group* g = group_for(key);
        if (!g) {
            ORF_TRY(new_group(key, std::make_unique<Group2D<R>>()));
            g = groups.back().g.get();
        }
        static_cast<Group2D<R>*>(g)->add(j.get());
        ORF_TRY(resume(J, j.get(), g));
        J->group = g;
        J->pl = &j->pl;
        J->job = std::move(j);
        return ORF_OK;
    }
    template <class R>
    int admit3d(SrvJob* J, size_t left, bool* fits) {
        auto j = std::make_unique<Job3D<R>>();
        j->ctx = ctx;
        j->budget = left;
        const int st = j->create(&J->s3);
        J->need = j->need;
        if (st != ORF_OK) {
            *fits = !((st == ORF_ETOOLARGE && j->need > left) || st == ORF_ENOMEM_DEVICE);
            return st;
        }
        const int64_t key = 3 | (int64_t)(sizeof(R) == 8) << 2 | (int64_t)j->idxw << 8 | (int64_t)j->zc << 16 |
                            size_class(j->cells()) << 24;
        Group* g = group_for(key);
        if (!g) {
            ORF_TRY(new_group(key, std::make_unique<Group3D<R>>()));
            g = groups.back().g.get();
        }
        static_cast<Group3D<R>*>(g)->add(j.get());
        ORF_TRY(resume(J, j.get(), g));
        J->group = g;
        J->pl = &j->pl;
        J->job = std::move(j);
        return ORF_OK;
    }

    // a preempted job continues from its checkpoint, restored into the field
    // buffer its group launches from next (the group's members share one
    // buffer parity)
    int resume(SrvJob* J, orf_job* j, Group* g) {
        if (J->snapshot.empty()) return ORF_OK;
        const int st = job_restore(j, J->snapshot.data(), J->snapshot.size(), g->eng.par);
        if (st != ORF_OK) {
            g->remove(j);
            return st;
        }
        std::vector<unsigned char>().swap(J->snapshot);
        return ORF_OK;
    }

    // move a resident job's state to host memory and queue it again (at the
    // end); called between scheduling rounds, when no group work is in flight
    int preempt(int64_t ticket) {
        for (size_t q = 0; q < resident.size(); ++q) {
            if (resident[q]->ticket != ticket) continue;
            SrvJob* J = resident[q].get();
            orf_job* j = J->job.get();
            J->pl->poll(nullptr, nullptr);
            if (J->pl->done) return ORF_OK;   // finished: it retires at the next round
            size_t n = 0;
            ORF_TRY(job_checkpoint_size(j, &n));
            std::vector<unsigned char> snap(n);
            ORF_TRY(job_checkpoint(j, snap.data(), n));
            J->group->remove(j);
            J->group = nullptr;
            J->pl = nullptr;
            J->job.reset();
            used -= std::min(used, J->need);
            J->snapshot = std::move(snap);
            J->info.preemptions += 1;
            std::unique_ptr<SrvJob> P = std::move(resident[q]);
            resident.erase(resident.begin() + q);
            std::lock_guard<std::mutex> lk(mu);
            queue.push_back(std::move(P));
            return ORF_OK;
        }
        std::lock_guard<std::mutex> lk(mu);
        if (ticket < 1 || ticket >= next) {
            set_error("unknown ticket %lld", (long long)ticket);
            return ORF_EINVAL;
        }
        return ORF_OK;   // queued or finished: nothing to move
    }

    void fail(std::unique_ptr<SrvJob> J, int status) {
        J->info.status = status;
        J->info.t_done = clock();
        std::lock_guard<std::mutex> lk(mu);
        finished[J->ticket] = J->info;
    }

    // FIFO admission while slots and budget allow
    int admit() {
        bool any = false;
        while ((int)resident.size() < max_jobs) {
            std::unique_ptr<SrvJob> J;
            {
                std::lock_guard<std::mutex> lk(mu);
                if (queue.empty()) break;
                const size_t left = budget > used ? budget - used : 0;
                if (queue.front()->need && queue.front()->need > left && !resident.empty()) break;
                J = std::move(queue.front());
                queue.pop_front();
            }
            const size_t left = budget > used ? budget - used : 0;
            bool fits = true;
            int st;
            if (J->dims == 2)
                st = J->precision() == ORF_SINGLE ? admit2d<float>(J.get(), left, &fits)
                                                  : admit2d<double>(J.get(), left, &fits);
            else
                st = J->precision() == ORF_SINGLE ? admit3d<float>(J.get(), left, &fits)
                                                  : admit3d<double>(J.get(), left, &fits);
            if (st == ORF_OK) {
                if (J->info.preemptions == 0) J->info.t_admit = clock();   // the first admission
                J->info.device_bytes = (int64_t)J->need;
                used += J->need;
                resident.push_back(std::move(J));
                any = true;
                continue;
            }
            if (!fits && !resident.empty()) {
                // wait for memory at the head of the queue
                std::lock_guard<std::mutex> lk(mu);
                queue.push_front(std::move(J));
                break;
            }
            fail(std::move(J), st);
        }
        if (any) ORF_CUDA(cudaStreamSynchronize(ctx->stream));
        return ORF_OK;
    }

    int retire() {
        for (size_t q = 0; q < resident.size();) {
            SrvJob* J = resident[q].get();
            orf_job* j = J->job.get();
            J->pl->poll(nullptr, nullptr);
            if (!J->pl->done) {
                ++q;
                continue;
            }
            J->group->remove(j);
            const int st = J->dims == 2 ? j->finish2d(J->o2) : j->finish3d(J->o3);
            J->info.steps = J->dims == 2 ? J->o2->steps : J->o3->steps;
            ctx->stats.cell_updates += J->info.steps * j->cells();
            J->info.status = st;
            J->info.t_done = clock();
            if (J->dims == 2)
                J->o2->wall_time = J->info.t_done - J->info.t_submit;
            else
                J->o3->wall_time = J->info.t_done - J->info.t_submit;
            used -= std::min(used, J->need);
            J->job.reset();
            std::unique_ptr<SrvJob> done = std::move(resident[q]);
            resident.erase(resident.begin() + q);
            std::lock_guard<std::mutex> lk(mu);
            finished[done->ticket] = done->info;
        }
        return ORF_OK;
    }

    int step() {
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev != ctx->device) ORF_CUDA(cudaSetDevice(ctx->device));
        ORF_TRY(admit());
        // drop empty groups, rebuild changed ones
        for (size_t q = 0; q < groups.size();) {
            if (groups[q].g->size() == 0) {
                cudaStreamSynchronize(groups[q].stream);
                groups[q].g.reset();
                cudaStreamDestroy(groups[q].stream);
                groups.erase(groups.begin() + q);
                continue;
            }
            if (groups[q].g->dirty) ORF_TRY(groups[q].g->build(groups[q].stream));
            ++q;
        }
        std::vector<int> nch;
        plan_round(nch);
        for (size_t q = 0; q < groups.size(); ++q) ORF_TRY(groups[q].g->enqueue(nch[q], groups[q].stream));
        for (auto& s : groups) ORF_CUDA(cudaStreamSynchronize(s.stream));
        for (auto& s : groups) s.g->eng.collect_timing();
        return retire();
    }
};

// ------------------------------------------------------------------ C ABI --
extern "C" {

int32_t orf_serve_open(orf_ctx* ctx, const orf_serve_cfg* cfg, orf_server** srv) {
    if (!srv) {
        set_error("srv is NULL");
        return ORF_EINVAL;
    }
    *srv = nullptr;
    int st = ORF_OK;
    if (!ctx) ctx = default_ctx(&st);
    if (!ctx) return st;
    orf_serve_cfg c{};
    if (cfg) c = *cfg;
    if (c.max_device_bytes < 0 || c.max_jobs < 0 || c.macro_steps < 0) {
        set_error("orf_serve_cfg fields must be >= 0");
        return ORF_EINVAL;
    }
    ORF_ON_DEVICE(ctx->device);
    auto s = std::make_unique<orf_server>();
    s->ctx = ctx;
    if (c.max_device_bytes > 0) {
        s->budget = (size_t)c.max_device_bytes;
    } else {
        size_t fr = 0, tot = 0;
        dev_trim(ctx->device);   // cached blocks count as free memory here
        ORF_CUDA(cudaMemGetInfo(&fr, &tot));
        s->budget = (size_t)(0.9 * (double)fr);
    }
    s->max_jobs = c.max_jobs > 0 ? c.max_jobs : 1024;
    const int macro = c.macro_steps > 0 ? c.macro_steps : 200;
    // whole chunks; at most half the status ring between two reads of it
    s->chunks_per_step = std::max(1, std::min(kStatusRing / 2, (macro + kChunk - 1) / kChunk));
    s->t0 = now_s();
    ctx_retain(ctx);
    *srv = s.release();
    return ORF_OK;
}

int32_t orf_serve_submit2d(orf_server* srv, const orf_sim2d* sim, orf_out2d* out, int64_t* ticket) {
    if (!srv || !out || !ticket) {
        set_error("srv, out and ticket must not be NULL");
        return ORF_EINVAL;
    }
    ORF_TRY(validate2d(sim));
    auto J = std::make_unique<SrvJob>();
    J->copy2d(sim, out);
    J->info.t_submit = srv->clock();
    J->info.dims = 2;
    J->info.cells = (int64_t)sim->nx * sim->nz;
    std::lock_guard<std::mutex> lk(srv->mu);
    J->ticket = srv->next++;
    *ticket = J->ticket;
    srv->queue.push_back(std::move(J));
    return ORF_OK;
}

int32_t orf_serve_submit3d(orf_server* srv, const orf_sim3d* sim, orf_out3d* out, int64_t* ticket) {
    if (!srv || !out || !ticket) {
        set_error("srv, out and ticket must not be NULL");
        return ORF_EINVAL;
    }
    ORF_TRY(validate3d(sim));
    auto J = std::make_unique<SrvJob>();
    J->copy3d(sim, out);
    J->info.t_submit = srv->clock();
    J->info.dims = 3;
    J->info.cells = (int64_t)sim->nx * sim->ny * sim->nz;
    std::lock_guard<std::mutex> lk(srv->mu);
    J->ticket = srv->next++;
    *ticket = J->ticket;
    srv->queue.push_back(std::move(J));
    return ORF_OK;
}

int32_t orf_serve_step(orf_server* srv) {
    if (!srv) {
        set_error("srv is NULL");
        return ORF_EINVAL;
    }
    ORF_ON_DEVICE(srv->ctx->device);
    return srv->step();
}

int32_t orf_serve_poll(orf_server* srv, int64_t ticket, orf_serve_job_info* info) {
    if (!srv) {
        set_error("srv is NULL");
        return ORF_EINVAL;
    }
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->finished.find(ticket);
    if (it != srv->finished.end()) {
        if (info) *info = it->second;
        return ORF_OK;
    }
    if (ticket < 1 || ticket >= srv->next) {
        set_error("unknown ticket %lld", (long long)ticket);
        return ORF_EINVAL;
    }
    return ORF_EBUSY;
}

int32_t orf_serve_preempt(orf_server* srv, int64_t ticket) {
    if (!srv) {
        set_error("srv is NULL");
        return ORF_EINVAL;
    }
    ORF_ON_DEVICE(srv->ctx->device);
    return srv->preempt(ticket);
}

int32_t orf_serve_pending(orf_server* srv, int32_t* queued, int32_t* resident) {
    if (!srv) {
        set_error("srv is NULL");
        return ORF_EINVAL;
    }
    std::lock_guard<std::mutex> lk(srv->mu);
    if (queued) *queued = (int32_t)srv->queue.size();
    if (resident) *resident = (int32_t)srv->resident.size();
    return ORF_OK;
}

double orf_serve_clock(orf_server* srv) { return srv ? srv->clock() : 0.0; }

int32_t orf_serve_close(orf_server* srv) {
    if (!srv) return ORF_OK;
    orf_ctx* c = srv->ctx;
    {
        ORF_ON_DEVICE(c->device);
        delete srv;
        ctx_release(c);
    }
    return ORF_OK;
}

}  // extern "C"
