// checkpoint.cu -- checkpoint / resume of device-resident jobs
// (orf_job_checkpoint_size / orf_job_checkpoint / orf_job_restore).
//
// Between chunks a job's whole evolving state is: the field buffer holding
// the latest step (JobState.cur) with its CPML psi, the DFT sums, and the
// scalars of JobState (step, chunk, energy peak, done / converged).  The
// checkpoint is a header, those scalars, and the state regions of buffer
// `cur` in the order the job lists them (Job2D / Job3D::state_regions).  A
// restore writes the regions into buffer 0 of a job created from the same
// sim (the server: the buffer its group launches from next), sets cur and the
// counters, and re-arms the host's progress loop at the restored chunk: the
// kernels' arithmetic does not depend on the buffer parity or the tiling, so
// the continued run is bitwise the uninterrupted one.
#include "engine.cuh"

namespace orf {
namespace {

constexpr char kMagic[8] = {'O', 'R', 'F', 'C', 'K', 'P', 'T', '1'};

struct CkptHeader {
    char magic[8];
    int32_t dims;
    int32_t nregions;
    uint64_t key;
    uint64_t total;        // bytes of the whole checkpoint
    int64_t step, chunk;
    int32_t done, converged;
    double energy, peak;
};

size_t ckpt_bytes(const std::vector<std::pair<void*, size_t>>& regs) {
    size_t b = sizeof(CkptHeader) + regs.size() * sizeof(uint64_t);
    for (auto& r : regs) b += r.second;
    return b;
}

// every copy goes through the job's stream (non-blocking: the legacy default
// stream would not order against it), then that stream is synchronised
int read_state(orf_job* job, JobState* js) {
    cudaStream_t st = job->ctx->stream;
    ORF_CUDA(cudaMemcpyAsync(js, job->state_dev(), sizeof(JobState), cudaMemcpyDeviceToHost, st));
    ORF_CUDA(cudaStreamSynchronize(st));
    return ORF_OK;
}

}  // namespace

int job_checkpoint_size(orf_job* job, size_t* bytes) {
    std::vector<std::pair<void*, size_t>> regs;
    job->state_regions(0, regs);
    *bytes = ckpt_bytes(regs);
    return ORF_OK;
}

int job_checkpoint(orf_job* job, void* buf, size_t bytes) {
    JobState js{};
    ORF_TRY(read_state(job, &js));
    std::vector<std::pair<void*, size_t>> regs;
    job->state_regions(js.cur, regs);
    const size_t need = ckpt_bytes(regs);
    if (bytes < need) {
        set_error("checkpoint needs %zu bytes, the buffer has %zu", need, bytes);
        return ORF_EINVAL;
    }
    CkptHeader hd{};
    std::memcpy(hd.magic, kMagic, sizeof kMagic);
    hd.dims = job->dims;
    hd.nregions = (int32_t)regs.size();
    hd.key = job->state_key();
    hd.total = need;
    hd.step = js.step;
    hd.chunk = js.chunk;
    hd.done = js.done;
    hd.converged = js.converged;
    hd.energy = js.energy;
    hd.peak = js.peak;
    unsigned char* p = static_cast<unsigned char*>(buf);
    std::memcpy(p, &hd, sizeof hd);
    p += sizeof hd;
    for (auto& r : regs) {
        const uint64_t n = r.second;
        std::memcpy(p, &n, sizeof n);
        p += sizeof n;
    }
    for (auto& r : regs) {
        ORF_CUDA(cudaMemcpyAsync(p, r.first, r.second, cudaMemcpyDeviceToHost, job->ctx->stream));
        job->ctx->stats.d2h_bytes += (int64_t)r.second;
        p += r.second;
    }
    ORF_CUDA(cudaStreamSynchronize(job->ctx->stream));
    return ORF_OK;
}

int job_restore(orf_job* job, const void* buf, size_t bytes, int into) {
    CkptHeader hd{};
    if (bytes < sizeof hd) {
        set_error("not a checkpoint: %zu bytes", bytes);
        return ORF_EINVAL;
    }
    std::memcpy(&hd, buf, sizeof hd);
    std::vector<std::pair<void*, size_t>> regs;
    job->state_regions(into, regs);
    if (std::memcmp(hd.magic, kMagic, sizeof kMagic) != 0) {
        set_error("not a checkpoint of this library");
        return ORF_EINVAL;
    }
    if (hd.dims != job->dims || hd.key != job->state_key() || hd.nregions != (int32_t)regs.size() ||
        hd.total != ckpt_bytes(regs) || bytes < hd.total) {
        set_error("the checkpoint belongs to another run (dimension, precision, grid or monitors differ)");
        return ORF_EINVAL;
    }
    const unsigned char* p = static_cast<const unsigned char*>(buf) + sizeof hd;
    for (auto& r : regs) {
        uint64_t n = 0;
        std::memcpy(&n, p, sizeof n);
        p += sizeof n;
        if (n != r.second) {
            set_error("the checkpoint belongs to another run (state sizes differ)");
            return ORF_EINVAL;
        }
    }
    JobState js{};
    ORF_TRY(read_state(job, &js));
    for (auto& r : regs) {
        ORF_CUDA(cudaMemcpyAsync(r.first, p, r.second, cudaMemcpyHostToDevice, job->ctx->stream));
        job->ctx->stats.h2d_bytes += (int64_t)r.second;
        p += r.second;
    }
    js.step = hd.step;
    js.chunk = hd.chunk;
    js.converged = hd.converged;
    // the energy shutoff ends a run for good; a cancelled run, or one that
    // used up a smaller step budget, continues
    js.done = (hd.converged || hd.step >= job->nmax_steps()) ? 1 : 0;
    js.cur = into;
    js.fault = 0;
    js.energy = hd.energy;
    js.peak = hd.peak;
    ORF_CUDA(cudaMemcpyAsync(job->state_dev(), &js, sizeof js, cudaMemcpyHostToDevice, job->ctx->stream));
    ORF_CUDA(cudaStreamSynchronize(job->ctx->stream));
    job->resume_host(js);
    return ORF_OK;
}

}  // namespace orf

extern "C" {

int32_t orf_job_checkpoint_size(orf_job* job, size_t* bytes) {
    if (!job || !bytes) return ORF_EINVAL;
    ORF_ON_DEVICE(job->ctx->device);
    return orf::job_checkpoint_size(job, bytes);
}

int32_t orf_job_checkpoint(orf_job* job, void* buf, size_t bytes) {
    if (!job || !buf) return ORF_EINVAL;
    ORF_ON_DEVICE(job->ctx->device);
    return orf::job_checkpoint(job, buf, bytes);
}

int32_t orf_job_restore(orf_job* job, const void* buf, size_t bytes) {
    if (!job || !buf) return ORF_EINVAL;
    ORF_ON_DEVICE(job->ctx->device);
    return orf::job_restore(job, buf, bytes, 0);
}

}  // extern "C"
