// runtime.cuh -- host-side runtime shared by the 2D, 3D, batch and serve paths.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <atomic>
#include <memory>
#include <string>
#include <vector>

#include "orf_fdtd.h"
#include "orf_internal.cuh"

namespace orf {

// ------------------------------------------------------------------ errors --
void set_error(const char* fmt, ...);
const char* last_error();

struct Err {
    int code = ORF_OK;
    explicit operator bool() const { return code != ORF_OK; }
};

#define ORF_CUDA(call)                                                                    \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            ::orf::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
            return e_ == cudaErrorMemoryAllocation ? ORF_ENOMEM_DEVICE : ORF_ECUDA;       \
        }                                                                                 \
    } while (0)

#define ORF_TRY(expr)                      \
    do {                                   \
        int s_ = (expr);                   \
        if (s_ != ORF_OK) return s_;       \
    } while (0)

inline double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Makes `device` current for the scope of a C entry point and gives the
// calling thread its own current device back on every return path, so a call
// on a context of another GPU leaves the caller where it was.
struct DeviceScope {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceScope(int device) {
        if (cudaGetDevice(&prev) != cudaSuccess) {
            cudaGetLastError();
            prev = -1;
        }
        if (prev != device) err = cudaSetDevice(device);
    }
    DeviceScope(const DeviceScope&) = delete;
    DeviceScope& operator=(const DeviceScope&) = delete;
    ~DeviceScope() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};
#define ORF_ON_DEVICE(dev)                                                             \
    ::orf::DeviceScope orf_devscope_(dev);                                             \
    if (orf_devscope_.err != cudaSuccess) {                                            \
        ::orf::set_error("cudaSetDevice(%d): %s", (int)(dev), cudaGetErrorString(orf_devscope_.err)); \
        cudaGetLastError();                                                            \
        return ORF_ECUDA;                                                              \
    }

// --------------------------------------------------------- shared physics --
// These restate the reference's documented formulas; the CPU oracle holds an
// independent copy of the same definitions.
constexpr double kPi = 3.14159265358979323846;
constexpr double kPmlOrder = 3.0;          // cpmlCoefficients.m:6-8 grading law; constants chosen here
constexpr double kPmlKappaMax = 1.0;
static_assert(!kUnitKappa || kPmlKappaMax == 1.0, "the step kernels assume 1/kappa = 1 (kUnitKappa)");
constexpr double kPmlAlphaMaxPerK0 = 0.0;

// Gaussian pulse of relative 1/e spectral half-width bw (fdtd2DTE.m:14-15):
// g(t) = exp(-((t-t0)/tau)^2) sin(k0 (t-t0)), tau = 2/(bw k0), t0 = 5 tau, zero outside [0, 2 t0].
struct Pulse {
    double k0, tau, t0, tend;
    Pulse(double lambda0, double bw) {
        k0 = 2.0 * kPi / lambda0;
        tau = 2.0 / (bw * k0);
        t0 = 5.0 * tau;
        tend = 2.0 * t0;
    }
    double operator()(double t) const {
        if (t < 0.0 || t > tend) return 0.0;
        const double u = (t - t0) / tau;
        return std::exp(-u * u) * std::sin(k0 * (t - t0));
    }
};

// CPML (b, a, 1/kappa) at positions u = i + off on an n-point grid with npml
// cells per end (cpmlCoefficients.m:2-8); identity outside the layer.
void pml_profile(int n, int npts, int npml, double off, double dx, double S, double alpha_max,
                 std::vector<double>& bak, int* nslab);

int64_t max_steps(double max_time, double S);
double progress_fraction(double t, double src_end, double ratio, double shutoff);

// ---------------------------------------------------------------- context --
struct orf_ctx_impl;

// Device blocks for job and group arenas, with a per-process cache: a
// released block is kept (up to kPoolKeep bytes in all) and handed to a later
// request of about its size, so repeated runs map no new device memory.
// Release waits for the device to be idle, as cudaFree does, so no kernel
// still reads a block that is handed out again.
constexpr size_t kPoolGrain = size_t(2) << 20;   // block sizes: multiples of 2 MiB
constexpr size_t kPoolKeep = size_t(8) << 30;    // cached bytes kept for reuse
int dev_alloc(size_t bytes, void** out);
void dev_free(void* p);
void dev_trim(int device);                        // cudaFree the cached blocks of a device

// Small mapped (zero-copy) host buffers -- a job's status ring and cancel
// flag -- carved from pinned pages that the process keeps: a pair of
// cudaHostAlloc / cudaFreeHost per job costs far more than the job's own
// set-up when a batch holds hundreds of instances, and cudaFreeHost waits
// for the device.  Slots are reused by later jobs, never unpinned; their
// contents are not cleared.  dev receives the slot's device address.
int host_mapped_alloc(size_t bytes, void** host, void** dev);
void host_mapped_free(void* host);

// Pinned host staging buffers for device-to-host result copies, kept by the
// process and reused: a copy into pinned memory runs at the link's speed,
// and the host thread then moves it into the caller's (pageable) buffer, so
// the several host threads finishing a batch copy in parallel.  Each buffer
// holds kStageBytes; a thread takes one for the duration of its results.
constexpr size_t kStageBytes = size_t(4) << 20;
int pinned_stage_acquire(void** buf);
void pinned_stage_release(void* buf);
// Device-to-host copy of `bytes` from `src` into the pageable `dst` through
// the staging buffer `stage`, on stream st (synchronises st).
int copy_d2h_staged(void* dst, const void* src, size_t bytes, void* stage, cudaStream_t st);

// Exact dense index of the distinct values of a list of rows, in the order
// of their first occurrence when the rows are scanned in order: dst[i] of a
// row is the index of src[i] in vals.  Inputs of a million values or more
// are scanned by up to 16 host threads (a table per thread, merged in row
// order, so the indices are those of one sequential scan).
struct IndexRow {
    const double* src;
    uint32_t* dst;
    int n;
};
void index_values(const std::vector<IndexRow>& rows, std::vector<double>& vals);

// Index of the first of the n values that is not positive and finite (n if
// there is none), scanned by up to 16 host threads for long arrays.
size_t first_bad_positive(const double* v, size_t n);

// fn(r0, r1) over rows [0, n) split into contiguous ranges, on up to 16
// host threads when the n rows of cells_per_row cells hold a million or more
void parallel_rows_n(int n, size_t cells_per_row, const std::function<void(int, int)>& fn);

// Bump allocator over one device block: a job's buffers come from one block.
struct Arena {
    std::vector<std::pair<void**, size_t>> req;
    void* base = nullptr;
    size_t total = 0;
    template <class T>
    void add(T** p, size_t n) {
        req.push_back({reinterpret_cast<void**>(p), n * sizeof(T)});
    }
    void add_bytes(void** p, size_t bytes) { req.push_back({p, bytes}); }   // an untyped block
    size_t bytes() const {
        size_t s = 0;
        for (auto& r : req) s += (r.second + 255) & ~size_t(255);
        return s;
    }
    int alloc() {
        total = bytes();
        if (total == 0) return ORF_OK;
        const int rc = dev_alloc(total, &base);
        if (rc != ORF_OK) return rc;
        char* p = static_cast<char*>(base);
        for (auto& r : req) {
            *r.first = p;
            p += (r.second + 255) & ~size_t(255);
        }
        return ORF_OK;
    }
    // Carve the requests from caller-provided device memory instead of
    // cudaMalloc (no allocation); fails with ORF_ETOOLARGE if they do not fit.
    int check_budget(size_t budget, size_t* need) const {
        *need = bytes();
        if (*need > budget) {
            set_error("run needs %.1f MB of device memory, above the %.1f MB left in the budget", *need / 1048576.0,
                      budget / 1048576.0);
            return ORF_ETOOLARGE;
        }
        return ORF_OK;
    }
    int place(void* ext, size_t cap) {
        total = bytes();
        if (total > cap) {
            set_error("run needs %.1f MB of device scratch, above the %.1f MB limit", total / 1048576.0,
                      cap / 1048576.0);
            return ORF_ETOOLARGE;
        }
        base = ext;
        owned = false;
        char* p = static_cast<char*>(base);
        for (auto& r : req) {
            *r.first = p;
            p += (r.second + 255) & ~size_t(255);
        }
        return ORF_OK;
    }
    bool owned = true;
    void release() {
        if (base && owned) dev_free(base);
        base = nullptr;
    }
};

}  // namespace orf

struct orf_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int sm_count = 148;
    orf_tuning tuning{};
    bool timing = false;
    orf_kernel_stats stats{};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // bounded device waits of the 3D kernel (orf_ctx_set_wait_injection):
    // limit per plane wait in ns (0: one second), test-hook stall plane (-1: off)
    unsigned long long wait_ns = 0;
    int stall_plane = -1;
    // references: the creator's, plus one per job or server built on the
    // context; the context is freed when the last one is released
    std::atomic<int> refs{1};
};

namespace orf {
inline WaitCtl wait_ctl(const orf_ctx* c) { return WaitCtl{c->wait_ns, c->stall_plane}; }
// host-to-device byte counter of a context, safe from several host threads
void add_h2d(orf_ctx* c, int64_t bytes);
void add_d2h(orf_ctx* c, int64_t bytes);
void ctx_retain(orf_ctx* c);
void ctx_release(orf_ctx* c);
}  // namespace orf

// A device-resident run (2D or 3D).  Implemented in job2d.cu / job3d.cu.
struct orf_job {
    virtual ~orf_job() = default;
    orf_ctx* ctx = nullptr;
    int dims = 2;
    // admission: create() fails with ORF_ETOOLARGE, before allocating, when
    // the job's device arena would exceed `budget`; `need` holds its size
    size_t budget = ~size_t(0);
    size_t need = 0;
    virtual int advance(int64_t nsteps, orf_progress_fn progress, void* user) = 0;
    virtual int64_t steps_done() = 0;
    virtual int64_t step_budget() const = 0;
    virtual int64_t cells() const = 0;
    virtual int reset() = 0;
    virtual int get_fields(double* const* f, int nf) = 0;
    virtual int finish2d(orf_out2d*) { return ORF_EINVAL; }
    virtual int finish3d(orf_out3d*) { return ORF_EINVAL; }
    // 3D: enqueue exactly nsteps steps without waiting (orf_job3d_step), and
    // the device address of plane k of a field in a buffer (orf_job3d_plane)
    virtual int step_async(int64_t) { return ORF_EINVAL; }
    virtual int plane_ptr(int, int, int, void**, size_t*) { return ORF_EINVAL; }
    // checkpoint / resume (checkpoint.cu): the device regions of field
    // buffer b holding the run's state (fields, CPML psi, then the DFT sums,
    // which have one copy), a key of the grid and run options, the device
    // state block, and the host bookkeeping after a restore
    virtual void state_regions(int b, std::vector<std::pair<void*, size_t>>& out) = 0;
    virtual uint64_t state_key() const = 0;
    virtual orf::JobState* state_dev() const = 0;
    virtual int64_t nmax_steps() const = 0;
    virtual void resume_host(const orf::JobState& js) = 0;
};

namespace orf {
// checkpoint / resume (checkpoint.cu); restore writes into field buffer `into`
int job_checkpoint_size(orf_job* job, size_t* bytes);
int job_checkpoint(orf_job* job, void* buf, size_t bytes);
int job_restore(orf_job* job, const void* buf, size_t bytes, int into);
// scan_eps = false: the caller validated the sim, permittivity included
int make_job2d(orf_ctx* ctx, const orf_sim2d* sim, orf_job** out, bool scan_eps = true);
int make_job3d(orf_ctx* ctx, const orf_sim3d* sim, orf_job** out, bool scan_eps = true);
// a z slab of a larger 3D grid: local plane 0 is global plane z_off of nz_glob
int make_job3d_slab(orf_ctx* ctx, const orf_sim3d* sim, int z_off, int nz_glob, orf_job** out);
int batch2d_run(orf_ctx* ctx, int n, const orf_sim2d* sims, orf_out2d* outs, orf_progress_fn progress,
                void* user);
// scan_eps = false skips the per-cell permittivity scan (for callers that
// ran it already: a job's create() after make_job*, batch or serve checks)
int validate2d(const orf_sim2d* s, bool scan_eps = true);
// slab: the z position of a z-normal source is checked by the caller
// against the global grid
int validate3d(const orf_sim3d* s, bool slab = false, bool scan_eps = true);
orf_ctx* default_ctx(int* status);
}  // namespace orf
