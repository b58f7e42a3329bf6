// noalloc.cu -- orf_fdtd2d_run_noalloc: a 2D run that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the moment they want a run: a host
// whose device memory is handed out by its own pool (a MATLAB gpuArray
// session, a serving process with a fixed memory budget), a real-time loop
// that may not block on the allocator, or code that must not grow the
// process's device footprint after start-up.  This entry point runs the same
// kernels as orf_fdtd2d_run, but every device buffer of the run (fields and
// their ping-pong copies, CPML state, material index and tables, DFT samples
// and sums, flux) is carved from one file-scope static __device__ array of
// kNoAllocBytes.  The driver reserves that array on a GPU when this file's
// module is loaded there, and it stays reserved until the process exits.
//
// Set-up: the first call on a device, with that device current, looks up the
// array's device address with cudaGetSymbolAddress (host code cannot use the
// symbol itself: on the host it names a stand-in, not device memory).  CUDA
// loads modules lazily, so that first call is also the one that loads this
// module (reserving the array) and the 2D kernels (their code), on that
// device: make it at start-up, a small run is enough, before the device's
// memory is handed to the caller's pool and before any stream capture.  Later
// calls take no device memory at all.
//
// Limits and sharing: a run whose state exceeds kNoAllocBytes is rejected
// with ORF_ETOOLARGE before any device work.  Every call shares the one
// array, so calls that overlap on the GPU (from several threads or streams)
// race and corrupt each other; each call zeroes the part it uses first, so
// consecutive calls do not see each other's data.  There is no progress
// callback and no CUDA graph: chunks are launched directly on `stream`
// (cudaStreamPerThread when NULL) and the call returns when the run is done.
#include <mutex>

#include "job2d.cuh"

namespace orf {
namespace {

constexpr size_t kNoAllocBytes = (size_t)64 << 20;   // 64 MiB per device

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_addr_mu;
void* g_addr[64] = {nullptr};

// Device address of the scratch array on the current device (set-up on the
// first call per device).
int scratch_address(int dev, void** out) {
    if (dev < 0 || dev >= 64) {
        set_error("device %d out of range", dev);
        return ORF_ENODEV;
    }
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            set_error("cudaGetSymbolAddress of the no-allocation scratch array failed: %s", cudaGetErrorString(e));
            return ORF_ECUDA;
        }
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return ORF_OK;
}

template <class R>
int run_noalloc(const orf_sim2d* sim, orf_out2d* out, cudaStream_t stream, int dev) {
    void* base = nullptr;
    ORF_TRY(scratch_address(dev, &base));
    orf_ctx ctx;   // lives on the host stack: no stream or event is created
    ctx.device = dev;
    ctx.stream = stream;
    ctx.own_stream = false;
    cudaDeviceGetAttribute(&ctx.sm_count, cudaDevAttrMultiProcessorCount, dev);
    ctx.tuning = orf_tuning{};
    ctx.tuning.use_graph = 0;
    ctx.timing = false;
    const double t0 = now_s();
    int rc;
    {
        Job2D<R> job;
        job.ctx = &ctx;
        job.ext_base = base;
        job.ext_cap = kNoAllocBytes;
        rc = job.create(sim);
        if (rc == ORF_OK) rc = job.advance_all_direct();
        if (rc == ORF_OK) rc = job.finish2d(out);
    }
    if (rc == ORF_OK) out->wall_time = now_s() - t0;
    return rc;
}

}  // namespace
}  // namespace orf

using namespace orf;

extern "C" int32_t orf_fdtd2d_run_noalloc(const orf_sim2d* sim, orf_out2d* out, void* stream) {
    if (!out) {
        set_error("out is NULL");
        return ORF_EINVAL;
    }
    ORF_TRY(validate2d(sim));
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || orf_device_count() <= 0) {
        cudaGetLastError();
        set_error("no CUDA device available");
        return ORF_ENODEV;
    }
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : cudaStreamPerThread;
    // the scratch address is the current device's: the stream must be on it
    int sdev = dev;
    e = cudaStreamGetDevice(s, &sdev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaStreamGetDevice: %s", cudaGetErrorString(e));
        return ORF_EINVAL;
    }
    if (sdev != dev) {
        set_error("stream belongs to device %d but the current device is %d", sdev, dev);
        return ORF_EINVAL;
    }
    if (sim->precision == ORF_SINGLE) return run_noalloc<float>(sim, out, s, dev);
    return run_noalloc<double>(sim, out, s, dev);
}
