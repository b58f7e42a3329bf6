// runtime.cu -- errors, shared physics definitions, context, chunk engine.
#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <cfloat>
#include <thread>
#include <unordered_map>

#include "engine.cuh"

namespace orf {

namespace {
thread_local std::string g_err;
std::mutex g_stats_mu;
}

void add_h2d(orf_ctx* c, int64_t bytes) {
    std::lock_guard<std::mutex> g(g_stats_mu);
    c->stats.h2d_bytes += bytes;
}

void add_d2h(orf_ctx* c, int64_t bytes) {
    std::lock_guard<std::mutex> g(g_stats_mu);
    c->stats.d2h_bytes += bytes;
}

namespace {
struct DevPool {
    std::mutex mu;
    std::multimap<size_t, void*> idle;                           // cached blocks by size
    std::unordered_map<void*, std::pair<size_t, int>> blocks;    // every pool block: size, device
    size_t idle_bytes = 0;
};
DevPool& dev_pool() {
    static DevPool* p = new DevPool;   // never destroyed: blocks may be released during exit
    return *p;
}
}  // namespace

int dev_alloc(size_t bytes, void** out) {
    *out = nullptr;
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t want = (bytes + kPoolGrain - 1) / kPoolGrain * kPoolGrain;
    DevPool& P = dev_pool();
    {
        std::lock_guard<std::mutex> g(P.mu);
        // the smallest cached block of this device that fits, wasting at most a quarter
        for (auto it = P.idle.lower_bound(want); it != P.idle.end() && it->first <= want + want / 4 + kPoolGrain;
             ++it) {
            if (P.blocks[it->second].second != dev) continue;
            *out = it->second;
            P.idle_bytes -= it->first;
            P.idle.erase(it);
            return ORF_OK;
        }
    }
    cudaError_t e = cudaMalloc(out, want);
    if (e == cudaErrorMemoryAllocation) {   // give the cached blocks back and retry once
        cudaGetLastError();
        dev_trim(dev);
        e = cudaMalloc(out, want);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        set_error("device allocation of %.3f GB failed: %s", want / 1e9, cudaGetErrorString(e));
        return ORF_ENOMEM_DEVICE;
    }
    std::lock_guard<std::mutex> g(P.mu);
    P.blocks[*out] = {want, dev};
    return ORF_OK;
}

void dev_free(void* p) {
    if (!p) return;
    DevPool& P = dev_pool();
    size_t size = 0;
    int bdev = 0;
    {
        std::lock_guard<std::mutex> g(P.mu);
        auto it = P.blocks.find(p);
        if (it == P.blocks.end()) return;
        size = it->second.first;
        bdev = it->second.second;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != bdev) cudaSetDevice(bdev);
    const cudaError_t e = cudaDeviceSynchronize();
    std::vector<void*> evict;
    {
        std::lock_guard<std::mutex> g(P.mu);
        if (e != cudaSuccess) {   // a failed context: do not keep its memory
            P.blocks.erase(p);
            evict.push_back(p);
        } else {
            P.idle.insert({size, p});
            P.idle_bytes += size;
            while (P.idle_bytes > kPoolKeep) {   // drop the largest cached blocks
                auto last = std::prev(P.idle.end());
                P.idle_bytes -= last->first;
                evict.push_back(last->second);
                P.blocks.erase(last->second);
                P.idle.erase(last);
            }
        }
    }
    for (void* q : evict) cudaFree(q);
    if (cur != bdev) cudaSetDevice(cur);
}

void dev_trim(int device) {
    DevPool& P = dev_pool();
    std::vector<void*> evict;
    {
        std::lock_guard<std::mutex> g(P.mu);
        for (auto it = P.idle.begin(); it != P.idle.end();) {
            if (P.blocks[it->second].second == device) {
                P.idle_bytes -= it->first;
                evict.push_back(it->second);
                P.blocks.erase(it->second);
                it = P.idle.erase(it);
            } else {
                ++it;
            }
        }
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (!evict.empty() && cur != device) cudaSetDevice(device);
    for (void* q : evict) cudaFree(q);
    if (!evict.empty() && cur != device) cudaSetDevice(cur);
}

namespace {
constexpr size_t kHostSlab = size_t(1) << 20;   // pinned bytes per cudaHostAlloc
constexpr int kHostClasses = 9;                 // slot sizes 256 B .. 64 KiB (powers of two)
struct HostPool {
    std::mutex mu;
    std::vector<void*> idle[kHostClasses];
    std::unordered_map<void*, int> cls;         // every slot handed out: its size class
    char* cur = nullptr;                        // unused tail of the newest slab
    size_t left = 0;
};
HostPool& host_pool() {
    static HostPool* p = new HostPool;   // never destroyed: slots may be released during exit
    return *p;
}
}  // namespace

int host_mapped_alloc(size_t bytes, void** host, void** dev) {
    *host = *dev = nullptr;
    int c = 0;
    while (c < kHostClasses && (size_t(256) << c) < bytes) ++c;
    if (c == kHostClasses) {
        set_error("mapped host buffer of %zu bytes above the slot limit", bytes);
        return ORF_EINVAL;
    }
    const size_t sz = size_t(256) << c;
    HostPool& P = host_pool();
    void* h = nullptr;
    {
        std::lock_guard<std::mutex> g(P.mu);
        if (!P.idle[c].empty()) {
            h = P.idle[c].back();
            P.idle[c].pop_back();
        } else {
            if (P.left < sz) {   // a new slab; the old tail stays unused
                void* s = nullptr;
                const cudaError_t e = cudaHostAlloc(&s, kHostSlab, cudaHostAllocMapped | cudaHostAllocPortable);
                if (e != cudaSuccess) {
                    cudaGetLastError();
                    set_error("pinned host allocation failed: %s", cudaGetErrorString(e));
                    return ORF_ECUDA;
                }
                P.cur = static_cast<char*>(s);
                P.left = kHostSlab;
            }
            h = P.cur;   // every slot starts on a 256-byte boundary
            P.cur += sz;
            P.left -= sz;
        }
        P.cls[h] = c;
    }
    const cudaError_t e = cudaHostGetDevicePointer(dev, h, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        host_mapped_free(h);
        *dev = nullptr;
        set_error("no device address for a mapped host buffer: %s", cudaGetErrorString(e));
        return ORF_ECUDA;
    }
    *host = h;
    return ORF_OK;
}

void host_mapped_free(void* host) {
    if (!host) return;
    HostPool& P = host_pool();
    std::lock_guard<std::mutex> g(P.mu);
    auto it = P.cls.find(host);
    if (it == P.cls.end()) return;
    P.idle[it->second].push_back(host);
    P.cls.erase(it);
}

namespace {
struct StagePool {
    std::mutex mu;
    std::vector<void*> idle;
};
StagePool& stage_pool() {
    static StagePool* p = new StagePool;   // never destroyed: buffers may be released during exit
    return *p;
}
}  // namespace

int pinned_stage_acquire(void** buf) {
    *buf = nullptr;
    StagePool& P = stage_pool();
    {
        std::lock_guard<std::mutex> g(P.mu);
        if (!P.idle.empty()) {
            *buf = P.idle.back();
            P.idle.pop_back();
            return ORF_OK;
        }
    }
    const cudaError_t e = cudaHostAlloc(buf, kStageBytes, cudaHostAllocPortable);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *buf = nullptr;
        set_error("pinned staging buffer: %s", cudaGetErrorString(e));
        return ORF_ECUDA;
    }
    return ORF_OK;
}

void pinned_stage_release(void* buf) {
    if (!buf) return;
    StagePool& P = stage_pool();
    std::lock_guard<std::mutex> g(P.mu);
    P.idle.push_back(buf);
}

int copy_d2h_staged(void* dst, const void* src, size_t bytes, void* stage, cudaStream_t st) {
    char* d = static_cast<char*>(dst);
    const char* s = static_cast<const char*>(src);
    for (size_t off = 0; off < bytes; off += kStageBytes) {
        const size_t n = std::min(kStageBytes, bytes - off);
        ORF_CUDA(cudaMemcpyAsync(stage, s + off, n, cudaMemcpyDeviceToHost, st));
        ORF_CUDA(cudaStreamSynchronize(st));
        std::memcpy(d + off, stage, n);
    }
    return ORF_OK;
}

namespace {
// one table: distinct values in first-occurrence order, with the last value
// remembered (neighbouring cells mostly share a material)
struct ValueTable {
    std::unordered_map<uint64_t, uint32_t> map;
    std::vector<double> vals;
    uint64_t last_key = ~uint64_t(0);
    uint32_t last_id = 0;
    uint32_t get(double v) {
        uint64_t key;
        std::memcpy(&key, &v, 8);
        if (key == last_key) return last_id;
        auto it = map.find(key);
        uint32_t id;
        if (it != map.end()) {
            id = it->second;
        } else {
            id = (uint32_t)vals.size();
            map.emplace(key, id);
            vals.push_back(v);
        }
        last_key = key;
        last_id = id;
        return id;
    }
};
}  // namespace

void index_values(const std::vector<IndexRow>& rows, std::vector<double>& vals) {
    size_t total = 0;
    for (const auto& r : rows) total += (size_t)r.n;
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int T = total >= (size_t(1) << 20) ? std::min(16, hw) : 1;
    // rows [cut[t], cut[t+1]) to thread t, about equal cells each
    std::vector<size_t> cut(T + 1, rows.size());
    cut[0] = 0;
    {
        size_t acc = 0;
        int t = 1;
        for (size_t q = 0; q < rows.size() && t < T; ++q) {
            acc += (size_t)rows[q].n;
            while (t < T && acc * T >= total * (size_t)t) cut[t++] = q + 1;
        }
    }
    std::vector<ValueTable> loc(T);
    auto scan = [&](int t) {
        for (size_t q = cut[t]; q < cut[t + 1]; ++q) {
            const IndexRow& r = rows[q];
            for (int i = 0; i < r.n; ++i) r.dst[i] = loc[t].get(r.src[i]);
        }
    };
    if (T == 1) {
        scan(0);
        vals = std::move(loc[0].vals);
        return;
    }
    {
        std::vector<std::thread> pool;
        for (int t = 0; t < T; ++t) pool.emplace_back(scan, t);
        for (auto& th : pool) th.join();
    }
    // the tables in row order: the global first occurrences
    ValueTable glob;
    std::vector<std::vector<uint32_t>> remap(T);
    for (int t = 0; t < T; ++t) {
        remap[t].resize(loc[t].vals.size());
        for (size_t l = 0; l < loc[t].vals.size(); ++l) remap[t][l] = glob.get(loc[t].vals[l]);
    }
    auto apply = [&](int t) {
        const uint32_t* m = remap[t].data();
        for (size_t q = cut[t]; q < cut[t + 1]; ++q) {
            const IndexRow& r = rows[q];
            for (int i = 0; i < r.n; ++i) r.dst[i] = m[r.dst[i]];
        }
    };
    {
        std::vector<std::thread> pool;
        for (int t = 0; t < T; ++t) pool.emplace_back(apply, t);
        for (auto& th : pool) th.join();
    }
    vals = std::move(glob.vals);
}

void parallel_rows_n(int n, size_t cells_per_row, const std::function<void(int, int)>& fn) {
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int T = (size_t)n * cells_per_row >= (size_t(1) << 20) ? std::min({16, hw, n}) : 1;
    if (T <= 1) {
        if (n > 0) fn(0, n);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < T; ++t) {
        const int a = (int)((int64_t)n * t / T), b = (int)((int64_t)n * (t + 1) / T);
        pool.emplace_back([&fn, a, b] { fn(a, b); });
    }
    for (auto& th : pool) th.join();
}

size_t first_bad_positive(const double* v, size_t n) {
    // blocks of 4096 values: a branch-free test of the whole block (positive
    // and at most the largest finite double: NaN fails both), then the exact
    // position inside the first block that fails
    constexpr size_t kBlock = 4096;
    const size_t nb = (n + kBlock - 1) / kBlock;
    std::atomic<size_t> bad{n};
    parallel_rows_n((int)nb, kBlock, [&](int b0, int b1) {
        for (int b = b0; b < b1; ++b) {
            const size_t a = (size_t)b * kBlock, e = std::min(n, a + kBlock);
            if (a >= bad.load(std::memory_order_relaxed)) return;
            bool ok = true;
            for (size_t q = a; q < e; ++q) ok &= (v[q] > 0.0) & (v[q] <= DBL_MAX);
            if (ok) continue;
            for (size_t q = a; q < e; ++q)
                if (!(v[q] > 0.0 && v[q] <= DBL_MAX)) {
                    size_t cur = bad.load();
                    while (q < cur && !bad.compare_exchange_weak(cur, q)) {
                    }
                    return;   // the rest of this range lies after q
                }
        }
    });
    return bad.load();
}

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
}
const char* last_error() { return g_err.c_str(); }

void pml_profile(int n, int npts, int npml, double off, double dx, double S, double alpha_max,
                 std::vector<double>& bak, int* nslab) {
    bak.assign((size_t)3 * npts, 0.0);
    int ns = 0;
    for (int i = 0; i < npts; ++i) {
        bak[3 * i] = 1.0;
        bak[3 * i + 1] = 0.0;
        bak[3 * i + 2] = 1.0;
        if (npml <= 0) continue;
        const double u = i + off;
        const double lo = npml, hi = (n - 1) - npml;
        double depth = 0.0;
        if (u < lo) depth = lo - u;
        else if (u > hi) depth = u - hi;
        if (depth <= 0.0) continue;
        const double m = kPmlOrder;
        const double sigma_max = 0.8 * (m + 1.0) / dx;
        const double r = std::min(depth / npml, 1.0);
        const double rm = std::pow(r, m);
        const double sigma = sigma_max * rm;
        const double kappa = 1.0 + (kPmlKappaMax - 1.0) * rm;
        const double alpha = alpha_max * (1.0 - r);
        const double b = std::exp(-(sigma / kappa + alpha) * S);
        const double den = sigma * kappa + kappa * kappa * alpha;
        bak[3 * i] = b;
        bak[3 * i + 1] = den > 0.0 ? sigma / den * (b - 1.0) : 0.0;
        bak[3 * i + 2] = 1.0 / kappa;
        ++ns;
    }
    if (nslab) *nslab = ns;
}

int64_t max_steps(double max_time, double S) {
    const double r = max_time / S;
    if (!(r < 4e18)) return (int64_t)4e18;   // effectively unbounded, no overflow
    const int64_t n = (int64_t)std::ceil(r - 1e-9);
    return n < 0 ? 0 : n;
}

// fdtdProgress.m:6-12
double progress_fraction(double t, double src_end, double ratio, double shutoff) {
    double frac;
    if (t <= src_end) {
        frac = 0.3 * t / src_end;
    } else {
        const double so = shutoff > 0.0 ? shutoff : 1e-300;
        const double decay = std::log(std::max(ratio, so)) / std::log(so);
        frac = 0.3 + 0.7 * std::max(0.0, std::min(1.0, decay));
    }
    return std::max(0.0, std::min(1.0, frac));
}

// ----------------------------------------------------------- ChunkEngine --
KernelTimer::~KernelTimer() {
    for (auto e : pool) cudaEventDestroy(e);
}

int KernelTimer::begin(cudaStream_t s, cudaEvent_t* a) {
    if (used >= pool.size()) {
        cudaEvent_t e;
        ORF_CUDA(cudaEventCreate(&e));
        pool.push_back(e);
    }
    *a = pool[used++];
    ORF_CUDA(cudaEventRecord(*a, s));
    return ORF_OK;
}

int KernelTimer::end(cudaStream_t s, int kind, int64_t cells, cudaEvent_t a) {
    if (used >= pool.size()) {
        cudaEvent_t e;
        ORF_CUDA(cudaEventCreate(&e));
        pool.push_back(e);
    }
    cudaEvent_t b = pool[used++];
    ORF_CUDA(cudaEventRecord(b, s));
    recs.push_back({kind, cells, a, b});
    return ORF_OK;
}

void KernelTimer::collect(orf_kernel_stats* st) {
    for (auto& r : recs) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess) continue;
        if (r.kind == 0) {
            st->interior_ms += ms;
            st->interior_launches += 1;
            st->interior_cell_updates += r.cells;
        } else if (r.kind == 1) {
            st->frame_ms += ms;
            st->frame_launches += 1;
            st->frame_cell_updates += r.cells;
        } else {
            st->flush_ms += ms;
            st->flush_launches += 2;
        }
    }
    cudaGetLastError();
    recs.clear();
    used = 0;
}

ChunkEngine::~ChunkEngine() { drop_graph(); }

void ChunkEngine::drop_graph() {
    if (gexec) cudaGraphExecDestroy(gexec);
    gexec = nullptr;
    gchunks = 0;
    gpar = -1;
}

int ChunkEngine::enqueue_chunk(cudaStream_t s, bool timed) {
    KernelTimer* tm = timed ? &timer : nullptr;
    for (int off = 0; off < kChunk; off += T) {
        const int nsub = std::min(T, kChunk - off);
        const int we = (off + nsub == kChunk) ? 1 : 0;
        ORF_CUDA(step(off, nsub, par, we, s, tm));
        par ^= 1;
    }
    cudaEvent_t a = nullptr;
    if (tm) ORF_TRY(tm->begin(s, &a));
    ORF_CUDA(launch_flush(fp64, d_streams, d_items, nitems, s));
    ORF_CUDA(launch_check(d_states, nstates, s));
    if (tm) ORF_TRY(tm->end(s, 2, 0, a));
    return ORF_OK;
}

int ChunkEngine::enqueue(int nchunks, cudaStream_t s) {
    const bool timed = ctx->timing;
    const bool use_graph = ctx->tuning.use_graph != 0 && !timed;
    const int lpc = launches_per_chunk();
    // graph of G chunks with an even launch count, so the buffer parity is
    // the same before and after every replay
    const int G = (lpc & 1) ? 8 : 4;
    while (nchunks > 0) {
        if (use_graph && nchunks >= G) {
            if (!gexec || gpar != par || gchunks != G) {
                drop_graph();
                const int p0 = par;
                cudaGraph_t g = nullptr;
                ORF_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                int st = ORF_OK;
                for (int c = 0; c < G && st == ORF_OK; ++c) st = enqueue_chunk(s, false);
                cudaError_t ce = cudaStreamEndCapture(s, &g);
                par = p0;   // capture only recorded the launches
                if (st != ORF_OK) {
                    if (g) cudaGraphDestroy(g);
                    return st;
                }
                ORF_CUDA(ce);
                cudaError_t ie = cudaGraphInstantiate(&gexec, g, 0);
                cudaGraphDestroy(g);
                ORF_CUDA(ie);
                gpar = p0;
                gchunks = G;
            }
            ORF_CUDA(cudaGraphLaunch(gexec, s));
            par ^= (G * lpc) & 1;
            nchunks -= G;
        } else {
            ORF_TRY(enqueue_chunk(s, timed));
            nchunks -= 1;
        }
    }
    return ORF_OK;
}

void ChunkEngine::collect_timing() {
    if (!ctx->timing) return;
    timer.collect(&ctx->stats);
}

// ---------------------------------------------------------- ProgressLoop --
int ProgressLoop::poll(orf_progress_fn progress, void* user) {
    if (!ring) return ORF_OK;
    for (;;) {
        const volatile ChunkStatus* r = ring + (seen % kStatusRing);
        const long long seq = r->seq;
        if (seq != seen + 1) break;
        std::atomic_thread_fence(std::memory_order_acquire);
        const long long step = r->step;
        const double e = r->energy, pk = r->peak;
        const int dn = r->done;
        ++seen;
        last_step = step;
        if (progress && !done) {
            const double t = step * S;
            const double ratio = pk > 0.0 ? e / pk : 1.0;
            const double fr = r->converged ? 1.0 : progress_fraction(t, src_end, ratio, shutoff);
            char msg[96];
            std::snprintf(msg, sizeof msg, "step %lld, t = %.3g um", step, t);
            if (progress(fr, msg, user)) {
                if (cancel) *cancel = 1;
                done = true;
                cancelled = true;
                return ORF_ECANCELLED;
            }
        }
        if (dn) {
            done = true;
            break;
        }
    }
    return ORF_OK;
}

int run_chunks(ChunkEngine& eng, ProgressLoop& pl, orf_ctx* ctx, int64_t chunks, orf_progress_fn progress,
               void* user) {
    cudaStream_t st = ctx->stream;
    constexpr int kBatch = 8, kInFlight = 4;
    std::vector<cudaEvent_t> evs;
    int64_t enq = 0;
    size_t head = 0;
    int rc = ORF_OK;
    while (!pl.done) {
        while (enq < chunks && evs.size() - head < (size_t)kInFlight && !pl.done) {
            const int n = (int)std::min<int64_t>(kBatch, chunks - enq);
            ORF_TRY(eng.enqueue(n, st));
            enq += n;
            cudaEvent_t e;
            ORF_CUDA(cudaEventCreateWithFlags(&e, cudaEventBlockingSync | cudaEventDisableTiming));
            ORF_CUDA(cudaEventRecord(e, st));
            evs.push_back(e);
        }
        if (head < evs.size()) {
            ORF_CUDA(cudaEventSynchronize(evs[head]));
            ++head;
        }
        rc = pl.poll(progress, user);
        if (rc != ORF_OK) break;
        if (head == evs.size() && enq >= chunks) break;
    }
    cudaError_t e = cudaStreamSynchronize(st);
    for (auto ev : evs) cudaEventDestroy(ev);
    ORF_CUDA(e);
    if (rc == ORF_OK) rc = pl.poll(progress, user);
    return rc == ORF_ECANCELLED ? ORF_OK : rc;
}

}  // namespace orf
