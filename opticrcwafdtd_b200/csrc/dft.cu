// dft.cu -- running DFT monitors, energy shutoff and flux for the FDTD engine.
//
// The step kernels write each monitor line's fields for every step of a
// chunk into a sample buffer; flush folds those kChunk samples into the
// running sums with kernel e^{+i w t} (fdtd2DTE.m:18) in one pass, so the
// accumulators are read and written once per chunk instead of once per step.
// FP64 runs accumulate in double; FP32 runs accumulate in float with Kahan
// compensation and use FP64 only for the phase w*t and its sine/cosine.
// check advances the step counter, applies the energy shutoff
// (fdtd2DTE.m:19-21) and publishes progress; flux reduces the DFT lines to
// 1/2 Re sum P conj(B) dx (fdtd2DTE.m:27-31, fdtd3D.m:26) with warp shuffles.
#include "orf_internal.cuh"

namespace orf {
namespace {

constexpr int kFlushThreads = 128;
constexpr int kFlushLambdas = 8;

template <class R>
struct AccT;
template <>
struct AccT<double> {
    using T = double2;
};
template <>
struct AccT<float> {
    using T = float4;   // sum re, sum im, Kahan c re, c im
};

__device__ __forceinline__ void acc_add(double2& a, double re, double im) {
    a.x += re;
    a.y += im;
}
__device__ __forceinline__ void kahan(float& sum, float& c, float v) {
    const float y = v - c;
    const float t = sum + y;
    c = (t - sum) - y;
    sum = t;
}
__device__ __forceinline__ void acc_add(float4& a, float re, float im) {
    kahan(a.x, a.z, re);
    kahan(a.y, a.w, im);
}

template <class R>
__global__ void __launch_bounds__(kFlushThreads)
k_flush(const DftStream* __restrict__ streams, const FlushItem* __restrict__ items, int nitems) {
    using Acc = typename AccT<R>::T;
    __shared__ R ph[kFlushLambdas][kChunk][2];
    __shared__ int s_count;
    __shared__ long long s_n0;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        __syncthreads();
        const FlushItem w = items[it];
        const DftStream& S = streams[w.stream];
        if (threadIdx.x == 0) {
            const JobState* st = S.st;
            int cnt = 0;
            if (!st->done) cnt = (int)min((long long)kChunk, st->nmax - st->step);
            s_count = cnt;
            s_n0 = st->step;
        }
        __syncthreads();
        const int count = s_count;
        if (count <= 0) continue;
        const long long n0 = s_n0;
        const double dt = S.st->S;
        const int nlg = min(kFlushLambdas, S.nl - w.l0);
        // phases of the chunk's steps; zero past the last step of a partial
        // chunk, since those slots are multiplied by zero samples below and
        // shared memory may hold any bit pattern (0 * NaN = NaN)
        for (int q = threadIdx.x; q < nlg * kChunk; q += blockDim.x) {
            const int l = q / kChunk, j = q % kChunk;
            R c = R(0), s = R(0);
            if (j < count) {
                const double t = ((double)(n0 + j) + (S.half ? 0.5 : 1.0)) * dt;
                double sn, cs;
                sincos(S.omega[w.l0 + l] * t, &sn, &cs);
                c = (R)(cs * dt);
                s = (R)(sn * dt);
            }
            ph[l][j][0] = c;
            ph[l][j][1] = s;
        }
        __syncthreads();
        const int e = w.e0 + threadIdx.x;
        if (e < S.len) {
            const R* smp = reinterpret_cast<const R*>(S.samples) + S.soff + e;
            R x[kChunk];
#pragma unroll
            for (int j = 0; j < kChunk; ++j) x[j] = j < count ? smp[(size_t)j * S.sstride] : R(0);
            Acc* acc = reinterpret_cast<Acc*>(S.acc);
            for (int l = 0; l < nlg; ++l) {
                R re = R(0), im = R(0);
#pragma unroll
                for (int j = 0; j < kChunk; ++j) {
                    re += x[j] * ph[l][j][0];
                    im += x[j] * ph[l][j][1];
                }
                Acc a = acc[(size_t)(w.l0 + l) * S.len + e];
                acc_add(a, re, im);
                acc[(size_t)(w.l0 + l) * S.len + e] = a;
            }
        }
    }
}

__global__ void k_check(JobState* const* __restrict__ states, int n) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    JobState* st = states[q];
    if (st->done) return;
    const long long n0 = st->step;
    const long long cnt = min((long long)kChunk, st->nmax - n0);
    const long long step = n0 + (cnt > 0 ? cnt : 0);
    st->step = step;
    const double e = st->energy;
    st->energy = 0.0;
    int done = 0, conv = 0;
    if (step % kChunk == 0 && cnt == kChunk) {
        st->peak = fmax(st->peak, e);
        const double t = (double)step * st->S;
        if (t > st->src_end && st->shutoff > 0.0 && e < st->shutoff * st->peak) {
            done = 1;
            conv = 1;
        }
    }
    if (step >= st->nmax) done = 1;
    if (st->cancel && *st->cancel) done = 1;
    if (st->fault) done = 1;   // a step kernel gave up a bounded wait
    if (done) st->done = 1;
    if (conv) st->converged = 1;
    const long long c = st->chunk;
    st->chunk = c + 1;
    if (st->ring) {
        volatile ChunkStatus* r = st->ring + (c % kStatusRing);
        r->step = step;
        r->energy = e;
        r->peak = st->peak;
        r->done = done;
        r->converged = conv;
        __threadfence_system();
        r->seq = c + 1;
        __threadfence_system();
    }
}

template <class R>
__device__ __forceinline__ double2 acc_value(const void* acc, size_t q) {
    if constexpr (sizeof(R) == 8) {
        return reinterpret_cast<const double2*>(acc)[q];
    } else {
        const float4 a = reinterpret_cast<const float4*>(acc)[q];
        return make_double2((double)a.x - (double)a.z, (double)a.y - (double)a.w);
    }
}

template <class R>
__global__ void __launch_bounds__(256)
k_flux(const DftStream* __restrict__ streams, const FluxPair* __restrict__ pairs, int nl, double* out) {
    const FluxPair p = pairs[blockIdx.x];
    const int l = blockIdx.y;
    if (l >= nl) return;
    const DftStream& a1 = streams[p.a1];
    const DftStream& b1 = streams[p.b1];
    double s = 0.0;
    for (int e = threadIdx.x; e < a1.len; e += blockDim.x) {
        const double2 x = acc_value<R>(a1.acc, (size_t)l * a1.len + e);
        const double2 y = acc_value<R>(b1.acc, (size_t)l * b1.len + e);
        s += x.x * y.x + x.y * y.y;
        if (p.a2 >= 0) {
            const DftStream& a2 = streams[p.a2];
            const DftStream& b2 = streams[p.b2];
            const double2 u = acc_value<R>(a2.acc, (size_t)l * a2.len + e);
            const double2 v = acc_value<R>(b2.acc, (size_t)l * b2.len + e);
            s -= u.x * v.x + u.y * v.y;
        }
    }
    __shared__ double red[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        out[p.out + (size_t)p.ostride * l] = p.scale * tot;
    }
}

template <class R>
__global__ void k_acc_to_complex(const void* __restrict__ acc, size_t n, double2* __restrict__ out) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        out[q] = acc_value<R>(acc, q);
}

}  // namespace

cudaError_t launch_flush(bool fp64, const DftStream* streams, const FlushItem* items, int nitems, cudaStream_t s) {
    if (nitems <= 0) return cudaSuccess;
    const int grid = nitems < 4096 ? nitems : 4096;
    if (fp64)
        k_flush<double><<<grid, kFlushThreads, 0, s>>>(streams, items, nitems);
    else
        k_flush<float><<<grid, kFlushThreads, 0, s>>>(streams, items, nitems);
    return cudaGetLastError();
}

cudaError_t launch_check(JobState* const* states, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_check<<<(n + 127) / 128, 128, 0, s>>>(states, n);
    return cudaGetLastError();
}

cudaError_t launch_flux(bool fp64, const DftStream* streams, const FluxPair* pairs, int npairs, int nl,
                        double* out, cudaStream_t s) {
    if (npairs <= 0 || nl <= 0) return cudaSuccess;
    dim3 grid(npairs, nl);
    if (fp64)
        k_flux<double><<<grid, 256, 0, s>>>(streams, pairs, nl, out);
    else
        k_flux<float><<<grid, 256, 0, s>>>(streams, pairs, nl, out);
    return cudaGetLastError();
}

cudaError_t launch_acc_to_complex(bool fp64, const void* acc, size_t n, double2* out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const int grid = (int)((n + 255) / 256 < 2048 ? (n + 255) / 256 : 2048);
    if (fp64)
        k_acc_to_complex<double><<<grid, 256, 0, s>>>(acc, n, out);
    else
        k_acc_to_complex<float><<<grid, 256, 0, s>>>(acc, n, out);
    return cudaGetLastError();
}

}  // namespace orf
