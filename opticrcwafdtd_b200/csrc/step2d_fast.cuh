// step2d_fast.cuh -- pipelined interior 2D Yee step kernel for sm_100a.
//
// Same update as step2d_impl.cuh (toolbox/+orf/fdtd2D.m:3-7 P/A/B form, with
// the TF/SF corrections and DFT sampling of fdtd2DTE.m:11-18), for tiles whose
// whole dependency cone lies outside the CPML and inside the grid ("interior"
// tiles): no psi state and no boundary masks.
//
// Persistent CTA, software-pipelined over its tiles:
//   wait for tile t in shared memory -> move it to registers (fields) and to
//   a coefficient plane (material index -> C/eps through the table) ->
//   issue the cp.async prefetch of tile t+1 into the same shared buffer ->
//   run the T fused time steps of tile t from registers -> store its output.
// The prefetch of tile t+1 and the descriptor/state loads of tile t+2 are in
// flight while tile t computes, so the DRAM latency that bounded the simple
// kernel is hidden behind the stencil arithmetic.
#pragma once
#include "orf_internal.cuh"

namespace orf {
namespace fast {

__device__ __forceinline__ int pmod(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

__device__ __forceinline__ void cp_async4(void* sdst, const void* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async8(void* sdst, const void* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <class R>
__device__ __forceinline__ void cp_field(R* sdst, const R* gsrc) {
    if constexpr (sizeof(R) == 4) cp_async4(sdst, gsrc);
    else cp_async8(sdst, gsrc);
}

// Dynamic shared memory of one instantiation: prefetch planes of P, A, B and
// the material index (one or two), then the coefficient planes.
template <class R, class IT, bool TE, int KS, int WX, int WZ>
constexpr size_t dyn_smem() {
    constexpr size_t cells = (size_t)32 * WX * KS * WZ;
    constexpr size_t idxb = ((cells * sizeof(IT) * (TE ? 1 : 2)) + 15) & ~size_t(15);
    return cells * sizeof(R) * 3 + idxb + cells * sizeof(R) * (TE ? 1 : 2);
}

template <class R, class IT, bool TE, int KS, int WX, int WZ>
__global__ void __launch_bounds__(32 * WX * WZ, 1)
k_step2d_fast(const FastTile2D* __restrict__ tiles, int ntiles, int launch_off, int nsub_max, int par,
              int want_energy) {
    constexpr int NW = WX * WZ;
    constexpr int NT = 32 * NW;
    constexpr int LX = 32 * WX;
    constexpr int LZ = KS * WZ;
    constexpr int CELLS = LX * LZ;
    constexpr unsigned FULL = 0xffffffffu;
    constexpr int NIDX = TE ? 1 : 2;

    extern __shared__ __align__(16) unsigned char dsm[];
    R* pfP = reinterpret_cast<R*>(dsm);
    R* pfA = pfP + CELLS;
    R* pfB = pfA + CELLS;
    IT* pfI = reinterpret_cast<IT*>(pfB + CELLS);     // NIDX planes
    constexpr size_t idxb = ((CELLS * sizeof(IT) * NIDX) + 15) & ~size_t(15);
    R* c0s = reinterpret_cast<R*>(reinterpret_cast<unsigned char*>(pfI) + idxb);
    R* c1s = c0s + CELLS;                                // TM only

    __shared__ R xPc[NW][KS];
    __shared__ R xPr[NW][32];
    __shared__ R xBc[NW][KS];
    __shared__ R xAr[NW][32];
    __shared__ R slut[256];
    __shared__ const R* s_lutsrc;
    __shared__ double sg[2][kMaxSub];
    __shared__ double sred[NW];
    // descriptor ring (tiles t, t+G, t+2G) and snapshots of their job state,
    // both filled by cp.async so no thread waits on a dependent global load
    __shared__ __align__(16) FastTile2D s_desc[3];
    __shared__ __align__(16) long long s_state[3][4];   // step, nmax, chunk, (done | converged << 32)

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wx = warp % WX;
    const int wz = warp / WX;
    const int cx = 32 * wx + lane;
    const int ck0 = KS * wz;

    // ---- prefetch one tile's fields and material index into the shared buffer
    auto prefetch = [&](const FastTile2D& d) {
        const R* gP = reinterpret_cast<const R*>(d.f[par][0]);
        const R* gA = reinterpret_cast<const R*>(d.f[par][1]);
        const R* gB = reinterpret_cast<const R*>(d.f[par][2]);
        const int col = min(d.li0 + cx, d.pitch - 1);
#pragma unroll
        for (int j = 0; j < KS; ++j) {
            const int row = d.lk0 + ck0 + j;
            const int kk = d.periodic ? pmod(row, d.nz) : min(max(row, 0), d.nz - 1);
            const size_t off = (size_t)kk * d.pitch + col;
            const int c = (ck0 + j) * LX + cx;
            cp_field(pfP + c, gP + off);
            cp_field(pfA + c, gA + off);
            cp_field(pfB + c, gB + off);
        }
        // material index rows: 4-byte copies (li0 and pitch are multiples of 4 cells)
        constexpr int W4 = LX * (int)sizeof(IT) / 4;
        for (int q = threadIdx.x; q < NIDX * LZ * W4; q += NT) {
            const int plane = q / (LZ * W4);
            const int r = (q / W4) % LZ;
            const int c4 = q % W4;
            const int row = d.lk0 + r;
            const int kk = d.periodic ? pmod(row, d.nz) : min(max(row, 0), d.nz - 1);
            size_t boff = ((size_t)kk * d.pitch + d.li0) * sizeof(IT) + 4 * (size_t)c4;
            const size_t rowend = ((size_t)kk * d.pitch + d.pitch) * sizeof(IT);
            if (boff + 4 > rowend) boff = rowend - 4;
            const unsigned char* src = reinterpret_cast<const unsigned char*>(plane ? d.idx1 : d.idx0) + boff;
            cp_async4(reinterpret_cast<unsigned char*>(pfI) + (size_t)plane * CELLS * sizeof(IT) +
                          ((size_t)r * LX) * sizeof(IT) + 4 * (size_t)c4,
                      src);
        }
    };
    auto fetch_desc = [&](int tile, int slot) {   // threads 0..7: 8 x 16 B
        if (threadIdx.x < 8 && tile < ntiles) {
            const unsigned s = (unsigned)__cvta_generic_to_shared(reinterpret_cast<char*>(&s_desc[slot]) + 16 * threadIdx.x);
            const char* g = reinterpret_cast<const char*>(tiles + tile) + 16 * threadIdx.x;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(g) : "memory");
        }
    };
    auto fetch_state = [&](int slot) {            // threads 8..9: 2 x 16 B of JobState
        if (threadIdx.x >= 8 && threadIdx.x < 10) {
            const int q = threadIdx.x - 8;
            const unsigned s = (unsigned)__cvta_generic_to_shared(reinterpret_cast<char*>(&s_state[slot][0]) + 16 * q);
            const char* g = reinterpret_cast<const char*>(s_desc[slot].st) + 16 * q;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(g) : "memory");
        }
    };

    int t = blockIdx.x;
    if (t >= ntiles) return;
    if (threadIdx.x == 0) s_lutsrc = nullptr;
    // prologue: descriptor and state of the first tile, then its prefetch
    fetch_desc(t, 0);
    cp_commit();
    cp_wait_all();
    __syncthreads();
    fetch_state(0);
    cp_commit();
    cp_wait_all();
    __syncthreads();
    prefetch(s_desc[0]);
    fetch_desc(t + gridDim.x, 1);
    cp_commit();
    int it = 0;

    while (t < ntiles) {
        const int cs = it % 3, ns = (it + 1) % 3, nns = (it + 2) % 3;
        const int tn = t + gridDim.x;
        cp_wait_all();
        __syncthreads();   // tile t in shared memory, descriptor of tile tn and state of tile t landed
        const FastTile2D& d = s_desc[cs];
        int nsub = 0;
        {
            const long long step0 = s_state[cs][0], nmax = s_state[cs][1];
            const int done = (int)(s_state[cs][3] & 0xffffffffLL);
            if (!done) nsub = (int)max(0LL, min((long long)nsub_max, nmax - (step0 + launch_off)));
        }
        const long long n0 = s_state[cs][0] + launch_off;
        const Inst2D<R>* I = reinterpret_cast<const Inst2D<R>*>(d.inst);
        const R C = I->C;
        // coefficient table for uint8 indices (reloaded when the instance changes)
        if (sizeof(IT) == 1 && s_lutsrc != I->lutc) {
            __syncthreads();
            for (int q = threadIdx.x; q < 256; q += NT) slut[q] = I->lutc[q];
            __syncthreads();
            if (threadIdx.x == 0) s_lutsrc = I->lutc;
        }
        for (int q = threadIdx.x; q < nsub; q += NT) {
            const long long n = n0 + q;
            sg[0][q] = n < I->nsrc ? I->gE[n] : 0.0;
            sg[1][q] = n < I->nsrc ? I->gH[n] : 0.0;
        }
        // shared buffer -> registers / coefficient planes
        R P[KS], A[KS], B[KS];
#pragma unroll
        for (int j = 0; j < KS; ++j) {
            const int c = (ck0 + j) * LX + cx;
            P[j] = pfP[c];
            A[j] = pfA[c];
            B[j] = pfB[c];
            const int v0 = (int)pfI[c];
            c0s[c] = sizeof(IT) == 1 ? slut[v0] : __ldg(I->lutc + v0);
            if (!TE) {
                const int v1 = (int)pfI[CELLS + c];
                c1s[c] = sizeof(IT) == 1 ? slut[v1] : __ldg(I->lutc + v1);
            }
        }
        __syncthreads();   // shared buffer free; coefficient planes and sg ready
        if (tn < ntiles) {
            prefetch(s_desc[ns]);
            fetch_state(ns);
            fetch_desc(tn + gridDim.x, nns);
        }
        cp_commit();

        const int i = d.li0 + cx;
        const int kb = d.lk0 + ck0;
        if (nsub > 0) {
            const bool colown = i >= d.oi0 && i < d.oi0 + d.ow;
            unsigned own = 0;
#pragma unroll
            for (int j = 0; j < KS; ++j)
                if (colown && kb + j >= d.ok0 && kb + j < d.ok0 + d.oh) own |= 1u << j;
            const bool hs = (d.flags & 1) != 0;   // tile holds the TF/SF plane
            const int six = hs ? I->src_ix : -8;
            int xm = -1;
            unsigned zmask = 0;
            if (d.flags & 2)
                for (int m = 0; m < I->nmon; ++m)
                    if (I->mon[m] == i) { xm = m; break; }
            if (d.flags & 4) {
#pragma unroll
                for (int j = 0; j < KS; ++j) {
                    const int kk = d.periodic ? pmod(kb + j, d.nz) : kb + j;
                    for (int m = 0; m < I->nmonz; ++m)
                        if (I->monz[m] == kk) zmask |= ((own >> j) & 1u) << j;
                }
            }
            const int nz = d.nz;
            for (int s = 0; s < nsub; ++s) {
                // ----- H half step
                if (lane == 0) {
#pragma unroll
                    for (int j = 0; j < KS; ++j) xPc[warp][j] = P[j];
                }
                xPr[warp][lane] = P[0];
                __syncthreads();
                const R Pdn = (wz + 1 < WZ) ? xPr[warp + WX][lane] : P[KS - 1];
#pragma unroll
                for (int j = 0; j < KS; ++j) {
                    R pr = __shfl_down_sync(FULL, P[j], 1);
                    const R pe = (wx + 1 < WX) ? xPc[warp + 1][j] : pr;
                    pr = (lane == 31) ? pe : pr;
                    const R pk = (j + 1 < KS) ? P[j + 1] : Pdn;
                    const R ca = TE ? C : c0s[(ck0 + j) * LX + cx];
                    A[j] += ca * (pk - P[j]);
                    const R cb = TE ? C : c1s[(ck0 + j) * LX + cx];
                    B[j] -= cb * (pr - P[j]);
                }
                if (hs && i == six - 1) {
                    const R ge = (R)sg[0][s];
#pragma unroll
                    for (int j = 0; j < KS; ++j) {
                        const int kk = d.periodic ? pmod(kb + j, nz) : kb + j;
                        B[j] += __ldg(I->srcB + kk) * ge;
                    }
                }
                // ----- E half step (branch-free stencil loop)
                if (lane == 31) {
#pragma unroll
                    for (int j = 0; j < KS; ++j) xBc[warp][j] = B[j];
                }
                xAr[warp][lane] = A[KS - 1];
                __syncthreads();
                const R Aup = (wz > 0) ? xAr[warp - WX][lane] : A[0];
#pragma unroll
                for (int j = 0; j < KS; ++j) {
                    R bl = __shfl_up_sync(FULL, B[j], 1);
                    const R be = (wx > 0) ? xBc[warp - 1][j] : bl;
                    bl = (lane == 0) ? be : bl;
                    const R am = (j > 0) ? A[j - 1] : Aup;
                    const R cp = TE ? c0s[(ck0 + j) * LX + cx] : C;
                    P[j] += cp * ((A[j] - am) - (B[j] - bl));
                }
                // rare paths, each behind a tile-uniform flag
                if (hs && i == six) {   // TF/SF: the plane is total field
                    const R gh = (R)sg[1][s];
#pragma unroll
                    for (int j = 0; j < KS; ++j) {
                        const int kk = d.periodic ? pmod(kb + j, nz) : kb + j;
                        P[j] += __ldg(I->srcP + kk) * gh;
                    }
                }
                if (d.flags & 6) {      // DFT monitor samples of this step
                    const int sslot = launch_off + s;
                    R* smp0 = I->samples + (size_t)sslot * I->sstride;
#pragma unroll
                    for (int j = 0; j < KS; ++j) {
                        R bl = __shfl_up_sync(FULL, B[j], 1);
                        const R be = (wx > 0) ? xBc[warp - 1][j] : bl;
                        bl = (lane == 0) ? be : bl;
                        if (xm >= 0 && ((own >> j) & 1u)) {
                            R* smp = smp0 + (size_t)xm * 2 * nz;
                            smp[kb + j] = P[j];
                            smp[nz + kb + j] = R(0.5) * (bl + B[j]);
                        }
                        if ((zmask >> j) & 1u) {
                            const R am = (j > 0) ? A[j - 1] : Aup;
                            for (int m = 0; m < I->nmonz; ++m) {
                                if (I->monz[m] != kb + j) continue;
                                R* smp = smp0 + (size_t)I->nmon * 2 * nz + (size_t)m * 2 * I->nx;
                                smp[i] = P[j];
                                smp[I->nx + i] = R(0.5) * (am + A[j]);
                            }
                        }
                    }
                }
            }
            // ----- energy on the chunk's last launch
            if (want_energy) {
                double e = 0.0;
#pragma unroll
                for (int j = 0; j < KS; ++j) {
                    if ((own >> j) & 1u) {
                        const size_t o = (size_t)(kb + j) * d.pitch + i;
                        const double p = P[j], a = A[j], b = B[j];
                        const int v0 = (int)reinterpret_cast<const IT*>(d.idx0)[o];
                        if (TE) {
                            e += I->lute[v0] * p * p + a * a + b * b;
                        } else {
                            const int v1 = (int)reinterpret_cast<const IT*>(d.idx1)[o];
                            e += p * p + I->lute[v0] * a * a + I->lute[v1] * b * b;
                        }
                    }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(FULL, e, o);
                if (lane == 0) sred[warp] = e;
                __syncthreads();
                if (threadIdx.x == 0) {
                    double tot = 0.0;
                    for (int w = 0; w < NW; ++w) tot += sred[w];
                    atomicAdd(&d.st->energy, tot);
                }
            }
            // ----- store the output rectangle
            R* __restrict__ Pout = reinterpret_cast<R*>(const_cast<void*>(d.f[par ^ 1][0]));
            R* __restrict__ Aout = reinterpret_cast<R*>(const_cast<void*>(d.f[par ^ 1][1]));
            R* __restrict__ Bout = reinterpret_cast<R*>(const_cast<void*>(d.f[par ^ 1][2]));
#pragma unroll
            for (int j = 0; j < KS; ++j) {
                if ((own >> j) & 1u) {
                    const size_t o = (size_t)(kb + j) * d.pitch + i;
                    Pout[o] = P[j];
                    Aout[o] = A[j];
                    Bout[o] = B[j];
                }
            }
            if (threadIdx.x == 0) d.st->cur = par ^ 1;
        }
        // advance the pipeline
        t = tn;
        ++it;
        __syncthreads();   // everyone is done with sg, the exchange buffers and descriptor slot cs
    }
}

}  // namespace fast
}  // namespace orf
