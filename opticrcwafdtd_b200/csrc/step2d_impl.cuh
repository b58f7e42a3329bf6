// step2d_impl.cuh -- fused, temporally blocked 2D Yee step kernel for sm_100a.
//
// Replaces the time loop of toolbox/+orf/fdtd2D.m:3-7 (P/A/B form):
//   A += cA dP/dz,  B -= cB dP/dx,  P += cP (dA/dz - dB/dx)
// with CPML (cpmlCoefficients.m:4-8), the one-sided TF/SF plane
// (fdtd2DTE.m:11-15, fdtd2D.m:21-23) and DFT sampling of the monitor lines
// (fdtd2DTE.m:16-18) fused into one launch that advances up to T time steps.
//
// Layout and work split (B200-first):
//   - a CTA owns a tile of LX = 32*WX columns by LZ = KS*WZ rows; each thread
//     keeps a vertical strip of KS cells of P, A and B in registers for the
//     whole launch, so the T fused steps touch HBM once per field (load at
//     the start, store at the end);
//   - x neighbours come from warp shuffles, neighbours across warps from two
//     small shared-memory exchange buffers (one __syncthreads per half step);
//   - tiles overlap by T cells on every side (trapezoidal temporal
//     blocking): after T steps only the inner (LX-2T) x (LZ-2T) output
//     rectangle is valid and written back, so neighbouring CTAs never need
//     each other's results inside a launch;
//   - fields are read from buffer `par` and written to buffer 1-par
//     (ping-pong), which makes the overlapping tiles race-free;
//   - the update coefficients come from a uint8/uint16 material index and a
//     lookup table of C/eps (exact: the table holds the distinct values);
//   - CPML tiles keep their psi state in shared memory (dynamic), interior
//     tiles are a separate instantiation with no CPML code at all;
//   - the CTA is persistent: it walks the tile list (tiles of one or many
//     instances) with a grid stride.
#pragma once
#include "orf_internal.cuh"

#include <cstdio>

namespace orf {
namespace {

__device__ __forceinline__ int pmod(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

template <class IT>
__device__ __forceinline__ int ld_idx(const void* p, size_t off) {
    return (int)__ldg(reinterpret_cast<const IT*>(p) + off);
}

template <class R>
__device__ __forceinline__ R ldg(const R* p) { return __ldg(p); }

// compact CPML slab index of a coordinate (-1 outside the absorbing layer)
__device__ __forceinline__ int slab_int(int u, int n, int np) {
    if (np <= 0 || u < 0 || u >= n) return -1;
    if (u < np) return u;
    if (u >= n - np) return np + u - (n - np);
    return -1;
}
__device__ __forceinline__ int slab_half(int u, int n, int np) {   // positions u+1/2, u < n-1
    if (np <= 0 || u < 0 || u >= n - 1) return -1;
    if (u < np) return u;
    if (u >= n - 1 - np) return np + u - (n - 1 - np);
    return -1;
}

template <class R, class IT, bool TE, bool PML, int KS, int WX, int WZ>
__global__ void __launch_bounds__(32 * WX * WZ)
k_step2d(const Inst2D<R>* __restrict__ insts, const Tile2D* __restrict__ tiles, int ntiles, int halo,
         int launch_off, int nsub_max, int par, int want_energy) {
    constexpr int NW = WX * WZ;
    constexpr int LX = 32 * WX;
    constexpr int LZ = KS * WZ;
    constexpr unsigned FULL = 0xffffffffu;
    static_assert(KS <= 32, "strip mask is 32 bits");

    __shared__ R xPc[NW][KS];   // lane-0 column of P per warp (x neighbour for lane 31)
    __shared__ R xPr[NW][32];   // row 0 of P per warp (z neighbour for the row KS-1)
    __shared__ R xBc[NW][KS];   // lane-31 column of B per warp (x neighbour for lane 0)
    __shared__ R xAr[NW][32];   // row KS-1 of A per warp (z neighbour for row 0)
    __shared__ double sg[2][kMaxSub];
    __shared__ double sred[NW];
    __shared__ long long s_step0;
    __shared__ int s_nsub;
    __shared__ R spz[PML ? LZ : 1][3];    // CPML profile of the tile rows (P positions)
    __shared__ R spzh[PML ? LZ : 1][3];   // ... at A positions
    // dynamic shared memory: per-cell update coefficients of the tile
    // (TE: cP; TM: cA, cB), then the four CPML psi planes (PML tiles only)
    extern __shared__ __align__(16) unsigned char dsm[];
    R* c0s = reinterpret_cast<R*>(dsm);                 // [LZ][LX]
    R* c1s = c0s + LX * LZ;                             // TM only
    R* psiAs = c0s + (TE ? 1 : 2) * LX * LZ;            // [LZ][LX] each, PML only
    R* psiBs = psiAs + LX * LZ;
    R* psiPxs = psiBs + LX * LZ;
    R* psiPzs = psiPxs + LX * LZ;

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wx = warp % WX;
    const int wz = warp / WX;
    const int cx = 32 * wx + lane;

    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        __syncthreads();   // previous tile is done with the shared scalars
        const Tile2D tile = tiles[t];
        const Inst2D<R>* __restrict__ I = insts + tile.inst;
        JobState* st = I->st;
        if (threadIdx.x == 0) {
            long long step0 = st->done ? -1 : st->step;
            int nsub = 0;
            if (step0 >= 0) {
                long long rem = st->nmax - (step0 + launch_off);
                nsub = (int)max(0LL, min((long long)nsub_max, rem));
            }
            s_step0 = step0;
            s_nsub = nsub;
        }
        __syncthreads();
        const int nsub = s_nsub;
        if (nsub <= 0) continue;
        const long long n0 = s_step0 + launch_off;

        const int nx = I->nx, nz = I->nz, pitch = I->pitch, nzA = I->nzA, nxB = I->nxB;
        const bool per = I->periodic != 0;
        const R C = I->C;
        for (int q = threadIdx.x; q < nsub; q += blockDim.x) {
            const long long n = n0 + q;
            sg[0][q] = n < I->nsrc ? I->gE[n] : 0.0;
            sg[1][q] = n < I->nsrc ? I->gH[n] : 0.0;
        }
        const int kt0 = tile.ok0 - halo;        // first (unwrapped) row of the tile
        const int i = tile.oi0 - halo + cx;     // this thread's column
        const bool cv = i >= 0 && i < nx;
        const bool cvB = i >= 0 && i < nxB;
        if (PML) {
            for (int q = threadIdx.x; q < LZ; q += blockDim.x) {
                const int k = kt0 + q;
                const int kk = per ? pmod(k, nz) : k;
                const bool rv = kk >= 0 && kk < nz;
                for (int c = 0; c < 3; ++c) {
                    spz[q][c] = rv ? I->pmlz[3 * kk + c] : R(c == 0 || c == 2 ? 1 : 0);
                    spzh[q][c] = (rv && kk < nzA) ? I->pmlzh[3 * kk + c] : R(c == 0 || c == 2 ? 1 : 0);
                }
            }
        }

        // ---------------------------------------------------------- load
        const R* __restrict__ Pin = I->P[par];
        const R* __restrict__ Ain = I->A[par];
        const R* __restrict__ Bin = I->B[par];
        R P[KS], A[KS], B[KS];
        unsigned mP = 0, mA = 0, mB = 0, own = 0;
        const int kb = kt0 + KS * wz;
        const bool colown = (cx - halo) >= 0 && (cx - halo) < tile.ow;
#pragma unroll
        for (int j = 0; j < KS; ++j) {
            const int k = kb + j;
            const int kk = per ? pmod(k, nz) : k;
            const bool rv = per || (k >= 0 && k < nz);
            P[j] = R(0);
            A[j] = R(0);
            B[j] = R(0);
            R c0 = R(0), c1 = R(0);
            if (rv && cv) {
                const size_t o = (size_t)kk * pitch + i;
                P[j] = Pin[o];
                A[j] = Ain[o];
                B[j] = Bin[o];
                c0 = __ldg(I->lutc + ld_idx<IT>(I->idx0, o));
                if (!TE) c1 = __ldg(I->lutc + ld_idx<IT>(I->idx1, o));
                mP |= 1u << j;
                if (kk < nzA) mA |= 1u << j;
            }
            c0s[(KS * wz + j) * LX + cx] = c0;
            if (!TE) c1s[(KS * wz + j) * LX + cx] = c1;
            if (rv && cvB) mB |= 1u << j;
            const int r = KS * wz + j - halo;
            if (colown && r >= 0 && r < tile.oh) own |= 1u << j;
        }
        // column CPML profiles (identity outside the layer)
        R pxb = R(1), pxa = R(0), pxk = R(1), phb = R(1), pha = R(0), phk = R(1);
        int sxP = -1, sxB = -1;
        if (PML) {
            if (cv) {
                pxb = I->pmlx[3 * i];
                pxa = I->pmlx[3 * i + 1];
                pxk = I->pmlx[3 * i + 2];
                sxP = slab_int(i, nx, I->npx);
            }
            if (cvB) {
                phb = I->pmlxh[3 * i];
                pha = I->pmlxh[3 * i + 1];
                phk = I->pmlxh[3 * i + 2];
                sxB = slab_half(i, nx, I->npx);
            }
            const R* __restrict__ gA = I->psiA[par];
            const R* __restrict__ gB = I->psiB[par];
            const R* __restrict__ gPx = I->psiPx[par];
            const R* __restrict__ gPz = I->psiPz[par];
#pragma unroll
            for (int j = 0; j < KS; ++j) {
                const int ck = KS * wz + j;
                const int k = kb + j;
                const int kk = per ? pmod(k, nz) : k;
                R a = R(0), b = R(0), px = R(0), pz = R(0);
                if ((mP >> j) & 1u) {
                    const int szA = slab_half(kk, nz, I->npz);
                    const int szP = slab_int(kk, nz, I->npz);
                    if (szA >= 0) a = gA[(size_t)szA * nx + i];
                    if (szP >= 0) pz = gPz[(size_t)szP * nx + i];
                    if (sxP >= 0) px = gPx[(size_t)kk * (2 * I->npx) + sxP];
                }
                if (((mB >> j) & 1u) && sxB >= 0) b = gB[(size_t)kk * (2 * I->npx) + sxB];
                psiAs[ck * LX + cx] = a;
                psiBs[ck * LX + cx] = b;
                psiPxs[ck * LX + cx] = px;
                psiPzs[ck * LX + cx] = pz;
            }
        }
        // monitors on this column / these rows
        int xm = -1;
        for (int m = 0; m < I->nmon; ++m)
            if (I->mon[m] == i && cv) { xm = m; break; }
        unsigned zmask = 0;
        if (I->nmonz > 0) {
#pragma unroll
            for (int j = 0; j < KS; ++j) {
                const int kk = per ? pmod(kb + j, nz) : kb + j;
                for (int m = 0; m < I->nmonz; ++m)
                    if (I->monz[m] == kk) zmask |= ((own >> j) & 1u) << j;
            }
        }
        const int six = I->src_ix;
        const bool has_mon = __syncthreads_or(xm >= 0 || zmask != 0) != 0;   // also: sg / spz / psi ready

        // ---------------------------------------------------------- steps
        for (int s = 0; s < nsub; ++s) {
            // ----- H half step: A (d/dz P), B (d/dx P)
            if (lane == 0) {
#pragma unroll
                for (int j = 0; j < KS; ++j) xPc[warp][j] = P[j];
            }
            xPr[warp][lane] = P[0];
            __syncthreads();
            const R Pdn = (wz + 1 < WZ) ? xPr[warp + WX][lane] : R(0);
#pragma unroll
            for (int j = 0; j < KS; ++j) {
                R pr = __shfl_down_sync(FULL, P[j], 1);
                if (lane == 31) pr = (wx + 1 < WX) ? xPc[warp + 1][j] : R(0);
                const R pk = (j + 1 < KS) ? P[j + 1] : Pdn;
                R d = pk - P[j];
                if (PML) {
                    const int ck = KS * wz + j;
                    R& ps = psiAs[ck * LX + cx];
                    ps = spzh[ck][0] * ps + spzh[ck][1] * d;
                    d = d * spzh[ck][2] + ps;
                }
                const R ca = TE ? C : c0s[(KS * wz + j) * LX + cx];
                if ((mA >> j) & 1u) A[j] += ca * d;
                R e = pr - P[j];
                if (PML) {
                    const int ck = KS * wz + j;
                    R& ps = psiBs[ck * LX + cx];
                    ps = phb * ps + pha * e;
                    e = e * phk + ps;
                }
                const R cb = TE ? C : c1s[(KS * wz + j) * LX + cx];
                if ((mB >> j) & 1u) B[j] -= cb * e;
            }
            if (i == six - 1) {   // TF/SF: the B column left of the plane is scattered field
                const R ge = (R)sg[0][s];
#pragma unroll
                for (int j = 0; j < KS; ++j) {
                    if ((mB >> j) & 1u) {
                        const int kk = per ? pmod(kb + j, nz) : kb + j;
                        B[j] += ldg(I->srcB + kk) * ge;
                    }
                }
            }
            // ----- E half step: P
            if (lane == 31) {
#pragma unroll
                for (int j = 0; j < KS; ++j) xBc[warp][j] = B[j];
            }
            xAr[warp][lane] = A[KS - 1];
            __syncthreads();
            const R Aup = (wz > 0) ? xAr[warp - WX][lane] : R(0);
#pragma unroll
            for (int j = 0; j < KS; ++j) {
                R bl = __shfl_up_sync(FULL, B[j], 1);
                if (lane == 0) bl = (wx > 0) ? xBc[warp - 1][j] : R(0);
                const R am = (j > 0) ? A[j - 1] : Aup;
                R da = A[j] - am;
                R db = B[j] - bl;
                if (PML) {
                    const int ck = KS * wz + j;
                    R& pz = psiPzs[ck * LX + cx];
                    pz = spz[ck][0] * pz + spz[ck][1] * da;
                    da = da * spz[ck][2] + pz;
                    R& px = psiPxs[ck * LX + cx];
                    px = pxb * px + pxa * db;
                    db = db * pxk + px;
                }
                const R cp = TE ? c0s[(KS * wz + j) * LX + cx] : C;
                if ((mP >> j) & 1u) P[j] += cp * (da - db);
            }
            if (i == six) {   // TF/SF: the plane is total field
                const R gh = (R)sg[1][s];
#pragma unroll
                for (int j = 0; j < KS; ++j) {
                    if ((mP >> j) & 1u) {
                        const int kk = per ? pmod(kb + j, nz) : kb + j;
                        P[j] += ldg(I->srcP + kk) * gh;
                    }
                }
            }
            if (has_mon) {    // DFT monitor samples of this step (block-uniform flag)
                const int slot = launch_off + s;
#pragma unroll
                for (int j = 0; j < KS; ++j) {
                    R bl = __shfl_up_sync(FULL, B[j], 1);
                    if (lane == 0) bl = (wx > 0) ? xBc[warp - 1][j] : R(0);
                    if (xm >= 0 && ((own >> j) & 1u)) {
                        const int kk = per ? pmod(kb + j, nz) : kb + j;
                        R* smp = I->samples + (size_t)slot * I->sstride + (size_t)xm * 2 * nz;
                        smp[kk] = P[j];
                        smp[nz + kk] = R(0.5) * (bl + B[j]);
                    }
                    if ((zmask >> j) & 1u) {
                        const R am = (j > 0) ? A[j - 1] : Aup;
                        const int kk = per ? pmod(kb + j, nz) : kb + j;
                        for (int m = 0; m < I->nmonz; ++m) {
                            if (I->monz[m] != kk) continue;
                            R* smp = I->samples + (size_t)slot * I->sstride + (size_t)I->nmon * 2 * nz +
                                     (size_t)m * 2 * nx;
                            smp[i] = P[j];
                            smp[nx + i] = R(0.5) * (am + A[j]);
                        }
                    }
                }
            }
        }

        // ---------------------------------------------------------- energy
        if (want_energy) {
            double e = 0.0;
#pragma unroll
            for (int j = 0; j < KS; ++j) {
                if ((own >> j) & 1u) {
                    const double p = P[j], a = A[j], b = B[j];
                    const size_t o = (size_t)(kb + j) * pitch + i;
                    if (TE) {
                        e += I->lute[ld_idx<IT>(I->idx0, o)] * p * p + a * a + b * b;
                    } else {
                        e += p * p + (((mA >> j) & 1u) ? I->lute[ld_idx<IT>(I->idx0, o)] * a * a : 0.0) +
                             (((mB >> j) & 1u) ? I->lute[ld_idx<IT>(I->idx1, o)] * b * b : 0.0);
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
                atomicAdd(&st->energy, tot);
            }
        }

        // ---------------------------------------------------------- store
        R* __restrict__ Pout = I->P[1 - par];
        R* __restrict__ Aout = I->A[1 - par];
        R* __restrict__ Bout = I->B[1 - par];
#pragma unroll
        for (int j = 0; j < KS; ++j) {
            if ((own >> j) & 1u) {
                const int kk = kb + j;   // owned rows never wrap
                const size_t o = (size_t)kk * pitch + i;
                Pout[o] = P[j];
                Aout[o] = A[j];
                Bout[o] = B[j];
            }
        }
        if (PML) {
            R* __restrict__ gA = I->psiA[1 - par];
            R* __restrict__ gB = I->psiB[1 - par];
            R* __restrict__ gPx = I->psiPx[1 - par];
            R* __restrict__ gPz = I->psiPz[1 - par];
#pragma unroll
            for (int j = 0; j < KS; ++j) {
                if (!((own >> j) & 1u)) continue;
                const int ck = KS * wz + j;
                const int kk = kb + j;
                const int szA = slab_half(kk, nz, I->npz);
                const int szP = slab_int(kk, nz, I->npz);
                if (szA >= 0) gA[(size_t)szA * nx + i] = psiAs[ck * LX + cx];
                if (szP >= 0) gPz[(size_t)szP * nx + i] = psiPzs[ck * LX + cx];
                if (sxP >= 0) gPx[(size_t)kk * (2 * I->npx) + sxP] = psiPxs[ck * LX + cx];
                if (sxB >= 0) gB[(size_t)kk * (2 * I->npx) + sxB] = psiBs[ck * LX + cx];
            }
        }
        if (threadIdx.x == 0) st->cur = 1 - par;
    }
}

// Dynamic shared memory of one instantiation.
template <class R, bool TE, bool PML, int KS, int WX, int WZ>
constexpr size_t step2d_dyn_smem() {
    return (size_t)((TE ? 1 : 2) + (PML ? 4 : 0)) * 32 * WX * KS * WZ * sizeof(R);
}

// Opt-in to the dynamic shared memory of an instantiation, once per device.
// Called from the occupancy query at job creation, so it never runs inside a
// stream capture.
template <class R, class IT, bool TE, bool PML, int KS, int WX, int WZ>
cudaError_t configure_one() {
    static int configured[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 64 || configured[dev]) return cudaSuccess;
    constexpr size_t smem = step2d_dyn_smem<R, TE, PML, KS, WX, WZ>();
    cudaError_t e = cudaFuncSetAttribute(k_step2d<R, IT, TE, PML, KS, WX, WZ>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) configured[dev] = 1;
    return e;
}

template <class R, class IT, bool TE, bool PML, int KS, int WX, int WZ>
cudaError_t launch_one(const void* insts, const Tile2D* tiles, int ntiles, int halo, int launch_off, int nsub,
                       int par, int want_energy, int grid, cudaStream_t s) {
    auto kern = k_step2d<R, IT, TE, PML, KS, WX, WZ>;
    constexpr size_t smem = step2d_dyn_smem<R, TE, PML, KS, WX, WZ>();
    kern<<<grid, 32 * WX * WZ, smem, s>>>(reinterpret_cast<const Inst2D<R>*>(insts), tiles, ntiles, halo,
                                          launch_off, nsub, par, want_energy);
    return cudaGetLastError();
}

template <class R, class IT, bool TE, bool PML, int KS, int WX, int WZ>
int occupancy_one() {
    auto kern = k_step2d<R, IT, TE, PML, KS, WX, WZ>;
    constexpr size_t smem = step2d_dyn_smem<R, TE, PML, KS, WX, WZ>();
    if (configure_one<R, IT, TE, PML, KS, WX, WZ>() != cudaSuccess) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 32 * WX * WZ, smem) != cudaSuccess) nb = 1;
    return nb;
}

template <class R, int KS, int WX, int WZ>
cudaError_t dispatch_v(bool te, bool idx16, bool pml, const void* insts, const Tile2D* tiles, int ntiles,
                       int halo, int off, int nsub, int par, int we, int grid, cudaStream_t s) {
#define ORF_L(IT, TEV, PMLV) \
    return launch_one<R, IT, TEV, PMLV, KS, WX, WZ>(insts, tiles, ntiles, halo, off, nsub, par, we, grid, s)
    if (!idx16) {
        if (te) { if (pml) ORF_L(uint8_t, true, true); else ORF_L(uint8_t, true, false); }
        else    { if (pml) ORF_L(uint8_t, false, true); else ORF_L(uint8_t, false, false); }
    } else {
        if (te) { if (pml) ORF_L(uint16_t, true, true); else ORF_L(uint16_t, true, false); }
        else    { if (pml) ORF_L(uint16_t, false, true); else ORF_L(uint16_t, false, false); }
    }
#undef ORF_L
}

template <class R, int KS, int WX, int WZ>
int occ_v(bool te, bool idx16, bool pml) {
#define ORF_O(IT, TEV, PMLV) return occupancy_one<R, IT, TEV, PMLV, KS, WX, WZ>()
    if (!idx16) {
        if (te) { if (pml) ORF_O(uint8_t, true, true); else ORF_O(uint8_t, true, false); }
        else    { if (pml) ORF_O(uint8_t, false, true); else ORF_O(uint8_t, false, false); }
    } else {
        if (te) { if (pml) ORF_O(uint16_t, true, true); else ORF_O(uint16_t, true, false); }
        else    { if (pml) ORF_O(uint16_t, false, true); else ORF_O(uint16_t, false, false); }
    }
#undef ORF_O
}

}  // namespace
}  // namespace orf
