// step2d_fast.cuh -- pipelined, temporally blocked 2D Yee step kernel (sm_100a).
//
// Replaces the time loop of toolbox/+orf/fdtd2D.m:3-7 (P/A/B form):
//   A += cA dP/dz,  B -= cB dP/dx,  P += cP (dA/dz - dB/dx)
// with CPML (cpmlCoefficients.m:4-8), the one-sided TF/SF plane
// (fdtd2DTE.m:11-15, fdtd2D.m:21-23) and DFT sampling of the monitor lines
// (fdtd2DTE.m:16-18), advancing up to T time steps per launch.
//
// Layout and work split:
//   - a CTA owns a tile of LX = 32*WX columns by LZ = KS*WZ rows; each thread
//     keeps a vertical strip of KS cells of P, A and B in registers for the
//     whole launch, so the T fused steps read and write HBM once per field;
//   - x neighbours come from warp shuffles, neighbours across warps from small
//     shared exchange buffers (one __syncthreads per half step);
//   - tiles overlap by T cells (trapezoidal temporal blocking): after T steps
//     only the inner output rectangle is valid and written back; fields
//     ping-pong between two buffers so overlapping tiles never race;
//   - the update coefficients come from a uint8/uint16 material index and a
//     table of C/eps (exact), looked up once per tile into registers;
//   - no memory access depends on a runtime branch inside the stencil loop:
//     neighbour-warp columns are read with 16-byte vector loads from a valid
//     slot (a tile-edge warp reads its own, a halo value) and selected;
//   - the CTA is persistent and software-pipelined over its tiles: while tile
//     t computes, the cp.async prefetch of tile t+1 (fields, material index)
//     and the descriptor and job-state snapshot of tile t+2 are in flight.
// Two instantiations per geometry: interior tiles (PML = false: every cell of
// the tile's dependency cone is a plain cell, no masks and no CPML code) and
// frame tiles (PML = true: CPML psi in a shared working plane, boundary
// masks, zero fill outside the grid), the latter specialised on the CPML axes
// a tile reaches.  Every update is written with explicit fma, so each
// instantiation performs, cell by cell, the same roundings (no contraction
// choice left to the compiler) and results do not depend on the tiling.
#pragma once
#include "orf_internal.cuh"

namespace orf {
namespace fast {

template <bool B>
struct Flag {
    static constexpr bool value = B;
};

// Checked build (compiled with -DORF_CHECK, lib/liborf_fdtd_check.so): every
// global access of the step kernel is tested against the extent of its
// buffer (and every stored cell against the grid); an index outside is
// counted here and the access skipped.  In the normal build the tests compile
// away.  The counter of each translation unit is read by fast2d_violations.
#ifdef ORF_CHECK
static __device__ unsigned long long g_check_violations;
__device__ __forceinline__ bool in_bounds(long long i, long long n) {
    const bool ok = i >= 0 && i < n;
    if (!ok) atomicAdd(&g_check_violations, 1ull);
    return ok;
}
#define ORF_IN(i, n) ::orf::fast::in_bounds((long long)(i), (long long)(n))
#else
#define ORF_IN(i, n) true
#endif

__device__ __forceinline__ int pmod(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

// cp.async of 4 / 8 bytes; when valid is false the destination is zero-filled
// (src-size 0) and src is not read.
__device__ __forceinline__ void cp_async4(void* sdst, const void* gsrc, bool valid = true) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    const unsigned n = valid ? 4u : 0u;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gsrc), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async8(void* sdst, const void* gsrc, bool valid = true) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    const unsigned n = valid ? 8u : 0u;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gsrc), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <class R>
__device__ __forceinline__ void cp_field(R* sdst, const R* gsrc, bool valid = true) {
    if constexpr (sizeof(R) == 4) cp_async4(sdst, gsrc, valid);
    else cp_async8(sdst, gsrc, valid);
}

// compact CPML slab index (-1 outside the absorbing layer)
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

// Dynamic shared memory: prefetch planes of P, A, B and the material index,
// then (PML) four psi planes and the row / column CPML profiles of the tile.
template <class R, class IT, bool TE, bool PML, int KS, int WX, int WZ>
constexpr size_t dyn_smem() {
    constexpr size_t LX = 32 * WX, LZ = (size_t)KS * WZ, cells = LX * LZ;
    constexpr size_t idxb = ((cells * sizeof(IT) * (TE ? 1 : 2)) + 15) & ~size_t(15);
    size_t b = cells * sizeof(R) * 3 + idxb;
    if (PML) b += cells * sizeof(R) * 4 + (LZ + LX) * 6 * sizeof(R);
    return b;
}

// 16 bytes of an exchange row (16-byte aligned) into registers
template <class R>
__device__ __forceinline__ void load16(R (&dst)[16 / sizeof(R)], const R* src) {
    if constexpr (sizeof(R) == 4) {
        const float4 v = *reinterpret_cast<const float4*>(src);
        dst[0] = v.x; dst[1] = v.y; dst[2] = v.z; dst[3] = v.w;
    } else {
        const double2 v = *reinterpret_cast<const double2*>(src);
        dst[0] = v.x; dst[1] = v.y;
    }
}
template <class R, int KS>
__device__ __forceinline__ void store_row(R* dst, const R (&src)[KS]) {
    if constexpr (sizeof(R) == 4 && KS % 4 == 0) {
#pragma unroll
        for (int q = 0; q < KS / 4; ++q)
            reinterpret_cast<float4*>(dst)[q] = make_float4(src[4 * q], src[4 * q + 1], src[4 * q + 2], src[4 * q + 3]);
    } else if constexpr (sizeof(R) == 8 && KS % 2 == 0) {
#pragma unroll
        for (int q = 0; q < KS / 2; ++q) reinterpret_cast<double2*>(dst)[q] = make_double2(src[2 * q], src[2 * q + 1]);
    } else {
#pragma unroll
        for (int j = 0; j < KS; ++j) dst[j] = src[j];
    }
}

template <class R, class IT, bool TE, bool PML, int KS, int WX, int WZ>
__global__ void __launch_bounds__(32 * WX * WZ, (PML && sizeof(R) == 4) ? 2 : 1)
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
    R* psA = reinterpret_cast<R*>(reinterpret_cast<unsigned char*>(pfI) + idxb);   // PML only: psi of A (z), B (x), P (x), P (z)
    R* psB = psA + CELLS;
    R* psPx = psB + CELLS;
    R* psPz = psPx + CELLS;
    R* prz = psPz + CELLS;                               // PML only: [LZ][6] rows: zP b,a,k ; zA b,a,k
    R* prx = prz + LZ * 6;                               // PML only: [LX][6] cols: xP b,a,k ; xB b,a,k

    __shared__ __align__(16) R xPc[NW][KS];
    __shared__ R xPr[NW][32];
    __shared__ __align__(16) R xBc[NW][KS];
    __shared__ R xAr[NW][32];
    __shared__ R slut[256];
    __shared__ const R* s_lutsrc;
    __shared__ double sg[2][kMaxSub];
    __shared__ double sred[NW];
    // descriptor ring (tiles t, t+G, t+2G) and snapshots of their job state,
    // both filled by cp.async so no thread waits on a dependent global load
    __shared__ __align__(16) FastTile2D s_desc[3];
    __shared__ __align__(16) long long s_state[3][4];   // step, nmax, chunk, done | converged << 32

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wx = warp % WX;
    const int wz = warp / WX;
    const int cx = 32 * wx + lane;
    const int ck0 = KS * wz;
    // neighbour warps in the tile; a warp on the tile edge names itself
    const bool hasR = wx + 1 < WX, hasL = wx > 0, hasDn = wz + 1 < WZ, hasUp = wz > 0;
    const int wR = hasR ? warp + 1 : warp, wL = hasL ? warp - 1 : warp;
    const int wDn = hasDn ? warp + WX : warp, wUp = hasUp ? warp - WX : warp;

    // ---- prefetch one tile's fields and material index into the shared buffer
    auto prefetch = [&](const FastTile2D& d) {
        const R* gP = reinterpret_cast<const R*>(d.f[par][0]);
        const R* gA = reinterpret_cast<const R*>(d.f[par][1]);
        const R* gB = reinterpret_cast<const R*>(d.f[par][2]);
        if constexpr (!PML) {
            // interior tiles: 16-byte chunks of rows (li0 is a multiple of 4
            // cells and the pitch of 32, so every chunk is 16-byte aligned);
            // chunks past the row end are clamped onto its last chunk, cells
            // no output's dependency cone reaches
            constexpr int VE = 16 / (int)sizeof(R);
            constexpr int CPR = LX / VE;
            constexpr int NCH = LZ * CPR;
            static_assert(NCH % NT == 0, "whole chunks per thread");
#pragma unroll
            for (int r = 0; r < NCH / NT; ++r) {
                const int c = (int)threadIdx.x + r * NT;
                const int row = c / CPR, cc = c - row * CPR;
                const int grow = d.lk0 + row;
                const int kk = d.periodic ? pmod(grow, d.nz) : min(max(grow, 0), d.nz - 1);
                const size_t off = (size_t)kk * d.pitch + min(d.li0 + VE * cc, d.pitch - VE);
                const int s = row * LX + VE * cc;
                if (!ORF_IN(off + VE - 1, (size_t)d.pitch * d.nz)) continue;
                cp_async16(pfP + s, gP + off);
                cp_async16(pfA + s, gA + off);
                cp_async16(pfB + s, gB + off);
            }
        } else {
            const int i = d.li0 + cx;
            const bool cv = i >= 0 && i < d.nx;
            const int col = min(max(i, 0), d.nx - 1);
#pragma unroll
            for (int j = 0; j < KS; ++j) {
                const int row = d.lk0 + ck0 + j;
                const bool rv = d.periodic || (row >= 0 && row < d.nz);
                const int kk = d.periodic ? pmod(row, d.nz) : min(max(row, 0), d.nz - 1);
                const size_t off = (size_t)kk * d.pitch + col;
                const int c = (ck0 + j) * LX + cx;
                const bool v = cv && rv && ORF_IN(off, (size_t)d.pitch * d.nz);
                cp_field(pfP + c, gP + off, v);
                cp_field(pfA + c, gA + off, v);
                cp_field(pfB + c, gB + off, v);
            }
        }
        // material index rows: 4-byte copies (li0 and pitch are multiples of 4 cells)
        constexpr int W4 = LX * (int)sizeof(IT) / 4;
        for (int q = threadIdx.x; q < NIDX * LZ * W4; q += NT) {
            const int plane = q / (LZ * W4);
            const int r = (q / W4) % LZ;
            const int c4 = q % W4;
            const int row = d.lk0 + r;
            const bool rv = d.periodic || (row >= 0 && row < d.nz);
            const int kk = d.periodic ? pmod(row, d.nz) : min(max(row, 0), d.nz - 1);
            const int c0 = d.li0 + 4 * c4 / (int)sizeof(IT);     // first cell of the word
            const bool v = rv && c0 >= 0 && c0 < d.pitch;
            const size_t base = (size_t)kk * d.pitch * sizeof(IT);
            size_t boff = base + (size_t)max(c0, 0) * sizeof(IT);
            const size_t rowend = base + (size_t)d.pitch * sizeof(IT);
            if (boff + 4 > rowend) boff = rowend - 4;
            const unsigned char* src = reinterpret_cast<const unsigned char*>(plane ? d.idx1 : d.idx0) + boff;
            if (v && !ORF_IN(boff + 3, (size_t)d.pitch * d.nz * sizeof(IT))) continue;
            cp_async4(reinterpret_cast<unsigned char*>(pfI) + (size_t)plane * CELLS * sizeof(IT) +
                          ((size_t)r * LX) * sizeof(IT) + 4 * (size_t)c4,
                      src, v);
        }
    };
    auto fetch_desc = [&](int tile, int slot) {   // threads 0..7: 8 x 16 B
        if (threadIdx.x < 8 && tile < ntiles)
            cp_async16(reinterpret_cast<char*>(&s_desc[slot]) + 16 * threadIdx.x,
                       reinterpret_cast<const char*>(tiles + tile) + 16 * threadIdx.x);
    };
    auto fetch_state = [&](int slot) {            // threads 8..9: 2 x 16 B of JobState
        if (threadIdx.x >= 8 && threadIdx.x < 10) {
            const int q = threadIdx.x - 8;
            cp_async16(reinterpret_cast<char*>(&s_state[slot][0]) + 16 * q,
                       reinterpret_cast<const char*>(s_desc[slot].st) + 16 * q);
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
        const int i = d.li0 + cx;
        const int kb = d.lk0 + ck0;
        const int nz = d.nz;
        // boundary masks (frame tiles): cells outside the grid, and the A row
        // nz-1 / B column nx-1 that do not exist, keep zero and are not updated
        unsigned mP = ~0u, mA = ~0u, mB = ~0u;
        int sxP = -1, sxB = -1;
        if (PML) {
            const int nzA = d.periodic ? nz : nz - 1;
            const bool cv = i >= 0 && i < d.nx, cvB = i >= 0 && i < d.nx - 1;
            mP = mA = mB = 0;
#pragma unroll
            for (int j = 0; j < KS; ++j) {
                const int k = kb + j;
                const bool rv = d.periodic || (k >= 0 && k < nz);
                const int kk = d.periodic ? pmod(k, nz) : k;
                if (rv && cv) mP |= 1u << j;
                if (rv && cv && kk < nzA) mA |= 1u << j;
                if (rv && cvB) mB |= 1u << j;
            }
            // CPML state of the tile: psi planes (zero outside the slabs) and
            // the row / column profiles (identity outside the slabs)
            const int npx = I->npx, npz = I->npz, nx = d.nx;
            sxP = cv ? slab_int(i, nx, npx) : -1;
            sxB = cvB ? slab_half(i, nx, npx) : -1;
            const R* gA = I->psiA[par];
            const R* gB = I->psiB[par];
            const R* gPx = I->psiPx[par];
            const R* gPz = I->psiPz[par];
#pragma unroll
            for (int j = 0; j < KS; ++j) {
                const int c = (ck0 + j) * LX + cx;
                const int k = kb + j;
                const int kk = d.periodic ? pmod(k, nz) : k;
                R a = R(0), b = R(0), px = R(0), pz = R(0);
                if ((mP >> j) & 1u) {
                    const int szA = slab_half(kk, nz, npz);
                    const int szP = slab_int(kk, nz, npz);
                    if (szA >= 0 && ORF_IN((size_t)szA * nx + i, (size_t)2 * npz * nx)) a = gA[(size_t)szA * nx + i];
                    if (szP >= 0 && ORF_IN((size_t)szP * nx + i, (size_t)2 * npz * nx)) pz = gPz[(size_t)szP * nx + i];
                    if (sxP >= 0 && ORF_IN((size_t)kk * (2 * npx) + sxP, (size_t)nz * 2 * npx))
                        px = gPx[(size_t)kk * (2 * npx) + sxP];
                }
                if (((mB >> j) & 1u) && sxB >= 0 && ORF_IN((size_t)kk * (2 * npx) + sxB, (size_t)nz * 2 * npx))
                    b = gB[(size_t)kk * (2 * npx) + sxB];
                psA[c] = a;
                psB[c] = b;
                psPx[c] = px;
                psPz[c] = pz;
            }
            for (int q = threadIdx.x; q < LZ; q += NT) {
                const int k = d.lk0 + q;
                const int kk = d.periodic ? pmod(k, nz) : k;
                const bool rv = kk >= 0 && kk < nz;
                for (int cc = 0; cc < 3; ++cc) {
                    const R id = R(cc == 1 ? 0 : 1);
                    prz[q * 6 + cc] = (rv && ORF_IN(3 * kk + cc, 3 * nz)) ? I->pmlz[3 * kk + cc] : id;
                    prz[q * 6 + 3 + cc] = (rv && kk < nzA && ORF_IN(3 * kk + cc, 3 * nzA)) ? I->pmlzh[3 * kk + cc] : id;
                }
            }
            for (int q = threadIdx.x; q < LX; q += NT) {
                const int ii = d.li0 + q;
                for (int cc = 0; cc < 3; ++cc) {
                    const R id = R(cc == 1 ? 0 : 1);
                    prx[q * 6 + cc] = (ii >= 0 && ii < nx && ORF_IN(3 * ii + cc, 3 * nx)) ? I->pmlx[3 * ii + cc] : id;
                    prx[q * 6 + 3 + cc] =
                        (ii >= 0 && ii < nx - 1 && ORF_IN(3 * ii + cc, 3 * (nx - 1))) ? I->pmlxh[3 * ii + cc] : id;
                }
            }
        }
        // shared buffer -> registers: fields and update coefficients
        // (TE: K0 = C/eps of P; TM: K0 = C/eps of A, K1 = C/eps of B)
        R P[KS], A[KS], B[KS], K0[KS], K1[KS];
#pragma unroll
        for (int j = 0; j < KS; ++j) {
            const int c = (ck0 + j) * LX + cx;
            P[j] = pfP[c];
            A[j] = pfA[c];
            B[j] = pfB[c];
            int v0 = (int)pfI[c];
            // a material index outside the table is a fault wherever it lies:
            // the loaded window holds cells of the grid, its zero padding or
            // zero fill, whose index is 0
            if (!ORF_IN(v0, max(I->nlut, 1))) v0 = 0;
            K0[j] = sizeof(IT) == 1 ? slut[v0] : __ldg(I->lutc + v0);
            if (!TE) {
                int v1 = (int)pfI[CELLS + c];
                if (!ORF_IN(v1, max(I->nlut, 1))) v1 = 0;
                K1[j] = sizeof(IT) == 1 ? slut[v1] : __ldg(I->lutc + v1);
            } else {
                K1[j] = R(0);
            }
        }
        __syncthreads();   // shared buffer free; sg and CPML state ready
        if (tn < ntiles) {
            prefetch(s_desc[ns]);
            fetch_state(ns);
            fetch_desc(tn + gridDim.x, nns);
        }
        cp_commit();

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
            R pxb = R(1), pxa = R(0), pxk = R(1), phb = R(1), pha = R(0), phk = R(1);
            if (PML) {
                pxb = prx[cx * 6 + 0]; pxa = prx[cx * 6 + 1]; pxk = prx[cx * 6 + 2];
                phb = prx[cx * 6 + 3]; pha = prx[cx * 6 + 4]; phk = prx[cx * 6 + 5];
            }
            // the fused steps, specialised on the CPML axes the tile reaches
            // (frame tiles: flags 16 = z slab, 8 = x slab); skipping an axis
            // the tile does not reach leaves every value unchanged
            auto steps = [&](auto zc, auto xc) {
                constexpr bool ZC = PML && decltype(zc)::value;
                constexpr bool XC = PML && decltype(xc)::value;
                for (int s = 0; s < nsub; ++s) {
                    // ----- H half step: A (d/dz P), B (d/dx P)
                    if (lane == 0) store_row<R, KS>(&xPc[warp][0], P);
                    xPr[warp][lane] = P[0];
                    __syncthreads();
                    R Pdn = xPr[wDn][lane];
                    if (!hasDn) Pdn = PML ? R(0) : P[KS - 1];
                    constexpr int VEC = 16 / sizeof(R);
                    static_assert(KS % VEC == 0, "KS must be a multiple of 16 bytes of R");
                    R pe[VEC];
    #pragma unroll
                    for (int j = 0; j < KS; ++j) {
                        const int c = (ck0 + j) * LX + cx;
                        if (j % VEC == 0) load16<R>(pe, &xPc[wR][j]);
                        R pr = __shfl_down_sync(FULL, P[j], 1);
                        const R pej = (PML && !hasR) ? R(0) : pe[j % VEC];
                        pr = (lane == 31) ? pej : pr;
                        const R pk = (j + 1 < KS) ? P[j + 1] : Pdn;
                        R dz = pk - P[j];
                        R dx = pr - P[j];
                        if (ZC) {
                            const R* pz = prz + (ck0 + j) * 6;
                            const R ps = fma(pz[3], psA[c], pz[4] * dz);
                            psA[c] = ps;
                            dz = kUnitKappa ? dz + ps : fma(dz, pz[5], ps);
                        }
                        if (XC) {
                            const R qs = fma(phb, psB[c], pha * dx);
                            psB[c] = qs;
                            dx = kUnitKappa ? dx + qs : fma(dx, phk, qs);
                        }
                        const R ca = TE ? C : K0[j];
                        const R cb = TE ? C : K1[j];
                        if (PML) {
                            if ((mA >> j) & 1u) A[j] = fma(ca, dz, A[j]);
                            if ((mB >> j) & 1u) B[j] = fma(-cb, dx, B[j]);
                        } else {
                            A[j] = fma(ca, dz, A[j]);
                            B[j] = fma(-cb, dx, B[j]);
                        }
                    }
                    // (an interior tile has no row masks, and its loaded rows
                    // may run past the grid's last row: the source profile is
                    // read for grid rows only)
                    if (hs && i == six - 1) {   // TF/SF: the B column left of the plane is scattered field
                        const R ge = (R)sg[0][s];
    #pragma unroll
                        for (int j = 0; j < KS; ++j) {
                            const int kk = d.periodic ? pmod(kb + j, nz) : kb + j;
                            if (((mB >> j) & 1u) && kk >= 0 && kk < nz && ORF_IN(kk, nz))
                                B[j] = fma(__ldg(I->srcB + kk), ge, B[j]);
                        }
                    }
                    // ----- E half step: P (branch-free stencil loop)
                    if (lane == 31) store_row<R, KS>(&xBc[warp][0], B);
                    xAr[warp][lane] = A[KS - 1];
                    __syncthreads();
                    R Aup = xAr[wUp][lane];
                    if (!hasUp) Aup = PML ? R(0) : A[0];
                    R be[VEC];
    #pragma unroll
                    for (int j = 0; j < KS; ++j) {
                        const int c = (ck0 + j) * LX + cx;
                        if (j % VEC == 0) load16<R>(be, &xBc[wL][j]);
                        R bl = __shfl_up_sync(FULL, B[j], 1);
                        const R bej = (PML && !hasL) ? R(0) : be[j % VEC];
                        bl = (lane == 0) ? bej : bl;
                        const R am = (j > 0) ? A[j - 1] : Aup;
                        R da = A[j] - am;
                        R db = B[j] - bl;
                        if (ZC) {
                            const R* pz = prz + (ck0 + j) * 6;
                            const R ps = fma(pz[0], psPz[c], pz[1] * da);
                            psPz[c] = ps;
                            da = kUnitKappa ? da + ps : fma(da, pz[2], ps);
                        }
                        if (XC) {
                            const R qs = fma(pxb, psPx[c], pxa * db);
                            psPx[c] = qs;
                            db = kUnitKappa ? db + qs : fma(db, pxk, qs);
                        }
                        const R cp = TE ? K0[j] : C;
                        if (PML) {
                            if ((mP >> j) & 1u) P[j] = fma(cp, da - db, P[j]);
                        } else {
                            P[j] = fma(cp, da - db, P[j]);
                        }
                    }
                    // rare paths, each behind a tile-uniform flag
                    if (hs && i == six) {   // TF/SF: the plane is total field
                        const R gh = (R)sg[1][s];
    #pragma unroll
                        for (int j = 0; j < KS; ++j) {
                            const int kk = d.periodic ? pmod(kb + j, nz) : kb + j;
                            if (((mP >> j) & 1u) && kk >= 0 && kk < nz && ORF_IN(kk, nz))
                                P[j] = fma(__ldg(I->srcP + kk), gh, P[j]);
                        }
                    }
                    if (d.flags & 6) {      // DFT monitor samples of this step
                        const int sslot = launch_off + s;
                        R* smp0 = I->samples + (size_t)sslot * I->sstride;
    #pragma unroll
                        for (int j = 0; j < KS; ++j) {
                            if (j % VEC == 0) load16<R>(be, &xBc[wL][j]);
                            R bl = __shfl_up_sync(FULL, B[j], 1);
                            const R bej = (PML && !hasL) ? R(0) : be[j % VEC];
                            bl = (lane == 0) ? bej : bl;
                            if (xm >= 0 && ((own >> j) & 1u)) {
                                R* smp = smp0 + (size_t)xm * 2 * nz;
                                if (ORF_IN((size_t)sslot * I->sstride + (size_t)xm * 2 * nz + nz + kb + j,
                                           (size_t)kChunk * I->sstride)) {
                                    smp[kb + j] = P[j];
                                    smp[nz + kb + j] = R(0.5) * (bl + B[j]);
                                }
                            }
                            if ((zmask >> j) & 1u) {
                                const R am = (j > 0) ? A[j - 1] : Aup;
                                for (int m = 0; m < I->nmonz; ++m) {
                                    if (I->monz[m] != kb + j) continue;
                                    R* smp = smp0 + (size_t)I->nmon * 2 * nz + (size_t)m * 2 * d.nx;
                                    if (!ORF_IN((size_t)sslot * I->sstride + (size_t)I->nmon * 2 * nz +
                                                    (size_t)m * 2 * d.nx + d.nx + i,
                                                (size_t)kChunk * I->sstride))
                                        continue;
                                    smp[i] = P[j];
                                    smp[d.nx + i] = R(0.5) * (am + A[j]);
                                }
                            }
                        }
                    }
                }
            };
            if constexpr (!PML) {
                steps(Flag<false>{}, Flag<false>{});
            } else {
                const bool zc = (d.flags & 16) != 0, xc = (d.flags & 8) != 0;
                if (zc && xc) steps(Flag<true>{}, Flag<true>{});
                else if (zc) steps(Flag<true>{}, Flag<false>{});
                else if (xc) steps(Flag<false>{}, Flag<true>{});
                else steps(Flag<false>{}, Flag<false>{});
            }
            // ----- energy on the chunk's last launch
            if (want_energy) {
                double e = 0.0;
#pragma unroll
                for (int j = 0; j < KS; ++j) {
                    if ((own >> j) & 1u) {
                        const size_t o = (size_t)(kb + j) * d.pitch + i;
                        if (!(ORF_IN(i, d.nx) && ORF_IN(kb + j, nz))) continue;
                        const double p = P[j], a = A[j], b = B[j];
                        const int v0 = (int)reinterpret_cast<const IT*>(d.idx0)[o];
                        if (TE) {
                            e += I->lute[v0] * p * p + a * a + b * b;
                        } else {
                            const int v1 = (int)reinterpret_cast<const IT*>(d.idx1)[o];
                            e += p * p + (((mA >> j) & 1u) ? I->lute[v0] * a * a : 0.0) +
                                 (((mB >> j) & 1u) ? I->lute[v1] * b * b : 0.0);
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
            // ----- store the output rectangle (owned rows never wrap)
            R* __restrict__ Pout = reinterpret_cast<R*>(const_cast<void*>(d.f[par ^ 1][0]));
            R* __restrict__ Aout = reinterpret_cast<R*>(const_cast<void*>(d.f[par ^ 1][1]));
            R* __restrict__ Bout = reinterpret_cast<R*>(const_cast<void*>(d.f[par ^ 1][2]));
#pragma unroll
            for (int j = 0; j < KS; ++j) {
                if ((own >> j) & 1u) {
                    const size_t o = (size_t)(kb + j) * d.pitch + i;
                    // an owned cell must be a cell of the grid
                    if (!(ORF_IN(i, d.nx) && ORF_IN(kb + j, nz))) continue;
                    Pout[o] = P[j];
                    Aout[o] = A[j];
                    Bout[o] = B[j];
                }
            }
            if (PML) {
                const int npx = I->npx, npz = I->npz, nx = d.nx;
                R* __restrict__ gA = I->psiA[par ^ 1];
                R* __restrict__ gB = I->psiB[par ^ 1];
                R* __restrict__ gPx = I->psiPx[par ^ 1];
                R* __restrict__ gPz = I->psiPz[par ^ 1];
#pragma unroll
                for (int j = 0; j < KS; ++j) {
                    if (!((own >> j) & 1u)) continue;
                    const int c = (ck0 + j) * LX + cx;
                    const int kk = kb + j;
                    const int szA = slab_half(kk, nz, npz);
                    const int szP = slab_int(kk, nz, npz);
                    if (szA >= 0 && ORF_IN((size_t)szA * nx + i, (size_t)2 * npz * nx)) gA[(size_t)szA * nx + i] = psA[c];
                    if (szP >= 0 && ORF_IN((size_t)szP * nx + i, (size_t)2 * npz * nx)) gPz[(size_t)szP * nx + i] = psPz[c];
                    if (sxP >= 0 && ORF_IN((size_t)kk * (2 * npx) + sxP, (size_t)nz * 2 * npx))
                        gPx[(size_t)kk * (2 * npx) + sxP] = psPx[c];
                    if (sxB >= 0 && ORF_IN((size_t)kk * (2 * npx) + sxB, (size_t)nz * 2 * npx))
                        gB[(size_t)kk * (2 * npx) + sxB] = psB[c];
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
