// step3d_fused.cu -- one 3D Yee time step per launch, H and E fused in a z-march
// (toolbox/+orf/fdtd3D.m:1-29) for sm_100a.
//
//   H_c -= C (D+_c1 E_c2 - D+_c2 E_c1),   E_c += C/eps_c (D-_c1 H_c2 - D-_c2 H_c1)
// with CPML on any axis (cpmlCoefficients.m:4-8), PEC or periodic boundaries,
// the one-sided TF/SF plane on any axis (fdtd3D.m:15-21) and planar DFT
// monitors with H averaged onto the E plane (fdtd3D.m:22, 26-28).
//
// A CTA owns a 32 x 8 column tile and a segment [k0, k1) of z planes and
// marches it plane by plane:
//   - plane p of E (the tile plus one halo cell on every side), H and the
//     material index arrive in a shared-memory ring (4 slots FP32, 3 FP64),
//     ahead of the plane being updated: one thread issues TMA tensor copies
//     (cp.async.bulk.tensor, x window [i0-4, i0+36) so the start stays 16-byte
//     aligned, zero fill outside the grid) completing on one mbarrier per
//     slot; tiles whose halo wraps around a periodic x / y edge fill the same
//     layout with per-element cp.async instead;
//   - H at plane k is updated on the tile plus its low x / y halo (the halo
//     values are recomputed, not read from the neighbour CTA, whose update of
//     them may not have happened yet) into a shared plane; the tile's own H
//     goes to global memory;
//   - E at plane k is then updated from that plane and the H of plane k-1,
//     which each thread keeps in registers from the previous iteration.
// Fields, and CPML psi, ping-pong between two buffers (read par, write
// par^1), so CTAs never see each other's partial results.  Each field is read
// and written once per step: 12 values plus 3 index bytes per cell, the
// algorithmic minimum.  The arithmetic of every update is that of the split
// H-then-E formulation, operation for operation.
#include <type_traits>

#include "orf_internal.cuh"

namespace orf {
namespace {

constexpr int TX = kTile3X, TY = kTile3Y, NT = TX * TY;
constexpr int RX = TX + 2, RY = TY + 2, RC = RX * RY;   // E region [i0-1, i0+TX] x [j0-1, j0+TY]
constexpr int SX = TX + 8;                                // smem row: x in [i0-4, i0+TX+4)
constexpr int CX = 3;                                     // smem column of x = i0-1
template <class R>
constexpr int NS = sizeof(R) == 4 ? 4 : 3;               // planes in the ring (FP64: 3, for occupancy)
constexpr int RPT = (RC + NT - 1) / NT;                   // region cells per thread
constexpr long long kSpinMax = 1ll << 20;                 // bounded mbarrier wait: at most this many polls,
constexpr unsigned long long kWaitNsDefault = 1000000000ull;   // and at most this long (ns) per plane
constexpr int kIssuer = NT - 32;   // issues the TMA copies and polls their mbarriers: lane 0 of the
                                   // last warp, which has no halo H cell to recompute

// per-slot layout (elements of R, each block 128-byte aligned for TMA)
template <class R>
constexpr int rnd128(int n) {
    return (int)((((size_t)n * sizeof(R) + 127) / 128) * 128 / sizeof(R));
}
template <class R>
constexpr int EB = rnd128<R>(SX * RY);        // one E component: [RY][SX]
template <class R>
constexpr int HB = rnd128<R>(SX * (RY - 1));  // one H component: [RY-1][SX]

__device__ __forceinline__ int wrapc(int u, int n, bool per, bool* ok) {
    if (u >= 0 && u < n) {
        *ok = true;
        return u;
    }
    if (per) {
        *ok = true;
        const int r = u % n;
        return r < 0 ? r + n : r;
    }
    *ok = false;
    return 0;
}

__device__ __forceinline__ int sel3(int a, int x, int y, int z) { return a == 0 ? x : (a == 1 ? y : z); }

__device__ __forceinline__ int slab(bool half, int u, int n, int np) {
    if (np <= 0) return -1;
    if (u < np) return u;
    const int hi = half ? n - 1 - np : n - np;
    return u >= hi ? np + (u - hi) : -1;
}

// CPML context of one instance, staged in shared memory by the CPML launches
// so that a stretched difference costs one psi load, not a chain of
// dependent descriptor loads.  kind 0: E update (integer positions, psiE),
// kind 1: H update (half positions, psiH).
template <class R>
struct Cpml3 {
    const R* prof[2][3];        // (b, a, 1/kappa) per coordinate, per axis
    const R* pin[2][3][3];      // psi of (component, axis), buffer par (read)
    R* pout[2][3][3];           // the same, buffer par^1 (written)
    int n[3], np[3], nsl[2][3];
    const R* zp[2];             // z profile of the segment's planes zk0 .. in shared memory
    int zk0;
};

// The six differences of one cell's H or E update, in the order
// (c, q) = (0,1) (0,2) (1,2) (1,0) (2,0) (2,1): component c, derivative axis q.
// CPML stretch d -> d/kappa + psi, psi <- b psi + a d (reading buffer par,
// writing par^1 when store) of those on an absorbing slab of their axis,
// axis by axis: the two psi loads of an axis are issued together, and a cell
// on the slab of a single axis (all but the slab corners) has all its psi
// loads in flight at once.  psi of buffer par is read-only during the launch.
// zpre: z0, z1 are this cell's two z-axis psi values, loaded ahead by the
// caller (the same values the loads here would return).
template <class R>
__device__ __forceinline__ void cpml6(const Cpml3<R>& X, int kind, bool store, int i, int j, int k, R (&d)[6],
                                      bool zpre = false, R z0 = R(0), R z1 = R(0)) {
    const bool half = kind == 1;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const int coord = q == 0 ? i : (q == 1 ? j : k);
        const int sl = slab(half, coord, X.n[q], X.np[q]);
        if (sl < 0) continue;
        // the entries on axis q: (component c1, entry e1), (c2, e2)
        constexpr int E1[3] = {3, 0, 1}, E2[3] = {4, 5, 2};
        constexpr int C1[3] = {1, 0, 0}, C2[3] = {2, 2, 1};
        const int v0 = q == 0 ? sl : i, v1 = q == 1 ? sl : j, v2 = q == 2 ? sl : k;
        const int d0 = q == 0 ? X.nsl[kind][0] : X.n[0], d1 = q == 1 ? X.nsl[kind][1] : X.n[1];
        const size_t o = (size_t)v0 + (size_t)d0 * ((size_t)v1 + (size_t)d1 * v2);
        const bool zs = q == 2 && X.zp[kind] != nullptr;   // z profile staged in shared memory
        const R* pr = zs ? X.zp[kind] + 3 * (coord - X.zk0) : X.prof[kind][q] + 3 * coord;
        R ps1, ps2;
        if (q == 2 && zpre) {
            ps1 = z0;
            ps2 = z1;
        } else {
            ps1 = __ldg(X.pin[kind][C1[q]][q] + o);
            ps2 = __ldg(X.pin[kind][C2[q]][q] + o);
        }
        R b, a, ki = R(1);
        if (zs) {
            b = pr[0];
            a = pr[1];
            if (!kUnitKappa) ki = pr[2];
        } else {
            b = __ldg(pr);
            a = __ldg(pr + 1);
            if (!kUnitKappa) ki = __ldg(pr + 2);
        }
        const R p1 = b * ps1 + a * d[E1[q]];
        const R p2 = b * ps2 + a * d[E2[q]];
        if (store) {
            X.pout[kind][C1[q]][q][o] = p1;
            X.pout[kind][C2[q]][q][o] = p2;
        }
        d[E1[q]] = kUnitKappa ? d[E1[q]] + p1 : d[E1[q]] * ki + p1;
        d[E2[q]] = kUnitKappa ? d[E2[q]] + p2 : d[E2[q]] * ki + p2;
    }
}

__device__ __forceinline__ void cp4(void* sdst, const void* gsrc, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gsrc), "r"(valid ? 4u : 0u) : "memory");
}
__device__ __forceinline__ void cp8(void* sdst, const void* gsrc, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gsrc), "r"(valid ? 8u : 0u) : "memory");
}
template <class R>
__device__ __forceinline__ void cpR(R* sdst, const R* gsrc, bool valid) {
    if constexpr (sizeof(R) == 4) cp4(sdst, gsrc, valid);
    else cp8(sdst, gsrc, valid);
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// FP32 CPML kernels carry the four z-axis psi planes of a cell's H and E
// updates in the ring too (ZR); FP64 ones load them from global memory
template <class R, bool PML>
constexpr bool kZRing = PML && sizeof(R) == 4;
template <class R, class IT, bool ZR>
constexpr size_t slot_bytes() {   // 3 E blocks, 3 H blocks, 3 index blocks (+ 4 psi blocks)
    return 3 * (size_t)EB<R> * sizeof(R) + 3 * (size_t)HB<R> * sizeof(R) + 3 * (size_t)NT * sizeof(IT) +
           (ZR ? 4 * (size_t)EB<R> * sizeof(R) : 0);
}
template <class R, class IT, bool ZR>
constexpr size_t smem_bytes() {   // the ring, then the new-H plane, + 128 for alignment
    return NS<R> * slot_bytes<R, IT, ZR>() + 3 * (size_t)EB<R> * sizeof(R) + 128;
}

__device__ __forceinline__ unsigned sm_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned cnt) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(sm_addr(b)), "r"(cnt) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(sm_addr(b)), "r"(bytes) : "memory");
}
// try_wait with a suspend-time hint: the polling thread sleeps until the
// phase completes or about hint_ns pass, instead of re-issuing the poll
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* b, unsigned parity, unsigned hint_ns) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(sm_addr(b)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;\n" : "=l"(t));
    return t;
}
// Wait for the phase of parity `parity` of mbarrier b to complete, giving up
// after kSpinMax polls or limit_ns nanoseconds; true when it completed.
constexpr unsigned kPollHintNs = 20000;   // longest sleep of one poll
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* b, unsigned parity,
                                                  unsigned long long limit_ns) {
    if (mbar_try_wait(b, parity, kPollHintNs)) return true;
    const unsigned long long t0 = global_ns();
    for (long long spins = 1; spins < kSpinMax; ++spins) {
        if (mbar_try_wait(b, parity, kPollHintNs)) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
    return false;
}

// 3D tiled TMA load of the box at (x, y, z) into shared memory, completing on b
__device__ __forceinline__ void tma_load3(void* sdst, const void* tmap, int x, int y, int z, unsigned long long* b) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(sm_addr(sdst)),
        "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(sm_addr(b))
        : "memory");
}

// H update of one cell (the split formulation's operations, in order)
template <bool PML, class R>
__device__ __forceinline__ void h_cell(const Inst3D<R>* __restrict__ I, const Cpml3<R>& X, bool store, int i, int j,
                                       int k, R ex, R ey, R ez, R ex_k, R ey_k, R ez_i, R ey_i, R ez_j, R ex_j, R& hx,
                                       R& hy, R& hz, R gE, bool src, bool zpre = false, R z0 = R(0),
                                       R z1 = R(0)) {
    const R C = I->C;
    // Hx -= C ((Ez(j+1) - Ez) - (Ey(k+1) - Ey))
    // Hy -= C ((Ex(k+1) - Ex) - (Ez(i+1) - Ez))
    // Hz -= C ((Ey(i+1) - Ey) - (Ex(j+1) - Ex))
    R dd[6] = {ez_j - ez, ey_k - ey, ex_k - ex, ez_i - ez, ey_i - ey, ex_j - ex};
    if (PML) cpml6(X, 1, store, i, j, k, dd, zpre, z0, z1);
    hx = hx - C * (dd[0] - dd[1]);
    hy = hy - C * (dd[2] - dd[3]);
    hz = hz - C * (dd[4] - dd[5]);
    // TF/SF: the H plane just below the source plane is scattered field
    // (src: sel3(sa, i, j, k) == ss - 1)
    if (src) {
        const int sa = I->sa;
        const int sb = (sa + 1) % 3, sc = (sa + 2) % 3;
        const size_t pq = (size_t)sel3(sb, i, j, k) + (size_t)I->na * sel3(sc, i, j, k);
        const R ua = __ldg(I->sHa + pq) * gE, ub = __ldg(I->sHb + pq) * gE;
        if (sa == 0) { hy += ua; hz += ub; }
        else if (sa == 1) { hz += ua; hx += ub; }
        else { hx += ua; hy += ub; }
    }
}

template <class R, class IT>
__device__ __forceinline__ R coef(const R* slut, const R* __restrict__ lutc, int v) {
    if constexpr (sizeof(IT) == 1) return slut[v];
    else return __ldg(lutc + v);
}

// Resident CTAs per SM: FP32 4 (interior) / 3 (CPML: the psi and profile
// values loaded ahead need the registers), FP64 3.
template <class R, class IT, bool PML>
__global__ void __launch_bounds__(NT, sizeof(R) == 4 ? (PML ? 3 : 4) : 3)
k_step3d(const Inst3D<R>* __restrict__ insts, const Tile3D* __restrict__ tiles, int par, int launch_off,
         int want_energy, WaitCtl wc) {
    const Tile3D tile = tiles[blockIdx.x];
    const Inst3D<R>* __restrict__ I = insts + tile.inst;
    JobState* st = I->st;
    if (st->done || st->fault) return;   // finished, or an earlier launch gave up a wait
    const long long n = st->step + launch_off;
    if (n >= st->nmax) return;

    extern __shared__ __align__(128) unsigned char dsm_raw[];
    // TMA destinations must be 128-byte aligned: align the base explicitly
    // (the launch requests 128 spare bytes)
    unsigned char* dsm = dsm_raw + ((128u - (sm_addr(dsm_raw) & 127u)) & 127u);
    constexpr int EBr = EB<R>, HBr = HB<R>;
    constexpr bool ZR = kZRing<R, PML>;
    constexpr size_t SB = slot_bytes<R, IT, ZR>();
    // slot s: E component q at sEq(s, q), H at sHq(s, q), index at sIq(s, q);
    // region cell (r, c) (x = i0-1+c, y = j0-1+r) at r * SX + c + CX
    auto sEq = [&](int s2, int q) { return reinterpret_cast<R*>(dsm + s2 * SB) + q * EBr; };
    auto sHq = [&](int s2, int q) { return reinterpret_cast<R*>(dsm + s2 * SB) + 3 * EBr + q * HBr; };
    auto sIq = [&](int s2, int q) {
        return reinterpret_cast<IT*>(dsm + s2 * SB + 3 * (EBr + HBr) * sizeof(R)) + q * NT;
    };
    // ZR: z psi block q of slot s (0, 1: psiH of Hx, Hy; 2, 3: psiE of Ex, Ey), the E layout
    auto sZq = [&](int s2, int q) {
        return reinterpret_cast<R*>(dsm + s2 * SB + 3 * (EBr + HBr) * sizeof(R) + 3 * NT * sizeof(IT)) + q * EBr;
    };
    constexpr int ns = NS<R>;
    R* sHn = reinterpret_cast<R*>(dsm + ns * SB);      // [3][EB]
    __shared__ R slut[sizeof(IT) == 1 ? 256 : 1];
    __shared__ __align__(8) unsigned long long sbar[ns];
    __shared__ Cpml3<R> sx;
    __shared__ int s_abort;   // set by the issuer when a plane wait runs out
    // planes the issuer has armed (TMA) and the last one whose wait completed
    // (the planes in between are in flight); only the issuer touches them
    __shared__ int s_issued, s_waited;

    const int t = threadIdx.x;
    if (PML && t < 18) {   // CPML context: thread (kind, c, q) copies one psi pair
        const int kind = t / 9, c = (t / 3) % 3, q = t % 3;
        sx.pin[kind][c][q] = kind ? I->psiH[par][c][q] : I->psiE[par][c][q];
        sx.pout[kind][c][q] = kind ? I->psiH[par ^ 1][c][q] : I->psiE[par ^ 1][c][q];
        if (c == 0) {
            sx.prof[kind][q] = kind ? I->pmlH[q] : I->pmlI[q];
            sx.nsl[kind][q] = kind ? I->nslabH[q] : I->nslabI[q];
            if (kind == 0) {
                sx.n[q] = I->n[q];
                sx.np[q] = I->np[q];
            }
        }
    }
    const int tx = t % TX, ty = t / TX;
    const int nx = I->n[0], ny = I->n[1], nz = I->n[2], pitch = I->pitch;
    const bool px = I->per[0] != 0, py = I->per[1] != 0, pz = I->per[2] != 0;
    const size_t plane = (size_t)ny * pitch;
    const int i0 = tile.i0, j0 = tile.j0, k0 = tile.k0, k1 = tile.k1;
    const R* __restrict__ Ein[3] = {I->E[par][0], I->E[par][1], I->E[par][2]};
    const R* __restrict__ Hin[3] = {I->H[par][0], I->H[par][1], I->H[par][2]};

    if constexpr (sizeof(IT) == 1) slut[t] = I->lutc[t];

    // TMA for tiles whose halo does not wrap around a periodic edge
    const bool wrapx = px && (i0 == 0 || i0 + TX >= nx), wrapy = py && (j0 == 0 || j0 + TY >= ny);
    const bool use_tma = I->tmap != nullptr && !wrapx && !wrapy;
    const char* tm = reinterpret_cast<const char*>(I->tmap);
    constexpr unsigned kTx = (unsigned)(3 * SX * RY * sizeof(R) + 3 * SX * (RY - 1) * sizeof(R) + 3 * NT * sizeof(IT));
    if (t == 0) s_abort = 0;
    if (t == kIssuer) s_issued = s_waited = k0 - 1;
    if (use_tma && t == 0) {
        for (int q = 0; q < ns; ++q) mbar_init(&sbar[q], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
    __syncthreads();
    // CPML tiles: the z profile (b, a, 1/kappa) of planes k0-1 .. k1 in shared
    // memory, the entry every cell of a plane reads
    __shared__ R szp[PML ? 2 : 1][PML ? 3 * (kSeg3 + 2) : 1];
    const int np2 = PML ? sx.np[2] : 0;
    // FP32 CPML tiles with a z slab on the TMA path take the z-axis psi of
    // their cells through the ring as well (slab planes of the psi arrays)
    const bool zring = ZR && use_tma && I->tma_psi != 0 && np2 > 0;
    const unsigned tx_bytes = kTx + (zring ? 4u * (unsigned)(SX * RY * sizeof(R)) : 0u);
    if constexpr (PML) {
        const int cnt = k1 - k0 + 2;
        if (np2 > 0) {
            for (int q = t; q < 6 * cnt; q += NT) {
                const int kind = q / (3 * cnt), r = q - kind * 3 * cnt, c = r / 3 + k0 - 1, f = r - 3 * (r / 3);
                szp[kind][r] = (c >= 0 && c < nz) ? sx.prof[kind][2][3 * c + f] : R(f == 1 ? 0 : 1);
            }
        }
        __syncthreads();   // every thread has read sx.np
        if (t == 0) {
            sx.zk0 = k0 - 1;
            sx.zp[0] = np2 > 0 ? &szp[0][0] : nullptr;
            sx.zp[1] = np2 > 0 ? &szp[1][0] : nullptr;
        }
        __syncthreads();
    }

    // ---- region addressing for the cp.async path, the same for every plane
    size_t roff[RPT];
    unsigned rmask = 0;
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int e = t + NT * r;
        roff[r] = 0;
        if (e < RC) {
            const int rr = e / RX, c = e % RX;
            bool iok, jok;
            const int ii = wrapc(i0 - 1 + c, nx, px, &iok), jj = wrapc(j0 - 1 + rr, ny, py, &jok);
            roff[r] = (size_t)jj * pitch + ii;
            if (iok && jok) rmask |= 1u << r;
        }
    }
    // material index of the tile's own cells: 4-byte words of its rows
    constexpr int WPR = TX * (int)sizeof(IT) / 4;   // words per row
    constexpr int NWI = 3 * TY * WPR;

    const unsigned long long wait_ns = wc.wait_ns ? wc.wait_ns : kWaitNsDefault;
    // ---- plane p (wrapped or zero outside the grid) into slot s
    auto load_plane = [&](int p, int s2) {
        bool pok;
        const int pw = wrapc(p, nz, pz, &pok);
        if (use_tma) {
            if (t == kIssuer) {
                const int zc = pok ? pw : -1;   // z = -1: the whole box reads as zero
                // order the block's earlier generic reads of this slot before the async writes
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                mbar_expect_tx(&sbar[s2], tx_bytes);
                s_issued = p;
                // failure-detection test hook (off unless set on the host):
                // the slot is armed but its copies are never issued
                if (wc.stall_plane >= 0 && p == k0 + wc.stall_plane) return;
                for (int q = 0; q < 3; ++q) {
                    tma_load3(sEq(s2, q), tm + 128 * (3 * par + q), i0 - 4, j0 - 1, zc, &sbar[s2]);
                    tma_load3(sHq(s2, q), tm + 128 * (6 + 3 * par + q), i0 - 4, j0 - 1, zc, &sbar[s2]);
                    tma_load3(sIq(s2, q), tm + 128 * (12 + q), i0, j0, zc, &sbar[s2]);
                }
                if (zring) {   // slab plane of the psi arrays, or z = -1 (zeros) off the slab
                    const int zh = pok ? slab(true, pw, nz, np2) : -1;
                    const int ze = pok ? slab(false, pw, nz, np2) : -1;
                    for (int c = 0; c < 2; ++c) {
                        tma_load3(sZq(s2, c), tm + 128 * (15 + 2 * par + c), i0 - 4, j0 - 1, zh, &sbar[s2]);
                        tma_load3(sZq(s2, 2 + c), tm + 128 * (19 + 2 * par + c), i0 - 4, j0 - 1, ze, &sbar[s2]);
                    }
                }
            }
            return;
        }
        const size_t po = (size_t)pw * plane;
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int e = t + NT * r;
            if (e >= RC) break;
            const bool v = pok && ((rmask >> r) & 1u);
            const size_t o = po + roff[r];
            const int rr = e / RX, c = e - rr * RX;
            const int se = rr * SX + c + CX;
#pragma unroll
            for (int q = 0; q < 3; ++q) cpR<R>(sEq(s2, q) + se, Ein[q] + o, v);
            if (rr < RY - 1 && c < RX - 1) {
#pragma unroll
                for (int q = 0; q < 3; ++q) cpR<R>(sHq(s2, q) + se, Hin[q] + o, v);
            }
        }
        for (int w = t; w < NWI; w += NT) {
            const int q = w / (TY * WPR), r = (w / WPR) % TY, cw = w % WPR;
            const int jj = j0 + r;
            const bool v = pok && jj < ny;
            const size_t o = (po + (size_t)(v ? jj : 0) * pitch + i0) * sizeof(IT) + 4 * (size_t)cw;
            cp4(reinterpret_cast<unsigned char*>(sIq(s2, q)) + (size_t)r * TX * sizeof(IT) + 4 * cw,
                reinterpret_cast<const unsigned char*>(I->idx[q]) + o, v);
        }
    };
    // wait for plane p in slot s (TMA: the issuer polls its mbarrier, the
    // barrier that follows orders the data for everyone; cp.async: each
    // thread's own groups, made visible by the same barrier)
    bool timed_out = false;
    auto wait_plane = [&](int p, int s2) {
        if (use_tma) {
            if (t != kIssuer || timed_out) return;
            const unsigned parity = (unsigned)(((p - k0) / ns) & 1);
            if (mbar_wait_bounded(&sbar[s2], parity, wait_ns)) {
                s_waited = p;
            } else {
                timed_out = true;
                s_abort = 1;   // read by every thread after the next barrier
            }
        } else {
            cp_wait<ns - 3>();   // all but the planes issued after p
        }
    };

    // planes k0 .. k0+ns-2 (a segment reads planes up to k1)
    for (int q = 0; q < ns - 1; ++q) {
        if (k0 + q <= k1) load_plane(k0 + q, q);
        cp_commit();
    }

    const R gE = (R)(n < I->nsrc ? I->gE[n] : 0.0);
    const R gH = (R)(n < I->nsrc ? I->gH[n] : 0.0);
    const bool own = tx < tile.tw && ty < tile.th;
    const int i = i0 + tx, j = j0 + ty;
    R* __restrict__ Eout[3] = {I->E[par ^ 1][0], I->E[par ^ 1][1], I->E[par ^ 1][2]};
    R* __restrict__ Hout[3] = {I->H[par ^ 1][0], I->H[par ^ 1][1], I->H[par ^ 1][2]};

    // ---- H of plane k0-1 at the own column (the E update of plane k0 needs
    // its x and y components); recomputed here, never stored
    R hxm = R(0), hym = R(0);
    if (own) {
        bool kok;
        const int km = wrapc(k0 - 1, nz, pz, &kok);
        if (kok) {
            bool iok, jok, kpk;
            const int ip = wrapc(i + 1, nx, px, &iok), jp = wrapc(j + 1, ny, py, &jok);
            const int kp = wrapc(km + 1, nz, pz, &kpk);
            const size_t o = (size_t)km * plane + (size_t)j * pitch + i;
            const size_t oi = (size_t)km * plane + (size_t)j * pitch + ip;
            const size_t oj = (size_t)km * plane + (size_t)jp * pitch + i;
            const size_t ok = (size_t)kp * plane + (size_t)j * pitch + i;
            const R ex = __ldg(Ein[0] + o), ey = __ldg(Ein[1] + o), ez = __ldg(Ein[2] + o);
            const R ex_k = kpk ? __ldg(Ein[0] + ok) : R(0), ey_k = kpk ? __ldg(Ein[1] + ok) : R(0);
            const R ez_i = iok ? __ldg(Ein[2] + oi) : R(0), ey_i = iok ? __ldg(Ein[1] + oi) : R(0);
            const R ez_j = jok ? __ldg(Ein[2] + oj) : R(0), ex_j = jok ? __ldg(Ein[0] + oj) : R(0);
            R hx = __ldg(Hin[0] + o), hy = __ldg(Hin[1] + o), hz = __ldg(Hin[2] + o);
            h_cell<PML>(I, sx, false, i, j, km, ex, ey, ez, ex_k, ey_k, ez_i, ey_i, ez_j, ex_j, hx, hy, hz, gE,
                        sel3(I->sa, i, j, km) == I->ss - 1);
            hxm = hx;
            hym = hy;
        }
    }

    // halo H cell of this thread (41 of them: row j0-1, then column i0-1)
    static_assert(kIssuer >= RX - 1 + TY, "the issuer warp has no halo cell");
    const bool hasHalo = t < RX - 1 + TY;
    const int hr = t < RX - 1 ? 0 : t - (RX - 1) + 1;
    const int hc = t < RX - 1 ? t : 0;
    bool hiok, hjok;
    const int hi = wrapc(i0 - 1 + hc, nx, px, &hiok), hj = wrapc(j0 - 1 + hr, ny, py, &hjok);
    const bool haloValid = hasHalo && hiok && hjok;
    const int eo = (ty + 1) * SX + (tx + 1) + CX;   // own cell in the region
    const int he = hr * SX + hc + CX;               // halo cell in the region

    // monitors this thread samples: x / y normal planes through its column
    // (every plane of the march), z normal planes (when k matches)
    unsigned mcol = 0, mz = 0;
    for (int m = 0; m < I->nmon; ++m) {
        const int ax = I->mon_axis[m], ix = I->mon_index[m];
        if (ax == 2) mz |= 1u << m;
        else if ((ax == 0 && i == ix) || (ax == 1 && j == ix)) mcol |= 1u << m;
    }
    // planes of the segment (k - k0 < kSeg3 <= 64) that carry a z normal monitor
    static_assert(kSeg3 <= 64, "one bit per plane of a segment");
    unsigned long long zpl = 0;
    for (unsigned b = mz; b; b &= b - 1) {
        const int dk = I->mon_index[__ffs(b) - 1] - k0;
        if (dk >= 0 && dk < k1 - k0) zpl |= 1ull << dk;
    }
    // the TF/SF plane: on an x / y plane a fixed set of columns, on a z plane
    // one plane of the march (sel3(sa, i, j, k) == ss - 1 for H, == ss for E)
    const int sa = I->sa, ss = I->ss;
    const int kSrcH = sa == 2 ? ss - 1 : -2, kSrcE = sa == 2 ? ss : -2;
    const bool ownSrcH = sa != 2 && sel3(sa, i, j, 0) == ss - 1;
    const bool ownSrcE = sa != 2 && sel3(sa, i, j, 0) == ss;
    const bool haloSrcH = sa != 2 && sel3(sa, hi, hj, 0) == ss - 1;
    double energy = 0.0;
    R* smp0 = I->samples + (size_t)launch_off * I->sstride;
    // CPML tiles with a z slab: the z-axis psi of the own and the halo cell's
    // H update are loaded a plane ahead, those of the own E update at the top
    // of the plane's iteration, so the loads overlap the barriers and the H
    // phase instead of stalling the update (psi of buffer par is read-only)
    // (FP32: in FP64 the values held ahead would spill at three CTAs per SM)
    const bool zpre = PML && sizeof(R) == 4 && np2 > 0 && !zring;
    const bool zgiven = zpre || zring;   // the z-axis psi reach cpml6 from outside
    R zHo0 = R(0), zHo1 = R(0), zHh0 = R(0), zHh1 = R(0), zEo0 = R(0), zEo1 = R(0);
    auto load_zH = [&](int p) {
        const int sl = slab(true, p, nz, np2);
        if (sl < 0) return;
        if (own) {
            const size_t o = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * sl);
            zHo0 = __ldg(sx.pin[1][0][2] + o);
            zHo1 = __ldg(sx.pin[1][1][2] + o);
        }
        if (haloValid) {
            const size_t o = (size_t)hi + (size_t)nx * ((size_t)hj + (size_t)ny * sl);
            zHh0 = __ldg(sx.pin[1][0][2] + o);
            zHh1 = __ldg(sx.pin[1][1][2] + o);
        }
    };
    auto load_zE = [&](int p) {
        const int sl = slab(false, p, nz, np2);
        if (sl < 0 || !own) return;
        const size_t o = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * sl);
        zEo0 = __ldg(sx.pin[0][0][2] + o);
        zEo1 = __ldg(sx.pin[0][1][2] + o);
    };
    // One plane of the march after its loads: H of plane k, then E.  SP: the
    // plane or the tile carries a TF/SF plane or a DFT monitor; in interior
    // tiles the other planes run a form without that code (same operations,
    // same bits).
    auto march_plane = [&](int k, int it, int s0, int s1, auto sp) {
        constexpr bool SP = decltype(sp)::value;
        const R* E0x = sEq(s0, 0);
        const R* E0y = sEq(s0, 1);
        const R* E0z = sEq(s0, 2);
        const R* E1x = sEq(s1, 0);
        const R* E1y = sEq(s1, 1);
        const R* H0x = sHq(s0, 0);
        const R* H0y = sHq(s0, 1);
        const R* H0z = sHq(s0, 2);
        // ---- H of plane k: the halo cell (its psi reads issued ahead of the
        // own cell's psi writes), then the own cell
        if (hasHalo) {
            const int e = he;
            R hx = R(0), hy = R(0), hz = R(0);
            if (haloValid) {
                hx = H0x[e];
                hy = H0y[e];
                hz = H0z[e];
                h_cell<PML>(I, sx, false, hi, hj, k, E0x[e], E0y[e], E0z[e], E1x[e], E1y[e], E0z[e + 1], E0y[e + 1],
                            E0z[e + SX], E0x[e + SX], hx, hy, hz, gE, SP && (haloSrcH || k == kSrcH), zgiven,
                            zring ? sZq(s0, 0)[e] : zHh0, zring ? sZq(s0, 1)[e] : zHh1);
            }
            sHn[e] = hx;
            sHn[EBr + e] = hy;
            sHn[2 * EBr + e] = hz;
        }
        // the own cell's E and new H stay in registers for the E update
        R exo = R(0), eyo = R(0), ezo = R(0), hxk = R(0), hyk = R(0), hzk = R(0);
        {
            const int e = eo;
            if (own) {
                exo = E0x[e];
                eyo = E0y[e];
                ezo = E0z[e];
                hxk = H0x[e];
                hyk = H0y[e];
                hzk = H0z[e];
                h_cell<PML>(I, sx, true, i, j, k, exo, eyo, ezo, E1x[e], E1y[e], E0z[e + 1], E0y[e + 1], E0z[e + SX],
                            E0x[e + SX], hxk, hyk, hzk, gE, SP && (ownSrcH || k == kSrcH), zgiven,
                            zring ? sZq(s0, 0)[e] : zHo0, zring ? sZq(s0, 1)[e] : zHo1);
                const size_t o = (size_t)k * plane + (size_t)j * pitch + i;
                Hout[0][o] = hxk;
                Hout[1][o] = hyk;
                Hout[2][o] = hzk;
            }
            sHn[e] = hxk;
            sHn[EBr + e] = hyk;
            sHn[2 * EBr + e] = hzk;
        }
        if (zpre && k + 1 < k1) load_zH(k + 1);   // consumed at the next plane's H phase
        __syncthreads();
        // ---- E of plane k at the own cell
        if (own) {
            const int e = eo;
            const R hy_i = sHn[EBr + e - 1], hz_i = sHn[2 * EBr + e - 1];
            const R hx_j = sHn[e - SX], hz_j = sHn[2 * EBr + e - SX];
            const int v0 = (int)sIq(s0, 0)[t], v1 = (int)sIq(s0, 1)[t], v2 = (int)sIq(s0, 2)[t];
            // Ex += cx ((Hz - Hz(j-1)) - (Hy - Hy(k-1)))
            // Ey += cy ((Hx - Hx(k-1)) - (Hz - Hz(i-1)))
            // Ez += cz ((Hy - Hy(i-1)) - (Hx - Hx(j-1)))
            R dd[6] = {hzk - hz_j, hyk - hym, hxk - hxm, hzk - hz_i, hyk - hy_i, hxk - hx_j};
            if (PML)
                cpml6(sx, 0, true, i, j, k, dd, zgiven, zring ? sZq(s0, 2)[e] : zEo0, zring ? sZq(s0, 3)[e] : zEo1);
            R ex = exo + coef<R, IT>(slut, I->lutc, v0) * (dd[0] - dd[1]);
            R ey = eyo + coef<R, IT>(slut, I->lutc, v1) * (dd[2] - dd[3]);
            R ez = ezo + coef<R, IT>(slut, I->lutc, v2) * (dd[4] - dd[5]);
            // TF/SF: the source plane is total field
            if (SP && (ownSrcE || k == kSrcE)) {
                const int sb = (sa + 1) % 3, sc = (sa + 2) % 3;
                const size_t pq = (size_t)sel3(sb, i, j, k) + (size_t)I->na * sel3(sc, i, j, k);
                const R ua = __ldg(I->sEa + pq) * gH, ub = __ldg(I->sEb + pq) * gH;
                if (sa == 0) { ey += ua; ez += ub; }
                else if (sa == 1) { ez += ua; ex += ub; }
                else { ex += ua; ey += ub; }
            }
            const size_t o = (size_t)k * plane + (size_t)j * pitch + i;
            Eout[0][o] = ex;
            Eout[1][o] = ey;
            Eout[2][o] = ez;
            // DFT samples: E on the plane, H averaged over the planes m-1, m of its normal
            unsigned hit = SP ? mcol : 0u;
            if (SP && ((zpl >> it) & 1ull)) {
                for (unsigned b = mz; b; b &= b - 1) {
                    const int m = __ffs(b) - 1;
                    if (k == I->mon_index[m]) hit |= 1u << m;
                }
            }
            for (; hit; hit &= hit - 1) {
                const int m = __ffs(hit) - 1;
                const int ax = I->mon_axis[m];
                R ea, eb, ha, hb;
                size_t p, npl;
                if (ax == 2) {          // a = x, b = y
                    ea = ex; eb = ey;
                    ha = R(0.5) * (hxk + hxm); hb = R(0.5) * (hyk + hym);
                    p = (size_t)i + (size_t)nx * j;
                    npl = (size_t)nx * ny;
                } else if (ax == 0) {   // a = y, b = z
                    ea = ey; eb = ez;
                    ha = R(0.5) * (hyk + hy_i); hb = R(0.5) * (hzk + hz_i);
                    p = (size_t)j + (size_t)ny * k;
                    npl = (size_t)ny * nz;
                } else {                // a = z, b = x
                    ea = ez; eb = ex;
                    ha = R(0.5) * (hzk + hz_j); hb = R(0.5) * (hxk + hx_j);
                    p = (size_t)k + (size_t)nz * i;
                    npl = (size_t)nz * nx;
                }
                R* smp = smp0 + I->mon_off[m];
                smp[p] = ea;
                smp[npl + p] = eb;
                smp[2 * npl + p] = ha;
                smp[3 * npl + p] = hb;
            }
            if (want_energy) {
                energy += I->lute[v0] * (double)ex * ex + I->lute[v1] * (double)ey * ey +
                          I->lute[v2] * (double)ez * ez + (double)hxk * hxk + (double)hyk * hyk +
                          (double)hzk * hzk;
            }
            hxm = hxk;
            hym = hyk;
        }
        // the next iteration's first barrier separates these reads of the
        // new-H plane and slot s0 from their reuse
    };
    // the tile has x / y normal source or monitor columns (every plane is special)
    const bool colSpecial = __syncthreads_or(ownSrcH || ownSrcE || haloSrcH || mcol != 0u) != 0;
    if (zpre) load_zH(k0);
    for (int k = k0; k < k1; ++k) {
        const int it = k - k0;
        const int s0 = it % ns, s1 = (it + 1) % ns, sn = (it + ns - 1) % ns;
        if (it == 0) wait_plane(k, s0);
        wait_plane(k + 1, s1);   // planes k and k+1 have landed (later ones may be in flight)
        __syncthreads();         // ... for every thread; everyone is done with plane k-1
        if (s_abort) break;      // a wait ran out: the whole CTA leaves the march here
        if (k + ns - 1 <= k1) load_plane(k + ns - 1, sn);   // into the slot of plane k-1
        cp_commit();
        if (zpre) load_zE(k);
        if constexpr (PML) {   // one form: the CPML loop is large enough without a second copy
            march_plane(k, it, s0, s1, std::true_type{});
        } else {
            const bool special = colSpecial || k == kSrcH || k == kSrcE || ((zpl >> it) & 1ull) != 0;
            if (special) march_plane(k, it, s0, s1, std::true_type{});
            else march_plane(k, it, s0, s1, std::false_type{});
        }
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");   // no cp.async copy outlives the CTA
    // Every TMA plane armed, k0 .. k1, was waited for inside the march unless
    // a wait ran out; then the planes armed after the last completed wait may
    // still be writing into this CTA's shared memory: the issuer (which keeps
    // the CTA resident) waits for each of them, with the same bound, before
    // the CTA exits.
    if (use_tma && t == kIssuer) {
        for (int p = s_waited + 1; p <= s_issued; ++p) {
            const int s2 = (p - k0) % ns;
            if (!mbar_wait_bounded(&sbar[s2], (unsigned)(((p - k0) / ns) & 1), wait_ns)) timed_out = true;
        }
    }
    if (timed_out) st->fault = 1;
    if (t == 0) st->cur = par ^ 1;   // every CTA of the instance writes the same value
    if (want_energy) {   // warp reduction, one atomic per warp
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) energy += __shfl_down_sync(0xffffffffu, energy, o);
        if ((t & 31) == 0 && energy != 0.0) atomicAdd(&st->energy, energy);
    }
}

template <class R, class IT, bool PML>
cudaError_t launch_one(const void* insts, const Tile3D* tiles, int ntiles, int par, int off, int we, WaitCtl wc,
                       cudaStream_t s) {
    constexpr size_t smem = smem_bytes<R, IT, kZRing<R, PML>>();
    static int done[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !done[dev]) {
        const cudaError_t e =
            cudaFuncSetAttribute(k_step3d<R, IT, PML>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        done[dev] = 1;
    }
    k_step3d<R, IT, PML><<<ntiles, NT, smem, s>>>(reinterpret_cast<const Inst3D<R>*>(insts), tiles, par, off, we, wc);
    return cudaGetLastError();
}

template <class R, bool PML>
cudaError_t launch_idx(int idxw, const void* insts, const Tile3D* tiles, int ntiles, int par, int off, int we,
                       WaitCtl wc, cudaStream_t s) {
    if (idxw == 1) return launch_one<R, uint8_t, PML>(insts, tiles, ntiles, par, off, we, wc, s);
    if (idxw == 2) return launch_one<R, uint16_t, PML>(insts, tiles, ntiles, par, off, we, wc, s);
    return launch_one<R, uint32_t, PML>(insts, tiles, ntiles, par, off, we, wc, s);
}

}  // namespace

cudaError_t launch_step3d(bool fp64, bool pml, int idxw, const void* insts, const Tile3D* tiles, int ntiles, int par,
                          int launch_off, int want_energy, WaitCtl wc, cudaStream_t s) {
    if (ntiles <= 0) return cudaSuccess;
    if (fp64)
        return pml ? launch_idx<double, true>(idxw, insts, tiles, ntiles, par, launch_off, want_energy, wc, s)
                   : launch_idx<double, false>(idxw, insts, tiles, ntiles, par, launch_off, want_energy, wc, s);
    return pml ? launch_idx<float, true>(idxw, insts, tiles, ntiles, par, launch_off, want_energy, wc, s)
               : launch_idx<float, false>(idxw, insts, tiles, ntiles, par, launch_off, want_energy, wc, s);
}

}  // namespace orf
