// step3d.cu -- 3D Yee half-step kernels (toolbox/+orf/fdtd3D.m:1-29) for sm_100a.
//
//   H_c -= C (D+_c1 E_c2 - D+_c2 E_c1),   E_c += C/eps_c (D-_c1 H_c2 - D-_c2 H_c1)
// with CPML on any axis (cpmlCoefficients.m:4-8), PEC or periodic boundaries,
// the one-sided TF/SF plane on any axis (fdtd3D.m:15-21) and planar DFT
// monitors with H averaged onto the E plane (fdtd3D.m:22, 26-28).
//
// One time step = the H kernel then the E kernel, each updating its fields
// in place (the H update reads only E, the E update only H, so no second
// buffer is needed and the 3D state takes 6 arrays, not 12).  A thread owns
// one (x, y) column and marches ZC planes of it: every load of the ZC planes
// is issued before the first update (the kernel reads the other field set
// only and each updated cell belongs to one thread, so the loads can all be
// in flight), the z-neighbour of the previous plane comes from the same
// register arrays, x/y neighbours from the L1 lines the neighbouring threads
// of the same CTA load.  Tiles that touch no CPML slab
// run an instantiation without any CPML code.  Every thread does the same
// work, so neither kernel needs a barrier or shared memory.
#include "orf_internal.cuh"

namespace orf {
namespace {

constexpr int TX = kTile3X, TY = kTile3Y, NT = TX * TY;
static_assert(NT == 256, "the E kernel fills a 256-entry table with one entry per thread");

__device__ __forceinline__ int wrap(int u, int n, bool per, bool* ok) {
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

// Compact slab index of a coordinate along an axis with np CPML cells per end
// (-1 outside): integer positions (E derivatives) have np + np entries, half
// positions u+1/2 (H derivatives, u < n) np + (np + 1).
__device__ __forceinline__ int slab(bool half, int u, int n, int np) {
    if (np <= 0) return -1;
    if (u < np) return u;
    const int hi = half ? n - 1 - np : n - np;
    return u >= hi ? np + (u - hi) : -1;
}

// CPML-stretched difference, psi updated in place (each psi cell belongs to
// exactly one thread): d -> d/kappa + psi, psi <- b psi + a d
template <bool PML, class R>
__device__ __forceinline__ R cpml(const Inst3D<R>* __restrict__ I, bool half, int c, int q, int coord, int i, int j,
                                  int k, R d) {
    if (!PML) return d;   // interior tiles: no cell within reach of an absorbing slab
    const int sl = slab(half, coord, I->n[q], I->np[q]);
    if (sl < 0) return d;
    const R* prof = half ? I->pmlH[q] : I->pmlI[q];
    const R b = prof[3 * coord], a = prof[3 * coord + 1], ki = prof[3 * coord + 2];
    int v[3] = {i, j, k};
    int dim[3] = {I->n[0], I->n[1], I->n[2]};
    v[q] = sl;
    dim[q] = half ? I->nslabH[q] : I->nslabI[q];
    const size_t o = (size_t)v[0] + (size_t)dim[0] * ((size_t)v[1] + (size_t)dim[1] * v[2]);
    R* ps = half ? I->psiH[0][c][q] : I->psiE[0][c][q];
    const R p = b * ps[o] + a * d;
    ps[o] = p;
    return d * ki + p;
}

template <class R, class IT>
__device__ __forceinline__ R coef(const R* slut, const R* __restrict__ lutc, int v) {
    if constexpr (sizeof(IT) == 1) return slut[v];
    else return __ldg(lutc + v);
}

template <class IT>
__device__ __forceinline__ int ldx(const void* p, size_t o) {
    return (int)__ldg(reinterpret_cast<const IT*>(p) + o);
}

template <class R, int ZC, bool PML>
__global__ void __launch_bounds__(NT, 2)
k_h3d(const Inst3D<R>* __restrict__ insts, const Tile3D* __restrict__ tiles, int launch_off) {
    const Tile3D tile = tiles[blockIdx.x];
    const Inst3D<R>* __restrict__ I = insts + tile.inst;
    const JobState* st = I->st;
    if (st->done) return;
    const long long n = st->step + launch_off;
    if (n >= st->nmax) return;
    const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
    if (tx >= tile.tw || ty >= tile.th) return;   // no barriers below
    const int nx = I->n[0], ny = I->n[1], nz = I->n[2], pitch = I->pitch;
    const bool px = I->per[0] != 0, py = I->per[1] != 0, pz = I->per[2] != 0;
    const size_t plane = (size_t)ny * pitch;
    const R C = I->C;
    const int sa = I->sa, sb = (sa + 1) % 3, sc = (sa + 2) % 3, ss = I->ss;
    const int i = tile.i0 + tx, j = tile.j0 + ty;
    bool iok, jok;
    const int ip = wrap(i + 1, nx, px, &iok);
    const int jp = wrap(j + 1, ny, py, &jok);
    const R* __restrict__ E0 = I->E[0][0];
    const R* __restrict__ E1 = I->E[0][1];
    const R* __restrict__ E2 = I->E[0][2];
    R* __restrict__ H0 = I->H[0][0];
    R* __restrict__ H1 = I->H[0][1];
    R* __restrict__ H2 = I->H[0][2];
    const size_t cij = (size_t)j * pitch + i;
    const size_t ci = (size_t)j * pitch + ip, cj = (size_t)jp * pitch + i;
    // all loads of the ZC planes first (E is read-only in this kernel, and
    // each H cell is read and written by its own thread), so they are in
    // flight together; then the updates and stores
    R ex[ZC + 1], ey[ZC + 1], ez[ZC], ezi[ZC], eyi[ZC], ezj[ZC], exj[ZC], h0[ZC], h1[ZC], h2[ZC];
    ex[0] = __ldg(E0 + (size_t)tile.k0 * plane + cij);
    ey[0] = __ldg(E1 + (size_t)tile.k0 * plane + cij);
#pragma unroll
    for (int kq = 0; kq < ZC; ++kq) {
        const int k = tile.k0 + kq;
        const bool kin = k < tile.k1;
        bool kok;
        const int kp = wrap(k + 1, nz, pz, &kok);
        const size_t o = (size_t)k * plane;
        const size_t ok = (size_t)kp * plane + cij;
        ex[kq + 1] = (kin && kok) ? __ldg(E0 + ok) : R(0);
        ey[kq + 1] = (kin && kok) ? __ldg(E1 + ok) : R(0);
        ez[kq] = kin ? __ldg(E2 + o + cij) : R(0);
        ezi[kq] = (kin && iok) ? __ldg(E2 + o + ci) : R(0);
        eyi[kq] = (kin && iok) ? __ldg(E1 + o + ci) : R(0);
        ezj[kq] = (kin && jok) ? __ldg(E2 + o + cj) : R(0);
        exj[kq] = (kin && jok) ? __ldg(E0 + o + cj) : R(0);
        h0[kq] = kin ? H0[o + cij] : R(0);
        h1[kq] = kin ? H1[o + cij] : R(0);
        h2[kq] = kin ? H2[o + cij] : R(0);
    }
    const R gE = (R)(n < I->nsrc ? I->gE[n] : 0.0);
#pragma unroll
    for (int kq = 0; kq < ZC; ++kq) {
        const int k = tile.k0 + kq;
        if (k >= tile.k1) break;
        const size_t o = (size_t)k * plane + cij;
        // Hx -= C ((Ez(j+1) - Ez) - (Ey(k+1) - Ey))
        R d1 = cpml<PML>(I, true, 0, 1, j, i, j, k, ezj[kq] - ez[kq]);
        R d2 = cpml<PML>(I, true, 0, 2, k, i, j, k, ey[kq + 1] - ey[kq]);
        R hx = h0[kq] - C * (d1 - d2);
        // Hy -= C ((Ex(k+1) - Ex) - (Ez(i+1) - Ez))
        d1 = cpml<PML>(I, true, 1, 2, k, i, j, k, ex[kq + 1] - ex[kq]);
        d2 = cpml<PML>(I, true, 1, 0, i, i, j, k, ezi[kq] - ez[kq]);
        R hy = h1[kq] - C * (d1 - d2);
        // Hz -= C ((Ey(i+1) - Ey) - (Ex(j+1) - Ex))
        d1 = cpml<PML>(I, true, 2, 0, i, i, j, k, eyi[kq] - ey[kq]);
        d2 = cpml<PML>(I, true, 2, 1, j, i, j, k, exj[kq] - ex[kq]);
        R hz = h2[kq] - C * (d1 - d2);
        // TF/SF: the H plane just below the source plane is scattered field
        if (sel3(sa, i, j, k) == ss - 1) {
            const size_t pq = (size_t)sel3(sb, i, j, k) + (size_t)I->na * sel3(sc, i, j, k);
            const R ua = __ldg(I->sHa + pq) * gE, ub = __ldg(I->sHb + pq) * gE;
            if (sa == 0) { hy += ua; hz += ub; }
            else if (sa == 1) { hz += ua; hx += ub; }
            else { hx += ua; hy += ub; }
        }
        H0[o] = hx;
        H1[o] = hy;
        H2[o] = hz;
    }
}

template <class R, class IT, int ZC, bool PML>
__global__ void __launch_bounds__(NT, 2)
k_e3d(const Inst3D<R>* __restrict__ insts, const Tile3D* __restrict__ tiles, int launch_off, int want_energy) {
    const Tile3D tile = tiles[blockIdx.x];
    const Inst3D<R>* __restrict__ I = insts + tile.inst;
    JobState* st = I->st;
    if (st->done) return;
    const long long n = st->step + launch_off;
    if (n >= st->nmax) return;
    const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
    const bool own = tx < tile.tw && ty < tile.th;
    // u8 index: the 256-entry coefficient table in shared memory, so the
    // coefficient lookup is not a second dependent global load
    __shared__ R slut[sizeof(IT) == 1 ? 256 : 1];
    if constexpr (sizeof(IT) == 1) {
        slut[threadIdx.x] = I->lutc[threadIdx.x];
        __syncthreads();
    }
    double energy = 0.0;
    if (own) {
        const int nx = I->n[0], ny = I->n[1], nz = I->n[2], pitch = I->pitch;
        const bool px = I->per[0] != 0, py = I->per[1] != 0, pz = I->per[2] != 0;
        const size_t plane = (size_t)ny * pitch;
        const int sa = I->sa, sb = (sa + 1) % 3, sc = (sa + 2) % 3, ss = I->ss;
        const int i = tile.i0 + tx, j = tile.j0 + ty;
        bool iok, jok, kok;
        const int im = wrap(i - 1, nx, px, &iok);
        const int jm = wrap(j - 1, ny, py, &jok);
        R* __restrict__ E0 = I->E[0][0];
        R* __restrict__ E1 = I->E[0][1];
        R* __restrict__ E2 = I->E[0][2];
        const R* __restrict__ H0 = I->H[0][0];
        const R* __restrict__ H1 = I->H[0][1];
        const R* __restrict__ H2 = I->H[0][2];
        const size_t cij = (size_t)j * pitch + i;
        const size_t ci = (size_t)j * pitch + im, cj = (size_t)jm * pitch + i;
        // loads of the ZC planes first (H is read-only here; each E cell is
        // read and written by its own thread), then the updates
        const int km0 = wrap(tile.k0 - 1, nz, pz, &kok);
        R hx[ZC + 1], hy[ZC + 1], hz[ZC], hyi[ZC], hzi[ZC], hxj[ZC], hzj[ZC], e0[ZC], e1[ZC], e2[ZC];
        int v0[ZC], v1[ZC], v2[ZC];
        hx[0] = kok ? __ldg(H0 + (size_t)km0 * plane + cij) : R(0);
        hy[0] = kok ? __ldg(H1 + (size_t)km0 * plane + cij) : R(0);
#pragma unroll
        for (int kq = 0; kq < ZC; ++kq) {
            const int k = tile.k0 + kq;
            const bool kin = k < tile.k1;
            const size_t o = (size_t)k * plane;
            hx[kq + 1] = kin ? __ldg(H0 + o + cij) : R(0);
            hy[kq + 1] = kin ? __ldg(H1 + o + cij) : R(0);
            hz[kq] = kin ? __ldg(H2 + o + cij) : R(0);
            hyi[kq] = (kin && iok) ? __ldg(H1 + o + ci) : R(0);
            hzi[kq] = (kin && iok) ? __ldg(H2 + o + ci) : R(0);
            hxj[kq] = (kin && jok) ? __ldg(H0 + o + cj) : R(0);
            hzj[kq] = (kin && jok) ? __ldg(H2 + o + cj) : R(0);
            v0[kq] = kin ? ldx<IT>(I->idx[0], o + cij) : 0;
            v1[kq] = kin ? ldx<IT>(I->idx[1], o + cij) : 0;
            v2[kq] = kin ? ldx<IT>(I->idx[2], o + cij) : 0;
            e0[kq] = kin ? E0[o + cij] : R(0);
            e1[kq] = kin ? E1[o + cij] : R(0);
            e2[kq] = kin ? E2[o + cij] : R(0);
        }
        const R gH = (R)(n < I->nsrc ? I->gH[n] : 0.0);
        R* smp0 = I->samples + (size_t)launch_off * I->sstride;
#pragma unroll
        for (int kq = 0; kq < ZC; ++kq) {
            const int k = tile.k0 + kq;
            if (k >= tile.k1) break;
            const size_t o = (size_t)k * plane + cij;
            const R hxk = hx[kq + 1], hyk = hy[kq + 1], hzk = hz[kq];
            const R hxm = hx[kq], hym = hy[kq];
            const R hy_i = hyi[kq], hz_i = hzi[kq], hx_j = hxj[kq], hz_j = hzj[kq];
            // Ex += cx ((Hz - Hz(j-1)) - (Hy - Hy(k-1)))
            R d1 = cpml<PML>(I, false, 0, 1, j, i, j, k, hzk - hz_j);
            R d2 = cpml<PML>(I, false, 0, 2, k, i, j, k, hyk - hym);
            R ex = e0[kq] + coef<R, IT>(slut, I->lutc, v0[kq]) * (d1 - d2);
            // Ey += cy ((Hx - Hx(k-1)) - (Hz - Hz(i-1)))
            d1 = cpml<PML>(I, false, 1, 2, k, i, j, k, hxk - hxm);
            d2 = cpml<PML>(I, false, 1, 0, i, i, j, k, hzk - hz_i);
            R ey = e1[kq] + coef<R, IT>(slut, I->lutc, v1[kq]) * (d1 - d2);
            // Ez += cz ((Hy - Hy(i-1)) - (Hx - Hx(j-1)))
            d1 = cpml<PML>(I, false, 2, 0, i, i, j, k, hyk - hy_i);
            d2 = cpml<PML>(I, false, 2, 1, j, i, j, k, hxk - hx_j);
            R ez = e2[kq] + coef<R, IT>(slut, I->lutc, v2[kq]) * (d1 - d2);
            // TF/SF: the source plane is total field
            if (sel3(sa, i, j, k) == ss) {
                const size_t pq = (size_t)sel3(sb, i, j, k) + (size_t)I->na * sel3(sc, i, j, k);
                const R ua = __ldg(I->sEa + pq) * gH, ub = __ldg(I->sEb + pq) * gH;
                if (sa == 0) { ey += ua; ez += ub; }
                else if (sa == 1) { ez += ua; ex += ub; }
                else { ex += ua; ey += ub; }
            }
            E0[o] = ex;
            E1[o] = ey;
            E2[o] = ez;
            // DFT samples: E on the plane, H averaged over the planes m-1, m of its normal
            for (int m = 0; m < I->nmon; ++m) {
                const int ax = I->mon_axis[m];
                if (sel3(ax, i, j, k) != I->mon_index[m]) continue;
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
                energy += I->lute[v0[kq]] * (double)ex * ex + I->lute[v1[kq]] * (double)ey * ey +
                          I->lute[v2[kq]] * (double)ez * ez + (double)hxk * hxk + (double)hyk * hyk +
                          (double)hzk * hzk;
            }
        }
    }
    if (want_energy) {   // warp reduction, one atomic per warp (no block barrier)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) energy += __shfl_down_sync(0xffffffffu, energy, o);
        if ((threadIdx.x & 31) == 0 && energy != 0.0) atomicAdd(&st->energy, energy);
    }
}

}  // namespace

cudaError_t launch_h3d(bool fp64, int zc, bool pml, const void* insts, const Tile3D* tiles, int ntiles,
                       int launch_off, cudaStream_t s) {
    if (ntiles <= 0) return cudaSuccess;
#define ORF_H3(R, Z, P) k_h3d<R, Z, P><<<ntiles, NT, 0, s>>>(reinterpret_cast<const Inst3D<R>*>(insts), tiles, launch_off)
#define ORF_H3Z(R, P) \
    if (zc == 4) ORF_H3(R, 4, P); else ORF_H3(R, 2, P)
    if (fp64) {
        if (pml) { ORF_H3Z(double, true); } else { ORF_H3Z(double, false); }
    } else {
        if (pml) { ORF_H3Z(float, true); } else { ORF_H3Z(float, false); }
    }
#undef ORF_H3Z
#undef ORF_H3
    return cudaGetLastError();
}

cudaError_t launch_e3d(bool fp64, int zc, bool pml, int idxw, const void* insts, const Tile3D* tiles, int ntiles,
                       int launch_off, int want_energy, cudaStream_t s) {
    if (ntiles <= 0) return cudaSuccess;
#define ORF_E3(R, IT, Z, P) \
    k_e3d<R, IT, Z, P><<<ntiles, NT, 0, s>>>(reinterpret_cast<const Inst3D<R>*>(insts), tiles, launch_off, want_energy)
#define ORF_E3Z(R, IT) \
    if (pml) { if (zc == 4) ORF_E3(R, IT, 4, true); else ORF_E3(R, IT, 2, true); } \
    else { if (zc == 4) ORF_E3(R, IT, 4, false); else ORF_E3(R, IT, 2, false); }
    if (fp64) {
        if (idxw == 1) { ORF_E3Z(double, uint8_t); }
        else if (idxw == 2) { ORF_E3Z(double, uint16_t); }
        else { ORF_E3Z(double, uint32_t); }
    } else {
        if (idxw == 1) { ORF_E3Z(float, uint8_t); }
        else if (idxw == 2) { ORF_E3Z(float, uint16_t); }
        else { ORF_E3Z(float, uint32_t); }
    }
#undef ORF_E3Z
#undef ORF_E3
    return cudaGetLastError();
}

}  // namespace orf
