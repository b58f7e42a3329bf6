// step3d.cu -- 3D Yee step kernel (toolbox/+orf/fdtd3D.m:1-29) for sm_100a.
//
//   H_c -= C (D+_c1 E_c2 - D+_c2 E_c1),   E_c += C/eps_c (D-_c1 H_c2 - D-_c2 H_c1)
// with CPML on any axis (cpmlCoefficients.m:4-8), PEC or periodic boundaries,
// the one-sided TF/SF plane on any axis (fdtd3D.m:15-21) and planar DFT
// monitors with H averaged onto the E plane (fdtd3D.m:22, 26-28).
//
// 2.5D z-march: a CTA owns a kTile3X x kTile3Y column of cells and walks its
// planes k = 0 .. nz-1.  Per plane it stages the old E of plane k+1 (tile
// plus a one-cell ring) in a double-buffered shared plane, computes the new H
// of plane k on the tile plus its low ring (the ring H is recomputed, never
// stored), then the new E of plane k from the new H of planes k and k-1 (the
// latter kept in registers from the previous plane).  Each field is read once
// and written once from HBM per step (plus the small ring overlap); buffers
// ping-pong between launches so CTAs at different planes never race.
#include "orf_internal.cuh"

namespace orf {
namespace {

constexpr int TX = kTile3X, TY = kTile3Y, NT = TX * TY;
constexpr int EX = TX + 2, EY = TY + 2;   // E plane with a one-cell ring (low and high)
constexpr int HX = TX + 1, HY = TY + 1;   // H plane with a one-cell ring on the low side

__device__ __forceinline__ int wrap(int u, int n, bool per, bool* ok) {
    if (u >= 0 && u < n) {
        *ok = true;
        return u;
    }
    if (per) {   // any number of periods: the staged ring can be wider than a tiny periodic axis
        *ok = true;
        const int r = u % n;
        return r < 0 ? r + n : r;
    }
    *ok = false;
    return 0;
}

template <class R>
__device__ __forceinline__ size_t psi_at(const Inst3D<R>* I, int q, int ns, int slab, int i, int j, int k) {
    int v[3] = {i, j, k};
    int d[3] = {I->n[0], I->n[1], I->n[2]};
    v[q] = slab;
    d[q] = ns;
    return (size_t)v[0] + (size_t)d[0] * ((size_t)v[1] + (size_t)d[1] * v[2]);
}

// CPML-stretched difference: d -> d/kappa + psi, psi <- b psi + a d (psi in
// difference units); identity outside the layer.
template <class R>
__device__ __forceinline__ R cpml(const Inst3D<R>* I, bool half, int c, int q, int coord, int i, int j, int k,
                                  int par, bool store, R d) {
    const int sl = half ? I->slabH[q][coord] : I->slabI[q][coord];
    if (sl < 0) return d;
    const R* prof = half ? I->pmlH[q] : I->pmlI[q];
    const R b = prof[3 * coord], a = prof[3 * coord + 1], ki = prof[3 * coord + 2];
    const size_t o = psi_at(I, q, half ? I->nslabH[q] : I->nslabI[q], sl, i, j, k);
    const R* pin = half ? I->psiH[par][c][q] : I->psiE[par][c][q];
    R* pout = half ? I->psiH[par ^ 1][c][q] : I->psiE[par ^ 1][c][q];
    const R ps = b * pin[o] + a * d;
    if (store) pout[o] = ps;
    return d * ki + ps;
}

__device__ __forceinline__ int sel3(int a, int x, int y, int z) { return a == 0 ? x : (a == 1 ? y : z); }

template <class IT>
__device__ __forceinline__ int ldx(const void* p, size_t o) {
    return (int)__ldg(reinterpret_cast<const IT*>(p) + o);
}

template <class R, class IT>
__global__ void __launch_bounds__(NT)
k_step3d(const Inst3D<R>* __restrict__ insts, const Tile3D* __restrict__ tiles, int ntiles, int launch_off, int par,
         int want_energy) {
    __shared__ R sE[2][3][EY][EX];
    __shared__ R sH[3][HY][HX];
    __shared__ double sred[NT / 32];
    const Tile3D tile = tiles[blockIdx.x];
    const Inst3D<R>* __restrict__ I = insts + tile.inst;
    JobState* st = I->st;
    if (st->done) return;
    const long long n = st->step + launch_off;
    if (n >= st->nmax) return;
    const int nx = I->n[0], ny = I->n[1], nz = I->n[2], pitch = I->pitch;
    const bool px = I->per[0] != 0, py = I->per[1] != 0, pz = I->per[2] != 0;
    const size_t plane = (size_t)ny * pitch;
    const R C = I->C;
    const R gE = (R)(n < I->nsrc ? I->gE[n] : 0.0);
    const R gH = (R)(n < I->nsrc ? I->gH[n] : 0.0);
    const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
    const int i = tile.i0 + tx, j = tile.j0 + ty;
    const bool own = tx < tile.tw && ty < tile.th;
    const R* Ein[3] = {I->E[par][0], I->E[par][1], I->E[par][2]};
    const R* Hin[3] = {I->H[par][0], I->H[par][1], I->H[par][2]};
    R* Eout[3] = {I->E[par ^ 1][0], I->E[par ^ 1][1], I->E[par ^ 1][2]};
    R* Hout[3] = {I->H[par ^ 1][0], I->H[par ^ 1][1], I->H[par ^ 1][2]};
    const int sa = I->sa, sb = (sa + 1) % 3, sc = (sa + 2) % 3, ss = I->ss;

    // stage old E of plane k (zero outside a non-periodic grid)
    auto loadE = [&](int k, int buf) {
        bool kok;
        const int kk = wrap(k, nz, pz, &kok);
        for (int q = threadIdx.x; q < EX * EY; q += NT) {
            const int ex = q % EX, ey = q / EX;
            bool iok, jok;
            const int gi = wrap(tile.i0 - 1 + ex, nx, px, &iok);
            const int gj = wrap(tile.j0 - 1 + ey, ny, py, &jok);
            const bool ok = kok && iok && jok;
            const size_t o = (size_t)kk * plane + (size_t)gj * pitch + gi;
#pragma unroll
            for (int c = 0; c < 3; ++c) sE[buf][c][ey][ex] = ok ? Ein[c][o] : R(0);
        }
    };

    // new H of the owned column at plane k-1 (z-backward neighbour of E(k))
    R hxp = R(0), hyp = R(0);
    if (pz && own) {
        // periodic z: E(0) needs H(nz-1) of this step; compute it up front
        // (the march recomputes the same value at k = nz-1)
        const int k = nz - 1;
        bool ok;
        const int jp = wrap(j + 1, ny, py, &ok);
        const bool jpo = ok;
        const int ip = wrap(i + 1, nx, px, &ok);
        const bool ipo = ok;
        const size_t o = (size_t)k * plane + (size_t)j * pitch + i;
        const size_t o0 = (size_t)j * pitch + i;   // plane 0
        const R ez = Ein[2][o], ey = Ein[1][o], ex = Ein[0][o];
        R d1 = (jpo ? Ein[2][(size_t)k * plane + (size_t)jp * pitch + i] : R(0)) - ez;
        R d2 = Ein[1][o0] - ey;
        d1 = cpml(I, true, 0, 1, j, i, j, k, par, false, d1);
        d2 = cpml(I, true, 0, 2, k, i, j, k, par, false, d2);
        R hx = Hin[0][o] - C * (d1 - d2);
        R e1 = Ein[0][o0] - ex;
        R e2 = (ipo ? Ein[2][(size_t)k * plane + (size_t)j * pitch + ip] : R(0)) - ez;
        e1 = cpml(I, true, 1, 2, k, i, j, k, par, false, e1);
        e2 = cpml(I, true, 1, 0, i, i, j, k, par, false, e2);
        R hy = Hin[1][o] - C * (e1 - e2);
        if (sel3(sa, i, j, k) == ss - 1) {   // TF/SF correction (scattered side of the plane)
            const size_t pq = (size_t)sel3(sb, i, j, k) + (size_t)I->na * sel3(sc, i, j, k);
            const R ua = __ldg(I->sHa + pq) * gE, ub = __ldg(I->sHb + pq) * gE;
            if (sa == 0) hy += ua;                 // H_a = Hy, H_b = Hz
            else if (sa == 1) hx += ub;            // H_a = Hz, H_b = Hx
            else { hx += ua; hy += ub; }           // H_a = Hx, H_b = Hy
        }
        hxp = hx;
        hyp = hy;
    }

    double energy = 0.0;
    loadE(0, 0);
    __syncthreads();
    for (int k = 0; k < nz; ++k) {
        const int cb = k & 1, nb = cb ^ 1;
        loadE(k + 1, nb);
        __syncthreads();
        // ---- new H of plane k on the tile and its low ring
        for (int q = threadIdx.x; q < HX * HY; q += NT) {
            const int hx_ = q % HX, hy_ = q / HX;
            bool iok, jok;
            const int gi = wrap(tile.i0 - 1 + hx_, nx, px, &iok);
            const int gj = wrap(tile.j0 - 1 + hy_, ny, py, &jok);
            R hn[3] = {R(0), R(0), R(0)};
            if (iok && jok) {
                const bool store = hx_ >= 1 && hy_ >= 1 && hx_ - 1 < tile.tw && hy_ - 1 < tile.th;
                const size_t o = (size_t)k * plane + (size_t)gj * pitch + gi;
                const int ex = hx_, ey = hy_;   // the same cell in the E plane tile (both start at i0-1, j0-1)
                const R Ex0 = sE[cb][0][ey][ex], Ey0 = sE[cb][1][ey][ex], Ez0 = sE[cb][2][ey][ex];
                // Hx -= C ((Ez(j+1) - Ez) - (Ey(k+1) - Ey))
                R d1 = sE[cb][2][ey + 1][ex] - Ez0;
                R d2 = sE[nb][1][ey][ex] - Ey0;
                d1 = cpml(I, true, 0, 1, gj, gi, gj, k, par, store, d1);
                d2 = cpml(I, true, 0, 2, k, gi, gj, k, par, store, d2);
                hn[0] = Hin[0][o] - C * (d1 - d2);
                // Hy -= C ((Ex(k+1) - Ex) - (Ez(i+1) - Ez))
                d1 = sE[nb][0][ey][ex] - Ex0;
                d2 = sE[cb][2][ey][ex + 1] - Ez0;
                d1 = cpml(I, true, 1, 2, k, gi, gj, k, par, store, d1);
                d2 = cpml(I, true, 1, 0, gi, gi, gj, k, par, store, d2);
                hn[1] = Hin[1][o] - C * (d1 - d2);
                // Hz -= C ((Ey(i+1) - Ey) - (Ex(j+1) - Ex))
                d1 = sE[cb][1][ey][ex + 1] - Ey0;
                d2 = sE[cb][0][ey + 1][ex] - Ex0;
                d1 = cpml(I, true, 2, 0, gi, gi, gj, k, par, store, d1);
                d2 = cpml(I, true, 2, 1, gj, gi, gj, k, par, store, d2);
                hn[2] = Hin[2][o] - C * (d1 - d2);
                // TF/SF: the H plane just below the source plane is scattered field
                if (sel3(sa, gi, gj, k) == ss - 1) {
                    const size_t pq = (size_t)sel3(sb, gi, gj, k) + (size_t)I->na * sel3(sc, gi, gj, k);
                    const R ua = __ldg(I->sHa + pq) * gE, ub = __ldg(I->sHb + pq) * gE;
                    if (sa == 0) { hn[1] += ua; hn[2] += ub; }
                    else if (sa == 1) { hn[2] += ua; hn[0] += ub; }
                    else { hn[0] += ua; hn[1] += ub; }
                }
                if (store) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) Hout[c][o] = hn[c];
                }
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) sH[c][hy_][hx_] = hn[c];
        }
        __syncthreads();
        // ---- new E of plane k on the owned column
        if (own) {
            const size_t o = (size_t)k * plane + (size_t)j * pitch + i;
            const int hx_ = tx + 1, hy_ = ty + 1;
            const R Hx = sH[0][hy_][hx_], Hy = sH[1][hy_][hx_], Hz = sH[2][hy_][hx_];
            const int ex = tx + 1, ey = ty + 1;
            R en[3];
            R c0 = __ldg(I->lutc + ldx<IT>(I->idx[0], o));
            R c1 = __ldg(I->lutc + ldx<IT>(I->idx[1], o));
            R c2 = __ldg(I->lutc + ldx<IT>(I->idx[2], o));
            // Ex += cx ((Hz - Hz(j-1)) - (Hy - Hy(k-1)))
            R d1 = Hz - sH[2][hy_ - 1][hx_];
            R d2 = Hy - hyp;
            d1 = cpml(I, false, 0, 1, j, i, j, k, par, true, d1);
            d2 = cpml(I, false, 0, 2, k, i, j, k, par, true, d2);
            en[0] = sE[cb][0][ey][ex] + c0 * (d1 - d2);
            // Ey += cy ((Hx - Hx(k-1)) - (Hz - Hz(i-1)))
            d1 = Hx - hxp;
            d2 = Hz - sH[2][hy_][hx_ - 1];
            d1 = cpml(I, false, 1, 2, k, i, j, k, par, true, d1);
            d2 = cpml(I, false, 1, 0, i, i, j, k, par, true, d2);
            en[1] = sE[cb][1][ey][ex] + c1 * (d1 - d2);
            // Ez += cz ((Hy - Hy(i-1)) - (Hx - Hx(j-1)))
            d1 = Hy - sH[1][hy_][hx_ - 1];
            d2 = Hx - sH[0][hy_ - 1][hx_];
            d1 = cpml(I, false, 2, 0, i, i, j, k, par, true, d1);
            d2 = cpml(I, false, 2, 1, j, i, j, k, par, true, d2);
            en[2] = sE[cb][2][ey][ex] + c2 * (d1 - d2);
            // TF/SF: the source plane is total field
            if (sel3(sa, i, j, k) == ss) {
                const size_t pq = (size_t)sel3(sb, i, j, k) + (size_t)I->na * sel3(sc, i, j, k);
                const R ua = __ldg(I->sEa + pq) * gH, ub = __ldg(I->sEb + pq) * gH;
                if (sa == 0) { en[1] += ua; en[2] += ub; }
                else if (sa == 1) { en[2] += ua; en[0] += ub; }
                else { en[0] += ua; en[1] += ub; }
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) Eout[c][o] = en[c];
            // DFT samples: E on the plane, H averaged over the two neighbouring
            // H planes along the monitor normal
            for (int m = 0; m < I->nmon; ++m) {
                const int ax = I->mon_axis[m];
                if (sel3(ax, i, j, k) != I->mon_index[m]) continue;
                // (Ea, Eb, Ha, Hb) with a = ax+1, b = ax+2; H over the planes m-1, m
                R ea, eb, ha, hb;
                size_t p, npl;
                if (ax == 2) {          // a = x, b = y
                    ea = en[0]; eb = en[1];
                    ha = R(0.5) * (Hx + hxp); hb = R(0.5) * (Hy + hyp);
                    p = (size_t)i + (size_t)nx * j;
                    npl = (size_t)nx * ny;
                } else if (ax == 0) {   // a = y, b = z
                    ea = en[1]; eb = en[2];
                    ha = R(0.5) * (Hy + sH[1][hy_][hx_ - 1]); hb = R(0.5) * (Hz + sH[2][hy_][hx_ - 1]);
                    p = (size_t)j + (size_t)ny * k;
                    npl = (size_t)ny * nz;
                } else {                // a = z, b = x
                    ea = en[2]; eb = en[0];
                    ha = R(0.5) * (Hz + sH[2][hy_ - 1][hx_]); hb = R(0.5) * (Hx + sH[0][hy_ - 1][hx_]);
                    p = (size_t)k + (size_t)nz * i;
                    npl = (size_t)nz * nx;
                }
                R* smp = I->samples + (size_t)launch_off * I->sstride + I->mon_off[m];
                smp[p] = ea;
                smp[npl + p] = eb;
                smp[2 * npl + p] = ha;
                smp[3 * npl + p] = hb;
            }
            if (want_energy) {
                energy += I->lute[ldx<IT>(I->idx[0], o)] * (double)en[0] * en[0] +
                          I->lute[ldx<IT>(I->idx[1], o)] * (double)en[1] * en[1] +
                          I->lute[ldx<IT>(I->idx[2], o)] * (double)en[2] * en[2] + (double)Hx * Hx +
                          (double)Hy * Hy + (double)Hz * Hz;
            }
            hxp = Hx;
            hyp = Hy;
        }
        __syncthreads();
    }
    if (want_energy) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) energy += __shfl_down_sync(0xffffffffu, energy, o);
        if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = energy;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < NT / 32; ++w) t += sred[w];
            atomicAdd(&st->energy, t);
        }
    }
    if (threadIdx.x == 0 && blockIdx.x == 0) st->cur = par ^ 1;
}

}  // namespace

cudaError_t launch_step3d(bool fp64, int idxw, const void* insts, const Tile3D* tiles, int ntiles, int launch_off,
                          int par, int want_energy, cudaStream_t s) {
    if (ntiles <= 0) return cudaSuccess;
#define ORF_L3(R, IT) \
    k_step3d<R, IT><<<ntiles, NT, 0, s>>>(reinterpret_cast<const Inst3D<R>*>(insts), tiles, ntiles, launch_off, par, want_energy)
    if (fp64) {
        if (idxw == 1) ORF_L3(double, uint8_t);
        else if (idxw == 2) ORF_L3(double, uint16_t);
        else ORF_L3(double, uint32_t);
    } else {
        if (idxw == 1) ORF_L3(float, uint8_t);
        else if (idxw == 2) ORF_L3(float, uint16_t);
        else ORF_L3(float, uint32_t);
    }
#undef ORF_L3
    return cudaGetLastError();
}

}  // namespace orf
