// job3d.cu -- one orf.fdtd3D run on the device (toolbox/+orf/fdtd3D.m:1-29).
//
// Host work at creation: validate the sim struct, turn the three eps arrays
// into material indices (uint8/16/32) plus a table of C/eps (exact), build the
// CPML profiles and slab maps of every axis, the TF/SF plane tables, the DFT
// streams of the monitor planes (Ea, Eb, Ha, Hb), the column tiles and z
// segments, and the TMA tensor maps, and upload everything into one device
// arena.  A time step is one launch of the fused H+E kernel over the interior
// tiles and one over the CPML tiles (step3d_fused.cu), reading one field
// buffer and writing the other; the shared ChunkEngine runs the loop.
#include <cuda.h>   // CUtensorMap and the cuTensorMapEncodeTiled signature (entry point fetched at run time)

#include <algorithm>
#include <unordered_map>

#include "job3d.cuh"

namespace orf {

int validate3d(const orf_sim3d* s, bool slab, bool scan_eps) {
    if (!s) { set_error("sim is NULL"); return ORF_EINVAL; }
    const int n[3] = {s->nx, s->ny, s->nz};
    for (int q = 0; q < 3; ++q)
        if (n[q] < 2) { set_error("every grid axis needs at least 2 points"); return ORF_EINVAL; }
    if ((int64_t)n[0] * n[1] * n[2] > ((int64_t)1 << 34)) { set_error("grid exceeds 2^34 cells"); return ORF_ETOOLARGE; }
    if (!(s->d > 0) || !std::isfinite(s->d)) { set_error("grid spacing must be positive"); return ORF_EINVAL; }
    if (!(s->courant > 0) || s->courant > 1.0 / std::sqrt(3.0) + 1e-12) {
        set_error("courant %.6g outside (0, 1/sqrt(3)] (3D Yee stability limit)", s->courant);
        return ORF_EINVAL;
    }
    if (!s->eps_x || !s->eps_y || !s->eps_z) { set_error("sim.eps.x/.y/.z are required"); return ORF_EINVAL; }
    const size_t N = (size_t)n[0] * n[1] * n[2];
    const double* e[3] = {s->eps_x, s->eps_y, s->eps_z};
    for (int c = 0; c < 3 && scan_eps; ++c) {
        const size_t q = first_bad_positive(e[c], N);
        if (q < N) {
            set_error("sim.eps.%c(%zu) = %g: permittivity must be positive and finite", "xyz"[c], q + 1, e[c][q]);
            return ORF_EINVAL;
        }
    }
    for (int q = 0; q < 3; ++q) {
        const int np = s->periodic[q] ? 0 : s->npml[q];
        if (np < 0 || 2 * np >= n[q] - 1) { set_error("npml(%d) = %d does not fit the grid", q + 1, np); return ORF_EINVAL; }
    }
    const int a = s->src_axis;
    if (a < 0 || a > 2) { set_error("source.axis must be 1, 2 or 3"); return ORF_EINVAL; }
    const int np = s->periodic[a] ? 0 : s->npml[a];
    if (s->src_index < 0 || s->src_index >= n[a]) { set_error("source.index outside the grid"); return ORF_EINVAL; }
    if (!(slab && a == 2) && (s->src_index < np || s->src_index >= n[a] - np)) {
        set_error("source.index lies inside the CPML");
        return ORF_EINVAL;
    }
    if (!s->src_Ea || !s->src_Eb || !s->src_Ha || !s->src_Hb) { set_error("source profiles Ea, Eb, Ha, Hb are required"); return ORF_EINVAL; }
    if (!(s->src_lambda0 > 0) || !(s->src_bw > 0)) { set_error("source.lambda0 and source.bw must be positive"); return ORF_EINVAL; }
    if (s->n_mon < 0 || s->n_mon > kMaxMon) { set_error("at most %d monitors", kMaxMon); return ORF_EINVAL; }
    for (int m = 0; m < s->n_mon; ++m) {
        const int q = s->mon_axis[m];
        if (q < 0 || q > 2) { set_error("monitors(%d).axis must be 1..3", m + 1); return ORF_EINVAL; }
        if (s->mon_index[m] < 0 || s->mon_index[m] >= n[q]) { set_error("monitors(%d).index outside the grid", m + 1); return ORF_EINVAL; }
    }
    if (s->n_lambda < 1 || !s->lambdas) { set_error("sim.lambdas must not be empty"); return ORF_EINVAL; }
    for (int l = 0; l < s->n_lambda; ++l)
        if (!(s->lambdas[l] > 0)) { set_error("lambdas(%d) must be positive", l + 1); return ORF_EINVAL; }
    if (!(s->max_time >= 0) || !(s->shutoff >= 0)) { set_error("maxTime and shutoff must be non-negative"); return ORF_EINVAL; }
    if (s->precision != ORF_DOUBLE && s->precision != ORF_SINGLE) { set_error("precision must be double or single"); return ORF_EINVAL; }
    return ORF_OK;
}


namespace {
// psi plane of position u of an n-point axis with an np-position layer at
// both ends (half: the positions u + 1/2), -1 outside: the step kernel's map
int slab_index(bool half, int u, int n, int np) {
    if (np <= 0) return -1;
    if (u < np) return u;
    const int hi = half ? n - 1 - np : n - np;
    return u >= hi ? np + (u - hi) : -1;
}
}  // namespace

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (no link-time dependency on libcuda)
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int encode_fn(EncodeTiledFn* out) {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p) {
            cudaGetLastError();
            set_error("cuTensorMapEncodeTiled is not available from the driver");
            return ORF_ECUDA;
        }
        fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    *out = fn;
    return ORF_OK;
}

template <class R>
int Job3D<R>::encode_tmap3(CUtensorMap* m, CUtensorMapDataType t, const void* base, size_t esz, int bx, int by,
                           int rows_pitch, int nplanes) {
    EncodeTiledFn fn;
    ORF_TRY(encode_fn(&fn));
    const int rp = rows_pitch > 0 ? rows_pitch : pitch;
    const int np = nplanes > 0 ? nplanes : n[2];
    const cuuint64_t dims[3] = {(cuuint64_t)n[0], (cuuint64_t)n[1], (cuuint64_t)np};
    const cuuint64_t strides[2] = {(cuuint64_t)rp * esz, (cuuint64_t)rp * n[1] * esz};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = fn(m, t, 3, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d) for a %d x %d x %d grid", (int)r, n[0], n[1], n[2]);
        return ORF_ECUDA;
    }
    return ORF_OK;
}

// Host-only plan of a 3D run's tiles: kTile3X x kTile3Y columns, a segment
// of up to kSeg3 planes each; a tile takes the CPML instantiation if any cell
// it updates or recomputes (one halo cell in x and y, the plane below the
// segment) lies within one cell of an absorbing slab along any axis.  z
// segments of at most kSeg3 planes never mix planes near a z slab with planes
// away from it, so only the planes that need CPML code run it.  Needs no
// device; orf_plan3d exposes it for checks of the tiling.
void plan3d(const orf_sim3d* s, std::vector<Tile3D>& tiles, std::vector<Tile3D>& tiles_pml, bool zlo, bool zhi) {
    const int n[3] = {s->nx, s->ny, s->nz};
    bool per[3];
    for (int q = 0; q < 3; ++q) per[q] = s->periodic[q] != 0;
    tiles.clear();
    tiles_pml.clear();
    auto near_pml = [&](int q, int lo, int hi) {   // cells [lo, hi) along axis q
        const int np = per[q] ? 0 : s->npml[q];
        if (np <= 0) return false;
        const bool at_lo = q != 2 || zlo, at_hi = q != 2 || zhi;
        return (at_lo && lo < np + 1) || (at_hi && hi > n[q] - np - 2);
    };
    std::vector<std::pair<int, int>> segs;
    for (int k0 = 0; k0 < n[2];) {
        const bool pz0 = near_pml(2, k0 - 1, k0 + 2);
        int k1 = k0 + 1;
        while (k1 < n[2] && k1 - k0 < kSeg3 && near_pml(2, k1 - 1, k1 + 2) == pz0) ++k1;
        segs.push_back({k0, k1});
        k0 = k1;
    }
    for (auto [k0, k1] : segs)
        for (int j0 = 0; j0 < n[1]; j0 += kTile3Y)
            for (int i0 = 0; i0 < n[0]; i0 += kTile3X) {
                Tile3D t;
                t.inst = 0;
                t.i0 = i0;
                t.j0 = j0;
                t.tw = (short)std::min(kTile3X, n[0] - i0);
                t.th = (short)std::min(kTile3Y, n[1] - j0);
                t.k0 = k0;
                t.k1 = k1;
                const bool pm = near_pml(0, t.i0 - 1, t.i0 + t.tw + 1) || near_pml(1, t.j0 - 1, t.j0 + t.th + 1) ||
                                near_pml(2, t.k0 - 1, t.k1 + 1);
                (pm ? tiles_pml : tiles).push_back(t);
            }
}

template <class R>
int Job3D<R>::create(const orf_sim3d* s) {
    ORF_TRY(validate3d(s, slab, false));   // every caller scanned the permittivity already
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != ctx->device) ORF_CUDA(cudaSetDevice(ctx->device));
    n[0] = s->nx; n[1] = s->ny; n[2] = s->nz;
    for (int q = 0; q < 3; ++q) per[q] = s->periodic[q] != 0;
    pitch = (n[0] + 31) & ~31;
    d = s->d;
    Cc = s->courant;
    S = Cc * d;
    nM = s->n_mon;
    nL = s->n_lambda;
    cudaStream_t st = ctx->stream;

    // ---- material indices (exact table of distinct eps values)
    // component by component, row by row (index_values: several host
    // threads for large grids, the indices of one sequential scan)
    // (uninitialised scratch: index_values writes the nx cells of every
    // row, the narrowing below the padding columns, both on several host
    // threads for large grids)
    const double* eps[3] = {s->eps_x, s->eps_y, s->eps_z};
    std::unique_ptr<uint32_t[]> ix[3];
    std::vector<IndexRow> irows;
    irows.reserve((size_t)3 * n[1] * n[2]);
    for (int c = 0; c < 3; ++c) {
        ix[c].reset(new uint32_t[NP()]);
        for (int k = 0; k < n[2]; ++k)
            for (int j = 0; j < n[1]; ++j)
                irows.push_back({eps[c] + (size_t)n[0] * ((size_t)j + (size_t)n[1] * k),
                                 ix[c].get() + ((size_t)k * n[1] + j) * pitch, n[0]});
    }
    std::vector<double> lvals;
    index_values(irows, lvals);
    const size_t nlut = lvals.size();
    idxw = nlut <= 256 ? 1 : (nlut <= 65536 ? 2 : 4);
    std::vector<R> hlutc(nlut);
    for (size_t v = 0; v < nlut; ++v) hlutc[v] = R(Cc / lvals[v]);

    // ---- CPML per axis
    const double alpha_max = kPmlAlphaMaxPerK0 * 2.0 * kPi / s->src_lambda0;
    std::vector<double> pI[3], pH[3];
    std::vector<int> slI[3], slH[3];
    int nsI[3], nsH[3];
    for (int q = 0; q < 3; ++q) {
        const int np = per[q] ? 0 : s->npml[q];
        if (slab && q == 2) {
            // the global grid's z profile at the slab's planes: identity at an
            // end that borders another slab.  psi keeps the layout of a
            // symmetric np-plane layer at both local ends (the kernel's slab
            // map); at an inner end it stays zero, and b = 1, a = 0 leave each
            // difference unchanged bit for bit.
            std::vector<double> gI, gH;
            pml_profile(nz_glob, nz_glob, np, 0.0, d, S, alpha_max, gI, nullptr);
            pml_profile(nz_glob, nz_glob, np, 0.5, d, S, alpha_max, gH, nullptr);
            pI[q].assign(gI.begin() + 3 * (size_t)z_off, gI.begin() + 3 * ((size_t)z_off + n[q]));
            pH[q].assign(gH.begin() + 3 * (size_t)z_off, gH.begin() + 3 * ((size_t)z_off + n[q]));
            slI[q].assign(n[q], -1);
            slH[q].assign(n[q], -1);
            const bool inner_lo = z_off > 0, inner_hi = z_off + n[q] < nz_glob;
            for (int u = 0; u < n[q]; ++u) {
                const int si = slab_index(false, u, n[q], np), sh = slab_index(true, u, n[q], np);
                slI[q][u] = si;
                slH[q][u] = sh;
                const bool ai = pI[q][3 * u + 1] != 0.0 || pI[q][3 * u] != 1.0 || pI[q][3 * u + 2] != 1.0;
                const bool ah = pH[q][3 * u + 1] != 0.0 || pH[q][3 * u] != 1.0 || pH[q][3 * u + 2] != 1.0;
                // the layer positions of an end that borders another slab
                // carry no absorption; every absorbing position has psi
                const bool lo_i = si >= 0 && u < np, lo_h = sh >= 0 && u < np;
                const bool bad = (ai && si < 0) || (ah && sh < 0) ||
                                 (inner_lo && ((ai && lo_i) || (ah && lo_h))) ||
                                 (inner_hi && ((ai && si >= 0 && !lo_i) || (ah && sh >= 0 && !lo_h)));
                if (bad) {
                    set_error("z slab [%d, %d) of %d planes: an end that borders another slab lies within %d "
                              "planes of the grid's %d-plane CPML",
                              z_off, z_off + n[q], nz_glob, np + 1, np);
                    return ORF_EINVAL;
                }
            }
            nsI[q] = np > 0 ? 2 * np : 0;
            nsH[q] = np > 0 ? 2 * np + 1 : 0;
            continue;
        }
        pml_profile(n[q], n[q], np, 0.0, d, S, alpha_max, pI[q], &nsI[q]);
        pml_profile(n[q], n[q], np, 0.5, d, S, alpha_max, pH[q], &nsH[q]);
        slI[q].assign(n[q], -1);
        slH[q].assign(n[q], -1);
        int a = 0, b = 0;
        for (int u = 0; u < n[q]; ++u) {
            if (pI[q][3 * u + 1] != 0.0 || pI[q][3 * u] != 1.0 || pI[q][3 * u + 2] != 1.0) slI[q][u] = a++;
            if (pH[q][3 * u + 1] != 0.0 || pH[q][3 * u] != 1.0 || pH[q][3 * u + 2] != 1.0) slH[q][u] = b++;
        }
        nsI[q] = a;
        nsH[q] = b;
    }

    // ---- TF/SF plane: d = axis, a = d+1, b = d+2 (fdtd3D.m:15-21)
    const int sa = s->src_axis, sb = (sa + 1) % 3, sc = (sa + 2) % 3, ss = s->src_index;
    const int Na = n[sb], Nb = n[sc];
    std::vector<R> hsHa((size_t)Na * Nb), hsHb(hsHa.size()), hsEa(hsHa.size()), hsEb(hsHa.size());
    for (int ib = 0; ib < Nb; ++ib)
        for (int ia = 0; ia < Na; ++ia) {
            const size_t pq = (size_t)ia + (size_t)Na * ib;
            int v[3];
            v[sa] = ss;
            v[sb] = ia;
            v[sc] = ib;
            const size_t q0 = (size_t)v[0] + (size_t)n[0] * ((size_t)v[1] + (size_t)n[1] * v[2]);
            hsHa[pq] = R(-Cc * s->src_Eb[pq]);
            hsHb[pq] = R(Cc * s->src_Ea[pq]);
            hsEa[pq] = R((Cc / eps[sb][q0]) * s->src_Hb[pq]);
            hsEb[pq] = R(-(Cc / eps[sc][q0]) * s->src_Ha[pq]);
        }
    const Pulse g(s->src_lambda0, s->src_bw);
    src_end = g.tend;
    nsrc = (int64_t)std::ceil(g.tend / S) + 2;
    std::vector<double> hgE(nsrc), hgH(nsrc);
    for (int64_t k = 0; k < nsrc; ++k) {
        hgE[k] = g(k * S);
        hgH[k] = g((k + 0.5) * S + s->src_neff * 0.5 * d);
    }
    nmax = max_steps(s->max_time, S);
    shutoff = s->shutoff;

    // ---- monitors -> DFT streams (Ea, Eb at t_{n+1}; Ha, Hb at t_{n+1/2})
    int sstride = 0;
    std::vector<int> moff(nM);
    planes.clear();
    for (int m = 0; m < nM; ++m) {
        const int q = s->mon_axis[m];
        const int na = n[(q + 1) % 3], nb = n[(q + 2) % 3];
        planes.push_back({na, nb});
        moff[m] = sstride;
        sstride += 4 * na * nb;
    }
    struct SDesc { int soff, len, half; };
    std::vector<SDesc> sd;
    for (int m = 0; m < nM; ++m) {
        const int np = planes[m].first * planes[m].second;
        for (int f = 0; f < 4; ++f) sd.push_back({moff[m] + f * np, np, f >= 2 ? 1 : 0});
    }
    nstreams = (int)sd.size();
    std::vector<FlushItem> items;
    for (int q = 0; q < nstreams; ++q)
        for (int e0 = 0; e0 < sd[q].len; e0 += 128)
            for (int l0 = 0; l0 < nL; l0 += 8) items.push_back({q, e0, l0, 0});
    nitems = (int)items.size();
    std::vector<FluxPair> pairs;
    for (int m = 0; m < nM; ++m)   // 1/2 Re sum(Ea Hb* - Eb Ha*) dA  (fdtd3D.m:26)
        pairs.push_back({4 * m, 4 * m + 3, 4 * m + 1, 4 * m + 2, m, nM, 0.5 * d * d});
    npairs = (int)pairs.size();

    // ---- tiles (plan3d)
    // a z slab's ends that border other slabs carry no CPML: their planes are
    // interior tiles (the psi planes of the layout there stay unused)
    plan3d(s, tiles, tiles_pml, !slab || z_off == 0, !slab || z_off + n[2] == nz_glob);
    zc = kSeg3;

    // ---- device arena
    // fields and psi ping-pong: a step reads buffer par and writes par^1
    Arena ar;
    for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 3; ++c) {
            ar.add(&h.E[b][c], NP());
            ar.add(&h.H[b][c], NP());
        }
    for (int c = 0; c < 3; ++c)
        for (int q = 0; q < 3; ++q)
            for (int b = 0; b < 2; ++b) {
                h.psiE[b][c][q] = nullptr;
                h.psiH[b][c][q] = nullptr;
                if (q == c) continue;
                if (nsI[q] > 0) ar.add(&h.psiE[b][c][q], N() / n[q] * nsI[q]);
                if (nsH[q] > 0) ar.add(&h.psiH[b][c][q], N() / n[q] * nsH[q]);
            }
    unsigned char* d_ix[3];
    for (int c = 0; c < 3; ++c) ar.add(&d_ix[c], NP() * idxw);
    R *d_lutc, *d_pI[3], *d_pH[3], *d_sHa, *d_sHb, *d_sEa, *d_sEb, *d_samples;
    int *d_slI[3], *d_slH[3];
    double *d_lute, *d_gE, *d_gH;
    // at least 256 entries: u8-index kernels copy the whole table to shared memory
    ar.add(&d_lutc, std::max<size_t>(nlut, 256));
    ar.add(&d_lute, std::max<size_t>(nlut, 256));
    for (int q = 0; q < 3; ++q) {
        ar.add(&d_pI[q], pI[q].size());
        ar.add(&d_pH[q], pH[q].size());
        ar.add(&d_slI[q], n[q]);
        ar.add(&d_slH[q], n[q]);
    }
    ar.add(&d_sHa, hsHa.size());
    ar.add(&d_sHb, hsHa.size());
    ar.add(&d_sEa, hsHa.size());
    ar.add(&d_sEb, hsHa.size());
    ar.add(&d_gE, nsrc);
    ar.add(&d_gH, nsrc);
    ar.add(&d_samples, (size_t)kChunk * sstride + 1);
    size_t acc_elems = 0;
    stage_elems = 1;
    for (auto& q : sd) {
        acc_elems += (size_t)q.len * nL;
        stage_elems = std::max(stage_elems, (size_t)q.len * nL);
    }
    ar.add_bytes(&d_acc, acc_elems * 16 + 16);
    ar.add(&d_omega, nL);
    ar.add(&d_flux, (size_t)nM * nL + 1);
    ar.add(&d_stage, stage_elems);
    ar.add(&d_inst, 1);
    ar.add(&d_st, 1);
    ar.add(&d_states, 1);
    ar.add(&d_tiles, tiles.size() + 1);
    ar.add(&d_tiles_pml, tiles_pml.size() + 1);
    ar.add(&d_streams, nstreams + 1);
    ar.add(&d_items, nitems + 1);
    ar.add(&d_pairs, npairs + 1);
    unsigned char* d_tmap = nullptr;
    ar.add(&d_tmap, kTmaps3 * sizeof(CUtensorMap));
    ORF_TRY(ar.check_budget(budget, &need));
    ORF_TRY(ar.alloc());
    arena = ar;
    ORF_CUDA(cudaMemsetAsync(arena.base, 0, arena.total, st));
    ORF_TRY(host_mapped_alloc(sizeof(ChunkStatus) * kStatusRing, (void**)&ring_h, (void**)&ring_d));
    std::memset(ring_h, 0, sizeof(ChunkStatus) * kStatusRing);
    void* ch = nullptr;
    ORF_TRY(host_mapped_alloc(sizeof(int), &ch, (void**)&cancel_d));
    cancel_h = static_cast<volatile int*>(ch);
    *cancel_h = 0;

    auto up = [&](void* dst, const void* src, size_t bytes) -> int {
        if (bytes == 0) return ORF_OK;
        ORF_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
        ORF_CUDA(cudaStreamSynchronize(st));   // host staging vectors are freed on return
        ctx->stats.h2d_bytes += (int64_t)bytes;
        return ORF_OK;
    };
    // the device index of a component: idxw-byte table indices in rows of
    // `pitch`, zero in the padding columns (the TMA boxes read them)
    std::unique_ptr<unsigned char[]> ib(new unsigned char[NP() * idxw]);
    for (int c = 0; c < 3; ++c) {
        const uint32_t* v = ix[c].get();
        unsigned char* dst = ib.get();
        const int w = n[0], iw = idxw;
        parallel_rows_n(n[1] * n[2], (size_t)pitch, [&](int r0, int r1) {
            for (int r = r0; r < r1; ++r) {
                const size_t o = (size_t)r * pitch;
                if (iw == 4) {
                    uint32_t* d = reinterpret_cast<uint32_t*>(dst) + o;
                    for (int i = 0; i < w; ++i) d[i] = v[o + i];
                    for (int i = w; i < pitch; ++i) d[i] = 0;
                } else if (iw == 2) {
                    uint16_t* d = reinterpret_cast<uint16_t*>(dst) + o;
                    for (int i = 0; i < w; ++i) d[i] = (uint16_t)v[o + i];
                    for (int i = w; i < pitch; ++i) d[i] = 0;
                } else {
                    unsigned char* d = dst + o;
                    for (int i = 0; i < w; ++i) d[i] = (unsigned char)v[o + i];
                    for (int i = w; i < pitch; ++i) d[i] = 0;
                }
            }
        });
        ix[c].reset();
        ORF_TRY(up(d_ix[c], ib.get(), NP() * idxw));
    }
    ORF_TRY(up(d_lutc, hlutc.data(), nlut * sizeof(R)));
    ORF_TRY(up(d_lute, lvals.data(), nlut * sizeof(double)));
    for (int q = 0; q < 3; ++q) {
        std::vector<R> a(pI[q].begin(), pI[q].end()), b(pH[q].begin(), pH[q].end());
        ORF_TRY(up(d_pI[q], a.data(), a.size() * sizeof(R)));
        ORF_TRY(up(d_pH[q], b.data(), b.size() * sizeof(R)));
        ORF_TRY(up(d_slI[q], slI[q].data(), n[q] * sizeof(int)));
        ORF_TRY(up(d_slH[q], slH[q].data(), n[q] * sizeof(int)));
    }
    ORF_TRY(up(d_sHa, hsHa.data(), hsHa.size() * sizeof(R)));
    ORF_TRY(up(d_sHb, hsHb.data(), hsHb.size() * sizeof(R)));
    ORF_TRY(up(d_sEa, hsEa.data(), hsEa.size() * sizeof(R)));
    ORF_TRY(up(d_sEb, hsEb.data(), hsEb.size() * sizeof(R)));
    ORF_TRY(up(d_gE, hgE.data(), nsrc * sizeof(double)));
    ORF_TRY(up(d_gH, hgH.data(), nsrc * sizeof(double)));
    std::vector<double> om(nL);
    for (int l = 0; l < nL; ++l) om[l] = 2.0 * kPi / s->lambdas[l];
    ORF_TRY(up(d_omega, om.data(), nL * sizeof(double)));

    for (int q = 0; q < 3; ++q) {
        h.n[q] = n[q];
        h.per[q] = per[q] ? 1 : 0;
        h.np[q] = per[q] ? 0 : s->npml[q];
        h.pmlI[q] = d_pI[q];
        h.pmlH[q] = d_pH[q];
        h.slabI[q] = d_slI[q];
        h.slabH[q] = d_slH[q];
        h.nslabI[q] = nsI[q];
        h.nslabH[q] = nsH[q];
        h.idx[q] = d_ix[q];
    }
    h.pitch = pitch;
    h.idxw = idxw;
    h.C = R(Cc);
    h.lutc = d_lutc;
    h.lute = d_lute;
    h.sa = sa; h.ss = ss; h.na = Na; h.nb = Nb;
    h.sHa = d_sHa; h.sHb = d_sHb; h.sEa = d_sEa; h.sEb = d_sEb;
    h.gE = d_gE; h.gH = d_gH; h.nsrc = nsrc;
    h.nmon = nM;
    h.sstride = sstride;
    for (int m = 0; m < kMaxMon; ++m) {
        h.mon_axis[m] = m < nM ? s->mon_axis[m] : 0;
        h.mon_index[m] = m < nM ? s->mon_index[m] : -1;
        h.mon_off[m] = m < nM ? moff[m] : 0;
    }
    h.samples = d_samples;
    {
        // TMA tensor maps of the plane loads: E[b][c] (box 40 x 10), H[b][c]
        // (box 40 x 9), index[c] (box 32 x 8); x extent nx, so reads past the
        // grid (the row padding included) are zero-filled
        std::vector<CUtensorMap> maps(kTmaps3);
        const CUtensorMapDataType ft = sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
        const CUtensorMapDataType it = idxw == 1 ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                       : idxw == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_UINT32;
        for (int b = 0; b < 2; ++b)
            for (int c = 0; c < 3; ++c) {
                ORF_TRY(encode_tmap3(&maps[3 * b + c], ft, h.E[b][c], sizeof(R), kTile3X + 8, kTile3Y + 2));
                ORF_TRY(encode_tmap3(&maps[6 + 3 * b + c], ft, h.H[b][c], sizeof(R), kTile3X + 8, kTile3Y + 1));
            }
        for (int c = 0; c < 3; ++c) ORF_TRY(encode_tmap3(&maps[12 + c], it, d_ix[c], idxw, kTile3X, kTile3Y));
        // FP32 CPML tiles: the z-axis psi of the H update (psiH[b][c][2]) and
        // of the E update (psiE[b][c][2]), c = 0, 1, planes of nx x ny in
        // slab order, box 40 x 10 like E; rows of nx values must be a
        // multiple of 16 bytes
        h.tma_psi = 0;
        bool zpsi = sizeof(R) == 4 && h.nslabH[2] > 0 && h.nslabI[2] > 0 && (n[0] * sizeof(R)) % 16 == 0;
        for (int b = 0; b < 2; ++b)
            for (int c = 0; c < 2; ++c) zpsi = zpsi && h.psiH[b][c][2] && h.psiE[b][c][2];
        if (zpsi) {
            for (int b = 0; b < 2; ++b)
                for (int c = 0; c < 2; ++c) {
                    ORF_TRY(encode_tmap3(&maps[15 + 2 * b + c], ft, h.psiH[b][c][2], sizeof(R), kTile3X + 8,
                                         kTile3Y + 2, n[0], h.nslabH[2]));
                    ORF_TRY(encode_tmap3(&maps[19 + 2 * b + c], ft, h.psiE[b][c][2], sizeof(R), kTile3X + 8,
                                         kTile3Y + 2, n[0], h.nslabI[2]));
                }
            h.tma_psi = 1;
        }
        ORF_TRY(up(d_tmap, maps.data(), maps.size() * sizeof(CUtensorMap)));
        h.tmap = d_tmap;
    }
    h.st = d_st;
    ORF_TRY(up(d_inst, &h, sizeof(h)));
    ORF_TRY(up(d_tiles, tiles.data(), tiles.size() * sizeof(Tile3D)));
    ORF_TRY(up(d_tiles_pml, tiles_pml.data(), tiles_pml.size() * sizeof(Tile3D)));
    std::vector<DftStream> hs(nstreams);
    size_t aoff = 0;
    for (int q = 0; q < nstreams; ++q) {
        hs[q].st = d_st;
        hs[q].samples = d_samples;
        hs[q].sstride = sstride;
        hs[q].soff = sd[q].soff;
        hs[q].len = sd[q].len;
        hs[q].half = sd[q].half;
        hs[q].nl = nL;
        hs[q].omega = d_omega;
        hs[q].acc = static_cast<char*>(d_acc) + aoff * 16;
        aoff += (size_t)sd[q].len * nL;
    }
    host_streams = hs;
    ORF_TRY(up(d_streams, hs.data(), hs.size() * sizeof(DftStream)));
    ORF_TRY(up(d_items, items.data(), items.size() * sizeof(FlushItem)));
    ORF_TRY(up(d_pairs, pairs.data(), pairs.size() * sizeof(FluxPair)));
    JobState* sp = d_st;
    ORF_TRY(up(d_states, &sp, sizeof(sp)));
    ORF_TRY(init_state());

    eng.ctx = ctx;
    eng.fp64 = sizeof(R) == 8;
    eng.T = 1;
    eng.par = 0;
    eng.d_streams = d_streams;
    eng.d_items = d_items;
    eng.nitems = nitems;
    eng.d_states = d_states;
    eng.nstates = 1;
    // cells of the interior and of the CPML tile launches (timing records)
    int64_t ncell_int = 0, ncell_pml = 0;
    for (const Tile3D& t : tiles) ncell_int += (int64_t)t.tw * t.th * (t.k1 - t.k0);
    for (const Tile3D& t : tiles_pml) ncell_pml += (int64_t)t.tw * t.th * (t.k1 - t.k0);
    if (!tiles.empty() && !tiles_pml.empty()) ORF_TRY(side.init());
    eng.step = [this, ncell_int, ncell_pml](int off, int nsub, int par, int we, cudaStream_t stream,
                                            KernelTimer* tm) -> cudaError_t {
        (void)nsub;
        cudaEvent_t a = nullptr;
        const bool f64 = sizeof(R) == 8;
        // the CPML tiles run next to the interior tiles (disjoint cells, both
        // read buffer par) unless launches are being timed (then one after
        // the other, each between its own events: kind 0 interior, 1 CPML)
        const bool overlap = !tm && side.ok();
        cudaError_t e = overlap ? side.fork(stream) : cudaSuccess;
        if (e == cudaSuccess && !tiles.empty()) {
            if (tm && tm->begin(stream, &a) != ORF_OK) return cudaErrorUnknown;
            e = launch_step3d(f64, false, idxw, d_inst, d_tiles, (int)tiles.size(), par, off, we, wait_ctl(ctx), stream);
            if (e == cudaSuccess && tm && tm->end(stream, 0, ncell_int, a) != ORF_OK) return cudaErrorUnknown;
        }
        if (e == cudaSuccess && !tiles_pml.empty()) {
            if (tm && tm->begin(stream, &a) != ORF_OK) return cudaErrorUnknown;
            e = launch_step3d(f64, true, idxw, d_inst, d_tiles_pml, (int)tiles_pml.size(), par, off, we,
                              wait_ctl(ctx), overlap ? side.s2 : stream);
            if (e == cudaSuccess && tm && tm->end(stream, 1, ncell_pml, a) != ORF_OK) return cudaErrorUnknown;
        }
        if (e == cudaSuccess && overlap) e = side.join(stream);
        return e;
    };
    ORF_CUDA(cudaStreamSynchronize(st));
    return ORF_OK;
}

template <class R>
int Job3D<R>::init_state() {
    JobState js{};
    js.nmax = nmax;
    js.done = nmax <= 0 ? 1 : 0;
    js.S = S;
    js.src_end = src_end;
    js.shutoff = shutoff;
    js.ring = ring_d;
    js.cancel = cancel_d;
    if (ring_h) std::memset(ring_h, 0, sizeof(ChunkStatus) * kStatusRing);
    if (cancel_h) *cancel_h = 0;
    enq_steps = 0;
    sdone = 0;
    soff = 0;
    ORF_CUDA(cudaMemcpyAsync(d_st, &js, sizeof js, cudaMemcpyHostToDevice, ctx->stream));
    ORF_CUDA(cudaStreamSynchronize(ctx->stream));
    pl = ProgressLoop{};
    pl.ring = ring_h;
    pl.cancel = cancel_h;
    pl.S = S;
    pl.src_end = src_end;
    pl.shutoff = shutoff;
    eng.par = 0;
    return ORF_OK;
}

template <class R>
int Job3D<R>::reset() {
    cudaStream_t st = ctx->stream;
    ORF_CUDA(cudaStreamSynchronize(st));
    for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 3; ++c) {
            ORF_CUDA(cudaMemsetAsync(h.E[b][c], 0, NP() * sizeof(R), st));
            ORF_CUDA(cudaMemsetAsync(h.H[b][c], 0, NP() * sizeof(R), st));
            for (int q = 0; q < 3; ++q) {
                if (h.psiE[b][c][q])
                    ORF_CUDA(cudaMemsetAsync(h.psiE[b][c][q], 0, N() / n[q] * h.nslabI[q] * sizeof(R), st));
                if (h.psiH[b][c][q])
                    ORF_CUDA(cudaMemsetAsync(h.psiH[b][c][q], 0, N() / n[q] * h.nslabH[q] * sizeof(R), st));
            }
        }
    size_t acc_elems = 0;
    for (auto& q : host_streams) acc_elems += (size_t)q.len * nL;
    ORF_CUDA(cudaMemsetAsync(d_acc, 0, acc_elems * 16, st));
    return init_state();
}

template <class R>
void Job3D<R>::state_regions(int b, std::vector<std::pair<void*, size_t>>& out) {
    out.clear();
    for (int c = 0; c < 3; ++c) out.push_back({h.E[b][c], NP() * sizeof(R)});
    for (int c = 0; c < 3; ++c) out.push_back({h.H[b][c], NP() * sizeof(R)});
    for (int c = 0; c < 3; ++c)
        for (int q = 0; q < 3; ++q) {
            if (h.psiE[b][c][q]) out.push_back({h.psiE[b][c][q], N() / n[q] * h.nslabI[q] * sizeof(R)});
            if (h.psiH[b][c][q]) out.push_back({h.psiH[b][c][q], N() / n[q] * h.nslabH[q] * sizeof(R)});
        }
    size_t acc_elems = 0;
    for (auto& q : host_streams) acc_elems += (size_t)q.len * nL;
    out.push_back({d_acc, acc_elems * 16});
}

template <class R>
uint64_t Job3D<R>::state_key() const {
    uint64_t k = 1469598103934665603ull;   // FNV-1a over the grid and run options
    auto mix = [&k](const void* p, size_t m) {
        const unsigned char* c = static_cast<const unsigned char*>(p);
        for (size_t q = 0; q < m; ++q) k = (k ^ c[q]) * 1099511628211ull;
    };
    const int v[] = {3, (int)sizeof(R), n[0], n[1], n[2], pitch, per[0], per[1], per[2],
                     h.np[0], h.np[1], h.np[2], h.sa, h.ss, nM, nL};
    mix(v, sizeof v);
    mix(h.mon_axis, sizeof h.mon_axis);
    mix(h.mon_index, sizeof h.mon_index);
    mix(&S, sizeof S);
    mix(&d, sizeof d);
    return k;
}

template <class R>
void Job3D<R>::resume_host(const JobState& js) {
    enq_steps = js.chunk * kChunk;
    sdone = js.step;
    soff = 0;
    pl = ProgressLoop{};
    pl.ring = ring_h;
    pl.cancel = cancel_h;
    pl.S = S;
    pl.src_end = src_end;
    pl.shutoff = shutoff;
    pl.seen = js.chunk;
    pl.last_step = js.step;
    pl.done = js.done != 0;
    if (ring_h) std::memset(ring_h, 0, sizeof(ChunkStatus) * kStatusRing);
    if (cancel_h) *cancel_h = 0;
    eng.par = js.cur;
    eng.drop_graph();   // a graph captured before encodes the old buffer parity
}

template <class R>
int Job3D<R>::advance(int64_t nsteps, orf_progress_fn progress, void* user) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != ctx->device) ORF_CUDA(cudaSetDevice(ctx->device));
    if (soff != 0) {
        set_error("advance: a chunk begun by orf_job3d_step is unfinished (%d of %d steps)", soff, kChunk);
        return ORF_EINVAL;
    }
    enq_steps = std::max(enq_steps, sdone);
    const int64_t left = std::max<int64_t>(0, nmax - enq_steps);
    const int64_t chunks = (std::min(nsteps, left) + kChunk - 1) / kChunk;
    enq_steps += chunks * kChunk;
    const int64_t steps0 = pl.last_step;
    ORF_TRY(run_chunks(eng, pl, ctx, chunks, progress, user));
    eng.collect_timing();
    ctx->stats.cell_updates += (pl.last_step - steps0) * (int64_t)N();
    return pl.cancelled ? ORF_ECANCELLED : ORF_OK;
}

// One launch pair per step, as in a chunk of advance(), with the sample slot
// of the step in its chunk; the chunk's DFT flush and check follow its last
// step, or the run's last one.  The host does not wait.
template <class R>
int Job3D<R>::step_async(int64_t nsteps) {
    if (nsteps < 0) return ORF_EINVAL;
    if (soff == 0) sdone = std::max(sdone, enq_steps);   // continue after whole chunks of advance()
    cudaStream_t st = ctx->stream;
    for (int64_t q = 0; q < nsteps && sdone < nmax; ++q) {
        const int we = soff == kChunk - 1 ? 1 : 0;
        ORF_CUDA(eng.step(soff, 1, eng.par, we, st, nullptr));
        eng.par ^= 1;
        ++soff;
        ++sdone;
        ctx->stats.cell_updates += (int64_t)N();
        if (soff == kChunk || sdone == nmax) {
            ORF_CUDA(launch_flush(sizeof(R) == 8, d_streams, d_items, nitems, st));
            ORF_CUDA(launch_check(d_states, 1, st));
            soff = 0;
        }
    }
    enq_steps = std::max(enq_steps, sdone - soff);
    return ORF_OK;
}

template <class R>
int Job3D<R>::plane_ptr(int b, int f, int k, void** dev, size_t* bytes) {
    if (b < 0 || b > 1 || f < 0 || f > 5 || k < 0 || k >= n[2] || !dev || !bytes) {
        set_error("plane: buffer 0/1, field 0..5 (Ex Ey Ez Hx Hy Hz), plane 0..%d", n[2] - 1);
        return ORF_EINVAL;
    }
    R* base = f < 3 ? h.E[b][f] : h.H[b][f - 3];
    *dev = base + (size_t)k * n[1] * pitch;
    *bytes = (size_t)n[1] * pitch * sizeof(R);
    return ORF_OK;
}

template <class R>
int64_t Job3D<R>::steps_done() {
    JobState js;
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return -1;
    if (cudaMemcpy(&js, d_st, sizeof js, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return js.step;
}

template <class R>
int Job3D<R>::finish3d(orf_out3d* o) {
    cudaStream_t st = ctx->stream;
    ORF_CUDA(cudaStreamSynchronize(st));
    JobState js;
    ORF_CUDA(cudaMemcpy(&js, d_st, sizeof js, cudaMemcpyDeviceToHost));
    if (js.fault) {
        set_error("a 3D step kernel gave up waiting for its plane loads at step %lld", js.step);
        return ORF_ETIMEOUT_DEVICE;
    }
    const bool f64 = sizeof(R) == 8;
    ORF_CUDA(launch_flux(f64, d_streams, d_pairs, npairs, nL, d_flux, st));
    std::vector<double> fl((size_t)nM * nL);
    if (!fl.empty()) ORF_CUDA(cudaMemcpyAsync(fl.data(), d_flux, fl.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    ctx->stats.d2h_bytes += (int64_t)(fl.size() * sizeof(double));
    for (int m = 0; m < nM; ++m) {
        double* const* dsts[4] = {o->mon_Ea, o->mon_Eb, o->mon_Ha, o->mon_Hb};
        for (int f = 0; f < 4; ++f) {
            if (!dsts[f] || !dsts[f][m]) continue;
            const DftStream& S = host_streams[4 * m + f];
            const size_t ne = (size_t)S.len * nL;
            if (f64) {
                ORF_CUDA(cudaMemcpyAsync(dsts[f][m], S.acc, ne * sizeof(double2), cudaMemcpyDeviceToHost, st));
            } else {
                ORF_CUDA(launch_acc_to_complex(false, S.acc, ne, d_stage, st));
                ORF_CUDA(cudaMemcpyAsync(dsts[f][m], d_stage, ne * sizeof(double2), cudaMemcpyDeviceToHost, st));
            }
            ORF_CUDA(cudaStreamSynchronize(st));
            ctx->stats.d2h_bytes += (int64_t)(ne * sizeof(double2));
        }
    }
    ORF_CUDA(cudaStreamSynchronize(st));
    if (o->flux)
        for (size_t q = 0; q < fl.size(); ++q) o->flux[q] = fl[q];
    o->converged = js.converged;
    o->steps = js.step;
    o->time = js.step * S;
    return ORF_OK;
}

template <class R>
int Job3D<R>::get_fields(double* const* f, int nf) {
    if (nf < 6) { set_error("3D fields are Ex Ey Ez Hx Hy Hz"); return ORF_EINVAL; }
    ORF_CUDA(cudaStreamSynchronize(ctx->stream));
    JobState js;
    ORF_CUDA(cudaMemcpy(&js, d_st, sizeof js, cudaMemcpyDeviceToHost));
    const int b = js.cur;   // buffer written by the last step
    std::vector<R> tmp(NP());
    for (int q = 0; q < 6; ++q) {
        if (!f[q]) continue;
        R* src = q < 3 ? h.E[b][q] : h.H[b][q - 3];
        ORF_CUDA(cudaMemcpy(tmp.data(), src, NP() * sizeof(R), cudaMemcpyDeviceToHost));
        for (int k = 0; k < n[2]; ++k)
            for (int j = 0; j < n[1]; ++j)
                for (int i = 0; i < n[0]; ++i)
                    f[q][(size_t)i + (size_t)n[0] * ((size_t)j + (size_t)n[1] * k)] =
                        (double)tmp[((size_t)k * n[1] + j) * pitch + i];
    }
    return ORF_OK;
}

template struct Job3D<float>;
template struct Job3D<double>;

int make_job3d(orf_ctx* ctx, const orf_sim3d* sim, orf_job** out, bool scan_eps) {
    *out = nullptr;
    ORF_TRY(validate3d(sim, false, scan_eps));
    if (sim->precision == ORF_SINGLE) {
        auto j = std::make_unique<Job3D<float>>();
        j->ctx = ctx;
        ORF_TRY(j->create(sim));
        *out = j.release();
    } else {
        auto j = std::make_unique<Job3D<double>>();
        j->ctx = ctx;
        ORF_TRY(j->create(sim));
        *out = j.release();
    }
    return ORF_OK;
}

int make_job3d_slab(orf_ctx* ctx, const orf_sim3d* sim, int z_off, int nz_glob, orf_job** out) {
    *out = nullptr;
    ORF_TRY(validate3d(sim, true));
    if (z_off < 0 || nz_glob < sim->nz || z_off + sim->nz > nz_glob) {
        set_error("z slab [%d, %d) outside the %d planes of the grid", z_off, z_off + sim->nz, nz_glob);
        return ORF_EINVAL;
    }
    if (sim->periodic[2]) {
        set_error("a z slab needs a non-periodic z axis");
        return ORF_EINVAL;
    }
    if (sim->shutoff != 0.0) {
        set_error("z slabs run a fixed step count: shutoff must be 0 (the energy of one slab is not the run's)");
        return ORF_EINVAL;
    }
    if (sim->src_axis == 2) {   // a z-normal source plane: outside the grid's CPML
        const int g = z_off + sim->src_index, np = sim->npml[2];
        if (g < np || g >= nz_glob - np) {
            set_error("source.index lies inside the CPML of the grid");
            return ORF_EINVAL;
        }
    }
    auto build = [&](auto* j) -> int {
        j->ctx = ctx;
        j->slab = true;
        j->z_off = z_off;
        j->nz_glob = nz_glob;
        return j->create(sim);
    };
    if (sim->precision == ORF_SINGLE) {
        auto j = std::make_unique<Job3D<float>>();
        ORF_TRY(build(j.get()));
        *out = j.release();
    } else {
        auto j = std::make_unique<Job3D<double>>();
        ORF_TRY(build(j.get()));
        *out = j.release();
    }
    return ORF_OK;
}

}  // namespace orf
