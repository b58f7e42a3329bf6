// job2d.cu -- one orf.fdtd2D run on the device (toolbox/+orf/fdtd2D.m:1-29).
//
// Host work at creation: validate the sim struct, turn the eps arrays into a
// material index plus a table of update coefficients (exact: the table holds
// every distinct eps value), build the CPML profiles, the TF/SF source
// tables and the tile lists, and upload everything into one device arena.
// The time loop is the shared ChunkEngine; outputs are the monitor DFT lines
// and the fluxes of fdtd2D.m:25-29.
#include <algorithm>
#include <unordered_map>

#include "engine.cuh"
#include "job2d.cuh"

namespace orf {

int validate2d(const orf_sim2d* s, bool scan_eps) {
    if (!s) { set_error("sim is NULL"); return ORF_EINVAL; }
    if (s->pol != ORF_TE && s->pol != ORF_TM) { set_error("sim.pol must be TE or TM"); return ORF_EINVAL; }
    if (s->nx < 3 || s->nz < 2) { set_error("grid must be at least 3 x 2 cells"); return ORF_EINVAL; }
    if ((int64_t)s->nx * s->nz > (int64_t)1 << 31) { set_error("grid exceeds 2^31 cells"); return ORF_ETOOLARGE; }
    if (!(s->dx > 0) || !std::isfinite(s->dx)) { set_error("grid spacing must be positive"); return ORF_EINVAL; }
    if (!(s->courant > 0) || s->courant > 1.0 / std::sqrt(2.0) + 1e-12) {
        set_error("courant %.6g outside (0, 1/sqrt(2)] (2D Yee stability limit)", s->courant);
        return ORF_EINVAL;
    }
    const bool per = s->periodic_z != 0;
    const int nz = s->nz, nx = s->nx, nzA = per ? nz : nz - 1;
    if (s->pol == ORF_TE && !s->eps) { set_error("sim.eps is required for TE"); return ORF_EINVAL; }
    if (s->pol == ORF_TM && (!s->eps_x || !s->eps_z)) { set_error("sim.epsX and sim.epsZ are required for TM"); return ORF_EINVAL; }
    auto chk = [&](const double* e, size_t n, const char* nm) {
        const size_t q = first_bad_positive(e, n);
        if (q < n) {
            set_error("%s(%zu) = %g: permittivity must be positive and finite", nm, q + 1, e[q]);
            return false;
        }
        return true;
    };
    if (scan_eps && s->pol == ORF_TE && !chk(s->eps, (size_t)nx * nz, "sim.eps")) return ORF_EINVAL;
    if (scan_eps && s->pol == ORF_TM &&
        (!chk(s->eps_x, (size_t)nx * nzA, "sim.epsX") || !chk(s->eps_z, (size_t)(nx - 1) * nz, "sim.epsZ")))
        return ORF_EINVAL;
    const int npz = per ? 0 : s->npml_z;
    if (s->npml_x < 0 || 2 * s->npml_x >= nx - 1) { set_error("npml(1) = %d does not fit numel(x) = %d", s->npml_x, nx); return ORF_EINVAL; }
    if (npz < 0 || 2 * npz >= nz - 1) { set_error("npml(2) = %d does not fit numel(z) = %d", npz, nz); return ORF_EINVAL; }
    if (s->src_ix < 0 || s->src_ix >= nx) { set_error("source.ix = %d outside 1..%d", s->src_ix + 1, nx); return ORF_EINVAL; }
    if (s->src_ix < s->npml_x || s->src_ix >= nx - s->npml_x) { set_error("source.ix = %d lies inside the CPML", s->src_ix + 1); return ORF_EINVAL; }
    if (!s->src_profile) { set_error("source.profile is required"); return ORF_EINVAL; }
    if (!(s->src_lambda0 > 0) || !(s->src_bw > 0)) { set_error("source.lambda0 and source.bw must be positive"); return ORF_EINVAL; }
    if (!std::isfinite(s->src_neff)) { set_error("source.neff must be finite"); return ORF_EINVAL; }
    if (s->n_mon < 0 || s->n_mon > kMaxMon || s->n_monz < 0 || s->n_monz > kMaxMon) {
        set_error("at most %d monitors per orientation", kMaxMon);
        return ORF_EINVAL;
    }
    for (int m = 0; m < s->n_mon; ++m)
        if (s->monitors[m] < 0 || s->monitors[m] >= nx) { set_error("monitors(%d) = %d outside 1..%d", m + 1, s->monitors[m] + 1, nx); return ORF_EINVAL; }
    for (int m = 0; m < s->n_monz; ++m)
        if (s->monitors_z[m] < 0 || s->monitors_z[m] >= nz) { set_error("monitorsZ(%d) = %d outside 1..%d", m + 1, s->monitors_z[m] + 1, nz); return ORF_EINVAL; }
    if (s->n_lambda < 1 || !s->lambdas) { set_error("sim.lambdas must not be empty"); return ORF_EINVAL; }
    for (int l = 0; l < s->n_lambda; ++l)
        if (!(s->lambdas[l] > 0)) { set_error("lambdas(%d) must be positive", l + 1); return ORF_EINVAL; }
    if (!(s->max_time >= 0) || !(s->shutoff >= 0)) { set_error("maxTime and shutoff must be non-negative"); return ORF_EINVAL; }
    if (s->precision != ORF_DOUBLE && s->precision != ORF_SINGLE) { set_error("precision must be double or single"); return ORF_EINVAL; }
    return ORF_OK;
}


// Host-only plan of a run's 2D tiles: the interior kernel variant and fused
// depth, the interior rectangle and the frame strips, and every tile's loaded
// window, output rectangle and flags (pointers left unset).  Needs no device;
// orf_plan2d exposes it for checks of the tiling.
int plan2d(const orf_sim2d* s, const orf_tuning& tuning, Plan2D* plan) {
    const bool f64 = s->precision == ORF_DOUBLE;
    const bool per = s->periodic_z != 0;
    const int nx = s->nx, nz = s->nz, npx = s->npml_x, npz = per ? 0 : s->npml_z;
    const int pitch = (nx + 31) & ~31;
    // defaults from the variant / depth sweeps on the 4000 x 1500 workload
    const int fvariant = tuning.variant > 0 ? tuning.variant : (f64 ? 2 : 1);
    Variant2D fv, pv;
    if (!fast2d_info(fvariant, f64, false, &fv)) {
        set_error("unknown 2D kernel variant %d", fvariant);
        return ORF_EINVAL;
    }
    fast2d_info(0, f64, true, &pv);
    // a tile's output keeps T cells (plus up to 3 of x alignment) from its edges
    const int tmax = std::min({kMaxSub, (pv.lz() - 1) / 2, (pv.lx() - 4) / 2, (fv.lz() - 1) / 2, (fv.lx() - 4) / 2});
    int T = tuning.tsteps > 0 ? tuning.tsteps : (f64 ? 6 : 8);
    if (T > tmax) T = tmax;
    if (T < 1) T = 1;

    // An output cell's T-step dependency cone needs correct (CPML-free,
    // unmasked) updates of P within distance T-1 and of A (B) within distance
    // T on the low side: A at rows >= npz, B at columns >= npx, P at rows and
    // columns >= 1.  On the high side P, A and B within distance T-1 must lie
    // below the upper slabs (A starts at nz-1-npz, B at nx-1-npx) and exist.
    int ax = npx + T, bx = nx - npx - T;
    int az = per ? 0 : npz + T, bz = per ? nz : nz - npz - T;
    // Frame tiles at the edge of the grid: outside the grid every field is
    // zero at every step (the mask keeps it so), so a tile whose loaded
    // window starts at the edge, or reaches past it, needs no T-cell margin
    // on that side: its output runs up to the edge.  The x / z strips are
    // widened to what whole frame tiles output anyway (the frame costs the
    // same number of tiles and the interior shrinks by the cells the frame
    // covers): a strip of one tile row is LZ - T rows high at the edge,
    // each further row adds LZ - 2T (x: LX - T, then LX - 2T - 3 at worst).
    {
        const int lzp = pv.lz(), lxp = pv.lx();
        if (!per && lzp - 2 * T > 0) {
            int h = lzp - T;
            while (h < az) h += lzp - 2 * T;
            az = h;
            bz = nz - h;
        }
        if (lxp - 2 * T - 3 > 0) {
            int w = lxp - T;
            while (w < ax) w += lxp - 2 * T - 3;
            ax = w;
            // the right strip: its first tile loads from ceil4(nx - LX) and so
            // reaches the edge, if that still leaves the npx + T columns the
            // interior needs; otherwise whole tiles of worst-case output
            const int c4 = ((nx - lxp) + 3) & ~3;
            if (nx - (c4 + T) >= npx + T) {
                bx = c4 + T;
            } else {
                int wr = lxp - 2 * T - 3;
                while (wr < nx - bx) wr += lxp - 2 * T - 3;
                bx = nx - wr;
            }
        }
    }
    if (bx - ax < 8 || bz - az < 4) { ax = bx = 0; az = bz = 0; }   // everything is frame
    std::vector<FastTile2D> inner, frame;
    // tile the rectangle [x0,x1) x [z0,z1) with a geometry of LX x LZ cells;
    // the loaded origin li0 is rounded down to a multiple of 4 cells.  Frame
    // tiles (edge = true) load from the grid edge when they start there and
    // output up to the edge when their window reaches it.
    auto tile_rect = [&](std::vector<FastTile2D>& out, const Variant2D& v, int x0, int x1, int z0, int z1,
                         bool edge) {
        for (int ok0 = z0; ok0 < z1;) {
            const bool zlo = edge && !per && ok0 == 0;
            const int lk0 = zlo ? 0 : ok0 - T;
            const bool zhi = edge && !per && lk0 + v.lz() >= nz;
            const int oh = std::min((zhi ? nz : lk0 + v.lz() - T) - ok0, z1 - ok0);
            for (int oi0 = x0; oi0 < x1;) {
                const int a = oi0 - T;
                const int li0 = (edge && oi0 == 0) ? 0 : a - ((a % 4) + 4) % 4;
                const bool xhi = edge && li0 + v.lx() >= nx;
                const int ow = std::min((xhi ? nx : li0 + v.lx() - T) - oi0, x1 - oi0);
                FastTile2D t{};
                t.pitch = pitch;
                t.nz = nz;
                t.nx = nx;
                t.periodic = per ? 1 : 0;
                t.li0 = li0;
                t.lk0 = lk0;
                t.oi0 = oi0;
                t.ok0 = ok0;
                t.ow = ow;
                t.oh = oh;
                out.push_back(t);
                oi0 += ow;
            }
            ok0 += oh;
        }
    };
    if (bx > ax) {
        tile_rect(inner, fv, ax, bx, az, bz, false);
        tile_rect(frame, pv, 0, nx, 0, az, true);
        tile_rect(frame, pv, 0, nx, bz, nz, true);
        tile_rect(frame, pv, 0, ax, az, bz, true);
        tile_rect(frame, pv, bx, nx, az, bz, true);
    } else {
        tile_rect(frame, pv, 0, nx, 0, nz, true);
    }
    plan->fvariant = fvariant;
    plan->T = T;
    plan->nfast = (int)inner.size();
    plan->nframe = (int)frame.size();
    plan->lx_int = fv.lx();
    plan->lx_pml = pv.lx();
    plan->lz_pml = pv.lz();
    plan->tiles = inner;
    plan->tiles.insert(plan->tiles.end(), frame.begin(), frame.end());
    const int sx = s->src_ix;
    for (size_t q = 0; q < plan->tiles.size(); ++q) {
        FastTile2D& t = plan->tiles[q];
        const int lxt = (int)q < plan->nfast ? plan->lx_int : plan->lx_pml;
        t.flags = 0;
        if ((sx - 1 >= t.li0 && sx - 1 < t.li0 + lxt) || (sx >= t.li0 && sx < t.li0 + lxt)) t.flags |= 1;
        if ((int)q >= plan->nfast) {
            // frame tile: CPML slabs of x (columns < npx, >= nx-1-npx) and of
            // z (rows < npz, >= nz-1-npz) that its loaded cells reach, with a
            // cell of margin; the kernel skips the psi updates of an axis
            // whose slabs the tile does not reach (they would leave every
            // value unchanged: psi 0, profile (1, 0, 1))
            if (npx > 0 && (t.li0 < npx + 1 || t.li0 + lxt > nx - npx - 2)) t.flags |= 8;
            if (npz > 0 && (t.lk0 < npz + 1 || t.lk0 + plan->lz_pml > nz - npz - 2)) t.flags |= 16;
        }
        for (int m = 0; m < s->n_mon; ++m)
            if (s->monitors[m] >= t.oi0 && s->monitors[m] < t.oi0 + t.ow) t.flags |= 2;
        for (int m = 0; m < s->n_monz; ++m)
            if (s->monitors_z[m] >= t.ok0 && s->monitors_z[m] < t.ok0 + t.oh) t.flags |= 4;
    }
    sort_frame_tiles(plan->tiles.begin() + plan->nfast, plan->tiles.end());
    return ORF_OK;
}

template <class R>
int Job2D<R>::create(const orf_sim2d* s) {
    ORF_TRY(validate2d(s, false));   // every caller scanned the permittivity already
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != ctx->device) ORF_CUDA(cudaSetDevice(ctx->device));
    te = s->pol == ORF_TE;
    per = s->periodic_z != 0;
    nx = s->nx;
    nz = s->nz;
    nzA = per ? nz : nz - 1;
    nxB = nx - 1;
    pitch = (nx + 31) & ~31;
    dx = s->dx;
    Cc = s->courant;
    S = Cc * dx;
    nM = s->n_mon;
    nMZ = s->n_monz;
    nL = s->n_lambda;
    const int npx = s->npml_x, npz = per ? 0 : s->npml_z;
    const size_t cellsP = (size_t)pitch * nz;

    // ---- material index + coefficient table
    // one plane at a time, row by row (index_values: several host threads
    // for large grids, the indices of one sequential scan)
    // (host scratch of the calling thread, kept between jobs: large grids
    // then touch no new pages; entries outside the planes are never read)
    thread_local std::vector<uint32_t> ix0, ix1;
    ix0.resize(std::max(ix0.size(), cellsP));
    if (!te) ix1.resize(std::max(ix1.size(), cellsP));
    std::vector<IndexRow> irows;
    auto add_plane = [&](const double* e, int w, int h, std::vector<uint32_t>& ix) {
        for (int k = 0; k < h; ++k) irows.push_back({e + (size_t)w * k, ix.data() + (size_t)k * pitch, w});
    };
    if (te) {
        add_plane(s->eps, nx, nz, ix0);
    } else {
        add_plane(s->eps_x, nx, nzA, ix0);
        add_plane(s->eps_z, nxB, nz, ix1);
    }
    std::vector<double> lvals;
    index_values(irows, lvals);
    if (lvals.size() > 65536) {
        set_error("more than 65536 distinct permittivity values");
        return ORF_ETOOLARGE;
    }
    nlut = (int)lvals.size();
    idx16 = nlut > 256;
    std::vector<R> hlutc(nlut);
    for (int v = 0; v < nlut; ++v) hlutc[v] = R(Cc / lvals[v]);

    // ---- CPML profiles
    const double alpha_max = kPmlAlphaMaxPerK0 * 2.0 * kPi / s->src_lambda0;
    std::vector<double> px, pxh, pz, pzh;
    int ns;
    pml_profile(nx, nx, npx, 0.0, dx, S, alpha_max, px, &ns);
    pml_profile(nx, nxB, npx, 0.5, dx, S, alpha_max, pxh, &ns);
    pml_profile(nz, nz, npz, 0.0, dx, S, alpha_max, pz, &ns);
    pml_profile(nz, nzA, npz, 0.5, dx, S, alpha_max, pzh, &ns);
    auto toR = [](const std::vector<double>& v) { return std::vector<R>(v.begin(), v.end()); };

    // ---- source
    const int sx = s->src_ix;
    const Pulse g(s->src_lambda0, s->src_bw);
    src_end = g.tend;
    std::vector<R> hsrcB(nz), hsrcP(nz);
    for (int k = 0; k < nz; ++k) {
        const double f = s->src_profile[k];
        const double epsB = te ? 1.0 : (sx >= 1 ? s->eps_z[(sx - 1) + (size_t)nxB * k] : 1.0);
        const double cB = te ? Cc : (sx >= 1 ? Cc / s->eps_z[(sx - 1) + (size_t)nxB * k] : 0.0);
        const double cP = te ? Cc / s->eps[sx + (size_t)nx * k] : Cc;
        hsrcB[k] = R(cB * f);
        hsrcP[k] = R(cP * (s->src_neff * f / epsB));
    }
    nsrc = (int64_t)std::ceil(g.tend / S) + 2;
    std::vector<double> hgE(nsrc), hgH(nsrc);
    for (int64_t n = 0; n < nsrc; ++n) {
        hgE[n] = g(n * S);
        hgH[n] = g((n + 0.5) * S + s->src_neff * 0.5 * dx);
    }
    nmax = max_steps(s->max_time, S);
    shutoff = s->shutoff;

    // ---- tiles
    ORF_TRY(pick_tiling(s));

    // ---- DFT streams: x monitors (P, B lines), z monitors (P, A lines)
    const int sstride = 2 * nz * nM + 2 * nx * nMZ;
    struct SDesc { int soff, len, half; };
    std::vector<SDesc> sd;
    for (int m = 0; m < nM; ++m) {
        sd.push_back({m * 2 * nz, nz, 0});
        sd.push_back({m * 2 * nz + nz, nz, 1});
    }
    for (int m = 0; m < nMZ; ++m) {
        sd.push_back({nM * 2 * nz + m * 2 * nx, nx, 0});
        sd.push_back({nM * 2 * nz + m * 2 * nx + nx, nx, 1});
    }
    nstreams = (int)sd.size();
    std::vector<FlushItem> items;
    for (int q = 0; q < nstreams; ++q)
        for (int e0 = 0; e0 < sd[q].len; e0 += 128)
            for (int l0 = 0; l0 < nL; l0 += 8) items.push_back({q, e0, l0, 0});
    nitems = (int)items.size();
    std::vector<FluxPair> pairs;
    for (int m = 0; m < nM; ++m) pairs.push_back({2 * m, 2 * m + 1, -1, -1, m, nM, 0.5 * dx});
    for (int m = 0; m < nMZ; ++m)
        pairs.push_back({2 * nM + 2 * m, 2 * nM + 2 * m + 1, -1, -1, nM * nL + m, nMZ, -0.5 * dx});
    npairs = (int)pairs.size();

    // ---- device arena
    Arena ar;
    for (int b = 0; b < 2; ++b) {
        ar.add(&h.P[b], cellsP);
        ar.add(&h.A[b], cellsP);
        ar.add(&h.B[b], cellsP);
        ar.add(&h.psiB[b], (size_t)nz * 2 * npx + 1);
        ar.add(&h.psiPx[b], (size_t)nz * 2 * npx + 1);
        ar.add(&h.psiA[b], (size_t)2 * npz * nx + 1);
        ar.add(&h.psiPz[b], (size_t)2 * npz * nx + 1);
    }
    const size_t isz = idx16 ? 2 : 1;
    unsigned char *d_ix0 = nullptr, *d_ix1 = nullptr;
    ar.add(&d_ix0, cellsP * isz);
    if (!te) ar.add(&d_ix1, cellsP * isz);
    R *d_lutc, *d_px, *d_pxh, *d_pz, *d_pzh, *d_srcB, *d_srcP, *d_samples;
    double *d_lute, *d_gE, *d_gH;
    // at least 256 entries: u8-index kernels copy the whole table to shared memory
    ar.add(&d_lutc, std::max<size_t>(nlut, 256));
    ar.add(&d_lute, std::max<size_t>(nlut, 256));
    ar.add(&d_px, px.size());
    ar.add(&d_pxh, pxh.size() + 3);
    ar.add(&d_pz, pz.size());
    ar.add(&d_pzh, pzh.size() + 3);
    ar.add(&d_srcB, nz);
    ar.add(&d_srcP, nz);
    ar.add(&d_gE, nsrc);
    ar.add(&d_gH, nsrc);
    ar.add(&d_samples, (size_t)kChunk * sstride + 1);
    size_t acc_elems = 0;
    for (auto& q : sd) acc_elems += (size_t)q.len * nL;
    ar.add_bytes(&d_acc, acc_elems * 16 + 16);
    ar.add(&d_omega, nL);
    ar.add(&d_flux, (size_t)(nM + nMZ) * nL + 1);
    ar.add(&d_stage, (size_t)std::max(nx, nz) * nL);
    ar.add(&d_inst, 1);
    ar.add(&d_st, 1);
    ar.add(&d_states, 1);
    ar.add(&d_ftiles, ftiles_host.size() + 1);
    ar.add(&d_streams, nstreams + 1);
    ar.add(&d_items, nitems + 1);
    ar.add(&d_pairs, npairs + 1);
    ORF_TRY(ar.check_budget(budget, &need));
    if (ext_base) {
        ORF_TRY(ar.place(ext_base, ext_cap));
    } else {
        ORF_TRY(ar.alloc());
    }
    arena = ar;
    cudaStream_t st = ctx->stream;
    ORF_CUDA(cudaMemsetAsync(arena.base, 0, arena.total, st));

    // mapped host status ring and cancel flag (not in no-allocation mode)
    if (!ext_base) {
        ORF_TRY(host_mapped_alloc(sizeof(ChunkStatus) * kStatusRing, (void**)&ring_h, (void**)&ring_d));
        std::memset(ring_h, 0, sizeof(ChunkStatus) * kStatusRing);
        void* ch = nullptr;
        ORF_TRY(host_mapped_alloc(sizeof(int), &ch, (void**)&cancel_d));
        cancel_h = static_cast<volatile int*>(ch);
        *cancel_h = 0;
    }

    // ---- upload
    thread_local std::vector<unsigned char> ib0, ib1;
    ib0.resize(cellsP * isz);
    ib1.resize(te ? 0 : cellsP * isz);
    // the device index: 16-bit or 8-bit table indices of a plane of w x h
    // cells in rows of `pitch`, zero outside the plane (rows split over
    // host threads)
    auto narrow = [&](const std::vector<uint32_t>& src, int w, int hh, std::vector<unsigned char>& dst) {
        const uint32_t* v = src.data();
        parallel_rows_n(nz, (size_t)pitch, [&](int k0, int k1) {
            for (int k = k0; k < k1; ++k) {
                const size_t o = (size_t)k * pitch;
                const int ww = k < hh ? w : 0;
                if (idx16) {
                    uint16_t* d = reinterpret_cast<uint16_t*>(dst.data()) + o;
                    for (int i = 0; i < ww; ++i) d[i] = (uint16_t)v[o + i];
                    for (int i = ww; i < pitch; ++i) d[i] = 0;
                } else {
                    unsigned char* d = dst.data() + o;
                    for (int i = 0; i < ww; ++i) d[i] = (unsigned char)v[o + i];
                    for (int i = ww; i < pitch; ++i) d[i] = 0;
                }
            }
        });
    };
    if (te) {
        narrow(ix0, nx, nz, ib0);
    } else {
        narrow(ix0, nx, nzA, ib0);
        narrow(ix1, nxB, nz, ib1);
    }
    // (bytes counted here and added to the context's counter once, under a
    // lock: a batch creates its instances on several host threads)
    int64_t h2d = 0;
    auto up = [&](void* d, const void* hsrc, size_t bytes) -> int {
        if (bytes == 0) return ORF_OK;
        ORF_CUDA(cudaMemcpyAsync(d, hsrc, bytes, cudaMemcpyHostToDevice, st));
        h2d += (int64_t)bytes;
        return ORF_OK;
    };
    ORF_TRY(up(d_ix0, ib0.data(), ib0.size()));
    if (!te) ORF_TRY(up(d_ix1, ib1.data(), ib1.size()));
    ORF_TRY(up(d_lutc, hlutc.data(), hlutc.size() * sizeof(R)));
    ORF_TRY(up(d_lute, lvals.data(), lvals.size() * sizeof(double)));
    auto pxR = toR(px), pxhR = toR(pxh), pzR = toR(pz), pzhR = toR(pzh);
    ORF_TRY(up(d_px, pxR.data(), pxR.size() * sizeof(R)));
    ORF_TRY(up(d_pxh, pxhR.data(), pxhR.size() * sizeof(R)));
    ORF_TRY(up(d_pz, pzR.data(), pzR.size() * sizeof(R)));
    ORF_TRY(up(d_pzh, pzhR.data(), pzhR.size() * sizeof(R)));
    ORF_TRY(up(d_srcB, hsrcB.data(), nz * sizeof(R)));
    ORF_TRY(up(d_srcP, hsrcP.data(), nz * sizeof(R)));
    ORF_TRY(up(d_gE, hgE.data(), nsrc * sizeof(double)));
    ORF_TRY(up(d_gH, hgH.data(), nsrc * sizeof(double)));
    std::vector<double> om(nL);
    for (int l = 0; l < nL; ++l) om[l] = 2.0 * kPi / s->lambdas[l];
    ORF_TRY(up(d_omega, om.data(), nL * sizeof(double)));

    h.nx = nx; h.nz = nz; h.pitch = pitch; h.nzA = nzA; h.nxB = nxB;
    h.periodic = per ? 1 : 0; h.te = te ? 1 : 0; h.npx = npx; h.npz = npz; h.idx16 = idx16 ? 1 : 0;
    h.nlut = nlut;
    h.C = R(Cc);
    h.idx0 = d_ix0; h.idx1 = d_ix1; h.lutc = d_lutc; h.lute = d_lute;
    h.pmlx = d_px; h.pmlxh = d_pxh; h.pmlz = d_pz; h.pmlzh = d_pzh;
    h.src_ix = sx; h.nmon = nM; h.nmonz = nMZ; h.sstride = sstride;
    h.srcB = d_srcB; h.srcP = d_srcP; h.gE = d_gE; h.gH = d_gH; h.nsrc = nsrc;
    for (int m = 0; m < kMaxMon; ++m) {
        h.mon[m] = m < nM ? s->monitors[m] : -1;
        h.monz[m] = m < nMZ ? s->monitors_z[m] : -1;
    }
    h.samples = d_samples;
    h.st = d_st;
    ORF_TRY(up(d_inst, &h, sizeof(h)));
    for (FastTile2D& t : ftiles_host) {   // flags come from the plan
        for (int b = 0; b < 2; ++b) {
            t.f[b][0] = h.P[b];
            t.f[b][1] = h.A[b];
            t.f[b][2] = h.B[b];
        }
        t.idx0 = d_ix0;
        t.idx1 = te ? d_ix0 : d_ix1;
        t.st = d_st;
        t.inst = d_inst;
    }
    ORF_TRY(up(d_ftiles, ftiles_host.data(), ftiles_host.size() * sizeof(FastTile2D)));
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
    eng.T = T;
    eng.par = 0;
    eng.d_streams = d_streams;
    eng.d_items = d_items;
    eng.nitems = nitems;
    eng.d_states = d_states;
    eng.nstates = 1;
    int64_t interior_cells = 0;
    for (int q = 0; q < nfast; ++q) interior_cells += (int64_t)ftiles_host[q].ow * ftiles_host[q].oh;
    if (!ext_base && nfast && nframe) ORF_TRY(side.init());   // no extra stream in no-allocation mode
    eng.step = [this, interior_cells](int off, int nsub, int par, int we, cudaStream_t stream,
                                      KernelTimer* tm) -> cudaError_t {
        const bool f64 = sizeof(R) == 8;
        cudaError_t e = cudaSuccess;
        cudaEvent_t a = nullptr;
        // frame next to the interior on the side stream (not while timing
        // individual launches); the interior is submitted first, the side
        // stream waits only for the fork recorded before it
        const bool overlap = !tm && side.ok();
        cudaStream_t fs = stream;
        if (overlap) {
            e = side.fork(stream);
            if (e != cudaSuccess) return e;
            fs = side.s2;
        }
        if (nfast) {
            if (tm && tm->begin(stream, &a) != ORF_OK) return cudaErrorUnknown;
            e = launch_fast2d(f64, te, idx16, false, fvariant, d_ftiles, nfast, off, nsub, par, we, grid_fast, stream);
            if (e != cudaSuccess) return e;
            if (tm && tm->end(stream, 0, interior_cells * nsub, a) != ORF_OK) return cudaErrorUnknown;
        }
        if (nframe) {
            if (tm && tm->begin(fs, &a) != ORF_OK) return cudaErrorUnknown;
            e = launch_fast2d(f64, te, idx16, true, 0, d_ftiles + nfast, nframe, off, nsub, par, we, grid_frame, fs);
            if (e != cudaSuccess) return e;
            if (tm && tm->end(fs, 1, ((int64_t)nx * nz - interior_cells) * nsub, a) != ORF_OK)
                return cudaErrorUnknown;
        }
        if (overlap) e = side.join(stream);
        return e;
    };
    ORF_CUDA(cudaStreamSynchronize(st));
    add_h2d(ctx, h2d);
    return ORF_OK;
}

template <class R>
int Job2D<R>::pick_tiling(const orf_sim2d* s) {
    const bool f64 = sizeof(R) == 8;
    Plan2D plan;
    ORF_TRY(plan2d(s, ctx->tuning, &plan));
    fvariant = plan.fvariant;
    T = plan.T;
    nfast = plan.nfast;
    nframe = plan.nframe;
    ftiles_host = std::move(plan.tiles);
    const int bps_f = nfast ? fast2d_blocks_per_sm(f64, te, idx16, false, fvariant) : 1;
    const int bps_p = nframe ? fast2d_blocks_per_sm(f64, te, idx16, true, 0) : 1;
    if (bps_f < 1 || bps_p < 1) {
        set_error("2D kernel variant %d cannot be resident on this device (%s)", fvariant,
                  cudaGetErrorString(cudaGetLastError()));
        return ORF_ECUDA;
    }
    grid_fast = (int)std::min<size_t>(nfast, (size_t)ctx->sm_count * bps_f);
    grid_frame = (int)std::min<size_t>(nframe, (size_t)ctx->sm_count * bps_p);
    return ORF_OK;
}

template <class R>
int Job2D<R>::init_state() {
    JobState js{};
    js.step = 0;
    js.nmax = nmax;
    js.chunk = 0;
    js.done = nmax <= 0 ? 1 : 0;
    js.converged = 0;
    js.cur = 0;
    js.energy = 0;
    js.peak = 0;
    js.S = S;
    js.src_end = src_end;
    js.shutoff = shutoff;
    js.ring = ring_d;
    js.cancel = cancel_d;
    if (ring_h) std::memset(ring_h, 0, sizeof(ChunkStatus) * kStatusRing);
    if (cancel_h) *cancel_h = 0;
    enq_steps = 0;
    ORF_CUDA(cudaMemcpyAsync(d_st, &js, sizeof js, cudaMemcpyHostToDevice, ctx->stream));
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
Job2D<R>::~Job2D() {
    if (arena.base) {
        cudaStreamSynchronize(ctx->stream);
        arena.release();
    }
    host_mapped_free(ring_h);
    host_mapped_free((void*)cancel_h);
}

template <class R>
int Job2D<R>::reset() {
    cudaStream_t st = ctx->stream;
    ORF_CUDA(cudaStreamSynchronize(st));
    for (int b = 0; b < 2; ++b) {
        ORF_CUDA(cudaMemsetAsync(h.P[b], 0, sizeof(R) * pitch * nz, st));
        ORF_CUDA(cudaMemsetAsync(h.A[b], 0, sizeof(R) * pitch * nz, st));
        ORF_CUDA(cudaMemsetAsync(h.B[b], 0, sizeof(R) * pitch * nz, st));
        ORF_CUDA(cudaMemsetAsync(h.psiB[b], 0, sizeof(R) * ((size_t)nz * 2 * h.npx + 1), st));
        ORF_CUDA(cudaMemsetAsync(h.psiPx[b], 0, sizeof(R) * ((size_t)nz * 2 * h.npx + 1), st));
        ORF_CUDA(cudaMemsetAsync(h.psiA[b], 0, sizeof(R) * ((size_t)2 * h.npz * nx + 1), st));
        ORF_CUDA(cudaMemsetAsync(h.psiPz[b], 0, sizeof(R) * ((size_t)2 * h.npz * nx + 1), st));
    }
    size_t acc_elems = 0;
    for (auto& q : host_streams) acc_elems += (size_t)q.len * nL;
    ORF_CUDA(cudaMemsetAsync(d_acc, 0, acc_elems * 16, st));
    ORF_TRY(init_state());
    ORF_CUDA(cudaStreamSynchronize(st));
    return ORF_OK;
}

template <class R>
void Job2D<R>::state_regions(int b, std::vector<std::pair<void*, size_t>>& out) {
    const size_t fb = sizeof(R) * pitch * nz;
    const size_t px = sizeof(R) * ((size_t)nz * 2 * h.npx + 1), pz = sizeof(R) * ((size_t)2 * h.npz * nx + 1);
    out.clear();
    out.push_back({h.P[b], fb});
    out.push_back({h.A[b], fb});
    out.push_back({h.B[b], fb});
    out.push_back({h.psiB[b], px});
    out.push_back({h.psiPx[b], px});
    out.push_back({h.psiA[b], pz});
    out.push_back({h.psiPz[b], pz});
    size_t acc_elems = 0;
    for (auto& q : host_streams) acc_elems += (size_t)q.len * nL;
    out.push_back({d_acc, acc_elems * 16});
}

template <class R>
uint64_t Job2D<R>::state_key() const {
    uint64_t k = 1469598103934665603ull;   // FNV-1a over the grid and run options
    auto mix = [&k](const void* p, size_t n) {
        const unsigned char* c = static_cast<const unsigned char*>(p);
        for (size_t q = 0; q < n; ++q) k = (k ^ c[q]) * 1099511628211ull;
    };
    const int v[] = {2, (int)sizeof(R), te, per, nx, nz, pitch, h.npx, h.npz, h.src_ix, nM, nMZ, nL};
    mix(v, sizeof v);
    mix(h.mon, sizeof h.mon);
    mix(h.monz, sizeof h.monz);
    mix(&S, sizeof S);
    mix(&dx, sizeof dx);
    return k;
}

template <class R>
void Job2D<R>::resume_host(const JobState& js) {
    enq_steps = js.chunk * kChunk;
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
int Job2D<R>::advance(int64_t nsteps, orf_progress_fn progress, void* user) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != ctx->device) ORF_CUDA(cudaSetDevice(ctx->device));
    const int64_t left = std::max<int64_t>(0, nmax - enq_steps);
    const int64_t chunks = (std::min(nsteps, left) + kChunk - 1) / kChunk;
    enq_steps += chunks * kChunk;
    const int64_t steps0 = pl.last_step;
    ORF_TRY(run_chunks(eng, pl, ctx, chunks, progress, user));
    eng.collect_timing();
    ctx->stats.cell_updates += (pl.last_step - steps0) * (int64_t)nx * nz;
    return pl.cancelled ? ORF_ECANCELLED : ORF_OK;
}

template <class R>
int Job2D<R>::advance_all_direct() {
    const int64_t chunks = (std::max<int64_t>(0, nmax - enq_steps) + kChunk - 1) / kChunk;
    enq_steps += chunks * kChunk;
    for (int64_t c = 0; c < chunks; ++c) ORF_TRY(eng.enqueue_chunk(ctx->stream, false));
    ORF_CUDA(cudaStreamSynchronize(ctx->stream));
    return ORF_OK;
}

template <class R>
int64_t Job2D<R>::steps_done() {
    JobState js;
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return -1;
    if (cudaMemcpy(&js, d_st, sizeof js, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return js.step;
}

template <class R>
int Job2D<R>::finish2d(orf_out2d* o) {
    return finish2d_on(o, ctx->stream);
}

// Results on stream st (a batch finishes its instances on several host
// threads, each with a stream of its own, after the time loop has ended)
template <class R>
int Job2D<R>::finish2d_on(orf_out2d* o, cudaStream_t st) {
    int64_t d2h = 0;
    JobState js;   // read after the stream's last synchronisation below
    ORF_CUDA(cudaMemcpyAsync(&js, d_st, sizeof js, cudaMemcpyDeviceToHost, st));
    const bool f64 = sizeof(R) == 8;
    ORF_CUDA(launch_flux(f64, d_streams, d_pairs, npairs, nL, d_flux, st));
    std::vector<double> fl((size_t)(nM + nMZ) * nL);
    if (!fl.empty()) ORF_CUDA(cudaMemcpyAsync(fl.data(), d_flux, fl.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    d2h += (int64_t)(fl.size() * sizeof(double));
    // DFT lines: stream q -> complex [l][e], through a pinned staging buffer
    // (in no-allocation mode straight into the caller's buffers)
    void* stage = nullptr;
    if (!ext_base) ORF_TRY(pinned_stage_acquire(&stage));
    struct StageGuard {
        void* p;
        ~StageGuard() { pinned_stage_release(p); }
    } stage_guard{stage};
    auto fetch = [&](int q, double* dst) -> int {
        if (!dst) return ORF_OK;
        const DftStream& S = host_streams[q];
        const size_t n = (size_t)S.len * nL;
        d2h += (int64_t)(n * sizeof(double2));
        const void* src = S.acc;
        if (!f64) {   // FP32 sums with their compensation -> complex doubles
            ORF_CUDA(launch_acc_to_complex(false, S.acc, n, d_stage, st));
            src = d_stage;
        }
        if (!stage) {
            ORF_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(double2), cudaMemcpyDeviceToHost, st));
            ORF_CUDA(cudaStreamSynchronize(st));   // the device staging buffer is reused
            return ORF_OK;
        }
        return copy_d2h_staged(dst, src, n * sizeof(double2), stage, st);
    };
    for (int m = 0; m < nM; ++m) {
        ORF_TRY(fetch(2 * m, o->P ? o->P + (size_t)2 * nz * nL * m : nullptr));
        ORF_TRY(fetch(2 * m + 1, o->B ? o->B + (size_t)2 * nz * nL * m : nullptr));
    }
    for (int m = 0; m < nMZ; ++m) {
        ORF_TRY(fetch(2 * nM + 2 * m, o->PZ ? o->PZ + (size_t)2 * nx * nL * m : nullptr));
        ORF_TRY(fetch(2 * nM + 2 * m + 1, o->AZ ? o->AZ + (size_t)2 * nx * nL * m : nullptr));
    }
    ORF_CUDA(cudaStreamSynchronize(st));
    if (o->flux)
        for (size_t q = 0; q < (size_t)nM * nL; ++q) o->flux[q] = fl[q];
    if (o->flux_z)
        for (size_t q = 0; q < (size_t)nMZ * nL; ++q) o->flux_z[q] = fl[(size_t)nM * nL + q];
    o->converged = js.converged;
    o->steps = js.step;
    o->time = js.step * S;
    add_d2h(ctx, d2h);
    return ORF_OK;
}

template <class R>
int Job2D<R>::get_fields(double* const* f, int nf) {
    if (nf < 3) { set_error("2D fields are P, A, B"); return ORF_EINVAL; }
    ORF_CUDA(cudaStreamSynchronize(ctx->stream));
    JobState js;
    ORF_CUDA(cudaMemcpy(&js, d_st, sizeof js, cudaMemcpyDeviceToHost));
    const int b = js.cur;
    std::vector<R> tmp((size_t)pitch * nz);
    R* src[3] = {h.P[b], h.A[b], h.B[b]};
    const int w[3] = {nx, nx, nxB}, hh[3] = {nz, nzA, nz};
    for (int q = 0; q < 3; ++q) {
        if (!f[q]) continue;
        ORF_CUDA(cudaMemcpy(tmp.data(), src[q], tmp.size() * sizeof(R), cudaMemcpyDeviceToHost));
        for (int k = 0; k < hh[q]; ++k)
            for (int i = 0; i < w[q]; ++i) f[q][i + (size_t)w[q] * k] = (double)tmp[(size_t)k * pitch + i];
    }
    return ORF_OK;
}

template struct Job2D<float>;
template struct Job2D<double>;

int make_job2d(orf_ctx* ctx, const orf_sim2d* sim, orf_job** out, bool scan_eps) {
    *out = nullptr;
    ORF_TRY(validate2d(sim, scan_eps));
    if (sim->precision == ORF_SINGLE) {
        auto j = std::make_unique<Job2D<float>>();
        j->ctx = ctx;
        ORF_TRY(j->create(sim));
        *out = j.release();
    } else {
        auto j = std::make_unique<Job2D<double>>();
        j->ctx = ctx;
        ORF_TRY(j->create(sim));
        *out = j.release();
    }
    return ORF_OK;
}

}  // namespace orf
