// eps3d.cu -- subpixel-averaged 3D permittivity on the GPU (orf_eps3d).
//
// The device form of epsComponents3D (toolbox/+orf/epsComponents3D.m:1-27,
// documented behaviour; host form in opticrcwafdtd_b200/geometry.py): for
// each Yee E component c, every cell at (x_i, y_j, z_k) + h e_c is painted by
// the shapes in order at its centre; cells an interface may cross (the
// shapes' band tests) are sub-sampled at NSub^3 points and take the
// directional mean -- harmonic along c, then arithmetic over the other two
// axes -- or the Kottke diagonal.  One thread per cell; the sub-samples are
// painted on the fly.
//
// Every operation is the host generator's, in its order, with explicit
// round-to-nearest intrinsics (no contraction): the two produce the same
// bits.  A 600 x 600 x 300 pillar lattice takes milliseconds per component
// instead of the host's seconds.
#include "engine.cuh"

namespace orf {
namespace {

struct DevShape {
    int kind, n0, n1, pad;
    double n2;
    double lo[3], hi[3];
    double p[8];
    const double* data;
};

struct EpsArgs {
    const double *x, *y, *z;
    int nx, ny, nz;
    int c;             // component 0 / 1 / 2
    double h, d;       // half cell, cell
    double bg2;        // background n^2
    double Lx, Ly;     // fold periods (0: none)
    int nsub, nshape;
    int method;        // 0 directional, 1 Kottke
    const double* off; // sub-sample offsets, nsub
    const DevShape* sh;
};

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

// v folded into [-L/2, L/2): mod(v + L/2, L) - L/2 with a floored modulo
__device__ __forceinline__ double fold(double v, double L) {
    if (!(L > 0.0) || isinf(L)) return v;
    const double a = add(v, dvd(L, 2.0));
    double m = fmod(a, L);
    if (m != 0.0 && (m < 0.0) != (L < 0.0)) m = add(m, L);
    return sub(m, dvd(L, 2.0));
}

__device__ __forceinline__ double clip01(double v) { return fmin(fmax(v, 0.0), 1.0); }

__device__ bool inside(const DevShape& s, double X, double Y, double Z) {
    switch (s.kind) {
        case ORF_SHAPE_BOX:
            return X >= s.lo[0] && X < s.hi[0] && Y >= s.lo[1] && Y < s.hi[1] && Z >= s.lo[2] && Z < s.hi[2];
        case ORF_SHAPE_CONE: {   // p: cx cy r1 r2 z1 z2
            const bool zin = Z >= s.p[4] && Z < s.p[5];
            const double t = clip01(dvd(sub(Z, s.p[4]), fmax(sub(s.p[5], s.p[4]), 1e-300)));
            const double r = add(s.p[2], mul(sub(s.p[3], s.p[2]), t));
            const double dx = sub(X, s.p[0]), dy = sub(Y, s.p[1]);
            return zin && add(mul(dx, dx), mul(dy, dy)) < mul(r, r);
        }
        case ORF_SHAPE_POLYGON: {   // p: z1 z2; data: x0 y0 x1 y1 ...
            const bool zin = Z >= s.p[0] && Z < s.p[1];
            bool in = false;
            const double* xy = s.data;
            for (int a = 0; a < s.n0; ++a) {
                const int b = (a + 1) % s.n0;
                const double xa = xy[2 * a], ya = xy[2 * a + 1], xb = xy[2 * b], yb = xy[2 * b + 1];
                const bool cond = (ya > Y) != (yb > Y);
                const double den = yb != ya ? sub(yb, ya) : 1.0;
                const double xc = add(dvd(mul(sub(xb, xa), sub(Y, ya)), den), xa);
                in ^= cond && (X < xc);
            }
            return zin && in;
        }
        case ORF_SHAPE_LATTICE: {   // p: x0 y0 period z1 z2 dRdz; data: R[n0][n1]
            const long long ix = (long long)rint(dvd(sub(X, s.p[0]), s.p[2]));
            const long long iy = (long long)rint(dvd(sub(Y, s.p[1]), s.p[2]));
            const bool ok = ix >= 0 && ix < s.n0 && iy >= 0 && iy < s.n1;
            const long long ixc = ix < 0 ? 0 : (ix > s.n0 - 1 ? s.n0 - 1 : ix);
            const long long iyc = iy < 0 ? 0 : (iy > s.n1 - 1 ? s.n1 - 1 : iy);
            const double r = add(s.data[ixc * s.n1 + iyc], mul(s.p[5], sub(Z, s.p[3])));
            const double cx = add(s.p[0], mul((double)ixc, s.p[2]));
            const double cy = add(s.p[1], mul((double)iyc, s.p[2]));
            const bool zin = Z >= s.p[3] && Z < s.p[4];
            const double dx = sub(X, cx), dy = sub(Y, cy);
            return ok && zin && r > 0.0 && add(mul(dx, dx), mul(dy, dy)) < mul(r, r);
        }
    }
    return false;
}

// cells (centre X, Y, Z, half size h) the shape's boundary may cross
__device__ bool band(const DevShape& s, double X, double Y, double Z, double h) {
    const bool near = X >= sub(s.lo[0], h) && X <= add(s.hi[0], h) && Y >= sub(s.lo[1], h) &&
                      Y <= add(s.hi[1], h) && Z >= sub(s.lo[2], h) && Z <= add(s.hi[2], h);
    if (!near) return false;
    if (s.kind == ORF_SHAPE_BOX) {
        const bool full = sub(X, h) >= s.lo[0] && add(X, h) < s.hi[0] && sub(Y, h) >= s.lo[1] &&
                          add(Y, h) < s.hi[1] && sub(Z, h) >= s.lo[2] && add(Z, h) < s.hi[2];
        return !full;
    }
    const double z1 = s.kind == ORF_SHAPE_CONE ? s.p[4] : (s.kind == ORF_SHAPE_POLYGON ? s.p[0] : s.p[3]);
    const double z2 = s.kind == ORF_SHAPE_CONE ? s.p[5] : (s.kind == ORF_SHAPE_POLYGON ? s.p[1] : s.p[4]);
    if (fabs(sub(Z, z1)) <= h || fabs(sub(Z, z2)) <= h) return true;
    const double hd = mul(mul(h, sqrt(2.0)), 1.0000001);
    if (s.kind == ORF_SHAPE_CONE) {
        const double dx = sub(X, s.p[0]), dy = sub(Y, s.p[1]);
        const double rho = sqrt(add(mul(dx, dx), mul(dy, dy)));
        const double rlo = fmin(s.p[2], s.p[3]), rhi = fmax(s.p[2], s.p[3]);
        return rho >= sub(rlo, hd) && rho <= add(rhi, hd);
    }
    if (s.kind == ORF_SHAPE_LATTICE) {
        const double dz = mul(fabs(s.p[5]), h);
        const long long ix0 = (long long)rint(dvd(sub(X, s.p[0]), s.p[2]));
        const long long iy0 = (long long)rint(dvd(sub(Y, s.p[1]), s.p[2]));
        for (int di = -1; di <= 1; ++di)
            for (int dj = -1; dj <= 1; ++dj) {
                const long long ix = ix0 + di, iy = iy0 + dj;
                const bool ok = ix >= 0 && ix < s.n0 && iy >= 0 && iy < s.n1;
                const long long ixc = ix < 0 ? 0 : (ix > s.n0 - 1 ? s.n0 - 1 : ix);
                const long long iyc = iy < 0 ? 0 : (iy > s.n1 - 1 ? s.n1 - 1 : iy);
                const double r = s.p[5] != 0.0 ? add(s.data[ixc * s.n1 + iyc], mul(s.p[5], sub(Z, s.p[3])))
                                               : add(s.data[ixc * s.n1 + iyc], 0.0);
                const double dx = sub(X, add(s.p[0], mul((double)ixc, s.p[2])));
                const double dy = sub(Y, add(s.p[1], mul((double)iyc, s.p[2])));
                const double rho = sqrt(add(mul(dx, dx), mul(dy, dy)));
                if (ok && fabs(sub(rho, r)) <= add(hd, dz)) return true;
            }
        return false;
    }
    // polygon: distance to any edge
    const double* xy = s.data;
    double dmin = INFINITY;
    for (int a = 0; a < s.n0; ++a) {
        const int b = (a + 1) % s.n0;
        const double xa = xy[2 * a], ya = xy[2 * a + 1];
        const double ex = sub(xy[2 * b], xa), ey = sub(xy[2 * b + 1], ya);
        const double L2 = fmax(add(mul(ex, ex), mul(ey, ey)), 1e-300);
        const double t = clip01(dvd(add(mul(sub(X, xa), ex), mul(sub(Y, ya), ey)), L2));
        const double u = sub(sub(X, xa), mul(t, ex)), v = sub(sub(Y, ya), mul(t, ey));
        dmin = fmin(dmin, sqrt(add(mul(u, u), mul(v, v))));
    }
    return dmin <= hd;
}

__device__ __forceinline__ double paint(const EpsArgs& a, double X, double Y, double Z) {
    double e = a.bg2;
    for (int q = 0; q < a.nshape; ++q)
        if (inside(a.sh[q], X, Y, Z)) e = a.sh[q].n2;
    return e;
}

__global__ void k_eps3d(EpsArgs a, double* __restrict__ out) {
    const size_t ncell = (size_t)a.nx * a.ny * a.nz;
    for (size_t cell = (size_t)blockIdx.x * blockDim.x + threadIdx.x; cell < ncell;
         cell += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(cell % a.nx);
        const int j = (int)((cell / a.nx) % a.ny);
        const int k = (int)(cell / ((size_t)a.nx * a.ny));
        const double X = add(a.x[i], a.c == 0 ? a.h : 0.0);
        const double Y = add(a.y[j], a.c == 1 ? a.h : 0.0);
        const double Z = add(a.z[k], a.c == 2 ? a.h : 0.0);
        const double Xf = fold(X, a.Lx), Yf = fold(Y, a.Ly);
        double e = a.bg2;
        bool bnd = false;
        for (int q = 0; q < a.nshape; ++q) {
            if (inside(a.sh[q], Xf, Yf, Z)) e = a.sh[q].n2;
            bnd = bnd || band(a.sh[q], Xf, Yf, Z, a.h);
        }
        if (a.nsub > 1 && bnd && a.method == 1) {
            // Kottke: <eps>, <1/eps> and the first moment g of the samples,
            // each summed sequentially in row-major (x, y, z) order;
            // 1/eps_cc = n_c^2 <1/eps> + (1 - n_c^2)/<eps>, n = g / |g|
            const int N = a.nsub, N3 = N * N * N;
            double se = 0.0, si = 0.0, g[3] = {0.0, 0.0, 0.0};
            for (int u = 0; u < N; ++u)
                for (int v = 0; v < N; ++v)
                    for (int w = 0; w < N; ++w) {
                        const double sx = fold(add(X, mul(a.off[u], a.d)), a.Lx);
                        const double sy = fold(add(Y, mul(a.off[v], a.d)), a.Ly);
                        const double sz = add(Z, mul(a.off[w], a.d));
                        const double ev = paint(a, sx, sy, sz);
                        const double iv = dvd(1.0, ev);
                        const double p0 = mul(ev, a.off[u]), p1 = mul(ev, a.off[v]), p2 = mul(ev, a.off[w]);
                        if (u == 0 && v == 0 && w == 0) {
                            se = ev;
                            si = iv;
                            g[0] = p0;
                            g[1] = p1;
                            g[2] = p2;
                        } else {
                            se = add(se, ev);
                            si = add(si, iv);
                            g[0] = add(g[0], p0);
                            g[1] = add(g[1], p1);
                            g[2] = add(g[2], p2);
                        }
                    }
            const double me = dvd(se, (double)N3), mi = dvd(si, (double)N3);
            const double gn = sqrt(add(add(mul(g[0], g[0]), mul(g[1], g[1])), mul(g[2], g[2])));
            double nc2 = 0.0;
            if (gn > 0.0) {
                const double r = dvd(g[a.c], gn);
                nc2 = mul(r, r);
            }
            e = dvd(1.0, add(mul(nc2, mi), dvd(sub(1.0, nc2), me)));
        } else if (a.nsub > 1 && bnd) {
            // sample (s0, s1, s2) along (x, y, z); the sum along c is
            // sequential, then the NSub^2 harmonic means are summed in
            // row-major order of the two remaining axes
            const int N = a.nsub;
            const int r1ax = a.c == 0 ? 1 : 0, r2ax = a.c == 2 ? 1 : 2;
            double tot = 0.0;
            for (int u = 0; u < N; ++u)
                for (int v = 0; v < N; ++v) {
                    double acc = 0.0;
                    for (int w = 0; w < N; ++w) {
                        int sidx[3];
                        sidx[a.c] = w;
                        sidx[r1ax] = u;
                        sidx[r2ax] = v;
                        const double sx = fold(add(X, mul(a.off[sidx[0]], a.d)), a.Lx);
                        const double sy = fold(add(Y, mul(a.off[sidx[1]], a.d)), a.Ly);
                        const double sz = add(Z, mul(a.off[sidx[2]], a.d));
                        const double inv = dvd(1.0, paint(a, sx, sy, sz));
                        acc = w == 0 ? inv : add(acc, inv);
                    }
                    const double rv = dvd(1.0, dvd(acc, (double)N));
                    tot = (u == 0 && v == 0) ? rv : add(tot, rv);
                }
            e = dvd(tot, (double)(N * N));
        }
        out[cell] = e;
    }
}

}  // namespace

int eps3d(orf_ctx* ctx, const double* x, const double* y, const double* z, int nx, int ny, int nz, double nbg,
          int nsub, int method, const double* period, int nshape, const orf_eps_shape* shapes,
          double* const* outs) {
    if (nx < 2 || ny < 1 || nz < 1 || nsub < 1 || nsub > 16 || nshape < 0 || (nshape && !shapes) || !x || !y ||
        !z || method < 0 || method > 1) {
        set_error("orf_eps3d: invalid grid, NSub (1..16), method (0, 1) or shape list");
        return ORF_EINVAL;
    }
    cudaStream_t st = ctx->stream;
    // shapes and their tables: one device block
    std::vector<DevShape> hs(nshape);
    size_t tab = 0;
    for (int q = 0; q < nshape; ++q) {
        const orf_eps_shape& s = shapes[q];
        if (s.kind < ORF_SHAPE_BOX || s.kind > ORF_SHAPE_LATTICE) {
            set_error("orf_eps3d: shape %d has unknown kind %d", q + 1, s.kind);
            return ORF_EINVAL;
        }
        if ((s.kind == ORF_SHAPE_POLYGON && (s.n0 < 3 || !s.data)) ||
            (s.kind == ORF_SHAPE_LATTICE && (s.n0 < 1 || s.n1 < 1 || !s.data || !(s.p[2] > 0.0)))) {
            set_error("orf_eps3d: shape %d lacks its vertex or radius table", q + 1);
            return ORF_EINVAL;
        }
        if (s.kind == ORF_SHAPE_POLYGON) tab += 2 * (size_t)s.n0;
        if (s.kind == ORF_SHAPE_LATTICE) tab += (size_t)s.n0 * s.n1;
    }
    Arena ar;
    double *d_x, *d_y, *d_z, *d_off, *d_tab, *d_out;
    DevShape* d_sh;
    const size_t ncell = (size_t)nx * ny * nz;
    ar.add(&d_x, nx);
    ar.add(&d_y, ny);
    ar.add(&d_z, nz);
    ar.add(&d_off, nsub);
    ar.add(&d_tab, tab + 1);
    ar.add(&d_sh, nshape + 1);
    ar.add(&d_out, ncell);
    ORF_TRY(ar.alloc());
    struct Release {
        Arena& a;
        ~Release() { a.release(); }
    } rel{ar};
    std::vector<double> htab;
    htab.reserve(tab + 1);
    for (int q = 0; q < nshape; ++q) {
        const orf_eps_shape& s = shapes[q];
        DevShape& d = hs[q];
        d.kind = s.kind;
        d.n0 = s.n0;
        d.n1 = s.n1;
        d.n2 = s.n * s.n;
        for (int t = 0; t < 3; ++t) {
            d.lo[t] = s.lo[t];
            d.hi[t] = s.hi[t];
        }
        for (int t = 0; t < 8; ++t) d.p[t] = s.p[t];
        d.data = nullptr;
        const size_t len = s.kind == ORF_SHAPE_POLYGON ? 2 * (size_t)s.n0
                           : s.kind == ORF_SHAPE_LATTICE ? (size_t)s.n0 * s.n1 : 0;
        if (len) {
            d.data = d_tab + htab.size();
            htab.insert(htab.end(), s.data, s.data + len);
        }
    }
    std::vector<double> off(nsub);
    for (int q = 0; q < nsub; ++q) off[q] = ((q + 1) - (nsub + 1) / 2.0) / nsub;   // as the host's offsets
    ORF_CUDA(cudaMemcpyAsync(d_x, x, nx * sizeof(double), cudaMemcpyHostToDevice, st));
    ORF_CUDA(cudaMemcpyAsync(d_y, y, ny * sizeof(double), cudaMemcpyHostToDevice, st));
    ORF_CUDA(cudaMemcpyAsync(d_z, z, nz * sizeof(double), cudaMemcpyHostToDevice, st));
    ORF_CUDA(cudaMemcpyAsync(d_off, off.data(), nsub * sizeof(double), cudaMemcpyHostToDevice, st));
    if (!htab.empty())
        ORF_CUDA(cudaMemcpyAsync(d_tab, htab.data(), htab.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    if (nshape)
        ORF_CUDA(cudaMemcpyAsync(d_sh, hs.data(), nshape * sizeof(DevShape), cudaMemcpyHostToDevice, st));
    EpsArgs a{};
    a.x = d_x;
    a.y = d_y;
    a.z = d_z;
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.d = x[1] - x[0];
    a.h = a.d / 2;
    a.bg2 = nbg * nbg;
    a.Lx = period ? period[0] : 0.0;
    a.Ly = period ? period[1] : 0.0;
    a.nsub = nsub;
    a.method = method;
    a.nshape = nshape;
    a.off = d_off;
    a.sh = d_sh;
    const int threads = 256;
    const int blocks = (int)std::min<size_t>((ncell + threads - 1) / threads, (size_t)ctx->sm_count * 16);
    for (int c = 0; c < 3; ++c) {
        a.c = c;
        k_eps3d<<<blocks, threads, 0, st>>>(a, d_out);
        ORF_CUDA(cudaGetLastError());
        ORF_CUDA(cudaMemcpyAsync(outs[c], d_out, ncell * sizeof(double), cudaMemcpyDeviceToHost, st));
        ctx->stats.d2h_bytes += (int64_t)(ncell * sizeof(double));
    }
    ORF_CUDA(cudaStreamSynchronize(st));
    return ORF_OK;
}

}  // namespace orf

extern "C" int32_t orf_eps3d(orf_ctx* ctx, const double* x, const double* y, const double* z, int32_t nx, int32_t ny,
                             int32_t nz, double nbg, int32_t nsub, int32_t method, const double* period,
                             int32_t nshape, const orf_eps_shape* shapes, double* ex, double* ey, double* ez) {
    int st = ORF_OK;
    if (!ctx) ctx = orf::default_ctx(&st);
    if (!ctx) return st;
    if (!ex || !ey || !ez) {
        orf::set_error("orf_eps3d: output arrays are NULL");
        return ORF_EINVAL;
    }
    ORF_ON_DEVICE(ctx->device);
    double* outs[3] = {ex, ey, ez};
    return orf::eps3d(ctx, x, y, z, nx, ny, nz, nbg, nsub, method, period, nshape, shapes, outs);
}
