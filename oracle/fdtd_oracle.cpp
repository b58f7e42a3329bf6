// fdtd_oracle.cpp -- CPU restatement of OpticRCWAFDTD's Yee FDTD time loop.
//
// TEST INFRASTRUCTURE ONLY.  This file is the oracle: tests/, the smoke check
// and the cpu_baseline / reference leg of bench.py call it as the checker.
// The product (liborf_fdtd.so) never links, loads or calls it.
//
// The reference implementation (toolbox/+orf/fdtd2D.p, fdtd3D.p,
// cpmlCoefficients.p) is closed P-code and is never opened.  This code
// restates what the open help text and tests document:
//   - 2D P/A/B update, TE/TM mapping, Yee positions:   fdtd2D.m:1-7
//   - sim/out fields:                                   fdtd2D.m:9-29, fdtd2DTE.m:5-32
//   - 3D six-component update, D+/D-, PEC or wrap:      fdtd3D.m:1-9
//   - 3D source planes, monitors, H averaged onto E:    fdtd3D.m:15-28
//   - CPML (Roden-Gedney) grading and psi recursion:    cpmlCoefficients.m:1-8
//   - TF/SF one-sided plane, Ey_inc = f g(t-neff(x-xs)),
//     B_inc = neff f / eps_B:                           fdtd2DTE.m:11-15, fdtd2D.m:21-23
//   - running DFT with kernel e^{+i w t}:                fdtd2DTE.m:18
//   - flux 1/2 Re int P B* dz, -1/2 Re int P A* dx:      fdtd2DTE.m:27-31
//   - shutoff on field energy, progress every 50 steps: fdtd2DTE.m:19-21, fdtd2D.m:18-20
//   - progress fraction:                                fdtdProgress.m:1-13
// Details the closed code does not document (CPML m/kappa/alpha, pulse delay,
// DFT time stamps, energy definition) are chosen here and shared, as a
// specification, with the CUDA engine; they are listed in the repository's
// design notes.
//
// Parity status: the physics is pinned against the reference's own tests
// (tests/TestFDTD2D.m, TestFDTD3D.m, TestCPO.m tolerances: TMM slab R/T,
// exact-Yee dispersion, unidirectional source, empty-domain reflection);
// bit-level parity with the closed P-code is unpinned (it cannot run here).
#include "orf_fdtd.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.14159265358979323846;

// CPML constants (cpmlCoefficients.m:6-8 gives the grading law; the constants
// are not documented and are chosen here).
constexpr double kPmlOrder = 3.0;
constexpr double kPmlKappaMax = 1.0;
constexpr double kPmlAlphaMaxPerK0 = 0.0;   // alpha' = this * 2*pi/lambda0

// Gaussian pulse of relative 1/e spectral half-width bw at lambda0
// (fdtd2DTE.m:14-15): g(t) = exp(-((t-t0)/tau)^2) sin(k0 (t-t0)),
// tau = 2/(bw k0), t0 = 5 tau, g = 0 outside [0, 2 t0].
struct Pulse {
    double k0, tau, t0, tend;
    Pulse(double lambda0, double bw) {
        k0 = 2.0 * kPi / lambda0;
        tau = 2.0 / (bw * k0);
        t0 = 5.0 * tau;
        tend = 2.0 * t0;
    }
    double operator()(double t) const {
        if (t < 0.0 || t > tend) return 0.0;
        double u = (t - t0) / tau;
        return std::exp(-u * u) * std::sin(k0 * (t - t0));
    }
};

// 1-D CPML profile at positions u = i + off (cell units, off = 0 or 0.5),
// n points on the integer grid 0..n-1, npml cells at each end.
struct Pml1D {
    std::vector<double> b, a, kinv;
    std::vector<int> slab;   // compact slab index, -1 outside the PML
    int nslab = 0;
};

Pml1D make_pml(int n, int npts, int npml, double off, double dx, double S, double alpha_max) {
    Pml1D p;
    p.b.assign(npts, 1.0);
    p.a.assign(npts, 0.0);
    p.kinv.assign(npts, 1.0);
    p.slab.assign(npts, -1);
    if (npml <= 0) return p;
    const double m = kPmlOrder;
    const double sigma_max = 0.8 * (m + 1.0) / dx;
    const double lo = npml, hi = (n - 1) - npml;
    for (int i = 0; i < npts; ++i) {
        double u = i + off;
        double depth = 0.0;
        if (u < lo) depth = lo - u;
        else if (u > hi) depth = u - hi;
        if (depth <= 0.0) continue;
        double r = std::min(depth / npml, 1.0);
        double rm = std::pow(r, m);
        double sigma = sigma_max * rm;
        double kappa = 1.0 + (kPmlKappaMax - 1.0) * rm;
        double alpha = alpha_max * (1.0 - r);
        double b = std::exp(-(sigma / kappa + alpha) * S);
        double den = sigma * kappa + kappa * kappa * alpha;
        p.b[i] = b;
        p.a[i] = den > 0.0 ? sigma / den * (b - 1.0) : 0.0;
        p.kinv[i] = 1.0 / kappa;
        p.slab[i] = p.nslab++;
    }
    return p;
}

// fdtdProgress.m:6-12
double progress_fraction(double t, double src_end, double ratio, double shutoff) {
    double frac;
    if (t <= src_end) {
        frac = 0.3 * t / src_end;
    } else {
        double so = shutoff > 0.0 ? shutoff : 1e-300;
        double decay = std::log(std::max(ratio, so)) / std::log(so);
        frac = 0.3 + 0.7 * std::max(0.0, std::min(1.0, decay));
    }
    return std::max(0.0, std::min(1.0, frac));
}

int64_t max_steps(double max_time, double S) {
    double r = max_time / S;
    int64_t n = (int64_t)std::ceil(r - 1e-9);
    return n < 0 ? 0 : n;
}

constexpr int kCheckEvery = 50;

// ------------------------------------------------------------------ 2D --
template <class R>
int run2d(const orf_sim2d* s, orf_out2d* o, orf_progress_fn progress, void* user, double* const* fields) {
    auto t_start = std::chrono::steady_clock::now();
    const int nx = s->nx, nz = s->nz;
    const bool per = s->periodic_z != 0;
    const bool te = s->pol == ORF_TE;
    const int nzA = per ? nz : nz - 1;
    const int nxB = nx - 1;
    const double C = s->courant;
    const double dx = s->dx;
    const double S = C * dx;
    const int npx = s->npml_x, npz = per ? 0 : s->npml_z;

    auto iP = [&](int i, int k) { return (size_t)i + (size_t)nx * k; };
    auto iB = [&](int i, int k) { return (size_t)i + (size_t)nxB * k; };

    std::vector<R> P((size_t)nx * nz, R(0)), A((size_t)nx * std::max(nzA, 0), R(0)),
        B((size_t)std::max(nxB, 0) * nz, R(0));
    std::vector<R> cP(P.size()), cA(A.size()), cB(B.size());
    for (size_t q = 0; q < P.size(); ++q) cP[q] = te ? R(C / s->eps[q]) : R(C);
    for (size_t q = 0; q < A.size(); ++q) cA[q] = te ? R(C) : R(C / s->eps_x[q]);
    for (size_t q = 0; q < B.size(); ++q) cB[q] = te ? R(C) : R(C / s->eps_z[q]);

    const double alpha_max = kPmlAlphaMaxPerK0 * 2.0 * kPi / s->src_lambda0;
    Pml1D px = make_pml(nx, nx, npx, 0.0, dx, S, alpha_max);      // P columns
    Pml1D pxh = make_pml(nx, nxB, npx, 0.5, dx, S, alpha_max);    // B columns
    Pml1D pz = make_pml(nz, nz, npz, 0.0, dx, S, alpha_max);      // P rows
    Pml1D pzh = make_pml(nz, nzA, npz, 0.5, dx, S, alpha_max);    // A rows
    // psi in compact slabs, in units of field differences
    std::vector<R> psiBx((size_t)pxh.nslab * nz, R(0)), psiPx((size_t)px.nslab * nz, R(0));
    std::vector<R> psiAz((size_t)nx * pzh.nslab, R(0)), psiPz((size_t)nx * pz.nslab, R(0));
    std::vector<R> pxh_b(pxh.b.begin(), pxh.b.end()), pxh_a(pxh.a.begin(), pxh.a.end()), pxh_k(pxh.kinv.begin(), pxh.kinv.end());
    std::vector<R> px_b(px.b.begin(), px.b.end()), px_a(px.a.begin(), px.a.end()), px_k(px.kinv.begin(), px.kinv.end());
    std::vector<R> pzh_b(pzh.b.begin(), pzh.b.end()), pzh_a(pzh.a.begin(), pzh.a.end()), pzh_k(pzh.kinv.begin(), pzh.kinv.end());
    std::vector<R> pz_b(pz.b.begin(), pz.b.end()), pz_a(pz.a.begin(), pz.a.end()), pz_k(pz.kinv.begin(), pz.kinv.end());

    // source (one-sided TF/SF plane at P column ix toward +x)
    const int sx = s->src_ix;
    const Pulse g(s->src_lambda0, s->src_bw);
    std::vector<double> fB(nz, 0.0), fP(nz, 0.0);   // B_inc / P_inc profiles
    for (int k = 0; k < nz; ++k) {
        double f = s->src_profile[k];
        double epsB = te ? 1.0 : s->eps_z[iB(sx - 1, k)];
        fP[k] = f;
        fB[k] = s->src_neff * f / epsB;
    }

    // DFT accumulators (always double, fdtd2DTE.m:24-25)
    const int nL = s->n_lambda, nM = s->n_mon, nMZ = s->n_monz;
    std::vector<double> w(nL);
    for (int l = 0; l < nL; ++l) w[l] = 2.0 * kPi / s->lambdas[l];
    std::vector<double> dP((size_t)2 * nz * nL * nM, 0.0), dB(dP.size(), 0.0);
    std::vector<double> dPZ((size_t)2 * nx * nL * nMZ, 0.0), dAZ(dPZ.size(), 0.0);

    const int64_t nmax = max_steps(s->max_time, S);
    const double src_end = g.tend;
    double peak = 0.0;
    bool converged = false;
    int64_t n = 0;
    char msg[128];

    for (n = 0; n < nmax; ++n) {
        const double tn = n * S;                  // P time level
        const double th = (n + 0.5) * S;          // A, B time level after the H update
        const double gE = g(tn);
        const double gH = g(th + s->src_neff * 0.5 * dx);

        // ---- H update: A (d/dz of P), B (d/dx of P)
#pragma omp parallel for schedule(static)
        for (int k = 0; k < nzA; ++k) {
            const int kp = (k + 1 < nz) ? k + 1 : 0;   // only wraps when periodic
            const int sz = pzh.slab[k];
            for (int i = 0; i < nx; ++i) {
                R d = P[iP(i, kp)] - P[iP(i, k)];
                if (sz >= 0) {
                    R& ps = psiAz[(size_t)i + (size_t)nx * sz];
                    ps = pzh_b[k] * ps + pzh_a[k] * d;
                    d = d * pzh_k[k] + ps;
                }
                A[iP(i, k)] += cA[iP(i, k)] * d;
            }
        }
#pragma omp parallel for schedule(static)
        for (int k = 0; k < nz; ++k) {
            for (int i = 0; i < nxB; ++i) {
                R d = P[iP(i + 1, k)] - P[iP(i, k)];
                const int sxs = pxh.slab[i];
                if (sxs >= 0) {
                    R& ps = psiBx[(size_t)sxs + (size_t)pxh.nslab * k];
                    ps = pxh_b[i] * ps + pxh_a[i] * d;
                    d = d * pxh_k[i] + ps;
                }
                B[iB(i, k)] -= cB[iB(i, k)] * d;
            }
            // TF/SF: the B column left of the plane is scattered field; it saw
            // the total P at the plane, so remove the incident part.
            if (sx >= 1) B[iB(sx - 1, k)] += cB[iB(sx - 1, k)] * R(fP[k] * gE);
        }

        // ---- E update: P
#pragma omp parallel for schedule(static)
        for (int k = 0; k < nz; ++k) {
            const int km = k > 0 ? k - 1 : (per ? nz - 1 : -1);
            const int szp = pz.slab[k];
            for (int i = 0; i < nx; ++i) {
                R a1 = (k < nzA) ? A[iP(i, k)] : R(0);
                R a0 = (km >= 0) ? A[iP(i, km)] : R(0);
                R b1 = (i < nxB) ? B[iB(i, k)] : R(0);
                R b0 = (i >= 1) ? B[iB(i - 1, k)] : R(0);
                R da = a1 - a0, db = b1 - b0;
                if (szp >= 0) {
                    R& ps = psiPz[(size_t)i + (size_t)nx * szp];
                    ps = pz_b[k] * ps + pz_a[k] * da;
                    da = da * pz_k[k] + ps;
                }
                const int sxp = px.slab[i];
                if (sxp >= 0) {
                    R& ps = psiPx[(size_t)sxp + (size_t)px.nslab * k];
                    ps = px_b[i] * ps + px_a[i] * db;
                    db = db * px_k[i] + ps;
                }
                P[iP(i, k)] += cP[iP(i, k)] * (da - db);
            }
            // TF/SF: the plane is total field; its left B neighbour is scattered.
            P[iP(sx, k)] += cP[iP(sx, k)] * R(fB[k] * gH);
        }

        // ---- running DFT: P at t_{n+1}, B (A) averaged onto the P line at t_{n+1/2}
        const double t1 = (n + 1) * S;
        for (int l = 0; l < nL; ++l) {
            const double cp = std::cos(w[l] * t1) * S, sp = std::sin(w[l] * t1) * S;
            const double ch = std::cos(w[l] * th) * S, sh = std::sin(w[l] * th) * S;
            for (int m = 0; m < nM; ++m) {
                const int ix = s->monitors[m];
                double* Pm = &dP[2 * ((size_t)nz * (l + (size_t)nL * m))];
                double* Bm = &dB[2 * ((size_t)nz * (l + (size_t)nL * m))];
                for (int k = 0; k < nz; ++k) {
                    double pv = P[iP(ix, k)];
                    double b1 = ix < nxB ? (double)B[iB(ix, k)] : 0.0;
                    double b0 = ix >= 1 ? (double)B[iB(ix - 1, k)] : 0.0;
                    double bv = 0.5 * (b0 + b1);
                    Pm[2 * k] += pv * cp;  Pm[2 * k + 1] += pv * sp;
                    Bm[2 * k] += bv * ch;  Bm[2 * k + 1] += bv * sh;
                }
            }
            for (int m = 0; m < nMZ; ++m) {
                const int kz = s->monitors_z[m];
                double* Pm = &dPZ[2 * ((size_t)nx * (l + (size_t)nL * m))];
                double* Am = &dAZ[2 * ((size_t)nx * (l + (size_t)nL * m))];
                const int km = kz > 0 ? kz - 1 : (per ? nz - 1 : -1);
                for (int i = 0; i < nx; ++i) {
                    double pv = P[iP(i, kz)];
                    double a1 = kz < nzA ? (double)A[iP(i, kz)] : 0.0;
                    double a0 = km >= 0 ? (double)A[iP(i, km)] : 0.0;
                    double av = 0.5 * (a0 + a1);
                    Pm[2 * i] += pv * cp;  Pm[2 * i + 1] += pv * sp;
                    Am[2 * i] += av * ch;  Am[2 * i + 1] += av * sh;
                }
            }
        }

        // ---- energy check and progress every 50 steps
        if ((n + 1) % kCheckEvery == 0) {
            double e = 0.0;
#pragma omp parallel for reduction(+ : e) schedule(static)
            for (int k = 0; k < nz; ++k) {
                double ek = 0.0;
                for (int i = 0; i < nx; ++i) {
                    double p = P[iP(i, k)];
                    ek += (te ? s->eps[iP(i, k)] : 1.0) * p * p;
                    if (k < nzA) { double a = A[iP(i, k)]; ek += (te ? 1.0 : s->eps_x[iP(i, k)]) * a * a; }
                    if (i < nxB) { double b = B[iB(i, k)]; ek += (te ? 1.0 : s->eps_z[iB(i, k)]) * b * b; }
                }
                e += ek;
            }
            peak = std::max(peak, e);
            double ratio = peak > 0.0 ? e / peak : 1.0;
            bool stop = (t1 > src_end) && (s->shutoff > 0.0) && (e < s->shutoff * peak);
            if (progress) {
                double fr = stop ? 1.0 : progress_fraction(t1, src_end, ratio, s->shutoff);
                std::snprintf(msg, sizeof msg, "step %lld, t = %.3g um", (long long)(n + 1), t1);
                if (progress(fr, msg, user)) return ORF_ECANCELLED;
            }
            if (stop) { converged = true; ++n; break; }
        }
    }

    // ---- outputs
    if (fields) {
        for (size_t q = 0; q < P.size(); ++q) if (fields[0]) fields[0][q] = P[q];
        for (size_t q = 0; q < A.size(); ++q) if (fields[1]) fields[1][q] = A[q];
        for (size_t q = 0; q < B.size(); ++q) if (fields[2]) fields[2][q] = B[q];
    }
    const int64_t steps = n;
    if (o->flux) {
        for (int m = 0; m < nM; ++m)
            for (int l = 0; l < nL; ++l) {
                const double* Pm = &dP[2 * ((size_t)nz * (l + (size_t)nL * m))];
                const double* Bm = &dB[2 * ((size_t)nz * (l + (size_t)nL * m))];
                double acc = 0.0;
                for (int k = 0; k < nz; ++k) acc += Pm[2 * k] * Bm[2 * k] + Pm[2 * k + 1] * Bm[2 * k + 1];
                o->flux[m + (size_t)nM * l] = 0.5 * acc * dx;
            }
    }
    if (o->flux_z) {
        for (int m = 0; m < nMZ; ++m)
            for (int l = 0; l < nL; ++l) {
                const double* Pm = &dPZ[2 * ((size_t)nx * (l + (size_t)nL * m))];
                const double* Am = &dAZ[2 * ((size_t)nx * (l + (size_t)nL * m))];
                double acc = 0.0;
                for (int i = 0; i < nx; ++i) acc += Pm[2 * i] * Am[2 * i] + Pm[2 * i + 1] * Am[2 * i + 1];
                o->flux_z[m + (size_t)nMZ * l] = -0.5 * acc * dx;
            }
    }
    if (o->P) std::memcpy(o->P, dP.data(), dP.size() * sizeof(double));
    if (o->B) std::memcpy(o->B, dB.data(), dB.size() * sizeof(double));
    if (o->PZ) std::memcpy(o->PZ, dPZ.data(), dPZ.size() * sizeof(double));
    if (o->AZ) std::memcpy(o->AZ, dAZ.data(), dAZ.size() * sizeof(double));
    o->converged = converged ? 1 : 0;
    o->steps = steps;
    o->time = steps * S;
    o->wall_time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    return ORF_OK;
}

// ------------------------------------------------------------------ 3D --
template <class R>
struct F3 {
    int n[3];
    bool per[3];
    size_t idx(int i, int j, int k) const { return (size_t)i + (size_t)n[0] * ((size_t)j + (size_t)n[1] * k); }
};

template <class R>
int run3d(const orf_sim3d* s, orf_out3d* o, orf_progress_fn progress, void* user, double* const* fields) {
    auto t_start = std::chrono::steady_clock::now();
    const int n[3] = {s->nx, s->ny, s->nz};
    const bool per[3] = {s->periodic[0] != 0, s->periodic[1] != 0, s->periodic[2] != 0};
    const size_t N = (size_t)n[0] * n[1] * n[2];
    const double C = s->courant, d = s->d, S = C * d;
    auto idx = [&](int i, int j, int k) { return (size_t)i + (size_t)n[0] * ((size_t)j + (size_t)n[1] * k); };
    const size_t st[3] = {1, (size_t)n[0], (size_t)n[0] * n[1]};

    std::vector<R> E[3], H[3], cE[3];
    const double* epsc[3] = {s->eps_x, s->eps_y, s->eps_z};
    for (int c = 0; c < 3; ++c) {
        E[c].assign(N, R(0));
        H[c].assign(N, R(0));
        cE[c].resize(N);
        for (size_t q = 0; q < N; ++q) cE[c][q] = R(C / epsc[c][q]);
    }
    const double alpha_max = kPmlAlphaMaxPerK0 * 2.0 * kPi / s->src_lambda0;
    Pml1D pI[3], pH[3];   // integer (E-derivative) and half (H-derivative) positions
    int np[3];
    for (int q = 0; q < 3; ++q) {
        np[q] = per[q] ? 0 : s->npml[q];
        pI[q] = make_pml(n[q], n[q], np[q], 0.0, d, S, alpha_max);
        pH[q] = make_pml(n[q], n[q], np[q], 0.5, d, S, alpha_max);
    }
    // psi for (field component c, derivative axis q != c): compact along q
    auto psi_size = [&](const Pml1D& p, int q) {
        size_t sz = 1;
        for (int a = 0; a < 3; ++a) sz *= (a == q) ? (size_t)p.nslab : (size_t)n[a];
        return sz;
    };
    std::vector<R> psiE[3][3], psiH[3][3];
    for (int c = 0; c < 3; ++c)
        for (int q = 0; q < 3; ++q) {
            if (q == c) continue;
            psiE[c][q].assign(psi_size(pI[q], q), R(0));
            psiH[c][q].assign(psi_size(pH[q], q), R(0));
        }
    auto psi_idx = [&](const Pml1D& p, int q, int slab, int i, int j, int k) {
        int v[3] = {i, j, k};
        v[q] = slab;
        int m[3] = {n[0], n[1], n[2]};
        m[q] = p.nslab;
        return (size_t)v[0] + (size_t)m[0] * ((size_t)v[1] + (size_t)m[1] * v[2]);
    };

    // source plane
    const int sa = s->src_axis, sb = (sa + 1) % 3, sc = (sa + 2) % 3;   // d, a, b
    const int ss = s->src_index;
    const int Na = n[sb], Nb = n[sc];
    const Pulse g(s->src_lambda0, s->src_bw);

    const int nL = s->n_lambda, nM = s->n_mon;
    std::vector<double> w(nL);
    for (int l = 0; l < nL; ++l) w[l] = 2.0 * kPi / s->lambdas[l];
    std::vector<std::vector<double>> mEa(nM), mEb(nM), mHa(nM), mHb(nM);
    for (int m = 0; m < nM; ++m) {
        int q = s->mon_axis[m];
        size_t sz = (size_t)2 * n[(q + 1) % 3] * n[(q + 2) % 3] * nL;
        mEa[m].assign(sz, 0.0); mEb[m].assign(sz, 0.0); mHa[m].assign(sz, 0.0); mHb[m].assign(sz, 0.0);
    }

    const int64_t nmax = max_steps(s->max_time, S);
    const double src_end = g.tend;
    double peak = 0.0;
    bool converged = false;
    int64_t step = 0;
    char msg[128];

    // neighbour access with PEC (zero) or wrap
    auto fwd = [&](const std::vector<R>& F, int q, int i, int j, int k) -> R {
        int v[3] = {i, j, k};
        v[q] += 1;
        if (v[q] >= n[q]) { if (!per[q]) return R(0); v[q] = 0; }
        return F[idx(v[0], v[1], v[2])];
    };
    auto bwd = [&](const std::vector<R>& F, int q, int i, int j, int k) -> R {
        int v[3] = {i, j, k};
        v[q] -= 1;
        if (v[q] < 0) { if (!per[q]) return R(0); v[q] = n[q] - 1; }
        return F[idx(v[0], v[1], v[2])];
    };

    for (step = 0; step < nmax; ++step) {
        const double tn = step * S, th = (step + 0.5) * S;
        const double gE = g(tn), gH = g(th + s->src_neff * 0.5 * d);

        // H_c -= C (D+_{c1} E_{c2} - D+_{c2} E_{c1})   (fdtd3D.m:7)
        for (int c = 0; c < 3; ++c) {
            const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
#pragma omp parallel for schedule(static)
            for (int k = 0; k < n[2]; ++k)
                for (int j = 0; j < n[1]; ++j)
                    for (int i = 0; i < n[0]; ++i) {
                        const int v[3] = {i, j, k};
                        const size_t q0 = idx(i, j, k);
                        R d1 = fwd(E[c2], c1, i, j, k) - E[c2][q0];
                        R d2 = fwd(E[c1], c2, i, j, k) - E[c1][q0];
                        int s1 = pH[c1].slab[v[c1]];
                        if (s1 >= 0) {
                            R& ps = psiH[c][c1][psi_idx(pH[c1], c1, s1, i, j, k)];
                            ps = R(pH[c1].b[v[c1]]) * ps + R(pH[c1].a[v[c1]]) * d1;
                            d1 = d1 * R(pH[c1].kinv[v[c1]]) + ps;
                        }
                        int s2 = pH[c2].slab[v[c2]];
                        if (s2 >= 0) {
                            R& ps = psiH[c][c2][psi_idx(pH[c2], c2, s2, i, j, k)];
                            ps = R(pH[c2].b[v[c2]]) * ps + R(pH[c2].a[v[c2]]) * d2;
                            d2 = d2 * R(pH[c2].kinv[v[c2]]) + ps;
                        }
                        H[c][q0] -= R(C) * (d1 - d2);
                    }
        }
        // TF/SF on the H plane at index ss-1 (scattered side)
        if (ss >= 1) {
            for (int ib = 0; ib < Nb; ++ib)
                for (int ia = 0; ia < Na; ++ia) {
                    int v[3]; v[sa] = ss - 1; v[sb] = ia; v[sc] = ib;
                    size_t q0 = idx(v[0], v[1], v[2]);
                    size_t pq = (size_t)ia + (size_t)Na * ib;
                    H[sb][q0] -= R(C) * R(s->src_Eb[pq] * gE);
                    H[sc][q0] += R(C) * R(s->src_Ea[pq] * gE);
                }
        }
        // E_c += C/eps_c (D-_{c1} H_{c2} - D-_{c2} H_{c1})
        for (int c = 0; c < 3; ++c) {
            const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
#pragma omp parallel for schedule(static)
            for (int k = 0; k < n[2]; ++k)
                for (int j = 0; j < n[1]; ++j)
                    for (int i = 0; i < n[0]; ++i) {
                        const int v[3] = {i, j, k};
                        const size_t q0 = idx(i, j, k);
                        R d1 = H[c2][q0] - bwd(H[c2], c1, i, j, k);
                        R d2 = H[c1][q0] - bwd(H[c1], c2, i, j, k);
                        int s1 = pI[c1].slab[v[c1]];
                        if (s1 >= 0) {
                            R& ps = psiE[c][c1][psi_idx(pI[c1], c1, s1, i, j, k)];
                            ps = R(pI[c1].b[v[c1]]) * ps + R(pI[c1].a[v[c1]]) * d1;
                            d1 = d1 * R(pI[c1].kinv[v[c1]]) + ps;
                        }
                        int s2 = pI[c2].slab[v[c2]];
                        if (s2 >= 0) {
                            R& ps = psiE[c][c2][psi_idx(pI[c2], c2, s2, i, j, k)];
                            ps = R(pI[c2].b[v[c2]]) * ps + R(pI[c2].a[v[c2]]) * d2;
                            d2 = d2 * R(pI[c2].kinv[v[c2]]) + ps;
                        }
                        E[c][q0] += cE[c][q0] * (d1 - d2);
                    }
        }
        // TF/SF on the E plane at index ss (total side)
        for (int ib = 0; ib < Nb; ++ib)
            for (int ia = 0; ia < Na; ++ia) {
                int v[3]; v[sa] = ss; v[sb] = ia; v[sc] = ib;
                size_t q0 = idx(v[0], v[1], v[2]);
                size_t pq = (size_t)ia + (size_t)Na * ib;
                E[sb][q0] += cE[sb][q0] * R(s->src_Hb[pq] * gH);
                E[sc][q0] -= cE[sc][q0] * R(s->src_Ha[pq] * gH);
            }

        // DFT on monitor planes
        const double t1 = (step + 1) * S;
        for (int m = 0; m < nM; ++m) {
            const int q = s->mon_axis[m], qa = (q + 1) % 3, qb = (q + 2) % 3;
            const int mi = s->mon_index[m];
            const int na = n[qa], nb = n[qb];
            for (int ib = 0; ib < nb; ++ib)
                for (int ia = 0; ia < na; ++ia) {
                    int v[3]; v[q] = mi; v[qa] = ia; v[qb] = ib;
                    size_t q0 = idx(v[0], v[1], v[2]);
                    double ea = E[qa][q0], eb = E[qb][q0];
                    double ha = 0.5 * ((double)H[qa][q0] + (double)bwd(H[qa], q, v[0], v[1], v[2]));
                    double hb = 0.5 * ((double)H[qb][q0] + (double)bwd(H[qb], q, v[0], v[1], v[2]));
                    size_t p = (size_t)ia + (size_t)na * ib;
                    for (int l = 0; l < nL; ++l) {
                        const double cp = std::cos(w[l] * t1) * S, sp = std::sin(w[l] * t1) * S;
                        const double ch = std::cos(w[l] * th) * S, sh = std::sin(w[l] * th) * S;
                        size_t o2 = 2 * (p + (size_t)na * nb * l);
                        mEa[m][o2] += ea * cp; mEa[m][o2 + 1] += ea * sp;
                        mEb[m][o2] += eb * cp; mEb[m][o2 + 1] += eb * sp;
                        mHa[m][o2] += ha * ch; mHa[m][o2 + 1] += ha * sh;
                        mHb[m][o2] += hb * ch; mHb[m][o2 + 1] += hb * sh;
                    }
                }
        }

        if ((step + 1) % kCheckEvery == 0) {
            double e = 0.0;
#pragma omp parallel for reduction(+ : e) schedule(static)
            for (int k = 0; k < n[2]; ++k) {
                double ek = 0.0;
                for (int j = 0; j < n[1]; ++j)
                    for (int i = 0; i < n[0]; ++i) {
                        size_t q0 = idx(i, j, k);
                        for (int c = 0; c < 3; ++c) {
                            double ev = E[c][q0], hv = H[c][q0];
                            ek += epsc[c][q0] * ev * ev + hv * hv;
                        }
                    }
                e += ek;
            }
            peak = std::max(peak, e);
            double ratio = peak > 0.0 ? e / peak : 1.0;
            bool stop = (t1 > src_end) && (s->shutoff > 0.0) && (e < s->shutoff * peak);
            if (progress) {
                double fr = stop ? 1.0 : progress_fraction(t1, src_end, ratio, s->shutoff);
                std::snprintf(msg, sizeof msg, "step %lld, t = %.3g um", (long long)(step + 1), t1);
                if (progress(fr, msg, user)) return ORF_ECANCELLED;
            }
            if (stop) { converged = true; ++step; break; }
        }
    }
    (void)st;
    if (fields) {
        for (int c = 0; c < 3; ++c) {
            if (fields[c]) for (size_t q = 0; q < N; ++q) fields[c][q] = E[c][q];
            if (fields[3 + c]) for (size_t q = 0; q < N; ++q) fields[3 + c][q] = H[c][q];
        }
    }

    for (int m = 0; m < nM; ++m) {
        const int q = s->mon_axis[m];
        const size_t np2 = (size_t)n[(q + 1) % 3] * n[(q + 2) % 3];
        for (int l = 0; l < nL; ++l) {
            double acc = 0.0;
            for (size_t p = 0; p < np2; ++p) {
                size_t o2 = 2 * (p + np2 * l);
                // Re(Ea Hb* - Eb Ha*)
                acc += mEa[m][o2] * mHb[m][o2] + mEa[m][o2 + 1] * mHb[m][o2 + 1];
                acc -= mEb[m][o2] * mHa[m][o2] + mEb[m][o2 + 1] * mHa[m][o2 + 1];
            }
            if (o->flux) o->flux[m + (size_t)nM * l] = 0.5 * acc * d * d;
        }
        if (o->mon_Ea && o->mon_Ea[m]) std::memcpy(o->mon_Ea[m], mEa[m].data(), mEa[m].size() * sizeof(double));
        if (o->mon_Eb && o->mon_Eb[m]) std::memcpy(o->mon_Eb[m], mEb[m].data(), mEb[m].size() * sizeof(double));
        if (o->mon_Ha && o->mon_Ha[m]) std::memcpy(o->mon_Ha[m], mHa[m].data(), mHa[m].size() * sizeof(double));
        if (o->mon_Hb && o->mon_Hb[m]) std::memcpy(o->mon_Hb[m], mHb[m].data(), mHb[m].size() * sizeof(double));
    }
    o->converged = converged ? 1 : 0;
    o->steps = step;
    o->time = step * S;
    o->wall_time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    return ORF_OK;
}

}  // namespace

extern "C" {

// precision: 0 = FP64 fields, 1 = FP32 fields (DFT always FP64).
int oracle_fdtd2d_run(const orf_sim2d* s, orf_out2d* o, orf_progress_fn progress, void* user,
                      int threads, double* const* fields) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    if (s->precision == ORF_SINGLE) return run2d<float>(s, o, progress, user, fields);
    return run2d<double>(s, o, progress, user, fields);
}

int oracle_fdtd3d_run(const orf_sim3d* s, orf_out3d* o, orf_progress_fn progress, void* user,
                      int threads, double* const* fields) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    if (s->precision == ORF_SINGLE) return run3d<float>(s, o, progress, user, fields);
    return run3d<double>(s, o, progress, user, fields);
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Pulse value, exposed so tests can check the shared pulse definition.
double oracle_pulse(double lambda0, double bw, double t) { return Pulse(lambda0, bw)(t); }

}  // extern "C"
