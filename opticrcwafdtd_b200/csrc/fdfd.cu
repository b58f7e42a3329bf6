// fdfd.cu -- orf_fdfd2d_*: the 2D TE frequency-domain solver with its adjoint
// (toolbox/+orf/fdfd2D.m:1-19) on the device.
//
//   (1/s_x) d/dx((1/s_x) dE/dx) + (1/s_z) d/dz((1/s_z) dE/dz) + k0^2 eps E = -J
//
// on the FDTD's E_y points, E = 0 outside the grid, stretched-coordinate PML
// s = 1 + i a (depth / L)^3 (e^{-i w t}), discretised with the 5-point
// stencil.  Ordered block by block along the longer axis, the matrix is block
// tridiagonal: blocks of m = min(nx, nz) unknowns (one line across the
// shorter axis), tridiagonal diagonal blocks, diagonal couplings to the
// neighbouring lines.  The factorisation is the block LU of that structure,
//   D_0 = A_00,  D_b = A_bb - B_b D_{b-1}^{-1} C_{b-1},
// with every D_b inverted by Gauss-Jordan elimination with partial pivoting
// and the inverses kept on the device; a solve is then a forward and a
// backward sweep of matrix-vector products with them (m^2 per line), for A
// and, with the same inverses, for A.' (the adjoint, fdfd2D.m:13-15).
//
// The block inversions run on one thread-block cluster of 8 CTAs (16, a
// non-portable cluster size, for blocks above 128 points): CTA c
// holds rows [c R, c R + R) of the block in registers (one column per
// thread, the rows split over up to four thread groups).
// At each pivot step every CTA stores its pivot candidate into the shared
// memory of every CTA of the cluster; after a cluster barrier all pick the
// same pivot, its owner stores the pivot row into every CTA (and the owner
// of row k that row into the pivot row's owner), and after a second barrier
// each CTA eliminates from local copies: no remote read, one row broadcast
// per pivot.  The next block's Schur complement is formed from the
// inverse while it is still in registers.  Cluster barriers are hardware
// barriers: no CTA spins on memory.
#include <cooperative_groups.h>

#include <complex>

#include "runtime.cuh"

namespace cg = cooperative_groups;

namespace orf {
namespace {

constexpr int kFdMaxM = 384;      // largest block (the shorter grid axis)
constexpr int kFdMaxC = 16;       // largest cluster
constexpr int kSolveThreads = 256;

struct FdfdDev {
    int m, nb;                 // block size, number of blocks
    const double2* diag;       // [nb][m]
    const double2* wm;         // [nb][m]: coupling to p - 1 inside the block
    const double2* wp;         // [nb][m]: to p + 1
    const double2* bm;         // [nb][m]: to the same p of block b - 1
    const double2* bp;         // [nb][m]: to block b + 1
    double2* inv;              // [nb][m][m]: D_b^{-1}, row-major
    int* fault;                // a zero pivot (singular block)
    double2* xpan;             // [m][kPanel]: the blocked factorisation's panel, every row
    double2* xrow;             // [kPanel][m]: its pivot rows
};

struct FdCand {   // a CTA's pivot candidate: |value|^2 and row (m: none)
    double v;
    int i, pad;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }

// Block LU of the whole operator: block b inverted in place, stored to
// P.inv[b], then turned into D_{b+1} = A - B D_b^{-1} C in registers.
// Thread (j, h) = (t % mp, t / mp) holds column j of the CTA's rows
// h*RS .. h*RS + RS - 1 (TPC groups of RS rows; mp = m rounded up to a warp),
// so that a pivot step's row work is spread over TPC times as many warps.
template <int RS, int TPC, int NT>
__global__ void __launch_bounds__(NT, 1) k_fdfd_factor(FdfdDev P) {
    constexpr int RM = RS * TPC;   // rows per CTA at most
    cg::cluster_group cl = cg::this_cluster();
    const int C = (int)cl.num_blocks();
    const int c = (int)cl.block_rank();
    const int m = P.m;
    const int mp = (m + 31) / 32 * 32;
    const int R = (m + C - 1) / C;
    const int r0 = c * R;
    const int nr = max(0, min(m, r0 + R) - r0);
    const int t = threadIdx.x;
    const int j = t % mp, h = t / mp;
    const int q0 = h * RS;            // first of this thread's rows, local to the CTA
    const int r1 = r0 + q0;           // ... as a row of the block
    const int nq = max(0, min(RS, nr - q0));   // this thread's rows
    const bool col = j < m;

    // Exchange buffers, per pivot parity, written by the other CTAs of the
    // cluster (remote stores before a cluster barrier) and read locally after
    // it: every CTA's pivot candidate (|value|^2, row), the pivot row, and
    // row k (sent to the pivot row's owner only).
    __shared__ FdCand s_cv[2][kFdMaxC];
    // s_prow[2] and s_rowk[2] in the pivot steps; the column exchange of a
    // finished block (up to 4 row groups) reuses them: no CTA writes them
    // again before the next block's first candidate barrier, which this CTA
    // reaches only after its exchange
    __shared__ double2 s_ex[4][kFdMaxM];
    double2 (*s_prow)[kFdMaxM] = s_ex;
    double2 (*s_rowk)[kFdMaxM] = s_ex + 2;
    __shared__ double2 s_colk[2][RM];   // column k of the owned rows, before the exchange
    __shared__ FdCand s_hc[2][TPC];     // the row groups' candidates
    __shared__ int s_piv[kFdMaxM];
    __shared__ int s_perm[kFdMaxM];
    static_assert(TPC <= 4, "the column exchange uses s_ex");

    double2 a[RS];
#pragma unroll
    for (int u = 0; u < RS; ++u) a[u] = make_double2(0.0, 0.0);
    long long g = 0;   // pivot steps so far (buffer parity)

    for (int b = 0; b < P.nb; ++b) {
        // ---- D_b: the tridiagonal block minus B_b D_{b-1}^{-1} C_{b-1}
        if (col) {
            const double2 cpj = b > 0 ? P.bp[(size_t)(b - 1) * m + j] : make_double2(0.0, 0.0);
#pragma unroll
            for (int u = 0; u < RS; ++u) {
                if (u >= nq) break;
                const int p = r1 + u;
                const size_t o = (size_t)b * m + p;
                double2 v = make_double2(0.0, 0.0);
                if (b > 0) {
                    const double2 s = cmul(cmul(P.bm[o], a[u]), cpj);
                    v = make_double2(-s.x, -s.y);
                }
                if (j == p) v = cadd(v, P.diag[o]);
                else if (j == p - 1) v = cadd(v, P.wm[o]);
                else if (j == p + 1) v = cadd(v, P.wp[o]);
                a[u] = v;
            }
        }
        // ---- Gauss-Jordan inversion in place, partial pivoting
        for (int k = 0; k < m; ++k, ++g) {
            const int par = (int)(g & 1);
            if (j == k) {   // the group's candidate: the largest |a| of column k on its rows >= k
                double best = -1.0;
                int bi = m;
#pragma unroll
                for (int u = 0; u < RS; ++u) {
                    if (q0 + u < RM) s_colk[par][q0 + u] = a[u];
                    if (u >= nq) continue;
                    const int r = r1 + u;
                    const double v = cabs2(a[u]);
                    if (r >= k && v > best) {
                        best = v;
                        bi = r;
                    }
                }
                s_hc[par][h] = FdCand{best, bi, 0};
            }
            __syncthreads();
            // the CTA's candidate (the same in every thread)
            double cbest = -1.0;
            int bl = m;
#pragma unroll
            for (int hh = 0; hh < TPC; ++hh) {
                const FdCand cd = s_hc[par][hh];
                if (cd.i < m && (cd.v > cbest || (cd.v == cbest && cd.i < bl))) {
                    cbest = cd.v;
                    bl = cd.i;
                }
            }
            if (t == 0) {   // the CTA's candidate into every CTA
                const FdCand cd{cbest, bl, 0};
                for (int c2 = 0; c2 < C; ++c2) *cl.map_shared_rank(&s_cv[par][c], c2) = cd;
            }
            cl.sync();   // every CTA's candidate is here
            // the pivot row: the largest candidate, the lowest row on a tie;
            // lane c2 of every warp reads CTA c2's candidate and the warp
            // reduces (every warp decides the same)
            int p;
            {
                const int lane = t & 31;
                double best = -1.0;
                int bi = m;
                if (lane < C) {
                    const FdCand cd = s_cv[par][lane];
                    if (cd.i < m) {
                        best = cd.v;
                        bi = cd.i;
                    }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                    if (ob > best || (ob == best && oi < bi)) {
                        best = ob;
                        bi = oi;
                    }
                }
                p = bi;
            }
            if (col) {   // the pivot row into every CTA, row k into the pivot row's owner
                const bool hasp = p >= r1 && p < r1 + nq, hask = p != k && k >= r1 && k < r1 + nq;
                if (hasp || hask) {
                    double2 vp = make_double2(0.0, 0.0), vk = make_double2(0.0, 0.0);
#pragma unroll
                    for (int u = 0; u < RS; ++u) {
                        if (r1 + u == p) vp = a[u];
                        if (r1 + u == k) vk = a[u];
                    }
                    if (hasp)
                        for (int c2 = 0; c2 < C; ++c2) cl.map_shared_rank(&s_prow[par][0], c2)[j] = vp;
                    if (hask) cl.map_shared_rank(&s_rowk[par][0], p / R)[j] = vk;
                }
            }
            cl.sync();   // the pivot row (and, at its owner, row k) is here
            const double2* prow_all = &s_prow[par][0];
            const double2* rowk = &s_rowk[par][0];
            const double2 pk = prow_all[k];
            const double dd = cabs2(pk);
            const double inv_dd = dd == 0.0 ? 0.0 : 1.0 / dd;
            const double2 ip = make_double2(pk.x * inv_dd, -pk.y * inv_dd);
            if (t == 0) {
                s_piv[k] = p;
                if (dd == 0.0) atomicExch(P.fault, 1);
            }
            if (col && nq > 0) {
                const double2 prow = prow_all[j];
                const double2 pr = j == k ? ip : cmul(prow, ip);   // the scaled pivot row
                const bool swap = p != k && p >= r1 && p < r1 + nq;   // row p takes the old row k
                const double2 rkj = rowk[j], rkk = rowk[k];
#pragma unroll
                for (int u = 0; u < RS; ++u) {
                    if (u >= nq) break;
                    const int r = r1 + u;
                    if (r == k) {
                        a[u] = pr;
                    } else {
                        // column k of the inverse: -f / pivot (pr = 1 / pivot there)
                        const bool sw = swap && r == p;
                        const double2 f = sw ? rkk : s_colk[par][q0 + u];
                        const double2 cur = j == k ? make_double2(0.0, 0.0) : (sw ? rkj : a[u]);
                        a[u] = csub(cur, cmul(f, pr));
                    }
                }
            }
        }
        // ---- undo the row exchanges on the columns of the inverse, last first:
        // column j of D_b^{-1} is column perm[j] of what the threads hold
        __syncthreads();
        if (t == 0) {
            for (int q = 0; q < m; ++q) s_perm[q] = q;
            for (int k = m - 1; k >= 0; --k) {
                const int pk = s_piv[k];
                if (pk != k) {
                    const int tmp = s_perm[k];
                    s_perm[k] = s_perm[pk];
                    s_perm[pk] = tmp;
                }
            }
        }
        __syncthreads();
        const int src = col ? s_perm[j] : 0;
#pragma unroll
        for (int u = 0; u < RS; ++u) {
            if (col) s_ex[h][j] = a[u];
            __syncthreads();
            if (col) a[u] = s_ex[h][src];
            __syncthreads();
        }
        if (col) {
            double2* out = P.inv + (size_t)b * m * m;
#pragma unroll
            for (int u = 0; u < RS; ++u) {
                if (u >= nq) break;
                out[(size_t)(r1 + u) * m + j] = a[u];
            }
        }
    }
    cl.sync();   // no CTA leaves while another may still read its shared memory
}

// Blocked form of the same elimination for blocks of up to 256 points:
// pivots chosen and applied kPanel columns at a time.  Every CTA reads the
// panel columns of all rows (each CTA writes its rows' entries to a global
// scratch panel, cluster barrier, every CTA reads it back from L2: the
// fan-out goes through L2, not through one SM's port), runs the panel's
// pivot steps on that copy with block barriers only (pivot rows by partial
// pivoting among the rows not yet used, the lowest row on a tie: every CTA
// decides the same), reads the panel's pivot rows the same way (second
// cluster barrier), and applies the rank-kPanel update
//   pivot rows:  A[K, N] <- P^-1 A[K, N],   others: A[r, N] -= A[r, K0] P^-1 A[K, N]
// to its own rows (P: the panel block of the pivot rows, N: the columns
// outside the panel); the panel columns take the replica's values.  Rows
// are not exchanged: the inverse is the result with its rows taken in pivot
// order and its columns in the inverse order, and is stored to P.inv row by
// row in its true place, then read back for the next block.
constexpr int kPanel = 8;
constexpr int kPanelMaxM = 256;

inline size_t fd_panel_smem(int m) {   // s_pan[m][W], s_pn[m][W], s_rk[W][m], s_u[W][m], s_rows[2][m][W]
    return (size_t)6 * m * kPanel * sizeof(double2);
}

template <int RS, int TPC, int NT>
__global__ void __launch_bounds__(NT, 1) k_fdfd_factor_panel(FdfdDev P) {
    cg::cluster_group cl = cg::this_cluster();
    const int C = (int)cl.num_blocks();
    const int c = (int)cl.block_rank();
    const int m = P.m;
    const int mp = (m + 31) / 32 * 32;
    const int R = (m + C - 1) / C;
    const int r0 = c * R;
    const int nr = max(0, min(m, r0 + R) - r0);
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int nt = (int)blockDim.x, nwarps = nt / 32;   // TPC x mp threads (at most NT)
    const int j = t % mp, h = t / mp;
    const int q0 = h * RS;
    const int r1 = r0 + q0;
    const int nq = max(0, min(RS, nr - q0));
    const bool col = j < m;
    constexpr int W = kPanel;

    extern __shared__ double2 s_dyn[];
    double2* s_pan = s_dyn;                          // [m][W]: the panel, every row (old values)
    double2* s_pn = s_pan + (size_t)m * W;           // [m][W]: the panel after its pivot steps
    double2* s_rk = s_pn + (size_t)m * W;            // [W][m]: the panel's pivot rows (old values)
    double2* s_u = s_rk + (size_t)W * m;             // [W][m]: P^-1 times them
    double2* s_rows = s_u + (size_t)W * m;           // [2][m][W]: the copy's rows, per pivot step
    __shared__ FdCand s_wc[2][NT / 32];              // per warp candidates, per pivot step
    __shared__ int s_K[W];                           // pivot rows of the panel
    __shared__ signed char s_kidx[kPanelMaxM];       // index of a row in s_K, or -1
    __shared__ int s_piv[kPanelMaxM];
    __shared__ int s_ipiv[kPanelMaxM];

    double2 a[RS];
#pragma unroll
    for (int u = 0; u < RS; ++u) a[u] = make_double2(0.0, 0.0);

    for (int b = 0; b < P.nb; ++b) {
        // ---- D_b: the tridiagonal block minus B_b D_{b-1}^{-1} C_{b-1}
        if (col) {
            const double2 cpj = b > 0 ? P.bp[(size_t)(b - 1) * m + j] : make_double2(0.0, 0.0);
#pragma unroll
            for (int u = 0; u < RS; ++u) {
                if (u >= nq) break;
                const int p = r1 + u;
                const size_t o = (size_t)b * m + p;
                double2 v = make_double2(0.0, 0.0);
                if (b > 0) {
                    const double2 s = cmul(cmul(P.bm[o], a[u]), cpj);
                    v = make_double2(-s.x, -s.y);
                }
                if (j == p) v = cadd(v, P.diag[o]);
                else if (j == p - 1) v = cadd(v, P.wm[o]);
                else if (j == p + 1) v = cadd(v, P.wp[o]);
                a[u] = v;
            }
        }
        bool myused = false;   // row t (thread t < m) is the pivot row of an earlier column
        for (int k0 = 0; k0 < m; k0 += W) {
            const int we = min(W, m - k0);
            double2* pan = s_pan;
            // ---- the panel entries of the own rows to the scratch panel; every
            // CTA reads the whole panel back (L2, bypassing L1: the scratch is
            // rewritten every panel).  The scratch is written again only after
            // the next cluster barrier, which every reader reaches after its read.
            if (col && j >= k0 && j < k0 + we) {
#pragma unroll
                for (int u = 0; u < RS; ++u)
                    if (u < nq) P.xpan[(size_t)(r1 + u) * W + (j - k0)] = a[u];
            }
            __threadfence();
            cl.sync();   // the whole panel is in memory
            // ---- the panel's pivot steps on the copy: thread r holds row r
            double2 pr[W];
            if (t < m) {
#pragma unroll
                for (int l = 0; l < W; ++l) {
                    pr[l] = l < we ? __ldcg(P.xpan + (size_t)t * W + l) : make_double2(0.0, 0.0);
                    pan[(size_t)t * W + l] = pr[l];
                }
            }
            // one block barrier per pivot step: every row thread publishes its
            // row and every warp its candidate (buffers alternate by step), then
            // every warp reduces the candidates itself and reads the pivot row
            // (unrolled: a row's entries are registers indexed by the step)
#pragma unroll
            for (int aa = 0; aa < W; ++aa) {
                if (aa >= we) break;
                const int sp2 = aa & 1;
                double2* rows = s_rows + (size_t)sp2 * m * W;
                double best = -1.0;
                int bi = m;
                if (t < m) {
#pragma unroll
                    for (int l = 0; l < W; ++l) rows[(size_t)t * W + l] = pr[l];
                    if (!myused) {
                        best = cabs2(pr[aa]);
                        bi = t;
                    }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                    if (ob > best || (ob == best && oi < bi)) {
                        best = ob;
                        bi = oi;
                    }
                }
                if (lane == 0) s_wc[sp2][warp] = FdCand{best, bi, 0};
                __syncthreads();
                best = -1.0;
                bi = m;
                if (lane < nwarps) {
                    const FdCand cd = s_wc[sp2][lane];
                    best = cd.v;
                    bi = cd.i;
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                    if (ob > best || (ob == best && oi < bi)) {
                        best = ob;
                        bi = oi;
                    }
                }
                const bool bad = bi >= m || best == 0.0;
                const int p = bi >= m ? 0 : bi;
                if (t == 0) {
                    if (bad) atomicExch(P.fault, 1);
                    s_piv[k0 + aa] = p;
                    s_K[aa] = p;
                }
                if (t == p) myused = true;
                const double2* prw = rows + (size_t)p * W;
                const double2 pk = prw[aa];
                const double dd = cabs2(pk);
                const double inv_dd = dd == 0.0 ? 0.0 : 1.0 / dd;
                const double2 ip = make_double2(pk.x * inv_dd, -pk.y * inv_dd);
                if (t < m) {
                    const double2 f = pr[aa];
#pragma unroll
                    for (int l = 0; l < W; ++l) {
                        const double2 sp = l == aa ? ip : cmul(prw[l], ip);   // the scaled pivot row
                        if (t == p) pr[l] = sp;
                        else pr[l] = csub(l == aa ? make_double2(0.0, 0.0) : pr[l], cmul(f, sp));
                    }
                }
            }
            __syncthreads();   // s_K, s_piv
            if (t < m) {
#pragma unroll
                for (int l = 0; l < W; ++l) s_pn[(size_t)t * W + l] = pr[l];
                s_kidx[t] = -1;
            }
            __syncthreads();
            if (t < we) s_kidx[s_K[t]] = (signed char)t;
            // ---- the panel's pivot rows (old values, every column) through the
            // scratch rows, read back by every CTA
            if (col) {
#pragma unroll
                for (int u = 0; u < RS; ++u) {
                    if (u >= nq) break;
                    const int r = r1 + u;
                    for (int i = 0; i < we; ++i)
                        if (s_K[i] == r) P.xrow[(size_t)i * m + j] = a[u];
                }
            }
            __threadfence();
            cl.sync();   // the pivot rows are in memory
            for (int e = t; e < we * m; e += nt) s_rk[e] = __ldcg(P.xrow + e);
            __syncthreads();
            // ---- U = P^-1 (pivot rows): row i of U by the threads of group i % TPC
            if (col) {
                for (int i = h; i < we; i += TPC) {
                    double2 acc = make_double2(0.0, 0.0);
                    const double2* pinv = s_pn + (size_t)s_K[i] * W;
                    for (int l = 0; l < we; ++l) acc = cadd(acc, cmul(pinv[l], s_rk[(size_t)l * m + j]));
                    s_u[(size_t)i * m + j] = acc;
                }
            }
            __syncthreads();
            // ---- the rank-we update of the own rows
            if (col) {
                const bool inpan = j >= k0 && j < k0 + we;
#pragma unroll
                for (int u = 0; u < RS; ++u) {
                    if (u >= nq) break;
                    const int r = r1 + u;
                    if (inpan) {
                        a[u] = s_pn[(size_t)r * W + (j - k0)];
                    } else if (s_kidx[r] >= 0) {
                        a[u] = s_u[(size_t)s_kidx[r] * m + j];
                    } else {
                        double2 v = a[u];
                        for (int l = 0; l < we; ++l) v = csub(v, cmul(pan[(size_t)r * W + l], s_u[(size_t)l * m + j]));
                        a[u] = v;
                    }
                }
            }
            __syncthreads();   // s_kidx, s_u and s_pn are rewritten by the next panel
        }
        // ---- the inverse: row ipiv[r] is row r of what the threads hold,
        // with column j taken from column ipiv[j]
        if (t < m) s_ipiv[s_piv[t]] = t;
        __syncthreads();
        double2* s_ex = s_u;   // [TPC][m] (TPC <= kPanel)
        const int src = col ? s_ipiv[j] : 0;
#pragma unroll
        for (int u = 0; u < RS; ++u) {
            if (col) s_ex[(size_t)h * m + j] = a[u];
            __syncthreads();
            if (col) a[u] = s_ex[(size_t)h * m + src];
            __syncthreads();
        }
        double2* out = P.inv + (size_t)b * m * m;
        if (col) {
#pragma unroll
            for (int u = 0; u < RS; ++u)
                if (u < nq) out[(size_t)s_ipiv[r1 + u] * m + j] = a[u];
        }
        __threadfence();
        cl.sync();   // every CTA's rows of the inverse are in memory
        if (col) {
#pragma unroll
            for (int u = 0; u < RS; ++u)
                if (u < nq) a[u] = out[(size_t)(r1 + u) * m + j];
        }
        __syncthreads();
    }
    cl.sync();   // no CTA leaves while another may still read its shared memory
}

// Forward and backward sweeps with the stored inverses.
//   mode 0: A x = -rhs:   w_b = -rhs_b - B_b y_{b-1},  y_b = D_b^{-1} w_b,
//                         x_b = y_b - D_b^{-1} C_b x_{b+1}
//   mode 1: A.' x = rhs:  z_b = D_b^{-T} (rhs_b - C_{b-1} z_{b-1}),
//                         x_{b-1} = z_{b-1} - D_{b-1}^{-T} B_b x_b
// Vector entries are owned by the CTA that owns the row of the same index;
// the products gather the whole vector (mode 0) or reduce partial sums over
// the owned rows (mode 1) through distributed shared memory, one cluster
// barrier per line.
__global__ void __launch_bounds__(kSolveThreads, 1) k_fdfd_solve(FdfdDev P, const double2* rhs, double2* x,
                                                                  double2* Y, int mode) {
    cg::cluster_group cl = cg::this_cluster();
    const int C = (int)cl.num_blocks();
    const int c = (int)cl.block_rank();
    const int m = P.m, nb = P.nb;
    const int R = (m + C - 1) / C;
    const int r0 = c * R;
    const int nr = max(0, min(m, r0 + R) - r0);
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    constexpr int NW = kSolveThreads / 32;
    __shared__ double2 s_pub[2][kFdMaxM];   // published own entries (mode 0) / partial sums (mode 1)
    __shared__ double2 s_full[kFdMaxM];     // mode 0: the gathered vector
    __shared__ double2 s_u[kFdMaxM];        // mode 1: the owned entries of the multiplied vector
    long long g = 0;
    auto warp_sum = [&](double2 v) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
            v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
        }
        return v;
    };
    if (mode == 0) {
        // dst_b = D_b^{-1} s_full on the owned rows (base_b minus it when base is given)
        auto gemv_rows = [&](int b, const double2* base, double2* dst) {
            const double2* Ib = P.inv + (size_t)b * m * m;
            for (int q = warp; q < nr; q += NW) {
                const int p = r0 + q;
                const double2* row = Ib + (size_t)p * m;
                double2 acc = make_double2(0.0, 0.0);
                for (int jj = lane; jj < m; jj += 32) acc = cadd(acc, cmul(row[jj], s_full[jj]));
                acc = warp_sum(acc);
                if (lane == 0) dst[(size_t)b * m + p] = base ? csub(base[(size_t)b * m + p], acc) : acc;
            }
        };
        for (int b = 0; b < nb; ++b, ++g) {
            const int par = (int)(g & 1);
            for (int q = t; q < nr; q += kSolveThreads) {
                const int p = r0 + q;
                const size_t o = (size_t)b * m + p;
                double2 w = make_double2(-rhs[o].x, -rhs[o].y);
                if (b > 0) w = csub(w, cmul(P.bm[o], Y[o - m]));
                s_pub[par][p] = w;
            }
            cl.sync();
            for (int jj = t; jj < m; jj += kSolveThreads) s_full[jj] = cl.map_shared_rank(&s_pub[par][0], jj / R)[jj];
            __syncthreads();
            gemv_rows(b, nullptr, Y);
            __syncthreads();
        }
        for (int q = t; q < nr; q += kSolveThreads) {
            const size_t o = (size_t)(nb - 1) * m + r0 + q;
            x[o] = Y[o];
        }
        __syncthreads();
        for (int b = nb - 2; b >= 0; --b, ++g) {
            const int par = (int)(g & 1);
            for (int q = t; q < nr; q += kSolveThreads) {
                const int p = r0 + q;
                const size_t o = (size_t)b * m + p;
                s_pub[par][p] = cmul(P.bp[o], x[o + m]);
            }
            cl.sync();
            for (int jj = t; jj < m; jj += kSolveThreads) s_full[jj] = cl.map_shared_rank(&s_pub[par][0], jj / R)[jj];
            __syncthreads();
            gemv_rows(b, Y, x);
            __syncthreads();
        }
    } else {
        // partial sums of D_b^{-T} u over the owned rows, for every column
        auto partial = [&](int b, int par) {
            const double2* Ib = P.inv + (size_t)b * m * m;
            for (int jj = t; jj < m; jj += kSolveThreads) {
                double2 acc = make_double2(0.0, 0.0);
                for (int q = 0; q < nr; ++q) acc = cadd(acc, cmul(Ib[(size_t)(r0 + q) * m + jj], s_u[q]));
                s_pub[par][jj] = acc;
            }
        };
        auto reduce_own = [&](int par, int q) {
            double2 s = make_double2(0.0, 0.0);
            for (int c2 = 0; c2 < C; ++c2) s = cadd(s, cl.map_shared_rank(&s_pub[par][0], c2)[r0 + q]);
            return s;
        };
        for (int b = 0; b < nb; ++b, ++g) {
            const int par = (int)(g & 1);
            for (int q = t; q < nr; q += kSolveThreads) {
                const size_t o = (size_t)b * m + r0 + q;
                double2 u = rhs[o];
                if (b > 0) u = csub(u, cmul(P.bp[o - m], Y[o - m]));
                s_u[q] = u;
            }
            __syncthreads();
            partial(b, par);
            cl.sync();
            for (int q = t; q < nr; q += kSolveThreads) Y[(size_t)b * m + r0 + q] = reduce_own(par, q);
            __syncthreads();
        }
        for (int q = t; q < nr; q += kSolveThreads) {
            const size_t o = (size_t)(nb - 1) * m + r0 + q;
            x[o] = Y[o];
        }
        __syncthreads();
        for (int b = nb - 1; b >= 1; --b, ++g) {
            const int par = (int)(g & 1);
            for (int q = t; q < nr; q += kSolveThreads) {
                const size_t o = (size_t)b * m + r0 + q;
                s_u[q] = cmul(P.bm[o], x[o]);
            }
            __syncthreads();
            partial(b - 1, par);
            cl.sync();
            for (int q = t; q < nr; q += kSolveThreads) {
                const size_t o = (size_t)(b - 1) * m + r0 + q;
                x[o] = csub(Y[o], reduce_own(par, q));
            }
            __syncthreads();
        }
    }
    cl.sync();   // no CTA leaves while another may still read its shared memory
}

// Factor kernel shape for block size m: CTAs of the cluster, rows per CTA
// at most (RM), thread groups per column (TPC); threads TPC x m rounded up
// to a warp.  m <= 128: 8 CTAs, 4 groups of 4 rows; m <= 256: 16 CTAs, 4
// groups of 4 rows; m <= 384: 16 CTAs, one group of 24 rows.
int fd_shape(int m, int* C, int* RM) {
    static const int kC[3] = {8, 16, 16}, kR[3] = {16, 16, 24};
    for (int q = 0; q < 3; ++q)
        if (kC[q] * kR[q] >= m) {
            *C = kC[q];
            *RM = kR[q];
            return ORF_OK;
        }
    set_error("fdfd2D: the shorter grid axis has %d points, above the %d this solver takes", m, kFdMaxM);
    return ORF_ETOOLARGE;
}

template <class K, class... Args>
cudaError_t launch_cluster(K kern, int C, int threads, size_t smem, cudaStream_t s, Args... args) {
    if (C > 8) {
        const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)C, 1, 1);
    cfg.blockDim = dim3((unsigned)threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

using cplx = std::complex<double>;

// s at the integer points (half = false) or at the half points u = -1/2 ..
// n-1/2 (half = true) of one axis: s = 1 + i a (depth / L)^3 inside the
// npml-cell layers, depth = npml - u below the low edge, u - (n-1-npml)
// above the high edge (the FDTD's CPML convention), a = 2 ln(1/R) / (k0 L)
std::vector<cplx> fd_stretch(int n, int npml, double d, double k0, double R, bool half) {
    const int npts = half ? n + 1 : n;
    std::vector<cplx> s(npts, cplx(1.0, 0.0));
    if (npml <= 0) return s;
    const double L = npml * d;
    const double a = 2.0 * std::log(1.0 / R) / (k0 * L);
    const double lo = npml, hi = (n - 1) - npml;
    for (int q = 0; q < npts; ++q) {
        const double u = half ? q - 0.5 : (double)q;
        double depth = 0.0;
        if (u < lo) depth = lo - u;
        else if (u > hi) depth = u - hi;
        const double r = depth * d / L;
        s[q] = cplx(1.0, a * r * r * r);
    }
    return s;
}

}  // namespace
}  // namespace orf

using namespace orf;

struct orf_fdfd {
    orf_ctx* ctx = nullptr;
    int nx = 0, nz = 0, m = 0, nb = 0, C = 8, RM = 16;
    bool along_x = true;   // blocks are lines of constant x (m = nz)
    Arena ar;
    double2 *diag = nullptr, *wm = nullptr, *wp = nullptr, *bm = nullptr, *bp = nullptr;
    double2 *inv = nullptr, *Y = nullptr, *vin = nullptr, *vout = nullptr, *xpan = nullptr, *xrow = nullptr;
    int* fault = nullptr;
    ~orf_fdfd() {
        if (ar.base) {
            cudaStreamSynchronize(ctx->stream);
            ar.release();
        }
        if (ctx) ctx_release(ctx);
    }
    FdfdDev dev() const { return FdfdDev{m, nb, diag, wm, wp, bm, bp, inv, fault, xpan, xrow}; }
    // (i, k) of the grid <-> entry b * m + p of the block layout
    size_t at(int i, int k) const { return along_x ? (size_t)i * m + k : (size_t)k * m + i; }
};

extern "C" int32_t orf_fdfd2d_factor(orf_ctx* ctx, const orf_fdfd2d* pr, orf_fdfd** out) {
    if (!out) {
        set_error("out is null");
        return ORF_EINVAL;
    }
    *out = nullptr;
    if (!ctx || !pr || !pr->eps) {
        set_error("ctx, problem and eps are required");
        return ORF_EINVAL;
    }
    const int nx = pr->nx, nz = pr->nz;
    if (nx < 3 || nz < 3 || !(pr->dx > 0) || !(pr->lambda0 > 0)) {
        set_error("fdfd2D: needs at least 3 x 3 points, dx > 0 and lambda0 > 0");
        return ORF_EINVAL;
    }
    if (pr->npml_x < 0 || pr->npml_z < 0 || 2 * pr->npml_x >= nx || 2 * pr->npml_z >= nz) {
        set_error("fdfd2D: Npml must leave interior points on both axes");
        return ORF_EINVAL;
    }
    if (!(pr->pml_reflection > 0 && pr->pml_reflection < 1)) {
        set_error("fdfd2D: PmlReflection must lie in (0, 1)");
        return ORF_EINVAL;
    }
    ORF_ON_DEVICE(ctx->device);
    auto F = std::make_unique<orf_fdfd>();
    F->nx = nx;
    F->nz = nz;
    F->along_x = nz <= nx;
    F->m = F->along_x ? nz : nx;
    F->nb = F->along_x ? nx : nz;
    ORF_TRY(fd_shape(F->m, &F->C, &F->RM));
    const int m = F->m, nb = F->nb;
    const size_t N = (size_t)nx * nz;

    // ---- operator coefficients, rows scaled as in A E = -J
    const double d = pr->dx, k0 = 2.0 * kPi / pr->lambda0, R = pr->pml_reflection;
    const auto sxi = fd_stretch(nx, pr->npml_x, d, k0, R, false), sxh = fd_stretch(nx, pr->npml_x, d, k0, R, true);
    const auto szi = fd_stretch(nz, pr->npml_z, d, k0, R, false), szh = fd_stretch(nz, pr->npml_z, d, k0, R, true);
    std::vector<double2> hd(N), hwm(N), hwp(N), hbm(N), hbp(N);
    const double h2 = 1.0 / (d * d);
    auto d2 = [](cplx v) { return make_double2(v.real(), v.imag()); };
    for (int k = 0; k < nz; ++k)
        for (int i = 0; i < nx; ++i) {
            const cplx cxm = h2 / (sxi[i] * sxh[i]), cxp = h2 / (sxi[i] * sxh[i + 1]);
            const cplx czm = h2 / (szi[k] * szh[k]), czp = h2 / (szi[k] * szh[k + 1]);
            const size_t g = (size_t)i + (size_t)nx * k;
            const cplx eps(pr->eps[2 * g], pr->eps[2 * g + 1]);
            const cplx dg = -(cxm + cxp + czm + czp) + k0 * k0 * eps;
            const size_t o = F->at(i, k);
            hd[o] = d2(dg);
            hwm[o] = d2(F->along_x ? czm : cxm);
            hwp[o] = d2(F->along_x ? czp : cxp);
            hbm[o] = d2(F->along_x ? cxm : czm);
            hbp[o] = d2(F->along_x ? cxp : czp);
        }

    F->ctx = ctx;
    ctx_retain(ctx);
    Arena& ar = F->ar;
    ar.add(&F->diag, N);
    ar.add(&F->wm, N);
    ar.add(&F->wp, N);
    ar.add(&F->bm, N);
    ar.add(&F->bp, N);
    ar.add(&F->inv, (size_t)nb * m * m);
    ar.add(&F->Y, N);
    ar.add(&F->vin, N);
    ar.add(&F->vout, N);
    ar.add(&F->fault, 1);
    ar.add(&F->xpan, (size_t)m * 8);
    ar.add(&F->xrow, (size_t)8 * m);
    ORF_TRY(ar.alloc());
    cudaStream_t st = ctx->stream;
    ORF_CUDA(cudaMemcpyAsync(F->diag, hd.data(), N * sizeof(double2), cudaMemcpyHostToDevice, st));
    ORF_CUDA(cudaMemcpyAsync(F->wm, hwm.data(), N * sizeof(double2), cudaMemcpyHostToDevice, st));
    ORF_CUDA(cudaMemcpyAsync(F->wp, hwp.data(), N * sizeof(double2), cudaMemcpyHostToDevice, st));
    ORF_CUDA(cudaMemcpyAsync(F->bm, hbm.data(), N * sizeof(double2), cudaMemcpyHostToDevice, st));
    ORF_CUDA(cudaMemcpyAsync(F->bp, hbp.data(), N * sizeof(double2), cudaMemcpyHostToDevice, st));
    ORF_CUDA(cudaMemsetAsync(F->fault, 0, sizeof(int), st));
    add_h2d(ctx, (int64_t)(5 * N * sizeof(double2)));
    const int mp = (m + 31) / 32 * 32;
    const FdfdDev P = F->dev();
    cudaError_t e;
    const size_t fsm = 0;
    const size_t psm = fd_panel_smem(m);
    if (F->RM == 16 && mp <= 128) e = launch_cluster(k_fdfd_factor_panel<4, 4, 512>, F->C, 4 * mp, psm, st, P);
    else if (F->RM == 16) e = launch_cluster(k_fdfd_factor_panel<8, 2, 512>, F->C, 2 * mp, psm, st, P);
    else e = launch_cluster(k_fdfd_factor<24, 1, 384>, F->C, mp, fsm, st, P);
    ORF_CUDA(e);
    int fault = 0;
    ORF_CUDA(cudaMemcpyAsync(&fault, F->fault, sizeof(int), cudaMemcpyDeviceToHost, st));
    ORF_CUDA(cudaStreamSynchronize(st));
    if (fault) {
        set_error("fdfd2D: the operator is singular (a zero pivot in the block elimination)");
        return ORF_EINVAL;
    }
    *out = F.release();
    return ORF_OK;
}

extern "C" int32_t orf_fdfd2d_solve(orf_fdfd* F, const double* rhs, double* x, int32_t transpose) {
    if (!F || !rhs || !x) {
        set_error("fdfd handle, rhs and x are required");
        return ORF_EINVAL;
    }
    ORF_ON_DEVICE(F->ctx->device);
    const size_t N = (size_t)F->nx * F->nz;
    std::vector<double2> h(N);
    for (int k = 0; k < F->nz; ++k)
        for (int i = 0; i < F->nx; ++i) {
            const size_t g = (size_t)i + (size_t)F->nx * k;
            h[F->at(i, k)] = make_double2(rhs[2 * g], rhs[2 * g + 1]);
        }
    cudaStream_t st = F->ctx->stream;
    ORF_CUDA(cudaMemcpyAsync(F->vin, h.data(), N * sizeof(double2), cudaMemcpyHostToDevice, st));
    add_h2d(F->ctx, (int64_t)(N * sizeof(double2)));
    ORF_CUDA(launch_cluster(k_fdfd_solve, F->C, kSolveThreads, 0, st, F->dev(), (const double2*)F->vin, F->vout, F->Y,
                            transpose ? 1 : 0));
    ORF_CUDA(cudaMemcpyAsync(h.data(), F->vout, N * sizeof(double2), cudaMemcpyDeviceToHost, st));
    ORF_CUDA(cudaStreamSynchronize(st));
    add_d2h(F->ctx, (int64_t)(N * sizeof(double2)));
    for (int k = 0; k < F->nz; ++k)
        for (int i = 0; i < F->nx; ++i) {
            const size_t g = (size_t)i + (size_t)F->nx * k;
            const double2 v = h[F->at(i, k)];
            x[2 * g] = v.x;
            x[2 * g + 1] = v.y;
        }
    return ORF_OK;
}

extern "C" void orf_fdfd2d_release(orf_fdfd* F) {
    if (!F) return;
    DeviceScope ds(F->ctx->device);
    delete F;
}

extern "C" int32_t orf_fdfd2d_info(const orf_fdfd* F, int32_t* block, int32_t* nblocks, int32_t* cluster) {
    if (!F) {
        set_error("fdfd handle is null");
        return ORF_EINVAL;
    }
    if (block) *block = F->m;
    if (nblocks) *nblocks = F->nb;
    if (cluster) *cluster = F->C;
    return ORF_OK;
}
