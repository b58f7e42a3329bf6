// orf_internal.cuh -- device-side data model of the B200 Yee-FDTD engine.
//
// One "instance" is one orf.fdtd2D / orf.fdtd3D run.  Instances live in a
// device table; the step kernels walk a list of tiles (instance, output
// rectangle) so that a single run, a batch of hundreds of runs and the
// serving loop all use the same kernels.  Every instance advances in
// "chunks" of kChunk steps: the step kernels (each fusing up to T time steps
// of the H and E updates, CPML, TF/SF source and DFT sampling), then one DFT
// flush kernel and one energy/shutoff check kernel.  Chunk boundaries are
// where the reference calls its progress callback (fdtd2D.m:18-20).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace orf {

constexpr int kChunk = 50;        // steps between energy checks and progress calls
constexpr int kMaxMon = 16;       // monitors per orientation per instance
constexpr int kMaxSub = 32;       // max time steps fused in one step-kernel launch
// The CPML grading uses kappa_max = 1, so 1/kappa is 1 at every position and
// the stretched difference d/kappa + psi is d + psi: the step kernels skip the
// 1/kappa factor (fma(d, 1, psi) and d + psi round alike).
constexpr bool kUnitKappa = true;
constexpr int kStatusRing = 64;   // status ring entries per job (mapped host memory)

// Written by the check kernel into mapped pinned host memory.
struct ChunkStatus {
    long long seq;          // chunk number + 1 (written last)
    long long step;         // steps completed
    double energy;
    double peak;
    int done;
    int converged;
};

// Device-resident run state of one instance.
struct JobState {
    long long step;         // steps completed
    long long nmax;         // step budget from maxTime
    long long chunk;        // chunks completed
    int done;               // no more steps (shutoff, budget or cancel)
    int converged;          // stopped by the energy shutoff
    int cur;                // field buffer (0/1) holding the latest state
    int fault;              // a bounded device-side wait ran out (ORF_ETIMEOUT_DEVICE)
    double energy;          // energy accumulator of the current chunk
    double peak;
    double S;               // c0*dt [um]
    double src_end;         // end of the source pulse (c0*t)
    double shutoff;
    ChunkStatus* ring;      // mapped host ring, kStatusRing entries (may be null)
    const volatile int* cancel;   // mapped host flag: non-zero stops the run at the next check
};

// One DFT stream: a monitor line (or plane) of one field, sampled every step
// into the chunk's sample buffer and folded into running DFT sums by the
// flush kernel.  Kernel e^{+i w t} (fdtd2DTE.m:18).
struct DftStream {
    JobState* st;
    const void* samples;    // sample buffer of the instance (Real)
    int sstride;            // elements per step in that buffer
    int soff;               // offset of this stream inside one step's samples
    int len;                // elements
    int half;               // 1: field lives at t_{n+1/2}, 0: at t_{n+1}
    int nl;                 // wavelengths
    int pad;
    const double* omega;    // 2*pi/lambda, nl values
    void* acc;              // FP64: double2[nl][len]; FP32: float4[nl][len] (sum re, im; Kahan c re, im)
};

struct FlushItem {          // one block of the flush kernel
    int stream;
    int e0;                 // first element
    int l0;                 // first wavelength
    int pad;
};

// --------------------------------------------------------------------- 2D --
// P/A/B fields (fdtd2D.m:3-7): TE P=Ey A=Hx B=Hz, TM P=Hy A=-Ex B=-Ez.
// Device layout: every field is [nz][pitch] with x fastest, pitch a multiple
// of 32 elements; A's row nz-1 (non-periodic) and B's column nx-1 do not
// exist in the reference and stay zero here.
template <class R>
struct Inst2D {
    int nx, nz, pitch, nzA, nxB;
    int periodic, te;
    int npx, npz;           // CPML cells per end (npz = 0 when periodic)
    int idx16;              // material index width: 0 = uint8, 1 = uint16
    int nlut;               // distinct materials (entries of lutc / lute in use)
    R C;                    // courant number c0*dt/dx
    R* P[2];
    R* A[2];
    R* B[2];
    const void* idx0;       // TE: material index at P; TM: at A
    const void* idx1;       // TM: material index at B
    const R* lutc;          // C / eps per material index
    const double* lute;     // eps per material index (energy)
    // CPML profiles, (b, a, 1/kappa) interleaved: columns at P (x_i) and at
    // B (x_i+1/2), rows at P (z_k) and at A (z_k+1/2)
    const R* pmlx;
    const R* pmlxh;
    const R* pmlz;
    const R* pmlzh;
    // psi in compact slabs, ping-pong: x slabs [nz][2*npx], z slabs [2*npz][nx]
    R* psiB[2];
    R* psiPx[2];
    R* psiA[2];
    R* psiPz[2];
    // TF/SF plane at P column src_ix: B column src_ix-1 gets srcB[k]*gE[n],
    // P column src_ix gets srcP[k]*gH[n]
    int src_ix;
    int nmon, nmonz;
    int sstride;            // samples per step: 2*nz*nmon + 2*nx*nmonz
    const R* srcB;
    const R* srcP;
    const double* gE;
    const double* gH;
    long long nsrc;         // table length (pulse is zero beyond)
    int mon[kMaxMon];
    int monz[kMaxMon];
    R* samples;             // [kChunk][sstride]
    JobState* st;
};

// Self-contained descriptor of a tile for the pipelined kernel
// (step2d_fast.cuh): everything its prefetch needs, 128 bytes, copied into
// shared memory with cp.async two tiles ahead.
struct alignas(16) FastTile2D {
    const void* f[2][3];    // P, A, B of buffer 0 and 1
    const void* idx0;
    const void* idx1;
    JobState* st;
    const void* inst;       // Inst2D<R>* (source, monitors, tables, CPML state)
    int pitch, nz, periodic;
    int li0, lk0;           // loaded origin; li0 is a multiple of 4 cells (may be negative)
    int oi0, ok0, ow, oh;   // output rectangle
    int flags;              // 1: TF/SF plane in the loaded columns, 2: x monitor, 4: z monitor,
                            // 8 / 16: (frame tiles) the loaded cells reach an x / z CPML slab
    int nx;
    int pad;
};
static_assert(sizeof(FastTile2D) == 128, "FastTile2D must stay 128 bytes");

// --------------------------------------------------------------------- 3D --
// Six components at their Yee positions (fdtd3D.m:2-5); every array is
// [nz][ny][pitch] with x fastest.  Component c of E/H: 0 = x, 1 = y, 2 = z.
template <class R>
struct Inst3D {
    int n[3];
    int pitch;
    int per[3];
    int np[3];              // CPML cells per end per axis (0 on periodic axes)
    int idxw;               // material index width in bytes: 1, 2 or 4
    R C;                    // courant number
    R* E[2][3];             // ping-pong
    R* H[2][3];
    const void* idx[3];     // material index of Ex, Ey, Ez
    const R* lutc;          // C / eps per material index
    const double* lute;     // eps per material index
    // CPML per axis q: (b, a, 1/kappa) at integer (E-derivative) and half
    // (H-derivative) positions, n[q] entries each; slab index per coordinate
    // (-1 outside the absorbing layer)
    const R* pmlI[3];
    const R* pmlH[3];
    const int* slabI[3];
    const int* slabH[3];
    int nslabI[3], nslabH[3];
    // psi of (component c, derivative axis q != c), compact along q, ping-pong
    R* psiE[2][3][3];
    R* psiH[2][3][3];
    // TF/SF plane normal to axis sa at index ss (a = sa+1, b = sa+2 cyclic):
    // H_a[ss-1] += sHa*gE, H_b[ss-1] += sHb*gE, E_a[ss] += sEa*gH, E_b[ss] += sEb*gH
    int sa, ss, na, nb;
    const R* sHa;           // -C * Eb profile
    const R* sHb;           // +C * Ea profile
    const R* sEa;           // +(C/eps_a) * Hb profile
    const R* sEb;           // -(C/eps_b) * Ha profile
    const double* gE;
    const double* gH;
    long long nsrc;
    int nmon;
    int sstride;            // samples per step
    int mon_axis[kMaxMon];
    int mon_index[kMaxMon];
    int mon_off[kMaxMon];   // offset of the monitor's Ea, Eb, Ha, Hb planes in one step's samples
    R* samples;
    JobState* st;
    // TMA tensor maps (CUtensorMap, 128 B each) in device memory, or null:
    // [0..5] E[b][c] boxes 40 x 10 x 1, [6..11] H[b][c] boxes 40 x 9 x 1,
    // [12..14] index[c] boxes 32 x 8 x 1 (b = buffer, c = component);
    // when tma_psi: [15..18] psiH[b][c][2], [19..22] psiE[b][c][2] (c = 0, 1),
    // boxes 40 x 10 x 1 over nx x ny x slab planes
    const void* tmap;
    int tma_psi;
};

struct Tile3D {
    int inst;
    int i0, j0;             // column origin in x, y
    short tw, th;           // extent in x, y (<= kTile3X x kTile3Y)
    int k0, k1;             // z planes [k0, k1) marched by the CTA
};

// ------------------------------------------------------------- launchers --
// Implemented in step2d.cu / step3d.cu / dft.cu.
struct Variant2D {
    int id;
    int ks, wx, wz;         // strip length, warps along x, warps along z
    int lx() const { return 32 * wx; }
    int lz() const { return ks * wz; }
};
int variant2d_count();

// Pipelined kernel (step2d_fast.cuh).  pml = false: interior tiles (no CPML
// or boundary cell in reach); pml = true: CPML / boundary tiles.
bool fast2d_info(int id, bool fp64, bool pml, Variant2D* v);
cudaError_t launch_fast2d(bool fp64, bool te, bool idx16, bool pml, int variant, const FastTile2D* tiles, int ntiles,
                          int launch_off, int nsub, int par, int want_energy, int grid, cudaStream_t s);
int fast2d_blocks_per_sm(bool fp64, bool te, bool idx16, bool pml, int variant);
int fast2d_violations_f32(unsigned long long* n, int reset);
int fast2d_violations_f64(unsigned long long* n, int reset);

constexpr int kTile3X = 32, kTile3Y = 8;   // 3D CTA tile (x, y)
constexpr int kSeg3 = 60;                  // z planes marched by one 3D CTA
// One 3D time step (step3d_fused.cu): reads fields and psi of buffer par,
// writes buffer par^1.  pml = false only for tiles with no cell (halo and
// the plane below the segment included) near a CPML slab.
// Bounds of the 3D kernel's plane waits: wait_ns per plane (0: one second);
// stall_plane >= 0 is the failure-detection test hook (the plane k0 +
// stall_plane of every TMA tile is armed but never loaded, so its wait runs
// out), -1 in every production launch.
struct WaitCtl {
    unsigned long long wait_ns;
    int stall_plane;
};
cudaError_t launch_step3d(bool fp64, bool pml, int idxw, const void* insts, const Tile3D* tiles, int ntiles, int par,
                          int launch_off, int want_energy, WaitCtl wc, cudaStream_t s);

cudaError_t launch_flush(bool fp64, const DftStream* streams, const FlushItem* items, int nitems,
                         cudaStream_t s);
cudaError_t launch_check(JobState* const* states, int n, cudaStream_t s);
// flux[out + ostride*l] = scale * sum_e (Re(a1 conj(b1)) - Re(a2 conj(b2)))
struct FluxPair {
    int a1, b1, a2, b2;     // stream indices; a2 < 0: no second product
    int out, ostride;
    double scale;
};
cudaError_t launch_flux(bool fp64, const DftStream* streams, const FluxPair* pairs, int npairs, int nl,
                        double* out, cudaStream_t s);
cudaError_t launch_acc_to_complex(bool fp64, const void* acc, size_t n, double2* out, cudaStream_t s);

}  // namespace orf
