/*
 * orf_fdtd.h -- C ABI of the B200 Yee-FDTD engine (liborf_fdtd.so).
 *
 * Drop-in for the time loop behind OpticRCWAFDTD's orf.fdtd2D / orf.fdtd2DTE /
 * orf.fdtd3D.  Every struct is plain data: pointers, sizes, doubles.  A MATLAB
 * MEX gateway (mex/orf_fdtd_mex.c), Python ctypes, or any C caller binds the
 * same symbols.
 *
 * Conventions (toolbox/+orf/fdtd2D.m:1-7, fdtd3D.m:1-9, docs/CONVENTIONS.md:17):
 *   - real fields, H~ = eta0*H, time as c0*t in micrometres;
 *   - arrays are column-major with x fastest (MATLAB ndgrid layout);
 *   - every index in these structs is 0-based (the MEX gateway and the Python
 *     mirror subtract 1 from MATLAB's 1-based indices);
 *   - complex outputs are interleaved (re, im) doubles, MATLAB's
 *     interleaved-complex layout (R2018a+).
 *
 * Ownership: input arrays are borrowed for the duration of the call.  Output
 * arrays are allocated by the caller; orf_out2d_sizes / orf_out3d_sizes give
 * their element counts.  Device memory is owned by an orf_ctx.
 */
#ifndef ORF_FDTD_H
#define ORF_FDTD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORF_ABI_VERSION 1

#if defined(_WIN32)
#define ORF_API __declspec(dllexport)
#else
#define ORF_API __attribute__((visibility("default")))
#endif

/* Status codes.  The MEX gateway maps them to MATLAB error identifiers
 * (ORF_ECANCELLED -> 'orf:cancelled', tests/TestGUISupport.m:39-43). */
typedef enum orf_status {
    ORF_OK = 0,
    ORF_EINVAL = 1,            /* malformed sim struct / out-of-range index   */
    ORF_ENOMEM_DEVICE = 2,     /* not enough free device memory                */
    ORF_ECANCELLED = 3,        /* progress callback asked to stop              */
    ORF_ETIMEOUT_DEVICE = 4,   /* a bounded device-side wait ran out           */
    ORF_ECUDA = 5,             /* CUDA runtime error (message in orf_last_error)*/
    ORF_ENODEV = 6,            /* no CUDA device / library built without one   */
    ORF_EBUSY = 7,             /* serving queue full / ticket not finished     */
    ORF_ETOOLARGE = 8          /* request exceeds a documented size limit      */
} orf_status;

enum { ORF_TE = 0, ORF_TM = 1 };                 /* sim.pol        */
enum { ORF_DOUBLE = 0, ORF_SINGLE = 1 };         /* sim.precision  */

/* Progress callback, invoked on the calling thread every 50 simulated steps
 * (fdtd2D.m:18-20).  frac follows orf.fdtdProgress (fdtdProgress.m:1-13).
 * Return non-zero to cancel the run: the call then returns ORF_ECANCELLED. */
typedef int (*orf_progress_fn)(double frac, const char* msg, void* user);

/* ---------------------------------------------------------------- 2D ---- */
/* Mirrors the sim struct of orf.fdtd2D / orf.fdtd2DTE
 * (fdtd2D.m:9-23, fdtd2DTE.m:7-25). */
typedef struct orf_sim2d {
    int32_t pol;               /* ORF_TE (P=Ey,A=Hx,B=Hz) or ORF_TM (P=Hy,A=-Ex,B=-Ez) */
    int32_t nx, nz;            /* numel(sim.x), numel(sim.z)                          */
    double x0, z0, dx;         /* sim.x(1), sim.z(1), uniform spacing                 */
    const double* eps;         /* TE: nx*nz eps at P                                   */
    const double* eps_x;       /* TM: nx*(nz-1) (nx*nz if periodic_z) eps at A        */
    const double* eps_z;       /* TM: (nx-1)*nz eps at B                               */
    int32_t npml_x, npml_z;    /* sim.npml = [nx nz] CPML cells per end               */
    int32_t periodic_z;        /* sim.periodicZ                                        */
    int32_t src_ix;            /* sim.source.ix (0-based P column)                    */
    const double* src_profile; /* sim.source.profile, nz values                       */
    double src_neff, src_lambda0, src_bw;
    int32_t n_mon;             /* sim.monitors: P columns of x = const lines          */
    const int32_t* monitors;
    int32_t n_monz;            /* sim.monitorsZ: P rows of z = const lines            */
    const int32_t* monitors_z;
    int32_t n_lambda;          /* sim.lambdas [um]                                     */
    const double* lambdas;
    double max_time;           /* sim.maxTime (c0*t, um), default 1e4                 */
    double shutoff;            /* sim.shutoff, default 1e-10                           */
    double courant;            /* sim.courant, default 0.99/sqrt(2)                   */
    int32_t precision;         /* ORF_DOUBLE or ORF_SINGLE                             */
    int32_t flags;             /* reserved, 0                                          */
} orf_sim2d;

/* Mirrors the out struct (fdtd2D.m:25-29, fdtd2DTE.m:27-32).  Any pointer may
 * be NULL to skip that output. */
typedef struct orf_out2d {
    double* flux;      /* n_mon  x n_lambda, column-major                        */
    double* flux_z;    /* n_monz x n_lambda                                      */
    double* P;         /* complex nz x n_lambda x n_mon  (out.P, TE Ey / TM Hy)  */
    double* B;         /* complex nz x n_lambda x n_mon  (out.B, TE Hz / TM -Ez) */
    double* PZ;        /* complex nx x n_lambda x n_monz (out.PZ)                */
    double* AZ;        /* complex nx x n_lambda x n_monz (out.AZ, TE Hx / TM -Ex)*/
    int32_t converged; /* 0: maxTime reached (fdtd2D:notConverged)               */
    int32_t _pad;
    int64_t steps;
    double time;       /* steps * courant * dx                                   */
    double wall_time;  /* seconds                                                */
} orf_out2d;

/* ---------------------------------------------------------------- 3D ---- */
/* Mirrors the sim struct of orf.fdtd3D (fdtd3D.m:11-24). */
typedef struct orf_sim3d {
    int32_t nx, ny, nz;
    int32_t _pad0;
    double x0, y0, z0, d;
    const double* eps_x;       /* sim.eps.x, nx*ny*nz at Ex (x+d/2, y, z)   */
    const double* eps_y;       /* sim.eps.y at Ey                            */
    const double* eps_z;       /* sim.eps.z at Ez                            */
    int32_t npml[3];           /* sim.npml                                   */
    int32_t periodic[3];       /* sim.periodic                               */
    int32_t src_axis;          /* sim.source.axis - 1  (0 = x, 1 = y, 2 = z) */
    int32_t src_index;         /* sim.source.index - 1                       */
    const double* src_Ea;      /* Na*Nb profiles, a = axis+1, b = axis+2     */
    const double* src_Eb;
    const double* src_Ha;
    const double* src_Hb;
    double src_neff, src_lambda0, src_bw;
    int32_t n_mon;
    int32_t _pad1;
    const int32_t* mon_axis;   /* sim.monitors(q).axis - 1                   */
    const int32_t* mon_index;  /* sim.monitors(q).index - 1                  */
    int32_t n_lambda;
    int32_t _pad2;
    const double* lambdas;
    double max_time, shutoff, courant;   /* courant default 0.99/sqrt(3)     */
    int32_t precision;
    int32_t flags;
} orf_sim3d;

typedef struct orf_out3d {
    double* flux;              /* n_mon x n_lambda                                  */
    double* const* mon_Ea;     /* n_mon pointers, each complex Na x Nb x n_lambda   */
    double* const* mon_Eb;
    double* const* mon_Ha;     /* H averaged onto the E plane (fdtd3D.m:27-28)      */
    double* const* mon_Hb;
    int32_t converged;
    int32_t _pad;
    int64_t steps;
    double time;
    double wall_time;
} orf_out3d;

/* ------------------------------------------------------------ context --- */
typedef struct orf_ctx orf_ctx;

/* Tuning knobs of the 2D/3D step kernels; zero fields mean "autotuned". */
typedef struct orf_tuning {
    int32_t tsteps;            /* time steps fused per launch (temporal block depth) */
    int32_t variant;           /* kernel tile variant id, 0 = the precision's default */
    int32_t use_graph;         /* 1: capture the time loop in CUDA graphs            */
    int32_t _pad;
} orf_tuning;

/* Per-kernel timing, collected when orf_ctx_set_timing(ctx, 1): CUDA events
 * around every launch on the context's stream.  "interior" is the pipelined
 * step kernel of tiles away from the CPML, "frame" the step kernel of the
 * CPML/boundary tiles (2D), "flush" the DFT flush + check kernels. */
typedef struct orf_kernel_stats {
    double interior_ms;
    int64_t interior_launches;
    int64_t interior_cell_updates;   /* cells x time steps those launches advanced */
    double frame_ms;
    int64_t frame_launches;
    int64_t frame_cell_updates;
    double flush_ms;
    int64_t flush_launches;
    int64_t cell_updates;            /* all cells x time steps advanced           */
    int64_t h2d_bytes;               /* host->device bytes copied by run/create   */
    int64_t d2h_bytes;               /* device->host bytes copied by finish       */
    /* host wall time of orf_batch2d_run calls, by phase: instance setup (host
     * tables, device allocation, uploads, groups), the time loop, and the
     * copy-out of results (with the release of the instances' memory) */
    double setup_ms;
    double loop_ms;
    double finish_ms;
} orf_kernel_stats;

ORF_API int32_t     orf_abi_version(void);
ORF_API const char* orf_status_string(int32_t status);
/* Copies the last error message of this thread (NUL-terminated). */
ORF_API int32_t     orf_last_error(char* buf, size_t len);
ORF_API int32_t     orf_device_count(void);

/* Creates a context on `device`.  `stream` is a cudaStream_t or NULL (the
 * context then creates its own non-blocking stream). */
ORF_API int32_t orf_ctx_create(int32_t device, void* stream, orf_ctx** out);
/* Releases the caller's reference.  Every job and server built on the
 * context holds one more, so the context (its stream, tuning and counters)
 * lives until the last of them is destroyed: contexts, jobs and servers may
 * be destroyed in any order.  The device memory of finished runs is kept for
 * reuse by later runs (up to 8 GiB per process, released blocks first wait
 * for the device to be idle); releasing the last reference to a context
 * returns its device's cached memory to the driver. */
ORF_API int32_t orf_ctx_destroy(orf_ctx* ctx);
ORF_API int32_t orf_ctx_set_tuning(orf_ctx* ctx, const orf_tuning* t);
ORF_API int32_t orf_ctx_set_timing(orf_ctx* ctx, int32_t on);
ORF_API int32_t orf_ctx_get_stats(orf_ctx* ctx, orf_kernel_stats* st);
/* No counterpart in the reference (whose CPU / gpuArray loop has no device
 * waits).  Bounds of the 3D kernel's only device-side waits, the TMA plane
 * loads of its z-march: each wait gives up after wait_ns nanoseconds (0 = one
 * second, the default) and the run then returns ORF_ETIMEOUT_DEVICE from its
 * finish (the CTA that gave up first waits, with the same bound, for the
 * plane copies it still has in flight, and later launches of the run return
 * at once).  stall_plane >= 0 is a failure-detection test hook: in 3D jobs
 * created on this context afterwards, every tile loaded by TMA arms the ring
 * slot of its z-plane k0 + stall_plane without issuing the copies, so that
 * wait runs out; -1 (the default) turns it off.  Runs created before the call
 * keep their launch arguments (CUDA graphs). */
ORF_API int32_t orf_ctx_set_wait_injection(orf_ctx* ctx, int32_t stall_plane, int64_t wait_ns);
ORF_API int32_t orf_ctx_reset_stats(orf_ctx* ctx);
/* No counterpart in the reference.  Times every 2D kernel variant and fused
 * step depth (4, 6, 8, 10) on `steps` steps (0 = 200) of the n sims (shutoff
 * off) -- one run for n = 1, one batched orf_batch2d_run for n > 1 -- keeps
 * the fastest in ctx's tuning and returns it in *best (may be NULL).  Only
 * speed depends on the choice: every candidate computes the same values. */
ORF_API int32_t orf_autotune2d(orf_ctx* ctx, int32_t n, const orf_sim2d* sims, int32_t steps, orf_tuning* best);

/* One tile of a 2D run's plan (orf_plan2d): a CTA loads the lx x lz window at
 * (li0, lk0), advances it by the fused depth and stores the output rectangle
 * (oi0, ok0, ow, oh).  kind 0: interior tile (no CPML code), 1: frame tile
 * (CPML and boundary masks).  flags: 1 the loaded columns hold the TF/SF
 * plane, 2 / 4 the output holds an x / z monitor line, 8 / 16 (frame) the
 * loaded cells reach an x / z CPML slab. */
typedef struct orf_tile2d {
    int32_t kind;
    int32_t li0, lk0, lx, lz;
    int32_t oi0, ok0, ow, oh;
    int32_t flags;
} orf_tile2d;

/* No counterpart in the reference.  Host-only view of the tiles a 2D run of
 * `sim` would use under `tuning` (NULL: the defaults): the fused depth, the
 * interior kernel variant and every tile, interior tiles first.  Needs no
 * device, so tests and tools can check the tiling on any host.  The counts
 * are always written; the tiles only when tiles != NULL and cap holds them
 * all (ORF_ETOOLARGE when cap > 0 is too small). */
ORF_API int32_t orf_plan2d(const orf_sim2d* sim, const orf_tuning* tuning, orf_tile2d* tiles, int32_t cap,
                           int32_t* n_interior, int32_t* n_frame, int32_t* tsteps, int32_t* variant);

/* One tile of a 3D run's plan (orf_plan3d): a CTA marches the tw x th column
 * at (i0, j0) through the z planes [k0, k1).  kind 0: interior tile (no CPML
 * code), 1: CPML tile.  tma: 1 when its planes arrive by TMA tensor copies
 * (every tile whose halo does not wrap around a periodic x / y edge), whose
 * boxes start at x = tma_x (fields) and x = tma_index_x (material index). */
typedef struct orf_tile3d {
    int32_t kind;
    int32_t i0, j0, tw, th, k0, k1;
    int32_t tma, tma_x, tma_index_x;
} orf_tile3d;

/* No counterpart in the reference.  Host-only view of the tiles a 3D run of
 * `sim` would use, interior tiles first; needs no device.  Counts always
 * written; tiles when tiles != NULL and cap holds them all (ORF_ETOOLARGE
 * when cap > 0 is too small). */
ORF_API int32_t orf_plan3d(const orf_sim3d* sim, orf_tile3d* tiles, int32_t cap, int32_t* n_interior,
                           int32_t* n_cpml);

/* No counterpart in the reference.  The checked build of this library
 * (lib/liborf_fdtd_check.so, compiled with ORF_CHECK) tests every global
 * access of the 2D step kernels against its buffer and every stored cell
 * against the grid; an access that fails is counted and skipped.  Writes the
 * count on the current device since the last reset (reset != 0: clear it
 * after reading).  The normal build returns ORF_EINVAL. */
ORF_API int32_t orf_check_violations(uint64_t* count, int32_t reset);

/* ------------------------------------------------------------ 2D runs --- */
/* Element counts of the caller-allocated out arrays (complex counts are in
 * complex elements; allocate twice as many doubles). */
ORF_API int32_t orf_out2d_sizes(const orf_sim2d* sim, int64_t* n_flux, int64_t* n_flux_z,
                        int64_t* n_P, int64_t* n_PZ);

/* One orf.fdtd2D(sim) call: host arrays in, host arrays out.
 * Replaces toolbox/+orf/fdtd2D.m:1-29 (and fdtd2DTE.m:33-34 with pol = TE). */
ORF_API int32_t orf_fdtd2d_run(const orf_sim2d* sim, orf_out2d* out,
                       orf_progress_fn progress, void* user);
ORF_API int32_t orf_fdtd2d_run_ctx(orf_ctx* ctx, const orf_sim2d* sim, orf_out2d* out,
                           orf_progress_fn progress, void* user);

/* Device-resident form of the same run, for benchmarks and callers that keep
 * fields on the GPU: create (uploads + allocates), advance (enqueues steps,
 * asynchronous), finish (flux + copy-out, synchronous). */
typedef struct orf_job orf_job;
ORF_API int32_t orf_job2d_create(orf_ctx* ctx, const orf_sim2d* sim, orf_job** job);
ORF_API int32_t orf_job3d_create(orf_ctx* ctx, const orf_sim3d* sim, orf_job** job);
ORF_API int32_t orf_job_advance(orf_job* job, int64_t nsteps);
ORF_API int32_t orf_job_sync(orf_job* job);
ORF_API int32_t orf_job_reset(orf_job* job);       /* fields, DFT sums, step counter -> 0 */
ORF_API int64_t orf_job_steps_done(orf_job* job);
ORF_API int64_t orf_job_cells(orf_job* job);
ORF_API int32_t orf_job2d_finish(orf_job* job, orf_out2d* out);
ORF_API int32_t orf_job3d_finish(orf_job* job, orf_out3d* out);
/* Copies the current fields to host: 2D fills P, A, B with nx*nz, nx*nzA,
 * (nx-1)*nz doubles; 3D fills the six components (nx*ny*nz each, order
 * Ex Ey Ez Hx Hy Hz).  For parity tests. */
ORF_API int32_t orf_job_get_fields(orf_job* job, double* const* fields, int32_t nfields);

/* No counterpart in the reference (fdtd3D.m:1-29 runs one grid).  One z slab
 * of a 3D grid too large for one GPU: `slab` describes planes [z_offset,
 * z_offset + slab->nz) of a grid of nz_global planes -- their eps, the
 * source and monitors in local indices, npml of the whole grid.  Its CPML
 * profile in z is the whole grid's at those planes (none at an end that
 * borders another slab), so the slab's cells update bit for bit as in the
 * whole grid once its edge planes hold the neighbours' values: an inner end
 * carries one ghost plane, written by the caller after every step from the
 * neighbouring slab (below: Ex Ey Ez Hx Hy of its last own plane; above: Ex
 * Ey of its first own plane).  Needs a non-periodic z axis, shutoff = 0
 * (fixed step count) and inner ends outside the grid's CPML (ORF_EINVAL).
 * Fields are [nz][ny][pitch] per component, pitch = nx rounded up to 32. */
ORF_API int32_t orf_job3d_create_slab(orf_ctx* ctx, const orf_sim3d* slab, int32_t z_offset,
                                      int32_t nz_global, orf_job** job);
/* Enqueues exactly nsteps more steps of a 3D job on its context's stream
 * (the DFT fold and check after the 50th step of each chunk and after the
 * run's last step) and returns without waiting; after s steps from the start
 * the state is in buffer s % 2.  Does not mix with an unfinished chunk of
 * orf_job_advance (ORF_EINVAL). */
ORF_API int32_t orf_job3d_step(orf_job* job, int64_t nsteps);
/* Device address and size of plane k of field `field` (0..5: Ex Ey Ez Hx Hy
 * Hz) in field buffer `buffer` (0 or 1) of a 3D job: ny * pitch elements of
 * the run's precision, contiguous.  For halo exchanges between slabs. */
ORF_API int32_t orf_job3d_plane(orf_job* job, int32_t buffer, int32_t field, int32_t k, void** dev,
                                size_t* bytes);
ORF_API int32_t orf_job_destroy(orf_job* job);

/* Checkpoint / resume (no counterpart in the reference).  The state of a job
 * between chunks -- current fields, CPML psi, DFT sums, step and chunk
 * counters, energy peak -- as one self-describing host buffer of
 * orf_job_checkpoint_size bytes.  orf_job_restore loads it into a job created
 * from the same sim (maxTime may differ): advancing that job continues the
 * run exactly, bitwise, whatever the tuning of its context.  A run stopped
 * by cancellation or by its step budget resumes; one stopped by the energy
 * shutoff stays finished.  Both calls synchronise the job's stream; restore
 * fails with ORF_EINVAL on a buffer of another size, dimension, precision or
 * grid. */
ORF_API int32_t orf_job_checkpoint_size(orf_job* job, size_t* bytes);
ORF_API int32_t orf_job_checkpoint(orf_job* job, void* buf, size_t bytes);
ORF_API int32_t orf_job_restore(orf_job* job, const void* buf, size_t bytes);

/* No counterpart in the reference.  orf.fdtd2D(sim) for callers that cannot
 * allocate device memory at call time (a host with its own device memory
 * pool, such as a MATLAB gpuArray session, a serving process with a fixed
 * budget, or a loop that must not block on the allocator).  Runs the same
 * kernels as orf_fdtd2d_run but calls no cudaMalloc/cudaFree and no other
 * allocating routine.  All device state lives in one 64 MiB static
 * __device__ array that every GPU loading this library reserves until exit.
 * Runs needing more return ORF_ETOOLARGE, before any device work (the
 * 800 x 300 FP64 grating coupler with 51 wavelengths needs
 * about 20 MiB).  The first call on a device does a one-time set-up there:
 * it looks up the array's address and, CUDA loading modules lazily, loads the
 * module that holds the array (which reserves it) and the 2D kernels' code.
 * Make that first call (a small run is enough) at start-up, before the
 * device's memory goes to the caller's pool and before any stream capture;
 * later calls take no device memory.  `stream` (a cudaStream_t; NULL = the
 * per-thread default stream) must belong to the current device (ORF_EINVAL
 * otherwise): the array's address is the current device's.  Calls share the
 * array: calls that overlap on the GPU race, and each call zeroes what it
 * uses first.  There is no progress callback; the call returns when the run
 * is done. */
ORF_API int32_t orf_fdtd2d_run_noalloc(const orf_sim2d* sim, orf_out2d* out, void* stream);

/* ------------------------------------------------------------ 3D runs --- */
/* Plane sizes Na, Nb of each monitor (arrays of n_mon). */
ORF_API int32_t orf_out3d_sizes(const orf_sim3d* sim, int32_t* na, int32_t* nb);
/* One orf.fdtd3D(sim) call.  Replaces toolbox/+orf/fdtd3D.m:1-29. */
ORF_API int32_t orf_fdtd3d_run(const orf_sim3d* sim, orf_out3d* out,
                       orf_progress_fn progress, void* user);
ORF_API int32_t orf_fdtd3d_run_ctx(orf_ctx* ctx, const orf_sim3d* sim, orf_out3d* out,
                           orf_progress_fn progress, void* user);

/* ------------------------------------------------------------ batches --- */
/* Many independent 2D runs advanced together: runs of one kernel
 * configuration share each persistent-kernel launch, and the time loop is
 * captured in CUDA graphs.  All sims of one call must share the precision
 * (ORF_EINVAL otherwise); TE and TM runs may be mixed.  Replaces the sequential orf.fdtd2D calls of the
 * sweeps (examples/cpo_box_scan.m:23-31, optimizeGratingCoupler.m:1-12). */
ORF_API int32_t orf_batch2d_run(orf_ctx* ctx, int32_t n, const orf_sim2d* sims,
                        orf_out2d* outs, orf_progress_fn progress, void* user);

/* ------------------------------------------------------------ serving --- */
typedef struct orf_server orf_server;
typedef struct orf_serve_cfg {
    int64_t max_device_bytes;   /* admission budget; 0 = 90% of free memory   */
    int32_t max_jobs;           /* slot count; 0 = 1024                        */
    int32_t macro_steps;        /* steps advanced between admissions; 0 = 200  */
} orf_serve_cfg;
typedef struct orf_serve_job_info {
    double t_submit, t_admit, t_done;   /* seconds on the server's clock       */
    int64_t steps;
    int64_t cells;
    int32_t status;            /* the job's orf_status                        */
    int32_t dims;              /* 2 or 3                                       */
    int64_t device_bytes;      /* device memory the job held while resident    */
    int32_t preemptions;       /* times orf_serve_preempt moved it off the GPU */
    int32_t reserved;
} orf_serve_job_info;

ORF_API int32_t orf_serve_open(orf_ctx* ctx, const orf_serve_cfg* cfg, orf_server** srv);
/* The sim and its arrays are copied at submit.  The out struct, the arrays
 * it points to (and, in 3D, its per-monitor pointer arrays) must stay valid
 * until the ticket completes: the server writes them when it retires the
 * job, and sets out->wall_time to the job's latency (done - submit). */
ORF_API int32_t orf_serve_submit2d(orf_server* srv, const orf_sim2d* sim, orf_out2d* out,
                           int64_t* ticket);
ORF_API int32_t orf_serve_submit3d(orf_server* srv, const orf_sim3d* sim, orf_out3d* out,
                           int64_t* ticket);
/* Runs one scheduling round: admits queued jobs that fit, advances every
 * resident job by up to macro_steps, retires finished jobs. */
ORF_API int32_t orf_serve_step(orf_server* srv);
/* ORF_OK when the ticket is done (info filled), ORF_EBUSY otherwise. */
ORF_API int32_t orf_serve_poll(orf_server* srv, int64_t ticket, orf_serve_job_info* info);
ORF_API int32_t orf_serve_pending(orf_server* srv, int32_t* queued, int32_t* resident);
/* Preemption: a resident job's state (as orf_job_checkpoint) moves to host
 * memory, its device memory returns to the budget, and it joins the end of
 * the queue; re-admitted, it continues where it stopped, and its result is
 * bitwise that of the job run alone.  A queued or finished ticket is left
 * as it is.  Call from the thread that calls orf_serve_step. */
ORF_API int32_t orf_serve_preempt(orf_server* srv, int64_t ticket);
ORF_API double  orf_serve_clock(orf_server* srv);
ORF_API int32_t orf_serve_close(orf_server* srv);

/* Subpixel-averaged permittivity of a 3D grid on the GPU (the device form
 * of epsComponents3D, toolbox/+orf/epsComponents3D.m:1-27): for each Yee E
 * component, cells whose centre an interface passes near are sampled at
 * nsub^3 points; method 0 ("directional") takes the harmonic mean along the
 * component's axis, then the arithmetic mean over the other two; method 1
 * ("kottke") 1/eps_cc = n_c^2 <1/eps> + (1 - n_c^2)/<eps> with n the first
 * moment of the samples; shapes paint in order over the background nbg.  x, y, z are the cell centres
 * (uniform, one spacing); period = {Lx, Ly} folds x and y into [-L/2, L/2)
 * (NULL: no folding).  ex, ey, ez receive nx*ny*nz doubles each, column-major
 * (x fastest), at (x+d/2, y, z), (x, y+d/2, z), (x, y, z+d/2).  The values
 * are bitwise those of the package's host generator. */
enum {
    ORF_SHAPE_BOX = 0,      /* lo / hi: the box                                        */
    ORF_SHAPE_CONE = 1,     /* p: cx cy r1 r2 z1 z2 (a cylinder when r1 = r2)          */
    ORF_SHAPE_POLYGON = 2,  /* p: z1 z2; data: n0 vertices x0 y0 x1 y1 ...             */
    ORF_SHAPE_LATTICE = 3   /* p: x0 y0 period z1 z2 dRdz; data: radii R[n0][n1], row-major */
};
typedef struct orf_eps_shape {
    int32_t kind;
    int32_t n0, n1;
    int32_t reserved;
    double n;               /* refractive index                                        */
    double lo[3], hi[3];    /* bounding box (the band test's "near" region, minus h)   */
    double p[8];
    const double* data;
} orf_eps_shape;
ORF_API int32_t orf_eps3d(orf_ctx* ctx, const double* x, const double* y, const double* z, int32_t nx,
                          int32_t ny, int32_t nz, double nbg, int32_t nsub, int32_t method,
                          const double* period,
                          int32_t nshape, const orf_eps_shape* shapes, double* ex, double* ey, double* ez);

/* ---------------------------------------------------------------- FDFD --
 * The 2D TE frequency-domain solver with its adjoint (toolbox/+orf/fdfd2D.m:1-19,
 * `out = orf.fdfd2D(x, z, epsr, lambda0, J)`, out.solve, out.adjoint):
 *   (1/s_x) d/dx((1/s_x) dE/dx) + (1/s_z) d/dz((1/s_z) dE/dz) + k0^2 eps E = -J
 * for E = E_y on the grid's points (those of orf.fdtd2DTE), E = 0 outside,
 * stretched-coordinate PML s = 1 + i a (depth/L)^3 (e^{-i w t} convention)
 * of npml cells per side, a = 2 ln(1/R) / (k0 L), L = npml dx.
 * orf_fdfd2d_factor builds the operator and factors it on the device (block
 * LU along the longer axis; the shorter axis may hold at most 384 points);
 * each orf_fdfd2d_solve is then one forward and one backward sweep.
 * Complex arrays are interleaved (re, im) pairs of nx*nz entries in
 * column-major order (entry (i, k) at i + nx*k), as MATLAB's interleaved
 * complex API hands them over. */
typedef struct orf_fdfd2d {
    int32_t nx, nz;
    double dx;                 /* grid spacing, the same on both axes [um] */
    const double* eps;         /* relative permittivity, complex (nx*nz pairs) */
    double lambda0;            /* vacuum wavelength [um]; k0 = 2 pi / lambda0 */
    int32_t npml_x, npml_z;    /* PML cells per side (Npml, default 30 30) */
    double pml_reflection;     /* PmlReflection (default 1e-8) */
} orf_fdfd2d;
typedef struct orf_fdfd orf_fdfd;   /* factored operator, device-resident */

ORF_API int32_t orf_fdfd2d_factor(orf_ctx* ctx, const orf_fdfd2d* problem, orf_fdfd** out);
/* transpose 0: solves A x = -rhs (the field E for a current J = rhs, out.E /
 * out.solve(J2)); transpose 1: solves A.' x = rhs (out.adjoint(g): for a
 * figure of merit c = sum(g .* E), dc/deps = -k0^2 x .* E). */
ORF_API int32_t orf_fdfd2d_solve(orf_fdfd* f, const double* rhs, double* x, int32_t transpose);
/* block size (shorter axis), number of blocks, CTAs of the solver's cluster */
ORF_API int32_t orf_fdfd2d_info(const orf_fdfd* f, int32_t* block, int32_t* nblocks, int32_t* cluster);
ORF_API void    orf_fdfd2d_release(orf_fdfd* f);

#ifdef __cplusplus
}
#endif
#endif /* ORF_FDTD_H */
