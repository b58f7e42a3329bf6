/* orf_fdtd_mex.c -- MATLAB MEX gateway of liborf_fdtd.so (include/orf_fdtd.h).
 *
 * MATLAB stays the host of OpticRCWAFDTD; this gateway is what the +orf
 * wrappers in ../matlab/+orf call instead of the reference's P-code:
 *
 *   out = orf_fdtd_mex('fdtd2D', sim)     orf.fdtd2D   (toolbox/+orf/fdtd2D.m:1-29)
 *   out = orf_fdtd_mex('fdtd2DTE', sim)   orf.fdtd2DTE (fdtd2DTE.m:33-34: pol forced to TE)
 *   out = orf_fdtd_mex('fdtd3D', sim)     orf.fdtd3D   (fdtd3D.m:1-29)
 *   c   = orf_fdtd_mex('marshal2d', sim)  the orf_sim2d the call would pass, as a struct
 *   c   = orf_fdtd_mex('marshal3d', sim)  the orf_sim3d likewise (for checking defaults)
 *   v   = orf_fdtd_mex('version')         orf_abi_version()
 *
 *   id  = orf_fdtd_mex('fdfd2D_factor', x, z, epsr, lambda0, Npml, PmlReflection)
 *   E   = orf_fdtd_mex('fdfd2D_solve', id, rhs, transpose)
 *         orf_fdtd_mex('fdfd2D_release', id)
 *         the frequency-domain solver of orf.fdfd2D (toolbox/+orf/fdfd2D.m:1-19):
 *         the factors stay on the device under a small integer id (at most
 *         64 at once) until released; transpose 0 returns E with A E = -rhs,
 *         1 returns lam with A.' lam = rhs.  epsr and rhs are nx x nz,
 *         real or complex; E is complex nx x nz.  +orf/fdfd2D.m builds the
 *         reference's result struct on these (out.solve, out.adjoint, fluxes).
 *
 * Inputs: every sim field of fdtd2D.m:9-23 / fdtd2DTE.m:7-25 / fdtd3D.m:11-24
 * with the reference's defaults (pol "TE", periodicZ false, npml 0,
 * source.neff 1, source.bw 0.2, maxTime 1e4, shutoff 1e-10, courant
 * 0.99/sqrt(2) in 2D and 0.99/sqrt(3) in 3D, precision "double"); MATLAB's
 * 1-based indices (source.ix / .index, monitors, monitorsZ, monitors(q).index)
 * become the ABI's 0-based ones.  Text fields must be char: the +orf wrappers
 * turn string scalars into char before the call.  sim.useGPU is accepted and
 * ignored: every run is on the GPU.  Arrays are column-major doubles, as the
 * ABI expects, so they are passed without a copy.
 *
 * Outputs: out.flux, out.fluxZ, out.P, out.B, out.PZ, out.AZ and the aliases
 * TE: Ey, Hz, EyZ, HxZ; TM: Hy, Ez = -B, HyZ, ExZ = -AZ (physical signs,
 * fdtd2D.m:26-27); 3D: out.flux and out.mon(q).Ea/Eb/Ha/Hb; then converged,
 * steps, time, wallTime.  Complex arrays use MATLAB's interleaved storage
 * (build with -R2018a), the ABI's layout.
 *
 * Errors: a non-zero status raises the MATLAB error identifier of its code
 * (orf:invalidInput, orf:outOfDeviceMemory, orf:deviceTimeout, orf:cuda,
 * orf:noDevice, ...) with the library's message.  An error thrown by
 * sim.progress cancels the run, and that same error is rethrown unchanged
 * (orf:cancelled in tests/TestGUISupport.m:39-43).  A run that reaches
 * maxTime issues the warning fdtd2D:notConverged / fdtd3D:notConverged.
 *
 * Build (MATLAB):  mex -R2018a -I<repo>/include orf_fdtd_mex.c -L<repo>/opticrcwafdtd_b200/lib -lorf_fdtd
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "mex.h"
#include "orf_fdtd.h"

#define MAXMON 64

/* ------------------------------------------------------------ helpers --- */
static void bad(const char* fmt, const char* a) { mexErrMsgIdAndTxt("orf:invalidInput", fmt, a); }

static const char* status_id(int32_t st) {
    switch (st) {
        case ORF_EINVAL: return "orf:invalidInput";
        case ORF_ENOMEM_DEVICE: return "orf:outOfDeviceMemory";
        case ORF_ECANCELLED: return "orf:cancelled";
        case ORF_ETIMEOUT_DEVICE: return "orf:deviceTimeout";
        case ORF_ECUDA: return "orf:cuda";
        case ORF_ENODEV: return "orf:noDevice";
        case ORF_EBUSY: return "orf:busy";
        case ORF_ETOOLARGE: return "orf:tooLarge";
    }
    return "orf:error";
}

static void fail(int32_t st) {
    char msg[2048];
    orf_last_error(msg, sizeof msg);
    mexErrMsgIdAndTxt(status_id(st), "%s (%s)", msg, orf_status_string(st));
}

/* a field of a scalar struct; missing or [] reads as absent */
static const mxArray* fld(const mxArray* s, const char* name) {
    const mxArray* a = mxGetField(s, 0, name);
    return (a && !mxIsEmpty(a)) ? a : NULL;
}

static double num(const mxArray* s, const char* name, double dflt) {
    const mxArray* a = fld(s, name);
    if (!a) return dflt;
    if ((!mxIsNumeric(a) && !mxIsLogical(a)) || mxGetNumberOfElements(a) != 1) bad("sim.%s must be a numeric scalar", name);
    return mxGetScalar(a);   /* the real part, as the reference reads neff */
}

static double need_num(const mxArray* s, const char* name, const char* what) {
    if (!fld(s, name)) bad("%s is required", what);
    return num(s, name, 0.0);
}

/* a real double array of exactly n elements (NULL when absent and n may be 0) */
static const double* dbl(const mxArray* a, size_t n, const char* what) {
    if (!mxIsDouble(a) || mxIsComplex(a)) bad("%s must be a real double array", what);
    if (mxGetNumberOfElements(a) != n) {
        char m[256];
        snprintf(m, sizeof m, "%s must have %zu elements, not %zu", what, n, (size_t)mxGetNumberOfElements(a));
        mexErrMsgIdAndTxt("orf:invalidInput", "%s", m);
    }
    return mxGetDoubles(a);
}

static const double* need_arr(const mxArray* s, const char* name, size_t n, const char* what) {
    const mxArray* a = fld(s, name);
    if (!a) bad("%s is required", what);
    return dbl(a, n, what);
}

/* uniform increasing grid vector */
static void grid(const mxArray* s, const char* name, int32_t* n, double* x0, double* d) {
    const mxArray* a = fld(s, name);
    if (!a || !mxIsDouble(a) || mxIsComplex(a) || mxGetNumberOfElements(a) < 2)
        bad("sim.%s must be a real vector of at least two points", name);
    const double* v = mxGetDoubles(a);
    const size_t m = mxGetNumberOfElements(a);
    const double h = v[1] - v[0];
    double dev = 0.0;
    for (size_t i = 1; i < m; ++i) dev = fmax(dev, fabs((v[i] - v[i - 1]) - h));
    if (!(h > 0) || dev > 1e-9 * fmax(1.0, fabs(h)) * (double)m) bad("sim.%s must be uniform and increasing", name);
    *n = (int32_t)m;
    *x0 = v[0];
    *d = h;
}

/* char field compared case-insensitively; dflt when absent */
static void text(const mxArray* s, const char* name, const char* dflt, char* out, size_t cap) {
    const mxArray* a = fld(s, name);
    if (!a) {
        snprintf(out, cap, "%s", dflt);
        return;
    }
    if (!mxIsChar(a) || mxGetString(a, out, (mwSize)cap) != 0) bad("sim.%s must be text (char)", name);
    for (char* p = out; *p; ++p)
        if (*p >= 'A' && *p <= 'Z') *p = (char)(*p - 'A' + 'a');
}

/* 1-based MATLAB indices -> 0-based int32 */
static int32_t index_vec(const mxArray* s, const char* name, int32_t* out, const char* what) {
    const mxArray* a = fld(s, name);
    if (!a) return 0;
    if (!mxIsDouble(a) || mxIsComplex(a)) bad("%s must be real doubles (1-based indices)", what);
    const size_t n = mxGetNumberOfElements(a);
    if (n > MAXMON) bad("%s: too many monitors", what);
    const double* v = mxGetDoubles(a);
    for (size_t i = 0; i < n; ++i) {
        if (v[i] != floor(v[i])) bad("%s must hold integer indices", what);
        out[i] = (int32_t)v[i] - 1;
    }
    return (int32_t)n;
}

static int32_t precision(const mxArray* s) {
    char p[16];
    text(s, "precision", "double", p, sizeof p);
    if (!strcmp(p, "double")) return ORF_DOUBLE;
    if (!strcmp(p, "single")) return ORF_SINGLE;
    bad("sim.precision must be \"double\" or \"single\"%s", "");
    return ORF_DOUBLE;
}

/* ------------------------------------------------------ progress (GUI) --- */
typedef struct {
    const mxArray* fn;
    mxArray* exc;   /* the error the callback threw */
} progress_box;

static int progress_cb(double frac, const char* msg, void* user) {
    progress_box* p = (progress_box*)user;
    mxArray* args[3];
    args[0] = (mxArray*)p->fn;
    args[1] = mxCreateDoubleScalar(frac);
    args[2] = mxCreateString(msg ? msg : "");
    mxArray* exc = mexCallMATLABWithTrap(0, NULL, 3, args, "feval");
    mxDestroyArray(args[1]);
    mxDestroyArray(args[2]);
    if (exc) {
        p->exc = exc;
        return 1;   /* cancel the run */
    }
    return 0;
}

static orf_progress_fn progress_of(const mxArray* sim, progress_box* box) {
    box->fn = fld(sim, "progress");
    box->exc = NULL;
    if (!box->fn) return NULL;
    if (!mxIsClass(box->fn, "function_handle")) bad("sim.progress must be a function handle%s", "");
    return progress_cb;
}

static void finish_status(int32_t st, progress_box* box) {
    if (st == ORF_ECANCELLED && box->exc) mexCallMATLAB(0, NULL, 1, &box->exc, "rethrow");
    if (st != ORF_OK) fail(st);
}

/* --------------------------------------------------------------- 2D ----- */
static void marshal2d(const mxArray* s, int force_te, orf_sim2d* c, int32_t* mons, int32_t* monz) {
    memset(c, 0, sizeof *c);
    char pol[8];
    text(s, "pol", "te", pol, sizeof pol);
    if (force_te) strcpy(pol, "te");
    if (strcmp(pol, "te") && strcmp(pol, "tm")) bad("sim.pol must be \"TE\" or \"TM\"%s", "");
    c->pol = strcmp(pol, "te") ? ORF_TM : ORF_TE;
    double dz;
    grid(s, "x", &c->nx, &c->x0, &c->dx);
    grid(s, "z", &c->nz, &c->z0, &dz);
    if (fabs(dz - c->dx) > 1e-9 * c->dx) bad("sim.x and sim.z must share one spacing%s", "");
    c->periodic_z = num(s, "periodicZ", 0.0) != 0.0;
    const size_t nx = (size_t)c->nx, nz = (size_t)c->nz;
    if (c->pol == ORF_TE) {
        c->eps = need_arr(s, "eps", nx * nz, "sim.eps (numel(x) x numel(z))");
    } else {
        const size_t nzA = c->periodic_z ? nz : nz - 1;
        c->eps_x = need_arr(s, "epsX", nx * nzA, "sim.epsX (numel(x) x numel(z)-1, or numel(z) if periodic)");
        c->eps_z = need_arr(s, "epsZ", (nx - 1) * nz, "sim.epsZ (numel(x)-1 x numel(z))");
    }
    const mxArray* np = fld(s, "npml");
    if (np) {
        const size_t k = mxGetNumberOfElements(np);
        if (!mxIsDouble(np) || (k != 1 && k != 2)) bad("sim.npml must be [nx nz]%s", "");
        c->npml_x = (int32_t)mxGetDoubles(np)[0];
        c->npml_z = (int32_t)mxGetDoubles(np)[k - 1];
    }
    const mxArray* src = fld(s, "source");
    if (!src || !mxIsStruct(src)) bad("sim.source is required%s", "");
    c->src_ix = (int32_t)need_num(src, "ix", "sim.source.ix") - 1;
    c->src_profile = need_arr(src, "profile", nz, "sim.source.profile (numel(z) values)");
    c->src_neff = num(src, "neff", 1.0);
    c->src_lambda0 = need_num(src, "lambda0", "sim.source.lambda0");
    c->src_bw = num(src, "bw", 0.2);
    c->n_mon = index_vec(s, "monitors", mons, "sim.monitors");
    c->monitors = mons;
    c->n_monz = index_vec(s, "monitorsZ", monz, "sim.monitorsZ");
    c->monitors_z = monz;
    const mxArray* lam = fld(s, "lambdas");
    if (!lam) bad("sim.lambdas is required%s", "");
    c->n_lambda = (int32_t)mxGetNumberOfElements(lam);
    c->lambdas = dbl(lam, (size_t)c->n_lambda, "sim.lambdas");
    c->max_time = num(s, "maxTime", 1e4);
    c->shutoff = num(s, "shutoff", 1e-10);
    c->courant = num(s, "courant", 0.99 / sqrt(2.0));
    c->precision = precision(s);
}

static mxArray* cplx3(size_t a, size_t b, size_t c) {
    mwSize d[3] = {(mwSize)a, (mwSize)b, (mwSize)c};
    return mxCreateNumericArray(3, d, mxDOUBLE_CLASS, mxCOMPLEX);
}

static double* cdata(mxArray* a) {
    return mxGetNumberOfElements(a) ? (double*)mxGetComplexDoubles(a) : NULL;
}

static mxArray* negated(const mxArray* a) {
    mxArray* r = mxDuplicateArray(a);
    double* v = cdata(r);
    for (size_t i = 0; v && i < 2 * mxGetNumberOfElements(r); ++i) v[i] = -v[i];
    return r;
}

static void run2d(int nlhs, mxArray* plhs[], const mxArray* s, int force_te) {
    orf_sim2d c;
    int32_t mons[MAXMON], monz[MAXMON];
    marshal2d(s, force_te, &c, mons, monz);
    const size_t nl = (size_t)c.n_lambda, nm = (size_t)c.n_mon, nmz = (size_t)c.n_monz;
    mxArray* flux = mxCreateDoubleMatrix((mwSize)nm, (mwSize)nl, mxREAL);
    mxArray* fluxz = mxCreateDoubleMatrix((mwSize)nmz, (mwSize)nl, mxREAL);
    mxArray* P = cplx3((size_t)c.nz, nl, nm);
    mxArray* B = cplx3((size_t)c.nz, nl, nm);
    mxArray* PZ = cplx3((size_t)c.nx, nl, nmz);
    mxArray* AZ = cplx3((size_t)c.nx, nl, nmz);
    orf_out2d o;
    memset(&o, 0, sizeof o);
    o.flux = nm ? mxGetDoubles(flux) : NULL;
    o.flux_z = nmz ? mxGetDoubles(fluxz) : NULL;
    o.P = cdata(P);
    o.B = cdata(B);
    o.PZ = cdata(PZ);
    o.AZ = cdata(AZ);
    progress_box box;
    const orf_progress_fn cb = progress_of(s, &box);
    finish_status(orf_fdtd2d_run(&c, &o, cb, &box), &box);
    static const char* te_names[] = {"flux", "fluxZ", "P", "B", "PZ", "AZ", "Ey", "Hz", "EyZ", "HxZ",
                                     "converged", "steps", "time", "wallTime"};
    static const char* tm_names[] = {"flux", "fluxZ", "P", "B", "PZ", "AZ", "Hy", "Ez", "HyZ", "ExZ",
                                     "converged", "steps", "time", "wallTime"};
    const int te = c.pol == ORF_TE;
    mxArray* out = mxCreateStructMatrix(1, 1, 14, te ? te_names : tm_names);
    mxSetFieldByNumber(out, 0, 0, flux);
    mxSetFieldByNumber(out, 0, 1, fluxz);
    mxSetFieldByNumber(out, 0, 6, mxDuplicateArray(P));
    mxSetFieldByNumber(out, 0, 7, te ? mxDuplicateArray(B) : negated(B));
    mxSetFieldByNumber(out, 0, 8, mxDuplicateArray(PZ));
    mxSetFieldByNumber(out, 0, 9, te ? mxDuplicateArray(AZ) : negated(AZ));
    mxSetFieldByNumber(out, 0, 2, P);
    mxSetFieldByNumber(out, 0, 3, B);
    mxSetFieldByNumber(out, 0, 4, PZ);
    mxSetFieldByNumber(out, 0, 5, AZ);
    mxSetFieldByNumber(out, 0, 10, mxCreateLogicalScalar(o.converged != 0));
    mxSetFieldByNumber(out, 0, 11, mxCreateDoubleScalar((double)o.steps));
    mxSetFieldByNumber(out, 0, 12, mxCreateDoubleScalar(o.time));
    mxSetFieldByNumber(out, 0, 13, mxCreateDoubleScalar(o.wall_time));
    if (!o.converged)
        mexWarnMsgIdAndTxt("fdtd2D:notConverged", "maxTime reached after %lld steps, before the field energy fell "
                           "below shutoff x its peak", (long long)o.steps);
    (void)nlhs;
    plhs[0] = out;
}

/* --------------------------------------------------------------- 3D ----- */
typedef struct {
    int32_t mon_axis[MAXMON], mon_index[MAXMON];
    double* prof[4];   /* source planes built here (mxMalloc: freed when the call ends) */
} store3d;

static void marshal3d(const mxArray* s, orf_sim3d* c, store3d* st) {
    memset(c, 0, sizeof *c);
    double dy, dz;
    grid(s, "x", &c->nx, &c->x0, &c->d);
    grid(s, "y", &c->ny, &c->y0, &dy);
    grid(s, "z", &c->nz, &c->z0, &dz);
    if (fabs(dy - c->d) > 1e-9 * c->d || fabs(dz - c->d) > 1e-9 * c->d)
        bad("sim.x, sim.y and sim.z must share one spacing%s", "");
    const int32_t n[3] = {c->nx, c->ny, c->nz};
    const size_t N = (size_t)n[0] * n[1] * n[2];
    const mxArray* e = fld(s, "eps");
    if (!e || !mxIsStruct(e)) bad("sim.eps (struct .x .y .z) is required%s", "");
    c->eps_x = need_arr(e, "x", N, "sim.eps.x (numel(x) x numel(y) x numel(z))");
    c->eps_y = need_arr(e, "y", N, "sim.eps.y");
    c->eps_z = need_arr(e, "z", N, "sim.eps.z");
    const mxArray* per = fld(s, "periodic");
    const mxArray* np = fld(s, "npml");
    for (int q = 0; q < 3; ++q) {
        int p = 0;
        if (per) {
            const size_t k = mxGetNumberOfElements(per);
            if ((k != 1 && k != 3) || !(mxIsLogical(per) || mxIsDouble(per)))
                bad("sim.periodic must be a logical or double [px py pz]%s", "");
            p = mxGetScalar(per) != 0.0;
            if (k == 3) p = mxIsLogical(per) ? mxGetLogicals(per)[q] != 0 : mxGetDoubles(per)[q] != 0.0;
        }
        int32_t m = 0;
        if (np) {
            const size_t k = mxGetNumberOfElements(np);
            if (!mxIsDouble(np) || (k != 1 && k != 3)) bad("sim.npml must be [nx ny nz]%s", "");
            m = (int32_t)mxGetDoubles(np)[k == 3 ? q : 0];
        }
        c->periodic[q] = p;
        c->npml[q] = p ? 0 : m;   /* no CPML on a periodic axis */
    }
    const mxArray* src = fld(s, "source");
    if (!src || !mxIsStruct(src)) bad("sim.source is required%s", "");
    const int ax = (int)need_num(src, "axis", "sim.source.axis") - 1;
    if (ax < 0 || ax > 2) bad("sim.source.axis must be 1, 2 or 3%s", "");
    c->src_axis = ax;
    c->src_index = (int32_t)need_num(src, "index", "sim.source.index") - 1;
    const size_t na = (size_t)n[(ax + 1) % 3], nb = (size_t)n[(ax + 2) % 3];
    static const char* pn[4] = {"Ea", "Eb", "Ha", "Hb"};
    const double* pp[4];
    for (int f = 0; f < 4; ++f) {
        const mxArray* a = fld(src, pn[f]);
        if (a && mxGetNumberOfElements(a) == na * nb) {
            pp[f] = dbl(a, na * nb, "sim.source plane profile (Na x Nb)");
            st->prof[f] = NULL;
            continue;
        }
        if (a && mxGetNumberOfElements(a) != 1) bad("sim.source.%s must be a scalar or Na x Nb", pn[f]);
        const double v = a ? mxGetScalar(a) : 0.0;   /* missing: zero, scalar: filled plane */
        st->prof[f] = (double*)mxMalloc(na * nb * sizeof(double));
        for (size_t i = 0; i < na * nb; ++i) st->prof[f][i] = v;
        pp[f] = st->prof[f];
    }
    c->src_Ea = pp[0];
    c->src_Eb = pp[1];
    c->src_Ha = pp[2];
    c->src_Hb = pp[3];
    c->src_neff = num(src, "neff", 1.0);
    c->src_lambda0 = need_num(src, "lambda0", "sim.source.lambda0");
    c->src_bw = num(src, "bw", 0.2);
    const mxArray* mons = fld(s, "monitors");
    if (mons) {
        if (!mxIsStruct(mons)) bad("sim.monitors must be a struct array with axis, index%s", "");
        const size_t k = mxGetNumberOfElements(mons);
        if (k > MAXMON) bad("sim.monitors: too many monitors%s", "");
        for (size_t q = 0; q < k; ++q) {
            const mxArray* a = mxGetField(mons, (mwIndex)q, "axis");
            const mxArray* i = mxGetField(mons, (mwIndex)q, "index");
            if (!a || !i) bad("sim.monitors(q) needs axis and index%s", "");
            st->mon_axis[q] = (int32_t)mxGetScalar(a) - 1;
            st->mon_index[q] = (int32_t)mxGetScalar(i) - 1;
        }
        c->n_mon = (int32_t)k;
    }
    c->mon_axis = st->mon_axis;
    c->mon_index = st->mon_index;
    const mxArray* lam = fld(s, "lambdas");
    if (!lam) bad("sim.lambdas is required%s", "");
    c->n_lambda = (int32_t)mxGetNumberOfElements(lam);
    c->lambdas = dbl(lam, (size_t)c->n_lambda, "sim.lambdas");
    c->max_time = num(s, "maxTime", 1e4);
    c->shutoff = num(s, "shutoff", 1e-10);
    c->courant = num(s, "courant", 0.99 / sqrt(3.0));
    c->precision = precision(s);
}

static void run3d(int nlhs, mxArray* plhs[], const mxArray* s) {
    orf_sim3d c;
    store3d st;
    marshal3d(s, &c, &st);
    const size_t nl = (size_t)c.n_lambda, nm = (size_t)c.n_mon;
    int32_t na[MAXMON], nb[MAXMON];
    const int32_t s3 = orf_out3d_sizes(&c, na, nb);
    if (s3 != ORF_OK) fail(s3);
    mxArray* flux = mxCreateDoubleMatrix((mwSize)nm, (mwSize)nl, mxREAL);
    static const char* mnames[] = {"Ea", "Eb", "Ha", "Hb"};
    mxArray* mon = mxCreateStructMatrix(1, (mwSize)nm, 4, mnames);
    double* ptrs[4][MAXMON];
    for (size_t q = 0; q < nm; ++q)
        for (int f = 0; f < 4; ++f) {
            mxArray* a = cplx3((size_t)na[q], (size_t)nb[q], nl);
            ptrs[f][q] = cdata(a);
            mxSetField(mon, (mwIndex)q, mnames[f], a);
        }
    orf_out3d o;
    memset(&o, 0, sizeof o);
    o.flux = nm ? mxGetDoubles(flux) : NULL;
    o.mon_Ea = ptrs[0];
    o.mon_Eb = ptrs[1];
    o.mon_Ha = ptrs[2];
    o.mon_Hb = ptrs[3];
    progress_box box;
    const orf_progress_fn cb = progress_of(s, &box);
    finish_status(orf_fdtd3d_run(&c, &o, cb, &box), &box);
    static const char* names[] = {"flux", "mon", "converged", "steps", "time", "wallTime"};
    mxArray* out = mxCreateStructMatrix(1, 1, 6, names);
    mxSetFieldByNumber(out, 0, 0, flux);
    mxSetFieldByNumber(out, 0, 1, mon);
    mxSetFieldByNumber(out, 0, 2, mxCreateLogicalScalar(o.converged != 0));
    mxSetFieldByNumber(out, 0, 3, mxCreateDoubleScalar((double)o.steps));
    mxSetFieldByNumber(out, 0, 4, mxCreateDoubleScalar(o.time));
    mxSetFieldByNumber(out, 0, 5, mxCreateDoubleScalar(o.wall_time));
    if (!o.converged)
        mexWarnMsgIdAndTxt("fdtd3D:notConverged", "maxTime reached after %lld steps, before the field energy fell "
                           "below shutoff x its peak", (long long)o.steps);
    (void)nlhs;
    plhs[0] = out;
}

/* ------------------------------------------------ marshal (inspection) --- */
static double sum(const double* v, size_t n) {
    double t = 0.0;
    for (size_t i = 0; v && i < n; ++i) t += v[i];
    return t;
}

static mxArray* ivec(const int32_t* v, int32_t n) {
    mxArray* a = mxCreateDoubleMatrix(1, (mwSize)n, mxREAL);
    for (int32_t i = 0; i < n; ++i) mxGetDoubles(a)[i] = v[i];
    return a;
}

static mxArray* dvec(const double* v, size_t n) {
    mxArray* a = mxCreateDoubleMatrix(1, (mwSize)n, mxREAL);
    if (n) memcpy(mxGetDoubles(a), v, n * sizeof(double));
    return a;
}

/* the orf_sim2d as a struct: scalars by field name, index vectors 0-based,
 * arrays by their sums (eps_sum, eps_x_sum, eps_z_sum) and the profile */
static void show2d(mxArray* plhs[], const mxArray* s) {
    orf_sim2d c;
    int32_t mons[MAXMON], monz[MAXMON];
    marshal2d(s, 0, &c, mons, monz);
    static const char* names[] = {"pol", "nx", "nz", "x0", "z0", "dx", "npml_x", "npml_z", "periodic_z", "src_ix",
                                  "src_neff", "src_lambda0", "src_bw", "monitors", "monitors_z", "lambdas",
                                  "max_time", "shutoff", "courant", "precision", "eps_sum", "eps_x_sum", "eps_z_sum",
                                  "src_profile"};
    mxArray* o = mxCreateStructMatrix(1, 1, 24, names);
    const double sc[13] = {(double)c.pol, (double)c.nx, (double)c.nz, c.x0, c.z0, c.dx, (double)c.npml_x,
                           (double)c.npml_z, (double)c.periodic_z, (double)c.src_ix, c.src_neff, c.src_lambda0,
                           c.src_bw};
    for (int f = 0; f < 13; ++f) mxSetFieldByNumber(o, 0, f, mxCreateDoubleScalar(sc[f]));
    mxSetFieldByNumber(o, 0, 13, ivec(c.monitors, c.n_mon));
    mxSetFieldByNumber(o, 0, 14, ivec(c.monitors_z, c.n_monz));
    mxSetFieldByNumber(o, 0, 15, dvec(c.lambdas, (size_t)c.n_lambda));
    mxSetFieldByNumber(o, 0, 16, mxCreateDoubleScalar(c.max_time));
    mxSetFieldByNumber(o, 0, 17, mxCreateDoubleScalar(c.shutoff));
    mxSetFieldByNumber(o, 0, 18, mxCreateDoubleScalar(c.courant));
    mxSetFieldByNumber(o, 0, 19, mxCreateDoubleScalar((double)c.precision));
    const size_t nx = (size_t)c.nx, nz = (size_t)c.nz, nzA = c.periodic_z ? nz : nz - 1;
    mxSetFieldByNumber(o, 0, 20, mxCreateDoubleScalar(sum(c.eps, nx * nz)));
    mxSetFieldByNumber(o, 0, 21, mxCreateDoubleScalar(sum(c.eps_x, nx * nzA)));
    mxSetFieldByNumber(o, 0, 22, mxCreateDoubleScalar(sum(c.eps_z, (nx - 1) * nz)));
    mxSetFieldByNumber(o, 0, 23, dvec(c.src_profile, nz));
    plhs[0] = o;
}

static void show3d(mxArray* plhs[], const mxArray* s) {
    orf_sim3d c;
    store3d st;
    marshal3d(s, &c, &st);
    static const char* names[] = {"nx", "ny", "nz", "x0", "y0", "z0", "d", "npml", "periodic", "src_axis",
                                  "src_index", "src_neff", "src_lambda0", "src_bw", "mon_axis", "mon_index",
                                  "lambdas", "max_time", "shutoff", "courant", "precision", "eps_sums",
                                  "src_sums"};
    mxArray* o = mxCreateStructMatrix(1, 1, 23, names);
    const double sc[7] = {(double)c.nx, (double)c.ny, (double)c.nz, c.x0, c.y0, c.z0, c.d};
    for (int f = 0; f < 7; ++f) mxSetFieldByNumber(o, 0, f, mxCreateDoubleScalar(sc[f]));
    mxSetFieldByNumber(o, 0, 7, ivec(c.npml, 3));
    mxSetFieldByNumber(o, 0, 8, ivec(c.periodic, 3));
    mxSetFieldByNumber(o, 0, 9, mxCreateDoubleScalar((double)c.src_axis));
    mxSetFieldByNumber(o, 0, 10, mxCreateDoubleScalar((double)c.src_index));
    mxSetFieldByNumber(o, 0, 11, mxCreateDoubleScalar(c.src_neff));
    mxSetFieldByNumber(o, 0, 12, mxCreateDoubleScalar(c.src_lambda0));
    mxSetFieldByNumber(o, 0, 13, mxCreateDoubleScalar(c.src_bw));
    mxSetFieldByNumber(o, 0, 14, ivec(c.mon_axis, c.n_mon));
    mxSetFieldByNumber(o, 0, 15, ivec(c.mon_index, c.n_mon));
    mxSetFieldByNumber(o, 0, 16, dvec(c.lambdas, (size_t)c.n_lambda));
    mxSetFieldByNumber(o, 0, 17, mxCreateDoubleScalar(c.max_time));
    mxSetFieldByNumber(o, 0, 18, mxCreateDoubleScalar(c.shutoff));
    mxSetFieldByNumber(o, 0, 19, mxCreateDoubleScalar(c.courant));
    mxSetFieldByNumber(o, 0, 20, mxCreateDoubleScalar((double)c.precision));
    const size_t N = (size_t)c.nx * c.ny * c.nz;
    const int32_t n[3] = {c.nx, c.ny, c.nz};
    const size_t np = (size_t)n[(c.src_axis + 1) % 3] * n[(c.src_axis + 2) % 3];
    const double es[3] = {sum(c.eps_x, N), sum(c.eps_y, N), sum(c.eps_z, N)};
    const double ss[4] = {sum(c.src_Ea, np), sum(c.src_Eb, np), sum(c.src_Ha, np), sum(c.src_Hb, np)};
    mxSetFieldByNumber(o, 0, 21, dvec(es, 3));
    mxSetFieldByNumber(o, 0, 22, dvec(ss, 4));
    plhs[0] = o;
}

/* -------------------------------------------------------------- FDFD ----- */
#define MAXFDFD 64
static orf_fdfd* g_fdfd[MAXFDFD];   /* factored operators by id - 1 */
static int32_t g_fdfd_n[MAXFDFD][2];

/* uniform increasing vector of at least three points */
static void vgrid(const mxArray* a, const char* name, int32_t* n, double* d) {
    if (!mxIsDouble(a) || mxIsComplex(a) || mxGetNumberOfElements(a) < 3)
        bad("%s must be a real vector of at least three points", name);
    const double* v = mxGetDoubles(a);
    const size_t m = mxGetNumberOfElements(a);
    const double h = v[1] - v[0];
    double dev = 0.0;
    for (size_t i = 1; i < m; ++i) dev = fmax(dev, fabs((v[i] - v[i - 1]) - h));
    if (!(h > 0) || dev > 1e-9 * fmax(1.0, fabs(h)) * (double)m) bad("%s must be uniform and increasing", name);
    *n = (int32_t)m;
    *d = h;
}

/* an nx x nz double array as interleaved complex: the array's own storage
 * when complex, else a complex copy in *tmp (destroyed by the caller) */
static const double* cplx_arg(const mxArray* a, size_t n, const char* what, mxArray** tmp) {
    *tmp = NULL;
    if (!mxIsDouble(a) || mxGetNumberOfElements(a) != n) bad("%s must be a double array of nx x nz elements", what);
    if (mxIsComplex(a)) return (const double*)mxGetComplexDoubles(a);
    *tmp = mxCreateDoubleMatrix((mwSize)n, 1, mxCOMPLEX);
    mxComplexDouble* c = mxGetComplexDoubles(*tmp);
    const double* r = mxGetDoubles(a);
    for (size_t q = 0; q < n; ++q) {
        c[q].real = r[q];
        c[q].imag = 0.0;
    }
    return (const double*)c;
}

static double real_scalar(const mxArray* a, const char* what) {
    if (!mxIsDouble(a) || mxIsComplex(a) || mxGetNumberOfElements(a) != 1) bad("%s must be a real scalar", what);
    return mxGetScalar(a);
}

static int fdfd_id(const mxArray* a) {
    const double v = real_scalar(a, "the fdfd2D id");
    const int id = (int)v;
    if ((double)id != v || id < 1 || id > MAXFDFD || !g_fdfd[id - 1]) bad("no factored operator has this id%s", "");
    return id - 1;
}

static void fdfd_factor(mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    if (nrhs != 7)
        mexErrMsgIdAndTxt("orf:invalidInput",
                          "usage: id = orf_fdtd_mex('fdfd2D_factor', x, z, epsr, lambda0, Npml, PmlReflection)");
    int32_t nx, nz;
    double dx, dz;
    vgrid(prhs[1], "x", &nx, &dx);
    vgrid(prhs[2], "z", &nz, &dz);
    if (fabs(dx - dz) > 1e-9 * dx) bad("x and z must have the same spacing%s", "");
    const double lambda0 = real_scalar(prhs[4], "lambda0");
    const mxArray* np = prhs[5];
    const size_t nn = mxGetNumberOfElements(np);
    if (!mxIsDouble(np) || mxIsComplex(np) || (nn != 1 && nn != 2)) bad("Npml must be one or two cell counts%s", "");
    const double* npv = mxGetDoubles(np);
    const double R = real_scalar(prhs[6], "PmlReflection");
    int slot = -1;
    for (int q = 0; q < MAXFDFD && slot < 0; ++q)
        if (!g_fdfd[q]) slot = q;
    if (slot < 0) bad("%s", "64 factored operators are held already: release some");
    mxArray* tmp = NULL;
    const double* eps = cplx_arg(prhs[3], (size_t)nx * nz, "epsr", &tmp);
    orf_fdfd2d pr;
    pr.nx = nx;
    pr.nz = nz;
    pr.dx = dx;
    pr.eps = eps;
    pr.lambda0 = lambda0;
    pr.npml_x = (int32_t)npv[0];
    pr.npml_z = (int32_t)npv[nn - 1];
    pr.pml_reflection = R;
    orf_ctx* ctx = NULL;
    int32_t st = orf_ctx_create(0, NULL, &ctx);
    orf_fdfd* f = NULL;
    if (st == ORF_OK) {
        st = orf_fdfd2d_factor(ctx, &pr, &f);
        orf_ctx_destroy(ctx);   /* the factors keep their context alive */
    }
    if (tmp) mxDestroyArray(tmp);
    if (st != ORF_OK) fail(st);
    g_fdfd[slot] = f;
    g_fdfd_n[slot][0] = nx;
    g_fdfd_n[slot][1] = nz;
    plhs[0] = mxCreateDoubleScalar((double)(slot + 1));
}

static void fdfd_solve(mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    if (nrhs != 4) mexErrMsgIdAndTxt("orf:invalidInput", "usage: E = orf_fdtd_mex('fdfd2D_solve', id, rhs, transpose)");
    const int q = fdfd_id(prhs[1]);
    const int32_t nx = g_fdfd_n[q][0], nz = g_fdfd_n[q][1];
    const double tr = real_scalar(prhs[3], "transpose");
    mxArray* tmp = NULL;
    const double* rhs = cplx_arg(prhs[2], (size_t)nx * nz, "the right-hand side", &tmp);
    mxArray* out = mxCreateDoubleMatrix((mwSize)nx, (mwSize)nz, mxCOMPLEX);
    const int32_t st = orf_fdfd2d_solve(g_fdfd[q], rhs, (double*)mxGetComplexDoubles(out), tr != 0.0);
    if (tmp) mxDestroyArray(tmp);
    if (st != ORF_OK) {
        mxDestroyArray(out);
        fail(st);
    }
    plhs[0] = out;
}

static void fdfd_release(int nrhs, const mxArray* prhs[]) {
    if (nrhs != 2) mexErrMsgIdAndTxt("orf:invalidInput", "usage: orf_fdtd_mex('fdfd2D_release', id)");
    const int q = fdfd_id(prhs[1]);
    orf_fdfd2d_release(g_fdfd[q]);
    g_fdfd[q] = NULL;
}

/* ------------------------------------------------------------- entry ----- */
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    char cmd[32];
    if (nrhs < 1 || !mxIsChar(prhs[0]) || mxGetString(prhs[0], cmd, sizeof cmd) != 0)
        mexErrMsgIdAndTxt("orf:invalidInput", "usage: out = orf_fdtd_mex(command, sim)");
    if (!strcmp(cmd, "version")) {
        plhs[0] = mxCreateDoubleScalar((double)orf_abi_version());
        return;
    }
    if (!strcmp(cmd, "fdfd2D_factor")) {
        fdfd_factor(plhs, nrhs, prhs);
        return;
    }
    if (!strcmp(cmd, "fdfd2D_solve")) {
        fdfd_solve(plhs, nrhs, prhs);
        return;
    }
    if (!strcmp(cmd, "fdfd2D_release")) {
        fdfd_release(nrhs, prhs);
        return;
    }
    if (nrhs != 2 || !mxIsStruct(prhs[1]) || mxGetNumberOfElements(prhs[1]) != 1)
        mexErrMsgIdAndTxt("orf:invalidInput", "orf_fdtd_mex('%s', sim): sim must be a scalar struct", cmd);
    if (!strcmp(cmd, "fdtd2D")) run2d(nlhs, plhs, prhs[1], 0);
    else if (!strcmp(cmd, "fdtd2DTE")) run2d(nlhs, plhs, prhs[1], 1);
    else if (!strcmp(cmd, "fdtd3D")) run3d(nlhs, plhs, prhs[1]);
    else if (!strcmp(cmd, "marshal2d")) show2d(plhs, prhs[1]);
    else if (!strcmp(cmd, "marshal3d")) show3d(plhs, prhs[1]);
    else mexErrMsgIdAndTxt("orf:invalidInput", "unknown command '%s'", cmd);
}
