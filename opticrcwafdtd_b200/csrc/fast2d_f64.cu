// fast2d_f64.cu -- double instantiations of the pipelined 2D step kernel (step2d_fast.cuh).
#include "orf_fdtd.h"
#include "step2d_fast.cuh"

namespace orf {
namespace {

template <class IT, bool TE, bool PML, int KS, int WX, int WZ>
cudaError_t configure() {
    static int done[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && done[dev]) return cudaSuccess;
    constexpr size_t smem = fast::dyn_smem<double, IT, TE, PML, KS, WX, WZ>();
    cudaError_t e = cudaFuncSetAttribute(fast::k_step2d_fast<double, IT, TE, PML, KS, WX, WZ>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && dev < 64) done[dev] = 1;
    return e;
}

template <class IT, bool TE, bool PML, int KS, int WX, int WZ>
cudaError_t launch(const FastTile2D* tiles, int ntiles, int off, int nsub, int par, int we, int grid, cudaStream_t s) {
    constexpr size_t smem = fast::dyn_smem<double, IT, TE, PML, KS, WX, WZ>();
    fast::k_step2d_fast<double, IT, TE, PML, KS, WX, WZ><<<grid, 32 * WX * WZ, smem, s>>>(tiles, ntiles, off, nsub, par, we);
    return cudaGetLastError();
}

template <class IT, bool TE, bool PML, int KS, int WX, int WZ>
int occ() {
    if (configure<IT, TE, PML, KS, WX, WZ>() != cudaSuccess) return 0;
    constexpr size_t smem = fast::dyn_smem<double, IT, TE, PML, KS, WX, WZ>();
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fast::k_step2d_fast<double, IT, TE, PML, KS, WX, WZ>,
                                                      32 * WX * WZ, smem) != cudaSuccess)
        return 0;
    return nb;
}

template <bool PML, int KS, int WX, int WZ>
cudaError_t dispatch(bool te, bool idx16, const FastTile2D* tiles, int ntiles, int off, int nsub, int par, int we,
                     int grid, cudaStream_t s) {
    if (!idx16) return te ? launch<uint8_t, true, PML, KS, WX, WZ>(tiles, ntiles, off, nsub, par, we, grid, s)
                          : launch<uint8_t, false, PML, KS, WX, WZ>(tiles, ntiles, off, nsub, par, we, grid, s);
    return te ? launch<uint16_t, true, PML, KS, WX, WZ>(tiles, ntiles, off, nsub, par, we, grid, s)
              : launch<uint16_t, false, PML, KS, WX, WZ>(tiles, ntiles, off, nsub, par, we, grid, s);
}

template <bool PML, int KS, int WX, int WZ>
int occv(bool te, bool idx16) {
    if (!idx16) return te ? occ<uint8_t, true, PML, KS, WX, WZ>() : occ<uint8_t, false, PML, KS, WX, WZ>();
    return te ? occ<uint16_t, true, PML, KS, WX, WZ>() : occ<uint16_t, false, PML, KS, WX, WZ>();
}

}  // namespace

cudaError_t launch_fast2d_f64(bool te, bool idx16, bool pml, int variant, const FastTile2D* tiles, int ntiles,
                              int off, int nsub, int par, int we, int grid, cudaStream_t s) {
    if (pml) return dispatch<true, 8, 2, 5>(te, idx16, tiles, ntiles, off, nsub, par, we, grid, s);
    switch (variant) {
        case 1: return dispatch<false, 8, 4, 4>(te, idx16, tiles, ntiles, off, nsub, par, we, grid, s);
        case 2: return dispatch<false, 8, 2, 8>(te, idx16, tiles, ntiles, off, nsub, par, we, grid, s);
    }
    return cudaErrorInvalidValue;
}

// Out-of-bounds accesses caught by the checked build's double kernels (reset: set
// the counter back to zero); ORF_EINVAL in the normal build.
int fast2d_violations_f64(unsigned long long* n, int reset) {
#ifdef ORF_CHECK
    cudaError_t e = cudaMemcpyFromSymbol(n, fast::g_check_violations, sizeof *n);
    if (e == cudaSuccess && reset) {
        const unsigned long long z = 0;
        e = cudaMemcpyToSymbol(fast::g_check_violations, &z, sizeof z);
    }
    return e == cudaSuccess ? ORF_OK : ORF_ECUDA;
#else
    (void)reset;
    *n = 0;
    return ORF_EINVAL;
#endif
}

int occ_fast2d_f64(bool te, bool idx16, bool pml, int variant) {
    if (pml) return occv<true, 8, 2, 5>(te, idx16);
    switch (variant) {
        case 1: return occv<false, 8, 4, 4>(te, idx16);
        case 2: return occv<false, 8, 2, 8>(te, idx16);
    }
    return 0;
}

}  // namespace orf
