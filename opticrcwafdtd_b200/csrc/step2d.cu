// step2d.cu -- tile geometries and dispatch of the 2D step kernel.
#include "orf_internal.cuh"

namespace orf {

cudaError_t launch_fast2d_f32(bool te, bool idx16, bool pml, int variant, const FastTile2D* tiles, int ntiles, int off,
                              int nsub, int par, int we, int grid, cudaStream_t s);
cudaError_t launch_fast2d_f64(bool te, bool idx16, bool pml, int variant, const FastTile2D* tiles, int ntiles, int off,
                              int nsub, int par, int we, int grid, cudaStream_t s);
int occ_fast2d_f32(bool te, bool idx16, bool pml, int variant);
int occ_fast2d_f64(bool te, bool idx16, bool pml, int variant);

namespace {
struct VDesc {
    int id, ks, wx, wz;
};
// tile = 32*wx columns x ks*wz rows; must match fast2d_f32.cu / fast2d_f64.cu
constexpr VDesc kF32[] = {{1, 16, 4, 4}, {2, 8, 4, 4}};
constexpr VDesc kF64[] = {{1, 8, 4, 4}, {2, 8, 2, 8}};
// CPML / boundary tiles: 64 x 40 covers a (npml + T)-cell frame strip in
// one tile row or column for npml = 20, T <= 6 (two rows at T = 8, which
// still wins overall in FP32: the interior dominates)
constexpr VDesc kF32Pml = {0, 8, 2, 5};
constexpr VDesc kF64Pml = {0, 8, 2, 5};
}  // namespace

int variant2d_count() { return 2; }

bool fast2d_info(int id, bool fp64, bool pml, Variant2D* v) {
    const VDesc* d = nullptr;
    if (pml) {
        d = fp64 ? &kF64Pml : &kF32Pml;
    } else {
        const VDesc* tab = fp64 ? kF64 : kF32;
        for (int q = 0; q < 2; ++q)
            if (tab[q].id == id) d = &tab[q];
    }
    if (!d) return false;
    v->id = d->id;
    v->ks = d->ks;
    v->wx = d->wx;
    v->wz = d->wz;
    return true;
}

cudaError_t launch_fast2d(bool fp64, bool te, bool idx16, bool pml, int variant, const FastTile2D* tiles, int ntiles,
                          int launch_off, int nsub, int par, int want_energy, int grid, cudaStream_t s) {
    if (nsub < 1 || nsub > kMaxSub || ntiles <= 0) return cudaErrorInvalidValue;
    if (fp64)
        return launch_fast2d_f64(te, idx16, pml, variant, tiles, ntiles, launch_off, nsub, par, want_energy, grid, s);
    return launch_fast2d_f32(te, idx16, pml, variant, tiles, ntiles, launch_off, nsub, par, want_energy, grid, s);
}

int fast2d_blocks_per_sm(bool fp64, bool te, bool idx16, bool pml, int variant) {
    return fp64 ? occ_fast2d_f64(te, idx16, pml, variant) : occ_fast2d_f32(te, idx16, pml, variant);
}

}  // namespace orf
