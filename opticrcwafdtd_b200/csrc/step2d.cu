// step2d.cu -- variant table and dispatch of the 2D step kernel.
#include "orf_internal.cuh"

namespace orf {

cudaError_t launch_step2d_f32(bool te, bool idx16, bool pml, int variant, const void* insts, const Tile2D* tiles,
                              int ntiles, int halo, int off, int nsub, int par, int we, int grid, cudaStream_t s);
cudaError_t launch_step2d_f64(bool te, bool idx16, bool pml, int variant, const void* insts, const Tile2D* tiles,
                              int ntiles, int halo, int off, int nsub, int par, int we, int grid, cudaStream_t s);
int occ_step2d_f32(bool te, bool idx16, bool pml, int variant);
int occ_step2d_f64(bool te, bool idx16, bool pml, int variant);

namespace {
struct VDesc {
    int id, ks, wx, wz;
};
// tile = 32*wx columns x ks*wz rows; must match step2d_f32.cu / step2d_f64.cu
constexpr VDesc kV32[] = {{1, 16, 2, 4}, {2, 8, 4, 4}};
constexpr VDesc kV64[] = {{1, 8, 2, 8}, {2, 8, 2, 4}};
}  // namespace

int variant2d_count() { return 2; }

bool variant2d_info(int id, bool fp64, Variant2D* v) {
    const VDesc* tab = fp64 ? kV64 : kV32;
    for (int q = 0; q < 2; ++q) {
        if (tab[q].id == id) {
            v->id = id;
            v->ks = tab[q].ks;
            v->wx = tab[q].wx;
            v->wz = tab[q].wz;
            return true;
        }
    }
    return false;
}

size_t step2d_smem(bool fp64, bool te, bool pml, int variant) {
    Variant2D v;
    if (!variant2d_info(variant, fp64, &v)) return 0;
    return (size_t)((te ? 1 : 2) + (pml ? 4 : 0)) * v.lx() * v.lz() * (fp64 ? 8 : 4);
}

cudaError_t launch_step2d(bool fp64, bool te, bool idx16, bool pml, int variant, const void* insts,
                          const Tile2D* tiles, int ntiles, int halo, int launch_off, int nsub, int par,
                          int want_energy, int grid, cudaStream_t s) {
    if (nsub < 1 || nsub > kMaxSub || ntiles <= 0) return cudaErrorInvalidValue;
    if (fp64)
        return launch_step2d_f64(te, idx16, pml, variant, insts, tiles, ntiles, halo, launch_off, nsub, par,
                                 want_energy, grid, s);
    return launch_step2d_f32(te, idx16, pml, variant, insts, tiles, ntiles, halo, launch_off, nsub, par,
                             want_energy, grid, s);
}

int step2d_blocks_per_sm(bool fp64, bool te, bool idx16, bool pml, int variant) {
    return fp64 ? occ_step2d_f64(te, idx16, pml, variant) : occ_step2d_f32(te, idx16, pml, variant);
}

}  // namespace orf

namespace orf {

cudaError_t launch_fast2d_f32(bool te, bool idx16, int variant, const FastTile2D* tiles, int ntiles, int off,
                              int nsub, int par, int we, int grid, cudaStream_t s);
cudaError_t launch_fast2d_f64(bool te, bool idx16, int variant, const FastTile2D* tiles, int ntiles, int off,
                              int nsub, int par, int we, int grid, cudaStream_t s);
int occ_fast2d_f32(bool te, bool idx16, int variant);
int occ_fast2d_f64(bool te, bool idx16, int variant);

namespace {
// pipelined interior kernel geometries; must match fast2d_f32.cu / fast2d_f64.cu
constexpr VDesc kF32[] = {{1, 16, 4, 4}, {2, 8, 4, 4}};
constexpr VDesc kF64[] = {{1, 8, 4, 4}, {2, 8, 2, 8}};
}  // namespace

bool fast2d_info(int id, bool fp64, Variant2D* v) {
    const VDesc* tab = fp64 ? kF64 : kF32;
    for (int q = 0; q < 2; ++q) {
        if (tab[q].id == id) {
            v->id = id;
            v->ks = tab[q].ks;
            v->wx = tab[q].wx;
            v->wz = tab[q].wz;
            return true;
        }
    }
    return false;
}

cudaError_t launch_fast2d(bool fp64, bool te, bool idx16, int variant, const FastTile2D* tiles, int ntiles,
                          int launch_off, int nsub, int par, int want_energy, int grid, cudaStream_t s) {
    if (nsub < 1 || nsub > kMaxSub || ntiles <= 0) return cudaErrorInvalidValue;
    if (fp64) return launch_fast2d_f64(te, idx16, variant, tiles, ntiles, launch_off, nsub, par, want_energy, grid, s);
    return launch_fast2d_f32(te, idx16, variant, tiles, ntiles, launch_off, nsub, par, want_energy, grid, s);
}

int fast2d_blocks_per_sm(bool fp64, bool te, bool idx16, int variant) {
    return fp64 ? occ_fast2d_f64(te, idx16, variant) : occ_fast2d_f32(te, idx16, variant);
}

}  // namespace orf
