// step2d_f32.cu -- float instantiations of the 2D step kernel (step2d_impl.cuh).
#include "step2d_impl.cuh"

namespace orf {

cudaError_t launch_step2d_f32(bool te, bool idx16, bool pml, int variant, const void* insts, const Tile2D* tiles,
                             int ntiles, int halo, int off, int nsub, int par, int we, int grid, cudaStream_t s) {
    switch (variant) {
        case 1: return dispatch_v<float, 16, 2, 4>(te, idx16, pml, insts, tiles, ntiles, halo, off, nsub, par, we, grid, s);
        case 2: return dispatch_v<float, 8, 4, 4>(te, idx16, pml, insts, tiles, ntiles, halo, off, nsub, par, we, grid, s);
    }
    return cudaErrorInvalidValue;
}

int occ_step2d_f32(bool te, bool idx16, bool pml, int variant) {
    switch (variant) {
        case 1: return occ_v<float, 16, 2, 4>(te, idx16, pml);
        case 2: return occ_v<float, 8, 4, 4>(te, idx16, pml);
    }
    return 1;
}

}  // namespace orf
