// Dispatch of the tiled FB_p_v kernel forms (lean, full, PML / face; flat
// or terrain-following grid) to their translation units.
#include "fdtd_kernels.hpp"

namespace fdtd {

template <typename R>
const void* tile_kernel_ptr(int form, bool wind, bool ter) {
    if (form >= 3) return ter ? tile_pml_kernel_ptr<R, true>(form - 3, wind) : tile_pml_kernel_ptr<R, false>(form - 3, wind);
    return ter ? tile_base_ptr<R, true>(form, wind) : tile_base_ptr<R, false>(form, wind);
}

template <typename R>
void run_tile(int form, bool wind, bool ter, dim3 grd, dim3 blk, size_t smem, cudaStream_t s, const Dev<R>& d,
              const TileMaps& maps, const TileGeo& tg, const TileBox* work, int par) {
    if (form >= 3) {
        if (ter) run_tile_pml<R, true>(form - 3, wind, grd, blk, smem, s, d, maps, tg, work, par);
        else run_tile_pml<R, false>(form - 3, wind, grd, blk, smem, s, d, maps, tg, work, par);
    } else {
        if (ter) run_tile_base<R, true>(form, wind, grd, blk, smem, s, d, maps, tg, work, par);
        else run_tile_base<R, false>(form, wind, grd, blk, smem, s, d, maps, tg, work, par);
    }
}

template const void* tile_kernel_ptr<float>(int, bool, bool);
template const void* tile_kernel_ptr<double>(int, bool, bool);
template void run_tile<float>(int, bool, bool, dim3, dim3, size_t, cudaStream_t, const Dev<float>&, const TileMaps&,
                              const TileGeo&, const TileBox*, int);
template void run_tile<double>(int, bool, bool, dim3, dim3, size_t, cudaStream_t, const Dev<double>&,
                               const TileMaps&, const TileGeo&, const TileBox*, int);

}  // namespace fdtd
