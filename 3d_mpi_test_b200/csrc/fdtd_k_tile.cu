// Tiled FB_p_v kernel (lean and full tile forms), instantiated for float
// (4-column vectors) and double (2-column vectors); the single-layer PML
// forms live in fdtd_k_tile_pml.cu.
#include "fdtd_kernels.hpp"

namespace fdtd {

template <typename R>
const void* tile_kernel_ptr(int form, bool wind) {
    constexpr int V = static_cast<int>(16 / sizeof(R));
    if (form >= 3) return tile_pml_kernel_ptr<R>(form - 3, wind);
    switch (form) {
        case 0:
            return wind ? reinterpret_cast<const void*>(k_tile<R, true, V, false, false>)
                        : reinterpret_cast<const void*>(k_tile<R, false, V, false, false>);
        case 1:
            return wind ? reinterpret_cast<const void*>(k_tile<R, true, V, true, false>)
                        : reinterpret_cast<const void*>(k_tile<R, false, V, true, false>);
        default:
            return wind ? reinterpret_cast<const void*>(k_tile<R, true, V, true, true>)
                        : reinterpret_cast<const void*>(k_tile<R, false, V, true, true>);
    }
}

template <typename R>
void run_tile(int form, bool wind, dim3 grd, dim3 blk, size_t smem, cudaStream_t s, const Dev<R>& d,
              const TileMaps& maps, const TileGeo& tg, const TileBox* work, int par) {
    constexpr int V = static_cast<int>(16 / sizeof(R));
    if (form >= 3) {
        run_tile_pml<R>(form - 3, wind, grd, blk, smem, s, d, maps, tg, work, par);
        return;
    }
    switch (form) {
        case 0:
            if (wind) k_tile<R, true, V, false, false><<<grd, blk, smem, s>>>(d, maps, tg, work, par);
            else k_tile<R, false, V, false, false><<<grd, blk, smem, s>>>(d, maps, tg, work, par);
            break;
        case 1:
            if (wind) k_tile<R, true, V, true, false><<<grd, blk, smem, s>>>(d, maps, tg, work, par);
            else k_tile<R, false, V, true, false><<<grd, blk, smem, s>>>(d, maps, tg, work, par);
            break;
        default:
            if (wind) k_tile<R, true, V, true, true><<<grd, blk, smem, s>>>(d, maps, tg, work, par);
            else k_tile<R, false, V, true, true><<<grd, blk, smem, s>>>(d, maps, tg, work, par);
            break;
    }
}

template const void* tile_kernel_ptr<float>(int, bool);
template const void* tile_kernel_ptr<double>(int, bool);
template void run_tile<float>(int, bool, dim3, dim3, size_t, cudaStream_t, const Dev<float>&, const TileMaps&,
                              const TileGeo&, const TileBox*, int);
template void run_tile<double>(int, bool, dim3, dim3, size_t, cudaStream_t, const Dev<double>&, const TileMaps&,
                               const TileGeo&, const TileBox*, int);

}  // namespace fdtd
