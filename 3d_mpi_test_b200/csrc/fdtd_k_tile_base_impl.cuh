// Launchers of the lean and full tile forms of k_tile for one grid kind
// (flat or terrain-following), included by one translation unit per kind.
#pragma once

#include "fdtd_kernels.hpp"

namespace fdtd {

template <typename R, bool TER>
const void* tile_base_ptr(int form, bool wind) {
    constexpr int V = static_cast<int>(16 / sizeof(R));
    switch (form) {
        case 0:
            return wind ? reinterpret_cast<const void*>(k_tile<R, true, V, false, false, TER>)
                        : reinterpret_cast<const void*>(k_tile<R, false, V, false, false, TER>);
        case 1:
            return wind ? reinterpret_cast<const void*>(k_tile<R, true, V, true, false, TER>)
                        : reinterpret_cast<const void*>(k_tile<R, false, V, true, false, TER>);
        default:
            return wind ? reinterpret_cast<const void*>(k_tile<R, true, V, true, true, TER>)
                        : reinterpret_cast<const void*>(k_tile<R, false, V, true, true, TER>);
    }
}

template <typename R, bool TER>
void run_tile_base(int form, bool wind, dim3 grd, dim3 blk, size_t smem, cudaStream_t s, const Dev<R>& d,
                   const TileMaps& maps, const TileGeo& tg, const TileBox* work, int par) {
    constexpr int V = static_cast<int>(16 / sizeof(R));
    switch (form) {
        case 0:
            if (wind) k_tile<R, true, V, false, false, TER><<<grd, blk, smem, s>>>(d, maps, tg, work, par);
            else k_tile<R, false, V, false, false, TER><<<grd, blk, smem, s>>>(d, maps, tg, work, par);
            break;
        case 1:
            if (wind) k_tile<R, true, V, true, false, TER><<<grd, blk, smem, s>>>(d, maps, tg, work, par);
            else k_tile<R, false, V, true, false, TER><<<grd, blk, smem, s>>>(d, maps, tg, work, par);
            break;
        default:
            if (wind) k_tile<R, true, V, true, true, TER><<<grd, blk, smem, s>>>(d, maps, tg, work, par);
            else k_tile<R, false, V, true, true, TER><<<grd, blk, smem, s>>>(d, maps, tg, work, par);
            break;
    }
}

}  // namespace fdtd
