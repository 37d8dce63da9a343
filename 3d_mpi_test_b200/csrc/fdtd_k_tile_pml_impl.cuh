// Launchers of the PML / face tile kernel for the eight layer sets (bit 0
// x, bit 1 y, bit 2 z), included by one translation unit per precision.
#pragma once

#include "fdtd_kernels.hpp"

namespace fdtd {

template <typename R, int LM, bool TER>
static const void* pml_ptr(bool wind) {
    return wind ? reinterpret_cast<const void*>(k_tile_pml_wind<R, true, LM, TER>)
                : reinterpret_cast<const void*>(k_tile_pml_calm<R, false, LM, TER>);
}

template <typename R, bool TER>
const void* tile_pml_kernel_ptr(int lm, bool wind) {
    switch (lm & 7) {
        case 0: return pml_ptr<R, 0, TER>(wind);
        case 1: return pml_ptr<R, 1, TER>(wind);
        case 2: return pml_ptr<R, 2, TER>(wind);
        case 3: return pml_ptr<R, 3, TER>(wind);
        case 4: return pml_ptr<R, 4, TER>(wind);
        case 5: return pml_ptr<R, 5, TER>(wind);
        case 6: return pml_ptr<R, 6, TER>(wind);
        default: return pml_ptr<R, 7, TER>(wind);
    }
}

template <typename R, int LM, bool TER>
static void pml_run(bool wind, dim3 grd, dim3 blk, size_t smem, cudaStream_t s, const Dev<R>& d,
                    const TileMaps& maps, const TileGeo& tg, const TileBox* work, int par) {
    if (wind) k_tile_pml_wind<R, true, LM, TER><<<grd, blk, smem, s>>>(d, maps, tg, work, par);
    else k_tile_pml_calm<R, false, LM, TER><<<grd, blk, smem, s>>>(d, maps, tg, work, par);
}

template <typename R, bool TER>
void run_tile_pml(int lm, bool wind, dim3 grd, dim3 blk, size_t smem, cudaStream_t s, const Dev<R>& d,
                  const TileMaps& maps, const TileGeo& tg, const TileBox* work, int par) {
    switch (lm & 7) {
        case 0: pml_run<R, 0, TER>(wind, grd, blk, smem, s, d, maps, tg, work, par); break;
        case 1: pml_run<R, 1, TER>(wind, grd, blk, smem, s, d, maps, tg, work, par); break;
        case 2: pml_run<R, 2, TER>(wind, grd, blk, smem, s, d, maps, tg, work, par); break;
        case 3: pml_run<R, 3, TER>(wind, grd, blk, smem, s, d, maps, tg, work, par); break;
        case 4: pml_run<R, 4, TER>(wind, grd, blk, smem, s, d, maps, tg, work, par); break;
        case 5: pml_run<R, 5, TER>(wind, grd, blk, smem, s, d, maps, tg, work, par); break;
        case 6: pml_run<R, 6, TER>(wind, grd, blk, smem, s, d, maps, tg, work, par); break;
        default: pml_run<R, 7, TER>(wind, grd, blk, smem, s, d, maps, tg, work, par); break;
    }
}

}  // namespace fdtd
