// Lean and full forms of the tiled kernel (fdtd_tile.cuh), terrain-following grid.
#include "fdtd_k_tile_base_impl.cuh"

namespace fdtd {

template const void* tile_base_ptr<float, true>(int, bool);
template const void* tile_base_ptr<double, true>(int, bool);
template void run_tile_base<float, true>(int, bool, dim3, dim3, size_t, cudaStream_t, const Dev<float>&,
                                        const TileMaps&, const TileGeo&, const TileBox*, int);
template void run_tile_base<double, true>(int, bool, dim3, dim3, size_t, cudaStream_t, const Dev<double>&,
                                         const TileMaps&, const TileGeo&, const TileBox*, int);

}  // namespace fdtd
