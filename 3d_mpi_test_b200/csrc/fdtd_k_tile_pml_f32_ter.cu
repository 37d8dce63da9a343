// PML / face tile kernel (fdtd_tile_pml.cuh), float, terrain-following grid.
#include "fdtd_k_tile_pml_impl.cuh"

namespace fdtd {

template const void* tile_pml_kernel_ptr<float, true>(int, bool);
template void run_tile_pml<float, true>(int, bool, dim3, dim3, size_t, cudaStream_t, const Dev<float>&, const TileMaps&,
                                     const TileGeo&, const TileBox*, int);

}  // namespace fdtd
