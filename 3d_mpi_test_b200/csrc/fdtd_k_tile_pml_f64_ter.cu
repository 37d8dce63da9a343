// PML / face tile kernel (fdtd_tile_pml.cuh), double, terrain-following grid.
#include "fdtd_k_tile_pml_impl.cuh"

namespace fdtd {

template const void* tile_pml_kernel_ptr<double, true>(int, bool);
template void run_tile_pml<double, true>(int, bool, dim3, dim3, size_t, cudaStream_t, const Dev<double>&, const TileMaps&,
                                     const TileGeo&, const TileBox*, int);

}  // namespace fdtd
