// Launchers of the time-marching kernels. Each kernel family is compiled in
// its own translation unit (fdtd_k_*.cu) with explicit instantiations for
// float and double, so the host solver never instantiates a kernel template
// itself and the families compile in parallel.
#pragma once

#include <cuda_runtime.h>

#include "fdtd_device.cuh"
#include "fdtd_march.cuh"
#include "fdtd_tile.cuh"
#include "fdtd_tile_pml.cuh"

namespace fdtd {

// two-pass kernels (fdtd_k_twopass.cu): pressure or velocity pass
template <typename R>
void run_two_pass(bool pressure, bool wind, dim3 grd, dim3 blk, cudaStream_t s, const Dev<R>& d, int code);

// moving-frame row shift (fdtd_k_twopass.cu)
template <typename R>
void run_shift_rows(cudaStream_t s, R* a, int rows, int nj, int sh, int lead, int tempJ, int J, int west_copy);

// impedance ground after a step at parity par (fdtd_k_twopass.cu); d holds
// the step's fused parameters (new level = 1 - par)
template <typename R>
void run_ground_tdbc(cudaStream_t s, const Dev<R>& d, const GroundC& gc, int par);

// row marching kernel (fdtd_k_march.cu); VW columns per thread (4: FP32 only)
template <typename R>
const void* march_kernel_ptr(int VW, bool wind, bool xf);
template <typename R>
void run_march(int VW, bool wind, bool xf, dim3 grd, dim3 blk, size_t smem, cudaStream_t s, const Dev<R>& d,
               const MarchTiling& t, int par);

// batched row marching kernel of the ensemble (fdtd_k_march.cu)
template <typename R>
const void* march_batch_kernel_ptr(int VW, bool wind, bool xf);
template <typename R>
void run_march_batch(int VW, bool wind, bool xf, dim3 grd, dim3 blk, size_t smem, cudaStream_t s,
                     const BatchWork* work, const BatchEntry<R>* entries, int nm, int phase);

// tiled kernel; form 0: lean tiles, 1: full tiles, 2: full tiles with the
// rarer features (inclusion mask, east TDBC, vectors holding both y
// layers), 3 + LM: PML / face tiles with the layers of set LM compiled in
// (bit 0 x, bit 1 y, bit 2 z); ter: terrain-following grid. Dispatch in
// fdtd_k_tile.cu.
template <typename R>
const void* tile_kernel_ptr(int form, bool wind, bool ter);
template <typename R>
void run_tile(int form, bool wind, bool ter, dim3 grd, dim3 blk, size_t smem, cudaStream_t s, const Dev<R>& d,
              const TileMaps& maps, const TileGeo& tg, const TileBox* work, int par);

// forms 0..2 (fdtd_k_tile_flat.cu, fdtd_k_tile_ter.cu)
template <typename R, bool TER>
const void* tile_base_ptr(int form, bool wind);
template <typename R, bool TER>
void run_tile_base(int form, bool wind, dim3 grd, dim3 blk, size_t smem, cudaStream_t s, const Dev<R>& d,
                   const TileMaps& maps, const TileGeo& tg, const TileBox* work, int par);

// PML / face tiles with layer set lm (fdtd_k_tile_pml_{f32,f64}{,_ter}.cu)
template <typename R, bool TER>
const void* tile_pml_kernel_ptr(int lm, bool wind);
template <typename R, bool TER>
void run_tile_pml(int lm, bool wind, dim3 grd, dim3 blk, size_t smem, cudaStream_t s, const Dev<R>& d,
                  const TileMaps& maps, const TileGeo& tg, const TileBox* work, int par);

}  // namespace fdtd
