// Registry of the two-level temporally blocked kernels (fdtd3d_tb.cuh).
// The kernels are instantiated in tb_kernels.cu (its own translation unit, so
// the library's sources compile in parallel); the host code in capi.cu picks
// a launch shape from this table.
#pragma once

#include <vector>

#include "fdtd3d_tb.cuh"

namespace jxf {

using TbKernel = void (*)(const Step3D, const MapsTB, const TbExtra);

struct TbConfig {
  int ry, nw, stages;
  int threads;  // 32 * nw
  int nr, ty;   // region rows, tile rows (nr - 3); the tile is TB_TZ columns wide
  size_t smem[2];     // [0 absorb / PEC, 1 CPML over all axes]
  TbKernel k[3][2];   // [0 absorb, 1 cpml (kappa = 1), 2 cpml (kappa > 1)][cbarr]
  size_t smem_ax[3];  // CPML (kappa = 1) for blocks touching one axis's slab [x, y, z]
  TbKernel kax[3][2];
  size_t smem_ax2[3];  // CPML (kappa = 1) for blocks touching two axes' slabs [xy, xz, yz]
  TbKernel kax2[3][2];
};

const std::vector<TbConfig>& tb_configs();

}  // namespace jxf
