// Registry of the one-step TMA kernels (fdtd3d_kernels.cuh): the launch shapes
// the autotuner chooses from.  The kernels are instantiated in tma_kernels.cu
// (its own translation unit, compiled in parallel with the host code).
#pragma once

#include <vector>

#include "fdtd3d_kernels.cuh"

namespace jxf {

using TmaKernel = void (*)(const Step3D, const Maps3D);
using TmaBatchKernel = void (*)(const TmaBatchArgs);

struct TmaConfig {
  int tz, ty, ry, stages;
  int threads;
  size_t smem[2];     // [mode: 0 absorb, 1 cpml]
  TmaKernel k[3][2];  // [0 absorb, 1 cpml (kappa = 1), 2 cpml (kappa > 1)][cbarr]
  // CPML (kappa = 1) for blocks touching the slab of one axis only [x, y, z][cbarr]
  size_t smem_ax[3];
  TmaKernel kax[3][2];
  // persistent batch kernels (same indices; nullptr: shape not offered for batches)
  TmaBatchKernel kb[3][2];
  TmaBatchKernel kbax[3][2];
};

const std::vector<TmaConfig>& tma_configs();

}  // namespace jxf
