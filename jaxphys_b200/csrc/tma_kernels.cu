// Instantiations of the one-step TMA kernels (single grids and persistent
// batches) and their launch-shape registry (tma_registry.h).
#include "tma_registry.h"

namespace jxf {

namespace {

template <int TZ, int TY, int RY, int ST, bool BATCH>
TmaConfig make_cfg() {
  TmaConfig c{};
  c.tz = TZ;
  c.ty = TY;
  c.ry = RY;
  c.stages = ST;
  c.threads = TZ * (TY / RY);
  c.smem[0] = TmaLayout<TZ, TY, RY, ST, true, false>::SMEM_BYTES;
  c.smem[1] = TmaLayout<TZ, TY, RY, ST, true, true>::SMEM_BYTES;
  c.k[0][0] = k3d_tma<TZ, TY, RY, ST, MODE_ABSORB, false, false>;
  c.k[0][1] = k3d_tma<TZ, TY, RY, ST, MODE_ABSORB, true, false>;
  c.k[1][0] = k3d_tma<TZ, TY, RY, ST, MODE_CPML, false, false>;
  c.k[1][1] = k3d_tma<TZ, TY, RY, ST, MODE_CPML, true, false>;
  c.k[2][0] = k3d_tma<TZ, TY, RY, ST, MODE_CPML, false, true>;
  c.k[2][1] = k3d_tma<TZ, TY, RY, ST, MODE_CPML, true, true>;
  c.smem_ax[0] = TmaLayout<TZ, TY, RY, ST, true, true, 1>::SMEM_BYTES;
  c.smem_ax[1] = TmaLayout<TZ, TY, RY, ST, true, true, 2>::SMEM_BYTES;
  c.smem_ax[2] = TmaLayout<TZ, TY, RY, ST, true, true, 4>::SMEM_BYTES;
  c.kax[0][0] = k3d_tma<TZ, TY, RY, ST, MODE_CPML, false, false, 1>;
  c.kax[0][1] = k3d_tma<TZ, TY, RY, ST, MODE_CPML, true, false, 1>;
  c.kax[1][0] = k3d_tma<TZ, TY, RY, ST, MODE_CPML, false, false, 2>;
  c.kax[1][1] = k3d_tma<TZ, TY, RY, ST, MODE_CPML, true, false, 2>;
  c.kax[2][0] = k3d_tma<TZ, TY, RY, ST, MODE_CPML, false, false, 4>;
  c.kax[2][1] = k3d_tma<TZ, TY, RY, ST, MODE_CPML, true, false, 4>;
  if constexpr (BATCH) {
    c.kb[0][0] = k3d_tma_batch<TZ, TY, RY, ST, MODE_ABSORB, false, false>;
    c.kb[0][1] = k3d_tma_batch<TZ, TY, RY, ST, MODE_ABSORB, true, false>;
    c.kb[1][0] = k3d_tma_batch<TZ, TY, RY, ST, MODE_CPML, false, false>;
    c.kb[1][1] = k3d_tma_batch<TZ, TY, RY, ST, MODE_CPML, true, false>;
    c.kb[2][0] = k3d_tma_batch<TZ, TY, RY, ST, MODE_CPML, false, true>;
    c.kb[2][1] = k3d_tma_batch<TZ, TY, RY, ST, MODE_CPML, true, true>;
    c.kbax[0][0] = k3d_tma_batch<TZ, TY, RY, ST, MODE_CPML, false, false, 1>;
    c.kbax[0][1] = k3d_tma_batch<TZ, TY, RY, ST, MODE_CPML, true, false, 1>;
    c.kbax[1][0] = k3d_tma_batch<TZ, TY, RY, ST, MODE_CPML, false, false, 2>;
    c.kbax[1][1] = k3d_tma_batch<TZ, TY, RY, ST, MODE_CPML, true, false, 2>;
    c.kbax[2][0] = k3d_tma_batch<TZ, TY, RY, ST, MODE_CPML, false, false, 4>;
    c.kbax[2][1] = k3d_tma_batch<TZ, TY, RY, ST, MODE_CPML, true, false, 4>;
  }
  return c;
}

}  // namespace

const std::vector<TmaConfig>& tma_configs() {
  static const std::vector<TmaConfig> cfgs = {
      make_cfg<32, 8, 1, 4, true>(),   make_cfg<32, 16, 2, 4, false>(),
      make_cfg<64, 8, 2, 3, true>(),   make_cfg<32, 16, 4, 4, false>(),
      make_cfg<64, 16, 4, 3, false>(),
      // small-grid shapes: 128-thread blocks (more blocks per SM, less
      // shared memory per block), 3-stage ring
      make_cfg<32, 4, 1, 4, false>(),  make_cfg<32, 8, 2, 4, false>(),
      make_cfg<32, 8, 1, 3, true>(),   make_cfg<64, 4, 1, 3, true>(),
      make_cfg<32, 4, 1, 3, false>(),  make_cfg<16, 8, 1, 3, false>(),
      make_cfg<64, 8, 1, 3, true>(),
  };
  return cfgs;
}

}  // namespace jxf
