// Instantiations of the two-level temporally blocked kernels and their
// launch-shape registry (tb_registry.h).
#include "tb_registry.h"

namespace jxf {

namespace {

template <int RY, int NW, int ST>
TbConfig make_tb() {
  TbConfig c;
  c.ry = RY;
  c.nw = NW;
  c.stages = ST;
  c.threads = 32 * NW;
  c.nr = RY * NW;
  c.ty = RY * NW - 3;
  c.smem[0] = TbLayout<RY, NW, ST, true, false>::SMEM_BYTES;
  c.smem[1] = TbLayout<RY, NW, ST, true, true>::SMEM_BYTES;
  c.k[0][0] = k3d_tb2<RY, NW, ST, MODE_ABSORB, false, false>;
  c.k[0][1] = k3d_tb2<RY, NW, ST, MODE_ABSORB, true, false>;
  c.k[1][0] = k3d_tb2<RY, NW, ST, MODE_CPML, false, false>;
  c.k[1][1] = k3d_tb2<RY, NW, ST, MODE_CPML, true, false>;
  c.k[2][0] = k3d_tb2<RY, NW, ST, MODE_CPML, false, true>;
  c.k[2][1] = k3d_tb2<RY, NW, ST, MODE_CPML, true, true>;
  c.smem_ax[0] = TbLayout<RY, NW, ST, true, true, 1>::SMEM_BYTES;
  c.smem_ax[1] = TbLayout<RY, NW, ST, true, true, 2>::SMEM_BYTES;
  c.smem_ax[2] = TbLayout<RY, NW, ST, true, true, 4>::SMEM_BYTES;
  c.kax[0][0] = k3d_tb2<RY, NW, ST, MODE_CPML, false, false, 1>;
  c.kax[0][1] = k3d_tb2<RY, NW, ST, MODE_CPML, true, false, 1>;
  c.kax[1][0] = k3d_tb2<RY, NW, ST, MODE_CPML, false, false, 2>;
  c.kax[1][1] = k3d_tb2<RY, NW, ST, MODE_CPML, true, false, 2>;
  c.kax[2][0] = k3d_tb2<RY, NW, ST, MODE_CPML, false, false, 4>;
  c.kax[2][1] = k3d_tb2<RY, NW, ST, MODE_CPML, true, false, 4>;
  c.smem_ax2[0] = TbLayout<RY, NW, ST, true, true, 3>::SMEM_BYTES;
  c.smem_ax2[1] = TbLayout<RY, NW, ST, true, true, 5>::SMEM_BYTES;
  c.smem_ax2[2] = TbLayout<RY, NW, ST, true, true, 6>::SMEM_BYTES;
  c.kax2[0][0] = k3d_tb2<RY, NW, ST, MODE_CPML, false, false, 3>;
  c.kax2[0][1] = k3d_tb2<RY, NW, ST, MODE_CPML, true, false, 3>;
  c.kax2[1][0] = k3d_tb2<RY, NW, ST, MODE_CPML, false, false, 5>;
  c.kax2[1][1] = k3d_tb2<RY, NW, ST, MODE_CPML, true, false, 5>;
  c.kax2[2][0] = k3d_tb2<RY, NW, ST, MODE_CPML, false, false, 6>;
  c.kax2[2][1] = k3d_tb2<RY, NW, ST, MODE_CPML, true, false, 6>;
  return c;
}

}  // namespace

const std::vector<TbConfig>& tb_configs() {
  static const std::vector<TbConfig> cfgs = {
      make_tb<4, 8, 3>(),   // 32-row region (29-row tile), 256 threads
      make_tb<2, 16, 3>(),  // 32-row region, 512 threads
      make_tb<2, 8, 3>(),   // 16-row region (13-row tile), 256 threads
      make_tb<2, 12, 3>(),  // 24-row region (21-row tile), 384 threads
      make_tb<1, 16, 3>(),  // 16-row region, one row per thread, 512 threads
      make_tb<4, 4, 3>(),   // 16-row region, four rows per thread, 128 threads
  };
  return cfgs;
}

}  // namespace jxf
