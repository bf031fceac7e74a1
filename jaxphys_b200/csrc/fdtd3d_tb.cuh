// Two-level temporally blocked 3D Yee march (sm_100a).
//
// One launch advances the grid by TWO leapfrog steps of the reference's scan
// body (jaxphys src/neurosim/em/fdtd3d.py:280-379, applied twice):
//   H^{n+1/2} = H^{n-1/2} - a curl E^n,   E^{n+1} = (E^n + cb curl H^{n+1/2}) d + src_n
//   H^{n+3/2} = H^{n+1/2} - a curl E^{n+1}, E^{n+2} = (E^{n+1} + cb curl H^{n+3/2}) d + src_{n+1}
// so every field crosses HBM once per two steps (2.5D temporal blocking: the
// intermediate level n+1 lives only in registers and shared memory).
//
// Geometry.  A block owns a tile of TB_TZ = 28 columns (z) by TY = NR - 3 rows
// (y) and marches along x over a chunk of planes.  Its 32 lanes cover the
// columns z0-2 .. z0+29 and its NW warps the rows y0-2 .. y0+NR-3 (RY
// consecutive rows per thread): the tile plus the halo that the two levels
// need, recomputed rather than exchanged (every block computes its halo cells
// with the same operations as their owner, so the values are bit-identical).
// Validity shrinks level by level: H^{n+1/2} on lanes 0..30 / rows 0..NR-1,
// E^{n+1} on lanes 1..30 / rows 1..NR-1, H^{n+3/2} on lanes 1..29 / rows
// 1..NR-2, E^{n+2} on the tile (lanes 2..29, rows 2..NR-2).
//
// Neighbours: along z by warp shuffles; along y by registers inside a
// thread's rows and through small shared-memory edge buffers between warps;
// along x by registers (the level-1 planes q and q-1, the level-2 plane q-2).
// Level 2 runs one plane behind level 1: at march step q the block forms
// H^{n+1/2}(q), E^{n+1}(q), then H^{n+3/2}(q-1), E^{n+2}(q-1).  Two CTA
// barriers per march step (one per time level and plane, as in the one-step
// kernel).  E^n, H^{n-1/2} and cb planes arrive by TMA into a ring of
// mbarrier-tracked stages; every wait is bounded.
//
// CPML: psi^n is read from the input psi set for every region cell in a slab,
// psi^{n+1} of each cell is kept in shared memory (private to the thread that
// owns the cell, by plane parity) until level 2 uses it one march step later,
// and psi^{n+2} of the tile cells is written to the output set.
//
// All arithmetic uses __fadd_rn / __fsub_rn / __fmul_rn in the order of the
// one-step kernels, so two blocked steps equal two generic steps bit for bit.
#pragma once

#include "fdtd3d_kernels.cuh"

namespace jxf {

constexpr int TB_TZ = 28;  // tile columns
constexpr int TB_BW = 36;  // staged box width: z0-4 .. z0+31 (16-byte aligned start)

struct alignas(64) MapsTB {
  CUtensorMap e[3];  // box {36, NR+1, 1} at (z0-4, y0-2, x)
  CUtensorMap h[3];  // box {36, NR,   1} at (z0-4, y0-2, x)
  CUtensorMap cb;    // box {36, NR,   1} at (z0-4, y0-2, x)
};

// Per-block soft-source entry of the blocked kernel.  off = row * 32 + lane
// inside the block's region; lv bit 0: apply at level 1 (step n, any region
// cell), bit 1: at level 2 (step n+1, tile cells of the block's own planes).
struct TbSrc {
  int x;
  int off;
  int comp;
  int wave;
  float amp;
  int lv;
  int pad0, pad1;
};
// Per-block probe entry: a probe cell inside the block's tile and planes,
// recorded after level 1 (the state after step n+1) by its owner thread.
struct TbProbe {
  int x;
  int off;
  int comp;  // 0..5 = ex..hz
  int slot;
};

struct TbExtra {
  const int* src_ptr;  // CSR over blocks (grid order), or nullptr
  const TbSrc* src;
  const int* probe_ptr;  // CSR over blocks, or nullptr
  const TbProbe* probe;
  float* probe_mid;  // row of the state after the first step, or nullptr
};

template <int RY, int NW, int STAGES, bool CBARR, bool CPML, int AXES = 7>
struct TbLayout {
  static constexpr int NR = RY * NW;  // region rows
  static constexpr int TY = NR - 3;   // tile rows
  static constexpr int NT = 32 * NW;
  static constexpr int EH = NR + 1, HH = NR;
  static constexpr int E_STRIDE = round32(EH * TB_BW);
  static constexpr int H_STRIDE = round32(HH * TB_BW);
  static constexpr int CB_STRIDE = CBARR ? round32(HH * TB_BW) : 0;
  static constexpr int STAGE_FLOATS = 3 * E_STRIDE + 3 * H_STRIDE + CB_STRIDE;
  static constexpr uint32_t STAGE_TX =
      (uint32_t)(3 * EH * TB_BW + 3 * HH * TB_BW + (CBARR ? HH * TB_BW : 0)) * 4u;
  // warp edge buffers: XH1[2][NW][32], XE1[2 parity][2][NW][32], XH2[2][NW][32]
  static constexpr int X_FLOATS = 8 * NW * 32;
  static constexpr int NPSI = CPML ? psi_count(AXES) : 0;
  // psi per thread and cell in shared memory.  Ring (when it fits): three
  // slots by plane mod 3 -- psi^n of plane q+1 arrives by cp.async during
  // march step q, level 1 of plane q turns its slot into psi^{n+1} in place,
  // level 2 reads it one step later.  Otherwise two slots by plane parity
  // hold psi^{n+1} and psi^n is read from global memory where it is used.
  static constexpr size_t BASE_BYTES =
      128 + sizeof(float) * ((size_t)STAGES * STAGE_FLOATS + X_FLOATS);
  static constexpr bool RING =
      CPML && BASE_BYTES + sizeof(float) * 3 * (size_t)NPSI * NR * 32 <= 227 * 1024;
  static constexpr int NSLOT = RING ? 3 : 2;
  static constexpr int PS_FLOATS = NSLOT * NPSI * NR * 32;
  static constexpr size_t SMEM_BYTES = BASE_BYTES + sizeof(float) * (size_t)PS_FLOATS;
  static_assert(NR >= 8, "region too small");
  static_assert(STAGES >= 3 && STAGES <= 6, "ring needs >= 3 stages");
  static_assert(NT <= 1024, "block too large");
  static_assert(NR + 1 <= 256, "TMA box height");
  static_assert(SMEM_BYTES <= 227 * 1024, "shared memory per block exceeds 227 KB");
};

template <int RY, int NW, int STAGES, int MODE, bool CBARR, bool KAPPA, int AXES = 7>
__global__ void __launch_bounds__(32 * NW)
    k3d_tb2(const __grid_constant__ Step3D p, const __grid_constant__ MapsTB maps,
            const __grid_constant__ TbExtra ex) {
  constexpr bool CPML = (MODE == MODE_CPML);
  constexpr bool AX = CPML && (AXES & 1) != 0;
  constexpr bool AY = CPML && (AXES & 2) != 0;
  constexpr bool AZ = CPML && (AXES & 4) != 0;
  using L = TbLayout<RY, NW, STAGES, CBARR, CPML, AXES>;
  constexpr int NR = L::NR;
  constexpr int NT = L::NT;
  constexpr unsigned FULL = 0xffffffffu;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
  float* stages = reinterpret_cast<float*>(smem_raw + 128);
  float* XB = stages + STAGES * L::STAGE_FLOATS;
  float* PS = XB + L::X_FLOATS;
  // edge buffers
  float* XH1 = XB;                  // [2][NW][32]: H^{n+1/2} hx, hz of each warp's last row
  float* XE1 = XB + 2 * NW * 32;    // [2][2][NW][32]: E^{n+1} ex, ez of the first row, by parity
  float* XH2 = XB + 6 * NW * 32;    // [2][NW][32]: H^{n+3/2} hx, hz of the last row

  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int w = tid >> 5;
  int tzi = blockIdx.x, tyi = blockIdx.y, ci = blockIdx.z;
  if (p.blk_list != nullptr) {
    tzi = p.blk_list[3 * blockIdx.x];
    tyi = p.blk_list[3 * blockIdx.x + 1];
    ci = p.blk_list[3 * blockIdx.x + 2] & BLK_CHUNK_MASK;
  }
  const int z0 = tzi * TB_TZ;
  const int y0 = tyi * L::TY;
  const int z = z0 - 2 + lane;
  const bool zin = z >= 0 && z < nz;
  const int xb = ci * p.x_chunk;
  const int xe = min(xb + p.x_chunk, nx);
  const int qs = max(xb - 2, 0);          // first level-1 plane
  const int ql = min(xe + 1, nx - 1);     // last staged plane
  const int nload = ql - qs + 1;
  const float a = p.a;
  const int r0 = w * RY;  // first region row of this thread

  if (p.pdl & PDL_WAIT_START) grid_dep_wait();
  if (p.pdl & PDL_TRIGGER) grid_dep_launch_dependents();

  // probes of the input state (the state after the previous step)
  if (p.probe_out != nullptr && tzi == 0 && tyi == 0 && ci == 0) {
    for (int i = tid; i < p.n_probes; i += NT) p.probe_out[i] = p.in[p.probe_comp[i]][p.probe_cell[i]];
  }

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
    fence_barrier_init();
    for (int c = 0; c < 3; ++c) {
      prefetch_tmap(&maps.e[c]);
      prefetch_tmap(&maps.h[c]);
    }
    if (CBARR) prefetch_tmap(&maps.cb);
  }
  __syncthreads();

  auto issue = [&](int l) {
    if (l == p.drop_stage) return;  // fault injection: this stage never arrives
    const int slot = l % STAGES;
    float* st = stages + slot * L::STAGE_FLOATS;
    const int q = qs + l;
    mbar_arrive_expect_tx(&bars[slot], L::STAGE_TX);
#pragma unroll
    for (int c = 0; c < 3; ++c)
      tma_load_3d(st + c * L::E_STRIDE, &maps.e[c], z0 - 4, y0 - 2, q, &bars[slot]);
#pragma unroll
    for (int c = 0; c < 3; ++c)
      tma_load_3d(st + 3 * L::E_STRIDE + c * L::H_STRIDE, &maps.h[c], z0 - 4, y0 - 2, q,
                  &bars[slot]);
    if (CBARR)
      tma_load_3d(st + 3 * L::E_STRIDE + 3 * L::H_STRIDE, &maps.cb, z0 - 4, y0 - 2, q,
                  &bars[slot]);
  };
  if (tid == 0) {
    for (int l = 0; l < min(STAGES, nload); ++l) issue(l);
  }
  int issued = min(STAGES, nload);
  int consumed = 0;

  // ---- per-lane (z) and per-row (y) constants
  int yv[RY];
  bool rin[RY];  // row inside the grid
#pragma unroll
  for (int k = 0; k < RY; ++k) {
    yv[k] = y0 - 2 + r0 + k;
    rin[k] = yv[k] >= 0 && yv[k] < ny;
  }
  // tile membership (stores): rows 2..NR-2, lanes 2..29
  bool trow[RY];
#pragma unroll
  for (int k = 0; k < RY; ++k) trow[k] = (r0 + k) >= 2 && (r0 + k) <= NR - 2 && rin[k];
  const bool tlane = lane >= 2 && lane <= 29 && zin;

  // CPML constants
  const int SY = CPML ? p.pml.L[1] * nz : 0;  // y-slab arrays: [nx][L1][nz]
  const int SZ = CPML ? ny * p.pml.L[2] : 0;  // z-slab arrays: [nx][ny][L2]
  const int SX = ny * nz;                     // x-slab arrays: [L0][ny][nz]
  bool inz = false;
  float zbh = 1.f, zch = 0.f, zbe = 1.f, zce = 0.f, zikh = 1.f, zike = 1.f;
  int km = -1;
  bool iny[RY];
  int oy[RY], oz[RY], ox[RY];
  float ybh[RY], ych[RY], ybe[RY], yce[RY], yikh[RY], yike[RY];
#pragma unroll
  for (int k = 0; k < RY; ++k) {
    iny[k] = false;
    oy[k] = oz[k] = ox[k] = 0;
    ybh[k] = ybe[k] = 1.f;
    ych[k] = yce[k] = 0.f;
    yikh[k] = yike[k] = 1.f;
  }
  if (CPML) {
    if (zin) {
      km = slab_map(z, nz, p.pml.P[2]);
      inz = AZ && km >= 0;
      zbh = __ldg(p.pml.tab[2][TAB_BH] + z);
      zch = __ldg(p.pml.tab[2][TAB_CH] + z);
      zbe = __ldg(p.pml.tab[2][TAB_BE] + z);
      zce = __ldg(p.pml.tab[2][TAB_CE] + z);
      if (KAPPA) {
        zikh = __ldg(p.pml.tab[2][TAB_IKH] + z);
        zike = __ldg(p.pml.tab[2][TAB_IKE] + z);
      }
    }
#pragma unroll
    for (int k = 0; k < RY; ++k) {
      const int y = yv[k];
      if (rin[k]) {
        const int jm = slab_map(y, ny, p.pml.P[1]);
        iny[k] = AY && zin && jm >= 0;
        oy[k] = jm * nz + z;
        oz[k] = y * p.pml.L[2] + km;
        ox[k] = y * nz + z;
        ybh[k] = __ldg(p.pml.tab[1][TAB_BH] + y);
        ych[k] = __ldg(p.pml.tab[1][TAB_CH] + y);
        ybe[k] = __ldg(p.pml.tab[1][TAB_BE] + y);
        yce[k] = __ldg(p.pml.tab[1][TAB_CE] + y);
        if (KAPPA) {
          yikh[k] = __ldg(p.pml.tab[1][TAB_IKH] + y);
          yike[k] = __ldg(p.pml.tab[1][TAB_IKE] + y);
        }
      }
    }
  }
  // damping factors of this thread's column and rows (ABSORB; PEC: ones)
  float dz = 1.f, dyr[RY];
#pragma unroll
  for (int k = 0; k < RY; ++k) dyr[k] = 1.f;
  if (MODE == MODE_ABSORB) {
    if (zin) dz = __ldg(p.damp[2] + z);
#pragma unroll
    for (int k = 0; k < RY; ++k)
      if (rin[k]) dyr[k] = __ldg(p.damp[1] + yv[k]);
  }

#define PSV(slot, id, k) PS[((((slot) * L::NPSI + psi_slot(AXES, (id))) * NR) + r0 + (k)) * 32 + lane]
// psi^n of a level-1 cell: from the ring slot, or from global memory
#define PSN(id, off, k) (L::RING ? PSV(s1, id, k) : __ldg(p.pml.in[id] + (off)))
  // cp.async of psi^n of plane qq (this thread's slab cells) into ring slot qq % 3
  auto issue_psi = [&](int qq) {
    const int sl = qq % 3;
    const int imq = AX ? slab_map(qq, nx, p.pml.P[0]) : -1;
#pragma unroll
    for (int k = 0; k < RY; ++k) {
      const bool valid = rin[k] && zin;
      if (AY && iny[k]) {
        const int o = qq * SY + oy[k];
        cp_async4(&PSV(sl, PSI_HXY, k), p.pml.in[PSI_HXY] + o);
        cp_async4(&PSV(sl, PSI_HZY, k), p.pml.in[PSI_HZY] + o);
        cp_async4(&PSV(sl, PSI_EXY, k), p.pml.in[PSI_EXY] + o);
        cp_async4(&PSV(sl, PSI_EZY, k), p.pml.in[PSI_EZY] + o);
      }
      if (AZ && inz && valid) {
        const int o = qq * SZ + oz[k];
        cp_async4(&PSV(sl, PSI_HXZ, k), p.pml.in[PSI_HXZ] + o);
        cp_async4(&PSV(sl, PSI_HYZ, k), p.pml.in[PSI_HYZ] + o);
        cp_async4(&PSV(sl, PSI_EXZ, k), p.pml.in[PSI_EXZ] + o);
        cp_async4(&PSV(sl, PSI_EYZ, k), p.pml.in[PSI_EYZ] + o);
      }
      if (AX && imq >= 0 && valid) {
        const int o = imq * SX + ox[k];
        cp_async4(&PSV(sl, PSI_HYX, k), p.pml.in[PSI_HYX] + o);
        cp_async4(&PSV(sl, PSI_HZX, k), p.pml.in[PSI_HZX] + o);
        cp_async4(&PSV(sl, PSI_EYX, k), p.pml.in[PSI_EYX] + o);
        cp_async4(&PSV(sl, PSI_EZX, k), p.pml.in[PSI_EZX] + o);
      }
    }
  };
  const int q1last = min(xe, nx - 1);  // last level-1 plane
  if (L::RING) {
    if (qs <= q1last) issue_psi(qs);
    cp_async_commit();
  }

  // source / probe lists of this block
  const int bid = (ci * p.ntiles_y + tyi) * p.ntiles_z + tzi;
  int sp1 = 0, sp2 = 0, se = 0;
  if (ex.src_ptr != nullptr) {
    sp1 = sp2 = ex.src_ptr[bid];
    se = ex.src_ptr[bid + 1];
  }
  int pp = 0, pe = 0;
  if (ex.probe_ptr != nullptr && ex.probe_mid != nullptr) {
    pp = ex.probe_ptr[bid];
    pe = ex.probe_ptr[bid + 1];
  }

  // ---- march state (registers)
  float ec[3][RY], en[3][RY];    // E^n at planes q, q+1
  float h1[3][RY], h1p[3][RY];   // H^{n+1/2} at q, q-1
  float e1[3][RY], e1p[3][RY];   // E^{n+1} at q, q-1
  float h2p[2][RY];              // H^{n+3/2} (y, z comps) at q-2
  float cbc[RY], cbp[RY];        // cb at q, q-1
#pragma unroll
  for (int k = 0; k < RY; ++k) {
#pragma unroll
    for (int c = 0; c < 3; ++c) ec[c][k] = en[c][k] = h1[c][k] = h1p[c][k] = e1[c][k] = e1p[c][k] = 0.f;
    h2p[0][k] = h2p[1][k] = 0.f;
    cbc[k] = cbp[k] = p.cb_const;
  }

  int fail_l = -1;
  bool aborted = false;
  const long long wl = p.wave_len;

  // first plane's E^n into ec
  {
    bool ok = mbar_wait_bounded(&bars[0], 0u, p.wait_ns);
    if (!ok) fail_l = 0;
    const float* Es = stages;
#pragma unroll
    for (int k = 0; k < RY; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) ec[c][k] = Es[c * L::E_STRIDE + (r0 + k) * TB_BW + lane + 2];
    if (__syncthreads_or(ok ? 0 : 1)) aborted = true;
  }

  for (int q = qs; q <= xe && !aborted; ++q) {
    const int l = q - qs;
    const bool lvl1 = q <= nx - 1;         // level 1 exists at plane q
    const bool have_next = q + 1 <= ql;    // plane q+1 staged
    const int slot = l % STAGES;
    const int par = q & 1;
    // psi slots: level 1 (plane q) and level 2 (plane q-1)
    const int s1 = L::RING ? q % 3 : par;
    const int s2 = L::RING ? (q + 2) % 3 : par ^ 1;
    if (L::RING) {
      if (q + 1 <= q1last) issue_psi(q + 1);
      cp_async_commit();                 // (possibly empty) group of plane q+1
      cp_async_wait_pending<1>();        // plane q's psi^n has landed
    }
    bool ok = true;
    if (have_next) {
      ok = mbar_wait_bounded(&bars[(l + 1) % STAGES], (uint32_t)(((l + 1) / STAGES) & 1),
                             p.wait_ns);
      if (!ok) fail_l = l + 1;
    }
    const float* Es = stages + slot * L::STAGE_FLOATS;
    const float* En = stages + ((l + 1) % STAGES) * L::STAGE_FLOATS;
    const float* Hs = Es + 3 * L::E_STRIDE;
    const float* CBs = Hs + 3 * L::H_STRIDE;
#define ES(c, r) Es[(c) * L::E_STRIDE + (r) * TB_BW + lane + 2]
#define ENS(c, r) En[(c) * L::E_STRIDE + (r) * TB_BW + lane + 2]
#define HS(c, r) Hs[(c) * L::H_STRIDE + (r) * TB_BW + lane + 2]

    // x-slab of plane q (level 1) and q-1 (level 2)
    int imq = -1, imp = -1;
    float xbh = 1.f, xch = 0.f, xikh = 1.f, xbe = 1.f, xce = 0.f, xike = 1.f;
    float pbh = 1.f, pch = 0.f, pikh = 1.f, pbe = 1.f, pce = 0.f, pike = 1.f;
    if (AX) {
      if (lvl1) {
        imq = slab_map(q, nx, p.pml.P[0]);
        if (imq >= 0) {
          xbh = __ldg(p.pml.tab[0][TAB_BH] + q);
          xch = __ldg(p.pml.tab[0][TAB_CH] + q);
          xbe = __ldg(p.pml.tab[0][TAB_BE] + q);
          xce = __ldg(p.pml.tab[0][TAB_CE] + q);
          if (KAPPA) {
            xikh = __ldg(p.pml.tab[0][TAB_IKH] + q);
            xike = __ldg(p.pml.tab[0][TAB_IKE] + q);
          }
        }
      }
      if (q >= 1) {
        imp = slab_map(q - 1, nx, p.pml.P[0]);
        if (imp >= 0) {
          pbh = __ldg(p.pml.tab[0][TAB_BH] + q - 1);
          pch = __ldg(p.pml.tab[0][TAB_CH] + q - 1);
          pbe = __ldg(p.pml.tab[0][TAB_BE] + q - 1);
          pce = __ldg(p.pml.tab[0][TAB_CE] + q - 1);
          if (KAPPA) {
            pikh = __ldg(p.pml.tab[0][TAB_IKH] + q - 1);
            pike = __ldg(p.pml.tab[0][TAB_IKE] + q - 1);
          }
        }
      }
    }

    // ================= level 1: H^{n+1/2}(q) =================
    if (lvl1) {
#pragma unroll
      for (int k = 0; k < RY; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c) en[c][k] = have_next ? ENS(c, r0 + k) : 0.f;
      const bool inx = AX && imq >= 0;
#pragma unroll
      for (int k = 0; k < RY; ++k) {
        const int y = yv[k];
        const bool valid = rin[k] && zin;
        // y+1 neighbours (Ez, Ex)
        const float ezy = (k + 1 < RY) ? ec[2][(k + 1) % RY] : ES(2, r0 + RY);
        const float exy = (k + 1 < RY) ? ec[0][(k + 1) % RY] : ES(0, r0 + RY);
        // z+1 neighbours (Ey, Ex)
        const float eyz = __shfl_down_sync(FULL, ec[1][k], 1);
        const float exz = __shfl_down_sync(FULL, ec[0][k], 1);
        const float exc = ec[0][k], eyc = ec[1][k], ezc = ec[2][k];
        float hx = HS(0, r0 + k), hy = HS(1, r0 + k), hz = HS(2, r0 + k);
        const bool ux = valid && y < ny - 1 && z < nz - 1;
        const bool uy = valid && q < nx - 1 && z < nz - 1;
        const bool uz = valid && q < nx - 1 && y < ny - 1;
        const float dyEz = fsub(ezy, ezc), dzEy = fsub(eyz, eyc);
        const float dzEx = fsub(exz, exc), dxEz = fsub(en[2][k], ezc);
        const float dxEy = fsub(en[1][k], eyc), dyEx = fsub(exy, exc);
        const bool cy = iny[k], cz = inz && valid, cx = inx && valid;
        if (CPML && __any_sync(FULL, cy || cz || cx)) {
          const int oyq = q * SY + oy[k], ozq = q * SZ + oz[k], oxq = imq * SX + ox[k];
          if (ux) {
            const float p1 = pnext(cy, ybh[k], ych[k], cy ? PSN(PSI_HXY, oyq, k) : 0.f, dyEz);
            const float p2 = pnext(cz, zbh, zch, cz ? PSN(PSI_HXZ, ozq, k) : 0.f, dzEy);
            if (cy) PSV(s1, PSI_HXY, k) = p1;
            if (cz) PSV(s1, PSI_HXZ, k) = p2;
            hx = h_sel<KAPPA>(hx, a, dyEz, dzEy, cy, cz, p1, p2, yikh[k], zikh);
          }
          if (uy) {
            const float p1 = pnext(cz, zbh, zch, cz ? PSN(PSI_HYZ, ozq, k) : 0.f, dzEx);
            const float p2 = pnext(cx, xbh, xch, cx ? PSN(PSI_HYX, oxq, k) : 0.f, dxEz);
            if (cz) PSV(s1, PSI_HYZ, k) = p1;
            if (cx) PSV(s1, PSI_HYX, k) = p2;
            hy = h_sel<KAPPA>(hy, a, dzEx, dxEz, cz, cx, p1, p2, zikh, xikh);
          }
          if (uz) {
            const float p1 = pnext(cx, xbh, xch, cx ? PSN(PSI_HZX, oxq, k) : 0.f, dxEy);
            const float p2 = pnext(cy, ybh[k], ych[k], cy ? PSN(PSI_HZY, oyq, k) : 0.f, dyEx);
            if (cx) PSV(s1, PSI_HZX, k) = p1;
            if (cy) PSV(s1, PSI_HZY, k) = p2;
            hz = h_sel<KAPPA>(hz, a, dxEy, dyEx, cx, cy, p1, p2, xikh, yikh[k]);
          }
        } else {
          if (ux) hx = h_plain(hx, a, dyEz, dzEy);
          if (uy) hy = h_plain(hy, a, dzEx, dxEz);
          if (uz) hz = h_plain(hz, a, dxEy, dyEx);
        }
        h1[0][k] = hx;
        h1[1][k] = hy;
        h1[2][k] = hz;
      }
      XH1[(0 * NW + w) * 32 + lane] = h1[0][RY - 1];
      XH1[(1 * NW + w) * 32 + lane] = h1[2][RY - 1];
    }

    // ---- barrier 1: XH1 visible; stage slot of plane q-1 long free
    if (__syncthreads_or(ok ? 0 : 1)) {
      aborted = true;
      break;
    }

    // ================= level 1: E^{n+1}(q) =================
    if (lvl1) {
      const bool inx = AX && imq >= 0;
      const float dxq = MODE == MODE_ABSORB ? __ldg(p.damp[0] + q) : 1.f;
#pragma unroll
      for (int k = 0; k < RY; ++k) {
        const int y = yv[k];
        const bool valid = rin[k] && zin;
        cbc[k] = CBARR ? CBs[(r0 + k) * TB_BW + lane + 2] : p.cb_const;
        const float hzy = k > 0 ? h1[2][(k + RY - 1) % RY]
                                : (w > 0 ? XH1[(1 * NW + w - 1) * 32 + lane] : 0.f);
        const float hxy = k > 0 ? h1[0][(k + RY - 1) % RY]
                                : (w > 0 ? XH1[(0 * NW + w - 1) * 32 + lane] : 0.f);
        const float hyz = __shfl_up_sync(FULL, h1[1][k], 1);
        const float hxz = __shfl_up_sync(FULL, h1[0][k], 1);
        const float hxc = h1[0][k], hyc = h1[1][k], hzc = h1[2][k];
        float exv = ec[0][k], eyv = ec[1][k], ezv = ec[2][k];
        const float cb = cbc[k];
        const bool ux = valid && y >= 1 && z >= 1;
        const bool uy = valid && q >= 1 && z >= 1;
        const bool uz = valid && q >= 1 && y >= 1;
        const float dyHz = fsub(hzc, hzy), dzHy = fsub(hyc, hyz);
        const float dzHx = fsub(hxc, hxz), dxHz = fsub(hzc, h1p[2][k]);
        const float dxHy = fsub(hyc, h1p[1][k]), dyHx = fsub(hxc, hxy);
        const bool cy = iny[k], cz = inz && valid, cx = inx && valid;
        if (CPML && __any_sync(FULL, cy || cz || cx)) {
          const int oyq = q * SY + oy[k], ozq = q * SZ + oz[k], oxq = imq * SX + ox[k];
          if (ux) {
            const float p1 = pnext(cy, ybe[k], yce[k], cy ? PSN(PSI_EXY, oyq, k) : 0.f, dyHz);
            const float p2 = pnext(cz, zbe, zce, cz ? PSN(PSI_EXZ, ozq, k) : 0.f, dzHy);
            if (cy) PSV(s1, PSI_EXY, k) = p1;
            if (cz) PSV(s1, PSI_EXZ, k) = p2;
            exv = e_sel<KAPPA>(exv, cb, dyHz, dzHy, cy, cz, p1, p2, yike[k], zike);
          }
          if (uy) {
            const float p1 = pnext(cz, zbe, zce, cz ? PSN(PSI_EYZ, ozq, k) : 0.f, dzHx);
            const float p2 = pnext(cx, xbe, xce, cx ? PSN(PSI_EYX, oxq, k) : 0.f, dxHz);
            if (cz) PSV(s1, PSI_EYZ, k) = p1;
            if (cx) PSV(s1, PSI_EYX, k) = p2;
            eyv = e_sel<KAPPA>(eyv, cb, dzHx, dxHz, cz, cx, p1, p2, zike, xike);
          }
          if (uz) {
            const float p1 = pnext(cx, xbe, xce, cx ? PSN(PSI_EZX, oxq, k) : 0.f, dxHy);
            const float p2 = pnext(cy, ybe[k], yce[k], cy ? PSN(PSI_EZY, oyq, k) : 0.f, dyHx);
            if (cx) PSV(s1, PSI_EZX, k) = p1;
            if (cy) PSV(s1, PSI_EZY, k) = p2;
            ezv = e_sel<KAPPA>(ezv, cb, dxHy, dyHx, cx, cy, p1, p2, xike, yike[k]);
          }
        } else {
          if (ux) exv = e_plain(exv, cb, dyHz, dzHy);
          if (uy) eyv = e_plain(eyv, cb, dzHx, dxHz);
          if (uz) ezv = e_plain(ezv, cb, dxHy, dyHx);
        }
        if (MODE == MODE_ABSORB && valid) {
          const float f = fmul(fmul(dxq, dyr[k]), dz);
          exv = fmul(exv, f);
          eyv = fmul(eyv, f);
          ezv = fmul(ezv, f);
        }
        e1[0][k] = exv;
        e1[1][k] = eyv;
        e1[2][k] = ezv;
      }
      // soft sources of step n at plane q (every region cell that holds one)
      while (sp1 < se) {
        const TbSrc s = ex.src[sp1];
        if (s.x > q) break;
        if (s.x == q && (s.lv & 1)) {
          const int rr = s.off >> 5, ll = s.off & 31;
          if (ll == lane && rr >= r0 && rr < r0 + RY) {
            const float v = fmul(s.amp, p.wave[(long long)s.wave * wl + p.step]);
#pragma unroll
            for (int k = 0; k < RY; ++k)
              if (r0 + k == rr) {
                if (s.comp == 0) e1[0][k] = fadd(e1[0][k], v);
                else if (s.comp == 1) e1[1][k] = fadd(e1[1][k], v);
                else e1[2][k] = fadd(e1[2][k], v);
              }
          }
        }
        ++sp1;
      }
      // probes of the state after step n (owner threads)
      while (pp < pe) {
        const TbProbe pr = ex.probe[pp];
        if (pr.x > q) break;
        if (pr.x == q) {
          const int rr = pr.off >> 5, ll = pr.off & 31;
          if (ll == lane && rr >= r0 && rr < r0 + RY) {
#pragma unroll
            for (int k = 0; k < RY; ++k)
              if (r0 + k == rr) {
                float v;
                switch (pr.comp) {
                  case 0: v = e1[0][k]; break;
                  case 1: v = e1[1][k]; break;
                  case 2: v = e1[2][k]; break;
                  case 3: v = h1[0][k]; break;
                  case 4: v = h1[1][k]; break;
                  default: v = h1[2][k]; break;
                }
                ex.probe_mid[pr.slot] = v;
              }
          }
        }
        ++pp;
      }
      XE1[((par * 2 + 0) * NW + w) * 32 + lane] = e1[0][0];
      XE1[((par * 2 + 1) * NW + w) * 32 + lane] = e1[2][0];
    }

    // ================= level 2: H^{n+3/2}(q-1) =================
    const int x2 = q - 1;  // level-2 plane
    const bool lvl2h = x2 >= 0 && x2 >= xb - 1;
    float h2[3][RY];
#pragma unroll
    for (int k = 0; k < RY; ++k) h2[0][k] = h2[1][k] = h2[2][k] = 0.f;
    if (lvl2h) {
      const int ppar = x2 & 1;
      const bool inx = AX && imp >= 0;
      const bool own_plane = x2 >= xb;
#pragma unroll
      for (int k = 0; k < RY; ++k) {
        const int y = yv[k];
        const bool valid = rin[k] && zin;
        const float ezy = (k + 1 < RY) ? e1p[2][(k + 1) % RY]
                                       : (w + 1 < NW ? XE1[((ppar * 2 + 1) * NW + w + 1) * 32 + lane] : 0.f);
        const float exy = (k + 1 < RY) ? e1p[0][(k + 1) % RY]
                                       : (w + 1 < NW ? XE1[((ppar * 2 + 0) * NW + w + 1) * 32 + lane] : 0.f);
        const float eyz = __shfl_down_sync(FULL, e1p[1][k], 1);
        const float exz = __shfl_down_sync(FULL, e1p[0][k], 1);
        const float exc = e1p[0][k], eyc = e1p[1][k], ezc = e1p[2][k];
        float hx = h1p[0][k], hy = h1p[1][k], hz = h1p[2][k];
        const bool ux = valid && y < ny - 1 && z < nz - 1;
        const bool uy = valid && x2 < nx - 1 && z < nz - 1;
        const bool uz = valid && x2 < nx - 1 && y < ny - 1;
        const float dyEz = fsub(ezy, ezc), dzEy = fsub(eyz, eyc);
        const float dzEx = fsub(exz, exc), dxEz = fsub(e1[2][k], ezc);
        const float dxEy = fsub(e1[1][k], eyc), dyEx = fsub(exy, exc);
        const bool cy = iny[k], cz = inz && valid, cx = inx && valid;
        if (CPML && __any_sync(FULL, cy || cz || cx)) {
          const bool own = own_plane && trow[k] && tlane;
          const int oyq = x2 * SY + oy[k], ozq = x2 * SZ + oz[k], oxq = imp * SX + ox[k];
          if (ux) {
            const float p1 = pnext(cy, ybh[k], ych[k], cy ? PSV(s2, PSI_HXY, k) : 0.f, dyEz);
            const float p2 = pnext(cz, zbh, zch, cz ? PSV(s2, PSI_HXZ, k) : 0.f, dzEy);
            if (own && cy) p.pml.out[PSI_HXY][oyq] = p1;
            if (own && cz) p.pml.out[PSI_HXZ][ozq] = p2;
            hx = h_sel<KAPPA>(hx, a, dyEz, dzEy, cy, cz, p1, p2, yikh[k], zikh);
          }
          if (uy) {
            const float p1 = pnext(cz, zbh, zch, cz ? PSV(s2, PSI_HYZ, k) : 0.f, dzEx);
            const float p2 = pnext(cx, pbh, pch, cx ? PSV(s2, PSI_HYX, k) : 0.f, dxEz);
            if (own && cz) p.pml.out[PSI_HYZ][ozq] = p1;
            if (own && cx) p.pml.out[PSI_HYX][oxq] = p2;
            hy = h_sel<KAPPA>(hy, a, dzEx, dxEz, cz, cx, p1, p2, zikh, pikh);
          }
          if (uz) {
            const float p1 = pnext(cx, pbh, pch, cx ? PSV(s2, PSI_HZX, k) : 0.f, dxEy);
            const float p2 = pnext(cy, ybh[k], ych[k], cy ? PSV(s2, PSI_HZY, k) : 0.f, dyEx);
            if (own && cx) p.pml.out[PSI_HZX][oxq] = p1;
            if (own && cy) p.pml.out[PSI_HZY][oyq] = p2;
            hz = h_sel<KAPPA>(hz, a, dxEy, dyEx, cx, cy, p1, p2, pikh, yikh[k]);
          }
        } else {
          if (ux) hx = h_plain(hx, a, dyEz, dzEy);
          if (uy) hy = h_plain(hy, a, dzEx, dxEz);
          if (uz) hz = h_plain(hz, a, dxEy, dyEx);
        }
        h2[0][k] = hx;
        h2[1][k] = hy;
        h2[2][k] = hz;
      }
      XH2[(0 * NW + w) * 32 + lane] = h2[0][RY - 1];
      XH2[(1 * NW + w) * 32 + lane] = h2[2][RY - 1];
    }

    // ---- barrier 2: XH2 visible; every thread is done with stage `slot`
    __syncthreads();
    consumed = l + 1;
    if (issued < nload && issued < consumed + STAGES) {
      if (tid == 0) issue(issued);
      ++issued;
    }

    // ================= level 2: E^{n+2}(q-1), stores =================
    if (lvl2h && x2 >= xb) {
      const bool inx = AX && imp >= 0;
      const float dxq = MODE == MODE_ABSORB ? __ldg(p.damp[0] + x2) : 1.f;
      float eo[3][RY];
#pragma unroll
      for (int k = 0; k < RY; ++k) {
        const int y = yv[k];
        const bool valid = rin[k] && zin;
        const float hzy = k > 0 ? h2[2][(k + RY - 1) % RY]
                                : (w > 0 ? XH2[(1 * NW + w - 1) * 32 + lane] : 0.f);
        const float hxy = k > 0 ? h2[0][(k + RY - 1) % RY]
                                : (w > 0 ? XH2[(0 * NW + w - 1) * 32 + lane] : 0.f);
        const float hyz = __shfl_up_sync(FULL, h2[1][k], 1);
        const float hxz = __shfl_up_sync(FULL, h2[0][k], 1);
        const float hxc = h2[0][k], hyc = h2[1][k], hzc = h2[2][k];
        float exv = e1p[0][k], eyv = e1p[1][k], ezv = e1p[2][k];
        const float cb = cbp[k];
        const bool ux = valid && y >= 1 && z >= 1;
        const bool uy = valid && x2 >= 1 && z >= 1;
        const bool uz = valid && x2 >= 1 && y >= 1;
        const float dyHz = fsub(hzc, hzy), dzHy = fsub(hyc, hyz);
        const float dzHx = fsub(hxc, hxz), dxHz = fsub(hzc, h2p[1][k]);
        const float dxHy = fsub(hyc, h2p[0][k]), dyHx = fsub(hxc, hxy);
        const bool cy = iny[k], cz = inz && valid, cx = inx && valid;
        if (CPML && __any_sync(FULL, cy || cz || cx)) {
          const bool own = trow[k] && tlane;
          const int oyq = x2 * SY + oy[k], ozq = x2 * SZ + oz[k], oxq = imp * SX + ox[k];
          if (ux) {
            const float p1 = pnext(cy, ybe[k], yce[k], cy ? PSV(s2, PSI_EXY, k) : 0.f, dyHz);
            const float p2 = pnext(cz, zbe, zce, cz ? PSV(s2, PSI_EXZ, k) : 0.f, dzHy);
            if (own && cy) p.pml.out[PSI_EXY][oyq] = p1;
            if (own && cz) p.pml.out[PSI_EXZ][ozq] = p2;
            exv = e_sel<KAPPA>(exv, cb, dyHz, dzHy, cy, cz, p1, p2, yike[k], zike);
          }
          if (uy) {
            const float p1 = pnext(cz, zbe, zce, cz ? PSV(s2, PSI_EYZ, k) : 0.f, dzHx);
            const float p2 = pnext(cx, pbe, pce, cx ? PSV(s2, PSI_EYX, k) : 0.f, dxHz);
            if (own && cz) p.pml.out[PSI_EYZ][ozq] = p1;
            if (own && cx) p.pml.out[PSI_EYX][oxq] = p2;
            eyv = e_sel<KAPPA>(eyv, cb, dzHx, dxHz, cz, cx, p1, p2, zike, pike);
          }
          if (uz) {
            const float p1 = pnext(cx, pbe, pce, cx ? PSV(s2, PSI_EZX, k) : 0.f, dxHy);
            const float p2 = pnext(cy, ybe[k], yce[k], cy ? PSV(s2, PSI_EZY, k) : 0.f, dyHx);
            if (own && cx) p.pml.out[PSI_EZX][oxq] = p1;
            if (own && cy) p.pml.out[PSI_EZY][oyq] = p2;
            ezv = e_sel<KAPPA>(ezv, cb, dxHy, dyHx, cx, cy, p1, p2, pike, yike[k]);
          }
        } else {
          if (ux) exv = e_plain(exv, cb, dyHz, dzHy);
          if (uy) eyv = e_plain(eyv, cb, dzHx, dxHz);
          if (uz) ezv = e_plain(ezv, cb, dxHy, dyHx);
        }
        if (MODE == MODE_ABSORB && valid) {
          const float f = fmul(fmul(dxq, dyr[k]), dz);
          exv = fmul(exv, f);
          eyv = fmul(eyv, f);
          ezv = fmul(ezv, f);
        }
        eo[0][k] = exv;
        eo[1][k] = eyv;
        eo[2][k] = ezv;
      }
      // soft sources of step n+1 at plane x2 (tile cells)
      while (sp2 < se) {
        const TbSrc s = ex.src[sp2];
        if (s.x > x2) break;
        if (s.x == x2 && (s.lv & 2)) {
          const int rr = s.off >> 5, ll = s.off & 31;
          if (ll == lane && rr >= r0 && rr < r0 + RY) {
            const float v = fmul(s.amp, p.wave[(long long)s.wave * wl + p.step + 1]);
#pragma unroll
            for (int k = 0; k < RY; ++k)
              if (r0 + k == rr) {
                if (s.comp == 0) eo[0][k] = fadd(eo[0][k], v);
                else if (s.comp == 1) eo[1][k] = fadd(eo[1][k], v);
                else eo[2][k] = fadd(eo[2][k], v);
              }
          }
        }
        ++sp2;
      }
      if (tlane) {
#pragma unroll
        for (int k = 0; k < RY; ++k) {
          if (trow[k]) {
            const long long idx = ((long long)x2 * ny + yv[k]) * nz + z;
            p.out[0][idx] = eo[0][k];
            p.out[1][idx] = eo[1][k];
            p.out[2][idx] = eo[2][k];
            p.out[3][idx] = h2[0][k];
            p.out[4][idx] = h2[1][k];
            p.out[5][idx] = h2[2][k];
          }
        }
      }
    }

    // ---- rotate the march registers
#pragma unroll
    for (int k = 0; k < RY; ++k) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ec[c][k] = en[c][k];
        h1p[c][k] = h1[c][k];
        e1p[c][k] = e1[c][k];
      }
      h2p[0][k] = h2[1][k];
      h2p[1][k] = h2[2][k];
      cbp[k] = cbc[k];
    }
#undef ES
#undef ENS
#undef HS
  }
#undef PSV
#undef PSN
  if (L::RING) cp_async_wait_all();

  if (aborted) {
    // A staged copy never arrived.  Record it, then wait (bounded) for every
    // copy this block issued so none lands in shared memory after exit.
    if (tid == 0) {
      report_error(p.err, ERR_TIMEOUT_BASE | 2, bid, fail_l, issued);
      for (int l = consumed; l < issued; ++l)
        (void)mbar_wait_bounded(&bars[l % STAGES], (uint32_t)((l / STAGES) & 1), p.wait_ns);
    }
    __syncthreads();
  }
  if (p.pdl & PDL_WAIT_END) grid_dep_wait();
}

}  // namespace jxf
