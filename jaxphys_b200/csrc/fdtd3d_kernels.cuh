// 3D Yee leapfrog kernels for sm_100a.
//
// One time step of the reference's scan body (jaxphys src/neurosim/em/
// fdtd3d.py:280-379):
//   H^{n+1/2} = H^{n-1/2} - a * curl(E^n)                    (:303-330)
//   E^{n+1}   = (E^n + cb * curl(H^{n+1/2})) * damping + src  (:332-369)
// with a = dt/(mu0 dx), cb = dt/(eps0 dx eps_r), the reference's index ranges
// (H not updated on the last index of its differencing axes, E not updated on
// index 0), its separable damping exp(-sigma_avg dt/eps0) and soft sources.
//
// Two implementations:
//   * generic: one thread per cell, H kernel then E kernel, in place; handles
//     every boundary mode (periodic wrap included) and any shape.
//   * tma: the fast path.  A block owns a (TY x TZ) tile of the (y, z) plane
//     and marches along x over a chunk of planes.  E, H and cb planes of the
//     tile (+ halo) are staged into shared memory by TMA through a ring of
//     mbarrier-tracked stages; H^{n+1/2} is formed for the tile plus a one
//     cell low halo in y and z (recomputed, not exchanged), then E^{n+1}; the
//     H^{n+1/2} plane x-1 stays in registers.  Reads come from buffer set A
//     and results go to buffer set B (ping-pong), so recomputed halo values
//     never race with a neighbour's writes.  Fields cross HBM once per step:
//     read 6 components + cb, write 6.
#pragma once

#include "fdtd_common.cuh"

namespace jxf {

// ---------------------------------------------------------------------------
// shared arithmetic (identical bits in every kernel)
// ---------------------------------------------------------------------------

// H update without CPML: h - a*(d1 - d2)
__device__ __forceinline__ float h_plain(float h, float a, float d1, float d2) {
  return fsub(h, fmul(a, fsub(d1, d2)));
}
// E update without CPML: e + cb*(d1 - d2)
__device__ __forceinline__ float e_plain(float e, float cb, float d1, float d2) {
  return fadd(e, fmul(cb, fsub(d1, d2)));
}
// psi <- b*psi + c*d
__device__ __forceinline__ float psi_next(float b, float psi, float c, float d) {
  return fadd(fmul(b, psi), fmul(c, d));
}

__device__ __forceinline__ long long xs_index(int im, int y, int z, int ny, int nz) {
  return ((long long)im * ny + y) * nz + z;
}
__device__ __forceinline__ long long ys_index(int x, int jm, int z, int L1, int nz) {
  return ((long long)x * L1 + jm) * nz + z;
}
__device__ __forceinline__ long long zs_index(int x, int y, int km, int ny, int L2) {
  return ((long long)x * ny + y) * L2 + km;
}

template <bool B>
struct BoolC {
  static constexpr bool value = B;
};

// One CPML term of a field component: the derivative along one axis.
struct PsiTerm {
  bool on;     // cell inside this axis' slab (psi stored)
  float b, c;  // recurrence coefficients at the component's position
  float ik;    // 1/kappa at that position (1 outside the slab)
  float old;   // psi_in (valid when on)
  float* out;  // where to store the new psi, or nullptr
};

// curl' = (ik1 d1 - ik2 d2) + (psi1 - psi2), psi <- b psi + c d.
// Outside both slabs the component uses the plain update instead (same value:
// psi = 0 and ik = 1 there), so both kernels branch on the same condition.
template <bool KAPPA>
__device__ __forceinline__ float curl_cpml(float d1, float d2, const PsiTerm& t1,
                                           const PsiTerm& t2) {
  float p1 = 0.0f, p2 = 0.0f;
  if (t1.on) {
    p1 = psi_next(t1.b, t1.old, t1.c, d1);
    if (t1.out) *t1.out = p1;
  }
  if (t2.on) {
    p2 = psi_next(t2.b, t2.old, t2.c, d2);
    if (t2.out) *t2.out = p2;
  }
  const float u1 = KAPPA ? fmul(t1.ik, d1) : d1;
  const float u2 = KAPPA ? fmul(t2.ik, d2) : d2;
  return fadd(fsub(u1, u2), fsub(p1, p2));
}
template <bool KAPPA>
__device__ __forceinline__ float h_cpml(float h, float a, float d1, float d2, const PsiTerm& t1,
                                        const PsiTerm& t2) {
  if (!(t1.on || t2.on)) return h_plain(h, a, d1, d2);
  return fsub(h, fmul(a, curl_cpml<KAPPA>(d1, d2, t1, t2)));
}
template <bool KAPPA>
__device__ __forceinline__ float e_cpml(float e, float cb, float d1, float d2, const PsiTerm& t1,
                                        const PsiTerm& t2) {
  if (!(t1.on || t2.on)) return e_plain(e, cb, d1, d2);
  return fadd(e, fmul(cb, curl_cpml<KAPPA>(d1, d2, t1, t2)));
}

// Coefficients of one position on one axis (H: half-integer, E: integer).
struct AxisCoef {
  float bh, ch, ikh, be, ce, ike;
};
__device__ __forceinline__ AxisCoef axis_coef(const CpmlDev& P, int axis, int pos) {
  AxisCoef c;
  c.bh = __ldg(P.tab[axis][TAB_BH] + pos);
  c.ch = __ldg(P.tab[axis][TAB_CH] + pos);
  c.ikh = __ldg(P.tab[axis][TAB_IKH] + pos);
  c.be = __ldg(P.tab[axis][TAB_BE] + pos);
  c.ce = __ldg(P.tab[axis][TAB_CE] + pos);
  c.ike = __ldg(P.tab[axis][TAB_IKE] + pos);
  return c;
}
// Term with coefficients loaded only when the cell is in the slab.
__device__ __forceinline__ PsiTerm term_h_at(const CpmlDev& P, int axis, int pos, bool on,
                                             float old, float* out) {
  PsiTerm t{on, 0.0f, 0.0f, 1.0f, old, out};
  if (on) {
    t.b = __ldg(P.tab[axis][TAB_BH] + pos);
    t.c = __ldg(P.tab[axis][TAB_CH] + pos);
    t.ik = __ldg(P.tab[axis][TAB_IKH] + pos);
  }
  return t;
}
__device__ __forceinline__ PsiTerm term_e_at(const CpmlDev& P, int axis, int pos, bool on,
                                             float old, float* out) {
  PsiTerm t{on, 0.0f, 0.0f, 1.0f, old, out};
  if (on) {
    t.b = __ldg(P.tab[axis][TAB_BE] + pos);
    t.c = __ldg(P.tab[axis][TAB_CE] + pos);
    t.ik = __ldg(P.tab[axis][TAB_IKE] + pos);
  }
  return t;
}
__device__ __forceinline__ PsiTerm term_h(bool on, const AxisCoef& c, float old, float* out) {
  return PsiTerm{on, c.bh, c.ch, c.ikh, old, out};
}
__device__ __forceinline__ PsiTerm term_e(bool on, const AxisCoef& c, float old, float* out) {
  return PsiTerm{on, c.be, c.ce, c.ike, old, out};
}

// ---------------------------------------------------------------------------
// generic path
// ---------------------------------------------------------------------------

// psi term read/written in place in global memory (generic kernels)
__device__ __forceinline__ PsiTerm g_term(const CpmlDev& P, int id, bool on, float b, float c,
                                          float ik, long long idx) {
  return PsiTerm{on, b, c, ik, on ? P.out[id][idx] : 0.0f, on ? P.out[id] + idx : nullptr};
}

// Body of the generic H pass over the owned cells k0, k0+kstep, ...
template <int MODE>
__device__ __forceinline__ void generic_h_body(const Step3D& p, long long k0, long long kstep) {
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const long long plane = (long long)ny * nz;
  const long long n = (long long)(p.x_hi - p.x_lo) * plane;  // owned cells
  const long long base = (long long)p.x_lo * plane;
  const float a = p.a;
  const float* ex = p.in[0];
  const float* ey = p.in[1];
  const float* ez = p.in[2];
  for (long long k = k0; k < n; k += kstep) {
    const long long idx = base + k;
    int x, y, z;
    decode_cell(idx, nz, ny, p.idx32 != 0, p.div_nz, p.div_ny, x, y, z);
    const int xg = x + p.gx0;  // global plane
    long long ixp, iyp, izp;  // neighbours at +1
    bool ux, uy, uz;          // Hx, Hy, Hz updated here
    if (MODE == MODE_PERIODIC) {
      ixp = idx + (long long)((x + 1 == nx) ? -(nx - 1) : 1) * ny * nz;
      iyp = idx + (long long)((y + 1 == ny) ? -(ny - 1) : 1) * nz;
      izp = idx + ((z + 1 == nz) ? -(nz - 1) : 1);
      ux = uy = uz = true;
    } else {
      ixp = idx + (long long)ny * nz;
      iyp = idx + nz;
      izp = idx + 1;
      ux = (y < ny - 1) && (z < nz - 1);
      uy = (xg < p.gnx - 1) && (z < nz - 1);
      uz = (xg < p.gnx - 1) && (y < ny - 1);
    }
    const float exc = ex[idx], eyc = ey[idx], ezc = ez[idx];
    int im = -1, jm = -1, km = -1;
    AxisCoef cx{}, cy{}, cz{};
    if (MODE == MODE_CPML) {
      im = slab_map(xg, p.gnx, p.pml.P[0]);
      jm = slab_map(y, ny, p.pml.P[1]);
      km = slab_map(z, nz, p.pml.P[2]);
      cx = axis_coef(p.pml, 0, xg);
      cy = axis_coef(p.pml, 1, y);
      cz = axis_coef(p.pml, 2, z);
    }
    const long long ix = xs_index(im, y, z, ny, nz);
    const long long iy = ys_index(x, jm, z, p.pml.L[1], nz);
    const long long iz = zs_index(x, y, km, ny, p.pml.L[2]);
    if (ux) {
      const float d1 = fsub(ez[iyp], ezc), d2 = fsub(ey[izp], eyc);
      const float h = p.in[3][idx];
      p.out[3][idx] =
          MODE == MODE_CPML
              ? h_cpml<true>(h, a, d1, d2, g_term(p.pml, PSI_HXY, jm >= 0, cy.bh, cy.ch, cy.ikh, iy),
                             g_term(p.pml, PSI_HXZ, km >= 0, cz.bh, cz.ch, cz.ikh, iz))
              : h_plain(h, a, d1, d2);
    }
    if (uy) {
      const float d1 = fsub(ex[izp], exc), d2 = fsub(ez[ixp], ezc);
      const float h = p.in[4][idx];
      p.out[4][idx] =
          MODE == MODE_CPML
              ? h_cpml<true>(h, a, d1, d2, g_term(p.pml, PSI_HYZ, km >= 0, cz.bh, cz.ch, cz.ikh, iz),
                             g_term(p.pml, PSI_HYX, im >= 0, cx.bh, cx.ch, cx.ikh, ix))
              : h_plain(h, a, d1, d2);
    }
    if (uz) {
      const float d1 = fsub(ey[ixp], eyc), d2 = fsub(ex[iyp], exc);
      const float h = p.in[5][idx];
      p.out[5][idx] =
          MODE == MODE_CPML
              ? h_cpml<true>(h, a, d1, d2, g_term(p.pml, PSI_HZX, im >= 0, cx.bh, cx.ch, cx.ikh, ix),
                             g_term(p.pml, PSI_HZY, jm >= 0, cy.bh, cy.ch, cy.ikh, iy))
              : h_plain(h, a, d1, d2);
    }
  }
}

// Body of the generic E pass over the owned cells k0, k0+kstep, ...
template <int MODE>
__device__ __forceinline__ void generic_e_body(const Step3D& p, long long k0, long long kstep) {
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const long long plane = (long long)ny * nz;
  const long long n = (long long)(p.x_hi - p.x_lo) * plane;  // owned cells
  const long long base = (long long)p.x_lo * plane;
  const float* hx = p.out[3];  // H already advanced (in place)
  const float* hy = p.out[4];
  const float* hz = p.out[5];
  for (long long k = k0; k < n; k += kstep) {
    const long long idx = base + k;
    int x, y, z;
    decode_cell(idx, nz, ny, p.idx32 != 0, p.div_nz, p.div_ny, x, y, z);
    const int xg = x + p.gx0;  // global plane
    long long ixm, iym, izm;
    bool ux, uy, uz;
    if (MODE == MODE_PERIODIC) {
      ixm = idx - (long long)((x == 0) ? -(nx - 1) : 1) * ny * nz;
      iym = idx - (long long)((y == 0) ? -(ny - 1) : 1) * nz;
      izm = idx - ((z == 0) ? -(nz - 1) : 1);
      ux = uy = uz = true;
    } else {
      ixm = idx - (long long)ny * nz;
      iym = idx - nz;
      izm = idx - 1;
      ux = (y >= 1) && (z >= 1);
      uy = (xg >= 1) && (z >= 1);
      uz = (xg >= 1) && (y >= 1);
    }
    const float cb = p.cb ? p.cb[idx] : p.cb_const;
    const float hxc = hx[idx], hyc = hy[idx], hzc = hz[idx];
    float ex = p.in[0][idx], ey = p.in[1][idx], ez = p.in[2][idx];
    int im = -1, jm = -1, km = -1;
    AxisCoef cx{}, cy{}, cz{};
    if (MODE == MODE_CPML) {
      im = slab_map(xg, p.gnx, p.pml.P[0]);
      jm = slab_map(y, ny, p.pml.P[1]);
      km = slab_map(z, nz, p.pml.P[2]);
      cx = axis_coef(p.pml, 0, xg);
      cy = axis_coef(p.pml, 1, y);
      cz = axis_coef(p.pml, 2, z);
    }
    const long long ix = xs_index(im, y, z, ny, nz);
    const long long iy = ys_index(x, jm, z, p.pml.L[1], nz);
    const long long iz = zs_index(x, y, km, ny, p.pml.L[2]);
    if (ux) {
      const float d1 = fsub(hzc, hz[iym]), d2 = fsub(hyc, hy[izm]);
      ex = MODE == MODE_CPML
               ? e_cpml<true>(ex, cb, d1, d2, g_term(p.pml, PSI_EXY, jm >= 0, cy.be, cy.ce, cy.ike, iy),
                              g_term(p.pml, PSI_EXZ, km >= 0, cz.be, cz.ce, cz.ike, iz))
               : e_plain(ex, cb, d1, d2);
    }
    if (uy) {
      const float d1 = fsub(hxc, hx[izm]), d2 = fsub(hzc, hz[ixm]);
      ey = MODE == MODE_CPML
               ? e_cpml<true>(ey, cb, d1, d2, g_term(p.pml, PSI_EYZ, km >= 0, cz.be, cz.ce, cz.ike, iz),
                              g_term(p.pml, PSI_EYX, im >= 0, cx.be, cx.ce, cx.ike, ix))
               : e_plain(ey, cb, d1, d2);
    }
    if (uz) {
      const float d1 = fsub(hyc, hy[ixm]), d2 = fsub(hxc, hx[iym]);
      ez = MODE == MODE_CPML
               ? e_cpml<true>(ez, cb, d1, d2, g_term(p.pml, PSI_EZX, im >= 0, cx.be, cx.ce, cx.ike, ix),
                              g_term(p.pml, PSI_EZY, jm >= 0, cy.be, cy.ce, cy.ike, iy))
               : e_plain(ez, cb, d1, d2);
    }
    if (MODE == MODE_ABSORB) {
      const float f = fmul(fmul(__ldg(p.damp[0] + xg), __ldg(p.damp[1] + y)), __ldg(p.damp[2] + z));
      ex = fmul(ex, f);
      ey = fmul(ey, f);
      ez = fmul(ez, f);
    }
    p.out[0][idx] = ex;
    p.out[1][idx] = ey;
    p.out[2][idx] = ez;
  }
}

template <int MODE>
__global__ void __launch_bounds__(256) k3d_generic_h(const __grid_constant__ Step3D p) {
  generic_h_body<MODE>(p, (long long)blockIdx.x * blockDim.x + threadIdx.x,
                       (long long)gridDim.x * blockDim.x);
}
template <int MODE>
__global__ void __launch_bounds__(256) k3d_generic_e(const __grid_constant__ Step3D p) {
  generic_e_body<MODE>(p, (long long)blockIdx.x * blockDim.x + threadIdx.x,
                       (long long)gridDim.x * blockDim.x);
}

// Batched passes: many independent grids in one launch.  Block b works on
// grid blk_grid[b] (its blk_count[g] blocks start at blk_first[g]); each grid's
// parameters are read from global memory.
struct BatchBlocks {
  const Step3D* grids;
  const int* blk_grid;
  const int* blk_first;
  const int* blk_count;
};
template <int MODE>
__global__ void __launch_bounds__(256) k3d_batch_h(const __grid_constant__ BatchBlocks b) {
  const int g = b.blk_grid[blockIdx.x];
  generic_h_body<MODE>(b.grids[g],
                       (long long)(blockIdx.x - b.blk_first[g]) * blockDim.x + threadIdx.x,
                       (long long)b.blk_count[g] * blockDim.x);
}
template <int MODE>
__global__ void __launch_bounds__(256) k3d_batch_e(const __grid_constant__ BatchBlocks b) {
  const int g = b.blk_grid[blockIdx.x];
  generic_e_body<MODE>(b.grids[g],
                       (long long)(blockIdx.x - b.blk_first[g]) * blockDim.x + threadIdx.x,
                       (long long)b.blk_count[g] * blockDim.x);
}

// Soft sources, grouped by cell (list order within a cell), after the E update.
static __global__ void k3d_sources(float* ex, float* ey, float* ez, const SrcCell* cells, int n_cells,
                            const SrcTerm* terms, const float* wave, long long wave_len,
                            long long step) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_cells) return;
  const SrcCell c = cells[i];
  float* f = c.comp == 0 ? ex : (c.comp == 1 ? ey : ez);
  float v = f[c.cell];
  for (int k = 0; k < c.count; ++k) {
    const SrcTerm t = terms[c.first + k];
    v = fadd(v, fmul(t.amp, wave[(long long)t.wave * wave_len + step]));
  }
  f[c.cell] = v;
}

// Batched soft sources: one thread per (grid, source cell) entry.
struct BatchSrcGrid {
  float* e[3];
  const SrcCell* cells;
  const SrcTerm* terms;
  const float* wave;
  long long wave_len;
};
static __global__ void k3d_batch_sources(const BatchSrcGrid* grids, const int2* entries, int n,
                                  long long step) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int2 en = entries[i];
  const BatchSrcGrid& g = grids[en.x];
  const SrcCell c = g.cells[en.y];
  float* f = g.e[c.comp];
  float v = f[c.cell];
  for (int k = 0; k < c.count; ++k) {
    const SrcTerm t = g.terms[c.first + k];
    v = fadd(v, fmul(t.amp, g.wave[(long long)t.wave * g.wave_len + step]));
  }
  f[c.cell] = v;
}

// Batched probes: out[i] = grids[g_i].in[comp_i][cell_i] (state after the step)
struct BatchProbe {
  int grid, comp;
  long long cell;
};
static __global__ void k3d_batch_probes(const Step3D* grids, const BatchProbe* pr, int n, float* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const BatchProbe q = pr[i];
  out[i] = grids[q.grid].in[q.comp][q.cell];
}

struct FieldPtrs6 {
  const float* f[6];
};

// probe_out[i] = field[comp_i][cell_i]
static __global__ void k_probe_gather(FieldPtrs6 fp, const long long* cell, const int* comp, int n,
                               float* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = fp.f[comp[i]][cell[i]];
}

// ---------------------------------------------------------------------------
// TMA marching path
// ---------------------------------------------------------------------------

struct alignas(64) Maps3D {
  CUtensorMap e[3];  // box {TZ+8, TY+2, 1} at (z0-4, y0-1, x)
  CUtensorMap h[3];  // box {TZ+4, TY+1, 1} at (z0-4, y0-1, x)
  CUtensorMap cb;    // box {TZ, TY, 1}     at (z0,   y0,   x)
};

constexpr int round32(int v) { return (v + 31) / 32 * 32; }

// psi arrays by differencing axis (x: HYX HZX EYX EZX, y: HXY HZY EXY EZY,
// z: HXZ HYZ EXZ EYZ) and their slot in a block's psi ring when the block's
// cells touch only the slab axes in the bit set `axes` (1 = x, 2 = y, 4 = z):
// four slots per included axis; psi of excluded axes are never used.
__host__ __device__ constexpr int psi_axis(int id) {
  return (id == PSI_HYX || id == PSI_HZX || id == PSI_EYX || id == PSI_EZX)   ? 0
         : (id == PSI_HXY || id == PSI_HZY || id == PSI_EXY || id == PSI_EZY) ? 1
                                                                              : 2;
}
__host__ __device__ constexpr int psi_within(int id) {
  return (id == PSI_HYX || id == PSI_HXY || id == PSI_HXZ)   ? 0
         : (id == PSI_HZX || id == PSI_HZY || id == PSI_HYZ) ? 1
         : (id == PSI_EYX || id == PSI_EXY || id == PSI_EXZ) ? 2
                                                             : 3;
}
__host__ __device__ constexpr int psi_slot(int axes, int id) {
  return ((axes >> psi_axis(id)) & 1) == 0
             ? 0
             : 4 * (((axes & 1) && psi_axis(id) > 0 ? 1 : 0) +
                    ((axes & 2) && psi_axis(id) > 1 ? 1 : 0)) +
                   psi_within(id);
}
__host__ __device__ constexpr int psi_count(int axes) {
  return 4 * ((axes & 1 ? 1 : 0) + (axes & 2 ? 1 : 0) + (axes & 4 ? 1 : 0));
}

template <int TZ, int TY, int RY, int STAGES, bool CBARR, bool CPML, int AXES = 7>
struct TmaLayout {
  static constexpr int TYT = TY / RY;
  static constexpr int NT = TZ * TYT;
  static constexpr int EW = TZ + 8, EH = TY + 2;
  static constexpr int HW = TZ + 4, HH = TY + 1;
  static constexpr int NW = TZ + 1, NH = TY + 1;
  static constexpr int E_STRIDE = round32(EH * EW);
  static constexpr int H_STRIDE = round32(HH * HW);
  static constexpr int CB_STRIDE = CBARR ? round32(TY * TZ) : 0;
  static constexpr int STAGE_FLOATS = 3 * E_STRIDE + 3 * H_STRIDE + CB_STRIDE;
  static constexpr uint32_t STAGE_TX =
      (uint32_t)(3 * EH * EW + 3 * HH * HW + (CBARR ? TY * TZ : 0)) * 4u;
  static constexpr int HN_STRIDE = round32(NH * NW);
  // new-H plane buffers: two (one CTA barrier per plane) for one row per
  // thread; one (two barriers) for several rows per thread, whose larger
  // tiles would otherwise lose a resident block per SM to shared memory
  static constexpr int HNB = RY == 1 ? 2 : 1;
  // CPML: psi of the planes in flight, per thread: 12 core values per row and
  // 4 halo values, in a ring of PSB buffers (prefetch distance PSB-1 planes).
  static constexpr int PSB = 2;
  static constexpr int NPSI = psi_count(AXES);
  static constexpr int PSC_FLOATS = CPML ? PSB * NPSI * RY * NT : 0;
  static constexpr int PSH_FLOATS = CPML ? PSB * 4 * (TZ + TY) : 0;
  static constexpr size_t SMEM_BYTES =
      128 + sizeof(float) * ((size_t)STAGES * STAGE_FLOATS + 3 * HNB * (size_t)HN_STRIDE +
                             PSC_FLOATS + PSH_FLOATS);
  static_assert(TY % RY == 0, "rows per thread must divide the tile height");
  static_assert(TZ % 4 == 0, "tile width must keep TMA x coordinates 16-byte aligned");
  static_assert(STAGES >= 3 && STAGES <= 8, "ring needs >= 3 stages for one plane of lead");
  static_assert(NT <= 1024, "block too large");
  static_assert(TZ + TY <= NT, "halo pass needs TZ + TY threads");
  static_assert(SMEM_BYTES <= 227 * 1024, "shared memory per block exceeds 227 KB");
};

// CPML component update for a warp in which some lane is in a slab.  With
// kappa = 1 the CPML form alone serves every lane: a lane outside both slabs
// has p1 = p2 = 0 (pnext), and (d1 - d2) + 0 equals d1 - d2, so the result
// equals the plain update h - a (d1 - d2) of the generic kernel (which
// branches on the same condition) in value; only the sign of an exact zero
// can differ, which no later +, -, * turns into a different number.  With
// kappa > 1 the two values are formed and the plain one is selected (the
// same bits as the generic kernel).
template <bool KAPPA>
__device__ __forceinline__ float h_sel(float h, float a, float d1, float d2, bool on1, bool on2,
                                       float p1, float p2, float ik1, float ik2) {
  const float u1 = KAPPA ? fmul(ik1, d1) : d1;
  const float u2 = KAPPA ? fmul(ik2, d2) : d2;
  const float c = fsub(h, fmul(a, fadd(fsub(u1, u2), fsub(p1, p2))));
  if (!KAPPA) return c;
  return (on1 || on2) ? c : h_plain(h, a, d1, d2);
}
template <bool KAPPA>
__device__ __forceinline__ float e_sel(float e, float cb, float d1, float d2, bool on1, bool on2,
                                       float p1, float p2, float ik1, float ik2) {
  const float u1 = KAPPA ? fmul(ik1, d1) : d1;
  const float u2 = KAPPA ? fmul(ik2, d2) : d2;
  const float c = fadd(e, fmul(cb, fadd(fsub(u1, u2), fsub(p1, p2))));
  if (!KAPPA) return c;
  return (on1 || on2) ? c : e_plain(e, cb, d1, d2);
}
__device__ __forceinline__ float pnext(bool on, float b, float c, float old, float d) {
  return on ? psi_next(b, old, c, d) : 0.0f;
}

// Slab-first cell order of a CPML block (one row per thread): thread t takes
// the t-th cell of the tile counted over the cells that lie in a y or z psi
// slab first (y-slab rows whole, then the slab columns of the other rows,
// row by row), then over the rest.  A tile whose 32-wide warps each hold a
// few z-slab lanes (e.g. 11 of 32) would run every warp through the CPML
// update; in this order the slab cells fill the first warps and the other
// warps take the plain update.  The arithmetic of every cell is unchanged.
// useY / useZ: the block's kernel handles that axis's slab; P < 0 stores
// the whole axis.
template <int TZ, int TY>
__device__ __forceinline__ void slab_first_cell(int t, int z0, int y0, int nz, int ny, int P1,
                                                int P2, bool useY, bool useZ, int& tx, int& ty) {
  // CPML columns of a row outside the y slab: [0, c1) and [c2, cv)
  const int cv = min(TZ, nz - z0);
  int c1 = 0, c2 = cv;
  if (useZ) {
    if (P2 < 0) {
      c1 = cv;
    } else {
      c1 = min(max(P2 - z0, 0), cv);
      c2 = max(c1, min(max(nz - P2 - z0, 0), cv));
    }
  }
  const int ncz = c1 + (cv - c2);  // CPML cells of such a row
  const int gap = c2 - c1;         // its other cells: [c1, c2) then [cv, TZ)
  int k = t, nc = 0;
#pragma unroll
  for (int i = 0; i < TY; ++i) {
    const int y = y0 + i;
    const bool yin = useY && y < ny && (P1 < 0 || y < P1 || y >= ny - P1);
    nc += yin ? TZ : (y < ny ? ncz : 0);
  }
  const bool first = t < nc;
  if (!first) k = t - nc;
  tx = 0;
  ty = TY - 1;
  bool done = false;
#pragma unroll
  for (int i = 0; i < TY; ++i) {
    const int y = y0 + i;
    const bool valid = y < ny;
    const bool yin = useY && valid && (P1 < 0 || y < P1 || y >= ny - P1);
    const int cnt = first ? (yin ? TZ : (valid ? ncz : 0)) : (yin ? 0 : (valid ? TZ - ncz : TZ));
    if (!done && k < cnt) {
      ty = i;
      if (yin || !valid) tx = k;
      else if (first) tx = k < c1 ? k : c2 + (k - c1);
      else tx = k < gap ? c1 + k : cv + (k - gap);
      done = true;
    }
    if (!done) k -= cnt;
  }
}

// AXES (CPML only): the slab axes the block's cells may touch (1 = x, 2 = y,
// 4 = z); the code and psi storage of the other axes compile away.  The host
// launches single-axis variants for blocks that touch one slab axis only.
// One block of work: the tile (tzi, tyi) over x chunk ci.  Called by the
// single-grid kernel (one block per work item) and by the batch kernel (a
// persistent block looping over the items of many grids).
// WSRC: sources of a plane fetched by whole warps (single grids, where one
// block may hold a plane source); the persistent batch kernel keeps the
// per-entry loop, which measured faster there (its grids hold point sources).
template <int TZ, int TY, int RY, int STAGES, int MODE, bool CBARR, bool KAPPA, int AXES = 7,
          bool WSRC = true>
__device__ __forceinline__ void tma_block(const Step3D& p, const Maps3D& maps, int tzi, int tyi,
                                          int ci, bool slab_first, long long step) {
  constexpr bool CPML = (MODE == MODE_CPML);
  constexpr bool AX = (AXES & 1) != 0, AY = (AXES & 2) != 0, AZ = (AXES & 4) != 0;
  using L = TmaLayout<TZ, TY, RY, STAGES, CBARR, CPML, AXES>;
  constexpr int TYT = L::TYT;
  constexpr int NT = L::NT;
  constexpr int NH = TZ + TY;  // halo threads
  constexpr int EW = L::EW, HW = L::HW, NW = L::NW;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
  float* stages = reinterpret_cast<float*>(smem_raw + 128);
  // H of the current plane (tile + halo row / column).  With two buffers
  // (L::HNB == 2) they alternate by plane parity: plane l writes buffer l & 1
  // in its H phase and reads it in its E phase; plane l + 2 overwrites it only
  // after every thread has passed plane l + 1's barrier, i.e. finished plane
  // l's E phase, so a plane needs one CTA barrier (between its H and E
  // phases).  With one buffer a second barrier ends each plane.
  constexpr bool ONE_BARRIER = L::HNB == 2;
  float* HnB = stages + STAGES * L::STAGE_FLOATS;
  float* PSc = HnB + 3 * L::HNB * L::HN_STRIDE;
  float* PSh = PSc + L::PSC_FLOATS;

  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int tid = threadIdx.x;
  const int z0 = tzi * TZ;
  const int y0 = tyi * TY;
  int tx = tid % TZ;
  int ty = tid / TZ;
  if (CPML && RY == 1 && slab_first)
    slab_first_cell<TZ, TY>(tid, z0, y0, nz, ny, p.pml.P[1], p.pml.P[2], AY, AZ, tx, ty);
  // Planes marched: a whole grid marches over all of them.  An x-slab of a
  // decomposed grid marches over its owned planes [x_lo, x_hi) and the left
  // ghost plane before them, where H is recomputed as a bitwise replica of
  // the neighbour's last plane and E is not updated (the neighbour's E
  // arrives there before each step); on the first slab that ghost plane is
  // outside the grid and is skipped.  Boundaries, coefficient tables, x-slab
  // psi and damping use the global plane x + gx0.
  const int xbeg = p.gx0 < 0 ? 1 : 0;
  const int xb = xbeg + ci * p.x_chunk;
  const int xe = min(xb + p.x_chunk, p.x_hi);
  const int qs = xb > 0 ? xb - 1 : 0;  // first plane staged
  const int qe = min(xe, nx - 1);      // last plane staged
  const int nload = qe - qs + 1;
  const float a = p.a;
  const int z = z0 + tx;

  // Probes of the input state (= after the previous step).
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
      tma_load_3d(st + c * L::E_STRIDE, &maps.e[c], z0 - 4, y0 - 1, q, &bars[slot]);
#pragma unroll
    for (int c = 0; c < 3; ++c)
      tma_load_3d(st + 3 * L::E_STRIDE + c * L::H_STRIDE, &maps.h[c], z0 - 4, y0 - 1, q,
                  &bars[slot]);
    if (CBARR)
      tma_load_3d(st + 3 * L::E_STRIDE + 3 * L::H_STRIDE, &maps.cb, z0, y0, q, &bars[slot]);
  };
  if (tid == 0) {
    for (int l = 0; l < min(STAGES, nload); ++l) issue(l);
  }
  int issued = min(STAGES, nload);  // identical in every thread

  // ---- CPML per-thread state, fixed over the march along x.
  // psi offsets are 32-bit: plane stride * plane + in-plane offset.
  const int SY = CPML ? p.pml.L[1] * nz : 0;  // y-slab arrays: [nx][L1][nz]
  const int SZ = CPML ? ny * p.pml.L[2] : 0;  // z-slab arrays: [nx][ny][L2]
  const int SX = ny * nz;                     // x-slab arrays: [L0][ny][nz]
  bool iny[RY], inz = false;
  int oy[RY], oz[RY], ox[RY];
  float ybh[RY], ych[RY], ybe[RY], yce[RY], yikh[RY], yike[RY];
  float zbh = 1.f, zch = 0.f, zbe = 1.f, zce = 0.f, zikh = 1.f, zike = 1.f;
  // halo cell (row y0-1 for tid < TZ, column z0-1 for TZ <= tid < TZ+TY)
  int yh = -1, zh = -1;
  bool inyh = false, inzh = false;
  int oyh = 0, ozh = 0, oxh = 0;
  float hyb = 1.f, hyc = 0.f, hyik = 1.f, hzb = 1.f, hzc = 0.f, hzik = 1.f;
  if (CPML) {
    const int km = (z < nz) ? slab_map(z, nz, p.pml.P[2]) : -1;
    inz = AZ && km >= 0;
    if (z < nz) {
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
    for (int r = 0; r < RY; ++r) {
      const int y = y0 + ty + r * TYT;
      const bool valid = (y < ny) && (z < nz);
      const int jm = (y < ny) ? slab_map(y, ny, p.pml.P[1]) : -1;
      iny[r] = AY && valid && jm >= 0;
      oy[r] = jm * nz + z;
      oz[r] = y * p.pml.L[2] + km;
      ox[r] = y * nz + z;
      const int yc = y < ny ? y : ny - 1;
      ybh[r] = __ldg(p.pml.tab[1][TAB_BH] + yc);
      ych[r] = __ldg(p.pml.tab[1][TAB_CH] + yc);
      ybe[r] = __ldg(p.pml.tab[1][TAB_BE] + yc);
      yce[r] = __ldg(p.pml.tab[1][TAB_CE] + yc);
      yikh[r] = KAPPA ? __ldg(p.pml.tab[1][TAB_IKH] + yc) : 1.f;
      yike[r] = KAPPA ? __ldg(p.pml.tab[1][TAB_IKE] + yc) : 1.f;
    }
    if (tid < TZ) {
      if (y0 >= 1 && z0 + tid < nz) {
        yh = y0 - 1;
        zh = z0 + tid;
      }
    } else if (tid < NH) {
      if (z0 >= 1 && y0 + tid - TZ < ny) {
        yh = y0 + tid - TZ;
        zh = z0 - 1;
      }
    }
    if (yh >= 0) {
      const int jmh = slab_map(yh, ny, p.pml.P[1]);
      const int kmh = slab_map(zh, nz, p.pml.P[2]);
      inyh = AY && jmh >= 0;
      inzh = AZ && kmh >= 0;
      oyh = jmh * nz + zh;
      ozh = yh * p.pml.L[2] + kmh;
      oxh = yh * nz + zh;
      hyb = __ldg(p.pml.tab[1][TAB_BH] + yh);
      hyc = __ldg(p.pml.tab[1][TAB_CH] + yh);
      hzb = __ldg(p.pml.tab[2][TAB_BH] + zh);
      hzc = __ldg(p.pml.tab[2][TAB_CH] + zh);
      if (KAPPA) {
        hyik = __ldg(p.pml.tab[1][TAB_IKH] + yh);
        hzik = __ldg(p.pml.tab[2][TAB_IKH] + zh);
      }
    }
  } else {
#pragma unroll
    for (int r = 0; r < RY; ++r) {
      iny[r] = false;
      oy[r] = oz[r] = ox[r] = 0;
      ybh[r] = ych[r] = ybe[r] = yce[r] = yikh[r] = yike[r] = 0.f;
    }
  }
#define PSC(buf, id, r) PSc[(((buf) * L::NPSI + psi_slot(AXES, (id))) * RY + (r)) * NT + tid]
#define PSH(buf, k) PSh[((buf) * 4 + (k)) * NH + tid]
  // Prefetch psi_in of plane q into buffer `buf` (this thread's cells only).
  auto issue_psi = [&](int q, int buf) {
    const int imq = slab_map(q + p.gx0, p.gnx, p.pml.P[0]);
#pragma unroll
    for (int r = 0; r < RY; ++r) {
      if (iny[r]) {
        const int o = q * SY + oy[r];
        cp_async4(&PSC(buf, PSI_HXY, r), p.pml.in[PSI_HXY] + o);
        cp_async4(&PSC(buf, PSI_HZY, r), p.pml.in[PSI_HZY] + o);
        cp_async4(&PSC(buf, PSI_EXY, r), p.pml.in[PSI_EXY] + o);
        cp_async4(&PSC(buf, PSI_EZY, r), p.pml.in[PSI_EZY] + o);
      }
      const bool valid = (y0 + ty + r * TYT < ny) && (z < nz);
      if (inz && valid) {
        const int o = q * SZ + oz[r];
        cp_async4(&PSC(buf, PSI_HXZ, r), p.pml.in[PSI_HXZ] + o);
        cp_async4(&PSC(buf, PSI_HYZ, r), p.pml.in[PSI_HYZ] + o);
        cp_async4(&PSC(buf, PSI_EXZ, r), p.pml.in[PSI_EXZ] + o);
        cp_async4(&PSC(buf, PSI_EYZ, r), p.pml.in[PSI_EYZ] + o);
      }
      if (AX && imq >= 0 && valid) {
        const int o = imq * SX + ox[r];
        cp_async4(&PSC(buf, PSI_HYX, r), p.pml.in[PSI_HYX] + o);
        cp_async4(&PSC(buf, PSI_HZX, r), p.pml.in[PSI_HZX] + o);
        cp_async4(&PSC(buf, PSI_EYX, r), p.pml.in[PSI_EYX] + o);
        cp_async4(&PSC(buf, PSI_EZX, r), p.pml.in[PSI_EZX] + o);
      }
    }
    if (yh >= 0) {
      if (inyh) cp_async4(&PSH(buf, 0), p.pml.in[PSI_HXY] + q * SY + oyh);
      if (inzh) cp_async4(&PSH(buf, 1), p.pml.in[PSI_HXZ] + q * SZ + ozh);
      if (tid < TZ) {  // row halo: Hz needs hzx, hzy
        if (AX && imq >= 0) cp_async4(&PSH(buf, 2), p.pml.in[PSI_HZX] + imq * SX + oxh);
        if (inyh) cp_async4(&PSH(buf, 3), p.pml.in[PSI_HZY] + q * SY + oyh);
      } else {  // column halo: Hy needs hyz, hyx
        if (inzh) cp_async4(&PSH(buf, 2), p.pml.in[PSI_HYZ] + q * SZ + ozh);
        if (AX && imq >= 0) cp_async4(&PSH(buf, 3), p.pml.in[PSI_HYX] + imq * SX + oxh);
      }
    }
    cp_async_commit();
  };
  constexpr int PSB = L::PSB;
  if (CPML) {
#pragma unroll
    for (int k = 0; k < PSB - 1; ++k) {
      if (qs + k < xe) issue_psi(qs + k, k);
      else cp_async_commit();
    }
  }

  // source list of this block
  const int bid = (ci * p.ntiles_y + tyi) * p.ntiles_z + tzi;
  int sp = 0, se = 0;
  if (p.blk_src_ptr != nullptr) {
    sp = p.blk_src_ptr[bid];
    se = p.blk_src_ptr[bid + 1];
  }

  float hy_prev[RY], hz_prev[RY];
#pragma unroll
  for (int r = 0; r < RY; ++r) hy_prev[r] = hz_prev[r] = 0.0f;

  const int zz = tx + 4;  // column in E / H stage boxes
  const int zn = tx + 1;  // column in Hn
  int consumed = 0;       // planes fully consumed (slots released)
  int fail_l = -1;        // plane index whose wait gave up (diagnostics)
  bool aborted = false;

  for (int x = qs; x < xe; ++x) {
    const int l = x - qs;
    const int pb = l % PSB;  // psi buffer of this plane
    if (CPML) {
      if (x + PSB - 1 < xe) issue_psi(x + PSB - 1, (l + PSB - 1) % PSB);
      else cp_async_commit();            // empty group keeps the count uniform
      cp_async_wait_pending<PSB - 1>();  // this plane's psi has landed (own copies)
    }
    const int slot = l % STAGES;
    const bool have_next = (x + 1 <= qe);
    bool ok = mbar_wait_bounded(&bars[slot], (uint32_t)((l / STAGES) & 1), p.wait_ns);
    if (have_next)
      ok = ok && mbar_wait_bounded(&bars[(l + 1) % STAGES], (uint32_t)(((l + 1) / STAGES) & 1),
                                   p.wait_ns);
    if (!ok) fail_l = l;
    const float* Es = stages + slot * L::STAGE_FLOATS;
    const float* En = stages + ((l + 1) % STAGES) * L::STAGE_FLOATS;
    const float* Hs = Es + 3 * L::E_STRIDE;
    const float* CBs = Hs + 3 * L::H_STRIDE;
    float* const Hn = HnB + (ONE_BARRIER ? (l & 1) : 0) * 3 * L::HN_STRIDE;
#define E_AT(c, yy, zc) Es[(c) * L::E_STRIDE + (yy) * EW + (zc)]
#define EN_AT(c, yy, zc) En[(c) * L::E_STRIDE + (yy) * EW + (zc)]
#define H_AT(c, yy, zc) Hs[(c) * L::H_STRIDE + (yy) * HW + (zc)]
#define HN_AT(c, yy, zc) Hn[(c) * L::HN_STRIDE + (yy) * NW + (zc)]
    const bool warm = (x < xb);
    const int xg = x + p.gx0;  // global plane
    int imx = -1;
    float xbh = 1.f, xch = 0.f, xbe = 1.f, xce = 0.f, xikh = 1.f, xike = 1.f;
    if (CPML) {
      imx = AX ? slab_map(xg, p.gnx, p.pml.P[0]) : -1;
      if (imx >= 0) {
        xbh = __ldg(p.pml.tab[0][TAB_BH] + xg);
        xch = __ldg(p.pml.tab[0][TAB_CH] + xg);
        xbe = __ldg(p.pml.tab[0][TAB_BE] + xg);
        xce = __ldg(p.pml.tab[0][TAB_CE] + xg);
        if (KAPPA) {
          xikh = __ldg(p.pml.tab[0][TAB_IKH] + xg);
          xike = __ldg(p.pml.tab[0][TAB_IKE] + xg);
        }
      }
    }
    const bool inx = imx >= 0;


    // ---------------- H^{n+1/2} on the tile (registers + Hn) ----------------
    float exr[RY], eyr[RY], ezr[RY], hxr[RY], hyr[RY], hzr[RY], cbr[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) {
      const int yl = ty + r * TYT;
      const int y = y0 + yl;
      // Cb is read here, with the rest of the stage: after this plane's
      // barrier the stage slot is refilled
      cbr[r] = CBARR ? CBs[yl * TZ + tx] : p.cb_const;
      const int yy = yl + 1;
      const bool valid = (y < ny) && (z < nz);
      const bool own = !warm && valid;
      const float exc = E_AT(0, yy, zz), eyc = E_AT(1, yy, zz), ezc = E_AT(2, yy, zz);
      exr[r] = exc;
      eyr[r] = eyc;
      ezr[r] = ezc;
      float hx = H_AT(0, yy, zz), hy = H_AT(1, yy, zz), hz = H_AT(2, yy, zz);
      const bool ux = !warm && y < ny - 1 && z < nz - 1;
      const bool uy = xg < p.gnx - 1 && z < nz - 1 && y < ny;
      const bool uz = xg < p.gnx - 1 && y < ny - 1 && z < nz;
      const float dyEz = fsub(E_AT(2, yy + 1, zz), ezc), dzEy = fsub(E_AT(1, yy, zz + 1), eyc);
      const float dzEx = fsub(E_AT(0, yy, zz + 1), exc), dxEz = fsub(EN_AT(2, yy, zz), ezc);
      const float dxEy = fsub(EN_AT(1, yy, zz), eyc), dyEx = fsub(E_AT(0, yy + 1, zz), exc);
      const bool cinz = inz && valid, cinx = inx && valid;
      if (CPML && __any_sync(0xffffffffu, iny[r] || cinz || cinx)) {
        const int oyq = x * SY + oy[r], ozq = x * SZ + oz[r], oxq = imx * SX + ox[r];
        if (ux) {
          const float p1 = pnext(iny[r], ybh[r], ych[r], PSC(pb, PSI_HXY, r), dyEz);
          const float p2 = pnext(cinz, zbh, zch, PSC(pb, PSI_HXZ, r), dzEy);
          if (own && iny[r]) p.pml.out[PSI_HXY][oyq] = p1;
          if (own && cinz) p.pml.out[PSI_HXZ][ozq] = p2;
          hx = h_sel<KAPPA>(hx, a, dyEz, dzEy, iny[r], cinz, p1, p2, yikh[r], zikh);
        }
        if (uy) {
          const float p1 = pnext(cinz, zbh, zch, PSC(pb, PSI_HYZ, r), dzEx);
          const float p2 = pnext(cinx, xbh, xch, PSC(pb, PSI_HYX, r), dxEz);
          if (own && cinz) p.pml.out[PSI_HYZ][ozq] = p1;
          if (own && cinx) p.pml.out[PSI_HYX][oxq] = p2;
          hy = h_sel<KAPPA>(hy, a, dzEx, dxEz, cinz, cinx, p1, p2, zikh, xikh);
        }
        if (uz) {
          const float p1 = pnext(cinx, xbh, xch, PSC(pb, PSI_HZX, r), dxEy);
          const float p2 = pnext(iny[r], ybh[r], ych[r], PSC(pb, PSI_HZY, r), dyEx);
          if (own && cinx) p.pml.out[PSI_HZX][oxq] = p1;
          if (own && iny[r]) p.pml.out[PSI_HZY][oyq] = p2;
          hz = h_sel<KAPPA>(hz, a, dxEy, dyEx, cinx, iny[r], p1, p2, xikh, yikh[r]);
        }
      } else {
        if (ux) hx = h_plain(hx, a, dyEz, dzEy);
        if (uy) hy = h_plain(hy, a, dzEx, dxEz);
        if (uz) hz = h_plain(hz, a, dxEy, dyEx);
      }
      hxr[r] = hx;
      hyr[r] = hy;
      hzr[r] = hz;
      if (!warm) {
        HN_AT(0, yy, zn) = hx;
        HN_AT(1, yy, zn) = hy;
        HN_AT(2, yy, zn) = hz;
      }
    }

    // ---------------- halo H: row y0-1 (Hx, Hz) and column z0-1 (Hx, Hy) ------
    // recomputed from the staged E (the owner block writes these cells)
    if (!warm && tid < NH) {
      if (tid < TZ) {
        const int y = y0 - 1;
        const int zc = z0 + tid;
        const int zb = tid + 4;
        float hx = H_AT(0, 0, zb), hz = H_AT(2, 0, zb);
        if (y >= 0 && zc < nz) {
          const float ezc = E_AT(2, 0, zb), eyc = E_AT(1, 0, zb), exc = E_AT(0, 0, zb);
          if (zc < nz - 1) {  // y < ny-1 holds: y0 < ny
            const float d1 = fsub(E_AT(2, 1, zb), ezc), d2 = fsub(E_AT(1, 0, zb + 1), eyc);
            if (CPML)
              hx = h_sel<KAPPA>(hx, a, d1, d2, inyh, inzh, pnext(inyh, hyb, hyc, PSH(pb, 0), d1),
                                pnext(inzh, hzb, hzc, PSH(pb, 1), d2), hyik, hzik);
            else
              hx = h_plain(hx, a, d1, d2);
          }
          if (xg < p.gnx - 1) {
            const float d1 = fsub(EN_AT(1, 0, zb), eyc), d2 = fsub(E_AT(0, 1, zb), exc);
            if (CPML)
              hz = h_sel<KAPPA>(hz, a, d1, d2, inx, inyh, pnext(inx, xbh, xch, PSH(pb, 2), d1),
                                pnext(inyh, hyb, hyc, PSH(pb, 3), d2), xikh, hyik);
            else
              hz = h_plain(hz, a, d1, d2);
          }
        }
        HN_AT(0, 0, tid + 1) = hx;
        HN_AT(2, 0, tid + 1) = hz;
      } else {
        const int yl = tid - TZ;
        const int y = y0 + yl;
        const int zc = z0 - 1;
        const int yy = yl + 1;
        float hx = H_AT(0, yy, 3), hy = H_AT(1, yy, 3);
        if (zc >= 0 && y < ny) {
          const float ezc = E_AT(2, yy, 3), eyc = E_AT(1, yy, 3), exc = E_AT(0, yy, 3);
          if (y < ny - 1) {  // zc < nz-1 holds: z0 < nz
            const float d1 = fsub(E_AT(2, yy + 1, 3), ezc), d2 = fsub(E_AT(1, yy, 4), eyc);
            if (CPML)
              hx = h_sel<KAPPA>(hx, a, d1, d2, inyh, inzh, pnext(inyh, hyb, hyc, PSH(pb, 0), d1),
                                pnext(inzh, hzb, hzc, PSH(pb, 1), d2), hyik, hzik);
            else
              hx = h_plain(hx, a, d1, d2);
          }
          if (xg < p.gnx - 1) {
            const float d1 = fsub(E_AT(0, yy, 4), exc), d2 = fsub(EN_AT(2, yy, 3), ezc);
            if (CPML)
              hy = h_sel<KAPPA>(hy, a, d1, d2, inzh, inx, pnext(inzh, hzb, hzc, PSH(pb, 2), d1),
                                pnext(inx, xbh, xch, PSH(pb, 3), d2), hzik, xikh);
            else
              hy = h_plain(hy, a, d1, d2);
          }
        }
        HN_AT(0, yy, 0) = hx;
        HN_AT(1, yy, 0) = hy;
      }
    }

    if (__syncthreads_or(ok ? 0 : 1)) {
      aborted = true;
      break;
    }
    // Every thread is done with stage `slot` (this H phase and the previous
    // plane's read it; Cb came along above): refill it now.
    if (ONE_BARRIER) {
      consumed = l + 1;
      if (issued < nload && issued < consumed + STAGES) {
        if (tid == 0) issue(issued);
        ++issued;
      }
    }

    if (!warm) {
      // ---------------- E^{n+1} on the tile ----------------
      float exo[RY], eyo[RY], ezo[RY];
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        const int yl = ty + r * TYT;
        const int y = y0 + yl;
        const int yy = yl + 1;
        const bool own = (y < ny) && (z < nz);
        float ex = exr[r], ey = eyr[r], ez = ezr[r];
        const float hxc = hxr[r], hyc = hyr[r], hzc = hzr[r];
        const float cb = cbr[r];
        // E is not updated on a ghost plane (x < x_lo): it keeps its input
        const bool ep = x >= p.x_lo;
        const bool ux = ep && y >= 1 && z >= 1, uy = ep && xg >= 1 && z >= 1,
                   uz = ep && xg >= 1 && y >= 1;
        const float dyHz = fsub(hzc, HN_AT(2, yy - 1, zn)), dzHy = fsub(hyc, HN_AT(1, yy, zn - 1));
        const float dzHx = fsub(hxc, HN_AT(0, yy, zn - 1)), dxHz = fsub(hzc, hz_prev[r]);
        const float dxHy = fsub(hyc, hy_prev[r]), dyHx = fsub(hxc, HN_AT(0, yy - 1, zn));
        const bool cinz = inz && own, cinx = inx && own;
        if (CPML && __any_sync(0xffffffffu, iny[r] || cinz || cinx)) {
          const int oyq = x * SY + oy[r], ozq = x * SZ + oz[r], oxq = imx * SX + ox[r];
          if (ux) {
            const float p1 = pnext(iny[r], ybe[r], yce[r], PSC(pb, PSI_EXY, r), dyHz);
            const float p2 = pnext(cinz, zbe, zce, PSC(pb, PSI_EXZ, r), dzHy);
            if (iny[r]) p.pml.out[PSI_EXY][oyq] = p1;
            if (cinz) p.pml.out[PSI_EXZ][ozq] = p2;
            ex = e_sel<KAPPA>(ex, cb, dyHz, dzHy, iny[r], cinz, p1, p2, yike[r], zike);
          }
          if (uy) {
            const float p1 = pnext(cinz, zbe, zce, PSC(pb, PSI_EYZ, r), dzHx);
            const float p2 = pnext(cinx, xbe, xce, PSC(pb, PSI_EYX, r), dxHz);
            if (cinz) p.pml.out[PSI_EYZ][ozq] = p1;
            if (cinx) p.pml.out[PSI_EYX][oxq] = p2;
            ey = e_sel<KAPPA>(ey, cb, dzHx, dxHz, cinz, cinx, p1, p2, zike, xike);
          }
          if (uz) {
            const float p1 = pnext(cinx, xbe, xce, PSC(pb, PSI_EZX, r), dxHy);
            const float p2 = pnext(iny[r], ybe[r], yce[r], PSC(pb, PSI_EZY, r), dyHx);
            if (cinx) p.pml.out[PSI_EZX][oxq] = p1;
            if (iny[r]) p.pml.out[PSI_EZY][oyq] = p2;
            ez = e_sel<KAPPA>(ez, cb, dxHy, dyHx, cinx, iny[r], p1, p2, xike, yike[r]);
          }
        } else {
          if (ux) ex = e_plain(ex, cb, dyHz, dzHy);
          if (uy) ey = e_plain(ey, cb, dzHx, dxHz);
          if (uz) ez = e_plain(ez, cb, dxHy, dyHx);
        }
        if (MODE == MODE_ABSORB && own && ep) {
          const float f =
              fmul(fmul(__ldg(p.damp[0] + xg), __ldg(p.damp[1] + y)), __ldg(p.damp[2] + z));
          ex = fmul(ex, f);
          ey = fmul(ey, f);
          ez = fmul(ez, f);
        }
        exo[r] = ex;
        eyo[r] = ey;
        ezo[r] = ez;
      }
      // soft sources of plane x, in list order; a thread adds the entries of
      // its own cell
      auto add_src = [&](int off, int comp, float v) {
        const int yl_e = off / TZ;
        const int tz_e = off - yl_e * TZ;
        if (tz_e == tx && (yl_e % TYT) == ty) {
          const int r_e = yl_e / TYT;
#pragma unroll
          for (int r = 0; r < RY; ++r) {
            if (r == r_e) {
              if (comp == 0) exo[r] = fadd(exo[r], v);
              else if (comp == 1) eyo[r] = fadd(eyo[r], v);
              else ezo[r] = fadd(ezo[r], v);
            }
          }
        }
      };
      // The block's entries are sorted by plane and those of plane x come
      // first: lane k of every warp loads entry sp + k with its waveform
      // sample (two round trips per 32 entries instead of two per entry) and
      // the warp walks them in list order through shuffles.  sp < se is the
      // same in every thread of the block.
      while (WSRC && sp < se) {
        const int k = sp + (tid & 31);
        bool here = false;
        int s_off = 0, s_comp = 0;
        float s_v = 0.0f;
        if (k < se) {
          const SrcEntry e = p.src[k];
          here = e.x == x;
          if (here) {
            s_off = e.off;
            s_comp = e.comp;
            s_v = fmul(e.amp, p.wave[(long long)e.wave * p.wave_len + step]);
          }
        }
        const int s_n = __popc(__ballot_sync(0xffffffffu, here));  // lanes 0 .. s_n-1
        for (int j = 0; j < s_n; ++j)
          add_src(__shfl_sync(0xffffffffu, s_off, j), __shfl_sync(0xffffffffu, s_comp, j),
                  __shfl_sync(0xffffffffu, s_v, j));
        sp += s_n;
        if (s_n < 32) break;
      }
      while (!WSRC && sp < se) {  // one entry at a time
        const SrcEntry e = p.src[sp];
        if (e.x != x) break;
        add_src(e.off, e.comp, fmul(e.amp, p.wave[(long long)e.wave * p.wave_len + step]));
        ++sp;
      }
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        const int y = y0 + ty + r * TYT;
        if (y < ny && z < nz) {
          const long long idx = ((long long)x * ny + y) * nz + z;
          p.out[0][idx] = exo[r];
          p.out[1][idx] = eyo[r];
          p.out[2][idx] = ezo[r];
          p.out[3][idx] = hxr[r];
          p.out[4][idx] = hyr[r];
          p.out[5][idx] = hzr[r];
        }
      }
    }
#pragma unroll
    for (int r = 0; r < RY; ++r) {
      hy_prev[r] = hyr[r];
      hz_prev[r] = hzr[r];
    }
#undef E_AT
#undef EN_AT
#undef H_AT
#undef HN_AT
    if (!ONE_BARRIER) {
      __syncthreads();  // the H plane and stage `slot` are free again
      consumed = l + 1;
      if (issued < nload && issued < consumed + STAGES) {
        if (tid == 0) issue(issued);
        ++issued;
      }
    }
  }
#undef PSC
#undef PSH
  if (CPML) cp_async_wait_all();

  if (aborted) {
    // A staged copy never arrived.  Record it, then wait (bounded) for every
    // copy this block issued so none lands in shared memory after exit.
    if (tid == 0) {
      report_error(p.err, ERR_TIMEOUT_BASE | 1, bid, fail_l, issued);
      for (int l = consumed; l < issued; ++l)
        (void)mbar_wait_bounded(&bars[l % STAGES], (uint32_t)((l / STAGES) & 1), p.wait_ns);
    }
    __syncthreads();
  }
}

template <int TZ, int TY, int RY, int STAGES, int MODE, bool CBARR, bool KAPPA, int AXES = 7>
__global__ void __launch_bounds__(TZ*(TY / RY))
    k3d_tma(const __grid_constant__ Step3D p, const __grid_constant__ Maps3D maps) {
  int tzi = blockIdx.x, tyi = blockIdx.y, ci = blockIdx.z;
  bool slab_first = false;
  if (p.blk_list != nullptr) {
    tzi = p.blk_list[3 * blockIdx.x];
    tyi = p.blk_list[3 * blockIdx.x + 1];
    const int v = p.blk_list[3 * blockIdx.x + 2];
    ci = v & BLK_CHUNK_MASK;
    slab_first = (v & BLK_SLAB_FIRST) != 0;
  }
  // Programmatic dependent launch: a step kernel waits for the previous
  // step's grids before touching its inputs and then lets the next launch be
  // scheduled; the plain interior kernel of a CPML step overlaps the shell
  // kernel it depends on and only waits for it before exiting (so the next
  // step, which waits on the interior kernel, also sees the shell's writes).
  if (p.pdl & PDL_WAIT_START) grid_dep_wait();
  if (p.pdl & PDL_TRIGGER) grid_dep_launch_dependents();
  tma_block<TZ, TY, RY, STAGES, MODE, CBARR, KAPPA, AXES>(p, maps, tzi, tyi, ci, slab_first,
                                                          p.step);
  if (p.pdl & PDL_WAIT_END) grid_dep_wait();
}

// Batches of grids on the TMA kernel: one persistent launch per step (and per
// CPML part) over a work list of (grid, tile, chunk) items of every grid,
// heaviest first.  Blocks take items through an atomic counter; the last
// block to finish resets the counter for the next launch (which reads it only
// after its programmatic-dependent-launch wait, i.e. after this grid is done).
struct TmaBatchArgs {
  const Step3D* params;  // [2][n_grids]: parameters with input set 0 / 1
  const Maps3D* maps;    // [2][n_grids]
  int n_grids;
  int in_set;            // input set of this step (one parity for the batch)
  const int4* items;     // (grid, tile_z, tile_y, chunk word)
  int n_items;
  int* counter;          // [0] next item, [1] blocks done
  int pdl;
  long long step;        // step index of the batch (waveform sample of the sources)
};

__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// the tensor maps live in global memory (written by the host before launch)
__device__ __forceinline__ void tensormap_acquire(const void* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(
                   reinterpret_cast<uint64_t>(map))
               : "memory");
}

template <int TZ, int TY, int RY, int STAGES, int MODE, bool CBARR, bool KAPPA, int AXES = 7>
__global__ void __launch_bounds__(TZ*(TY / RY))
    k3d_tma_batch(const __grid_constant__ TmaBatchArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
  __shared__ int s_item;
  if (a.pdl & PDL_WAIT_START) grid_dep_wait();
  if (a.pdl & PDL_TRIGGER) grid_dep_launch_dependents();
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(&a.counter[0], 1);
    __syncthreads();
    const int it = s_item;
    if (it >= a.n_items) break;
    const int4 w = a.items[it];
    const int k = a.in_set * a.n_grids + w.x;
    const Maps3D& m = a.maps[k];
    if (threadIdx.x == 0) {
      for (int c = 0; c < 3; ++c) {
        tensormap_acquire(&m.e[c]);
        tensormap_acquire(&m.h[c]);
      }
      if (CBARR) tensormap_acquire(&m.cb);
    }
    tma_block<TZ, TY, RY, STAGES, MODE, CBARR, KAPPA, AXES, false>(
        a.params[k], m, w.y, w.z, w.w & BLK_CHUNK_MASK, (w.w & BLK_SLAB_FIRST) != 0, a.step);
    __syncthreads();  // every wait of the item is over
    if (threadIdx.x == 0)
      for (int s = 0; s < STAGES; ++s) mbar_inval(&bars[s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&a.counter[1], 1) == (int)gridDim.x - 1) {
      a.counter[0] = 0;
      a.counter[1] = 0;
      __threadfence();
    }
  }
  if (a.pdl & PDL_WAIT_END) grid_dep_wait();
}

}  // namespace jxf
