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

template <int MODE>
__global__ void __launch_bounds__(256) k3d_generic_h(const __grid_constant__ Step3D p) {
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const long long n = (long long)nx * ny * nz;
  const float a = p.a;
  const float* ex = p.in[0];
  const float* ey = p.in[1];
  const float* ez = p.in[2];
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(idx % nz);
    const long long t = idx / nz;
    const int y = (int)(t % ny);
    const int x = (int)(t / ny);
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
      uy = (x < nx - 1) && (z < nz - 1);
      uz = (x < nx - 1) && (y < ny - 1);
    }
    const float exc = ex[idx], eyc = ey[idx], ezc = ez[idx];
    int im = -1, jm = -1, km = -1;
    AxisCoef cx{}, cy{}, cz{};
    if (MODE == MODE_CPML) {
      im = slab_map(x, nx, p.pml.P[0]);
      jm = slab_map(y, ny, p.pml.P[1]);
      km = slab_map(z, nz, p.pml.P[2]);
      cx = axis_coef(p.pml, 0, x);
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

template <int MODE>
__global__ void __launch_bounds__(256) k3d_generic_e(const __grid_constant__ Step3D p) {
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const long long n = (long long)nx * ny * nz;
  const float* hx = p.out[3];  // H already advanced (in place)
  const float* hy = p.out[4];
  const float* hz = p.out[5];
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(idx % nz);
    const long long t = idx / nz;
    const int y = (int)(t % ny);
    const int x = (int)(t / ny);
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
      uy = (x >= 1) && (z >= 1);
      uz = (x >= 1) && (y >= 1);
    }
    const float cb = p.cb ? p.cb[idx] : p.cb_const;
    const float hxc = hx[idx], hyc = hy[idx], hzc = hz[idx];
    float ex = p.in[0][idx], ey = p.in[1][idx], ez = p.in[2][idx];
    int im = -1, jm = -1, km = -1;
    AxisCoef cx{}, cy{}, cz{};
    if (MODE == MODE_CPML) {
      im = slab_map(x, nx, p.pml.P[0]);
      jm = slab_map(y, ny, p.pml.P[1]);
      km = slab_map(z, nz, p.pml.P[2]);
      cx = axis_coef(p.pml, 0, x);
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
      const float f = fmul(fmul(__ldg(p.damp[0] + x), __ldg(p.damp[1] + y)), __ldg(p.damp[2] + z));
      ex = fmul(ex, f);
      ey = fmul(ey, f);
      ez = fmul(ez, f);
    }
    p.out[0][idx] = ex;
    p.out[1][idx] = ey;
    p.out[2][idx] = ez;
  }
}

// Soft sources, grouped by cell (list order within a cell), after the E update.
__global__ void k3d_sources(float* ex, float* ey, float* ez, const SrcCell* cells, int n_cells,
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

struct FieldPtrs6 {
  const float* f[6];
};

// probe_out[i] = field[comp_i][cell_i]
__global__ void k_probe_gather(FieldPtrs6 fp, const long long* cell, const int* comp, int n,
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

template <int TZ, int TY, int RY, int STAGES, bool CBARR, bool CPML>
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
  // CPML: psi of the current and next plane, per thread: 12 core values per
  // row and 4 halo values (double buffered).
  static constexpr int PSC_FLOATS = CPML ? 2 * PSI_COUNT * RY * NT : 0;
  static constexpr int PSH_FLOATS = CPML ? 2 * 4 * (TZ + TY) : 0;
  static constexpr size_t SMEM_BYTES =
      128 + sizeof(float) * ((size_t)STAGES * STAGE_FLOATS + 3 * (size_t)HN_STRIDE +
                             PSC_FLOATS + PSH_FLOATS);
  static_assert(TY % RY == 0, "rows per thread must divide the tile height");
  static_assert(TZ % 4 == 0, "tile width must keep TMA x coordinates 16-byte aligned");
  static_assert(STAGES >= 3 && STAGES <= 8, "ring needs >= 3 stages for one plane of lead");
  static_assert(NT <= 1024, "block too large");
  static_assert(TZ + TY <= NT, "halo pass needs TZ + TY threads");
  static_assert(SMEM_BYTES <= 227 * 1024, "shared memory per block exceeds 227 KB");
};

template <int TZ, int TY, int RY, int STAGES, int MODE, bool CBARR, bool KAPPA>
__global__ void __launch_bounds__(TZ*(TY / RY))
    k3d_tma(const __grid_constant__ Step3D p, const __grid_constant__ Maps3D maps) {
  constexpr bool CPML = (MODE == MODE_CPML);
  using L = TmaLayout<TZ, TY, RY, STAGES, CBARR, CPML>;
  constexpr int TYT = L::TYT;
  constexpr int NT = L::NT;
  constexpr int NH = TZ + TY;  // halo threads
  constexpr int EW = L::EW, HW = L::HW, NW = L::NW;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
  float* stages = reinterpret_cast<float*>(smem_raw + 128);
  float* Hn = stages + STAGES * L::STAGE_FLOATS;
  float* PSc = Hn + 3 * L::HN_STRIDE;
  float* PSh = PSc + L::PSC_FLOATS;

  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int tid = threadIdx.x;
  const int tx = tid % TZ;
  const int ty = tid / TZ;
  const int z0 = blockIdx.x * TZ;
  const int y0 = blockIdx.y * TY;
  const int xb = blockIdx.z * p.x_chunk;
  const int xe = min(xb + p.x_chunk, nx);
  const int qs = xb > 0 ? xb - 1 : 0;  // first plane staged
  const int qe = min(xe, nx - 1);      // last plane staged
  const int nload = qe - qs + 1;
  const float a = p.a;
  const int z = z0 + tx;

  // Probes of the input state (= after the previous step).
  if (p.probe_out != nullptr && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0) {
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

  // ---- CPML: slab coordinates and coefficients of this thread's cells
  // (fixed over the march along x)
  int jm_r[RY];
  int km = -1;
  AxisCoef cz{};
  int jm_h = -1, km_h = -1;  // halo cell slab indices
  int yh = -1, zh = -1;      // halo cell (-1: none)
  if (CPML) {
    km = (z < nz) ? slab_map(z, nz, p.pml.P[2]) : -1;
    if (z < nz) cz = axis_coef(p.pml, 2, z);
#pragma unroll
    for (int r = 0; r < RY; ++r) {
      const int y = y0 + ty + r * TYT;
      jm_r[r] = (y < ny) ? slab_map(y, ny, p.pml.P[1]) : -1;
    }
    if (tid < TZ) {  // row halo (y0-1, z0+tid)
      if (y0 >= 1 && z0 + tid < nz) {
        yh = y0 - 1;
        zh = z0 + tid;
      }
    } else if (tid < NH) {  // column halo (y0+tid-TZ, z0-1)
      if (z0 >= 1 && y0 + tid - TZ < ny) {
        yh = y0 + tid - TZ;
        zh = z0 - 1;
      }
    }
    if (yh >= 0) {
      jm_h = slab_map(yh, ny, p.pml.P[1]);
      km_h = slab_map(zh, nz, p.pml.P[2]);
    }
  }
#define PSC(buf, id, r) PSc[(((buf) * PSI_COUNT + (id)) * RY + (r)) * NT + tid]
#define PSH(buf, k) PSh[((buf) * 4 + (k)) * NH + tid]
  // Prefetch psi_in of plane q into buffer `buf` (this thread's cells only).
  auto issue_psi = [&](int q, int buf) {
    const int imq = slab_map(q, nx, p.pml.P[0]);
#pragma unroll
    for (int r = 0; r < RY; ++r) {
      const int y = y0 + ty + r * TYT;
      if (y < ny && z < nz) {
        const int jm = jm_r[r];
        if (jm >= 0) {
          const long long iy = ys_index(q, jm, z, p.pml.L[1], nz);
          cp_async4(&PSC(buf, PSI_HXY, r), p.pml.in[PSI_HXY] + iy);
          cp_async4(&PSC(buf, PSI_HZY, r), p.pml.in[PSI_HZY] + iy);
          cp_async4(&PSC(buf, PSI_EXY, r), p.pml.in[PSI_EXY] + iy);
          cp_async4(&PSC(buf, PSI_EZY, r), p.pml.in[PSI_EZY] + iy);
        }
        if (km >= 0) {
          const long long iz = zs_index(q, y, km, ny, p.pml.L[2]);
          cp_async4(&PSC(buf, PSI_HXZ, r), p.pml.in[PSI_HXZ] + iz);
          cp_async4(&PSC(buf, PSI_HYZ, r), p.pml.in[PSI_HYZ] + iz);
          cp_async4(&PSC(buf, PSI_EXZ, r), p.pml.in[PSI_EXZ] + iz);
          cp_async4(&PSC(buf, PSI_EYZ, r), p.pml.in[PSI_EYZ] + iz);
        }
        if (imq >= 0) {
          const long long ix = xs_index(imq, y, z, ny, nz);
          cp_async4(&PSC(buf, PSI_HYX, r), p.pml.in[PSI_HYX] + ix);
          cp_async4(&PSC(buf, PSI_HZX, r), p.pml.in[PSI_HZX] + ix);
          cp_async4(&PSC(buf, PSI_EYX, r), p.pml.in[PSI_EYX] + ix);
          cp_async4(&PSC(buf, PSI_EZX, r), p.pml.in[PSI_EZX] + ix);
        }
      }
    }
    if (yh >= 0) {
      if (jm_h >= 0)
        cp_async4(&PSH(buf, 0), p.pml.in[PSI_HXY] + ys_index(q, jm_h, zh, p.pml.L[1], nz));
      if (km_h >= 0)
        cp_async4(&PSH(buf, 1), p.pml.in[PSI_HXZ] + zs_index(q, yh, km_h, ny, p.pml.L[2]));
      if (tid < TZ) {  // row halo: Hz needs hzx, hzy
        if (imq >= 0)
          cp_async4(&PSH(buf, 2), p.pml.in[PSI_HZX] + xs_index(imq, yh, zh, ny, nz));
        if (jm_h >= 0)
          cp_async4(&PSH(buf, 3), p.pml.in[PSI_HZY] + ys_index(q, jm_h, zh, p.pml.L[1], nz));
      } else {  // column halo: Hy needs hyz, hyx
        if (km_h >= 0)
          cp_async4(&PSH(buf, 2), p.pml.in[PSI_HYZ] + zs_index(q, yh, km_h, ny, p.pml.L[2]));
        if (imq >= 0)
          cp_async4(&PSH(buf, 3), p.pml.in[PSI_HYX] + xs_index(imq, yh, zh, ny, nz));
      }
    }
    cp_async_commit();
  };
  if (CPML) issue_psi(qs, 0);

  // source list of this block
  const int bid = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
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
    const int pb = l & 1;  // psi buffer of this plane
    if (CPML) {
      if (x + 1 < xe) issue_psi(x + 1, pb ^ 1);
      else cp_async_commit();  // empty group keeps the wait_group count uniform
      cp_async_wait_prev();    // this plane's psi has landed (own copies only)
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
#define E_AT(c, yy, zc) Es[(c) * L::E_STRIDE + (yy) * EW + (zc)]
#define EN_AT(c, yy, zc) En[(c) * L::E_STRIDE + (yy) * EW + (zc)]
#define H_AT(c, yy, zc) Hs[(c) * L::H_STRIDE + (yy) * HW + (zc)]
#define HN_AT(c, yy, zc) Hn[(c) * L::HN_STRIDE + (yy) * NW + (zc)]
    const bool warm = (x < xb);
    int imx = -1;
    AxisCoef cx{};
    if (CPML) {
      imx = slab_map(x, nx, p.pml.P[0]);
      cx = axis_coef(p.pml, 0, x);
    }
    const bool inx = imx >= 0;

    // ---------------- H^{n+1/2} on the tile (registers + Hn) ----------------
    float exr[RY], eyr[RY], ezr[RY], hxr[RY], hyr[RY], hzr[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) {
      const int yl = ty + r * TYT;
      const int y = y0 + yl;
      const int yy = yl + 1;
      const bool own = !warm && (y < ny) && (z < nz);
      const float exc = E_AT(0, yy, zz), eyc = E_AT(1, yy, zz), ezc = E_AT(2, yy, zz);
      exr[r] = exc;
      eyr[r] = eyc;
      ezr[r] = ezc;
      float hx = H_AT(0, yy, zz), hy = H_AT(1, yy, zz), hz = H_AT(2, yy, zz);
      const bool iny = CPML && jm_r[r] >= 0, inz = CPML && km >= 0;
      // Cells outside every slab take the plain update (identical value: psi
      // is 0 and 1/kappa is 1 there) without touching any CPML state.
      auto h_phase = [&](auto cpm) {
        constexpr bool CP = decltype(cpm)::value;
        const long long ix = CP ? xs_index(imx, y, z, ny, nz) : 0;
        const long long iy = CP ? ys_index(x, jm_r[r], z, p.pml.L[1], nz) : 0;
        const long long iz = CP ? zs_index(x, y, km, ny, p.pml.L[2]) : 0;
        if (!warm && y < ny - 1 && z < nz - 1) {  // Hx: d/dy Ez - d/dz Ey
          const float d1 = fsub(E_AT(2, yy + 1, zz), ezc), d2 = fsub(E_AT(1, yy, zz + 1), eyc);
          if (CP)
            hx = h_cpml<KAPPA>(
                hx, a, d1, d2,
                term_h_at(p.pml, 1, y, iny, PSC(pb, PSI_HXY, r), own ? p.pml.out[PSI_HXY] + iy : nullptr),
                term_h(inz, cz, PSC(pb, PSI_HXZ, r), own ? p.pml.out[PSI_HXZ] + iz : nullptr));
          else
            hx = h_plain(hx, a, d1, d2);
        }
        if (x < nx - 1 && z < nz - 1 && y < ny) {  // Hy: d/dz Ex - d/dx Ez
          const float d1 = fsub(E_AT(0, yy, zz + 1), exc), d2 = fsub(EN_AT(2, yy, zz), ezc);
          if (CP)
            hy = h_cpml<KAPPA>(
                hy, a, d1, d2,
                term_h(inz, cz, PSC(pb, PSI_HYZ, r), own ? p.pml.out[PSI_HYZ] + iz : nullptr),
                term_h(inx, cx, PSC(pb, PSI_HYX, r), own ? p.pml.out[PSI_HYX] + ix : nullptr));
          else
            hy = h_plain(hy, a, d1, d2);
        }
        if (x < nx - 1 && y < ny - 1 && z < nz) {  // Hz: d/dx Ey - d/dy Ex
          const float d1 = fsub(EN_AT(1, yy, zz), eyc), d2 = fsub(E_AT(0, yy + 1, zz), exc);
          if (CP)
            hz = h_cpml<KAPPA>(
                hz, a, d1, d2,
                term_h(inx, cx, PSC(pb, PSI_HZX, r), own ? p.pml.out[PSI_HZX] + ix : nullptr),
                term_h_at(p.pml, 1, y, iny, PSC(pb, PSI_HZY, r), own ? p.pml.out[PSI_HZY] + iy : nullptr));
          else
            hz = h_plain(hz, a, d1, d2);
        }
      };
      if (CPML && (iny || inz || inx))
        h_phase(BoolC<CPML>{});
      else
        h_phase(BoolC<false>{});
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
              hx = h_cpml<KAPPA>(hx, a, d1, d2, term_h_at(p.pml, 1, y, jm_h >= 0, PSH(pb, 0), nullptr),
                                 term_h_at(p.pml, 2, zc, km_h >= 0, PSH(pb, 1), nullptr));
            else
              hx = h_plain(hx, a, d1, d2);
          }
          if (x < nx - 1) {
            const float d1 = fsub(EN_AT(1, 0, zb), eyc), d2 = fsub(E_AT(0, 1, zb), exc);
            if (CPML)
              hz = h_cpml<KAPPA>(hz, a, d1, d2, term_h(inx, cx, PSH(pb, 2), nullptr),
                                 term_h_at(p.pml, 1, y, jm_h >= 0, PSH(pb, 3), nullptr));
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
              hx = h_cpml<KAPPA>(hx, a, d1, d2, term_h_at(p.pml, 1, y, jm_h >= 0, PSH(pb, 0), nullptr),
                                 term_h_at(p.pml, 2, zc, km_h >= 0, PSH(pb, 1), nullptr));
            else
              hx = h_plain(hx, a, d1, d2);
          }
          if (x < nx - 1) {
            const float d1 = fsub(E_AT(0, yy, 4), exc), d2 = fsub(EN_AT(2, yy, 3), ezc);
            if (CPML)
              hy = h_cpml<KAPPA>(hy, a, d1, d2, term_h_at(p.pml, 2, zc, km_h >= 0, PSH(pb, 2), nullptr),
                                 term_h(inx, cx, PSH(pb, 3), nullptr));
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
        const float cb = CBARR ? CBs[yl * TZ + tx] : p.cb_const;
        const bool iny = CPML && own && jm_r[r] >= 0, inz = CPML && own && km >= 0;
        const bool inxo = own && inx;
        auto e_phase = [&](auto cpm) {
          constexpr bool CP = decltype(cpm)::value;
          const long long ix = CP ? xs_index(imx, y, z, ny, nz) : 0;
          const long long iy = CP ? ys_index(x, jm_r[r], z, p.pml.L[1], nz) : 0;
          const long long iz = CP ? zs_index(x, y, km, ny, p.pml.L[2]) : 0;
          if (y >= 1 && z >= 1) {  // Ex: d/dy Hz - d/dz Hy
            const float d1 = fsub(hzc, HN_AT(2, yy - 1, zn)), d2 = fsub(hyc, HN_AT(1, yy, zn - 1));
            if (CP)
              ex = e_cpml<KAPPA>(ex, cb, d1, d2,
                                 term_e_at(p.pml, 1, y, iny, PSC(pb, PSI_EXY, r), p.pml.out[PSI_EXY] + iy),
                                 term_e(inz, cz, PSC(pb, PSI_EXZ, r), p.pml.out[PSI_EXZ] + iz));
            else
              ex = e_plain(ex, cb, d1, d2);
          }
          if (x >= 1 && z >= 1) {  // Ey: d/dz Hx - d/dx Hz
            const float d1 = fsub(hxc, HN_AT(0, yy, zn - 1)), d2 = fsub(hzc, hz_prev[r]);
            if (CP)
              ey = e_cpml<KAPPA>(ey, cb, d1, d2,
                                 term_e(inz, cz, PSC(pb, PSI_EYZ, r), p.pml.out[PSI_EYZ] + iz),
                                 term_e(inxo, cx, PSC(pb, PSI_EYX, r), p.pml.out[PSI_EYX] + ix));
            else
              ey = e_plain(ey, cb, d1, d2);
          }
          if (x >= 1 && y >= 1) {  // Ez: d/dx Hy - d/dy Hx
            const float d1 = fsub(hyc, hy_prev[r]), d2 = fsub(hxc, HN_AT(0, yy - 1, zn));
            if (CP)
              ez = e_cpml<KAPPA>(ez, cb, d1, d2,
                                 term_e(inxo, cx, PSC(pb, PSI_EZX, r), p.pml.out[PSI_EZX] + ix),
                                 term_e_at(p.pml, 1, y, iny, PSC(pb, PSI_EZY, r), p.pml.out[PSI_EZY] + iy));
            else
              ez = e_plain(ez, cb, d1, d2);
          }
        };
        if (CPML && (iny || inz || inxo))
          e_phase(BoolC<CPML>{});
        else
          e_phase(BoolC<false>{});
        if (MODE == MODE_ABSORB && own) {
          const float f =
              fmul(fmul(__ldg(p.damp[0] + x), __ldg(p.damp[1] + y)), __ldg(p.damp[2] + z));
          ex = fmul(ex, f);
          ey = fmul(ey, f);
          ez = fmul(ez, f);
        }
        exo[r] = ex;
        eyo[r] = ey;
        ezo[r] = ez;
      }
      // soft sources of plane x (uniform loop: every thread reads each entry)
      while (sp < se) {
        const SrcEntry e = p.src[sp];
        if (e.x != x) break;
        const int yl_e = e.off / TZ;
        const int tz_e = e.off - yl_e * TZ;
        if (tz_e == tx && (yl_e % TYT) == ty) {
          const int r_e = yl_e / TYT;
          const float v = fmul(e.amp, p.wave[(long long)e.wave * p.wave_len + p.step]);
#pragma unroll
          for (int r = 0; r < RY; ++r) {
            if (r == r_e) {
              if (e.comp == 0) exo[r] = fadd(exo[r], v);
              else if (e.comp == 1) eyo[r] = fadd(eyo[r], v);
              else ezo[r] = fadd(ezo[r], v);
            }
          }
        }
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
    __syncthreads();  // Hn and stage `slot` are free again
    consumed = l + 1;
    if (issued < nload && issued < consumed + STAGES) {
      if (tid == 0) issue(issued);
      ++issued;
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

}  // namespace jxf
