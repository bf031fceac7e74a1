// Discrete adjoint of the 3D Yee step (reverse mode, time reversed).
//
// Forward step n (fdtd3d_kernels.cuh; CPML written generally, the damping
// boundary is the same with psi absent and a per-cell factor `damp`):
//   psiH' = bH psiH + cH D(E)                       D: forward differences
//   H'    = H - a (kH D(E) + S psiH')               S: +psi1 - psi2 per component
//   psiE' = bE psiE + cE G(H')                      G: backward differences
//   E'    = damp (E + cb (kE G(H') + S psiE')) + src
// Its transpose, applied to the adjoint (Ebar', Hbar', psibar') of the
// step's outputs, gives the adjoint of its inputs:
//   k3a_e : X = kE G(H') + S psiE' from the stored forward state;
//           dJ/dcb += damp Ebar' X (FP64); Xbar = cb damp Ebar';
//           psibarE' += S^T Xbar;  dbarE = kE^T Xbar + cE psibarE';
//           psibarE = bE psibarE';  Ebar = damp Ebar'
//   k3a_h : Hbar' += G^T dbarE (gather);  Ybar = -a Hbar';
//           psibarH' += S^T Ybar;  dbarH = kH^T Ybar + cH psibarH';
//           psibarH = bH psibarH';  Hbar = Hbar'
//   k3a_e2: Ebar += D^T dbarH (gather)
// Cells outside a component's update range are the identity (no curl term),
// exactly as in the forward step.  Adjoint fields are FP32; dJ/dcb is
// accumulated in FP64.
#pragma once

#include "fdtd3d_kernels.cuh"

namespace jxf {

// db arrays of the E phase (adjoint of the H differences used by E):
//   0: Ex / dHz/dy   1: Ex / dHy/dz   2: Ey / dHx/dz
//   3: Ey / dHz/dx   4: Ez / dHy/dx   5: Ez / dHx/dy
// dh arrays of the H phase (adjoint of the E differences used by H):
//   0: Hx / dEz/dy   1: Hx / dEy/dz   2: Hy / dEx/dz
//   3: Hy / dEz/dx   4: Hz / dEy/dx   5: Hz / dEx/dy
struct Adj3D {
  int nx, ny, nz;
  float a, cb_const;
  const float* cb;
  const float* damp[3];
  CpmlDev pml;                // tables, slab maps (in/out unused)
  const float* fh[3];         // forward H^{n+1/2} after the step
  const float* fpsiE[6];      // forward psi (EXY..EZY) after the step, slab layout
  float* lE[3];               // adjoint of E
  float* lH[3];               // adjoint of H
  float* lpsi[PSI_COUNT];     // adjoint of psi, slab layout
  float* db[6];
  float* dh[6];
  double* gcb;                // dJ/dcb accumulator
  FastDiv div_nz, div_ny;     // index decode (idx32: nx ny nz < 2^32)
  int idx32;
};

// psi adjoint through one term: tot = carried + u; new carried = b * tot;
// returns c * tot (the term's contribution to the difference adjoint).
__device__ __forceinline__ float adj_psi(float* lp, long long idx, float b, float c, float u) {
  const float tot = lp[idx] + u;
  lp[idx] = b * tot;
  return c * tot;
}

template <int MODE>
__global__ void __launch_bounds__(256) k3a_e(const __grid_constant__ Adj3D p) {
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const long long n = (long long)nx * ny * nz;
  constexpr bool CP = (MODE == MODE_CPML);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    decode_cell(i, nz, ny, p.idx32 != 0, p.div_nz, p.div_ny, x, y, z);
    const float cb = p.cb ? p.cb[i] : p.cb_const;
    float damp = 1.0f;
    if (MODE == MODE_ABSORB)
      damp = (p.damp[0][x] * p.damp[1][y]) * p.damp[2][z];
    int im = -1, jm = -1, km = -1;
    AxisCoef cx{}, cy{}, cz{};
    if (CP) {
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
    const float* hx = p.fh[0];
    const float* hy = p.fh[1];
    const float* hz = p.fh[2];
    double g = 0.0;
    float d[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    // one E component: terms (axis a1 with diff d1, slab s1, psi id q1) and
    // (axis a2, d2, s2, q2); X = (ik1 d1 - ik2 d2) + (psi1' - psi2')
    auto comp = [&](int c, float d1, float d2, bool s1, bool s2, int q1, int q2, long long o1,
                    long long o2, const AxisCoef& k1, const AxisCoef& k2, int out1, int out2) {
      const float eb = p.lE[c][i];
      float X;
      if (CP && (s1 || s2)) {
        const float p1 = s1 ? p.fpsiE[q1 - PSI_EXY][o1] : 0.0f;
        const float p2 = s2 ? p.fpsiE[q2 - PSI_EXY][o2] : 0.0f;
        X = (k1.ike * d1 - k2.ike * d2) + (p1 - p2);
      } else {
        X = d1 - d2;
      }
      g += (double)eb * (double)damp * (double)X;
      const float xb = cb * damp * eb;
      float u1 = xb, u2 = -xb;  // adjoints of ik*d terms before ik
      if (CP && (s1 || s2)) {
        const float c1 = s1 ? adj_psi(p.lpsi[q1], o1, k1.be, k1.ce, xb) : 0.0f;
        const float c2 = s2 ? adj_psi(p.lpsi[q2], o2, k2.be, k2.ce, -xb) : 0.0f;
        u1 = k1.ike * xb + c1;
        u2 = -k2.ike * xb + c2;
      }
      d[out1] = u1;
      d[out2] = u2;
    };
    if (y >= 1 && z >= 1)  // Ex: dHz/dy - dHy/dz
      comp(0, hz[i] - hz[i - nz], hy[i] - hy[i - 1], jm >= 0, km >= 0, PSI_EXY, PSI_EXZ, iy, iz,
           cy, cz, 0, 1);
    if (x >= 1 && z >= 1)  // Ey: dHx/dz - dHz/dx
      comp(1, hx[i] - hx[i - 1], hz[i] - hz[i - (long long)ny * nz], km >= 0, im >= 0, PSI_EYZ,
           PSI_EYX, iz, ix, cz, cx, 2, 3);
    if (x >= 1 && y >= 1)  // Ez: dHy/dx - dHx/dy
      comp(2, hy[i] - hy[i - (long long)ny * nz], hx[i] - hx[i - nz], im >= 0, jm >= 0, PSI_EZX,
           PSI_EZY, ix, iy, cx, cy, 4, 5);
    for (int k = 0; k < 6; ++k) p.db[k][i] = d[k];
    if (g != 0.0) p.gcb[i] += g;
    if (MODE == MODE_ABSORB)
      for (int c = 0; c < 3; ++c) p.lE[c][i] = damp * p.lE[c][i];
  }
}

template <int MODE>
__global__ void __launch_bounds__(256) k3a_h(const __grid_constant__ Adj3D p) {
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const long long n = (long long)nx * ny * nz;
  const long long sx = (long long)ny * nz;
  constexpr bool CP = (MODE == MODE_CPML);
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    decode_cell(j, nz, ny, p.idx32 != 0, p.div_nz, p.div_ny, x, y, z);
    // Hbar' = lH + G^T dbarE
    const float zp_db2 = (z + 1 < nz) ? p.db[2][j + 1] : 0.0f;
    const float yp_db5 = (y + 1 < ny) ? p.db[5][j + nz] : 0.0f;
    const float zp_db1 = (z + 1 < nz) ? p.db[1][j + 1] : 0.0f;
    const float xp_db4 = (x + 1 < nx) ? p.db[4][j + sx] : 0.0f;
    const float yp_db0 = (y + 1 < ny) ? p.db[0][j + nz] : 0.0f;
    const float xp_db3 = (x + 1 < nx) ? p.db[3][j + sx] : 0.0f;
    const float hxb = p.lH[0][j] + (p.db[2][j] - zp_db2) + (p.db[5][j] - yp_db5);
    const float hyb = p.lH[1][j] + (p.db[1][j] - zp_db1) + (p.db[4][j] - xp_db4);
    const float hzb = p.lH[2][j] + (p.db[0][j] - yp_db0) + (p.db[3][j] - xp_db3);
    p.lH[0][j] = hxb;
    p.lH[1][j] = hyb;
    p.lH[2][j] = hzb;
    int im = -1, jm = -1, km = -1;
    AxisCoef cx{}, cy{}, cz{};
    if (CP) {
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
    float d[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    auto comp = [&](float hb, bool s1, bool s2, int q1, int q2, long long o1, long long o2,
                    const AxisCoef& k1, const AxisCoef& k2, int out1, int out2) {
      const float yb = -p.a * hb;
      float u1 = yb, u2 = -yb;
      if (CP && (s1 || s2)) {
        const float c1 = s1 ? adj_psi(p.lpsi[q1], o1, k1.bh, k1.ch, yb) : 0.0f;
        const float c2 = s2 ? adj_psi(p.lpsi[q2], o2, k2.bh, k2.ch, -yb) : 0.0f;
        u1 = k1.ikh * yb + c1;
        u2 = -k2.ikh * yb + c2;
      }
      d[out1] = u1;
      d[out2] = u2;
    };
    if (y < ny - 1 && z < nz - 1)  // Hx: dEz/dy - dEy/dz
      comp(hxb, jm >= 0, km >= 0, PSI_HXY, PSI_HXZ, iy, iz, cy, cz, 0, 1);
    if (x < nx - 1 && z < nz - 1)  // Hy: dEx/dz - dEz/dx
      comp(hyb, km >= 0, im >= 0, PSI_HYZ, PSI_HYX, iz, ix, cz, cx, 2, 3);
    if (x < nx - 1 && y < ny - 1)  // Hz: dEy/dx - dEx/dy
      comp(hzb, im >= 0, jm >= 0, PSI_HZX, PSI_HZY, ix, iy, cx, cy, 4, 5);
    for (int k = 0; k < 6; ++k) p.dh[k][j] = d[k];
  }
}

// Ebar += D^T dbarH (forward differences transposed: gather from i - axis)
__global__ void __launch_bounds__(256) k3a_e2(const __grid_constant__ Adj3D p) {
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const long long n = (long long)nx * ny * nz;
  const long long sx = (long long)ny * nz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    decode_cell(i, nz, ny, p.idx32 != 0, p.div_nz, p.div_ny, x, y, z);
    const float zm_dh2 = z >= 1 ? p.dh[2][i - 1] : 0.0f;
    const float ym_dh5 = y >= 1 ? p.dh[5][i - nz] : 0.0f;
    const float zm_dh1 = z >= 1 ? p.dh[1][i - 1] : 0.0f;
    const float xm_dh4 = x >= 1 ? p.dh[4][i - sx] : 0.0f;
    const float ym_dh0 = y >= 1 ? p.dh[0][i - nz] : 0.0f;
    const float xm_dh3 = x >= 1 ? p.dh[3][i - sx] : 0.0f;
    p.lE[0][i] += (zm_dh2 - p.dh[2][i]) + (ym_dh5 - p.dh[5][i]);
    p.lE[1][i] += (zm_dh1 - p.dh[1][i]) + (xm_dh4 - p.dh[4][i]);
    p.lE[2][i] += (ym_dh0 - p.dh[0][i]) + (xm_dh3 - p.dh[3][i]);
  }
}

// adjoint seeds of the probe readout after step n: lambda[comp][cell] += g[p]
struct Lam6 {
  float* f[6];  // adjoint of Ex, Ey, Ez, Hx, Hy, Hz
};
__global__ void k3a_seed(Lam6 lam, const long long* cell, const int* comp, int n_probes,
                         const float* grad_row) {
  // one thread: probes may repeat a cell, so add in order
  if (blockIdx.x == 0 && threadIdx.x == 0)
    for (int k = 0; k < n_probes; ++k) lam.f[comp[k]][cell[k]] += grad_row[k];
}

// dJ/deps_r = dJ/dcb * dcb/deps_r = -dJ/dcb * cb^2 / coef_e
__global__ void k3a_finish(const double* gcb, const float* cb, float cb_const, double coef_e,
                           float* grad_eps, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double c = cb ? (double)cb[i] : (double)cb_const;
    grad_eps[i] = (float)(-gcb[i] * c * c / coef_e);
  }
}

}  // namespace jxf
