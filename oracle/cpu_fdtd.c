/*
 * FP64 CPU oracle for the 3D FDTD hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * The same step as oracle/ref_numpy.py (which restates jaxphys
 * src/neurosim/em/fdtd3d.py:280-379 and is pinned bit-for-bit to the
 * reference source by tests/golden), written as OpenMP loops so the parity
 * tests can run 64^3 x 500 and 128^3 x 1000 cases in seconds and bench.py can
 * time a CPU baseline.  Coefficients (per-cell cb = dt/(eps0 dx eps_r),
 * per-cell damping exp(-sigma_avg dt/eps0), CPML tables, source values per
 * step) come from oracle/ref_numpy.py, so this file holds only the stencil.
 *
 * Update order per step (fdtd3d.py:303-369):
 *   H (from old E) -> E (from new H, times cb) -> damping (absorbing only)
 *   -> sources in list order -> probes.
 * Index ranges: Hx on [:, :-1, :-1], Hy on [:-1, :, :-1], Hz on [:-1, :-1, :];
 * Ex on [:, 1:, 1:], Ey on [1:, :, 1:], Ez on [1:, 1:, :]; periodic: every
 * cell with wrap-around neighbours (fdtd3d.py:249-301).
 * CPML (extension): psi <- b psi + c d; curl' = (ik1 d1 - ik2 d2) + (psi1 - psi2).
 */
#include <stdint.h>
#include <stddef.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { M_ABSORB = 0, M_PERIODIC = 1, M_PEC = 2, M_CPML = 3 };
/* psi order: hxy hxz hyz hyx hzx hzy exy exz eyz eyx ezx ezy */
/* tables per axis: be ce ike bh ch ikh */

#define IDX(x, y, z) (((int64_t)(x) * ny + (y)) * nz + (z))

static void step_h(int nx, int ny, int nz, int mode, double a, double* const* f,
                   const double* const* tab, double* const* psi) {
  double *ex = f[0], *ey = f[1], *ez = f[2], *hx = f[3], *hy = f[4], *hz = f[5];
#pragma omp parallel for schedule(static)
  for (int x = 0; x < nx; ++x) {
    for (int y = 0; y < ny; ++y) {
      for (int z = 0; z < nz; ++z) {
        const int64_t i = IDX(x, y, z);
        if (mode == M_PERIODIC) {
          const int64_t ixp = IDX((x + 1) % nx, y, z), iyp = IDX(x, (y + 1) % ny, z),
                        izp = IDX(x, y, (z + 1) % nz);
          /* fdtd3d.py:253-263 and :293-295 */
          hx[i] = hx[i] - a * ((ez[iyp] - ez[i]) - (ey[izp] - ey[i]));
          hy[i] = hy[i] - a * ((ex[izp] - ex[i]) - (ez[ixp] - ez[i]));
          hz[i] = hz[i] - a * ((ey[ixp] - ey[i]) - (ex[iyp] - ex[i]));
          continue;
        }
        const int64_t ixp = i + (int64_t)ny * nz, iyp = i + nz, izp = i + 1;
        if (y < ny - 1 && z < nz - 1) {
          const double d1 = ez[iyp] - ez[i], d2 = ey[izp] - ey[i];
          if (mode == M_CPML) {
            psi[0][i] = tab[1 * 6 + 3][y] * psi[0][i] + tab[1 * 6 + 4][y] * d1;
            psi[1][i] = tab[2 * 6 + 3][z] * psi[1][i] + tab[2 * 6 + 4][z] * d2;
            hx[i] = hx[i] - a * ((tab[1 * 6 + 5][y] * d1 - tab[2 * 6 + 5][z] * d2) +
                                 (psi[0][i] - psi[1][i]));
          } else {
            hx[i] = hx[i] - a * (d1 - d2);
          }
        }
        if (x < nx - 1 && z < nz - 1) {
          const double d1 = ex[izp] - ex[i], d2 = ez[ixp] - ez[i];
          if (mode == M_CPML) {
            psi[2][i] = tab[2 * 6 + 3][z] * psi[2][i] + tab[2 * 6 + 4][z] * d1;
            psi[3][i] = tab[0 * 6 + 3][x] * psi[3][i] + tab[0 * 6 + 4][x] * d2;
            hy[i] = hy[i] - a * ((tab[2 * 6 + 5][z] * d1 - tab[0 * 6 + 5][x] * d2) +
                                 (psi[2][i] - psi[3][i]));
          } else {
            hy[i] = hy[i] - a * (d1 - d2);
          }
        }
        if (x < nx - 1 && y < ny - 1) {
          const double d1 = ey[ixp] - ey[i], d2 = ex[iyp] - ex[i];
          if (mode == M_CPML) {
            psi[4][i] = tab[0 * 6 + 3][x] * psi[4][i] + tab[0 * 6 + 4][x] * d1;
            psi[5][i] = tab[1 * 6 + 3][y] * psi[5][i] + tab[1 * 6 + 4][y] * d2;
            hz[i] = hz[i] - a * ((tab[0 * 6 + 5][x] * d1 - tab[1 * 6 + 5][y] * d2) +
                                 (psi[4][i] - psi[5][i]));
          } else {
            hz[i] = hz[i] - a * (d1 - d2);
          }
        }
      }
    }
  }
}

static void step_e(int nx, int ny, int nz, int mode, const double* cb, double cb_const,
                   const double* damp, double* const* f, const double* const* tab,
                   double* const* psi) {
  double *ex = f[0], *ey = f[1], *ez = f[2], *hx = f[3], *hy = f[4], *hz = f[5];
#pragma omp parallel for schedule(static)
  for (int x = 0; x < nx; ++x) {
    for (int y = 0; y < ny; ++y) {
      for (int z = 0; z < nz; ++z) {
        const int64_t i = IDX(x, y, z);
        const double c = cb ? cb[i] : cb_const;
        if (mode == M_PERIODIC) {
          const int64_t ixm = IDX((x + nx - 1) % nx, y, z), iym = IDX(x, (y + ny - 1) % ny, z),
                        izm = IDX(x, y, (z + nz - 1) % nz);
          /* fdtd3d.py:269-278 and :299-301 */
          ex[i] = ex[i] + c * ((hz[i] - hz[iym]) - (hy[i] - hy[izm]));
          ey[i] = ey[i] + c * ((hx[i] - hx[izm]) - (hz[i] - hz[ixm]));
          ez[i] = ez[i] + c * ((hy[i] - hy[ixm]) - (hx[i] - hx[iym]));
          continue;
        }
        const int64_t ixm = i - (int64_t)ny * nz, iym = i - nz, izm = i - 1;
        if (y >= 1 && z >= 1) {
          const double d1 = hz[i] - hz[iym], d2 = hy[i] - hy[izm];
          if (mode == M_CPML) {
            psi[6][i] = tab[1 * 6 + 0][y] * psi[6][i] + tab[1 * 6 + 1][y] * d1;
            psi[7][i] = tab[2 * 6 + 0][z] * psi[7][i] + tab[2 * 6 + 1][z] * d2;
            ex[i] = ex[i] + c * ((tab[1 * 6 + 2][y] * d1 - tab[2 * 6 + 2][z] * d2) +
                                 (psi[6][i] - psi[7][i]));
          } else {
            ex[i] = ex[i] + c * (d1 - d2);
          }
        }
        if (x >= 1 && z >= 1) {
          const double d1 = hx[i] - hx[izm], d2 = hz[i] - hz[ixm];
          if (mode == M_CPML) {
            psi[8][i] = tab[2 * 6 + 0][z] * psi[8][i] + tab[2 * 6 + 1][z] * d1;
            psi[9][i] = tab[0 * 6 + 0][x] * psi[9][i] + tab[0 * 6 + 1][x] * d2;
            ey[i] = ey[i] + c * ((tab[2 * 6 + 2][z] * d1 - tab[0 * 6 + 2][x] * d2) +
                                 (psi[8][i] - psi[9][i]));
          } else {
            ey[i] = ey[i] + c * (d1 - d2);
          }
        }
        if (x >= 1 && y >= 1) {
          const double d1 = hy[i] - hy[ixm], d2 = hx[i] - hx[iym];
          if (mode == M_CPML) {
            psi[10][i] = tab[0 * 6 + 0][x] * psi[10][i] + tab[0 * 6 + 1][x] * d1;
            psi[11][i] = tab[1 * 6 + 0][y] * psi[11][i] + tab[1 * 6 + 1][y] * d2;
            ez[i] = ez[i] + c * ((tab[0 * 6 + 2][x] * d1 - tab[1 * 6 + 2][y] * d2) +
                                 (psi[10][i] - psi[11][i]));
          } else {
            ez[i] = ez[i] + c * (d1 - d2);
          }
        }
        if (mode == M_ABSORB) { /* fdtd3d.py:362-366 */
          ex[i] = ex[i] * damp[i];
          ey[i] = ey[i] * damp[i];
          ez[i] = ez[i] * damp[i];
        }
      }
    }
  }
}

/* Advance n_steps.  src_val is [n_steps][n_src] (value already multiplied by
 * the amplitude, FP64); probe_out is [n_steps][n_probe]. */
int oracle3d_run(int nx, int ny, int nz, int mode, double a, const double* cb, double cb_const,
                 const double* damp, const double* const* tab, double* const* psi,
                 double* const* f, int n_src, const int64_t* src_cell, const int32_t* src_comp,
                 const double* src_val, int n_probe, const int64_t* probe_cell,
                 const int32_t* probe_comp, double* probe_out, int n_steps) {
  if (nx < 2 || ny < 2 || nz < 2 || n_steps < 0) return 1;
  if (mode == M_ABSORB && !damp) return 1;
  if (mode == M_CPML && (!tab || !psi)) return 1;
  for (int s = 0; s < n_steps; ++s) {
    step_h(nx, ny, nz, mode, a, f, tab, psi);
    step_e(nx, ny, nz, mode, cb, cb_const, damp, f, tab, psi);
    for (int k = 0; k < n_src; ++k) /* fdtd3d.py:236-244, list order */
      f[src_comp[k]][src_cell[k]] += src_val[(int64_t)s * n_src + k];
    for (int k = 0; k < n_probe; ++k)
      probe_out[(int64_t)s * n_probe + k] = f[probe_comp[k]][probe_cell[k]];
  }
  return 0;
}

int oracle_num_threads(void) {
  int n = 1;
#ifdef _OPENMP
#pragma omp parallel
  {
#pragma omp single
    n = omp_get_num_threads();
  }
#endif
  return n;
}
