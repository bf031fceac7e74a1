// 2D TM (Ez, Hx, Hy) Yee kernels for sm_100a.
//
// One step of the reference's scan body (jaxphys src/neurosim/em/fdtd.py:304-357):
//   Hx[:, :-1] -= a (Ez[:, 1:] - Ez[:, :-1])                 (:325-327)
//   Hy[:-1, :] += a (Ez[1:, :] - Ez[:-1, :])                 (:330-332)
//   Ez[1:, 1:] += b ((Hy[i]-Hy[i-1]) - (Hx[j]-Hx[j-1]))       (:335-340)
//   periodic: the same with wrap-around differences on every cell (:314-321)
// then, by boundary mode: damping exp(-sigma_avg dt/eps0) (:342-344), mirrored
// edges (:264-282) or wrapped edges (:284-302); then line sources on whole
// rows Ez[:, y] (:257-262,354) and conductor rows forced to 0 (:357).
#pragma once

#include "fdtd_common.cuh"

namespace jxf {

struct Step2D {
  int nx, ny;
  float a, b;
  float* ez;
  float* hx;
  float* hy;
  const float* damp[2];  // separable damping (ABSORBING)
  // line sources (list order)
  int n_src;
  const int* src_y;
  const float* src_amp;
  const int* src_wave;
  const float* wave;
  long long wave_len;
  long long step;
  // conductor rows
  int n_wall;
  const int* wall_y;
  const int* wall_g0;  // < 0: solid
  const int* wall_g1;
};

template <int MODE>
__global__ void __launch_bounds__(256) k2d_h(const __grid_constant__ Step2D p) {
  const int nx = p.nx, ny = p.ny;
  const long long n = (long long)nx * ny;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(idx % ny);
    const int x = (int)(idx / ny);
    const float e = p.ez[idx];
    if (MODE == MODE_PERIODIC) {
      const long long iyp = (y + 1 == ny) ? idx - (ny - 1) : idx + 1;
      const long long ixp = (x + 1 == nx) ? (long long)y : idx + ny;
      p.hx[idx] = fsub(p.hx[idx], fmul(p.a, fsub(p.ez[iyp], e)));
      p.hy[idx] = fadd(p.hy[idx], fmul(p.a, fsub(p.ez[ixp], e)));
    } else {
      if (y < ny - 1) p.hx[idx] = fsub(p.hx[idx], fmul(p.a, fsub(p.ez[idx + 1], e)));
      if (x < nx - 1) p.hy[idx] = fadd(p.hy[idx], fmul(p.a, fsub(p.ez[idx + ny], e)));
    }
  }
}

__device__ __forceinline__ float add_line_sources(const Step2D& p, int y, float v) {
  for (int s = 0; s < p.n_src; ++s) {
    if (p.src_y[s] == y)
      v = fadd(v, fmul(p.src_amp[s], p.wave[(long long)p.src_wave[s] * p.wave_len + p.step]));
  }
  return v;
}

__device__ __forceinline__ bool in_wall(const Step2D& p, int x, int y) {
  for (int w = 0; w < p.n_wall; ++w) {
    if (p.wall_y[w] == y) {
      const int g0 = p.wall_g0[w], g1 = p.wall_g1[w];
      if (g0 < 0 || x < g0 || x >= g1) return true;
    }
  }
  return false;
}

// E update.  FUSE_POST: damping, sources and conductors in the same pass
// (ABSORBING, where no edge rule runs between them).
template <int MODE, bool FUSE_POST>
__global__ void __launch_bounds__(256) k2d_e(const __grid_constant__ Step2D p) {
  const int nx = p.nx, ny = p.ny;
  const long long n = (long long)nx * ny;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(idx % ny);
    const int x = (int)(idx / ny);
    float e = p.ez[idx];
    if (MODE == MODE_PERIODIC) {
      const long long ixm = (x == 0) ? idx + (long long)(nx - 1) * ny : idx - ny;
      const long long iym = (y == 0) ? idx + (ny - 1) : idx - 1;
      const float dhy = fsub(p.hy[idx], p.hy[ixm]);
      const float dhx = fsub(p.hx[idx], p.hx[iym]);
      e = fadd(e, fmul(p.b, fsub(dhy, dhx)));
    } else if (x >= 1 && y >= 1) {
      const float dhy = fsub(p.hy[idx], p.hy[idx - ny]);
      const float dhx = fsub(p.hx[idx], p.hx[idx - 1]);
      e = fadd(e, fmul(p.b, fsub(dhy, dhx)));
    }
    if (FUSE_POST) {
      if (MODE == MODE_ABSORB) e = fmul(e, fmul(__ldg(p.damp[0] + x), __ldg(p.damp[1] + y)));
      e = add_line_sources(p, y, e);
      if (in_wall(p, x, y)) e = 0.0f;
    }
    p.ez[idx] = e;
  }
}

// Edge rules (periodic: wrap, reflecting: mirror) for Ez, Hx, Hy in the
// reference's order (rows 0 and nx-1, then columns 0 and ny-1, so the column
// copies see the row copies), then sources, then conductors.  One block.
template <int MODE>
__global__ void __launch_bounds__(1024) k2d_post(const __grid_constant__ Step2D p) {
  const int nx = p.nx, ny = p.ny;
  const int t = threadIdx.x, nt = blockDim.x;
  const bool per = (MODE == MODE_PERIODIC);
  float* fs[3] = {p.ez, p.hx, p.hy};
  // f[0,:] = f[-2,:] (periodic) / f[1,:] (reflecting)
  for (int c = 0; c < 3; ++c) {
    float* f = fs[c];
    for (int j = t; j < ny; j += nt) f[j] = per ? f[(long long)(nx - 2) * ny + j] : f[(long long)ny + j];
  }
  __syncthreads();
  // f[-1,:] = f[1,:] (periodic) / f[-2,:] (reflecting)
  for (int c = 0; c < 3; ++c) {
    float* f = fs[c];
    for (int j = t; j < ny; j += nt)
      f[(long long)(nx - 1) * ny + j] = per ? f[(long long)ny + j] : f[(long long)(nx - 2) * ny + j];
  }
  __syncthreads();
  // f[:,0] = f[:,-2] / f[:,1]
  for (int c = 0; c < 3; ++c) {
    float* f = fs[c];
    for (int i = t; i < nx; i += nt) {
      const long long r = (long long)i * ny;
      f[r] = per ? f[r + ny - 2] : f[r + 1];
    }
  }
  __syncthreads();
  // f[:,-1] = f[:,1] / f[:,-2]
  for (int c = 0; c < 3; ++c) {
    float* f = fs[c];
    for (int i = t; i < nx; i += nt) {
      const long long r = (long long)i * ny;
      f[r + ny - 1] = per ? f[r + 1] : f[r + ny - 2];
    }
  }
  __syncthreads();
  // sources over whole rows, then conductors
  for (int i = t; i < nx; i += nt) {
    for (int s = 0; s < p.n_src; ++s) {
      const long long idx = (long long)i * ny + p.src_y[s];
      p.ez[idx] = fadd(p.ez[idx],
                       fmul(p.src_amp[s], p.wave[(long long)p.src_wave[s] * p.wave_len + p.step]));
    }
  }
  __syncthreads();
  for (int i = t; i < nx; i += nt) {
    for (int w = 0; w < p.n_wall; ++w) {
      const int g0 = p.wall_g0[w], g1 = p.wall_g1[w];
      if (g0 < 0 || i < g0 || i >= g1) p.ez[(long long)i * ny + p.wall_y[w]] = 0.0f;
    }
  }
}

}  // namespace jxf
