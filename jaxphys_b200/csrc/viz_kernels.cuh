// Field viewers fed from device buffers: the |max| of strided 2D slices and
// their colour-mapped RGB images, computed where the fields already live so a
// viewer copies 3 bytes per pixel to the host instead of the FP32 frames.
//
// A slice is nu x nv samples at src[f*sf + c*su + r*sv] (frames f, columns c
// along the first in-plane axis, rows r along the second).  Images follow the
// reference viewer's imshow(data.T, origin="lower") (viz/fields.py:66-78):
// image row 0 is the highest r, image column c is slice column c.  Colour:
// t = (v / vmax + 1) / 2 mapped through a 256-entry table, index
// floor(t * 256) clamped to [0, 255] (values beyond +-vmax saturate).
#pragma once

#include <cstdint>

namespace jxf {

// max |v| over n_frames slices into *out (caller zeroes *out); non-negative
// floats order like their bit patterns, so an integer atomicMax does it.
__global__ void k_slice_absmax(const float* __restrict__ src, long long nu, long long nv,
                               long long su, long long sv, long long sf, long long n_total,
                               float* out) {
  float m = 0.0f;
  const long long per = nu * nv;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long f = i / per;
    const long long rem = i - f * per;
    const long long r = rem / nu;
    const long long c = rem - r * nu;
    m = fmaxf(m, fabsf(src[f * sf + c * su + r * sv]));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int*>(out), __float_as_int(m));
}

// One thread per output pixel of every frame: out[f][row][col][rgb].
__global__ void k_slice_rgb(const float* __restrict__ src, long long nu, long long nv,
                            long long su, long long sv, long long sf, long long n_total,
                            const float* vmax_dev, float vmax_host,
                            const uint8_t* __restrict__ lut, uint8_t* __restrict__ out) {
  float vmax = vmax_dev ? *vmax_dev : vmax_host;
  if (!(vmax > 0.0f)) vmax = 1.0f;  // all-zero frames (viz/fields.py:64-65)
  const long long per = nu * nv;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long f = i / per;
    const long long rem = i - f * per;
    const long long row = rem / nu;
    const long long c = rem - row * nu;
    const float v = src[f * sf + c * su + (nv - 1 - row) * sv];
    const float t = __fmul_rn(__fadd_rn(__fdiv_rn(v, vmax), 1.0f), 0.5f);
    const float x = __fmul_rn(t, 256.0f);
    int k = x >= 255.0f ? 255 : (x > 0.0f ? (int)x : 0);  // NaN -> 0
    uint8_t* o = out + i * 3;
    o[0] = lut[3 * k];
    o[1] = lut[3 * k + 1];
    o[2] = lut[3 * k + 2];
  }
}

}  // namespace jxf
