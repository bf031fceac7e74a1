// Learned absorbing band: a per-cell MLP that advances the outer cell layer
// of a PEC-walled grid as if the domain continued outward.
//
// Geometry.  Every cell of the outer layer belongs to exactly one face
// f = 2 * a + side (a = normal axis, side 0 = low, 1 = high): the only face it
// lies on; on an edge between the faces of axes a and b, the face whose first
// tangent axis t1 = (a + 1) % 3 is the other face's normal; on a corner, the
// x face.  The band is the 3 outermost layers l = 0, 1, 2 (l = 0 outermost).
//
// Features.  For an outer cell c of face (a, side): the six components
// (Ex, Ey, Ez, eta0 Hx, eta0 Hy, eta0 Hz) at the 3 x 3 stencil of band layers
// l = 0..2 along a and offsets w = -1, 0, 1 along t1 (positions outside the
// grid read 0), index comp * 9 + l * 3 + (w + 1); 54 values v, normalised by
// s = sqrt(mean(v^2) + 1e-30).
//
// Network (one per face).  54 -> 64 -> 64 -> 6, tanh-form GELU, BF16 weights
// and activations, FP32 accumulation in tensor memory (tcgen05.mma kind::f16,
// M = 128 samples per tile), FP32 biases.  Its output o is the normalised
// correction of c's six components after a plain Yee step:
//     X_c <- X_c + s * o        (H components rescaled by 1 / eta0).
#pragma once

#include <cuda_bf16.h>

#include "fdtd_common.cuh"
#include "tc_common.cuh"

namespace jxf {
namespace band {

constexpr int kIn = 54, kInP = 64, kHid = 64, kOut = 6, kOutP = 16;
// FP32 master parameters of one face.
constexpr int kW1 = 0;                      // [64][64] (out, in), in >= 54 zero
constexpr int kB1 = kW1 + kHid * kInP;      // [64]
constexpr int kW2 = kB1 + kHid;             // [64][64] (out, in)
constexpr int kB2 = kW2 + kHid * kHid;      // [64]
constexpr int kW3 = kB2 + kHid;             // [16][64] (out, in), out >= 6 zero
constexpr int kB3 = kW3 + kOutP * kHid;     // [16], >= 6 zero
constexpr int kParams = kB3 + kOutP;        // 9360
// Biases ride in the MMA: the input tile carries a constant 1 in column 54
// (an unused input), the hidden tiles in column 64 of a K = 80 image, and the
// weight images hold the BF16 bias in that column.
constexpr int kOneX = 54;
constexpr int kKH = 80;                     // K of the hidden-activation images
// BF16 operand images of one face (bytes).
constexpr int kImgW1 = 0;          // W1 | b1 at column 54, 64 x 64
constexpr int kImgW2 = 8192;       // W2 | b2 at column 64, 64 x 80
constexpr int kImgW3 = 18432;      // W3 | b3 at column 64, 16 x 80
constexpr int kImgFwdBytes = 20992;
constexpr int kImgW2T = 20992;     // W2^T, 64 x 64 (K = out)
constexpr int kImgW3T = 29184;     // W3^T, 64 x 16 (K = out)
constexpr int kImgBytes = 31232;
constexpr float kEta0 = 376.730313668f;
constexpr int kTile = 128;

struct GridRef {
  float* f[6];
  int nx, ny, nz;
  int pad;
};

__device__ __forceinline__ bool is_pad_param(int k) {
  if (k < kB1) return (k % kInP) >= kIn;
  if (k >= kW3 && k < kB3) return (k - kW3) / kHid >= kOut;
  if (k >= kB3) return (k - kB3) >= kOut;
  return false;
}

__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
constexpr float kGeluC0 = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float kGeluC1 = 0.044715f;

// GELU of two values in packed BF16 arithmetic (the activation is a BF16
// MMA operand anyway): x rounded to BF16, then
//   g = h + h tanh(x (c0 + c0 c1 x^2)),  h = x / 2,
// every product / FMA rounded to BF16, tanh by tanh.approx.bf16x2.
__device__ __forceinline__ uint32_t gelu2(float x0, float x1) {
  const __nv_bfloat162 x = __floats2bfloat162_rn(x0, x1);
  const __nv_bfloat162 c0 = __float2bfloat162_rn(kGeluC0);
  const __nv_bfloat162 c01 = __float2bfloat162_rn(kGeluC0 * kGeluC1);
  const __nv_bfloat162 half = __float2bfloat162_rn(0.5f);
  const __nv_bfloat162 p = __hfma2(__hmul2(x, x), c01, c0);
  const __nv_bfloat162 u = __hmul2(x, p);
  uint32_t ub = *reinterpret_cast<const uint32_t*>(&u), tb;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(tb) : "r"(ub));
  const __nv_bfloat162 t = *reinterpret_cast<const __nv_bfloat162*>(&tb);
  const __nv_bfloat162 h = __hmul2(x, half);
  const __nv_bfloat162 g = __hfma2(h, t, h);
  return *reinterpret_cast<const uint32_t*>(&g);
}
// d GELU / dx of the tanh form, FP32 (training backward).
__device__ __forceinline__ float gelu_grad(float x) {
  const float x2 = x * x;
  const float t = tanh_fast(x * fmaf(kGeluC0 * kGeluC1, x2, kGeluC0));
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * kGeluC0 * fmaf(3.0f * kGeluC1, x2, 1.0f);
}

// Store 64 packed-BF16 values (32 words) as row r of a K-column image.
__device__ __forceinline__ void put_row_packed(unsigned char* img, int r, const uint32_t* w,
                                               int K) {
#pragma unroll
  for (int c = 0; c < 8; ++c)
    *reinterpret_cast<uint4*>(img + tc::img_off(r, 8 * c, K)) =
        make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
}
// Store 64 FP32 values rounded to BF16 as row r of a K-column image.
__device__ __forceinline__ void put_row_f32(unsigned char* img, int r, const float* v, int K) {
  uint32_t w[32];
#pragma unroll
  for (int c = 0; c < 32; ++c) w[c] = tc::pack_bf16(v[2 * c], v[2 * c + 1]);
  put_row_packed(img, r, w, K);
}
// Column r (sample r) of a 64 x 128 image from 64 packed-BF16 values.
__device__ __forceinline__ void put_col_packed(unsigned char* imgT, int r, const uint32_t* w) {
#pragma unroll
  for (int q = 0; q < 32; ++q) {
    *reinterpret_cast<uint16_t*>(imgT + tc::img_off(2 * q, r, 128)) = (uint16_t)(w[q] & 0xFFFFu);
    *reinterpret_cast<uint16_t*>(imgT + tc::img_off(2 * q + 1, r, 128)) = (uint16_t)(w[q] >> 16);
  }
}
// Constant tail of a 128 x 80 hidden image: column 64 = 1, 65..79 = 0.
__device__ __forceinline__ void init_hidden_tail(unsigned char* img, int tid, int nthreads) {
  for (int r = tid; r < kTile; r += nthreads) {
    *reinterpret_cast<uint4*>(img + tc::img_off(r, 64, kKH)) = make_uint4(0x3F80u, 0u, 0u, 0u);
    *reinterpret_cast<uint4*>(img + tc::img_off(r, 72, kKH)) = make_uint4(0u, 0u, 0u, 0u);
  }
}

// Raw stencil of an outer cell (v[54], H scaled by eta0); returns s.  ctr
// receives the cell's own six components as stored (unscaled).
// Every load is issued before any value is used: positions outside the grid
// along the tangent are loaded from the clamped (in-grid) neighbour and then
// replaced by zero, so no load sits behind a branch and a thread keeps all
// 54 (x, y faces) or 18 (z faces) loads in flight at once.
__device__ __forceinline__ float gather(const GridRef& gref, int cell, int face, float* v,
                                        float* ctr) {
  const GridRef g = gref;
  const int a = face >> 1, side = face & 1;
  float ss = 0.0f;
  if (a == 2 && (g.nz & 3) == 0) {
    // z faces: the three band layers of a row are one aligned 16-byte load
    const long long row = (long long)cell - (side ? g.nz - 1 : 0) + (side ? g.nz - 4 : 0);
    const int x = cell / (g.nz * g.ny);
    const long long sx = (long long)g.ny * g.nz;
    float4 q[3][6];
#pragma unroll
    for (int w = 0; w < 3; ++w) {
      const int xw = min(max(x + w - 1, 0), g.nx - 1);
#pragma unroll
      for (int comp = 0; comp < 6; ++comp)
        q[w][comp] = __ldg(reinterpret_cast<const float4*>(g.f[comp] + row + (xw - x) * sx));
    }
#pragma unroll
    for (int comp = 0; comp < 6; ++comp) ctr[comp] = side ? q[1][comp].w : q[1][comp].x;
#pragma unroll
    for (int w = 0; w < 3; ++w) {
      const bool in = x + w - 1 >= 0 && x + w - 1 < g.nx;
#pragma unroll
      for (int comp = 0; comp < 6; ++comp) {
        const float sc = comp >= 3 ? kEta0 : 1.0f;
        const float4 r = q[w][comp];
        const float l0 = in ? (side ? r.w : r.x) * sc : 0.0f;
        const float l1 = in ? (side ? r.z : r.y) * sc : 0.0f;
        const float l2 = in ? (side ? r.y : r.z) * sc : 0.0f;
        v[comp * 9 + 0 * 3 + w] = l0;
        v[comp * 9 + 1 * 3 + w] = l1;
        v[comp * 9 + 2 * 3 + w] = l2;
        ss = fmaf(l0, l0, fmaf(l1, l1, fmaf(l2, l2, ss)));
      }
    }
    return sqrtf(ss * (1.0f / kIn) + 1e-30f);
  }
  const int t1 = a == 2 ? 0 : a + 1;
  const int z = cell % g.nz;
  const int y = (cell / g.nz) % g.ny;
  const int x = cell / (g.nz * g.ny);
  const long long sx = (long long)g.ny * g.nz;
  const long long sa = a == 0 ? sx : (a == 1 ? (long long)g.nz : 1ll);
  const long long st = t1 == 0 ? sx : (t1 == 1 ? (long long)g.nz : 1ll);
  const int ct = t1 == 0 ? x : (t1 == 1 ? y : z);
  const int nt = t1 == 0 ? g.nx : (t1 == 1 ? g.ny : g.nz);
  float raw[3][3][6];
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    const long long dn = side ? -l * sa : l * sa;
#pragma unroll
    for (int w = 0; w < 3; ++w) {
      const int cw = min(max(ct + w - 1, 0), nt - 1);
      const long long idx = (long long)cell + dn + (long long)(cw - ct) * st;
#pragma unroll
      for (int comp = 0; comp < 6; ++comp) raw[l][w][comp] = __ldg(g.f[comp] + idx);
    }
  }
#pragma unroll
  for (int comp = 0; comp < 6; ++comp) ctr[comp] = raw[0][1][comp];
#pragma unroll
  for (int l = 0; l < 3; ++l) {
#pragma unroll
    for (int w = 0; w < 3; ++w) {
      const bool in = ct + w - 1 >= 0 && ct + w - 1 < nt;
#pragma unroll
      for (int comp = 0; comp < 6; ++comp) {
        float val = in ? raw[l][w][comp] : 0.0f;
        if (comp >= 3) val *= kEta0;
        v[comp * 9 + l * 3 + w] = val;
        ss = fmaf(val, val, ss);
      }
    }
  }
  return sqrtf(ss * (1.0f / kIn) + 1e-30f);
}

// This thread waits for `bar`; true if the wait gave up (recorded in err).
__device__ __forceinline__ bool wait_one(uint64_t* bar, uint32_t phase, unsigned long long ns,
                                         int* err, int where) {
  const bool ok = mbar_wait_bounded(bar, phase, ns);
  if (!ok) report_error(err, ERR_TIMEOUT_BASE | 0x100 | where, blockIdx.x, blockIdx.y, threadIdx.x);
  return !ok;
}

// All threads wait for `bar`; false (for every thread) if any timed out.
__device__ __forceinline__ bool wait_all(uint64_t* bar, uint32_t phase, unsigned long long ns,
                                        int* err, int where) {
  const bool ok = mbar_wait_bounded(bar, phase, ns);
  if (!ok) report_error(err, ERR_TIMEOUT_BASE | 0x100 | where, blockIdx.x, blockIdx.y, threadIdx.x);
  return __syncthreads_or(!ok) == 0;
}

// ---------------------------------------------------------------------------
// Inference (tensor cores).  One CTA = 4 warps; thread t owns row t of each
// 128-cell tile.  Tiles are single-face; a CTA works through a contiguous
// range of tiles and reloads the face's weights when the face changes.  One
// activation image (X, then G1, then G2; each MMA has completed before the
// next epilogue overwrites it) and 64 TMEM columns (Z1, then Z2, then O).
// The launch bound keeps 5 CTAs per SM (<= 102 registers), the residency
// that shared memory and TMEM allow and that the grid is sized for.
enum InferSrc : int { SRC_GRIDS = 0, SRC_ROWS = 1 };

struct InferArgs {
  const GridRef* grids;
  const int2* cells;        // [n_tiles * 128]: (cell or row, grid); x < 0 = padding
  const int* tile_face;     // [n_tiles]
  int n_tiles;
  const unsigned char* wimg;  // [6][kImgBytes]
  const float* params;        // [6][kParams]
  // [n_tiles * 128][6]: SRC_GRIDS the corrected values of the six
  // components of each cell, SRC_ROWS the network outputs s * o
  float* delta;
  const float* rows;          // SRC_ROWS: [n][54] normalised features
  int* err;
  unsigned long long wait_ns;
  // fault injection for the failure-detection tests: every CTA leaves the
  // first MMA of its first tile unissued, so its bounded waits run out
  int drop_first_mma;
};

constexpr int kInfOffA = 0;        // activation image, 128 x 80
constexpr int kInfOffW = 20480;    // W1 | W2 | W3 images
constexpr int kInfOffBar = kInfOffW + kImgFwdBytes;
constexpr int kInfSmem = kInfOffBar + 16;
constexpr int kInfTmemCols = 64;

template <int SRC>
__global__ void __launch_bounds__(128, 5) k_band_infer(const __grid_constant__ InferArgs p) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* bufA = smem + kInfOffA;
  unsigned char* bufW = smem + kInfOffW;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kInfOffBar);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kInfOffBar + 8);
  const int tid = threadIdx.x;
  const int t0 = (int)((long long)blockIdx.x * p.n_tiles / gridDim.x);
  const int t1 = (int)((long long)(blockIdx.x + 1) * p.n_tiles / gridDim.x);
  if (t0 >= t1) return;
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_barrier_init();
  }
  init_hidden_tail(bufA, tid, 128);
  if (tid < 32) {
    tc::tmem_alloc(tslot, kInfTmemCols);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tm = *tslot;
  const uint32_t lane_base = tc::taddr(tm, (tid >> 5) * 32, 0);
  const uint32_t sA = smem_u32(bufA), sW = smem_u32(bufW);
  constexpr uint32_t id64 = tc::idesc_bf16(128, 64), id16 = tc::idesc_bf16(128, 16);
  // Every thread waits on the MMA barrier itself (so no CTA barrier follows
  // an MMA); a wait that gave up is voted at the next CTA barrier, before
  // the next MMA is issued.  Three CTA barriers per tile.
  uint32_t phase = 0;
  int cur_face = -1;
  bool ok = true, timed = false;
  int2 cg_next = p.cells[t0 * kTile + tid];  // (cell, grid) of the next tile, loaded a tile early
  for (int t = t0; t < t1 && ok; ++t) {
    const int face = p.tile_face[t];
    const int2 cg = cg_next;
    if (t + 1 < t1) cg_next = p.cells[(t + 1) * kTile + tid];
    if (face != cur_face) {
      const uint4* src = reinterpret_cast<const uint4*>(p.wimg + (size_t)face * kImgBytes);
      uint4* dst = reinterpret_cast<uint4*>(bufW);
      for (int k = tid; k < kImgFwdBytes / 16; k += 128) dst[k] = __ldg(src + k);
      cur_face = face;
    }
    const int i = t * kTile + tid;
    float v[kInP];
    float ctr[6];  // SRC_GRIDS: the cell's six components before the correction
    float s = 0.0f;
    if (cg.x >= 0) {
      if (SRC == SRC_GRIDS) {
        s = gather(p.grids[cg.y], cg.x, face, v, ctr);
        const float inv = 1.0f / s;
#pragma unroll
        for (int k = 0; k < kIn; ++k) v[k] *= inv;
      } else {
        s = 1.0f;
#pragma unroll
        for (int k = 0; k < kIn; ++k) v[k] = p.rows[(size_t)cg.x * kIn + k];
      }
    } else {
#pragma unroll
      for (int k = 0; k < kIn; ++k) v[k] = 0.0f;
    }
    v[kOneX] = 1.0f;
#pragma unroll
    for (int k = kOneX + 1; k < kInP; ++k) v[k] = 0.0f;
    put_row_f32(bufA, tid, v, kKH);
    fence_proxy_async();
    tc::fence_before_sync();
    if (__syncthreads_or(timed)) {
      ok = false;
      break;
    }
    // layer 1: Z1 = [X 1] [W1 b1]^T
    if (tid == 0 && !(p.drop_first_mma && t == t0)) {
      tc::fence_after_sync();
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        tc::mma(tm, tc::img_desc(sA, kKH, kk), tc::img_desc(sW + kImgW1, 64, kk), id64, kk);
      tc::commit(bar);
    }
    timed |= wait_one(bar, phase, p.wait_ns, p.err, 1);
    phase ^= 1;
    tc::fence_after_sync();
    uint32_t g[32];
    {
      float z[32];
#pragma unroll
      for (int hlf = 0; hlf < 2; ++hlf) {
        tc::ld32(lane_base + 32 * hlf, z);
#pragma unroll
        for (int c = 0; c < 16; ++c) g[16 * hlf + c] = gelu2(z[2 * c], z[2 * c + 1]);
      }
    }
    put_row_packed(bufA, tid, g, kKH);
    fence_proxy_async();
    tc::fence_before_sync();
    if (__syncthreads_or(timed)) {
      ok = false;
      break;
    }
    // layer 2: Z2 = [G1 1] [W2 b2]^T
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int kk = 0; kk < 5; ++kk)
        tc::mma(tm, tc::img_desc(sA, kKH, kk), tc::img_desc(sW + kImgW2, kKH, kk), id64, kk);
      tc::commit(bar);
    }
    timed |= wait_one(bar, phase, p.wait_ns, p.err, 2);
    phase ^= 1;
    tc::fence_after_sync();
    {
      float z[32];
#pragma unroll
      for (int hlf = 0; hlf < 2; ++hlf) {
        tc::ld32(lane_base + 32 * hlf, z);
#pragma unroll
        for (int c = 0; c < 16; ++c) g[16 * hlf + c] = gelu2(z[2 * c], z[2 * c + 1]);
      }
    }
    put_row_packed(bufA, tid, g, kKH);
    fence_proxy_async();
    tc::fence_before_sync();
    if (__syncthreads_or(timed)) {
      ok = false;
      break;
    }
    // layer 3: O = [G2 1] [W3 b3]^T  (columns 0..15)
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int kk = 0; kk < 5; ++kk)
        tc::mma(tm, tc::img_desc(sA, kKH, kk), tc::img_desc(sW + kImgW3, kKH, kk), id16, kk);
      tc::commit(bar);
    }
    timed |= wait_one(bar, phase, p.wait_ns, p.err, 3);
    phase ^= 1;
    tc::fence_after_sync();
    // Every thread saw the MMA complete before it reads O, so the next
    // tile's image and weight writes cannot race the MMAs of this one; the
    // next MMA is issued after the next CTA barrier, when every thread has
    // read its rows of O.
    tc::ld16(lane_base, v);
    if (cg.x >= 0 && !timed) {
      float* d = p.delta + (size_t)i * kOut;
      if (SRC == SRC_GRIDS) {
        // X_c + s o (H rescaled by 1 / eta0), rounded as separate steps
#pragma unroll
        for (int o = 0; o < kOut; ++o) {
          const float so = __fmul_rn(s, v[o]);
          d[o] = __fadd_rn(ctr[o], o >= 3 ? __fmul_rn(so, 1.0f / kEta0) : so);
        }
      } else {
#pragma unroll
        for (int o = 0; o < kOut; ++o) d[o] = s * v[o];
      }
    }
  }
  tc::fence_before_sync();
  if (__syncthreads_or(timed)) ok = false;
  if (!ok) {
    // the commit that timed out may still be outstanding: give it one more bounded wait
    mbar_wait_bounded(bar, phase ^ 1, p.wait_ns);
  }
  if (tid < 32) tc::tmem_dealloc(tm, kInfTmemCols);
}

// X_c <- the corrected values the inference wrote (padding entries skipped).
// A separate launch, because the stencils of other tiles read the
// uncorrected outer cells; the inference formed X_c + s o from the values
// it gathered, so the fields are only written here, never read (on z faces
// every component of a cell is its own DRAM sector).  The grid record is
// copied into registers once (through a reference into global memory every
// store would force the field pointers to be reloaded).  If the inference
// reported an error (a wait that gave up leaves tiles unwritten), nothing is
// stored: the fields keep the plain Yee step.
__global__ void k_band_apply(const GridRef* grids, const int2* cells, int n, const float* xnew,
                             const int* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (__ldcg(err) != 0) return;
  const int2 cg = cells[i];
  if (cg.x < 0) return;
  const GridRef g = grids[cg.y];
  float d[kOut];
#pragma unroll
  for (int c = 0; c < 6; ++c) d[c] = xnew[(size_t)i * kOut + c];
#pragma unroll
  for (int c = 0; c < 6; ++c) g.f[c][cg.x] = d[c];
}

// ---------------------------------------------------------------------------
// Training samples.  For the outer cells of a truncated grid T (its state
// after one plain step from the reference state at step n) and the reference
// state at step n + 1 (box of a larger grid at offset o):
//   row  = normalised features (BF16, 64 wide, zero padded)
//   tgt  = (X_ref(n+1) - X_T) / s   (H scaled by eta0)
//   w    = s^2
struct CollectArgs {
  GridRef t;
  const float* ref[6];
  int rnx, rny, rnz;
  int ox, oy, oz;
  const int* cells;   // entries (cell of T), grouped by face
  int first[7];       // entries of face f: [first[f], first[f+1])
  long long base[6];  // destination row of the first entry of face f
  __nv_bfloat16* feat[6];
  float* tgt[6];
  float* w[6];
};

__global__ void k_band_collect(const __grid_constant__ CollectArgs p) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= p.first[6]) return;
  int f = 0;
  while (e >= p.first[f + 1]) ++f;
  const int cell = p.cells[e];
  float v[kIn];
  float ctr[6];
  const float s = gather(p.t, cell, f, v, ctr);
  const float inv = 1.0f / s;
  const long long row = p.base[f] + (e - p.first[f]);
  __nv_bfloat16* fr = p.feat[f] + row * kInP;
  for (int k = 0; k < kInP; ++k) fr[k] = __float2bfloat16_rn(k < kIn ? v[k] * inv : 0.0f);
  const int z = cell % p.t.nz;
  const int y = (cell / p.t.nz) % p.t.ny;
  const int x = cell / (p.t.nz * p.t.ny);
  const long long ridx = ((long long)(x + p.ox) * p.rny + (y + p.oy)) * p.rnz + (z + p.oz);
  for (int c = 0; c < 6; ++c) {
    const float sc = c >= 3 ? kEta0 : 1.0f;
    p.tgt[f][row * kOut + c] = (p.ref[c][ridx] * sc - p.t.f[c][cell] * sc) * inv;
  }
  p.w[f][row] = s * s;
}

// ---------------------------------------------------------------------------
// Training step (tensor cores): forward, weighted MSE, backward and weight
// gradients for 128-sample tiles.  Block (b, f) works on face f's tiles
// b, b + gridDim.x, ...  Sample j of a tile is row
//   random mode:     hash(seed, j) mod count[f]
//   sequential mode: j (rows >= count[f] are padding with weight 0).
// Loss of face f = scale[f] * sum_j w_j |o_j - tgt_j|^2.  Weight gradients
// accumulate in TMEM across the block's tiles and are added to `grad` once.
struct TrainArgs {
  const __nv_bfloat16* feat[6];
  const float* tgt[6];
  const float* w[6];
  long long count[6];   // rows available (sequential) / to draw from (random)
  int tiles[6];         // tiles of face f in this pass
  float scale[6];
  int random;
  unsigned long long seed;
  const unsigned char* wimg;
  const float* params;
  float* grad;          // [6][kParams]
  float* loss;          // [6]
  int* err;
  unsigned long long wait_ns;
};

// smem map of the training kernel (bytes).  The A operands dO^T, dZ2^T and
// dZ1^T have fewer than 128 meaningful rows; the MMA reads the rows beyond
// them from the buffers that follow (D rows it never uses), so these three
// sit first, with at least 28 KB of the CTA's own shared memory after each.
constexpr int kTrOffDOT = 0;          // 16 x 128 (rows 0..5 used)
constexpr int kTrOffDZ2T = 4096;      // 64 x 128
constexpr int kTrOffDZ1T = 20480;     // 64 x 128
constexpr int kTrOffX = 36864;        // 128 x 64 (column 54 = 1)
constexpr int kTrOffXT = 53248;       // 64 x 128
constexpr int kTrOffG1 = 69632;       // 128 x 80 (column 64 = 1)
constexpr int kTrOffG1T = 90112;      // 64 x 128
constexpr int kTrOffG2 = 106496;      // 128 x 80 (column 64 = 1)
constexpr int kTrOffG2T = 126976;     // 64 x 128
constexpr int kTrOffDO = 143360;      // 128 x 16
constexpr int kTrOffDZ2 = 147456;     // 128 x 64
constexpr int kTrOffW = 163840;       // full image
constexpr int kTrOffF = kTrOffW + kImgBytes;   // gb (144), loss
constexpr int kTrOffBar = kTrOffF + 1280;
constexpr int kTrSmem = kTrOffBar + 16;
static_assert(kTrSmem <= 227 * 1024, "training kernel shared memory");
// TMEM columns
constexpr int kTmZ1 = 0, kTmZ2 = 64, kTmO = 128, kTmDG2 = 160, kTmDG1 = 224, kTmDW3 = 288,
              kTmDW2 = 352, kTmDW1 = 416;
constexpr int kTrTmemCols = 512;

__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return x;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(128, 1) k_band_train(const __grid_constant__ TrainArgs p) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int f = blockIdx.y;
  const int tid = threadIdx.x;
  const int n_tiles = p.tiles[f];
  if ((int)blockIdx.x >= n_tiles) return;
  unsigned char* sm = smem;
  float* gb = reinterpret_cast<float*>(sm + kTrOffF);
  float* lsum = gb + 144;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kTrOffBar);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kTrOffBar + 8);
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_barrier_init();
  }
  {
    const uint4* src = reinterpret_cast<const uint4*>(p.wimg + (size_t)f * kImgBytes);
    uint4* dst = reinterpret_cast<uint4*>(sm + kTrOffW);
    for (int k = tid; k < kImgBytes / 16; k += 128) dst[k] = __ldg(src + k);
    for (int k = tid; k < 144; k += 128) gb[k] = 0.0f;
    if (tid == 0) *lsum = 0.0f;
    init_hidden_tail(sm + kTrOffG1, tid, 128);
    init_hidden_tail(sm + kTrOffG2, tid, 128);
  }
  if (tid < 32) {
    tc::tmem_alloc(tslot, kTrTmemCols);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tm = *tslot;
  const uint32_t lb = tc::taddr(tm, (tid >> 5) * 32, 0);
  const uint32_t s0 = smem_u32(sm);
  const uint32_t sW = s0 + kTrOffW;
  constexpr uint32_t id64 = tc::idesc_bf16(128, 64), id16 = tc::idesc_bf16(128, 16);
  const __nv_bfloat16* feat = p.feat[f];
  const float* tgt = p.tgt[f];
  const float* wt = p.w[f];
  const long long cnt = p.count[f];
  const float scale = p.scale[f];
  uint32_t phase = 0;
  bool ok = true;
  bool first = true;
  float v[64], u[64];
  uint32_t g[32];
  for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
    const long long j = (long long)t * kTile + tid;
    long long row;
    if (p.random)
      row = cnt > 0 ? (long long)(mix64(p.seed ^ mix64((unsigned long long)j * 6 + f + 1)) %
                                  (unsigned long long)cnt)
                    : -1;
    else
      row = j < cnt ? j : -1;
    float w = 0.0f, tg[kOut];
    if (row >= 0) {
      const uint4* fr = reinterpret_cast<const uint4*>(feat + row * kInP);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const uint4 q = __ldg(fr + c);
        const uint32_t qq[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const __nv_bfloat162 b2 = *reinterpret_cast<const __nv_bfloat162*>(&qq[h]);
          v[8 * c + 2 * h] = __low2float(b2);
          v[8 * c + 2 * h + 1] = __high2float(b2);
        }
      }
      w = wt[row];
#pragma unroll
      for (int o = 0; o < kOut; ++o) tg[o] = tgt[row * kOut + o];
    } else {
#pragma unroll
      for (int k = 0; k < 64; ++k) v[k] = 0.0f;
#pragma unroll
      for (int o = 0; o < kOut; ++o) tg[o] = 0.0f;
    }
    v[kOneX] = 1.0f;
#pragma unroll
    for (int k = kOneX + 1; k < 64; ++k) v[k] = 0.0f;
    put_row_f32(sm + kTrOffX, tid, v, 64);
    tc::put_col(sm + kTrOffXT, tid, v, 64);
    fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    // forward layer 1
    if (tid == 0) {
      tc::fence_after_sync();
      for (int kk = 0; kk < 4; ++kk)
        tc::mma(tm + kTmZ1, tc::img_desc(s0 + kTrOffX, 64, kk),
                tc::img_desc(sW + kImgW1, 64, kk), id64, kk);
      tc::commit(bar);
    }
    ok = wait_all(bar, phase, p.wait_ns, p.err, 11);
    phase ^= 1;
    if (!ok) break;
    tc::fence_after_sync();
#pragma unroll
    for (int hlf = 0; hlf < 2; ++hlf) {
      tc::ld32(lb + kTmZ1 + 32 * hlf, u);
#pragma unroll
      for (int c = 0; c < 16; ++c) g[16 * hlf + c] = gelu2(u[2 * c], u[2 * c + 1]);
    }
    put_row_packed(sm + kTrOffG1, tid, g, kKH);
    put_col_packed(sm + kTrOffG1T, tid, g);
    fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    // forward layer 2
    if (tid == 0) {
      tc::fence_after_sync();
      for (int kk = 0; kk < 5; ++kk)
        tc::mma(tm + kTmZ2, tc::img_desc(s0 + kTrOffG1, kKH, kk),
                tc::img_desc(sW + kImgW2, kKH, kk), id64, kk);
      tc::commit(bar);
    }
    ok = wait_all(bar, phase, p.wait_ns, p.err, 12);
    phase ^= 1;
    if (!ok) break;
    tc::fence_after_sync();
#pragma unroll
    for (int hlf = 0; hlf < 2; ++hlf) {
      tc::ld32(lb + kTmZ2 + 32 * hlf, u);
#pragma unroll
      for (int c = 0; c < 16; ++c) g[16 * hlf + c] = gelu2(u[2 * c], u[2 * c + 1]);
    }
    put_row_packed(sm + kTrOffG2, tid, g, kKH);
    put_col_packed(sm + kTrOffG2T, tid, g);
    fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    // forward layer 3
    if (tid == 0) {
      tc::fence_after_sync();
      for (int kk = 0; kk < 5; ++kk)
        tc::mma(tm + kTmO, tc::img_desc(s0 + kTrOffG2, kKH, kk),
                tc::img_desc(sW + kImgW3, kKH, kk), id16, kk);
      tc::commit(bar);
    }
    ok = wait_all(bar, phase, p.wait_ns, p.err, 13);
    phase ^= 1;
    if (!ok) break;
    tc::fence_after_sync();
    tc::ld16(lb + kTmO, v);
    {
      float d[16], l = 0.0f;
#pragma unroll
      for (int o = 0; o < 16; ++o) d[o] = 0.0f;
#pragma unroll
      for (int o = 0; o < kOut; ++o) {
        const float r = v[o] - tg[o];
        l = fmaf(w * r, r, l);
        d[o] = 2.0f * scale * w * r;
      }
      // dO row (K = 16 image) and dO^T column (rows 0..5)
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        uint4 q;
        q.x = tc::pack_bf16(d[8 * c + 0], d[8 * c + 1]);
        q.y = tc::pack_bf16(d[8 * c + 2], d[8 * c + 3]);
        q.z = tc::pack_bf16(d[8 * c + 4], d[8 * c + 5]);
        q.w = tc::pack_bf16(d[8 * c + 6], d[8 * c + 7]);
        *reinterpret_cast<uint4*>(sm + kTrOffDO + tc::img_off(tid, 8 * c, 16)) = q;
      }
      tc::put_col(sm + kTrOffDOT, tid, d, kOut);
      l = warp_sum(l * scale);
      if ((tid & 31) == 0) atomicAdd(lsum, l);
#pragma unroll
      for (int o = 0; o < kOut; ++o) {
        const float sdo = warp_sum(d[o]);
        if ((tid & 31) == 0) atomicAdd(&gb[128 + o], sdo);
      }
    }
    fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    // backward: dG2 = dO W3 ; dW3 += dO^T G2
    if (tid == 0) {
      tc::fence_after_sync();
      tc::mma(tm + kTmDG2, tc::img_desc(s0 + kTrOffDO, 16, 0),
              tc::img_desc(sW + kImgW3T, 16, 0), id64, 0);
      for (int kk = 0; kk < 8; ++kk)
        tc::mma(tm + kTmDW3, tc::img_desc(s0 + kTrOffDOT, 128, kk),
                tc::img_desc(s0 + kTrOffG2T, 128, kk), id64, (first && kk == 0) ? 0 : 1);
      tc::commit(bar);
    }
    ok = wait_all(bar, phase, p.wait_ns, p.err, 14);
    phase ^= 1;
    if (!ok) break;
    tc::fence_after_sync();
    tc::ld32(lb + kTmDG2, v);
    tc::ld32(lb + kTmDG2 + 32, v + 32);
    tc::ld32(lb + kTmZ2, u);
    tc::ld32(lb + kTmZ2 + 32, u + 32);
#pragma unroll
    for (int k = 0; k < 64; ++k) v[k] *= gelu_grad(u[k]);
    put_row_f32(sm + kTrOffDZ2, tid, v, 64);
    tc::put_col(sm + kTrOffDZ2T, tid, v, 64);
#pragma unroll 4
    for (int k = 0; k < 64; ++k) {
      const float sk = warp_sum(v[k]);
      if ((tid & 31) == 0) atomicAdd(&gb[64 + k], sk);
    }
    fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    // dG1 = dZ2 W2 ; dW2 += dZ2^T G1
    if (tid == 0) {
      tc::fence_after_sync();
      for (int kk = 0; kk < 4; ++kk)
        tc::mma(tm + kTmDG1, tc::img_desc(s0 + kTrOffDZ2, 64, kk),
                tc::img_desc(sW + kImgW2T, 64, kk), id64, kk);
      for (int kk = 0; kk < 8; ++kk)
        tc::mma(tm + kTmDW2, tc::img_desc(s0 + kTrOffDZ2T, 128, kk),
                tc::img_desc(s0 + kTrOffG1T, 128, kk), id64, (first && kk == 0) ? 0 : 1);
      tc::commit(bar);
    }
    ok = wait_all(bar, phase, p.wait_ns, p.err, 15);
    phase ^= 1;
    if (!ok) break;
    tc::fence_after_sync();
    tc::ld32(lb + kTmDG1, v);
    tc::ld32(lb + kTmDG1 + 32, v + 32);
    tc::ld32(lb + kTmZ1, u);
    tc::ld32(lb + kTmZ1 + 32, u + 32);
#pragma unroll
    for (int k = 0; k < 64; ++k) v[k] *= gelu_grad(u[k]);
    tc::put_col(sm + kTrOffDZ1T, tid, v, 64);
#pragma unroll 4
    for (int k = 0; k < 64; ++k) {
      const float sk = warp_sum(v[k]);
      if ((tid & 31) == 0) atomicAdd(&gb[k], sk);
    }
    fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    // dW1 += dZ1^T X
    if (tid == 0) {
      tc::fence_after_sync();
      for (int kk = 0; kk < 8; ++kk)
        tc::mma(tm + kTmDW1, tc::img_desc(s0 + kTrOffDZ1T, 128, kk),
                tc::img_desc(s0 + kTrOffXT, 128, kk), id64, (first && kk == 0) ? 0 : 1);
      tc::commit(bar);
    }
    ok = wait_all(bar, phase, p.wait_ns, p.err, 16);
    phase ^= 1;
    first = false;
  }
  tc::fence_before_sync();
  __syncthreads();
  if (ok) {
    tc::fence_after_sync();
    float* gr = p.grad + (size_t)f * kParams;
    if (tid < 64) {  // warps 0 and 1 hold rows 0..63 of the weight gradients
      tc::ld32(lb + kTmDW1, v);
      tc::ld32(lb + kTmDW1 + 32, v + 32);
      tc::ld32(lb + kTmDW2, u);
      tc::ld32(lb + kTmDW2 + 32, u + 32);
      for (int k = 0; k < kIn; ++k) atomicAdd(&gr[kW1 + tid * kInP + k], v[k]);
      for (int k = 0; k < 64; ++k) atomicAdd(&gr[kW2 + tid * kHid + k], u[k]);
      tc::ld32(lb + kTmDW3, v);
      tc::ld32(lb + kTmDW3 + 32, v + 32);
      if (tid < kOut)
        for (int k = 0; k < 64; ++k) atomicAdd(&gr[kW3 + tid * kHid + k], v[k]);
    }
    for (int k = tid; k < 144; k += 128) {
      const int dst = k < 64 ? kB1 + k : (k < 128 ? kB2 + k - 64 : kB3 + k - 128);
      if (k < 128 || k - 128 < kOut) atomicAdd(&gr[dst], gb[k]);
    }
    if (tid == 0) atomicAdd(&p.loss[f], *lsum);
  } else {
    mbar_wait_bounded(bar, phase ^ 1, p.wait_ns);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (tid < 32) tc::tmem_dealloc(tm, kTrTmemCols);
}

// Adam on the FP32 master parameters; padding entries stay zero.
__global__ void k_band_adam(float* w, const float* g, float* m1, float* m2, int n, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (is_pad_param(i % kParams)) {
    w[i] = 0.0f;
    return;
  }
  const float gi = g[i];
  const float a = b1 * m1[i] + (1.0f - b1) * gi;
  const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  w[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

// Decode (r, k) from a byte offset inside a K-major image with K columns.
__device__ __forceinline__ void img_rc(int b, int K, int& r, int& k) {
  const int rem = b % (K * 16);
  r = (b / (K * 16)) * 8 + (rem % 128) / 16;
  k = (rem / 128) * 8 + (rem % 16) / 2;
}

// BF16 operand images of every face from the master parameters.
__global__ void k_band_pack(const float* params, unsigned char* wimg) {
  const int f = blockIdx.y;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;  // bf16 element of the image
  if (e >= kImgBytes / 2) return;
  const float* pf = params + (size_t)f * kParams;
  const int byte = e * 2;
  int r, k;
  float val = 0.0f;
  if (byte < kImgW2) {
    img_rc(byte - kImgW1, 64, r, k);  // W1 | b1 at column 54
    val = k < kIn ? pf[kW1 + r * kInP + k] : (k == kOneX ? pf[kB1 + r] : 0.0f);
  } else if (byte < kImgW3) {
    img_rc(byte - kImgW2, kKH, r, k);  // W2 | b2 at column 64
    val = k < kHid ? pf[kW2 + r * kHid + k] : (k == kHid ? pf[kB2 + r] : 0.0f);
  } else if (byte < kImgW2T) {
    img_rc(byte - kImgW3, kKH, r, k);  // W3 | b3 at column 64
    if (r < kOut) val = k < kHid ? pf[kW3 + r * kHid + k] : (k == kHid ? pf[kB3 + r] : 0.0f);
  } else if (byte < kImgW3T) {
    img_rc(byte - kImgW2T, 64, r, k);  // r = input unit, k = output unit
    val = pf[kW2 + k * kHid + r];
  } else {
    img_rc(byte - kImgW3T, 16, r, k);  // r = hidden unit, k = output
    if (k < kOut) val = pf[kW3 + k * kHid + r];
  }
  *reinterpret_cast<__nv_bfloat16*>(wimg + (size_t)f * kImgBytes + byte) =
      __float2bfloat16_rn(val);
}

}  // namespace band
}  // namespace jxf
