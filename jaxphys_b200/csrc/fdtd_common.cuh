// Shared device-side helpers for the FDTD kernels (sm_100a).
//
//  - the kernel parameter blocks shared by the 3D kernels
//  - mbarrier / TMA (cp.async.bulk.tensor) wrappers in inline PTX
//  - bounded waits: every spin on an mbarrier gives up after a time limit,
//    records where it gave up in a device error word and lets the block
//    return, so a lost transfer can never hang the GPU.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace jxf {

// chunk word of a blk_list entry: x chunk index | flags
constexpr int BLK_CHUNK_MASK = 0x3fffffff;
constexpr int BLK_SLAB_FIRST = 0x40000000;

enum Mode : int { MODE_ABSORB = 0, MODE_PERIODIC = 1, MODE_PEC = 2, MODE_CPML = 3 };

// psi array order (component of the field, then differencing axis)
enum PsiId : int {
  PSI_HXY = 0, PSI_HXZ, PSI_HYZ, PSI_HYX, PSI_HZX, PSI_HZY,
  PSI_EXY, PSI_EXZ, PSI_EYZ, PSI_EYX, PSI_EZX, PSI_EZY, PSI_COUNT
};
// table order per axis
enum TabId : int { TAB_BE = 0, TAB_CE, TAB_IKE, TAB_BH, TAB_CH, TAB_IKH, TAB_COUNT };

// Device error word values (high bits: code, low bits: where).
constexpr int ERR_TIMEOUT_BASE = 0x40000000;

// One soft-source entry of the per-block lists used by the TMA kernel.
struct SrcEntry {
  int x;       // plane
  int off;     // (y - y0) * TZ + (z - z0) inside the block tile
  int comp;    // 0..2
  int wave;    // waveform row
  float amp;
  int pad0, pad1, pad2;
};

// Grouped source entries for the generic path: one group per distinct cell,
// applied in list order.
struct SrcCell {
  long long cell;
  int comp;
  int first;   // index into SrcTerm array
  int count;
  int pad;
};
struct SrcTerm {
  float amp;
  int wave;
};

// Unsigned division of 32-bit numerators by a divisor fixed per launch:
// q = (umulhi(n, m) + n) >> s with s = ceil(log2 d) and
// m = floor(2^32 (2^s - d) / d) + 1 (the round-up multiply-high method,
// Granlund & Montgomery 1994 / Warren, Hacker's Delight 10-9); exact for every
// n < 2^32 (checked exhaustively for the divisor classes used).
struct FastDiv {
  uint32_t d, m, s;
};
inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f{d, 0u, 0u};
  while ((1ull << f.s) < d) ++f.s;
  f.m = (uint32_t)((((1ull << 32) * ((1ull << f.s) - d)) / d + 1ull) & 0xFFFFFFFFull);
  return f;
}
__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f) {
  return (uint32_t)(((unsigned long long)__umulhi(n, f.m) + n) >> f.s);
}
// (x, y, z) of linear index idx = (x ny + y) nz + z.
__device__ __forceinline__ void decode_cell(long long idx, int nz, int ny, bool idx32,
                                            const FastDiv& dnz, const FastDiv& dny, int& x,
                                            int& y, int& z) {
  if (idx32) {
    const uint32_t u = (uint32_t)idx;
    const uint32_t t = fdiv(u, dnz);
    const uint32_t xx = fdiv(t, dny);
    z = (int)(u - t * (uint32_t)nz);
    y = (int)(t - xx * (uint32_t)ny);
    x = (int)xx;
  } else {
    z = (int)(idx % nz);
    const long long t = idx / nz;
    y = (int)(t % ny);
    x = (int)(t / ny);
  }
}

struct CpmlDev {
  const float* tab[3][TAB_COUNT];  // per axis, length n_axis
  int L[3];                        // slab storage extent per axis
  int P[3];                        // slab half width, or -1 = whole axis stored
  const float* in[PSI_COUNT];
  float* out[PSI_COUNT];
};

struct Step3D {
  int nx, ny, nz;
  float a;                 // dt / (mu0 dx)
  float cb_const;          // dt / (eps0 dx) when cb == nullptr
  const float* cb;         // per-cell dt / (eps0 dx eps_r), or nullptr
  const float* in[6];
  float* out[6];
  const float* damp[3];    // separable damping factors (ABSORBING)
  CpmlDev pml;
  // sources
  const int* blk_src_ptr;  // TMA path: CSR over blocks
  const SrcEntry* src;
  const float* wave;
  long long wave_len;
  long long step;          // absolute step index of this launch
  // probes: record the INPUT state (after the previous step)
  int n_probes;
  const long long* probe_cell;
  const int* probe_comp;
  float* probe_out;        // nullptr = no recording in this launch
  int* err;                // [0] code, [1] block, [2] plane index, [3] stage slot
  unsigned long long wait_ns;  // bound on every mbarrier wait
  int x_chunk;
  int ntiles_y, ntiles_z;
  // Optional compact list of blocks (tile_z, tile_y, chunk) triples; nullptr
  // = the launch grid itself.  Used to run the shell and the interior of a
  // CPML grid as separate launches with different kernels.  The chunk word
  // carries BLK_SLAB_FIRST for blocks that order their cells slab-first.
  const int* blk_list;
  int pdl;  // PDL_* bits
  // x-slab of a decomposed grid (generic kernels): local planes [x_lo, x_hi)
  // are updated, local plane x is global plane x + gx0 of a grid of gnx
  // planes; planes outside the range are ghost copies of neighbouring ranks.
  int gx0, gnx, x_lo, x_hi;
  // index decode of the generic kernels (idx32: every local index < 2^32)
  FastDiv div_nz, div_ny;
  int idx32;
  // fault injection for the failure-detection tests: every block of the TMA
  // kernels leaves the copy of its staged plane with this index unissued, so
  // its bounded waits run out (-1: off; set from JXF_FAULT_DROP_STAGE)
  int drop_stage;
};

enum PdlBits : int { PDL_WAIT_START = 1, PDL_TRIGGER = 2, PDL_WAIT_END = 4 };

// griddepcontrol (programmatic dependent launch); no-ops for a grid launched
// without the programmatic-serialization attribute.
__device__ __forceinline__ void grid_dep_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}
__device__ __forceinline__ void grid_dep_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ int slab_map(int i, int n, int P) {
  if (P < 0) return i;
  if (i < P) return i;
  if (i >= n - P) return i - n + 2 * P;
  return -1;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for phase `parity` of `bar`, giving up after `limit_ns`.  Returns false
// on timeout.  try_wait itself suspends the thread for a hardware-chosen
// interval, so the loop does not hammer the barrier.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_timer_ns() - t0 > limit_ns) return false;
  }
}

// 3D tiled TMA load global -> shared, completion counted on `bar`.
// Coordinates are innermost first.  The innermost coordinate times 4 bytes
// must be a multiple of 16 (c0 % 4 == 0 for float32).
__device__ __forceinline__ void tma_load_3d(void* smem_dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

// 4-byte asynchronous global -> shared copy (per thread), grouped with
// commit/wait_group.  Used for the CPML psi values of the next plane.
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gmem_src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(smem_dst)),
               "l"(__cvta_generic_to_global(gmem_src))
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait_pending() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

__device__ __forceinline__ void report_error(int* err, int code, int where0 = 0, int where1 = 0,
                                             int where2 = 0) {
  if (err && atomicCAS(err, 0, code) == 0) {
    err[1] = where0;
    err[2] = where1;
    err[3] = where2;
  }
}

// Rounded-as-written arithmetic: the same expression always produces the same
// bits wherever it is evaluated (the TMA kernel recomputes halo values that a
// neighbouring block also computes), so the compiler must not contract or
// reassociate these.
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }

}  // namespace jxf
