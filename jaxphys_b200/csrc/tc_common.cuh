// 5th-generation tensor core (tcgen05) primitives for sm_100a in inline PTX.
//
// Operands live in shared memory as BF16 "core-matrix" images without
// swizzle: an R x K matrix (R, K multiples of 8), K-major, is stored as
// 8-row x 16-byte core matrices,
//     byte(r, k) = (r / 8) * (K * 16) + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// so core matrices adjacent along K are 128 bytes apart (leading byte
// offset) and 8-row groups are K * 16 bytes apart (stride byte offset).  One
// MMA consumes a K = 16 slice, i.e. the descriptor start advances 256 bytes
// per slice.  Accumulators are FP32 in tensor memory (TMEM): row m of an
// M = 128 tile is TMEM lane m, column n is TMEM column base + n.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "fdtd_common.cuh"

namespace jxf {
namespace tc {

// Byte offset of element (r, k) in a K-major core-matrix image with K columns.
__host__ __device__ __forceinline__ uint32_t img_off(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor (no swizzle, sm_100 descriptor version 1).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Descriptor of the K-slice `kk` (16 columns) of a K-major image with K columns.
__device__ __forceinline__ uint64_t img_desc(uint32_t saddr, int K, int kk) {
  return smem_desc(saddr + (uint32_t)kk * 256u, 128u, (uint32_t)K * 16u);
}

// Instruction descriptor: kind::f16 with BF16 A and B, FP32 D, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T for one K = 16 slice; issued by a single thread.
__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                    uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrive once on `bar` when every MMA issued so far by this thread is done.
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

// TMEM allocation (warp-wide): the base address is written to *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 16 / 32 consecutive FP32 columns of this thread's TMEM lane (warp w of the
// four accesses lanes 32 w .. 32 w + 31).  The load and its tcgen05.wait::ld
// are one asm statement, so the outputs exist only after the wait.
__device__ __forceinline__ void ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// TMEM address of (lane, column) relative to an allocation base.
__device__ __forceinline__ uint32_t taddr(uint32_t base, int lane, int col) {
  return base + ((uint32_t)lane << 16) + (uint32_t)col;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// Store row r (64 values) of a 128 x 64 K-major image (8 vector stores).
__device__ __forceinline__ void put_row64(unsigned char* img, int r, const float* v) {
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    uint4 q;
    q.x = pack_bf16(v[8 * c + 0], v[8 * c + 1]);
    q.y = pack_bf16(v[8 * c + 2], v[8 * c + 3]);
    q.z = pack_bf16(v[8 * c + 4], v[8 * c + 5]);
    q.w = pack_bf16(v[8 * c + 6], v[8 * c + 7]);
    *reinterpret_cast<uint4*>(img + img_off(r, 8 * c, 64)) = q;
  }
}
// Store sample r's 64 values as column r of a 64 x 128 K-major image
// (the transpose of a 128 x 64 tile), `n` values from row offset q0.
__device__ __forceinline__ void put_col(unsigned char* imgT, int r, const float* v, int n,
                                        int q0 = 0) {
  for (int q = 0; q < n; ++q)
    *reinterpret_cast<__nv_bfloat16*>(imgT + img_off(q0 + q, r, 128)) = __float2bfloat16_rn(v[q]);
}

}  // namespace tc
}  // namespace jxf
