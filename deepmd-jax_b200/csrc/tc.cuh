// tcgen05 / TMEM / mbarrier helpers for sm_100a (inline PTX).
//
// Operand tiles live in shared memory in the canonical no-swizzle
// ("interleave") layouts of the UMMA shared-memory descriptor: 8x8 core
// matrices of 128 contiguous bytes (16 bytes per row of 8 bf16).
//   K-major  tile (R rows x K):  byte(r,k)  = ((r/8)*(K/8) + k/8)*128 + (r%8)*16 + (k%8)*2
//            descriptor: LBO = 128 (next 8-wide K chunk), SBO = (K/8)*128 (next 8 rows)
//   MN-major tile (K x MN):      byte(k,mn) = ((k/8)*(MN/8) + mn/8)*128 + (k%8)*16 + (mn%8)*2
//            descriptor: LBO = (MN/8)*128 (next 8 K rows), SBO = 128 (next 8 MN)
// An MMA of K = 16 starts at the tile base plus the byte offset of its first
// K index.  Descriptor fields (64-bit): start >> 4 in [0,14), LBO >> 4 in
// [16,30), SBO >> 4 in [32,46), version 1 in [46,48), layout type (0 = no
// swizzle) in [61,64).  Instruction descriptor (kind::f16): D format F32 in
// [4,6), A/B format BF16 in [7,10)/[10,13), A/B major in bit 15/16,
// N >> 3 in [17,23), M >> 4 in [24,29).
//
// Every wait is bounded: on timeout the caller sets an error flag and returns
// instead of spinning forever.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace dpb {
namespace tc {

constexpr int kWaitLimit = 1 << 24;  // mbarrier polls before giving up

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__host__ __device__ constexpr uint64_t desc_fields(uint32_t lbo, uint32_t sbo) {
  return ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | desc_fields(lbo, sbo);
}

// BF16 x BF16 -> F32, M x N, A/B major: 0 = K-major, 1 = MN-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// F16 x F16 -> F32 (kind::f16 with A/B format 0), M x N, A/B major as above.
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// tcgen05.mma kind::f16 issued by one thread: D (TMEM) (+)= A . B with FP32
// accumulation; A and B are both BF16 or both FP16, as the instruction
// descriptor says (idesc_bf16 / idesc_f16).
__device__ __forceinline__ void mma_f16kind(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

// Wait for the phase with the given parity to complete; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity) {
  const uint32_t a = smem_u32(mbar);
  for (int it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// One warp allocates ncols (power of two >= 32) TMEM columns; the base
// address is written to *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 16 columns of 32-bit: thread t of the warp gets lane
// (32 * (warp % 4) + t), columns [col, col + 16).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// tanh.approx.f32: about 1e-5 relative error with no sign preference, far
// below the FP16 rounding step of the embedding's operands.  (The packed
// tanh.approx.f16x2 is cheaper but shrinks |tanh| by about 3.5e-4 on average,
// a bias that the embedding's tangents turn into a systematic scaling of the
// forces, so the FP16 kernels take tanh in FP32 and round the pair.)
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t *>(&h);
}

// ---- packed FP16 pairs (element k in the low half, k + 1 in the high half,
// the order of consecutive elements in the operand tiles)
__device__ __forceinline__ __half2 as_h2(uint32_t u) { return *reinterpret_cast<__half2 *>(&u); }
__device__ __forceinline__ uint32_t as_u32(__half2 h) { return *reinterpret_cast<uint32_t *>(&h); }
// (a, b) -> one register, round to nearest, saturating to the largest finite
// FP16 value instead of overflowing to infinity
__device__ __forceinline__ __half2 f2_to_h2(float a, float b) {
  uint32_t r;
  asm("cvt.rn.satfinite.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
  return as_h2(r);
}


// ---- warp-level MMA (mma.sync m16n8k16, FP16 operands, FP32 accumulators)
// for small per-warp products.  Fragments (PTX ISA layout; g = lane / 4,
// q = lane % 4): A (16 x 16, row-major) a[0] = (row g, cols 2q, 2q+1),
// a[1] = row g + 8, a[2] = cols + 8, a[3] = both; B (16 x 8, "col") b[0] =
// (rows 2q, 2q+1, col g), b[1] = rows + 8; C (16 x 8 FP32) c[0], c[1] = (row g,
// cols 2q, 2q+1), c[2], c[3] = row g + 8.
__device__ __forceinline__ void mma_16816(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// Four 8x8 b16 matrices from shared memory; lane l gives the row address of
// row l % 8 of matrix l / 8 (16-byte aligned); register i holds matrix i.
__device__ __forceinline__ void ldmatrix_x4(uint32_t (&r)[4], const void *row) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(row)));
}
// Two 8x8 b16 matrices (lanes 0-15 give the row addresses), as stored or
// transposed (.trans: lane l receives column l / 4, rows 2 (l % 4), +1).
__device__ __forceinline__ void ldmatrix_x2(uint32_t &r0, uint32_t &r1, const void *row) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(smem_u32(row)));
}
__device__ __forceinline__ void ldmatrix_x2_trans(uint32_t &r0, uint32_t &r1, const void *row) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];"
               : "=r"(r0), "=r"(r1)
               : "r"(smem_u32(row)));
}

// Asynchronous 16-byte global -> shared copies (no register round trip).
__device__ __forceinline__ void cp_async16(void *dst_smem, const void *src_gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst_smem)), "l"(src_gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Issue a 32 lanes x 16 columns TMEM load without waiting; pair with
// tmem_wait() before the registers are used.
__device__ __forceinline__ void tmem_ld16_issue(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// 32 lanes x 8 columns, issue only (pair with tmem_wait()).
__device__ __forceinline__ void tmem_ld8_issue(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}

// ---- mbarrier arrivals and bulk (TMA) copies
// Makes barrier initialisation visible to the async proxy (TMA complete_tx).
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(mbar)) : "memory");
}
// Arrive and add tx_bytes to the bytes the current phase waits for.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *mbar, uint32_t tx_bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(tx_bytes)
               : "memory");
}
// One poll of the phase with the given parity.
__device__ __forceinline__ bool mbar_test(uint32_t mbar_addr, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(mbar_addr), "r"(parity)
      : "memory");
  return done != 0;
}
// Bulk (TMA) copy of `bytes` contiguous bytes global -> shared, no multicast;
// completion is signalled on mbar as tx bytes.  Both addresses 16-byte
// aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(uint32_t dst_smem, const void *src, uint32_t bytes, uint64_t *mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   dst_smem),
               "l"(src), "r"(bytes), "r"(smem_u32(mbar))
               : "memory");
}

// Hint: bring the global line holding p into L2.
__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Byte offsets of the canonical layouts (see file comment).
__host__ __device__ constexpr uint32_t kmajor_off(int r, int k, int K) {
  return (uint32_t)(((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
__host__ __device__ constexpr uint32_t mnmajor_off(int k, int mn, int MN) {
  return (uint32_t)(((k >> 3) * (MN >> 3) + (mn >> 3)) * 128 + (k & 7) * 16 + (mn & 7) * 2);
}

}  // namespace tc
}  // namespace dpb
