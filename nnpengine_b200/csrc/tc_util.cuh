// tcgen05 (5th-generation tensor core) building blocks for sm_100a, written as inline PTX.
//
// Operand tiles live in shared memory in the K-major, no-swizzle canonical layout: the tile is a
// grid of 8x8 "core matrices" (8 rows x 16 bytes, 128 contiguous bytes each); core matrices that
// are adjacent along K are 128 B apart (leading-dimension byte offset, LBO) and groups of 8 rows
// are (K/8)*128 B apart (stride-dimension byte offset, SBO). One MMA consumes K=16 (two core
// matrices along K), so the k-th MMA of a chain starts 256*k bytes into the tile.
// Accumulators live in tensor memory (TMEM): row m of an M=128 tile is TMEM lane m, column n is
// TMEM column base+n; warp w of the CTA reads lanes 32*(w%4)..+31.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (r, k) in a K-major no-swizzle bf16 tile with K columns
__device__ __forceinline__ uint32_t kmajor_off(int r, int k, int K) {
  return ((uint32_t)(((r >> 3) * (K >> 3) + (k >> 3)) << 7)) + ((r & 7) << 4) + ((k & 7) << 1);
}

// shared-memory matrix descriptor (SWIZZLE_NONE, descriptor version 1)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}
// descriptor of the kk-th K=16 slice of a [rows][K] K-major tile at saddr
__device__ __forceinline__ uint64_t tile_desc(uint32_t saddr, int K, int kk) {
  return sdesc(saddr + 256u * kk, 128u, (uint32_t)(K >> 3) * 128u);
}

// instruction descriptor: kind::f16, A=B=BF16, D=F32, shape M x N; A and B K-major unless
// b_mn (bit 16) / a_mn (bit 15) select an MN-major B / A operand
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool b_mn = false, bool a_mn = false) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// MN-major no-swizzle tile [N rows (MN) x K]: core matrix (n/8, k/8) holds 8 K-rows of 8 contiguous
// MN elements; MN-adjacent core matrices are 128 B apart (SBO), K-adjacent ones (N/8)*128 B (LBO).
__device__ __forceinline__ uint32_t mnmajor_off(int n, int k, int N) {
  return ((uint32_t)(((k >> 3) * (N >> 3) + (n >> 3)) << 7)) + ((k & 7) << 4) + ((n & 7) << 1);
}
__device__ __forceinline__ uint64_t tile_desc_mn(uint32_t saddr, int N, int kk) {
  return sdesc(saddr + 2u * (uint32_t)(N >> 3) * 128u * kk, (uint32_t)(N >> 3) * 128u, 128u);
}
// K-major descriptor whose 8-row groups all alias the first one (SBO = 0): an M x K operand whose
// rows repeat with period 8, held in 8*K*2 bytes
__device__ __forceinline__ uint64_t tile_desc_bcast(uint32_t saddr, int K, int kk) {
  return sdesc(saddr + 256u * kk, 128u, 0u);
}
// MN-major counterpart: an M x K operand whose rows repeat with period 8, held as K rows of 8
// contiguous M elements (element (m, k) at 16 k + 2 (m % 8)); K-adjacent core matrices 128 B apart
// (LBO), MN-adjacent ones aliased (SBO = 0)
__device__ __forceinline__ uint64_t tile_desc_bcast_mn(uint32_t saddr, int kk) {
  return sdesc(saddr + 256u * kk, 128u, 0u);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy smem writes made visible to the tensor core's async proxy
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait (about max_cycles SM clocks); false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long max_cycles = 2000000000ll) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity))
    if (clock64() - t0 > max_cycles) return false;
  return true;
}

// One arrival that also expects `bytes` of asynchronous copies to complete on the barrier.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) from global memory into
// this CTA's shared memory, counted on the barrier's transaction count (a plain load, one destination CTA).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// TMEM allocation by one full warp; the base address is written to smem.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// 16 consecutive FP32 columns of this thread's lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// 2 x 16 FP32 columns (at ta and tb) of this thread's lane behind one wait; the wait names the
// destination registers so no use of them can be scheduled before it.
__device__ __forceinline__ void tmem_ld16x2(uint32_t ta, uint32_t tb, float* va, float* vb) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(ta));
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(tb));
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]),
                 "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]),
                 "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]),
                 "+r"(r[30]), "+r"(r[31])
               :
               : "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) { va[k] = __uint_as_float(r[k]); vb[k] = __uint_as_float(r[16 + k]); }
}

// 16-byte global -> shared copy that bypasses L1 (cp.async), and the wait for this thread's copies
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// wait until at most N of this thread's committed groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// 8 floats -> 8 bf16 packed in a 16-byte chunk
__device__ __forceinline__ uint4 pack8(const float* f) {
  uint4 u;
  __nv_bfloat162 a = __floats2bfloat162_rn(f[0], f[1]), b = __floats2bfloat162_rn(f[2], f[3]);
  __nv_bfloat162 c = __floats2bfloat162_rn(f[4], f[5]), d = __floats2bfloat162_rn(f[6], f[7]);
  u.x = *reinterpret_cast<uint32_t*>(&a); u.y = *reinterpret_cast<uint32_t*>(&b);
  u.z = *reinterpret_cast<uint32_t*>(&c); u.w = *reinterpret_cast<uint32_t*>(&d);
  return u;
}

}  // namespace tc
