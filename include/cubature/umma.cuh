// umma.cuh -- BF16 tensor-core GEMM tiles on sm_100a (tcgen05 + TMEM), the
// building block of the control-variate network's training and inference
// kernels (mlp.cuh).
//
//   D[M x N] (+)= A[M x K] * B[N x K]^T      A, B: bf16, both K-major
//                                            D: fp32 accumulators in TMEM
//
// One CTA of 128 threads owns a 128 x N output tile (N = 16 .. 256, a
// multiple of 16).  K is consumed in chunks of 64: the 128 threads copy the
// A and B chunks from global memory into shared memory in the canonical
// no-swizzle K-major layout, then one thread issues four
// tcgen05.mma.cta_group::1.kind::f16 (K = 16 each) and commits them to an
// mbarrier, which all threads wait on (bounded) before the next chunk
// overwrites the operands.  The epilogue reads the accumulators back with
// tcgen05.ld (thread t of warp w holds row 32 w + t).
//
// Shared-memory layout of a [R rows x 64] operand chunk (R = 128 or N), in
// 16-byte core rows: element (r, k) at byte
//     (k / 8) * (R * 16) + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// i.e. 8 x 8 core matrices of 128 contiguous bytes; core matrices adjacent
// in K are LBO = R * 16 bytes apart, adjacent in R are SBO = 128 bytes apart
// (the K-major SWIZZLE_NONE canonical form
// ((8,m),(T,2)):((1T,SBO),(1,LBO)) of CuTe's UMMA descriptors).
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace cubature {
namespace umma {

constexpr int kTileM = 128;
constexpr int kChunkK = 64;
constexpr long long kWaitSpins = 1ll << 20;  // bounded mbarrier waits

// 64-bit shared-memory matrix descriptor (tcgen05), SWIZZLE_NONE.
__host__ __device__ constexpr uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);  // version 1 (sm_100)
}

// 32-bit instruction descriptor: kind::f16, A = B = BF16, D = F32, both
// K-major, M = 128, N.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int n) {
  return (1u << 4)               // D format F32
         | (1u << 7)             // A format BF16
         | (1u << 10)            // B format BF16
         | ((uint32_t)(n >> 3) << 17)
         | ((uint32_t)(kTileM >> 4) << 24);
}

// Byte offset of element (r, k) of an R-row chunk in the layout above.
__host__ __device__ constexpr uint32_t chunk_offset(int rows, int r, int k) {
  return (uint32_t)((k / 8) * (rows * 16) + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Wait for phase `parity` of the mbarrier to complete; false after the
// spin limit.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (long long i = 0; i < kWaitSpins; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

// Generic-proxy shared-memory writes become visible to the tensor core.
__device__ __forceinline__ void fence_smem_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

// 32 consecutive fp32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_load32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive fp32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_load16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Operand pointers of one GEMM in a batch (element strides in bf16 units).
struct GemmArgs {
  const __nv_bfloat16* a;  // [M][lda], K-major
  const __nv_bfloat16* b;  // [N][ldb], K-major
  long long lda, ldb;
  long long batch_a, batch_b;  // element offsets between batch entries
  int m, k;                    // M (multiple of 128), K (multiple of 16)
  int* error;                  // set to 1 when a bounded wait gives up
};

// Copy an R-row x 64-column K-chunk (k0..k0+63, zero past k) into shared
// memory in the core-matrix layout; 16-byte vectors, 128 threads.
template <int R>
__device__ __forceinline__ void stage_chunk(uint8_t* dst, const __nv_bfloat16* src, long long ld,
                                            int r0, int k0, int k) {
  constexpr int kVec = R * (kChunkK / 8);  // 16-byte vectors in the chunk
  for (int v = threadIdx.x; v < kVec; v += blockDim.x) {
    const int r = v / (kChunkK / 8), kc = v % (kChunkK / 8);
    const int kk = k0 + kc * 8;
    uint4 val = make_uint4(0, 0, 0, 0);
    if (kk < k) val = *reinterpret_cast<const uint4*>(src + (long long)(r0 + r) * ld + kk);
    *reinterpret_cast<uint4*>(dst + chunk_offset(R, r, kc * 8)) = val;
  }
}

// Accumulate one 128 x N tile of A * B^T into TMEM at `tmem` (N columns),
// for batch entry `e` and row tile `mt`.  All 128 threads call it; returns
// false if a wait gave up (the tile is then incomplete).
template <int N>
__device__ __forceinline__ bool gemm_tile(const GemmArgs& g, int e, int mt, uint32_t tmem,
                                          uint8_t* sa, uint8_t* sb, uint64_t* bar,
                                          uint32_t& phase) {
  static_assert(N % 16 == 0 && N >= 16 && N <= 256, "UMMA N for M = 128");
  const __nv_bfloat16* A = g.a + (long long)e * g.batch_a;
  const __nv_bfloat16* B = g.b + (long long)e * g.batch_b;
  constexpr uint32_t idesc = instr_desc_bf16(N);
  bool ok = true;
  for (int k0 = 0; k0 < g.k; k0 += kChunkK) {
    stage_chunk<kTileM>(sa, A, g.lda, mt * kTileM, k0, g.k);
    stage_chunk<N>(sb, B, g.ldb, 0, k0, g.k);
    fence_smem_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      fence_after_sync();
      const int ksteps = (g.k - k0 < kChunkK ? g.k - k0 : kChunkK) / 16;
      for (int s = 0; s < ksteps; ++s) {
        // K = 16: two 8-element core-matrix columns, LBO apart
        const uint64_t ad = smem_desc(smem_u32(sa) + s * 2 * (kTileM * 16), kTileM * 16, 128);
        const uint64_t bd = smem_desc(smem_u32(sb) + s * 2 * (N * 16), N * 16, 128);
        mma_bf16(tmem, ad, bd, idesc, (k0 > 0 || s > 0) ? 1u : 0u);
      }
      mma_commit(bar);
    }
    // one verdict for the whole block: the epilogue's TMEM loads are
    // warp-collective
    ok = __syncthreads_and(mbar_wait(bar, phase) ? 1 : 0) && ok;
    phase ^= 1;
    fence_after_sync();
    if (!ok) break;
  }
  return ok;
}

}  // namespace umma
}  // namespace cubature
