// BF16 GEMM on the fifth-generation tensor cores (sm_100a): tcgen05.mma with
// both operands in shared memory, the FP32 accumulator in tensor memory
// (TMEM), read back by tcgen05.ld for the epilogue.  Used by the warm-start
// surrogate's layers (dsmc_gemm_bf16); the DSMC timestep has no contraction.
//
// One CTA of 128 threads computes a 128 x 128 tile of C = A B.  K advances
// 64 at a time through a two-stage ring of shared-memory tiles: all threads
// copy the next stage from global memory (16-byte vectors along each
// operand's contiguous dimension) while the tensor cores work on the
// current one; one thread issues the four K = 16 MMAs of a stage and commits
// them to the stage's mbarrier, which frees the stage again.
//
// Shared-memory operand layout: the canonical layout without swizzle.  A
// "core matrix" is 8 rows of 16 bytes (128 bytes, contiguous).  For a K-major
// operand (K contiguous in global memory) a 16-byte row holds 8 consecutive k
// of one m (or n); for an MN-major operand it holds 8 consecutive m (or n) of
// one k.  Core matrices are laid out with the 16 groups of 8 along M (or N)
// 128 bytes apart (the descriptor's stride byte offset) and the groups of 8
// along K 2048 bytes apart (its leading byte offset), the same numbers for
// both majors.
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

namespace dsmcb {
namespace umma {

constexpr int kBM = 128, kBN = 128, kBK = 64, kStages = 2, kThreads = 128;
constexpr int kTileBytes = kBM * kBK * 2;  // 16 KB per operand tile (kBM == kBN)
constexpr uint32_t kLbo = 2048;            // between groups of 8 along K
constexpr uint32_t kSbo = 128;             // between groups of 8 along M / N
constexpr uint32_t kTmemCols = 128;        // the FP32 accumulator: 128 lanes x 128 columns

struct __align__(128) Smem {
  __nv_bfloat16 a[kStages][kBM * kBK];
  __nv_bfloat16 b[kStages][kBN * kBK];
  unsigned long long mbar[kStages];
  uint32_t tmem_base;
  uint32_t failed;
};

// Byte offset of element (r, k) (r along M or N) in an operand tile.
__device__ __forceinline__ uint32_t kmajor_off(uint32_t r, uint32_t k) {
  return (k >> 3) * kLbo + (r >> 3) * kSbo + (r & 7u) * 16u + (k & 7u) * 2u;
}
__device__ __forceinline__ uint32_t mnmajor_off(uint32_t r, uint32_t k) {
  return (k >> 3) * kLbo + (r >> 3) * kSbo + (k & 7u) * 16u + (r & 7u) * 2u;
}

// Shared-memory matrix descriptor: start address, leading and stride byte
// offsets (all in 16-byte units), version 1 (sm100), no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((kLbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((kSbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  return d;
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B,
// operand majors (0 K, 1 MN), N = 128, M = 128.
__host__ __device__ constexpr uint32_t instr_desc(uint32_t a_mn, uint32_t b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn << 15) | (b_mn << 16) |
         ((uint32_t)(kBN >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
}

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void commit(unsigned long long* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   su32(mbar))
               : "memory");
}
// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
      "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
      "[%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

}  // namespace umma
}  // namespace dsmcb
