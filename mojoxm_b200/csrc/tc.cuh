// sm_100a tensor-core (tcgen05 / UMMA) and tensor-memory helpers, written as
// inline PTX.  Conventions (PTX ISA, tcgen05 family):
//  * shared-memory matrix descriptor, K-major, no swizzle: core matrices of
//    8 rows x 16 bytes stored contiguously (row r at +16r); LBO = byte
//    distance between the two core matrices along K of one MMA step, SBO =
//    byte distance between core matrices along M/N; version field = 1.
//  * instruction descriptor (kind::f16): F32 accumulator, BF16 A and B,
//    both K-major, N>>3 at bits [17,23), M>>4 at bits [24,29).
// The layout used by the kernels: element (row, k) of an R x Kp operand tile
// lives at byte  (k/8)*(R/8*128) + (row/8)*128 + (row%8)*16 + (k%8)*2,
// i.e. LBO = R*16 bytes and SBO = 128 bytes; an MMA K step of 16 advances
// the start address by 2*LBO.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "tma.cuh"

namespace mxm {

__host__ __device__ constexpr uint32_t umma_tile_offset(int row, int k, int rows) {
  return uint32_t((k >> 3) * (rows >> 3) * 128 + (row >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFFu);
  d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
  d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
  d |= uint64_t(1) << 46;  // descriptor version (sm_100)
  return d;                // base offset 0, legacy LBO mode, SWIZZLE_NONE
}

__host__ __device__ constexpr uint32_t umma_idesc_bf16_f32(int M, int N) {
  return (1u << 4)                       // D format F32
         | (1u << 7)                     // A format BF16
         | (1u << 10)                    // B format BF16
         | (uint32_t(N >> 3) << 17)      // N
         | (uint32_t(M >> 4) << 24);     // M
}

__device__ __forceinline__ void tc_mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

// Arrive on an mbarrier once all previously issued tcgen05.mma of this
// thread have completed.
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Whole warp: allocate `ncols` TMEM columns (power of two >= 32); the TMEM
// address is written to shared memory at `dst`.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns: thread i of the warp receives
// lane (warp's lane quarter + i), columns [col, col+16).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// x = hi + lo with hi, lo in bfloat16 (the split-precision operands)
__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// Two values at once: hi and lo of (a, b) as packed bf16 pairs, a in the low
// half (the lower address of a 4-byte word)
__device__ __forceinline__ void split_bf16x2(float a, float b, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

// x = hi + lo with hi, lo rounded to TF32 (11 significant bits, round to
// nearest, ties away from zero: cvt.rna.tf32.f32); x - hi is exact in FP32,
// so hi + lo carries 22 significant bits of x.
__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}

__device__ __forceinline__ void tc_mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

// Operand kinds of the split-precision contraction.  Both keep a value as
// hi + lo and form hi*hi + hi*lo + lo*hi in FP32 (three MMAs into one
// accumulator).  ELEM: bytes per operand element; KSTEP: K of one MMA;
// CM: elements in the 16 contiguous bytes of a core-matrix row; FMT: the
// A / B format code of the instruction descriptor.
// A_MN: whether the flux tile (the MMA's A operand) is stored MN-major.
//  * OpBF16 (kind::f16): 8 + 8 significant bits, relative error ~2^-16;
//    MN-major flux tile (two elements of one k share a 4-byte word);
//  * OpTF32 (kind::tf32): 11 + 11 significant bits, relative error ~2^-22,
//    twice the shared memory per operand; both operands K-major.
struct OpBF16 {
  static constexpr int ELEM = 2, KSTEP = 16, CM = 8;
  static constexpr bool A_MN = true;
  static constexpr uint32_t FMT = 1;
  __device__ static void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    tc_mma_bf16(d, a, b, idesc, acc);
  }
  // one value: hi at ph, lo at pl
  __device__ static void put1(unsigned char* ph, unsigned char* pl, float v) {
    __nv_bfloat16 h, l;
    split_bf16(v, h, l);
    *reinterpret_cast<__nv_bfloat16*>(ph) = h;
    *reinterpret_cast<__nv_bfloat16*>(pl) = l;
  }
  // two MN-adjacent values (rows r, r + 1 of one k; r even)
  __device__ static void put2(unsigned char* ph, unsigned char* pl, float a, float b) {
    uint32_t h, l;
    split_bf16x2(a, b, h, l);
    *reinterpret_cast<uint32_t*>(ph) = h;
    *reinterpret_cast<uint32_t*>(pl) = l;
  }
};
struct OpTF32 {
  static constexpr int ELEM = 4, KSTEP = 8, CM = 4;
  static constexpr bool A_MN = false;
  static constexpr uint32_t FMT = 2;
  __device__ static void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    tc_mma_tf32(d, a, b, idesc, acc);
  }
  __device__ static void put1(unsigned char* ph, unsigned char* pl, float v) {
    uint32_t h, l;
    split_tf32(v, h, l);
    *reinterpret_cast<uint32_t*>(ph) = h;
    *reinterpret_cast<uint32_t*>(pl) = l;
  }
  __device__ static void put2(unsigned char* ph, unsigned char* pl, float a, float b) {
    uint2 h, l;
    split_tf32(a, h.x, l.x);
    split_tf32(b, h.y, l.y);
    *reinterpret_cast<uint2*>(ph) = h;
    *reinterpret_cast<uint2*>(pl) = l;
  }
};

// Instruction descriptor: FP32 accumulator, A and B of format Op::FMT, A
// (the M side) MN-major when Op::A_MN, B K-major.
template <class Op>
__host__ __device__ constexpr uint32_t umma_idesc_f32acc(int M, int N) {
  return (1u << 4) | (Op::FMT << 7) | (Op::FMT << 10) | ((Op::A_MN ? 1u : 0u) << 15) | (uint32_t(N >> 3) << 17) |
         (uint32_t(M >> 4) << 24);
}

// No-swizzle core-matrix layouts (8 rows of 16 bytes per core matrix):
// MN-major `rows` x K tile: CM consecutive rows of one k in 16 bytes, the 8
// k of a core matrix 16 bytes apart, core matrices along the rows 128 bytes
// apart (SBO), along K rows/CM * 128 bytes apart (LBO);
template <class Op>
__host__ __device__ constexpr uint32_t umma_mn_off(int row, int k, int rows) {
  return uint32_t((k >> 3) * (rows / Op::CM) * 128 + (row / Op::CM) * 128 + (k & 7) * 16 + (row % Op::CM) * Op::ELEM);
}
// K-major `nn` x K tile: CM consecutive k of one row in 16 bytes, the 8 rows
// of a core matrix 16 bytes apart, core matrices along the rows 128 bytes
// apart (SBO), along K nn/8 * 128 bytes apart (LBO).
template <class Op>
__host__ __device__ constexpr uint32_t umma_k_off(int n, int k, int nn) {
  return uint32_t((k / Op::CM) * (nn >> 3) * 128 + (n >> 3) * 128 + (n & 7) * 16 + (k % Op::CM) * Op::ELEM);
}
// The flux tile (`rows` x K, the MMA's A operand) in Op's layout, its LBO
// and the start-address step of one MMA K step.
template <class Op>
__host__ __device__ constexpr uint32_t umma_a_off(int row, int k, int rows) {
  return Op::A_MN ? umma_mn_off<Op>(row, k, rows) : umma_k_off<Op>(row, k, rows);
}
template <class Op>
__host__ __device__ constexpr uint32_t umma_a_lbo(int rows) {
  return Op::A_MN ? uint32_t(rows / Op::CM) * 128 : uint32_t(rows / 8) * 128;
}
template <class Op>
__host__ __device__ constexpr uint32_t umma_a_kstep(int rows) {
  return Op::A_MN ? uint32_t(Op::KSTEP / 8) * umma_a_lbo<Op>(rows) : uint32_t(Op::KSTEP / Op::CM) * umma_a_lbo<Op>(rows);
}

}  // namespace mxm
