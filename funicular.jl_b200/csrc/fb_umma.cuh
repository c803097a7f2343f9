// The fifth-generation tensor core of sm_100a (tcgen05) as inline PTX: tensor
// memory allocation, shared-memory matrix descriptors, the instruction
// descriptor of the integer MMA, the MMA itself, its commit to an mbarrier,
// and loads of the accumulator out of tensor memory. The descriptor bit
// layouts follow the PTX ISA (tcgen05 "Shared memory descriptor" and
// "Instruction descriptor" tables), as CUTLASS's cute/arch/mma_sm100_desc.hpp
// also lays them out.
#pragma once

#include "fb_tma.cuh"

namespace fb {
namespace umma {

// Shared-memory matrix descriptor of a K-major operand tile whose rows are
// 64 bytes of K, stored with the 64-byte swizzle: eight-row core groups are
// 512 bytes apart (stride byte offset), the leading byte offset is unused by
// swizzled K-major layouts and set to 1, version 1 (Blackwell), base offset
// 0 (tiles start on 512-byte boundaries), layout type 4 = SWIZZLE_64B.
__device__ __forceinline__ uint64_t desc_kmajor_sw64(uint32_t smem_addr) {
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                 // leading byte offset (unused)
    d |= (uint64_t)(512 >> 4) << 32;        // stride byte offset
    d |= (uint64_t)1 << 46;                 // version
    d |= (uint64_t)4 << 61;                 // SWIZZLE_64B
    return d;
}

// Byte offset of element (row, k) inside such a tile: 16-byte chunk c of a
// 64-byte row r lands in chunk c ^ ((r >> 1) & 3) (address bits [4,6) XOR
// bits [7,9)).
__host__ __device__ __forceinline__ uint32_t sw64_offset(uint32_t row, uint32_t k) {
    const uint32_t chunk = (k >> 4) ^ ((row >> 1) & 3);
    return row * 64 + chunk * 16 + (k & 15);
}

// Instruction descriptor of kind::i8 with signed 8-bit A and B, both
// K-major, a signed 32-bit accumulator, shape M x N (bits: c_format [4,6) = 2,
// a_format [7,10) = 1, b_format [10,13) = 1, N >> 3 at [17,23), M >> 4 at
// [24,29)).
__host__ __device__ constexpr uint32_t idesc_s8s8_s32(int M, int N) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_s8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                       bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}

// D[tmem] (+)= A[tmem] B[smem]^T: A is M x K in tensor memory, row i in lane
// i, K packed four 8-bit values to a 32-bit column.
__device__ __forceinline__ void mma_s8_tmem_a(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                              bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p;\n\t}"
        ::"r"(d_tmem), "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}

// Arrives once on bar when every MMA this thread issued before has finished.
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Makes this thread's generic-proxy shared-memory writes visible to the
// tensor core (async proxy) reads that are ordered after it.
__device__ __forceinline__ void fence_smem_to_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Tensor memory allocation, by one whole warp. The address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(slot)), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 32 consecutive columns of 32-bit words: thread t of the warp
// gets lane (taddr lane + t), columns [col, col + 32). A warp may only touch
// the 32 lanes of its own quarter (warp id % 4).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
}

// 32 lanes x 16 consecutive columns, as tmem_ld32.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}

// Thread t of the warp writes two consecutive 32-bit columns of lane
// (taddr lane + t).
__device__ __forceinline__ void tmem_st2(uint32_t taddr, uint32_t r0, uint32_t r1) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(taddr), "r"(r0), "r"(r1) : "memory");
}

__device__ __forceinline__ void tmem_wait_st() {
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

}  // namespace umma
}  // namespace fb
