// Tensor memory (TMEM) as per-thread storage.
//
// Each SM of an sm_100a GPU has 256 KB of tensor memory: 128 lanes of 512
// 32-bit columns, allocated to CTAs in power-of-two column ranges. A warp
// reaches only the 32 lanes of its quadrant (warp index % 4); within it lane
// i of the warp reads and writes TMEM lane 32 * (warp % 4) + i. Loads and
// stores (tcgen05.ld / tcgen05.st, shape 32x32b) move N consecutive columns of
// the thread's own lane and do not use the shared-memory pipe. Every
// instruction here is warp-collective (.sync.aligned): the whole warp executes
// it with the same address.
#pragma once
#include <cstdint>

namespace exa {
namespace tmem {

// One warp allocates ncols columns (a power of two, 32..512) and writes the
// allocation's base address to *dst in shared memory; the CTA then gives up
// its permit to allocate again, so that other CTAs on the SM can allocate.
__device__ __forceinline__ void alloc(uint32_t* dst, uint32_t ncols) {
  const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(a), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// The allocating warp frees the allocation (after every warp is done with it).
__device__ __forceinline__ void dealloc(uint32_t base, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

// Order tensor-memory operations and allocation around a CTA barrier.
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Ten consecutive columns (five doubles) of this thread's lane. The loaded
// registers are valid only after wait_ld, which takes them as operands so
// that no use can be scheduled before it. Tensor memory is not memory the
// compiler sees, so these carry no memory clobber; being volatile, they keep
// their order among themselves.
__device__ __forceinline__ void ld10(uint32_t taddr, uint32_t (&r)[10]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(r[8]), "=r"(r[9]) : "r"(taddr + 8u));
}
__device__ __forceinline__ void wait_ld(uint32_t (&r)[10]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]));
}
__device__ __forceinline__ void st10(uint32_t taddr, const uint32_t (&r)[10]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
               "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]));
  asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(taddr + 8u), "r"(r[8]), "r"(r[9]));
}
// Stores of this thread are complete (visible to its later loads).
__device__ __forceinline__ void wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;"); }

// five doubles <-> ten 32-bit columns (low word first)
__device__ __forceinline__ void pack5(const double* q, uint32_t (&r)[10]) {
#pragma unroll
  for (int v = 0; v < 5; v++) {
    r[2 * v] = static_cast<uint32_t>(__double2loint(q[v]));
    r[2 * v + 1] = static_cast<uint32_t>(__double2hiint(q[v]));
  }
}
__device__ __forceinline__ void unpack5(const uint32_t (&r)[10], double* q) {
#pragma unroll
  for (int v = 0; v < 5; v++) q[v] = __hiloint2double(static_cast<int>(r[2 * v + 1]), static_cast<int>(r[2 * v]));
}

}  // namespace tmem
}  // namespace exa
