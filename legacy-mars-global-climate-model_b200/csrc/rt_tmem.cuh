// Tensor memory (TMEM) as per-thread scratch for the on-chip solves.
//
// Each SM has 256 KB of tensor memory: 128 lanes x 512 columns of 32 bits.
// Warp w of a CTA reaches lanes 32*(w%4) .. 32*(w%4)+31, one lane per
// thread, and every column of the CTA's allocation, so a lane is a private
// row of up to 2 KB for its thread.  The solves store doubles there as two
// consecutive columns (tcgen05.st/ld .32x32b: each thread moves consecutive
// columns of its own lane).  The tcgen05.ld/st instructions are .sync.aligned:
// all 32 threads of a warp execute them together with the same column, so
// callers keep warp-uniform control flow around them.
//
// Allocation (tcgen05.alloc) is issued by one warp for the whole CTA and the
// address handed to the others through shared memory; the same warp frees it
// before the CTA exits.  An allocation waits while other CTAs on the SM hold
// the columns it needs; every CTA here frees its columns when its work is
// done, so such a wait always ends.
#pragma once
#include <cstdint>

namespace mgcm {

__device__ __forceinline__ void tmem_alloc(uint32_t *smem_dst, uint32_t ncols) {
    const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Orders tcgen05 operations across a CTA barrier.
__device__ __forceinline__ void tmem_fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// One double per thread at taddr (two columns), store and wait.
__device__ __forceinline__ void tmem_put(uint32_t taddr, double x) {
    __syncwarp();   // the .sync.aligned forms need the whole warp converged
    const uint32_t lo = (uint32_t)__double2loint(x), hi = (uint32_t)__double2hiint(x);
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};\n"
        "tcgen05.wait::st.sync.aligned;" ::"r"(taddr),
        "r"(lo), "r"(hi)
        : "memory");
}

// One double per thread from taddr, load and wait (the registers are only
// defined after the wait, so both sit in one statement).
__device__ __forceinline__ double tmem_get(uint32_t taddr) {
    __syncwarp();
    uint32_t lo, hi;
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];\n"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(lo), "=r"(hi)
        : "r"(taddr)
        : "memory");
    return __hiloint2double((int)hi, (int)lo);
}

// Four doubles from taddr (eight columns) with one wait.
__device__ __forceinline__ void tmem_get4(uint32_t taddr, double &a, double &b, double &c, double &d) {
    __syncwarp();
    uint32_t r[8];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
        : "r"(taddr)
        : "memory");
    a = __hiloint2double((int)r[1], (int)r[0]);
    b = __hiloint2double((int)r[3], (int)r[2]);
    c = __hiloint2double((int)r[5], (int)r[4]);
    d = __hiloint2double((int)r[7], (int)r[6]);
}

}  // namespace mgcm
