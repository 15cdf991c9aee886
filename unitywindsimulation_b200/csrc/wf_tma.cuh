// wf_tma.cuh - tensor-memory-accelerator plumbing shared by the TMA-staged
// Jacobi passes (wf_pres_tma.cu, wf_vel_tma.cu): shared-memory addresses,
// bounded mbarrier waits, tiled bulk-tensor loads, and the host-side tensor
// map encoder.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "wf_common.cuh"

namespace wf {
namespace tma {

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for the phase of the given parity, bounded by limit_ns; false when
// it ran out.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, unsigned long long limit_ns) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try(bar, parity))
        if (global_ns() - t0 > limit_ns) return false;
    return true;
}
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_3d(unsigned dst, const CUtensorMap* map, int x, int y, int z, unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(dst),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tma_4d(unsigned dst, const CUtensorMap* map, int x, int y, int z, int q,
                                       unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(dst),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(q), "r"(bar)
        : "memory");
}

}  // namespace tma

// Tiled tensor map over `planes` consecutive N-float planes of the grid
// (rank 3 when planes == 1, else rank 4) with a box of box_w x box_h x 1 x
// box_planes floats and zero fill outside the grid.  False where the
// driver's encoder is missing or refuses the map (alignment).
bool tma_encode(CUtensorMap* m, const Params& P, const float* base, int planes, int box_w, int box_h,
                int box_planes);
// The driver's tensor-map encoder is present.
bool tma_available();

}  // namespace wf
