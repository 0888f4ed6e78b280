// Tensor-memory-accelerator (TMA) tile loads: tensor maps of this GPU's own buffers (no
// multicast anywhere), encoded on the host through the driver entry point, and the
// cp.async.bulk.tensor loads that complete on a shared-memory mbarrier.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace lsb {

// A 3-D FP64 tensor [nz][rows][nx] (nx fastest) with a box of box_x x box_rows x 1 and the
// 128-byte swizzle (box_x * 8 must be 128); false when the driver call is not available or
// refuses the map.  Cached by (base, dims, box): the map only encodes them.
bool tmap_f64_3d(CUtensorMap* out, const void* base, uint64_t nx, uint64_t rows, uint64_t nz, uint32_t box_x,
                 uint32_t box_rows);

// A 2-D tensor [rows][nx] of 4- or 8-byte elements with a box of box_x x 1 (one row piece),
// no swizzle: box_x <= 256 divides nx and box_x * elem_bytes is a multiple of 16.  Cached
// like tmap_f64_3d.
bool tmap_rows(CUtensorMap* out, const void* base, uint32_t elem_bytes, uint64_t nx, uint64_t rows, uint32_t box_x);

namespace tma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::); }

// one arrival that also announces `bytes` of transactions on the barrier's current phase
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// the phase of the given parity completed, with a time limit (about 0.2 s); false on time-out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    const long long t0 = clock64();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(ok)
            : "r"(addr), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > 400000000LL) return false;
    }
}

// box at (x, y, z) of the tensor map into shared memory at dst; completes on bar.  x must be
// a multiple of 2 (16 bytes of FP64): every caller passes twice a multiple of 8 columns.
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// box at (x, y) of a 2-D tensor map into shared memory at dst (128-byte aligned); completes
// on bar.  x * element size must be a multiple of 16 bytes.
__device__ __forceinline__ void load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// generic-proxy accesses of this thread (and, after a barrier, of the block) ordered before
// its later async-proxy (TMA) accesses to shared memory
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

}  // namespace tma
}  // namespace lsb
