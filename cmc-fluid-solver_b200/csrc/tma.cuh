// Tensor Memory Accelerator helpers shared by the TMA-fed X/Y sweeps
// (sweep_xytma.cu, sweep_xypair.cu): tile loads without multicast, mbarrier
// set-up and a bounded mbarrier wait, and the host-side tensor-map cache.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdint>

namespace adi {
namespace tma {

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 3D tiled copy global -> shared, completing on `bar` (complete_tx::bytes).
__device__ __forceinline__ void load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        :
        : "r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation visible to the async proxy.
__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Waits for phase `parity` of `bar` to complete: at most `tries` polls, each
// suspending for at most about 10 us.  Returns false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int tries)
{
    uint32_t done = 0;
    for (int it = 0; it < tries && !done; it++) {
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, 10000; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
    }
    return done != 0;
}

} // namespace tma

// Tensor map over a [nx][ny][nz] array (k fastest) whose box is {w, 1, Lb} for X
// lines or {w, Lb, 1} for Y lines; es = element bytes.  Encoded maps are cached
// by their arguments.  Returns false if the driver entry point is missing or the
// encoder rejects the arguments.
bool make_tile_map(CUtensorMap *m, const void *base, int dir, int nx, int ny, int nz, int w, int Lb, int es,
                   CUtensorMapDataType dt);
bool have_tensor_map_encoder();

// Tensor maps of one X/Y sweep launch (passed by value, in param space).
struct XYMaps {
    CUtensorMap cur[4];
    CUtensorMap tin[4];   // 16-wide boxes
    CUtensorMap fwide;    // advecting field of temp, 24-wide box (k0-4 .. k0+19)
    CUtensorMap code;
};

} // namespace adi
