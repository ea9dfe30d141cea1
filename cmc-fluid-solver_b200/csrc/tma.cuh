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

// 4D tiled copy global -> shared, completing on `bar` (complete_tx::bytes).
__device__ __forceinline__ void load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                        uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        :
        : "r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
          "r"(smem_u32(bar))
        : "memory");
}

// 4D tiled copy shared -> global (bulk-group completion).  The source must have
// been written before a fence.proxy.async.shared::cta and a barrier.
__device__ __forceinline__ void store_4d(const CUtensorMap *map, const void *src, int c0, int c1, int c2, int c3)
{
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%2, %3, %4, %5}], [%1];"
                 :
                 : "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// Waits until every committed bulk store has finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

// Makes this thread's generic-proxy shared-memory writes visible to the async proxy.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Asynchronous 4- or 8-byte copy global -> shared (cp.async, one group per call
// site; cp_async_wait_all waits for all of this thread's copies).
template <int BYTES>
__device__ __forceinline__ void cp_async(void *dst, const void *src)
{
    static_assert(BYTES == 4 || BYTES == 8, "4- or 8-byte copies");
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

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

// Chunk-major tile map over the same array: the line coordinate x = c K + i
// (line length L = P K) is split into a chunk index c (P values, global stride K
// rows) and a row-in-chunk i (K values, stride one row), ordered so that a box
// lands in shared memory as [i][c][w]: X lines dims {nz, ny, P, K}, box
// {w, 1, P, box_rows}; Y lines dims {nz, P, K, nx}, box {w, P, box_rows, 1}.
// box_rows = K covers whole lines, box_rows = 1 one row-in-chunk of every chunk.
bool make_chunk_map(CUtensorMap *m, const void *base, int dir, int nx, int ny, int nz, int w, int K, int es,
                    CUtensorMapDataType dt, int box_rows);
bool have_tensor_map_encoder();

// Tensor maps of one X/Y sweep launch (passed by value, in param space): 3D
// row-major maps (sweep_xypair.cu) or chunk-major maps (sweep_xytma.cu).
struct XYMaps {
    CUtensorMap cur[4];
    CUtensorMap tin[4];   // boxes as wide as the CTA's lines
    CUtensorMap fwide;    // advecting field of temp with a k halo on each side
    CUtensorMap code;
    CUtensorMap next[4];  // stores of the sweep's results (sweep_xytma.cu)
    CUtensorMap tout[4];
};

} // namespace adi
