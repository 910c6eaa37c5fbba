// tma_sm100.cuh — tensor-memory-accelerator (TMA) tile copies for sm_100a:
// a rank-5 tiled tensor map over a state vector, loads global -> shared
// completed on an mbarrier (bytes counted), stores shared -> global tracked
// by bulk async-groups.  No cluster multicast anywhere: every map covers
// this GPU's own memory and every copy has one destination CTA.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace yao {

// How a tile of a state vector moves between HBM and shared memory by TMA
// (one rank-5 tiled tensor map over the state).  Tensor dimension r spans
// the global bits [shift[r], shift[r] + width[r]); its box covers the low
// bits of that span, which are tile bits.  Dimension 0 starts at bit 0 and
// its box is the 128-byte run of the lowest tile bits (16 complex64 or 8
// complex128 amplitudes, two real elements each).  Tile bits beyond the box
// dimensions (at most 6, the highest tile positions) are enumerated: box
// copy e lands 1024-byte aligned at e * copy_bytes in shared memory.
struct TmaPlan {
    int8_t shift[5];
    int8_t width[5];
    int8_t ebits[6];     // enumerated global bits, ascending
    int32_t nebits;
    int32_t copy_bytes;  // bytes of one box
};

// Host: the plan and tensor map of a tile whose positions are the global
// bits tb[0] < ... < tb[tbits - 1] (sv_tiles.cu); false when it cannot move
// by TMA.  tma_enabled(): YAO_TMA=0 turns TMA tile copies off.
bool tma_make_plan(const int8_t* tb, int tbits, uint32_t nbits, size_t amp, void* st, TmaPlan& p, CUtensorMap* map);
bool tma_enabled();

namespace tma {

// Load of one box at coordinates c0..c4 (elements; c0 * element size is a
// multiple of 16 bytes) into shared memory at `dst` (shared-window address,
// 1024-byte aligned for the 128-byte swizzle); the barrier at `bar` counts
// the bytes as they land.
__device__ __forceinline__ void load5(uint32_t dst, const CUtensorMap* map, int32_t c0, int32_t c1, int32_t c2,
                                      int32_t c3, int32_t c4, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar)
        : "memory");
}

// Store of one box from shared memory at `src` to coordinates c0..c4
// (never negative); completion is tracked by the issuing thread's bulk
// async-groups.
__device__ __forceinline__ void store5(const CUtensorMap* map, int32_t c0, int32_t c1, int32_t c2, int32_t c3,
                                       int32_t c4, uint32_t src) {
    asm volatile(
        "cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group"
        " [%0, {%1, %2, %3, %4, %5}], [%6];\n" ::"l"(reinterpret_cast<uint64_t>(map)),
        "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(src)
        : "memory");
}

__device__ __forceinline__ void commit_group() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }

// Wait until at most N of this thread's committed store groups still read
// their shared-memory source.
template <int N>
__device__ __forceinline__ void wait_group_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;\n" ::"n"(N) : "memory");
}
// Wait until at most N of this thread's committed store groups are not
// complete (their writes performed).
template <int N>
__device__ __forceinline__ void wait_group() {
    asm volatile("cp.async.bulk.wait_group %0;\n" ::"n"(N) : "memory");
}

// The tensor map is read through the generic address of a __grid_constant__
// kernel parameter; this prefetches its descriptor.
__device__ __forceinline__ void prefetch_map(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Coordinates (elements) of the box whose tile base is `b`.
__device__ __forceinline__ void coords(const TmaPlan& p, uint64_t b, int32_t (&c)[5]) {
#pragma unroll
    for (int r = 0; r < 5; r++) c[r] = (int32_t)((b >> p.shift[r]) & ((1ull << p.width[r]) - 1));
    c[0] *= 2;  // two real elements per amplitude
}

// One thread: every box of the tile whose base index is `base` into shared
// memory at `dst`, completing on the barrier at `bar` (armed by the caller).
__device__ __forceinline__ void load_boxes(const CUtensorMap* map, const TmaPlan& p, uint64_t base, uint32_t dst,
                                           uint32_t bar) {
    const uint32_t nc = 1u << p.nebits;
    for (uint32_t e = 0; e < nc; e++) {
        uint64_t b = base;
        for (int q = 0; q < p.nebits; q++) b |= (uint64_t)((e >> q) & 1) << p.ebits[q];
        int32_t c[5];
        coords(p, b, c);
        load5(dst + e * (uint32_t)p.copy_bytes, map, c[0], c[1], c[2], c[3], c[4], bar);
    }
}

// One thread: every box of the tile at `base` from shared memory at `src`
// back to the state (the caller commits the group).
__device__ __forceinline__ void store_boxes(const CUtensorMap* map, const TmaPlan& p, uint64_t base, uint32_t src) {
    const uint32_t nc = 1u << p.nebits;
    for (uint32_t e = 0; e < nc; e++) {
        uint64_t b = base;
        for (int q = 0; q < p.nebits; q++) b |= (uint64_t)((e >> q) & 1) << p.ebits[q];
        int32_t c[5];
        coords(p, b, c);
        store5(map, c[0], c[1], c[2], c[3], c[4], src + e * (uint32_t)p.copy_bytes);
    }
}

}  // namespace tma
}  // namespace yao
