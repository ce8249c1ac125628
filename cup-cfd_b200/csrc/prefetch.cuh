// Tiles of 256 consecutive internal cells and the L2 prefetch of a tile's
// contiguous ranges (inline device code and plain structs only, so several
// translation units can include it).
//
// Because faces are numbered by owner slice, everything a tile reads in
// order is one contiguous range of device memory: its incidence entries,
// the records of the faces its cells own, and its cells' entries in every
// cell array. TileDesc holds those ranges, built once per mesh. In the
// prefetch kernels one lane per 256-cell tile asks L2 to fetch the ranges
// of the tile `dist` blocks ahead (cp.async.bulk.prefetch.L2), so the
// streamed loads of later blocks become L2 hits; shared memory and L1 are
// untouched and the per-cell arithmetic is that of the plain kernels.
#pragma once

#include "internal.cuh"

namespace cupcfd_gpu {

constexpr int TILE_CELLS = 256;

// Per-tile ranges, built once per mesh.
struct TileDesc {
    int entStart, entEnd;  // incidence entries of the tile's eight slices
    int fs, fe;            // faces owned by the tile's cells
    unsigned w03, w47;     // slice widths (entries per lane), one byte per slice
    int pad0, pad1;
};

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned) __cvta_generic_to_shared(p); }

struct PrefetchArgs {
    const TileDesc *desc;
    const int2 *inc;
    int nC, nF, nTiles, dist;
};

__device__ __forceinline__ void bulk_prefetch_l2(const void *p, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// The first half of a tile descriptor: {entStart, entEnd, fs, fe}.
__device__ __forceinline__ int4 load_ranges(const TileDesc *d) { return __ldg(reinterpret_cast<const int4 *>(d)); }

// The same 16 bytes fetched asynchronously into shared memory (cp.async),
// so no register is held while the thread works; ranges_ready() waits for it.
__device__ __forceinline__ void fetch_ranges_async(int4 *dst, const TileDesc *d) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n\tcp.async.commit_group;" ::"r"(smem_u32(dst)), "l"(d)
                 : "memory");
}
__device__ __forceinline__ int4 ranges_ready(const int4 *src) {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    return *src;
}

// Blocks smaller than a tile: TILE_CELLS / B blocks of B threads per tile,
// at the registers and warps per SM of 256-thread blocks. A block's slot
// frees when its own warps end instead of the slowest of eight. The last
// block of a tile prefetches for the tile (the lead lane: its last warp's
// first lane).
template <int B>
struct TileBlock {
    static_assert(TILE_CELLS % B == 0 && B % 32 == 0, "whole warps, whole tiles");
    static constexpr int P = TILE_CELLS / B;
    int c, tp;
    bool lead;
    __device__ __forceinline__ explicit TileBlock(const PrefetchArgs &pf) {
        c = blockIdx.x * B + threadIdx.x;
        tp = blockIdx.x / P + pf.dist;
        lead = blockIdx.x % P == P - 1 && threadIdx.x == B - 32 && tp < pf.nTiles;
    }
};

// One loss partial per warp, warp k of tile t at part[k nTiles + t] (stored
// warp-major, so that the loads which fold them coalesce); summed per tile in
// order from 0.0 (k_group_partials, k_reduce_partials<8>) they give the value
// a 256-thread block's reduction forms. Every lane takes part.
template <int B>
__device__ __forceinline__ void warp_partial_store(double l, int c, double *part) {
    for (int k = 16; k > 0; k >>= 1) l += __shfl_xor_sync(0xffffffffu, l, k);
    if ((threadIdx.x & 31) == 0)
        part[(size_t) ((c >> 5) % (TILE_CELLS / 32)) * (gridDim.x / TileBlock<B>::P) + c / TILE_CELLS] = l;
}

// Prefetches a tile's ranges: its entries, its owned faces' records (fgSize
// bytes each) and gface values (widened to whole 16-byte units inside the
// array), and, when the tile is whole, the cell arrays (cellBytes per tile).
template <int NCELL, class TG>
__device__ __forceinline__ void prefetch_tile(const PrefetchArgs &p, int t, const int4 &d, const void *fg,
                                              int fgSize, const TG *gface, const void *const (&cellSrc)[NCELL],
                                              const int (&cellBytes)[NCELL]) {
    constexpr int PER16 = 16 / (int) sizeof(TG);
    const int entStart = d.x, entEnd = d.y, fs = d.z, fe = d.w;
    if (entEnd > entStart) bulk_prefetch_l2(p.inc + entStart, (unsigned) (entEnd - entStart) * 8u);
    if (fe > fs)
        bulk_prefetch_l2(static_cast<const unsigned char *>(fg) + (size_t) fs * fgSize, (unsigned) (fe - fs) * (unsigned) fgSize);
    if (gface) {
        int gfA = fs & ~(PER16 - 1), gfB = (fe + PER16 - 1) & ~(PER16 - 1);
        if (gfB > p.nF) gfB = fe & ~(PER16 - 1);
        if (gfB > gfA) bulk_prefetch_l2(gface + gfA, (unsigned) (gfB - gfA) * (unsigned) sizeof(TG));
    }
    if ((long long) (t + 1) * TILE_CELLS <= (long long) p.nC)
        for (int i = 0; i < NCELL; i++)
            bulk_prefetch_l2(static_cast<const unsigned char *>(cellSrc[i]) + (size_t) t * cellBytes[i],
                             (unsigned) cellBytes[i]);
}

}  // namespace cupcfd_gpu
