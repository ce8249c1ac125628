// SELL-32 incidence-list access shared by the kernels of every translation
// unit (inline device functions only): the cell's first entry and slice
// width, and chunked entry loads. Layout in internal.cuh (struct Sell).
#pragma once

#include "internal.cuh"

namespace cupcfd_gpu {

struct SellView {
    const int *slicePtr;
    const int2 *inc;
    int width;  // common slice width, or 0 when widths vary
};

// The cell's first incidence entry and its slice width (entries per lane).
// With a common width (every hexahedral mesh) the position is arithmetic,
// which takes a dependent load off the head of every cell's load chain.
__device__ __forceinline__ const int2 *cell_entries(const SellView &sv, int c, int &w) {
    int s = c >> 5;
    if (sv.width) {
        w = sv.width;
        return sv.inc + (s * 32 * sv.width + (c & 31));  // entries fit in int (slicePtr is int)
    }
    int p0 = __ldg(sv.slicePtr + s);
    w = (__ldg(sv.slicePtr + s + 1) - p0) >> 5;
    return sv.inc + p0 + (c & 31);
}

// Read-only 8-byte load of an incidence entry. With CUPCFD_L2_PREFETCH the
// load asks L2 to fetch 256-byte blocks from DRAM (the incidence stream is
// read sequentially slice by slice).
__device__ __forceinline__ int2 ld_entry(const int2 *p) {
#ifdef CUPCFD_L2_PREFETCH
    int2 v;
    asm("ld.global.nc.L2::256B.v2.s32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p));
    return v;
#else
    return __ldg(p);
#endif
}

// Entries k0 .. k0+W-1 of the cell (padding {-1,-1} past its slice width).
template <int W>
__device__ __forceinline__ void load_entries(const int2 *e, int k0, int w, int2 (&en)[W]) {
#pragma unroll
    for (int j = 0; j < W; j++) en[j] = (k0 + j < w) ? ld_entry(e + 32 * (k0 + j)) : make_int2(-1, -1);
}

// The entries of the cell's next chunk into en: with PIPE they were loaded
// into nx before the current chunk's arithmetic (so their latency overlaps
// it; two more registers per entry), else they are loaded now.
template <int PIPE, int W>
__device__ __forceinline__ void next_entries(const int2 *e, int k0, int w, int2 (&en)[W], const int2 (&nx)[W]) {
    if (PIPE) {
#pragma unroll
        for (int j = 0; j < W; j++) en[j] = nx[j];
    } else {
        load_entries(e, k0, w, en);
    }
}

}  // namespace cupcfd_gpu
