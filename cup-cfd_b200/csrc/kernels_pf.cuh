// The face loops with an L2 prefetch of the tile one wave ahead, and the
// tile descriptors they read (built once per mesh).
//
// Cells are cut into tiles of TILE_CELLS = 256 consecutive internal cells
// (eight SELL slices). Because faces are numbered by owner slice, everything
// a tile reads in order is one contiguous range of device memory: its
// incidence entries, the records (and gface values) of the faces its cells
// own, and its cells' entries in every cell array (prefetch.cuh).
#pragma once

#include "kernels_adj.cuh"
#include "prefetch.cuh"

namespace cupcfd_gpu {

// ---------------------------------------------------------------------------
// L2 prefetch variant: the unstaged one-cell-per-thread kernels (the same
// per-cell bodies, so bit-identical results), where one lane per 256-cell
// block asks L2 to fetch the contiguous ranges of the tile `dist` blocks
// ahead (cp.async.bulk.prefetch.L2). Shared memory and L1 are untouched;
// the streamed loads of later blocks become L2 hits.
//
// WF: 0 for any mesh; 6 when every cell has exactly six incidences (all
// hexahedral meshes: every slice six entries wide, no padding). The cell
// loop then has a compile-time trip count: no padding checks, the chunks
// unrolled and their loads scheduled across chunks (same arithmetic in the
// same order, so the same bits).
// ---------------------------------------------------------------------------

// The separate forward and FP32 adjoint kernels run in blocks of
// CUPCFD_FWD_BLOCK = 64 threads (TileBlock), the forwards with one loss
// partial per warp, folded per tile by k_group_partials before the fixed-
// order sum. At 256^3 on one box: FP32 forward 0.477-0.485 ms against
// 0.503-0.533 in 256-thread blocks, FP32 adjoint 0.518-0.529 against
// 0.543-0.583, FP64 forward 0.698-0.704 against 0.707-0.717. The FP64
// adjoint keeps 256-thread blocks (slower in 64: 0.835 against 0.81 ms).
#ifndef CUPCFD_FWD_BLOCK
#define CUPCFD_FWD_BLOCK 64
#endif
template <int WF>
__global__ void __launch_bounds__(CUPCFD_FWD_BLOCK, CUPCFD_MINB_F32 *TILE_CELLS / CUPCFD_FWD_BLOCK)
    k_fwd_f32_pf(int nC, SellView sv, const float4 *__restrict__ fg, const float *__restrict__ phi,
                 const float *__restrict__ phiB, const double *__restrict__ vol, const float4 *__restrict__ st,
                 const float *__restrict__ gface, float *__restrict__ g, float *__restrict__ mflux,
                 double *__restrict__ lossPart, int64_t ldc, PrefetchArgs pf) {
    constexpr int T = TILE_CELLS;
    const TileBlock<CUPCFD_FWD_BLOCK> tb(pf);
    const int c = tb.c;
    __shared__ int4 s_rng;
    const void *const cellSrc[3] = {phi, st, vol};
    const int cellBytes[3] = {T * 4, T * 16, T * 8};
    if (tb.lead) fetch_ranges_async(&s_rng, pf.desc + tb.tp);
    double l = 0.0;
    if (c < nC) l = fwd_cell_f32<CUPCFD_FWD_CHUNK, WF>(c, sv, fg, phi, phiB, vol, st, gface, g, mflux, ldc);
    if (tb.lead) prefetch_tile<3>(pf, tb.tp, ranges_ready(&s_rng), fg, 16, gface, cellSrc, cellBytes);
    if (lossPart) warp_partial_store<CUPCFD_FWD_BLOCK>(l, c, lossPart);
}

template <int WF>
__global__ void __launch_bounds__(CUPCFD_FWD_BLOCK, CUPCFD_MINB_F32 *TILE_CELLS / CUPCFD_FWD_BLOCK)
    k_adj_f32_pf(int nC, SellView sv, const float4 *__restrict__ fg, const float *__restrict__ g, float hscale,
                 const float4 *__restrict__ st, const float *__restrict__ gface, float *__restrict__ phibar,
                 float *__restrict__ phibBar, float4 *__restrict__ stbar, int64_t ldc, PrefetchArgs pf) {
    constexpr int T = TILE_CELLS;
    const TileBlock<CUPCFD_FWD_BLOCK> tb(pf);
    const int c = tb.c;
    __shared__ int4 s_rng;
    const void *const cellSrc[4] = {g, g + ldc, g + 2 * ldc, st};
    const int cellBytes[4] = {T * 4, T * 4, T * 4, T * 16};
    if (tb.lead) fetch_ranges_async(&s_rng, pf.desc + tb.tp);
    if (c < nC) adj_cell_f32<false, CUPCFD_ADJ_CHUNK, 0, WF>(c, sv, fg, g, hscale, st, gface, phibar, phibBar, stbar, ldc);
    if (tb.lead) prefetch_tile<4>(pf, tb.tp, ranges_ready(&s_rng), fg, 16, gface, cellSrc, cellBytes);
}

// FP64 forward (fwd_cell_f64, exact reference arithmetic) with the same L2
// prefetch; the state's four component blocks are prefetched one by one.
template <int WF>
__global__ void __launch_bounds__(CUPCFD_FWD_BLOCK, CUPCFD_MINB_FWD_F64 *TILE_CELLS / CUPCFD_FWD_BLOCK)
    k_fwd_f64_pf(int nC, SellView sv, const double4 *__restrict__ fg, const double *__restrict__ phi,
                 const double *__restrict__ phiB, const double *__restrict__ vol, const double *__restrict__ st,
                 const double *__restrict__ gface, double *__restrict__ g, double *__restrict__ mflux,
                 double *__restrict__ lossPart, int64_t ldc, PrefetchArgs pf) {
    constexpr int T = TILE_CELLS;
    const TileBlock<CUPCFD_FWD_BLOCK> tb(pf);
    const int c = tb.c;
    __shared__ int4 s_rng;
    const void *const cellSrc[6] = {phi, vol, st, st + ldc, st + 2 * ldc, st + 3 * ldc};
    const int cellBytes[6] = {T * 8, T * 8, T * 8, T * 8, T * 8, T * 8};
    if (tb.lead) fetch_ranges_async(&s_rng, pf.desc + tb.tp);
    double l = 0.0;
    if (c < nC) l = fwd_cell_f64<CUPCFD_FWD_CHUNK_F64, WF>(c, sv, fg, phi, phiB, vol, st, gface, g, mflux, ldc);
    if (tb.lead) prefetch_tile<6>(pf, tb.tp, ranges_ready(&s_rng), fg, 32, gface, cellSrc, cellBytes);
    if (lossPart) warp_partial_store<CUPCFD_FWD_BLOCK>(l, c, lossPart);
}

// FP64 adjoint (adj_cell_f64) with the same L2 prefetch.
template <int WF>
__global__ void __launch_bounds__(TILE_CELLS, CUPCFD_MINB_ADJ_F64)
    k_adj_f64_pf(int nC, SellView sv, const double4 *__restrict__ fg, const double *__restrict__ g, double hscale,
                 const double *__restrict__ st, const double *__restrict__ gface, double *__restrict__ phibar,
                 double *__restrict__ phibBar, double *__restrict__ stbar, int64_t ldc, PrefetchArgs pf) {
    constexpr int T = TILE_CELLS;
    int c = blockIdx.x * T + threadIdx.x;
    const int tp = blockIdx.x + pf.dist;
    const bool lead = threadIdx.x == T - 32 && tp < pf.nTiles;
    __shared__ int4 s_rng;
    const void *const cellSrc[7] = {g, g + ldc, g + 2 * ldc, st, st + ldc, st + 2 * ldc, st + 3 * ldc};
    const int cellBytes[7] = {T * 8, T * 8, T * 8, T * 8, T * 8, T * 8, T * 8};
    if (lead) fetch_ranges_async(&s_rng, pf.desc + tp);
    if (c < nC) adj_cell_f64<false, CUPCFD_ADJ_CHUNK_F64, WF>(c, sv, fg, g, hscale, st, gface, phibar, phibBar, stbar, ldc);
    if (lead) prefetch_tile<7>(pf, tp, ranges_ready(&s_rng), fg, 32, gface, cellSrc, cellBytes);
}

// Forward with the mass-flux adjoint (fwd_madj_cell_f32), L2 prefetch as
// k_fwd_f32_pf. With k_gadj_f32_pf it forms the two-launch forward+adjoint:
// the state and gface are then read by one pass only.
//
// It runs in blocks of CUPCFD_FWD_MADJ_BLOCK = 64 threads, four per tile, at
// the same registers and warps per SM as 256-thread blocks: a block's slot
// frees when its two warps end instead of its slowest of eight (measured at
// 256^3: 0.543 ms against 0.568 ms; 32-thread blocks 0.540). The last block
// of a tile prefetches for the tile. The loss partials are one per warp,
// warp k of tile t at lossPart[k nTiles + t]; k_reduce_partials<8> sums each
// tile's eight in order, which gives the per-tile value of
// block_sum_store<256> bit for bit.
#ifndef CUPCFD_FWD_MADJ_CHUNK
#define CUPCFD_FWD_MADJ_CHUNK 2
#endif
#ifndef CUPCFD_MINB_FWD_MADJ
#define CUPCFD_MINB_FWD_MADJ 4  // in 256-cell tiles per SM
#endif
#ifndef CUPCFD_FWD_MADJ_BLOCK
#define CUPCFD_FWD_MADJ_BLOCK 64
#endif
template <int WF>
__global__ void __launch_bounds__(CUPCFD_FWD_MADJ_BLOCK, CUPCFD_MINB_FWD_MADJ *TILE_CELLS / CUPCFD_FWD_MADJ_BLOCK)
    k_fwd_madj_f32_pf(int nC, SellView sv, const float4 *__restrict__ fg, const float *__restrict__ phi,
                      const float *__restrict__ phiB, const double *__restrict__ vol, const float4 *__restrict__ st,
                      const float *__restrict__ gface, float *__restrict__ g, float *__restrict__ mflux,
                      float4 *__restrict__ stbar, double *__restrict__ lossPart, int64_t ldc, PrefetchArgs pf) {
    constexpr int T = TILE_CELLS;
    const TileBlock<CUPCFD_FWD_MADJ_BLOCK> tb(pf);
    const int c = tb.c;
    __shared__ int4 s_rng;
    const void *const cellSrc[3] = {phi, st, vol};
    const int cellBytes[3] = {T * 4, T * 16, T * 8};
    if (tb.lead) fetch_ranges_async(&s_rng, pf.desc + tb.tp);
    double l = 0.0;
    if (c < nC) l = fwd_madj_cell_f32<CUPCFD_FWD_MADJ_CHUNK, 0, WF>(c, sv, fg, phi, phiB, vol, st, gface, g, mflux, stbar, ldc);
    if (tb.lead) prefetch_tile<3>(pf, tb.tp, ranges_ready(&s_rng), fg, 16, gface, cellSrc, cellBytes);
    if (lossPart) warp_partial_store<CUPCFD_FWD_MADJ_BLOCK>(l, c, lossPart);
}

// Gradient part of the adjoint only (adj_cell_f32 without the mass part):
// phibar and phibBar. The next chunk's entries load during the current
// chunk's arithmetic (CUPCFD_GADJ_PIPE) within the 40 registers that six
// resident blocks per SM leave (CUPCFD_MINB_GADJ): chosen by measurement.
#ifndef CUPCFD_GADJ_PIPE
#define CUPCFD_GADJ_PIPE 1
#endif
#ifndef CUPCFD_MINB_GADJ
#define CUPCFD_MINB_GADJ 6
#endif
template <int WF>
__global__ void __launch_bounds__(TILE_CELLS, CUPCFD_MINB_GADJ)
    k_gadj_f32_pf(int nC, SellView sv, const float4 *__restrict__ fg, const float *__restrict__ g, float hscale,
                  float *__restrict__ phibar, float *__restrict__ phibBar, int64_t ldc, PrefetchArgs pf) {
    constexpr int T = TILE_CELLS;
    int c = blockIdx.x * T + threadIdx.x;
    const int tp = blockIdx.x + pf.dist;
    const bool lead = threadIdx.x == T - 32 && tp < pf.nTiles;
    __shared__ int4 s_rng;
    const void *const cellSrc[3] = {g, g + ldc, g + 2 * ldc};
    const int cellBytes[3] = {T * 4, T * 4, T * 4};
    if (lead) fetch_ranges_async(&s_rng, pf.desc + tp);
    if (c < nC)
        adj_cell_f32<false, CUPCFD_ADJ_CHUNK, CUPCFD_GADJ_PIPE, WF>(c, sv, fg, g, hscale, nullptr, nullptr, phibar,
                                                                phibBar, nullptr, ldc);
    if (lead) prefetch_tile<3>(pf, tp, ranges_ready(&s_rng), fg, 16, (const float *) nullptr, cellSrc, cellBytes);
}

// Mass-flux part of the adjoint only (adj_cell_f32 with hscale 0): stbar
// from the state and gface, with the L2 prefetch of their tile ranges. The
// host forward+adjoint call runs it once gface is in; with k_gadj_f32_pf for
// the gradient part it forms the same sums as k_adj_f32_pf, so the same bits.
template <int WF>
__global__ void __launch_bounds__(TILE_CELLS, CUPCFD_MINB_F32)
    k_madj_f32_pf(int nC, SellView sv, const float4 *__restrict__ fg, const float4 *__restrict__ st,
                  const float *__restrict__ gface, float4 *__restrict__ stbar, int64_t ldc, PrefetchArgs pf) {
    constexpr int T = TILE_CELLS;
    int c = blockIdx.x * T + threadIdx.x;
    const int tp = blockIdx.x + pf.dist;
    const bool lead = threadIdx.x == T - 32 && tp < pf.nTiles;
    __shared__ int4 s_rng;
    const void *const cellSrc[1] = {st};
    const int cellBytes[1] = {T * 16};
    if (lead) fetch_ranges_async(&s_rng, pf.desc + tp);
    if (c < nC)
        adj_cell_f32<false, CUPCFD_ADJ_CHUNK, 0, WF>(c, sv, fg, nullptr, 0.f, st, gface, nullptr, nullptr, stbar, ldc);
    if (lead) prefetch_tile<1>(pf, tp, ranges_ready(&s_rng), fg, 16, gface, cellSrc, cellBytes);
}

// Largest |c - neighbour| over the incidence lists (the numbering's bandwidth).
// Launched with whole warps (blockDim a multiple of 32), no early return.
__global__ void k_bandwidth(int nC, SellView sv, int *__restrict__ out) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    int bw = 0;
    if (c < nC) {
        int w;
        const int2 *e = cell_entries(sv, c, w);
        for (int k = 0; k < w; k++) {
            int2 en = e[32 * k];
            if (en.x < 0) break;
            if (en.y >= 0) bw = max(bw, abs(c - en.y));
        }
    }
    for (int s = 16; s > 0; s >>= 1) bw = max(bw, __shfl_xor_sync(0xffffffffu, bw, s));
    if ((threadIdx.x & 31) == 0) atomicMax(out, bw);
}

// ---------------------------------------------------------------------------
// Tile descriptors (mesh creation). Faces are numbered by owner slice, so
// the owner tile is non-decreasing in the face number; k_tile_face_start
// records where each tile's faces begin and flags any decrease.
// ---------------------------------------------------------------------------
__global__ void k_tile_face_start(int nF, int nTiles, const int2 *__restrict__ fcells, int *__restrict__ start,
                                  int *__restrict__ bad) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    int t = fcells[f].x / TILE_CELLS;
    int tp = f > 0 ? fcells[f - 1].x / TILE_CELLS : -1;
    if (t < tp) atomicOr(bad, 1);
    for (int u = tp + 1; u <= t; u++) start[u] = f;
    if (f == nF - 1)
        for (int u = t + 1; u <= nTiles; u++) start[u] = nF;
}

__global__ void k_tile_desc(int nTiles, int nSlices, const int *__restrict__ slicePtr, const int *__restrict__ start,
                            TileDesc *__restrict__ desc, int *__restrict__ maxima) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nTiles) return;
    int s0 = t * (TILE_CELLS / 32);
    TileDesc d;
    d.entStart = slicePtr[s0];
    d.entEnd = slicePtr[min(s0 + TILE_CELLS / 32, nSlices)];
    d.fs = start[t];
    d.fe = start[t + 1];
    unsigned w[2] = {0u, 0u};
    int wmax = 0;
    for (int i = 0; i < TILE_CELLS / 32; i++) {
        int s = s0 + i;
        int wi = s < nSlices ? (slicePtr[s + 1] - slicePtr[s]) >> 5 : 0;
        wmax = max(wmax, wi);
        w[i >> 2] |= (unsigned) min(wi, 255) << (8 * (i & 3));
    }
    d.w03 = w[0]; d.w47 = w[1];
    d.pad0 = 0; d.pad1 = 0;
    desc[t] = d;
    atomicMax(maxima + 0, d.entEnd - d.entStart);
    atomicMax(maxima + 1, d.fe - d.fs);
    atomicMax(maxima + 2, wmax);
}

}  // namespace cupcfd_gpu
