// Wavefront-fused forward + adjoint of the benchmark loss in ONE persistent
// launch, using the 126 MB L2 as the buffer between the two passes.
//
// A tile is 256 consecutive internal cell ids, one cell per thread. The
// launch's G CTAs (all co-resident: cooperative launch) work in rounds: in
// round r CTA b runs the forward of tile rG + b (gradient, owned mass
// fluxes, the tile's loss partial), counts it in done[r], then runs the
// adjoint of tile (r - L)G + b. The adjoint of tile j reads the gradients of
// its neighbours, all within aheadTiles = ceil(bandwidth / 256) + 1 tiles of
// j (bandwidth = the numbering's largest |c - neighbour|), so it needs the
// forward rounds up to (j + aheadTiles) / G; with L = 1 + ceil(aheadTiles /
// G) that is at most round r - 1, which the CTA waits for by polling one
// counter, done[r - 1 at most] == G. With a bandwidth-limited numbering (the
// reference's lexicographic order, or RCM) L is 2, and the adjoint of a tile
// runs about two rounds (two waves of tiles) after its forward, while the
// incidence entries and face records the forward read are still in L2. One
// lane per CTA also asks L2 to prefetch the contiguous ranges of the CTA's
// next forward tile (cp.async.bulk.prefetch.L2).
//
// Progress: a forward never waits, and the adjoint of round r waits only
// for forwards of earlier rounds, so the CTA at the lowest round can always
// proceed and every wait ends. Waits are bounded anyway: on expiry the error
// word is set, waiting stops everywhere and the launch finishes (the host
// reports CUPCFD_E_ERROR).
//
// Memory ordering (the grid-barrier pattern): after a forward tile,
// __syncthreads(), then thread 0 issues __threadfence() and atomicAdd(done[r]).
// A waiting thread 0 polls with volatile loads, then __threadfence() and
// __syncthreads(); gradients of other tiles are read with ld.global.cg (L2,
// the point of coherence), never through L1.
//
// Per-cell arithmetic and the per-tile loss partials are those of the
// two-launch path (fwd_cell_* / adj_cell_*, block sums in warp order), so
// both give bit-identical results.
#pragma once

#include "kernels_staged.cuh"

namespace cupcfd_gpu {

#ifndef CUPCFD_FUSED_FWD_CHUNK
#define CUPCFD_FUSED_FWD_CHUNK 1
#endif
#ifndef CUPCFD_FUSED_ADJ_CHUNK
#define CUPCFD_FUSED_ADJ_CHUNK 1
#endif
constexpr int FUSED_TILE = 256;
static_assert(FUSED_TILE == STAGED_TILE, "fused and prefetch tiles coincide");

struct FusedCtl {
    unsigned *done;  // [nRounds] forward tiles finished per round (zeroed per launch)
    int *err;        // bit 1: a wait expired
    int nTiles, nRounds, lagRounds, aheadTiles, spinLimit;
    PrefetchArgs pf; // pf.desc null: no prefetch
};

// Whole CTA: wait until every forward tile of rounds <= need is finished.
__device__ __forceinline__ void wait_round(const FusedCtl &k, int need) {
    if (threadIdx.x == 0) {
        const volatile unsigned *p = k.done + need;
        const unsigned G = gridDim.x;
        int spins = 0;
        while (*p < G) {
            if (*(volatile int *) k.err) break;
            if (++spins > k.spinLimit) {
                atomicOr(k.err, 1);
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
    }
    __syncthreads();
}

__device__ __forceinline__ void finish_round(const FusedCtl &k, int r) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(k.done + r, 1u);
    }
}

// Tile sum of v in the two-launch path's order, stored by thread 0.
__device__ __forceinline__ void tile_sum(double v, double *out, int idx) {
    __shared__ double red[FUSED_TILE / 32];
    for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < FUSED_TILE / 32; i++) t += red[i];
        out[idx] = t;
    }
}

__global__ void __launch_bounds__(FUSED_TILE, CUPCFD_MINB_FUSED_F32)
    k_fused_f32(int nC, FusedCtl k, SellView sv, const float4 *__restrict__ fg, const float *__restrict__ phi,
                const float *__restrict__ phiB, const double *__restrict__ vol, const float4 *__restrict__ st,
                const float *__restrict__ gface, float *g, float *__restrict__ mflux, float *__restrict__ phibar,
                float *__restrict__ phibBar, float4 *__restrict__ stbar, double *__restrict__ lossPart, int64_t ldc) {
    constexpr int T = FUSED_TILE;
    const int G = gridDim.x, b = blockIdx.x;
    const bool lead = threadIdx.x == T - 32 && k.pf.desc != nullptr;
    const void *const cellSrc[3] = {phi, st, vol};
    const int cellBytes[3] = {T * 4, T * 16, T * 8};
    const void *const adjSrc[4] = {g, g + ldc, g + 2 * ldc, st};
    const int adjBytes[4] = {T * 4, T * 4, T * 4, T * 16};
    for (int r = 0; r < k.nRounds + k.lagRounds; r++) {
        if (r < k.nRounds) {
            int t = r * G + b;
            if (t < k.nTiles) {
                int tn = t + G;
                __shared__ int4 s_rng;
                if (lead && tn < k.nTiles) fetch_ranges_async(&s_rng, k.pf.desc + tn);
                int c = t * T + threadIdx.x;
                double l = 0.0;
                if (c < nC) l = fwd_cell_f32<CUPCFD_FUSED_FWD_CHUNK>(c, sv, fg, phi, phiB, vol, st, gface, g, mflux, ldc);
                if (lead && tn < k.nTiles) prefetch_tile<3>(k.pf, tn, ranges_ready(&s_rng), fg, 16, gface, cellSrc, cellBytes);
                tile_sum(l, lossPart, t);
            }
            finish_round(k, r);
        }
        int ra = r - k.lagRounds;
        if (ra >= 0) {
            int ta = ra * G + b;
            if (ta < k.nTiles) {
                wait_round(k, min(k.nRounds - 1, (ta + k.aheadTiles) / G));
                // the next adjoint tile's ranges: a no-op where L2 still holds
                // them from its forward, a DRAM fetch ahead of use where not
                __shared__ int4 s_adj;
                int tn = ta + G;
                bool pfa = lead && tn < k.nTiles;
                if (pfa) fetch_ranges_async(&s_adj, k.pf.desc + tn);
                int c = ta * T + threadIdx.x;
                if (c < nC)
                    adj_cell_f32<true, CUPCFD_FUSED_ADJ_CHUNK>(c, sv, fg, g, 2.f, st, gface, phibar, phibBar, stbar, ldc);
                if (pfa) prefetch_tile<4>(k.pf, tn, ranges_ready(&s_adj), fg, 16, gface, adjSrc, adjBytes);
            }
        }
    }
}

__global__ void __launch_bounds__(FUSED_TILE, CUPCFD_MINB_FUSED_F64)
    k_fused_f64(int nC, FusedCtl k, SellView sv, const double4 *__restrict__ fg, const double *__restrict__ phi,
                const double *__restrict__ phiB, const double *__restrict__ vol, const double *__restrict__ st,
                const double *__restrict__ gface, double *g, double *__restrict__ mflux, double *__restrict__ phibar,
                double *__restrict__ phibBar, double *__restrict__ stbar, double *__restrict__ lossPart, int64_t ldc) {
    constexpr int T = FUSED_TILE;
    const int G = gridDim.x, b = blockIdx.x;
    for (int r = 0; r < k.nRounds + k.lagRounds; r++) {
        if (r < k.nRounds) {
            int t = r * G + b;
            if (t < k.nTiles) {
                int c = t * T + threadIdx.x;
                double l = 0.0;
                if (c < nC) l = fwd_cell_f64<CUPCFD_FWD_CHUNK_F64>(c, sv, fg, phi, phiB, vol, st, gface, g, mflux, ldc);
                tile_sum(l, lossPart, t);
            }
            finish_round(k, r);
        }
        int ra = r - k.lagRounds;
        if (ra >= 0) {
            int ta = ra * G + b;
            if (ta < k.nTiles) {
                wait_round(k, min(k.nRounds - 1, (ta + k.aheadTiles) / G));
                int c = ta * T + threadIdx.x;
                if (c < nC) adj_cell_f64<true>(c, sv, fg, g, 2.0, st, gface, phibar, phibBar, stbar, ldc);
            }
        }
    }
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

}  // namespace cupcfd_gpu
