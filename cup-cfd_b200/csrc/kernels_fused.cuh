// Wavefront-fused forward + adjoint of the benchmark loss in ONE persistent
// launch, using the 126 MB L2 as the buffer between the two passes.
//
// A work item is a tile of 256 consecutive internal cell ids, one cell per
// thread. Tiles are assigned round-robin to the launch's B CTAs: CTA b runs
// items b, b + B, b + 2B, ... in order. Item i runs the forward of tile i
// (gradient, owned mass fluxes, loss partials) and publishes it, then the
// adjoint of tile j = i - lag, which needs the forwards of tiles up to
// j + lagNeed, lagNeed = ceil(bandwidth / 256) + 1 (bandwidth = the
// numbering's largest |c - neighbour|): every neighbour gradient the adjoint
// reads is then final. lag = lagNeed + B: the adjoint of round r needs only
// rounds < r, so it rarely waits. With a bandwidth-limited numbering (the
// reference's lexicographic order, or RCM) the adjoint of tile j runs while
// the data its forward read are still in L2.
//
// No hot atomics: single-address atomics serialise at roughly 40 ns each, so
// neither work dispensing nor progress uses a shared counter. CTA b
// publishes prog[b] = rounds of forwards it has finished (one release store
// per item). A CTA that needs a newer bound reads all B counters, 256
// threads in parallel, and takes the lowest unfinished tile over all CTAs;
// it does so about once per round.
//
// Progress: the launch is cooperative (all CTAs co-resident); item i's
// adjoint needs forwards of items < i only, each run by a resident CTA once
// its earlier items are done, so by induction on the item index every wait
// ends. Waits are bounded anyway: on expiry the error word is set, waiting
// stops everywhere and the launch finishes (the host reports CUPCFD_E_ERROR).
//
// Memory ordering: results are written with ordinary stores, __syncthreads(),
// then thread 0 fences and st.release.gpu's prog[b]; readers use
// ld.acquire.gpu, synchronise the CTA, and read other tiles' gradients with
// ld.global.cg (L2, coherent), never through L1.
#pragma once

#include "kernels_adj.cuh"

namespace cupcfd_gpu {

#ifndef CUPCFD_FUSED_FWD_CHUNK
#define CUPCFD_FUSED_FWD_CHUNK 2
#endif
constexpr int FUSED_TILE = 256;

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

struct FusedCtl {
    unsigned *prog;    // [B] rounds of forward tiles each CTA has published (zeroed per launch)
    int *err;          // bit 1: a wait expired
    int nTiles, lagNeed, lag, spinLimit;
};

__device__ __forceinline__ double warp_sum(double v) {
    for (int k = 16; k > 0; k >>= 1) v += __shfl_xor_sync(0xffffffffu, v, k);
    return v;
}

// Lowest tile whose forward is not yet published (nTiles when all are),
// over all CTAs' progress counters. Whole CTA.
__device__ __forceinline__ int lowest_pending(const FusedCtl &k) {
    __shared__ int s_min;
    const int B = gridDim.x;
    if (threadIdx.x == 0) s_min = k.nTiles;
    __syncthreads();
    int m = k.nTiles;
    for (int b = threadIdx.x; b < B; b += blockDim.x) {
        long long next = (long long) b + (long long) ld_acquire(k.prog + b) * B;
        if (next < m) m = (int) next;
    }
    for (int s = 16; s > 0; s >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, s));
    if ((threadIdx.x & 31) == 0) atomicMin(&s_min, m);
    __syncthreads();
    return s_min;
}

// Wait until every forward tile < need is published; `known` caches the
// last bound this CTA saw. Whole CTA.
__device__ __forceinline__ void wait_tiles(const FusedCtl &k, int need, int &known) {
    int spins = 0;
    while (known < need) {
        known = lowest_pending(k);
        if (known >= need) break;
        __shared__ int s_stop;
        if (threadIdx.x == 0) {
            int dead = *(volatile int *) k.err;
            if (!dead && ++spins > k.spinLimit) {
                atomicOr(k.err, 1);
                dead = 1;
            }
            s_stop = dead;
        }
        __syncthreads();
        if (s_stop) {
            known = need;
            break;
        }
        __nanosleep(200);
    }
}

template <int BLOCK>
__device__ __forceinline__ void publish_round(const FusedCtl &k, unsigned rounds) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) st_release(k.prog + blockIdx.x, rounds);
}

__global__ void __launch_bounds__(FUSED_TILE, CUPCFD_MINB_FUSED_F32)
    k_fused_f32(int nC, FusedCtl k, SellView sv, const float4 *__restrict__ fg, const float *__restrict__ phi,
                const float *__restrict__ phiB, const double *__restrict__ vol, const float4 *__restrict__ st,
                const float *__restrict__ gface, float *g, float *__restrict__ mflux, float *__restrict__ phibar,
                float *__restrict__ phibBar, float4 *__restrict__ stbar, double *__restrict__ lossPart, int64_t ldc) {
    const int B = gridDim.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int total = k.nTiles + k.lag;
    int known = 0;
    unsigned rounds = 0;
    for (int i = blockIdx.x; i < total; i += B) {
        if (i < k.nTiles) {
            int c = i * FUSED_TILE + threadIdx.x;
            double l = 0.0;
            if (c < nC) l = fwd_cell_f32<CUPCFD_FUSED_FWD_CHUNK>(c, sv, fg, phi, phiB, vol, st, gface, g, mflux, ldc);
            l = warp_sum(l);
            if (lane == 0) lossPart[(int64_t) i * (FUSED_TILE / 32) + warp] = l;
            publish_round<FUSED_TILE>(k, ++rounds);
        }
        int j = i - k.lag;
        if (j >= 0) {
            wait_tiles(k, min(k.nTiles, j + k.lagNeed + 1), known);
            int c = j * FUSED_TILE + threadIdx.x;
            if (c < nC) adj_cell_f32<true>(c, sv, fg, g, 2.f, st, gface, phibar, phibBar, stbar, ldc);
        }
    }
}

__global__ void __launch_bounds__(FUSED_TILE, CUPCFD_MINB_FUSED_F64)
    k_fused_f64(int nC, FusedCtl k, SellView sv, const double4 *__restrict__ fg, const double *__restrict__ phi,
                const double *__restrict__ phiB, const double *__restrict__ vol, const double *__restrict__ st,
                const double *__restrict__ gface, double *g, double *__restrict__ mflux, double *__restrict__ phibar,
                double *__restrict__ phibBar, double *__restrict__ stbar, double *__restrict__ lossPart, int64_t ldc) {
    const int B = gridDim.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int total = k.nTiles + k.lag;
    int known = 0;
    unsigned rounds = 0;
    for (int i = blockIdx.x; i < total; i += B) {
        if (i < k.nTiles) {
            int c = i * FUSED_TILE + threadIdx.x;
            double l = 0.0;
            if (c < nC) l = fwd_cell_f64<CUPCFD_FUSED_FWD_CHUNK>(c, sv, fg, phi, phiB, vol, st, gface, g, mflux, ldc);
            l = warp_sum(l);
            if (lane == 0) lossPart[(int64_t) i * (FUSED_TILE / 32) + warp] = l;
            publish_round<FUSED_TILE>(k, ++rounds);
        }
        int j = i - k.lag;
        if (j >= 0) {
            wait_tiles(k, min(k.nTiles, j + k.lagNeed + 1), known);
            int c = j * FUSED_TILE + threadIdx.x;
            if (c < nC) adj_cell_f64<true>(c, sv, fg, g, 2.0, st, gface, phibar, phibBar, stbar, ldc);
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
