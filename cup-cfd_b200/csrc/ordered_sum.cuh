// Sums over the boundaries of one region type in boundary order, bit for bit
// the sums of a loop that walks ib = 0 .. nB-1 and adds each selected
// boundary's value into a running total and into its region's accumulator
// (FluxMassDolfynBoundaryLoop1-5, MassKernels.ipp:311-521;
// FluxUVWDolfynBndsLoop1, UVWKernels.ipp:527-544).
//
// IEEE addition is not associative, so each sum stays one chain of additions
// in boundary order; what runs in parallel is everything else. Three passes
// over all boundaries (count per block, scan of the counts, ordered write)
// gather the selected boundaries' values and regions into dense arrays in
// boundary order; one block then runs the chains: thread 0 the total, thread
// 32 + j region j's accumulators, each reading the dense values a block-sized
// batch at a time from shared memory. A chain costs one dependent add per
// selected boundary, against a shared-memory round trip and a branch per
// boundary when one thread walked all of them. F32: the chains add in float
// (the reference's T = float instantiation); values and accumulators stay in
// double arrays, which hold the float values exactly.
//
// Kernels and helpers sit in an unnamed namespace (at file scope, as in
// perm.cuh): each translation unit that includes this header gets its own
// copies, so no kernel symbol is defined twice.
#pragma once

#include <algorithm>

#include "internal.cuh"

namespace {

using namespace cupcfd_gpu;

constexpr int SEL_T = 1024;
constexpr int SEL_REGIONS = SEL_T - 32;  // regions per k_sel_sum launch (threads 32 ..)

struct SelArgs {
    int nB;
    const int *bndRegion, *regionType;
    int type;
};

__device__ __forceinline__ bool sel_flag(const SelArgs &a, int ib) {
    return ib < a.nB && a.regionType[a.bndRegion[ib]] == a.type;
}

// pass 1: selected boundaries per block of SEL_T
__global__ void __launch_bounds__(SEL_T) k_sel_count(SelArgs a, int *__restrict__ cnt) {
    const int n = __syncthreads_count(sel_flag(a, blockIdx.x * SEL_T + threadIdx.x));
    if (threadIdx.x == 0) cnt[blockIdx.x] = n;
}

// pass 2 (one block): exclusive prefix sums of cnt[0 .. n) in place, the
// total in cnt[n]
__global__ void __launch_bounds__(SEL_T) k_sel_scan(int n, int *__restrict__ cnt) {
    __shared__ int wsum[32];
    __shared__ int carry;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < n; b0 += SEL_T) {
        const int i = b0 + threadIdx.x;
        const int v = i < n ? cnt[i] : 0;
        int x = v;  // inclusive scan within the warp
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int t = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            wsum[lane] = t;
        }
        __syncthreads();
        const int excl = carry + (wid ? wsum[wid - 1] : 0) + x - v;
        if (i < n) cnt[i] = excl;
        __syncthreads();
        if (threadIdx.x == SEL_T - 1) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) cnt[n] = carry;
}

// pass 3: the selected boundaries' values (NV components at
// base[map[ib] * stride + offset + q], map null: ib) and regions, densely in
// boundary order
template <int NV>
__global__ void __launch_bounds__(SEL_T) k_sel_write(SelArgs a, const double *__restrict__ base, int stride,
                                                     int offset, const int *__restrict__ map,
                                                     const int *__restrict__ cnt, double *__restrict__ vals,
                                                     int *__restrict__ regs) {
    __shared__ int wcount[32];
    const int ib = blockIdx.x * SEL_T + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const bool f = sel_flag(a, ib);
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wcount[wid] = __popc(bal);
    __syncthreads();
    if (!f) return;
    int pos = cnt[blockIdx.x] + __popc(bal & ((1u << lane) - 1u));
    for (int w = 0; w < wid; w++) pos += wcount[w];
    const size_t j = (size_t) (map ? map[ib] : ib) * stride + offset;
#pragma unroll
    for (int q = 0; q < NV; q++) vals[(size_t) NV * pos + q] = base[j + q];
    regs[pos] = a.bndRegion[ib];
}

// pass 4 (one block): over the K = *total selected entries in order,
// *out = init + v_0 + v_1 + ... (NV = 1, when out is not null) and, for the
// regions r0 .. r0 + SEL_REGIONS - 1 below nR, regionAcc[NV r + q] +=
// v_k[q] over region r's entries (regionAcc in/out, may be null). Entries
// move through shared memory in batches of SB, double-buffered: each thread
// loads its entry of the next batch into registers before the chains of the
// current batch run, and stores it after them, so the loads' latency hides
// behind the chains and a batch costs one barrier.
template <int NV, bool F32 = false>
__global__ void __launch_bounds__(SEL_T) k_sel_sum(const int *__restrict__ total, const double *__restrict__ vals,
                                                   const int *__restrict__ regs, const double *init, double initValue,
                                                   double *out, double *regionAcc, int nR, int r0) {
    constexpr int SB = NV == 1 ? SEL_T : SEL_T / 2;  // 2 x (SB entries) fit the static shared memory
    __shared__ double sv[2][SB * NV];
    __shared__ int sr[2][SB];
    const int K = *total;
    const int tid = threadIdx.x;
    const bool doTotal = out != nullptr && tid == 0;
    const int myR = (regionAcc && tid >= 32 && r0 + tid - 32 < nR) ? r0 + tid - 32 : -1;
    double acc = doTotal ? (init ? *init : initValue) : 0.0;
    double racc[NV];
#pragma unroll
    for (int q = 0; q < NV; q++) racc[q] = myR >= 0 ? regionAcc[NV * (size_t) myR + q] : 0.0;
    if (tid < SB && tid < K) {
#pragma unroll
        for (int q = 0; q < NV; q++) sv[0][NV * tid + q] = vals[(size_t) NV * tid + q];
        sr[0][tid] = regs[tid];
    }
    __syncthreads();
    int buf = 0;
    for (int b0 = 0; b0 < K; b0 += SB) {
        const int kn = b0 + SB + tid;
        const bool hasNext = tid < SB && kn < K;
        double vn[NV];
        int rn = -1;
        if (hasNext) {
#pragma unroll
            for (int q = 0; q < NV; q++) vn[q] = vals[(size_t) NV * kn + q];
            rn = regs[kn];
        }
        const int n = min(SB, K - b0);
        const double *cv = sv[buf];
        const int *cr = sr[buf];
        if (doTotal) {
#pragma unroll 16
            for (int j = 0; j < n; j++) acc = F32 ? (double) __fadd_rn((float) acc, (float) cv[NV * j]) : __dadd_rn(acc, cv[NV * j]);
        } else if (myR >= 0) {
#pragma unroll 8
            for (int j = 0; j < n; j++)
                if (cr[j] == myR) {
#pragma unroll
                    for (int q = 0; q < NV; q++)
                        racc[q] = F32 ? (double) __fadd_rn((float) racc[q], (float) cv[NV * j + q])
                                      : __dadd_rn(racc[q], cv[NV * j + q]);
                }
        }
        if (hasNext) {
#pragma unroll
            for (int q = 0; q < NV; q++) sv[buf ^ 1][NV * tid + q] = vn[q];
            sr[buf ^ 1][tid] = rn;
        }
        __syncthreads();
        buf ^= 1;
    }
    if (doTotal) *out = acc;
    if (myR >= 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) regionAcc[NV * (size_t) myR + q] = racc[q];
    }
}

// The four passes. Scratch: cnt [nB / SEL_T + 2] ints, vals [NV nB]
// doubles, regs [nB] ints. out may be init (the sum continues from it).
template <int NV, bool F32 = false>
int launch_ordered_sum(const SelArgs &a, const double *base, int stride, int offset, const int *map,
                       const double *init, double initValue, double *out, double *regionAcc, int nR, int *cnt,
                       double *vals, int *regs, cudaStream_t st) {
    const int nBlk = (a.nB + SEL_T - 1) / SEL_T;
    if (nBlk > 0) {
        k_sel_count<<<nBlk, SEL_T, 0, st>>>(a, cnt);
        CG_LAUNCHED();
    }
    k_sel_scan<<<1, SEL_T, 0, st>>>(nBlk, cnt);
    CG_LAUNCHED();
    if (nBlk > 0) {
        k_sel_write<NV><<<nBlk, SEL_T, 0, st>>>(a, base, stride, offset, map, cnt, vals, regs);
        CG_LAUNCHED();
    }
    const int groups = regionAcc ? std::max(1, (nR + SEL_REGIONS - 1) / SEL_REGIONS) : 1;
    for (int g = 0; g < groups; g++) {
        k_sel_sum<NV, F32><<<1, SEL_T, 0, st>>>(cnt + nBlk, vals, regs, g == 0 ? init : nullptr, initValue,
                                           g == 0 ? out : nullptr, regionAcc, nR, g * SEL_REGIONS);
        CG_LAUNCHED();
    }
    return CUPCFD_E_SUCCESS;
}

}  // namespace
