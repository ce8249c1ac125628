// Staged face loops: the forward and adjoint cell loops with their
// contiguous input streams moved into shared memory by bulk async copies.
//
// Cells are cut into tiles of STAGED_TILE = 256 consecutive internal cells
// (eight SELL slices). Because faces are numbered by owner slice, everything
// a tile reads in order is one contiguous range of device memory:
//   - its incidence entries   inc[slicePtr[8t] .. slicePtr[8t + 8])
//   - the faces its cells own  fg32[fs .. fe), gface[fs .. fe)
//   - its cell scalars         phi/state/vol (forward), g/state (adjoint)
// A persistent grid walks the tiles round-robin. Thread 0 of each CTA keeps
// STAGES-1 tiles in flight: per tile it posts the byte count on that stage's
// mbarrier and issues one cp.async.bulk per range; the other threads wait on
// the mbarrier (bounded) and then compute one cell each. What is not in the
// tile's ranges (faces owned by other tiles, neighbour cells outside the
// tile, boundary values, the ragged ends of a range that does not fit the
// stage buffer) is read from global memory, mostly as L2 hits, so the stage
// capacities are a tuning choice, never a correctness condition.
//
// Per-cell arithmetic is the same, operation for operation and in the same
// face order, as fwd_cell_f32 / adj_cell_f32, and the loss partials are
// summed per 256-cell tile in the same order as k_fwd_f32's per-block sums,
// so staged and unstaged launches give bit-identical results.
//
// Requirements (checked on the host, which otherwise launches the unstaged
// kernels): user arrays copied in bulk start on 16-byte boundaries, and for
// the adjoint the gradient's component stride keeps each component block on
// a 16-byte boundary.
#pragma once

#include "kernels_adj.cuh"
#include "prefetch.cuh"

namespace cupcfd_gpu {


// What thread 0 actually staged for a tile, read by every thread of the CTA.
struct StageHdr {
    int entStart, entN;  // entries [entStart, entStart + entN) are in shared memory
    int fs, fgN;         // face records [fs, fs + fgN)
    int gfA, gfN;        // gface [gfA, gfA + gfN)
    int full;            // the tile's cell arrays are staged
    unsigned w03, w47;
    int pad[7];
};

// Shared-memory layout: mbarriers, stage headers, then STAGES stage buffers.
// Offsets inside a stage buffer are in bytes; every one is a multiple of 16.
struct StageLayout {
    int entCap, faceCap, gfCap;  // capacities in entries / faces / floats
    int ent, fg, gf;             // offsets of the three face-side ranges
    int c0, c1, c2, c3;          // offsets of the cell arrays
    int bytes;                   // one stage buffer
    int base;                    // offset of stage 0
};

struct StagedArgs {
    int nC, nF, nTiles;
    const TileDesc *desc;
    const int2 *inc;
    StageLayout L;
    int spinLimit;
    int *err;  // bit 1: a stage wait expired
};


__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// makes the initialised barriers visible to the async (bulk-copy) proxy
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// global -> shared bulk copy; both addresses 16-byte aligned, bytes a
// positive multiple of 16; completion is counted on `bar`
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// Waits for the phase of `bar` with the given parity to complete, at most
// `limit` polls (each poll may suspend the thread for a hardware-chosen
// interval). Returns false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int limit) {
    unsigned a = smem_u32(bar);
    for (int i = 0; i < limit; i++) {
        unsigned ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ TileDesc load_desc(const TileDesc *d) {
    const int4 *p = reinterpret_cast<const int4 *>(d);
    int4 a = __ldg(p), b = __ldg(p + 1);
    TileDesc r;
    r.entStart = a.x; r.entEnd = a.y; r.fs = a.z; r.fe = a.w;
    r.w03 = (unsigned) b.x; r.w47 = (unsigned) b.y; r.pad0 = b.z; r.pad1 = b.w;
    return r;
}

// Issues the face-side ranges of a tile into its stage and fills the header.
// Called by thread 0 only; cellSrc / cellBytes / cellOff list the
// cell-array copies (source array, bytes per tile, stage offset), made only
// when the tile lies wholly inside nC. The transaction count posted on the
// barrier equals the bytes issued.
template <int NCELL>
__device__ __forceinline__ void stage_issue(unsigned char *smem, const StagedArgs &a, int stage, int t,
                                            const TileDesc &d, const void *fg, int fgSize, const float *gface,
                                            const void *const (&cellSrc)[NCELL], const int (&cellBytes)[NCELL],
                                            const int (&cellOff)[NCELL]) {
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem) + stage;
    StageHdr *h = reinterpret_cast<StageHdr *>(smem + 64) + stage;
    unsigned char *buf = smem + a.L.base + stage * a.L.bytes;
    int entN = min(d.entEnd - d.entStart, a.L.entCap);
    int fgN = min(d.fe - d.fs, a.L.faceCap);
    int gfA = d.fs & ~3, gfN = 0;
    if (gface) {
        int gfB = (d.fe + 3) & ~3;
        if (gfB > a.nF) gfB = d.fe & ~3;  // never read past the array
        gfN = max(0, min(gfB - gfA, a.L.gfCap));
    }
    bool full = (long long) (t + 1) * STAGED_TILE <= (long long) a.nC;
    unsigned bytes = (unsigned) entN * 8u + (unsigned) fgN * (unsigned) fgSize + (unsigned) gfN * 4u;
    if (full)
        for (int i = 0; i < NCELL; i++) bytes += (unsigned) cellBytes[i];
    h->entStart = d.entStart; h->entN = entN;
    h->fs = d.fs; h->fgN = fgN;
    h->gfA = gfA; h->gfN = gfN;
    h->full = full;
    h->w03 = d.w03; h->w47 = d.w47;
    mbar_arrive_expect_tx(bar, bytes);
    if (entN > 0) bulk_g2s(buf + a.L.ent, a.inc + d.entStart, (unsigned) entN * 8u, bar);
    if (fgN > 0)
        bulk_g2s(buf + a.L.fg, static_cast<const unsigned char *>(fg) + (size_t) d.fs * fgSize,
                 (unsigned) fgN * (unsigned) fgSize, bar);
    if (gfN > 0) bulk_g2s(buf + a.L.gf, gface + gfA, (unsigned) gfN * 4u, bar);
    if (full)
        for (int i = 0; i < NCELL; i++)
            bulk_g2s(buf + cellOff[i], static_cast<const unsigned char *>(cellSrc[i]) + (size_t) t * cellBytes[i],
                     (unsigned) cellBytes[i], bar);
}

// This thread's slice width and the offset of its slice's first entry
// within the tile's entries.
__device__ __forceinline__ void slice_of(const StageHdr &h, int sl, int &w, int &off) {
    off = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        int wi = (int) (((i < 4 ? h.w03 : h.w47) >> (8 * (i & 3))) & 0xffu);
        if (i < sl) off += wi;
        if (i == sl) w = wi;
    }
    off *= 32;
}

// Sum of v over the CTA, in k_fwd_f32's order (warp butterfly, then warps
// in order), stored by thread 0 to out[idx].
__device__ __forceinline__ void tile_sum_store(double v, double *out, int idx, double *red) {
    for (int k = 16; k > 0; k >>= 1) v += __shfl_xor_sync(0xffffffffu, v, k);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < STAGED_TILE / 32; i++) t += red[i];
        out[idx] = t;
    }
}

// entries per chunk, and resident CTAs per SM the registers must allow
#ifndef CUPCFD_STAGED_CHUNK
#define CUPCFD_STAGED_CHUNK 6
#endif
#ifndef CUPCFD_STAGED_ADJ_CHUNK
#define CUPCFD_STAGED_ADJ_CHUNK 3
#endif
#ifndef CUPCFD_MINB_STAGED
#define CUPCFD_MINB_STAGED 2
#endif

// ---------------------------------------------------------------------------
// Staged forward, FP32 (same arithmetic as fwd_cell_f32).
// ---------------------------------------------------------------------------
template <int S>
__global__ void __launch_bounds__(STAGED_TILE, CUPCFD_MINB_STAGED)
    k_fwd_f32_staged(StagedArgs a, const float4 *__restrict__ fg, const float *__restrict__ phi,
                     const float *__restrict__ phiB, const double *__restrict__ vol, const float4 *__restrict__ st,
                     const float *__restrict__ gface, float *__restrict__ g, float *__restrict__ mflux,
                     double *__restrict__ lossPart, int64_t ldc) {
    constexpr int CH = CUPCFD_STAGED_CHUNK;
    constexpr int T = STAGED_TILE;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ double red[T / 32];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    const StageHdr *hdrs = reinterpret_cast<const StageHdr *>(smem + 64);
    const int tid = threadIdx.x, G = gridDim.x;
    const void *const cellSrc[3] = {phi, st, vol};
    const int cellBytes[3] = {T * 4, T * 16, T * 8};
    const int cellOff[3] = {a.L.c0, a.L.c1, a.L.c2};
    TileDesc nd;
    if (tid == 0) {
        for (int s = 0; s < S; s++) mbar_init(bars + s, 1);
        mbar_init_fence();
        for (int s = 0; s < S - 1; s++) {
            int t = blockIdx.x + s * G;
            if (t < a.nTiles) stage_issue<3>(smem, a, s, t, load_desc(a.desc + t), fg, 16, gface, cellSrc, cellBytes, cellOff);
        }
        int tn = blockIdx.x + (S - 1) * G;
        if (tn < a.nTiles) nd = load_desc(a.desc + tn);
    }
    __syncthreads();
    int n = 0;
    for (int t = blockIdx.x; t < a.nTiles; t += G, n++) {
        const int s = n % S;
        if (tid == 0) {
            int ti = t + (S - 1) * G;
            if (ti < a.nTiles) {
                stage_issue<3>(smem, a, (n + S - 1) % S, ti, nd, fg, 16, gface, cellSrc, cellBytes, cellOff);
                int tn = ti + G;
                if (tn < a.nTiles) nd = load_desc(a.desc + tn);
            }
        }
        if (!mbar_wait(bars + s, (unsigned) (n / S) & 1u, a.spinLimit)) atomicOr(a.err, 2);
        const StageHdr &h = hdrs[s];
        const unsigned char *buf = smem + a.L.base + s * a.L.bytes;
        const int2 *sent = reinterpret_cast<const int2 *>(buf + a.L.ent);
        const float4 *sfg = reinterpret_cast<const float4 *>(buf + a.L.fg);
        const float *sgf = reinterpret_cast<const float *>(buf + a.L.gf);
        const float *sphi = reinterpret_cast<const float *>(buf + a.L.c0);
        const float4 *sst = reinterpret_cast<const float4 *>(buf + a.L.c1);
        const double *svol = reinterpret_cast<const double *>(buf + a.L.c2);
        const int c0 = t * T, c = c0 + tid;
        const bool full = h.full;
        double l = 0.0;
        if (c < a.nC) {
            int w, off;
            slice_of(h, tid >> 5, w, off);
            const int q0 = off + (tid & 31);
            float phic = full ? sphi[tid] : phi[c];
            float4 sc = full ? sst[tid] : st[c];
            Acc2 ax, ay, az;
            double lsum = 0.0;
            for (int k0 = 0; k0 < w; k0 += CH) {
                int2 en[CH];
#pragma unroll
                for (int j = 0; j < CH; j++) {
                    int q = q0 + 32 * (k0 + j);
                    en[j] = (k0 + j < w) ? (q < h.entN ? sent[q] : __ldg(a.inc + h.entStart + q)) : make_int2(-1, -1);
                }
                float4 G4[CH], so[CH];
                float pv[CH], gf[CH];
#pragma unroll
                for (int j = 0; j < CH; j++) {
                    int code = en[j].x;
                    if (code < 0) continue;
                    int f = code >> 1, o = en[j].y;
                    G4[j] = (unsigned) (f - h.fs) < (unsigned) h.fgN ? sfg[f - h.fs] : __ldg(fg + f);
                    bool in = full && (unsigned) (o - c0) < (unsigned) T;
                    pv[j] = o >= 0 ? (in ? sphi[o - c0] : __ldg(phi + o)) : __ldg(phiB + (-1 - o));
                    if (o >= 0 && !(code & 1)) {
                        so[j] = in ? sst[o - c0] : __ldg(st + o);
                        gf[j] = gface ? ((unsigned) (f - h.gfA) < (unsigned) h.gfN ? sgf[f - h.gfA] : __ldg(gface + f)) : 0.f;
                    }
                }
#pragma unroll
                for (int j = 0; j < CH; j++) {
                    int code = en[j].x;
                    if (code < 0) continue;
                    bool isN = code & 1;
                    int o = en[j].y;
                    float phif;
                    if (o < 0) {
                        phif = pv[j];
                    } else {
                        float facn = G4[j].w, facp = 1.f - facn;
                        phif = isN ? fmaf(facn, phic, facp * pv[j]) : fmaf(facn, pv[j], facp * phic);
                        if (!isN) {
                            float denf = fmaf(facn, so[j].x, facp * sc.x);
                            float uF = fmaf(facn, so[j].y, facp * sc.y);
                            float vF = fmaf(facn, so[j].z, facp * sc.z);
                            float wF = fmaf(facn, so[j].w, facp * sc.w);
                            float m = denf * fmaf(uF, G4[j].x, fmaf(vF, G4[j].y, wF * G4[j].z));
                            mflux[code >> 1] = m;
                            lsum += (double) gf[j] * (double) m;
                        }
                    }
                    ax.add_prod(phif, G4[j].x); ay.add_prod(phif, G4[j].y); az.add_prod(phif, G4[j].z);
                }
            }
            double V = full ? svol[tid] : vol[c];
            double fact = 1.0 / V;
            float rx = (float) (ax.value() * fact), ry = (float) (ay.value() * fact), rz = (float) (az.value() * fact);
            g[c] = rx; g[ldc + c] = ry; g[2 * ldc + c] = rz;
            l = lsum + V * ((double) rx * rx + (double) ry * ry + (double) rz * rz);
        }
        if (lossPart) tile_sum_store(l, lossPart, t, red);
        __syncthreads();  // stage s and red[] are free again
    }
}

// ---------------------------------------------------------------------------
// Staged adjoint of the benchmark loss, FP32 (same arithmetic as
// adj_cell_f32 with both the gradient and the mass parts, hscale = 2).
// ---------------------------------------------------------------------------
template <int S>
__global__ void __launch_bounds__(STAGED_TILE, CUPCFD_MINB_STAGED)
    k_adj_f32_staged(StagedArgs a, const float4 *__restrict__ fg, const float *__restrict__ g, float hscale,
                     const float4 *__restrict__ st, const float *__restrict__ gface, float *__restrict__ phibar,
                     float *__restrict__ phibBar, float4 *__restrict__ stbar, int64_t ldc) {
    constexpr int CH = CUPCFD_STAGED_ADJ_CHUNK;
    constexpr int T = STAGED_TILE;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    const StageHdr *hdrs = reinterpret_cast<const StageHdr *>(smem + 64);
    const int tid = threadIdx.x, G = gridDim.x;
    const void *const cellSrc[4] = {g, g + ldc, g + 2 * ldc, st};
    const int cellBytes[4] = {T * 4, T * 4, T * 4, T * 16};
    const int cellOff[4] = {a.L.c0, a.L.c1, a.L.c2, a.L.c3};
    TileDesc nd;
    if (tid == 0) {
        for (int s = 0; s < S; s++) mbar_init(bars + s, 1);
        mbar_init_fence();
        for (int s = 0; s < S - 1; s++) {
            int t = blockIdx.x + s * G;
            if (t < a.nTiles) stage_issue<4>(smem, a, s, t, load_desc(a.desc + t), fg, 16, gface, cellSrc, cellBytes, cellOff);
        }
        int tn = blockIdx.x + (S - 1) * G;
        if (tn < a.nTiles) nd = load_desc(a.desc + tn);
    }
    __syncthreads();
    int n = 0;
    for (int t = blockIdx.x; t < a.nTiles; t += G, n++) {
        const int s = n % S;
        if (tid == 0) {
            int ti = t + (S - 1) * G;
            if (ti < a.nTiles) {
                stage_issue<4>(smem, a, (n + S - 1) % S, ti, nd, fg, 16, gface, cellSrc, cellBytes, cellOff);
                int tn = ti + G;
                if (tn < a.nTiles) nd = load_desc(a.desc + tn);
            }
        }
        if (!mbar_wait(bars + s, (unsigned) (n / S) & 1u, a.spinLimit)) atomicOr(a.err, 2);
        const StageHdr &h = hdrs[s];
        const unsigned char *buf = smem + a.L.base + s * a.L.bytes;
        const int2 *sent = reinterpret_cast<const int2 *>(buf + a.L.ent);
        const float4 *sfg = reinterpret_cast<const float4 *>(buf + a.L.fg);
        const float *sgf = reinterpret_cast<const float *>(buf + a.L.gf);
        const float *sg0 = reinterpret_cast<const float *>(buf + a.L.c0);
        const float *sg1 = reinterpret_cast<const float *>(buf + a.L.c1);
        const float *sg2 = reinterpret_cast<const float *>(buf + a.L.c2);
        const float4 *sst = reinterpret_cast<const float4 *>(buf + a.L.c3);
        const int c0 = t * T, c = c0 + tid;
        const bool full = h.full;
        if (c < a.nC) {
            int w, off;
            slice_of(h, tid >> 5, w, off);
            const int q0 = off + (tid & 31);
            float hx = hscale * (full ? sg0[tid] : __ldg(g + c));
            float hy = hscale * (full ? sg1[tid] : __ldg(g + ldc + c));
            float hz = hscale * (full ? sg2[tid] : __ldg(g + 2 * ldc + c));
            float4 sc = full ? sst[tid] : st[c];
            Acc2 pb, rb, ub, vb, wb;
            for (int k0 = 0; k0 < w; k0 += CH) {
                int2 en[CH];
#pragma unroll
                for (int j = 0; j < CH; j++) {
                    int q = q0 + 32 * (k0 + j);
                    en[j] = (k0 + j < w) ? (q < h.entN ? sent[q] : __ldg(a.inc + h.entStart + q)) : make_int2(-1, -1);
                }
                float4 G4[CH], so[CH];
                float go[CH][3], gf[CH];
#pragma unroll
                for (int j = 0; j < CH; j++) {
                    int code = en[j].x;
                    if (code < 0) continue;
                    int f = code >> 1, o = en[j].y;
                    G4[j] = (unsigned) (f - h.fs) < (unsigned) h.fgN ? sfg[f - h.fs] : __ldg(fg + f);
                    if (o < 0) continue;
                    bool in = full && (unsigned) (o - c0) < (unsigned) T;
                    if (in) {
                        go[j][0] = sg0[o - c0]; go[j][1] = sg1[o - c0]; go[j][2] = sg2[o - c0];
                        so[j] = sst[o - c0];
                    } else {
                        go[j][0] = __ldg(g + o); go[j][1] = __ldg(g + ldc + o); go[j][2] = __ldg(g + 2 * ldc + o);
                        so[j] = __ldg(st + o);
                    }
                    gf[j] = (unsigned) (f - h.gfA) < (unsigned) h.gfN ? sgf[f - h.gfA] : __ldg(gface + f);
                }
#pragma unroll
                for (int j = 0; j < CH; j++) {
                    int code = en[j].x;
                    if (code < 0) continue;
                    int o = en[j].y;
                    if (o < 0) {
                        phibBar[-1 - o] = fmaf(hx, G4[j].x, fmaf(hy, G4[j].y, hz * G4[j].z));
                        continue;
                    }
                    bool isN = code & 1;
                    float facn = G4[j].w, facp = 1.f - facn;
                    float wc = isN ? facn : facp, wo = isN ? facp : facn;
                    float sx = fmaf(hscale, go[j][0], hx), sy = fmaf(hscale, go[j][1], hy), sz = fmaf(hscale, go[j][2], hz);
                    pb.add_prod(wc, fmaf(sx, G4[j].x, fmaf(sy, G4[j].y, sz * G4[j].z)));
                    float denf = fmaf(wc, sc.x, wo * so[j].x);
                    float uF = fmaf(wc, sc.y, wo * so[j].y), vF = fmaf(wc, sc.z, wo * so[j].z), wF = fmaf(wc, sc.w, wo * so[j].w);
                    float am = wc * gf[j];
                    rb.add_prod(am, fmaf(uF, G4[j].x, fmaf(vF, G4[j].y, wF * G4[j].z)));
                    float b = am * denf;
                    ub.add_prod(b, G4[j].x); vb.add_prod(b, G4[j].y); wb.add_prod(b, G4[j].z);
                }
            }
            phibar[c] = (float) pb.value();
            stbar[c] = make_float4((float) rb.value(), (float) ub.value(), (float) vb.value(), (float) wb.value());
        }
        __syncthreads();  // stage s is free again
    }
}

// ---------------------------------------------------------------------------
// L2 prefetch variant: the unstaged one-cell-per-thread kernels (the same
// per-cell bodies, so bit-identical results), where one lane per 256-cell
// block asks L2 to fetch the contiguous ranges of the tile `dist` blocks
// ahead (cp.async.bulk.prefetch.L2). Shared memory and L1 are untouched;
// the streamed loads of later blocks become L2 hits.
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(STAGED_TILE, CUPCFD_MINB_F32)
    k_fwd_f32_pf(int nC, SellView sv, const float4 *__restrict__ fg, const float *__restrict__ phi,
                 const float *__restrict__ phiB, const double *__restrict__ vol, const float4 *__restrict__ st,
                 const float *__restrict__ gface, float *__restrict__ g, float *__restrict__ mflux,
                 double *__restrict__ lossPart, int64_t ldc, PrefetchArgs pf) {
    constexpr int T = STAGED_TILE;
    int c = blockIdx.x * T + threadIdx.x;
    const int tp = blockIdx.x + pf.dist;
    const bool lead = threadIdx.x == T - 32 && tp < pf.nTiles;
    __shared__ int4 s_rng;
    const void *const cellSrc[3] = {phi, st, vol};
    const int cellBytes[3] = {T * 4, T * 16, T * 8};
    if (lead) fetch_ranges_async(&s_rng, pf.desc + tp);
    double l = 0.0;
    if (c < nC) l = fwd_cell_f32<CUPCFD_FWD_CHUNK>(c, sv, fg, phi, phiB, vol, st, gface, g, mflux, ldc);
    if (lead) prefetch_tile<3>(pf, tp, ranges_ready(&s_rng), fg, 16, gface, cellSrc, cellBytes);
    if (lossPart) block_sum_store<T>(l, lossPart);
}

__global__ void __launch_bounds__(STAGED_TILE, CUPCFD_MINB_F32)
    k_adj_f32_pf(int nC, SellView sv, const float4 *__restrict__ fg, const float *__restrict__ g, float hscale,
                 const float4 *__restrict__ st, const float *__restrict__ gface, float *__restrict__ phibar,
                 float *__restrict__ phibBar, float4 *__restrict__ stbar, int64_t ldc, PrefetchArgs pf) {
    constexpr int T = STAGED_TILE;
    int c = blockIdx.x * T + threadIdx.x;
    const int tp = blockIdx.x + pf.dist;
    const bool lead = threadIdx.x == T - 32 && tp < pf.nTiles;
    __shared__ int4 s_rng;
    const void *const cellSrc[4] = {g, g + ldc, g + 2 * ldc, st};
    const int cellBytes[4] = {T * 4, T * 4, T * 4, T * 16};
    if (lead) fetch_ranges_async(&s_rng, pf.desc + tp);
    if (c < nC) adj_cell_f32<false>(c, sv, fg, g, hscale, st, gface, phibar, phibBar, stbar, ldc);
    if (lead) prefetch_tile<4>(pf, tp, ranges_ready(&s_rng), fg, 16, gface, cellSrc, cellBytes);
}

// FP64 forward (fwd_cell_f64, exact reference arithmetic) with the same L2
// prefetch; the state's four component blocks are prefetched one by one.
__global__ void __launch_bounds__(STAGED_TILE, CUPCFD_MINB_FWD_F64)
    k_fwd_f64_pf(int nC, SellView sv, const double4 *__restrict__ fg, const double *__restrict__ phi,
                 const double *__restrict__ phiB, const double *__restrict__ vol, const double *__restrict__ st,
                 const double *__restrict__ gface, double *__restrict__ g, double *__restrict__ mflux,
                 double *__restrict__ lossPart, int64_t ldc, PrefetchArgs pf) {
    constexpr int T = STAGED_TILE;
    int c = blockIdx.x * T + threadIdx.x;
    const int tp = blockIdx.x + pf.dist;
    const bool lead = threadIdx.x == T - 32 && tp < pf.nTiles;
    __shared__ int4 s_rng;
    const void *const cellSrc[6] = {phi, vol, st, st + ldc, st + 2 * ldc, st + 3 * ldc};
    const int cellBytes[6] = {T * 8, T * 8, T * 8, T * 8, T * 8, T * 8};
    if (lead) fetch_ranges_async(&s_rng, pf.desc + tp);
    double l = 0.0;
    if (c < nC) l = fwd_cell_f64<CUPCFD_FWD_CHUNK_F64>(c, sv, fg, phi, phiB, vol, st, gface, g, mflux, ldc);
    if (lead) prefetch_tile<6>(pf, tp, ranges_ready(&s_rng), fg, 32, gface, cellSrc, cellBytes);
    if (lossPart) block_sum_store<T>(l, lossPart);
}

// FP64 adjoint (adj_cell_f64) with the same L2 prefetch.
__global__ void __launch_bounds__(STAGED_TILE, CUPCFD_MINB_ADJ_F64)
    k_adj_f64_pf(int nC, SellView sv, const double4 *__restrict__ fg, const double *__restrict__ g, double hscale,
                 const double *__restrict__ st, const double *__restrict__ gface, double *__restrict__ phibar,
                 double *__restrict__ phibBar, double *__restrict__ stbar, int64_t ldc, PrefetchArgs pf) {
    constexpr int T = STAGED_TILE;
    int c = blockIdx.x * T + threadIdx.x;
    const int tp = blockIdx.x + pf.dist;
    const bool lead = threadIdx.x == T - 32 && tp < pf.nTiles;
    __shared__ int4 s_rng;
    const void *const cellSrc[7] = {g, g + ldc, g + 2 * ldc, st, st + ldc, st + 2 * ldc, st + 3 * ldc};
    const int cellBytes[7] = {T * 8, T * 8, T * 8, T * 8, T * 8, T * 8, T * 8};
    if (lead) fetch_ranges_async(&s_rng, pf.desc + tp);
    if (c < nC) adj_cell_f64<false>(c, sv, fg, g, hscale, st, gface, phibar, phibBar, stbar, ldc);
    if (lead) prefetch_tile<7>(pf, tp, ranges_ready(&s_rng), fg, 32, gface, cellSrc, cellBytes);
}

// Forward with the mass-flux adjoint (fwd_madj_cell_f32), L2 prefetch as
// k_fwd_f32_pf. With k_gadj_f32_pf it forms the two-launch forward+adjoint:
// the state and gface are then read by one pass only.
#ifndef CUPCFD_FWD_MADJ_CHUNK
#define CUPCFD_FWD_MADJ_CHUNK 2
#endif
#ifndef CUPCFD_MINB_FWD_MADJ
#define CUPCFD_MINB_FWD_MADJ 4
#endif
__global__ void __launch_bounds__(STAGED_TILE, CUPCFD_MINB_FWD_MADJ)
    k_fwd_madj_f32_pf(int nC, SellView sv, const float4 *__restrict__ fg, const float *__restrict__ phi,
                      const float *__restrict__ phiB, const double *__restrict__ vol, const float4 *__restrict__ st,
                      const float *__restrict__ gface, float *__restrict__ g, float *__restrict__ mflux,
                      float4 *__restrict__ stbar, double *__restrict__ lossPart, int64_t ldc, PrefetchArgs pf) {
    constexpr int T = STAGED_TILE;
    int c = blockIdx.x * T + threadIdx.x;
    const int tp = blockIdx.x + pf.dist;
    const bool lead = threadIdx.x == T - 32 && tp < pf.nTiles;
    __shared__ int4 s_rng;
    const void *const cellSrc[3] = {phi, st, vol};
    const int cellBytes[3] = {T * 4, T * 16, T * 8};
    if (lead) fetch_ranges_async(&s_rng, pf.desc + tp);
    double l = 0.0;
    if (c < nC) l = fwd_madj_cell_f32<CUPCFD_FWD_MADJ_CHUNK>(c, sv, fg, phi, phiB, vol, st, gface, g, mflux, stbar, ldc);
    if (lead) prefetch_tile<3>(pf, tp, ranges_ready(&s_rng), fg, 16, gface, cellSrc, cellBytes);
    if (lossPart) block_sum_store<T>(l, lossPart);
}

// Gradient part of the adjoint only (adj_cell_f32 without the mass part):
// phibar and phibBar.
__global__ void __launch_bounds__(STAGED_TILE, CUPCFD_MINB_F32)
    k_gadj_f32_pf(int nC, SellView sv, const float4 *__restrict__ fg, const float *__restrict__ g, float hscale,
                  float *__restrict__ phibar, float *__restrict__ phibBar, int64_t ldc, PrefetchArgs pf) {
    constexpr int T = STAGED_TILE;
    int c = blockIdx.x * T + threadIdx.x;
    const int tp = blockIdx.x + pf.dist;
    const bool lead = threadIdx.x == T - 32 && tp < pf.nTiles;
    __shared__ int4 s_rng;
    const void *const cellSrc[3] = {g, g + ldc, g + 2 * ldc};
    const int cellBytes[3] = {T * 4, T * 4, T * 4};
    if (lead) fetch_ranges_async(&s_rng, pf.desc + tp);
    if (c < nC) adj_cell_f32<false>(c, sv, fg, g, hscale, nullptr, nullptr, phibar, phibBar, nullptr, ldc);
    if (lead) prefetch_tile<3>(pf, tp, ranges_ready(&s_rng), fg, 16, (const float *) nullptr, cellSrc, cellBytes);
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
    int t = fcells[f].x / STAGED_TILE;
    int tp = f > 0 ? fcells[f - 1].x / STAGED_TILE : -1;
    if (t < tp) atomicOr(bad, 1);
    for (int u = tp + 1; u <= t; u++) start[u] = f;
    if (f == nF - 1)
        for (int u = t + 1; u <= nTiles; u++) start[u] = nF;
}

__global__ void k_tile_desc(int nTiles, int nSlices, const int *__restrict__ slicePtr, const int *__restrict__ start,
                            TileDesc *__restrict__ desc, int *__restrict__ maxima) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nTiles) return;
    int s0 = t * (STAGED_TILE / 32);
    TileDesc d;
    d.entStart = slicePtr[s0];
    d.entEnd = slicePtr[min(s0 + STAGED_TILE / 32, nSlices)];
    d.fs = start[t];
    d.fe = start[t + 1];
    unsigned w[2] = {0u, 0u};
    int wmax = 0;
    for (int i = 0; i < STAGED_TILE / 32; i++) {
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
