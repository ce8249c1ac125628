// Adjoint kernels, the fused forward pass and the full-semantics mass flux.
//
// Adjoints are the transposed gathers over the same SELL-32 incidence lists:
// a cell collects, over its faces in ascending reference face id, the
// sensitivities that the forward face loop spread from that face into both
// of its cells. One thread per cell, no floating-point atomics.
#pragma once

#include "kernels.cuh"

namespace cupcfd_gpu {

// ---------------------------------------------------------------------------
// Fused forward pass of the benchmark pipeline: gradient (nGradient = 1) and
// the plain mass flux of the faces this cell owns, plus the per-block FP64
// partial of L = sum_c V_c |g_c|^2 + sum_f gface_f m_f.
// FP64 version: same arithmetic as k_grad_f64 / k_mass_plain_f64.
// ---------------------------------------------------------------------------
template <int BLOCK>
__device__ __forceinline__ void block_sum_store(double v, double *out) {
    __shared__ double red[BLOCK / 32];
    for (int k = 16; k > 0; k >>= 1) v += __shfl_xor_sync(0xffffffffu, v, k);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < BLOCK / 32; i++) t += red[i];
        out[blockIdx.x] = t;
    }
}

// Per-cell body of the FP64 fused forward (exact reference arithmetic).
// Returns this cell's loss contribution (0 when gface is null).
template <int CH, int WF = 0>
__device__ __forceinline__ double fwd_cell_f64(int c, const SellView &sv, const double4 *__restrict__ fg,
                                               const double *__restrict__ phi, const double *__restrict__ phiB,
                                               const double *__restrict__ vol, const double *__restrict__ st,
                                               const double *__restrict__ gface, double *__restrict__ g,
                                               double *__restrict__ mflux, int64_t ldc) {
    int w;
    const int2 *e = cell_entries(sv, c, w);
    if (WF) w = WF;  // every cell has exactly WF entries (a full, uniform slice width)
    double phic = phi[c];
    double r0 = st[c], u0 = st[ldc + c], v0 = st[2 * ldc + c], w0 = st[3 * ldc + c];
    double ax = 0.0, ay = 0.0, az = 0.0, lsum = 0.0;
    for (int k0 = 0; k0 < w; k0 += CH) {
        int2 en[CH];
        load_entries(e, k0, w, en);
        double4 G[CH];
        double pv[CH], so[CH][4], gf[CH];
#pragma unroll
        for (int j = 0; j < CH; j++) {
            int code = en[j].x;
            if (!WF && code < 0) continue;
            int f = code >> 1, o = en[j].y;
            G[j] = ldg4(fg + f);
            pv[j] = o >= 0 ? __ldg(phi + o) : __ldg(phiB + (-1 - o));
            if (o >= 0 && !(code & 1)) {
                so[j][0] = __ldg(st + o); so[j][1] = __ldg(st + ldc + o);
                so[j][2] = __ldg(st + 2 * ldc + o); so[j][3] = __ldg(st + 3 * ldc + o);
                gf[j] = gface ? __ldg(gface + f) : 0.0;
            }
        }
#pragma unroll
        for (int j = 0; j < CH; j++) {
            int code = en[j].x;
            if (!WF && code < 0) continue;
            bool isN = code & 1;
            int o = en[j].y;
            double phif;
            if (o < 0) {
                phif = pv[j];
            } else {
                double facn = G[j].w, facp = ds(1.0, facn);
                phif = isN ? da(dm(phic, facn), dm(pv[j], facp)) : da(dm(pv[j], facn), dm(phic, facp));
                if (!isN) {  // the owner computes m_f: P = c, N = o
                    double denf = da(dm(so[j][0], facn), dm(r0, facp));
                    double uF = da(dm(so[j][1], facn), dm(u0, facp));
                    double vF = da(dm(so[j][2], facn), dm(v0, facp));
                    double wF = da(dm(so[j][3], facn), dm(w0, facp));
                    double m = dm(denf, da(da(dm(uF, G[j].x), dm(vF, G[j].y)), dm(wF, G[j].z)));
                    mflux[code >> 1] = m;
                    lsum = __fma_rn(gf[j], m, lsum);
                }
            }
            ax = da(ax, dm(phif, G[j].x)); ay = da(ay, dm(phif, G[j].y)); az = da(az, dm(phif, G[j].z));
        }
    }
    double V = vol[c];
    double fact = dvd(1.0, V);
    ax = dm(ax, fact); ay = dm(ay, fact); az = dm(az, fact);
    g[c] = ax; g[ldc + c] = ay; g[2 * ldc + c] = az;
    return __fma_rn(V, __fma_rn(ax, ax, __fma_rn(ay, ay, __dmul_rn(az, az))), lsum);
}

// Per-cell body of the FP32 fused forward; state as float4 {rho, u, v, w}.
template <int CH, int WF = 0>
__device__ __forceinline__ double fwd_cell_f32(int c, const SellView &sv, const float4 *__restrict__ fg,
                                               const float *__restrict__ phi, const float *__restrict__ phiB,
                                               const double *__restrict__ vol, const float4 *__restrict__ st,
                                               const float *__restrict__ gface, float *__restrict__ g,
                                               float *__restrict__ mflux, int64_t ldc) {
    int w;
    const int2 *e = cell_entries(sv, c, w);
    if (WF) w = WF;  // every cell has exactly WF entries (a full, uniform slice width)
    float phic = phi[c];
    float4 sc = st[c];
    Acc2x2 axy;  // (gx, gy) packed, gz alone
    Acc2 az;
    double lsum = 0.0;
    for (int k0 = 0; k0 < w; k0 += CH) {
        int2 en[CH];
        load_entries(e, k0, w, en);
        float4 G[CH], so[CH];
        float pv[CH], gf[CH];
#pragma unroll
        for (int j = 0; j < CH; j++) {
            int code = en[j].x;
            if (!WF && code < 0) continue;
            int f = code >> 1, o = en[j].y;
            G[j] = __ldg(fg + f);
            pv[j] = o >= 0 ? __ldg(phi + o) : __ldg(phiB + (-1 - o));
            if (o >= 0 && !(code & 1)) {
                so[j] = __ldg(st + o);
                gf[j] = gface ? __ldg(gface + f) : 0.f;
            }
        }
#pragma unroll
        for (int j = 0; j < CH; j++) {
            int code = en[j].x;
            if (!WF && code < 0) continue;
            bool isN = code & 1;
            int o = en[j].y;
            float phif;
            if (o < 0) {
                phif = pv[j];
            } else {
                const FaceW fw = face_weights(G[j].w, isN);
                phif = interp(fw, phic, pv[j]);
                if (!isN) {  // the owner computes m_f
                    const float4 sf = interp4(fw, sc, so[j]);
                    const float m = sf.x * udots(sf, G[j]);
                    mflux[code >> 1] = m;
                    lsum = __fma_rn((double) gf[j], (double) m, lsum);
                }
            }
            axy.add_prod(make_float2(phif, phif), make_float2(G[j].x, G[j].y));
            az.add_prod(phif, G[j].z);
        }
    }
    double V = vol[c];
    double fact = 1.0 / V;
    float rx = (float) (axy.x() * fact), ry = (float) (axy.y() * fact), rz = (float) (az.value() * fact);
    g[c] = rx; g[ldc + c] = ry; g[2 * ldc + c] = rz;
    return __fma_rn(V, __fma_rn((double) rx, (double) rx, __fma_rn((double) ry, (double) ry, __dmul_rn((double) rz, (double) rz))),
                    lsum);
}

// Per-cell body of the FP32 forward that also runs the mass-flux part of
// the adjoint (which needs only inputs: state, gface and geometry): the
// forward of fwd_cell_f32 plus, over every interior face, the rhobar / ubar
// accumulation of adj_cell_f32, with the same arithmetic in the same face
// order, so stbar equals the one the full adjoint writes bit for bit.
template <int CH, int PIPE = 0, int WF = 0>
__device__ __forceinline__ double fwd_madj_cell_f32(int c, const SellView &sv, const float4 *__restrict__ fg,
                                                    const float *__restrict__ phi, const float *__restrict__ phiB,
                                                    const double *__restrict__ vol, const float4 *__restrict__ st,
                                                    const float *__restrict__ gface, float *__restrict__ g,
                                                    float *__restrict__ mflux, float4 *__restrict__ stbar,
                                                    int64_t ldc) {
    int w;
    const int2 *e = cell_entries(sv, c, w);
    if (WF) w = WF;  // every cell has exactly WF entries (a full, uniform slice width)
    float phic = phi[c];
    float4 sc = st[c];
    // seven compensated sums in packed pairs: (gx, gy), (gz, rhobar), (ubar, vbar), wbar
    Acc2x2 axy, azr, uvb;
    Acc2 wb;
    double lsum = 0.0;
    int2 en[CH];
    load_entries(e, 0, w, en);
    for (int k0 = 0; k0 < w; k0 += CH) {
        float4 G[CH], so[CH];
        float pv[CH], gf[CH];
#pragma unroll
        for (int j = 0; j < CH; j++) {
            int code = en[j].x;
            if (!WF && code < 0) continue;
            int f = code >> 1, o = en[j].y;
            G[j] = __ldg(fg + f);
            pv[j] = o >= 0 ? __ldg(phi + o) : __ldg(phiB + (-1 - o));
            if (o >= 0) {
                so[j] = __ldg(st + o);
                gf[j] = __ldg(gface + f);
            }
        }
        int2 nx[CH];
        if (PIPE) load_entries(e, k0 + CH, w, nx);
#pragma unroll
        for (int j = 0; j < CH; j++) {
            int code = en[j].x;
            if (!WF && code < 0) continue;
            bool isN = code & 1;
            int o = en[j].y;
            float phif;
            if (o < 0) {
                phif = pv[j];
                axy.add_prod(make_float2(phif, phif), make_float2(G[j].x, G[j].y));
                azr.add_x(phif, G[j].z);
            } else {
                const FaceW fw = face_weights(G[j].w, isN);
                phif = interp(fw, phic, pv[j]);
                // rho_f and u_f . S_f from this cell's side: the owner's mass
                // flux and this cell's mass-adjoint terms (adj_cell_f32)
                const float4 sf = interp4(fw, sc, so[j]);
                const float q = udots(sf, G[j]);
                if (!isN) {
                    const float m = sf.x * q;
                    mflux[code >> 1] = m;
                    lsum = __fma_rn((double) gf[j], (double) m, lsum);
                }
                const float a = fw.wc * gf[j];
                const float b = a * sf.x;
                axy.add_prod(make_float2(phif, phif), make_float2(G[j].x, G[j].y));
                azr.add_prod(make_float2(phif, a), make_float2(G[j].z, q));
                uvb.add_prod(make_float2(b, b), make_float2(G[j].x, G[j].y));
                wb.add_prod(b, G[j].z);
            }
        }
        next_entries<PIPE>(e, k0 + CH, w, en, nx);
    }
    double V = vol[c];
    double fact = 1.0 / V;
    float rx = (float) (axy.x() * fact), ry = (float) (axy.y() * fact), rz = (float) (azr.x() * fact);
    g[c] = rx; g[ldc + c] = ry; g[2 * ldc + c] = rz;
    stbar[c] = make_float4(azr.yf(), uvb.xf(), uvb.yf(), wb.value_f());
    return __fma_rn(V, __fma_rn((double) rx, (double) rx, __fma_rn((double) ry, (double) ry, __dmul_rn((double) rz, (double) rz))),
                    lsum);
}

// ---------------------------------------------------------------------------
// Fused forward of the benchmark pipeline: gradient (nGradient = 1) and the
// plain mass flux of the faces each cell owns, plus the per-block FP64
// partial of L = sum_c V_c |g_c|^2 + sum_f gface_f m_f.
// ---------------------------------------------------------------------------
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, CUPCFD_MINB_FWD_F64) k_fwd_f64(int nC, SellView sv, const double4 *__restrict__ fg,
                                                   const double *__restrict__ phi, const double *__restrict__ phiB,
                                                   const double *__restrict__ vol, const double *__restrict__ st,
                                                   const double *__restrict__ gface, double *__restrict__ g,
                                                   double *__restrict__ mflux, double *__restrict__ lossPart, int64_t ldc) {
    int c = blockIdx.x * BLOCK + threadIdx.x;
    double l = 0.0;
    if (c < nC) l = fwd_cell_f64<CUPCFD_FWD_CHUNK_F64>(c, sv, fg, phi, phiB, vol, st, gface, g, mflux, ldc);
    if (lossPart) block_sum_store<BLOCK>(l, lossPart);
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, CUPCFD_MINB_F32) k_fwd_f32(int nC, SellView sv, const float4 *__restrict__ fg,
                                                   const float *__restrict__ phi, const float *__restrict__ phiB,
                                                   const double *__restrict__ vol, const float4 *__restrict__ st,
                                                   const float *__restrict__ gface, float *__restrict__ g,
                                                   float *__restrict__ mflux, double *__restrict__ lossPart, int64_t ldc) {
    int c = blockIdx.x * BLOCK + threadIdx.x;
    double l = 0.0;
    if (c < nC) l = fwd_cell_f32<CUPCFD_FWD_CHUNK>(c, sv, fg, phi, phiB, vol, st, gface, g, mflux, ldc);
    if (lossPart) block_sum_store<BLOCK>(l, lossPart);
}

// The benchmark loss from a forward already in memory (gradient g, mass
// fluxes m): per cell, gface_f m_f summed over the interior faces it owns in
// entry order, then V_c |g_c|^2 added, and the per-block partials of
// block_sum_store. The arithmetic and order are those of fwd_cell_f64 /
// fwd_cell_f32 / fwd_madj_cell_f32 (T = float: the FP32 values widened), so
// the partials, and the reduced loss, equal theirs bit for bit.
template <class T>
__global__ void __launch_bounds__(256) k_loss(int nC, SellView sv, const T *__restrict__ gface,
                                              const T *__restrict__ mflux, const T *__restrict__ g,
                                              const double *__restrict__ vol, double *__restrict__ lossPart,
                                              int64_t ldc) {
    int c = blockIdx.x * 256 + threadIdx.x;
    double l = 0.0;
    if (c < nC) {
        int w;
        const int2 *e = cell_entries(sv, c, w);
        double lsum = 0.0;
        for (int k = 0; k < w; k++) {
            int2 en = ld_entry(e + 32 * k);
            if (en.x < 0 || en.y < 0 || (en.x & 1)) continue;  // padding, boundary, or not the owner
            int f = en.x >> 1;
            lsum = __fma_rn((double) __ldg(gface + f), (double) __ldg(mflux + f), lsum);
        }
        double rx = g[c], ry = g[ldc + c], rz = g[2 * ldc + c];
        l = __fma_rn(vol[c], __fma_rn(rx, rx, __fma_rn(ry, ry, __dmul_rn(rz, rz))), lsum);
    }
    block_sum_store<256>(l, lossPart);
}

// Deterministic final reduction of per-block partials (fixed order): thread
// t adds part[t], part[t + blockDim], ... in that order, then a tree over
// the block. The loads of each group of 16 are issued before its adds, so
// they overlap instead of each add waiting on its own load.
// G > 1: the n block values are given as G partials each, partial k of
// block i at part[k n + i] (one per warp of a 256-cell tile, G = 8, stored
// warp-major so that these loads coalesce), summed in order from 0.0 first:
// the value block_sum_store<32 G> forms, so the result has the same bits.
template <int G>
__device__ __forceinline__ double group_value(const double *v) {
    if (G == 1) return v[0];
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < G; k++) s += v[k];
    return s;
}

// In place: part[t] becomes block t's value from its G partials (part[k n +
// t], k < G) summed in order from 0.0, the value k_reduce_partials<G> forms
// for it, so k_reduce_partials<1> over part[0, n) then gives k_reduce_partials
// <G>'s result bit for bit (each thread accumulates the same values in the
// same order). One thread per block value, reading and writing only its own
// column; many blocks, where k_reduce_partials<G> is one.
template <int G>
__global__ void __launch_bounds__(256) k_group_partials(int n, double *__restrict__ part) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double v[G];
#pragma unroll
    for (int k = 0; k < G; k++) v[k] = part[(size_t) k * n + t];
    part[t] = group_value<G>(v);
}

template <int G = 1>
__global__ void k_reduce_partials(int n, const double *__restrict__ part, double *__restrict__ out) {
    __shared__ double red[1024];
    constexpr int U = G >= 16 ? 1 : 16 / G;
    const int bd = blockDim.x;
    double t = 0.0;
    int i = threadIdx.x;
    for (; i + (U - 1) * bd < n; i += U * bd) {
        double v[U * G];
#pragma unroll
        for (int j = 0; j < U; j++)
#pragma unroll
            for (int k = 0; k < G; k++) v[j * G + k] = __ldg(part + (size_t) k * n + i + j * bd);
#pragma unroll
        for (int j = 0; j < U; j++) t += group_value<G>(v + j * G);
    }
    for (; i < n; i += bd) {
        double v[G];
#pragma unroll
        for (int k = 0; k < G; k++) v[k] = part[(size_t) k * n + i];
        t += group_value<G>(v);
    }
    red[threadIdx.x] = t;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if ((int) threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// ---------------------------------------------------------------------------
// Adjoint of the benchmark loss, one pass: with L = sum V|g|^2 + sum gface m,
// dL/dg_c = 2 V_c g_c, so h_c = dL/dg_c / V_c = 2 g_c and
//   phibar_c  = sum_{f in c, interior} w_cf (h_P + h_N) . S_f
//   phibBar_b = h_P . S_f                      (boundary face f of id b)
//   rhobar_c  = sum_f w_cf gface_f (u_f . S_f)
//   ubar_c    = sum_f w_cf gface_f rho_f S_f   (and v, w)
// with w_cf = 1 - lambda_f for the owner, lambda_f for the neighbour.
// hscale = 0 skips the gradient part (mass-only adjoint); a null gface
// skips the mass part. LDCG reads g with ld.global.cg (L2, coherent) for use
// inside a kernel that also writes g.
// ---------------------------------------------------------------------------
template <bool LDCG>
__device__ __forceinline__ float ldg_g(const float *p) { return LDCG ? __ldcg(p) : __ldg(p); }
template <bool LDCG>
__device__ __forceinline__ double ldg_g(const double *p) { return LDCG ? __ldcg(p) : __ldg(p); }

template <bool LDCG, int CH = CUPCFD_ADJ_CHUNK_F64, int WF = 0>
__device__ __forceinline__ void adj_cell_f64(int c, const SellView &sv, const double4 *__restrict__ fg,
                                             const double *g, double hscale, const double *__restrict__ st,
                                             const double *__restrict__ gface, double *__restrict__ phibar,
                                             double *__restrict__ phibBar, double *__restrict__ stbar, int64_t ldc) {
    int w;
    const int2 *e = cell_entries(sv, c, w);
    if (WF) w = WF;  // every cell has exactly WF entries (a full, uniform slice width)
    bool doG = hscale != 0.0, doM = gface != nullptr;
    double hx = 0, hy = 0, hz = 0;
    if (doG) { hx = hscale * ldg_g<LDCG>(g + c); hy = hscale * ldg_g<LDCG>(g + ldc + c); hz = hscale * ldg_g<LDCG>(g + 2 * ldc + c); }
    double r0 = 0, u0 = 0, v0 = 0, w0 = 0;
    if (doM) { r0 = st[c]; u0 = st[ldc + c]; v0 = st[2 * ldc + c]; w0 = st[3 * ldc + c]; }
    double pb = 0.0, rb = 0.0, ub = 0.0, vb = 0.0, wb = 0.0;
    for (int k0 = 0; k0 < w; k0 += CH) {
        int2 en[CH];
        load_entries(e, k0, w, en);
        double4 G[CH];
        double go[CH][3], so[CH][4], gf[CH];
#pragma unroll
        for (int j = 0; j < CH; j++) {
            int code = en[j].x;
            if (!WF && code < 0) continue;
            int f = code >> 1, o = en[j].y;
            G[j] = ldg4(fg + f);
            if (o < 0) continue;
            if (doG) { go[j][0] = ldg_g<LDCG>(g + o); go[j][1] = ldg_g<LDCG>(g + ldc + o); go[j][2] = ldg_g<LDCG>(g + 2 * ldc + o); }
            if (doM) {
                so[j][0] = __ldg(st + o); so[j][1] = __ldg(st + ldc + o);
                so[j][2] = __ldg(st + 2 * ldc + o); so[j][3] = __ldg(st + 3 * ldc + o);
                gf[j] = __ldg(gface + f);
            }
        }
#pragma unroll
        for (int j = 0; j < CH; j++) {
            int code = en[j].x;
            if (!WF && code < 0) continue;
            int o = en[j].y;
            if (o < 0) {
                if (doG) phibBar[-1 - o] = __fma_rn(hx, G[j].x, __fma_rn(hy, G[j].y, __dmul_rn(hz, G[j].z)));
                continue;
            }
            bool isN = code & 1;
            double facn = G[j].w, facp = 1.0 - facn;
            double wc = isN ? facn : facp, wo = isN ? facp : facn;
            if (doG)
                pb = __fma_rn(wc, __fma_rn(__fma_rn(hscale, go[j][0], hx), G[j].x,
                                           __fma_rn(__fma_rn(hscale, go[j][1], hy), G[j].y,
                                                    __dmul_rn(__fma_rn(hscale, go[j][2], hz), G[j].z))),
                              pb);
            if (doM) {
                double denf = __fma_rn(wc, r0, __dmul_rn(wo, so[j][0]));
                double uF = __fma_rn(wc, u0, __dmul_rn(wo, so[j][1]));
                double vF = __fma_rn(wc, v0, __dmul_rn(wo, so[j][2]));
                double wF = __fma_rn(wc, w0, __dmul_rn(wo, so[j][3]));
                double a = __dmul_rn(wc, gf[j]);
                rb = __fma_rn(a, __fma_rn(uF, G[j].x, __fma_rn(vF, G[j].y, __dmul_rn(wF, G[j].z))), rb);
                double b = __dmul_rn(a, denf);
                ub = __fma_rn(b, G[j].x, ub); vb = __fma_rn(b, G[j].y, vb); wb = __fma_rn(b, G[j].z, wb);
            }
        }
    }
    if (doG) phibar[c] = pb;
    if (doM) { stbar[c] = rb; stbar[ldc + c] = ub; stbar[2 * ldc + c] = vb; stbar[3 * ldc + c] = wb; }
}

template <bool LDCG, int CH = CUPCFD_ADJ_CHUNK, int PIPE = 0, int WF = 0>
__device__ __forceinline__ void adj_cell_f32(int c, const SellView &sv, const float4 *__restrict__ fg, const float *g,
                                             float hscale, const float4 *__restrict__ st,
                                             const float *__restrict__ gface, float *__restrict__ phibar,
                                             float *__restrict__ phibBar, float4 *__restrict__ stbar, int64_t ldc) {
    int w;
    const int2 *e = cell_entries(sv, c, w);
    if (WF) w = WF;  // every cell has exactly WF entries (a full, uniform slice width)
    bool doG = hscale != 0.f, doM = gface != nullptr;
    float hx = 0, hy = 0, hz = 0;
    if (doG) { hx = hscale * ldg_g<LDCG>(g + c); hy = hscale * ldg_g<LDCG>(g + ldc + c); hz = hscale * ldg_g<LDCG>(g + 2 * ldc + c); }
    float4 sc = make_float4(0, 0, 0, 0);
    if (doM) sc = st[c];
    Acc2 pb, rb, wb;
    Acc2x2 uvb;  // (ubar, vbar) packed
    int2 en[CH];
    load_entries(e, 0, w, en);
    for (int k0 = 0; k0 < w; k0 += CH) {
        float4 G[CH], so[CH];
        float go[CH][3], gf[CH];
#pragma unroll
        for (int j = 0; j < CH; j++) {
            int code = en[j].x;
            if (!WF && code < 0) continue;
            int f = code >> 1, o = en[j].y;
            G[j] = __ldg(fg + f);
            if (o < 0) continue;
            if (doG) { go[j][0] = ldg_g<LDCG>(g + o); go[j][1] = ldg_g<LDCG>(g + ldc + o); go[j][2] = ldg_g<LDCG>(g + 2 * ldc + o); }
            if (doM) { so[j] = __ldg(st + o); gf[j] = __ldg(gface + f); }
        }
        int2 nx[CH];
        if (PIPE) load_entries(e, k0 + CH, w, nx);
#pragma unroll
        for (int j = 0; j < CH; j++) {
            int code = en[j].x;
            if (!WF && code < 0) continue;
            int o = en[j].y;
            if (o < 0) {
                if (doG) phibBar[-1 - o] = fmaf(hx, G[j].x, fmaf(hy, G[j].y, hz * G[j].z));
                continue;
            }
            const FaceW fw = face_weights(G[j].w, code & 1);
            if (doG) {
                float sx = fmaf(hscale, go[j][0], hx), sy = fmaf(hscale, go[j][1], hy), sz = fmaf(hscale, go[j][2], hz);
                pb.add_prod(fw.wc, fmaf(sx, G[j].x, fmaf(sy, G[j].y, sz * G[j].z)));
            }
            if (doM) {
                const float4 sf = interp4(fw, sc, so[j]);
                const float a = fw.wc * gf[j];
                rb.add_prod(a, udots(sf, G[j]));
                const float b = a * sf.x;
                uvb.add_prod(make_float2(b, b), make_float2(G[j].x, G[j].y));
                wb.add_prod(b, G[j].z);
            }
        }
        next_entries<PIPE>(e, k0 + CH, w, en, nx);
    }
    if (doG) phibar[c] = pb.value_f();
    if (doM) stbar[c] = make_float4(rb.value_f(), uvb.xf(), uvb.yf(), wb.value_f());
}

__global__ void __launch_bounds__(256, CUPCFD_MINB_ADJ_F64) k_adj_f64(int nC, SellView sv, const double4 *__restrict__ fg,
                                                 const double *__restrict__ g, double hscale, const double *__restrict__ st,
                                                 const double *__restrict__ gface, double *__restrict__ phibar,
                                                 double *__restrict__ phibBar, double *__restrict__ stbar, int64_t ldc) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nC) adj_cell_f64<false>(c, sv, fg, g, hscale, st, gface, phibar, phibBar, stbar, ldc);
}

__global__ void __launch_bounds__(256, CUPCFD_MINB_F32) k_adj_f32(int nC, SellView sv, const float4 *__restrict__ fg,
                                                 const float *__restrict__ g, float hscale, const float4 *__restrict__ st,
                                                 const float *__restrict__ gface, float *__restrict__ phibar,
                                                 float *__restrict__ phibBar, float4 *__restrict__ stbar, int64_t ldc) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nC) adj_cell_f32<false>(c, sv, fg, g, hscale, st, gface, phibar, phibBar, stbar, ldc);
}

// General gradient adjoint (input gbar = dL/dg, any loss): h_c = gbar_c / V_c.
template <bool SIGNED, class T>
__global__ void __launch_bounds__(256) k_grad_adj_general(int nC, SellView sv, const double4 *__restrict__ fg64,
                                                          const float4 *__restrict__ fg32, const double *__restrict__ vol,
                                                          const T *__restrict__ gbar, T *__restrict__ phibar,
                                                          T *__restrict__ phibBar, int64_t ldc) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    int w;
    const int2 *e = cell_entries(sv, c, w);
    double iv = 1.0 / vol[c];
    double hx = (double) gbar[c] * iv, hy = (double) gbar[ldc + c] * iv, hz = (double) gbar[2 * ldc + c] * iv;
    double pb = 0.0;
    for (int k = 0; k < w; k++) {
        int2 en = __ldg(e + 32 * k);
        if (en.x < 0) break;
        int f = en.x >> 1, o = en.y;
        bool isN = en.x & 1;
        double Sx, Sy, Sz, lam;
        if (fg64) { double4 G = ldg4(fg64 + f); Sx = G.x; Sy = G.y; Sz = G.z; lam = G.w; }
        else { float4 G = __ldg(fg32 + f); Sx = G.x; Sy = G.y; Sz = G.z; lam = G.w; }
        double own = hx * Sx + hy * Sy + hz * Sz;
        if (o < 0) {
            phibBar[-1 - o] = (T) own;
            continue;
        }
        double ivo = 1.0 / __ldg(vol + o);
        double oth = ((double) gbar[o] * Sx + (double) gbar[ldc + o] * Sy + (double) gbar[2 * ldc + o] * Sz) * ivo;
        // d g_P / d phi_f = +S/V_P; d g_N / d phi_f = +S/V_N (reference) or -S/V_N (signed)
        double sOwn = (SIGNED && isN) ? -1.0 : 1.0, sOth = (SIGNED && !isN) ? -1.0 : 1.0;
        pb += (isN ? lam : 1.0 - lam) * (sOwn * own + sOth * oth);
    }
    phibar[c] = (T) pb;
}

// ---------------------------------------------------------------------------
// FluxMassDolfynFaceLoop, full semantics, FP64, one thread per face
// (MassKernels.ipp:95-306). Cell inputs are component blocks over ldc:
// grads = [dudx(3) dvdx(3) dwdx(3) dpdx(3)] (12 blocks), cs = [den u v w p ar]
// (6 blocks). rface is [2][nF] pairs in internal face order. Boundary
// branches per region type; the inlet su[ip] update is done afterwards by
// k_inlet_su in the reference's face order. cnt[4] counts the branches.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_mass_full_f64(
    int nF, const int2 *__restrict__ fcells, const double4 *__restrict__ fg, const double4 *__restrict__ fc,
    const double4 *__restrict__ fxp, const double4 *__restrict__ fxn, const double4 *__restrict__ cc,
    const double *__restrict__ vol, const double *__restrict__ grads, const double *__restrict__ cs, int64_t ldc,
    const int *__restrict__ bndRegion, const int *__restrict__ regionType, const double *__restrict__ regionUVW,
    const double *__restrict__ regionDen, double small, int flags, double *__restrict__ mflux,
    double *__restrict__ rface, double *__restrict__ denB, const double *__restrict__ bcIn, double *__restrict__ bcOut,
    int nB, int *__restrict__ cnt) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    int2 pn = fcells[f];
    double4 G = fg[f];
    int ip = pn.x;
    if (pn.y >= 0) {
        int in = pn.y;
        double4 xP = cc[ip], xN = cc[in];
        double4 X = fc[f];
        double facn = G.w, facp = ds(1.0, facn);
        const double *du = grads, *dvv = grads + 3 * ldc, *dw = grads + 6 * ldc, *dp = grads + 9 * ldc;
        double duac[3], dvac[3], dwac[3];
        for (int d = 0; d < 3; d++) {
            duac[d] = da(dm(du[d * ldc + in], facn), dm(du[d * ldc + ip], facp));
            dvac[d] = da(dm(dvv[d * ldc + in], facn), dm(dvv[d * ldc + ip], facp));
            dwac[d] = da(dm(dw[d * ldc + in], facn), dm(dw[d * ldc + ip], facp));
        }
        const double *den = cs, *u = cs + ldc, *v = cs + 2 * ldc, *w = cs + 3 * ldc, *p = cs + 4 * ldc, *ar = cs + 5 * ldc;
        double denf = da(dm(den[in], facn), dm(den[ip], facp));
        double xac0 = da(dm(xN.x, facn), dm(xP.x, facp));
        double xac1 = da(dm(xN.y, facn), dm(xP.y, facp));
        double xac2 = da(dm(xN.z, facn), dm(xP.z, facp));
        double de0 = ds(X.x, xac0), de1 = ds(X.y, xac1), de2 = ds(X.z, xac2);
        auto dot3 = [](double a0, double a1, double a2, double b0, double b1, double b2) {
            double d = 0.0;
            d = da(d, dm(a0, b0));
            d = da(d, dm(a1, b1));
            d = da(d, dm(a2, b2));
            return d;
        };
        double uF = da(da(dm(u[in], facn), dm(u[ip], facp)), dot3(duac[0], duac[1], duac[2], de0, de1, de2));
        double vF = da(da(dm(v[in], facn), dm(v[ip], facp)), dot3(dvac[0], dvac[1], dvac[2], de0, de1, de2));
        double wF = da(da(dm(w[in], facn), dm(w[ip], facp)), dot3(dwac[0], dwac[1], dwac[2], de0, de1, de2));
        double m = dm(denf, da(da(dm(uF, G.x), dm(vF, G.y)), dm(wF, G.z)));
        // xnorm = S / |S| (EuclideanVector::normalise, EuclideanVector.cpp:100-109)
        double n0 = G.x, n1 = G.y, n2 = G.z;
        double L = __dsqrt_rn(dot3(n0, n1, n2, n0, n1, n2));
        if (L != 0.0) {
            double sc = dvd(1.0, L);
            n0 = dm(n0, sc); n1 = dm(n1, sc); n2 = dm(n2, sc);
        }
        double xa0 = 0, xa1 = 0, xa2 = 0, xb0 = 0, xb1 = 0, xb2 = 0;
        if (fxp) {
            double4 a = fxp[f], b = fxn[f];
            xa0 = a.x; xa1 = a.y; xa2 = a.z; xb0 = b.x; xb1 = b.y; xb2 = b.z;
        }
        double dpP0 = dp[ip], dpP1 = dp[ldc + ip], dpP2 = dp[2 * ldc + ip];
        double pip = da(p[ip], dot3(dpP0, dpP1, dpP2, ds(xa0, xP.x), ds(xa1, xP.y), ds(xa2, xP.z)));
        double pin = da(p[in], dot3(dpP0, dpP1, dpP2, ds(xa0, xN.x), ds(xa1, xN.y), ds(xa2, xN.z)));  // dpdx[ip] (MassKernels.ipp:169)
        double xpn0 = ds(xb0, xa0), xpn1 = ds(xb1, xa1), xpn2 = ds(xb2, xa2);
        double apv1 = dm(den[ip], ar[ip]);
        double apv2 = dm(den[in], ar[in]);
        double apv = da(dm(apv2, facn), dm(apv1, facp));
        double factv = da(dm(vol[in], facn), dm(vol[ip], facp));
        apv = dm(apv, dvd(dm(X.w, factv), dot3(ds(xN.x, xP.x), ds(xN.y, xP.y), ds(xN.z, xP.z), n0, n1, n2)));
        double dpx = dm(da(dm(dp[in], facn), dm(dpP0, facp)), xpn0);
        double dpy = dm(da(dm(dp[ldc + in], facn), dm(dpP1, facp)), xpn1);
        double dpz = dm(da(dm(dp[2 * ldc + in], facn), dm(dpP2, facp)), xpn2);
        rface[2 * (int64_t) f] = -apv;
        rface[2 * (int64_t) f + 1] = -apv;
        mflux[f] = ds(m, dm(apv, ds(ds(ds(ds(pin, pip), dpx), dpy), dpz)));
        return;
    }
    int ib = -1 - pn.y;
    int ir = bndRegion[ib];
    int it = regionType[ir];
    if (it == CUPCFD_RTYPE_INLET) {
        atomicAdd(&cnt[0], 1);
        double d = 0.0;
        d = da(d, dm(regionUVW[3 * ir], G.x));
        d = da(d, dm(regionUVW[3 * ir + 1], G.y));
        d = da(d, dm(regionUVW[3 * ir + 2], G.z));
        mflux[f] = dm(regionDen[ir], d);
    } else if (it == CUPCFD_RTYPE_OUTLET) {
        atomicAdd(&cnt[1], 1);
        const double *den = cs, *u = cs + ldc, *v = cs + 2 * ldc, *w = cs + 3 * ldc;
        double denf = den[ip];
        denB[ib] = denf;
        double m = dm(denf, da(da(dm(u[ip], G.x), dm(v[ip], G.y)), dm(w[ip], G.z)));
        if (m < 0.0) {
            m = small;
            // bcIn = [te ed vis t] cell blocks, bcOut = [te ed vis t] boundary blocks
            for (int q = 0; q < 4; q++)
                if (flags & (1 << q)) bcOut[(int64_t) q * nB + ib] = bcIn[q * ldc + ip];
        }
        mflux[f] = m;
    } else if (it == CUPCFD_RTYPE_SYMP) {
        atomicAdd(&cnt[2], 1);
        mflux[f] = 0.0;
    } else if (it == CUPCFD_RTYPE_WALL) {
        atomicAdd(&cnt[3], 1);
        mflux[f] = 0.0;
    }
}

// ---------------------------------------------------------------------------
// FluxMassDolfynFaceLoop of the reference's T = float instantiation
// (MassKernels.ipp:95-306 with T = float; BenchmarkKernels.cpp:1134-1138
// instantiates it for CupCfdSoAMesh<int,float,int>), one thread per face:
// every product, sum and quotient rounds in float in the reference's operand
// order; facp = 1.0 - facn is evaluated in double and rounded to float (the
// literal is double); EuclideanVector::dotProduct accumulates from 0 in
// float; normalise takes the float square root of the float dot product
// (length() widens sqrtf's result to double, which the float scalar takes
// back exactly) and multiplies by 1.0f / length (EuclideanVector.cpp:83-109).
// The comparison massFlux < 0.0 widens to double, which changes nothing.
// Geometry is the mesh's FP32 copy (exact for a mesh uploaded from float
// arrays); volumes, xpac / xnac and region values are held in double and
// hold the float values exactly. Layouts as k_mass_full_f64.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdot0(float a0, float a1, float a2, float b0, float b1, float b2) {
    float d = 0.f;
    d = fa(d, fm(a0, b0));
    d = fa(d, fm(a1, b1));
    d = fa(d, fm(a2, b2));
    return d;
}

__global__ void __launch_bounds__(256) k_mass_full_f32ref(
    int nF, const int2 *__restrict__ fcells, const float4 *__restrict__ fg, const float4 *__restrict__ fc,
    const double4 *__restrict__ fxp, const double4 *__restrict__ fxn, const float4 *__restrict__ cc,
    const double *__restrict__ vol, const float *__restrict__ grads, const float *__restrict__ cs, int64_t ldc,
    const int *__restrict__ bndRegion, const int *__restrict__ regionType, const double *__restrict__ regionUVW,
    const double *__restrict__ regionDen, float small, int flags, float *__restrict__ mflux,
    float *__restrict__ rface, float *__restrict__ denB, const float *__restrict__ bcIn, float *__restrict__ bcOut,
    int nB, int *__restrict__ cnt) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    int2 pn = fcells[f];
    float4 G = fg[f];
    int ip = pn.x;
    if (pn.y >= 0) {
        int in = pn.y;
        float4 xP = cc[ip], xN = cc[in];
        float4 X = fc[f];
        float facn = G.w, facp = (float) (1.0 - (double) facn);
        const float *du = grads, *dvv = grads + 3 * ldc, *dw = grads + 6 * ldc, *dp = grads + 9 * ldc;
        float duac[3], dvac[3], dwac[3];
        for (int d = 0; d < 3; d++) {
            duac[d] = fa(fm(du[d * ldc + in], facn), fm(du[d * ldc + ip], facp));
            dvac[d] = fa(fm(dvv[d * ldc + in], facn), fm(dvv[d * ldc + ip], facp));
            dwac[d] = fa(fm(dw[d * ldc + in], facn), fm(dw[d * ldc + ip], facp));
        }
        const float *den = cs, *u = cs + ldc, *v = cs + 2 * ldc, *w = cs + 3 * ldc, *p = cs + 4 * ldc, *ar = cs + 5 * ldc;
        float denf = fa(fm(den[in], facn), fm(den[ip], facp));
        float xac0 = fa(fm(xN.x, facn), fm(xP.x, facp));
        float xac1 = fa(fm(xN.y, facn), fm(xP.y, facp));
        float xac2 = fa(fm(xN.z, facn), fm(xP.z, facp));
        float de0 = fs(X.x, xac0), de1 = fs(X.y, xac1), de2 = fs(X.z, xac2);
        float uF = fa(fa(fm(u[in], facn), fm(u[ip], facp)), fdot0(duac[0], duac[1], duac[2], de0, de1, de2));
        float vF = fa(fa(fm(v[in], facn), fm(v[ip], facp)), fdot0(dvac[0], dvac[1], dvac[2], de0, de1, de2));
        float wF = fa(fa(fm(w[in], facn), fm(w[ip], facp)), fdot0(dwac[0], dwac[1], dwac[2], de0, de1, de2));
        float m = fm(denf, fa(fa(fm(uF, G.x), fm(vF, G.y)), fm(wF, G.z)));
        float n0 = G.x, n1 = G.y, n2 = G.z;
        float L = __fsqrt_rn(fdot0(n0, n1, n2, n0, n1, n2));
        if (L != 0.f) {
            float sc = __fdiv_rn(1.f, L);
            n0 = fm(n0, sc); n1 = fm(n1, sc); n2 = fm(n2, sc);
        }
        float xa0 = 0, xa1 = 0, xa2 = 0, xb0 = 0, xb1 = 0, xb2 = 0;
        if (fxp) {
            double4 a = fxp[f], b = fxn[f];
            xa0 = (float) a.x; xa1 = (float) a.y; xa2 = (float) a.z;
            xb0 = (float) b.x; xb1 = (float) b.y; xb2 = (float) b.z;
        }
        float dpP0 = dp[ip], dpP1 = dp[ldc + ip], dpP2 = dp[2 * ldc + ip];
        float pip = fa(p[ip], fdot0(dpP0, dpP1, dpP2, fs(xa0, xP.x), fs(xa1, xP.y), fs(xa2, xP.z)));
        float pin = fa(p[in], fdot0(dpP0, dpP1, dpP2, fs(xa0, xN.x), fs(xa1, xN.y), fs(xa2, xN.z)));  // dpdx[ip] (MassKernels.ipp:169)
        float xpn0 = fs(xb0, xa0), xpn1 = fs(xb1, xa1), xpn2 = fs(xb2, xa2);
        float apv1 = fm(den[ip], ar[ip]);
        float apv2 = fm(den[in], ar[in]);
        float apv = fa(fm(apv2, facn), fm(apv1, facp));
        float factv = fa(fm((float) vol[in], facn), fm((float) vol[ip], facp));
        apv = fm(apv, __fdiv_rn(fm(X.w, factv), fdot0(fs(xN.x, xP.x), fs(xN.y, xP.y), fs(xN.z, xP.z), n0, n1, n2)));
        float dpx = fm(fa(fm(dp[in], facn), fm(dpP0, facp)), xpn0);
        float dpy = fm(fa(fm(dp[ldc + in], facn), fm(dpP1, facp)), xpn1);
        float dpz = fm(fa(fm(dp[2 * ldc + in], facn), fm(dpP2, facp)), xpn2);
        rface[2 * (int64_t) f] = -apv;
        rface[2 * (int64_t) f + 1] = -apv;
        mflux[f] = fs(m, fm(apv, fs(fs(fs(fs(pin, pip), dpx), dpy), dpz)));
        return;
    }
    int ib = -1 - pn.y;
    int ir = bndRegion[ib];
    int it = regionType[ir];
    if (it == CUPCFD_RTYPE_INLET) {
        atomicAdd(&cnt[0], 1);
        float d = fdot0((float) regionUVW[3 * ir], (float) regionUVW[3 * ir + 1], (float) regionUVW[3 * ir + 2], G.x, G.y,
                        G.z);
        mflux[f] = fm((float) regionDen[ir], d);
    } else if (it == CUPCFD_RTYPE_OUTLET) {
        atomicAdd(&cnt[1], 1);
        const float *den = cs, *u = cs + ldc, *v = cs + 2 * ldc, *w = cs + 3 * ldc;
        float denf = den[ip];
        denB[ib] = denf;
        float m = fm(denf, fa(fa(fm(u[ip], G.x), fm(v[ip], G.y)), fm(w[ip], G.z)));
        if (m < 0.f) {
            m = small;
            for (int q = 0; q < 4; q++)
                if (flags & (1 << q)) bcOut[(int64_t) q * nB + ib] = bcIn[q * ldc + ip];
        }
        mflux[f] = m;
    } else if (it == CUPCFD_RTYPE_SYMP) {
        atomicAdd(&cnt[2], 1);
        mflux[f] = 0.f;
    } else if (it == CUPCFD_RTYPE_WALL) {
        atomicAdd(&cnt[3], 1);
        mflux[f] = 0.f;
    }
}

// su[ip] -= massFlux over the cell's inlet faces in ascending reference face
// id (MassKernels.ipp:258), one thread per cell; T double or float (each
// subtraction rounds in T).
template <class T>
__global__ void __launch_bounds__(256) k_inlet_su(int nC, SellView sv, const int *__restrict__ bndRegion,
                                                  const int *__restrict__ regionType, const T *__restrict__ mflux,
                                                  T *__restrict__ su) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    int w;
    const int2 *e = cell_entries(sv, c, w);
    T v = su[c];
    bool touched = false;
    for (int k = 0; k < w; k++) {
        int2 en = e[32 * k];
        if (en.x < 0) break;
        if (en.y >= 0) continue;
        if (regionType[bndRegion[-1 - en.y]] != CUPCFD_RTYPE_INLET) continue;
        v = v - mflux[en.x >> 1];
        touched = true;
    }
    if (touched) su[c] = v;
}

}  // namespace cupcfd_gpu
