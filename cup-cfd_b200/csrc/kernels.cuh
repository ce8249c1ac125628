// Face-loop kernels (device code shared by the ABI translation units).
//
// Data layout (internal numbering, see internal.cuh):
//   faceCells[f] = {P, N} or {P, -1 - boundaryId}
//   fg64/fg32[f] = {Sx, Sy, Sz, lambda}: one 128-bit load per face in FP32
//   cell scalars T[nC]; cell vectors as three component blocks T[3][ldc]
//   SELL-32 incidence lists of int2 {face << 1 | role, other cell}: one
//   thread per cell, 32 consecutive cells per warp, entry k of the warp's
//   cells is one coalesced 256-byte load.
//
// Memory-level parallelism: a thread loads a chunk of incidence entries,
// then every face record and neighbour value of the chunk, and only then
// computes, so each thread keeps several independent gathers in flight
// instead of one dependent chain per face.
//
// Determinism: every cell sums its faces in ascending reference face id, one
// thread per cell, no floating-point atomics anywhere. FP64 kernels use
// explicit round-to-nearest intrinsics in the reference's operand order
// (GradientKernels.ipp:73-131, MassKernels.ipp:95-306), so results equal the
// reference CPU build bit for bit.
#pragma once

#include "arith.cuh"
#include "internal.cuh"
#include "sell.cuh"

namespace cupcfd_gpu {


// ---------------------------------------------------------------------------
// Compensated accumulation of products, after Dot2 (Ogita, Rump & Oishi,
// "Accurate sum and dot product", SIAM J. Sci. Comput. 26(6), 2005): the sum
// s is advanced by p = fl(a b) with Knuth's TwoSum, and the error of the
// product and of the addition are accumulated separately in e. CUPCFD_COMP:
//   3 (default): TwoSum computes nbp = s - t (t = s + p), av = t + nbp and
//     the exact ar = s - av; the product's error a b - p and TwoSum's exact
//     low part p - (t - s) are taken together as one FMA, fma(a, b, nbp)
//     = a b - (t - s), rounded once. That rounding is of the order u^2 |t|,
//     the order of Dot2's own error accumulation, so the result keeps
//     Dot2's bound (as if computed in twice the working precision) in 8
//     operations instead of Dot2's 10 (packed: 8 instead of 11).
//   2: Dot2 as published (TwoProduct by FMA, TwoSum, errors summed).
//   1: TwoSum without the product's error.
//   0: Kahan's compensated sum (Fast2Sum on p + e).
// ---------------------------------------------------------------------------
#ifndef CUPCFD_COMP
#define CUPCFD_COMP 3
#endif
//
// Every form starts from the rounded product p = fl(a b), written as
// fma(a, b, +0): the same value (a b + 0 rounds once; a zero product comes
// out +0, which no sum below tells apart from -0). The packed form needs it:
// with a plain packed multiply feeding a packed add, the add came out as one
// fused fma(a, b, s) on B200 with CUDA 12.9 (measured: the packed lanes then
// equal, bit for bit, an emulation of that fusion, and differ from the scalar
// form on 62% of random six-term sums), even when both were written as
// mul.rn.f32x2 / add.rn.f32x2 in inline PTX. That takes the product's
// rounding out of TwoSum's input and loses the error term where the sum
// cancels (checked in exact arithmetic: up to one ulp of the terms). The
// result of an FMA is not contracted again, and the scalar form uses the
// same expression so that a packed lane and Acc2 give the same bits.
struct Acc2 {
    float s = 0.f, e = 0.f;
    __device__ __forceinline__ void add_prod(float a, float b) {
        float p = __fmaf_rn(a, b, 0.f);
#if CUPCFD_COMP == 3
        float t = __fadd_rn(s, p);
        float nbp = __fsub_rn(s, t);
        float ar = __fsub_rn(s, __fadd_rn(t, nbp));
        float brp = __fmaf_rn(a, b, nbp);
        s = t;
        e = __fadd_rn(e, __fadd_rn(ar, brp));
#elif CUPCFD_COMP == 2
        float ep = __fmaf_rn(a, b, -p);
        float t = __fadd_rn(s, p);
        float bp = __fsub_rn(t, s);
        float es = __fadd_rn(__fsub_rn(s, __fsub_rn(t, bp)), __fsub_rn(p, bp));
        s = t;
        e = __fadd_rn(e, __fadd_rn(ep, es));
#elif CUPCFD_COMP == 1
        float t = __fadd_rn(s, p);
        float bp = __fsub_rn(t, s);
        float es = __fadd_rn(__fsub_rn(s, __fsub_rn(t, bp)), __fsub_rn(p, bp));
        s = t;
        e = __fadd_rn(e, es);
#else
        float y = __fadd_rn(p, e);
        float t = __fadd_rn(s, y);
        e = __fadd_rn(__fsub_rn(s, t), y);
        s = t;
#endif
    }
    __device__ __forceinline__ void sub_prod(float a, float b) { add_prod(-a, b); }
    __device__ __forceinline__ double value() const { return (double) s + (double) e; }
    // (float) value(), in one FP32 add and with the same bits: the double sum
    // of two floats is exact unless their exponents differ by more than 29,
    // and then |e| < 2^-29 |s| and both forms give s
    __device__ __forceinline__ float value_f() const { return __fadd_rn(s, e); }
};

// Two Acc2 sums advanced together by the sm_100 packed FP32x2 operations
// (__fmul2_rn, __ffma2_rn, __fadd2_rn): half the issued instructions. Each
// lane performs exactly Acc2::add_prod's IEEE operations, x - y being
// written fma(y, -1, x), which rounds the same exact value x + (-y), so the
// lanes are bit-identical to two Acc2. add_x advances lane x alone.
struct Acc2x2 {
    float2 s = {0.f, 0.f}, e = {0.f, 0.f};
    __device__ __forceinline__ void add_prod(float2 a, float2 b) {
        const float2 m1 = make_float2(-1.f, -1.f);
        float2 p = __ffma2_rn(a, b, make_float2(0.f, 0.f));
#if CUPCFD_COMP == 3
        float2 t = __fadd2_rn(s, p);
        float2 nbp = __ffma2_rn(t, m1, s);
        float2 ar = __ffma2_rn(__fadd2_rn(t, nbp), m1, s);
        float2 brp = __ffma2_rn(a, b, nbp);
        s = t;
        e = __fadd2_rn(e, __fadd2_rn(ar, brp));
#elif CUPCFD_COMP == 2
        float2 ep = __ffma2_rn(a, b, __fmul2_rn(p, m1));
        float2 t = __fadd2_rn(s, p);
        float2 bp = __ffma2_rn(s, m1, t);
        float2 es = __fadd2_rn(__ffma2_rn(__ffma2_rn(bp, m1, t), m1, s), __ffma2_rn(bp, m1, p));
        s = t;
        e = __fadd2_rn(e, __fadd2_rn(ep, es));
#elif CUPCFD_COMP == 1
        float2 t = __fadd2_rn(s, p);
        float2 bp = __ffma2_rn(s, m1, t);
        float2 es = __fadd2_rn(__ffma2_rn(__ffma2_rn(bp, m1, t), m1, s), __ffma2_rn(bp, m1, p));
        s = t;
        e = __fadd2_rn(e, es);
#else
        float2 y = __fadd2_rn(p, e);
        float2 t = __fadd2_rn(s, y);
        e = __fadd2_rn(__ffma2_rn(t, m1, s), y);
        s = t;
#endif
    }
    __device__ __forceinline__ void add_x(float a, float b) {
        Acc2 h;
        h.s = s.x; h.e = e.x;
        h.add_prod(a, b);
        s.x = h.s; e.x = h.e;
    }
    __device__ __forceinline__ double x() const { return (double) s.x + (double) e.x; }
    __device__ __forceinline__ double y() const { return (double) s.y + (double) e.y; }
    // (float) x(), (float) y() in FP32, the same bits (Acc2::value_f)
    __device__ __forceinline__ float xf() const { return __fadd_rn(s.x, e.x); }
    __device__ __forceinline__ float yf() const { return __fadd_rn(s.y, e.y); }
};

// ---------------------------------------------------------------------------
// FP32 face interpolation seen from one of the face's two cells: x_f =
// wc x_c + wo x_o (wc the weight of this cell's value, wo of the other's),
// rounded as fmaf(wc, x_c, wo * x_o). For the face's owner (cell1, P)
// wc = 1 - lambda and wo = lambda (MassKernels.ipp:140-153: lambda weights
// the neighbour). The owner's mass flux and both cells' adjoint terms use
// these same values, so the owner computes rho_f and u_f . S_f once for both.
// ---------------------------------------------------------------------------
struct FaceW {
    float wc, wo;
};
__device__ __forceinline__ FaceW face_weights(float lam, bool isN) {
    const float facp = 1.f - lam;
    return FaceW{isN ? lam : facp, isN ? facp : lam};
}
__device__ __forceinline__ float interp(const FaceW &w, float xc, float xo) { return fmaf(w.wc, xc, w.wo * xo); }
// {rho, u, v, w} in two packed FP32x2 operations; every lane rounds as interp()
__device__ __forceinline__ float4 interp4(const FaceW &w, float4 sc, float4 so) {
    const float2 wc2 = make_float2(w.wc, w.wc), wo2 = make_float2(w.wo, w.wo);
    const float2 a = __ffma2_rn(wc2, make_float2(sc.x, sc.y), __fmul2_rn(wo2, make_float2(so.x, so.y)));
    const float2 b = __ffma2_rn(wc2, make_float2(sc.z, sc.w), __fmul2_rn(wo2, make_float2(so.z, so.w)));
    return make_float4(a.x, a.y, b.x, b.y);
}
// u_f . S_f of an interpolated state {rho, u, v, w} and a face record {S, lambda}
__device__ __forceinline__ float udots(float4 s, float4 G) { return fmaf(s.y, G.x, fmaf(s.z, G.y, s.w * G.z)); }

// 32-byte read-only load as two 128-bit loads (no __ldg overload for double4)
__device__ __forceinline__ double4 ldg4(const double4 *p) {
    double2 a = __ldg(reinterpret_cast<const double2 *>(p));
    double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 ldg4(const float4 *p) { return __ldg(p); }


// Entries per chunk in the unrolled kernels (six covers a hex cell in one
// chunk; wider cells take more chunks) and the minimum resident blocks per
// SM the register allocation must allow, per kernel family. Chosen by
// measurement on B200; overridable at build time. The per-cell routines of
// the forward and adjoint also take WF: 0 for any mesh, or the number of
// incidences every cell has (6 for hexahedral meshes), which fixes the
// chunk loop's trip count at compile time and drops the padding tests
// (kernels_pf.cuh).
#ifndef CUPCFD_GRAD_CHUNK
#define CUPCFD_GRAD_CHUNK 6
#endif
#ifndef CUPCFD_FWD_CHUNK
#define CUPCFD_FWD_CHUNK 3
#endif
#ifndef CUPCFD_ADJ_CHUNK
#define CUPCFD_ADJ_CHUNK 2
#endif
#ifndef CUPCFD_MINB_F32
#define CUPCFD_MINB_F32 4
#endif
#ifndef CUPCFD_MINB_F64
#define CUPCFD_MINB_F64 2
#endif
#ifndef CUPCFD_FWD_CHUNK_F64
#define CUPCFD_FWD_CHUNK_F64 2
#endif
#ifndef CUPCFD_MINB_FWD_F64
#define CUPCFD_MINB_FWD_F64 3
#endif
#ifndef CUPCFD_ADJ_CHUNK_F64
#define CUPCFD_ADJ_CHUNK_F64 1
#endif
#ifndef CUPCFD_MINB_ADJ_F64
#define CUPCFD_MINB_ADJ_F64 4
#endif
#ifndef CUPCFD_MINB_FUSED_F32
#define CUPCFD_MINB_FUSED_F32 4
#endif
#ifndef CUPCFD_MINB_FUSED_F64
#define CUPCFD_MINB_FUSED_F64 2
#endif
constexpr int CHUNK = CUPCFD_GRAD_CHUNK;

// ---------------------------------------------------------------------------
// Gradient, FP64, reference arithmetic. CORR adds the non-orthogonal
// correction of the previous iterate (needed from the second iteration on;
// with a zero previous iterate the term is exactly +0 and is skipped).
// ---------------------------------------------------------------------------
template <bool CORR, bool SIGNED>
__global__ void __launch_bounds__(256, CUPCFD_MINB_F64) k_grad_f64(int nC, SellView sv, const double4 *__restrict__ fg,
                                                  const double4 *__restrict__ fc, const double4 *__restrict__ cc,
                                                  const double *__restrict__ phi, const double *__restrict__ phiB,
                                                  const double *__restrict__ vol, const double *__restrict__ go,
                                                  double *__restrict__ g, double *__restrict__ gcopy, int64_t ldc) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    int w;
    const int2 *e = cell_entries(sv, c, w);
    double phic = phi[c];
    double4 xc = make_double4(0, 0, 0, 0);
    double gc0 = 0, gc1 = 0, gc2 = 0;
    if (CORR) {
        xc = cc[c];
        gc0 = go[c]; gc1 = go[ldc + c]; gc2 = go[2 * ldc + c];
    }
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int k0 = 0; k0 < w; k0 += CHUNK) {
        int2 en[CHUNK];
        load_entries(e, k0, w, en);
        double4 G[CHUNK];
        double pv[CHUNK];
#pragma unroll
        for (int j = 0; j < CHUNK; j++) {
            if (en[j].x < 0) continue;
            G[j] = ldg4(fg + (en[j].x >> 1));
            int o = en[j].y;
            pv[j] = o >= 0 ? __ldg(phi + o) : __ldg(phiB + (-1 - o));
        }
#pragma unroll
        for (int j = 0; j < CHUNK; j++) {
            int code = en[j].x;
            if (code < 0) continue;
            bool isN = code & 1;
            int o = en[j].y;
            double phif;
            if (o < 0) {
                phif = pv[j];
            } else {
                double facn = G[j].w;
                double facp = ds(1.0, facn);
                double phN = isN ? phic : pv[j], phP = isN ? pv[j] : phic;
                phif = da(dm(phN, facn), dm(phP, facp));
                if (CORR) {
                    double4 xo = ldg4(cc + o);
                    double4 xf = ldg4(fc + (code >> 1));
                    double go0 = __ldg(go + o), go1 = __ldg(go + ldc + o), go2 = __ldg(go + 2 * ldc + o);
                    double4 xN = isN ? xc : xo, xP = isN ? xo : xc;
                    double gN0 = isN ? gc0 : go0, gN1 = isN ? gc1 : go1, gN2 = isN ? gc2 : go2;
                    double gP0 = isN ? go0 : gc0, gP1 = isN ? go1 : gc1, gP2 = isN ? go2 : gc2;
                    double xac0 = da(dm(xN.x, facn), dm(xP.x, facp));
                    double xac1 = da(dm(xN.y, facn), dm(xP.y, facp));
                    double xac2 = da(dm(xN.z, facn), dm(xP.z, facp));
                    double ga0 = da(dm(gN0, facn), dm(gP0, facp));
                    double ga1 = da(dm(gN1, facn), dm(gP1, facp));
                    double ga2 = da(dm(gN2, facn), dm(gP2, facp));
                    double d = 0.0;
                    d = da(d, dm(ga0, ds(xf.x, xac0)));
                    d = da(d, dm(ga1, ds(xf.y, xac1)));
                    d = da(d, dm(ga2, ds(xf.z, xac2)));
                    phif = da(phif, d);
                }
            }
            if (SIGNED && isN) {
                ax = ds(ax, dm(phif, G[j].x)); ay = ds(ay, dm(phif, G[j].y)); az = ds(az, dm(phif, G[j].z));
            } else {
                ax = da(ax, dm(phif, G[j].x)); ay = da(ay, dm(phif, G[j].y)); az = da(az, dm(phif, G[j].z));
            }
        }
    }
    double fact = dvd(1.0, vol[c]);
    ax = dm(ax, fact); ay = dm(ay, fact); az = dm(az, fact);
    g[c] = ax; g[ldc + c] = ay; g[2 * ldc + c] = az;
    if (gcopy) { gcopy[c] = ax; gcopy[ldc + c] = ay; gcopy[2 * ldc + c] = az; }
}

// ---------------------------------------------------------------------------
// Gradient, FP32 storage and arithmetic, compensated accumulation (Acc2), FP64 1/V.
// ---------------------------------------------------------------------------
template <bool CORR, bool SIGNED>
__global__ void __launch_bounds__(256, CUPCFD_MINB_F32) k_grad_f32(int nC, SellView sv, const float4 *__restrict__ fg,
                                                  const float4 *__restrict__ fc, const float4 *__restrict__ cc,
                                                  const float *__restrict__ phi, const float *__restrict__ phiB,
                                                  const double *__restrict__ vol, const float *__restrict__ go,
                                                  float *__restrict__ g, float *__restrict__ gcopy, int64_t ldc) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    int w;
    const int2 *e = cell_entries(sv, c, w);
    float phic = phi[c];
    float4 xc = make_float4(0, 0, 0, 0);
    float gc0 = 0, gc1 = 0, gc2 = 0;
    if (CORR) {
        xc = cc[c];
        gc0 = go[c]; gc1 = go[ldc + c]; gc2 = go[2 * ldc + c];
    }
    Acc2 ax, ay, az;
    for (int k0 = 0; k0 < w; k0 += CHUNK) {
        int2 en[CHUNK];
        load_entries(e, k0, w, en);
        float4 G[CHUNK];
        float pv[CHUNK];
#pragma unroll
        for (int j = 0; j < CHUNK; j++) {
            if (en[j].x < 0) continue;
            G[j] = __ldg(fg + (en[j].x >> 1));
            int o = en[j].y;
            pv[j] = o >= 0 ? __ldg(phi + o) : __ldg(phiB + (-1 - o));
        }
#pragma unroll
        for (int j = 0; j < CHUNK; j++) {
            int code = en[j].x;
            if (code < 0) continue;
            bool isN = code & 1;
            int o = en[j].y;
            float phif;
            if (o < 0) {
                phif = pv[j];
            } else {
                float facn = G[j].w, facp = 1.f - facn;
                phif = interp(face_weights(facn, isN), phic, pv[j]);
                if (CORR) {
                    float4 xo = __ldg(cc + o), xf = __ldg(fc + (code >> 1));
                    float go0 = __ldg(go + o), go1 = __ldg(go + ldc + o), go2 = __ldg(go + 2 * ldc + o);
                    float4 xN = isN ? xc : xo, xP = isN ? xo : xc;
                    float gN0 = isN ? gc0 : go0, gN1 = isN ? gc1 : go1, gN2 = isN ? gc2 : go2;
                    float gP0 = isN ? go0 : gc0, gP1 = isN ? go1 : gc1, gP2 = isN ? go2 : gc2;
                    float d0 = xf.x - fmaf(facn, xN.x, facp * xP.x);
                    float d1 = xf.y - fmaf(facn, xN.y, facp * xP.y);
                    float d2 = xf.z - fmaf(facn, xN.z, facp * xP.z);
                    phif += fmaf(facn, gN0, facp * gP0) * d0 + fmaf(facn, gN1, facp * gP1) * d1 +
                            fmaf(facn, gN2, facp * gP2) * d2;
                }
            }
            if (SIGNED && isN) {
                ax.sub_prod(phif, G[j].x); ay.sub_prod(phif, G[j].y); az.sub_prod(phif, G[j].z);
            } else {
                ax.add_prod(phif, G[j].x); ay.add_prod(phif, G[j].y); az.add_prod(phif, G[j].z);
            }
        }
    }
    double fact = 1.0 / vol[c];
    float rx = (float) (ax.value() * fact), ry = (float) (ay.value() * fact), rz = (float) (az.value() * fact);
    g[c] = rx; g[ldc + c] = ry; g[2 * ldc + c] = rz;
    if (gcopy) { gcopy[c] = rx; gcopy[ldc + c] = ry; gcopy[2 * ldc + c] = rz; }
}

// ---------------------------------------------------------------------------
// Gradient with the arithmetic of the reference's T=float instantiation
// (GradientKernels.ipp:38-136 with T = float): every product and sum rounds
// in float, facp = 1.0 - facn and fact = 1.0 / vol are evaluated in double
// and rounded to float (the literals are double), the correction's dot
// product accumulates from 0 in float (EuclideanVector.ipp dotProduct).
// vol holds the float volumes exactly (a mesh uploaded from float arrays).
// ---------------------------------------------------------------------------
template <bool CORR, bool SIGNED>
__global__ void __launch_bounds__(256, CUPCFD_MINB_F32) k_grad_f32ref(int nC, SellView sv, const float4 *__restrict__ fg,
                                                     const float4 *__restrict__ fc, const float4 *__restrict__ cc,
                                                     const float *__restrict__ phi, const float *__restrict__ phiB,
                                                     const double *__restrict__ vol, const float *__restrict__ go,
                                                     float *__restrict__ g, float *__restrict__ gcopy, int64_t ldc) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    int w;
    const int2 *e = cell_entries(sv, c, w);
    const float phic = phi[c];
    float4 xc = make_float4(0, 0, 0, 0);
    float gc0 = 0, gc1 = 0, gc2 = 0;
    if (CORR) {
        xc = cc[c];
        gc0 = go[c]; gc1 = go[ldc + c]; gc2 = go[2 * ldc + c];
    }
    float ax = 0.f, ay = 0.f, az = 0.f;
    for (int k = 0; k < w; k++) {
        const int2 en = ld_entry(e + 32 * k);
        const int code = en.x;
        if (code < 0) break;
        const bool isN = code & 1;
        const int o = en.y;
        const float4 G = __ldg(fg + (code >> 1));
        float phif;
        if (o < 0) {
            phif = __ldg(phiB + (-1 - o));
        } else {
            const float facn = G.w, facp = (float) (1.0 - (double) facn);
            const float pv = __ldg(phi + o);
            const float phN = isN ? phic : pv, phP = isN ? pv : phic;
            phif = __fadd_rn(__fmul_rn(phN, facn), __fmul_rn(phP, facp));
            if (CORR) {
                const float4 xo = __ldg(cc + o), xf = __ldg(fc + (code >> 1));
                const float go0 = __ldg(go + o), go1 = __ldg(go + ldc + o), go2 = __ldg(go + 2 * ldc + o);
                const float4 xN = isN ? xc : xo, xP = isN ? xo : xc;
                const float gN0 = isN ? gc0 : go0, gN1 = isN ? gc1 : go1, gN2 = isN ? gc2 : go2;
                const float gP0 = isN ? go0 : gc0, gP1 = isN ? go1 : gc1, gP2 = isN ? go2 : gc2;
                // xac = xN facn + xP facp; dPhidxac likewise; corr = xf - xac
                const float d0 = __fsub_rn(xf.x, __fadd_rn(__fmul_rn(xN.x, facn), __fmul_rn(xP.x, facp)));
                const float d1 = __fsub_rn(xf.y, __fadd_rn(__fmul_rn(xN.y, facn), __fmul_rn(xP.y, facp)));
                const float d2 = __fsub_rn(xf.z, __fadd_rn(__fmul_rn(xN.z, facn), __fmul_rn(xP.z, facp)));
                const float a0 = __fadd_rn(__fmul_rn(gN0, facn), __fmul_rn(gP0, facp));
                const float a1 = __fadd_rn(__fmul_rn(gN1, facn), __fmul_rn(gP1, facp));
                const float a2 = __fadd_rn(__fmul_rn(gN2, facn), __fmul_rn(gP2, facp));
                float dot = 0.f;
                dot = __fadd_rn(dot, __fmul_rn(a0, d0));
                dot = __fadd_rn(dot, __fmul_rn(a1, d1));
                dot = __fadd_rn(dot, __fmul_rn(a2, d2));
                phif = __fadd_rn(phif, dot);
            }
        }
        if (SIGNED && isN) {
            ax = __fsub_rn(ax, __fmul_rn(phif, G.x)); ay = __fsub_rn(ay, __fmul_rn(phif, G.y));
            az = __fsub_rn(az, __fmul_rn(phif, G.z));
        } else {
            ax = __fadd_rn(ax, __fmul_rn(phif, G.x)); ay = __fadd_rn(ay, __fmul_rn(phif, G.y));
            az = __fadd_rn(az, __fmul_rn(phif, G.z));
        }
    }
    const float fact = (float) (1.0 / vol[c]);
    const float rx = __fmul_rn(ax, fact), ry = __fmul_rn(ay, fact), rz = __fmul_rn(az, fact);
    g[c] = rx; g[ldc + c] = ry; g[2 * ldc + c] = rz;
    if (gcopy) { gcopy[c] = rx; gcopy[ldc + c] = ry; gcopy[2 * ldc + c] = rz; }
}

// ---------------------------------------------------------------------------
// Plain mass flux m_f = rho_f (u_f . S_f), one thread per face.
// F64: state as four component blocks [4][ldc] (rho, u, v, w).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_mass_plain_f64(int nF, const int2 *__restrict__ fcells,
                                                        const double4 *__restrict__ fg, const double *__restrict__ st,
                                                        int64_t ldc, double *__restrict__ mflux) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    int2 pn = fcells[f];
    if (pn.y < 0) return;
    double4 G = ldg4(fg + f);
    double facn = G.w, facp = ds(1.0, facn);
    int P = pn.x, N = pn.y;
    double denf = da(dm(__ldg(st + N), facn), dm(__ldg(st + P), facp));
    double uF = da(dm(__ldg(st + ldc + N), facn), dm(__ldg(st + ldc + P), facp));
    double vF = da(dm(__ldg(st + 2 * ldc + N), facn), dm(__ldg(st + 2 * ldc + P), facp));
    double wF = da(dm(__ldg(st + 3 * ldc + N), facn), dm(__ldg(st + 3 * ldc + P), facp));
    mflux[f] = dm(denf, da(da(dm(uF, G.x), dm(vF, G.y)), dm(wF, G.z)));
}

// F32: state as float4 {rho, u, v, w} per cell.
__global__ void __launch_bounds__(256) k_mass_plain_f32(int nF, const int2 *__restrict__ fcells,
                                                        const float4 *__restrict__ fg, const float4 *__restrict__ st,
                                                        float *__restrict__ mflux) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    int2 pn = fcells[f];
    if (pn.y < 0) return;
    float4 G = fg[f];
    float4 sP = __ldg(st + pn.x), sN = __ldg(st + pn.y);
    float4 sf = interp4(face_weights(G.w, false), sP, sN);  // seen from the owner
    mflux[f] = sf.x * udots(sf, G);
}

}  // namespace cupcfd_gpu
