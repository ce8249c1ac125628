// Momentum face loop of the reference, FP64 with its arithmetic
// (FluxUVWDolfynFaceLoop1, FluxUVWDolfynRegionLoop1, FluxUVWDolfynBndsLoop1;
// UVWKernels.ipp:38-544).
//
// The reference walks faces in label order and scatters each face's terms
// into su/sv/sw (both cells of an interior face) and au/av/aw (the owner of a
// boundary face). Here one thread per cell gathers them instead, over the
// cell's SELL-32 incidence list, which holds the cell's faces in ascending
// reference face id: the order in which the reference's updates reach that
// cell, so every cell's chain of roundings is the reference's. Both cells of
// an interior face evaluate its terms with the same operations (so the same
// bits); the owner alone writes the face's own outputs (rFace, boundary
// values, the outlet mass-flux clamp, wall shear).
//
// Values carried between faces. uFace/vFace/wFace and visFace are declared
// outside the reference's face loop (UVWKernels.ipp:74-75): interior faces
// read the uFace the last inlet or outlet face before them set, symmetry
// faces the visFace the last interior, inlet or outlet face set. A prefix
// maximum over reference face ids (k_carry_*) finds that face for every face
// once per region layout; carry[f] (internal face id) encodes it:
//   interior f: >= 0 the internal cell whose velocities the outlet took,
//               <= -2 the inlet region -2 - carry, -1 none (zero)
//   symmetry f: >= 0 the internal face whose visFace it reads, -1 none (zero)
// The reference reads uninitialised values where there is none; zero here.
#pragma once

#include <cstdint>

#include "arith.cuh"
#include "internal.cuh"
#include "prefetch.cuh"
#include "sell.cuh"

namespace cupcfd_gpu {

// Arithmetic of the two instantiations the reference compiles
// (BenchmarkKernels.cpp:1134-1138), one IEEE rounding per operator:
//   T = double: FP64 throughout.
//   T = float:  float throughout, except where the float build widens:
//     facp = 1.0 - facn (double literal, then rounded to float), 2.0 * visac
//     (double, exact, then float), and the wall's fabs(ut0) + fabs(ut1) +
//     fabs(ut2) (the C library's double fabs in the reference's scope, a
//     double sum rounded once to float). normalise() and the wall's
//     xpn.length() take the float square root of the float dot product
//     (length() widens sqrtf's result to double and the float scalar takes it
//     back exactly; EuclideanVector.cpp:93-109).
template <class T>
struct UvwReal;
template <>
struct UvwReal<double> {
    using V4 = double4;
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double sqrt_(double a) { return __dsqrt_rn(a); }
    static __device__ __forceinline__ double one_minus(double x) { return __dsub_rn(1.0, x); }
    static __device__ __forceinline__ double twice(double x) { return __dmul_rn(2.0, x); }
    static __device__ __forceinline__ double abs_sum3(double a, double b, double c) {
        return __dadd_rn(__dadd_rn(fabs(a), fabs(b)), fabs(c));
    }
};
template <>
struct UvwReal<float> {
    using V4 = float4;
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    static __device__ __forceinline__ float sqrt_(float a) { return __fsqrt_rn(a); }
    static __device__ __forceinline__ float one_minus(float x) { return (float) __dsub_rn(1.0, (double) x); }
    static __device__ __forceinline__ float twice(float x) { return (float) __dmul_rn(2.0, (double) x); }
    static __device__ __forceinline__ float abs_sum3(float a, float b, float c) {
        return (float) __dadd_rn(__dadd_rn(fabs((double) a), fabs((double) b)), fabs((double) c));
    }
};

// std::min / std::max of <algorithm>: min(a,b) = b < a ? b : a,
// max(a,b) = a < b ? b : a (the first argument wins ties and NaN compares).
template <class T>
__device__ __forceinline__ T std_min(T a, T b) { return (b < a) ? b : a; }
template <class T>
__device__ __forceinline__ T std_max(T a, T b) { return (a < b) ? b : a; }

// EuclideanVector::dotProduct (EuclideanVector.cpp:83-90): accumulated from 0.
template <class T>
__device__ __forceinline__ T dot0(T a0, T a1, T a2, T b0, T b1, T b2) {
    using R = UvwReal<T>;
    T d = T(0);
    d = R::add(d, R::mul(a0, b0));
    d = R::add(d, R::mul(a1, b1));
    d = R::add(d, R::mul(a2, b2));
    return d;
}

// EuclideanVector::normalise (EuclideanVector.cpp:100-109)
template <class T>
__device__ __forceinline__ void normalise(T &x, T &y, T &z) {
    using R = UvwReal<T>;
    T L = R::sqrt_(dot0(x, y, z, x, y, z));
    if (L != T(0)) {
        T sc = R::div(T(1), L);
        x = R::mul(x, sc); y = R::mul(y, sc); z = R::mul(z, sc);
    }
}

// Face geometry is the mesh's FP64 copy for T = double and its FP32 copy for
// T = float (exact for a mesh uploaded from float arrays); rlencos, boundary
// distances and region values are held in double (the float values exactly)
// and the boundary shears are written to the mesh's double array.
template <class T>
struct UvwArgs {
    using V4 = typename UvwReal<T>::V4;
    int nC;
    SellView sv;
    const int2 *fcells;
    const V4 *fg, *fc, *cc;                // {S, lambda}, {x_f, area}, {x_c, 0}
    const int *bndRegion, *regionType;
    const double *regionUVW;
    const double *rlencos;                 // [nF] internal, null = zero
    const double *bndDist;                 // [nB], null = zero
    const int *carry;                      // [nF] internal; null when no region is an inlet, outlet or symmetry
    T gammaBlend, small;
    const T *u, *v, *w, *visC;             // [nC] internal
    const T *visB;                         // [nB]
    const T *grads;                        // 9 blocks [ldg]: dudx xyz, dvdx xyz, dwdx xyz
    int64_t ldg;
    T *uB, *vB, *wB;                       // [nB]
    T *massFlux, *rFace;                   // [nF], [2 nF] internal
    double *shear;                         // [3 nB]
    T *su, *sv_, *sw, *au, *av, *aw;       // [nC] internal
};

// The values of the thread's own cell that every incidence reads (centre,
// velocity, viscosity, the nine gradient components): loaded once per cell
// instead of once per incidence. The terms use them exactly where the
// reference uses cell1's or cell2's values, so the arithmetic is unchanged.
template <class T>
struct UvwOwn {
    typename UvwReal<T>::V4 cc;
    T u, v, w, vis, g[9];
};
template <class T>
__device__ __forceinline__ UvwOwn<T> uvw_own(const UvwArgs<T> &a, int c) {
    UvwOwn<T> o;
    o.cc = a.cc[c]; o.u = a.u[c]; o.v = a.v[c]; o.w = a.w[c]; o.vis = a.visC[c];
#pragma unroll
    for (int q = 0; q < 9; q++) o.g[q] = a.grads[q * a.ldg + c];
    return o;
}

// visFace that face g leaves behind (interior, inlet and outlet faces set it,
// UVWKernels.ipp:160, 274, 335).
template <class T>
__device__ __forceinline__ T vis_face_of(const UvwArgs<T> &a, int g) {
    using R = UvwReal<T>;
    int2 pn = a.fcells[g];
    T rl = a.rlencos ? (T) a.rlencos[g] : T(0);
    T visac;
    if (pn.y >= 0) {
        T facn = a.fg[g].w, facp = R::one_minus(facn);
        visac = R::add(R::mul(a.visC[pn.y], facn), R::mul(a.visC[pn.x], facp));
    } else {
        int ib = -1 - pn.y;
        visac = a.regionType[a.bndRegion[ib]] == CUPCFD_RTYPE_INLET ? a.visB[ib] : a.visC[pn.x];
    }
    return R::mul(visac, rl);
}

// How an incidence's terms update its cell (t[0..9] from uvw_terms), in the
// reference's operand order:
enum UvwKind : int {
    UVW_NONE = 0,    // padding, default-region boundary
    UVW_OWNER = 1,   // interior, cell1: s = ((s - blend) + fde) - fdi          (UVWKernels.ipp:216-223)
    UVW_NEIGH = 2,   // interior, cell2: s = ((s + blend) - fde) + fdi
    UVW_INOUT = 3,   // inlet / outlet: a = a - f; s = ((s - f*uF) + fde) - fdi (:309-317, :370-378)
    UVW_WALLSYM = 4  // symmetry / wall: a = a + X; s = (s + X*u) - force       (:424-431, :490-497)
};

// The terms one incidence (entry en of cell c) contributes to its cell, and
// the face's own outputs when c owns the face. Returns the UvwKind.
template <class T>
__device__ __forceinline__ int uvw_terms(const UvwArgs<T> &a, int c, const UvwOwn<T> &own, int2 en, T (&t)[10]) {
    using R = UvwReal<T>;
    using V4 = typename UvwReal<T>::V4;
    const int64_t L = a.ldg;
    auto gr = [&](int q, int cell) { return a.grads[q * L + cell]; };
    const int f = en.x >> 1;
    const bool owner = (en.x & 1) == 0;
    const V4 G = a.fg[f];
    const T rl = a.rlencos ? (T) a.rlencos[f] : T(0);
    if (en.y >= 0) {
        // interior face (UVWKernels.ipp:145-228)
        const int o = en.y;  // the other cell: cell2 (in) for the owner, cell1 (ip) for the neighbour
        const T facn = G.w, facp = R::one_minus(facn);
        // the other cell's and this cell's weights: facn weights cell2 (in),
        // facp cell1 (ip); x_in*facn + x_ip*facp is then x_o*wO + x_c*wC for
        // either role (IEEE addition commutes exactly)
        const T wO = owner ? facn : facp, wC = owner ? facp : facn;
        T du[3], dv[3], dw[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            du[d] = R::add(R::mul(gr(d, o), wO), R::mul(own.g[d], wC));
            dv[d] = R::add(R::mul(gr(3 + d, o), wO), R::mul(own.g[3 + d], wC));
            dw[d] = R::add(R::mul(gr(6 + d, o), wO), R::mul(own.g[6 + d], wC));
        }
        const T visac = R::add(R::mul(a.visC[o], wO), R::mul(own.vis, wC));
        const V4 Co = a.cc[o];
        const V4 Cn = owner ? Co : own.cc, Cp = owner ? own.cc : Co;
        const T x0 = R::sub(Cn.x, Cp.x), x1 = R::sub(Cn.y, Cp.y), x2 = R::sub(Cn.z, Cp.z);
        const T visFace = R::mul(visac, rl);
        T uF = T(0), vF = T(0), wF = T(0);
        const int cr = a.carry ? a.carry[f] : -1;
        if (cr >= 0) {
            uF = a.u[cr]; vF = a.v[cr]; wF = a.w[cr];
        } else if (cr <= -2) {
            const double *r = a.regionUVW + 3 * (-2 - cr);
            uF = (T) r[0]; vF = (T) r[1]; wF = (T) r[2];
        }
        const T mf = a.massFlux[f];
        const T fmin = std_min(mf, T(0)), fmax = std_max(mf, T(0));
        const T mO = owner ? fmin : fmax, mC = owner ? fmax : fmin;  // fmin weights cell2, fmax cell1
        const T fuci = R::add(R::mul(mO, a.u[o]), R::mul(mC, own.u));
        const T fvci = R::add(R::mul(mO, a.v[o]), R::mul(mC, own.v));
        const T fwci = R::add(R::mul(mO, a.w[o]), R::mul(mC, own.w));
        t[0] = R::mul(a.gammaBlend, R::sub(R::mul(mf, uF), fuci));
        t[3] = R::mul(a.gammaBlend, R::sub(R::mul(mf, vF), fvci));
        t[6] = R::mul(a.gammaBlend, R::sub(R::mul(mf, wF), fwci));
        t[1] = R::mul(visac, R::add(R::add(R::mul(R::add(du[0], du[0]), G.x), R::mul(R::add(du[1], dv[0]), G.y)),
                                    R::mul(R::add(du[2], dw[0]), G.z)));
        t[4] = R::mul(visac, R::add(R::add(R::mul(R::add(du[1], dv[0]), G.x), R::mul(R::add(dv[1], dv[1]), G.y)),
                                    R::mul(R::add(dv[2], dw[1]), G.z)));
        t[7] = R::mul(visac, R::add(R::add(R::mul(R::add(du[2], dw[0]), G.x), R::mul(R::add(dw[1], dv[2]), G.y)),
                                    R::mul(R::add(dw[2], dw[2]), G.z)));
        t[2] = R::mul(visFace, dot0(du[0], du[1], du[2], x0, x1, x2));
        t[5] = R::mul(visFace, dot0(dv[0], dv[1], dv[2], x0, x1, x2));
        t[8] = R::mul(visFace, dot0(dw[0], dw[1], dw[2], x0, x1, x2));
        if (owner) {
            a.rFace[2 * (int64_t) f] = R::sub(-visFace, std_max(mf, T(0)));
            a.rFace[2 * (int64_t) f + 1] = R::add(-visFace, std_min(mf, T(0)));
        }
        return owner ? UVW_OWNER : UVW_NEIGH;
    }
    // boundary face: c is its owner
    const int ib = -1 - en.y;
    const int ir = a.bndRegion[ib];
    const int it = a.regionType[ir];
    if (it == CUPCFD_RTYPE_DEFAULT) return UVW_NONE;
    const V4 X = a.fc[f], Cp = own.cc;
    const T x0 = R::sub(X.x, Cp.x), x1 = R::sub(X.y, Cp.y), x2 = R::sub(X.z, Cp.z);
    const T uc = own.u, vc = own.v, wc = own.w;
    const T du0 = own.g[0], du1 = own.g[1], du2 = own.g[2];
    const T dv0 = own.g[3], dv1 = own.g[4], dv2 = own.g[5];
    const T dw0 = own.g[6], dw1 = own.g[7], dw2 = own.g[8];
    if (it == CUPCFD_RTYPE_INLET || it == CUPCFD_RTYPE_OUTLET) {
        // UVWKernels.ipp:259-382 (outlet: operands of two sums swapped,
        // which IEEE addition does not see)
        T uF, vF, wF, visac;
        if (it == CUPCFD_RTYPE_INLET) {
            const double *r = a.regionUVW + 3 * ir;
            uF = (T) r[0]; vF = (T) r[1]; wF = (T) r[2];
            visac = a.visB[ib];
        } else {
            uF = uc; vF = vc; wF = wc;
            visac = own.vis;
        }
        const T visFace = R::mul(visac, rl);
        T mf = a.massFlux[f];
        if (it == CUPCFD_RTYPE_OUTLET && mf < T(0)) {
            mf = a.small;
            a.massFlux[f] = mf;
        }
        const T fl = R::add(-visFace, std_min(mf, T(0)));
        t[0] = R::mul(fl, uF); t[3] = R::mul(fl, vF); t[6] = R::mul(fl, wF);
        t[1] = R::mul(visac, R::add(R::add(R::mul(R::add(du0, du0), G.x), R::mul(R::add(du1, dv0), G.y)),
                                    R::mul(R::add(du2, dw0), G.z)));
        t[4] = R::mul(visac, R::add(R::add(R::mul(R::add(du1, dv0), G.x), R::mul(R::add(dv1, dv1), G.y)),
                                    R::mul(R::add(dv2, dw1), G.z)));
        t[7] = R::mul(visac, R::add(R::add(R::mul(R::add(du2, dw0), G.x), R::mul(R::add(dw1, dv2), G.y)),
                                    R::mul(R::add(dw2, dw2), G.z)));
        t[2] = R::mul(visFace, dot0(du0, du1, du2, x0, x1, x2));
        t[5] = R::mul(visFace, dot0(dv0, dv1, dv2, x0, x1, x2));
        t[8] = R::mul(visFace, dot0(dw0, dw1, dw2, x0, x1, x2));
        t[9] = fl;
        a.uB[ib] = uF; a.vB[ib] = vF; a.wB[ib] = wF;
        return UVW_INOUT;
    }
    const T area = X.w;
    T Xc, f0 = T(0), f1 = T(0), f2 = T(0);
    if (it == CUPCFD_RTYPE_SYMP) {
        // UVWKernels.ipp:383-436; visFace carried from an earlier face
        const int g = a.carry ? a.carry[f] : -1;
        Xc = g >= 0 ? vis_face_of(a, g) : T(0);
        const T visac = own.vis;
        const T us0 = R::add(uc, dot0(du0, du1, du2, x0, x1, x2));
        const T us1 = R::add(vc, dot0(dv0, dv1, dv2, x0, x1, x2));
        const T us2 = R::add(wc, dot0(dw0, dw1, dw2, x0, x1, x2));
        T n0 = R::sub(T(0), G.x), n1 = R::sub(T(0), G.y), n2 = R::sub(T(0), G.z);
        normalise(n0, n1, n2);
        const T dp = dot0(us0, us1, us2, n0, n1, n2);
        const T dn = a.bndDist ? (T) a.bndDist[ib] : T(0);
        const T tv = R::twice(visac);
        f0 = R::mul(R::div(R::mul(tv, R::mul(dp, n0)), dn), area);
        f1 = R::mul(R::div(R::mul(tv, R::mul(dp, n1)), dn), area);
        f2 = R::mul(R::div(R::mul(tv, R::mul(dp, n2)), dn), area);
        a.uB[ib] = us0; a.vB[ib] = us1; a.wB[ib] = us2;
    } else {
        // wall, UVWKernels.ipp:437-510
        const double *uw = a.regionUVW + 3 * ir;
        const T uw0 = (T) uw[0], uw1 = (T) uw[1], uw2 = (T) uw[2];
        const T visac = a.visB[ib];
        Xc = R::div(R::mul(visac, area), R::sqrt_(dot0(x0, x1, x2, x0, x1, x2)));
        T n0 = G.x, n1 = G.y, n2 = G.z;
        normalise(n0, n1, n2);
        const T up0 = R::sub(uc, uw0), up1 = R::sub(vc, uw1), up2 = R::sub(wc, uw2);
        const T dp = dot0(up0, up1, up2, n0, n1, n2);
        const T ut0 = R::sub(up0, R::mul(dp, n0)), ut1 = R::sub(up1, R::mul(dp, n1)), ut2 = R::sub(up2, R::mul(dp, n2));
        const T uvel = R::abs_sum3(ut0, ut1, ut2);
        if (uvel > a.small) {
            const T dn = a.bndDist ? (T) a.bndDist[ib] : T(0);
            f0 = R::mul(R::div(R::mul(visac, ut0), dn), area);
            f1 = R::mul(R::div(R::mul(visac, ut1), dn), area);
            f2 = R::mul(R::div(R::mul(visac, ut2), dn), area);
        }
        a.shear[3 * (int64_t) ib] = (double) f0;
        a.shear[3 * (int64_t) ib + 1] = (double) f1;
        a.shear[3 * (int64_t) ib + 2] = (double) f2;
        a.uB[ib] = uw0; a.vB[ib] = uw1; a.wB[ib] = uw2;
    }
    t[0] = R::mul(Xc, uc); t[3] = R::mul(Xc, vc); t[6] = R::mul(Xc, wc);
    t[1] = f0; t[4] = f1; t[7] = f2;
    t[9] = Xc;
    return UVW_WALLSYM;
}

// Applies one incidence's terms to the cell's running su/sv/sw (s) and
// au/av/aw (ad).
template <class T>
__device__ __forceinline__ void uvw_fold(int kind, const T (&t)[10], T (&s)[3], T (&ad)[3]) {
    using R = UvwReal<T>;
    switch (kind) {
    case UVW_OWNER:
#pragma unroll
        for (int q = 0; q < 3; q++) s[q] = R::sub(R::add(R::sub(s[q], t[3 * q]), t[3 * q + 1]), t[3 * q + 2]);
        break;
    case UVW_NEIGH:
#pragma unroll
        for (int q = 0; q < 3; q++) s[q] = R::add(R::sub(R::add(s[q], t[3 * q]), t[3 * q + 1]), t[3 * q + 2]);
        break;
    case UVW_INOUT:
#pragma unroll
        for (int q = 0; q < 3; q++) {
            ad[q] = R::sub(ad[q], t[9]);
            s[q] = R::sub(R::add(R::sub(s[q], t[3 * q]), t[3 * q + 1]), t[3 * q + 2]);
        }
        break;
    case UVW_WALLSYM:
#pragma unroll
        for (int q = 0; q < 3; q++) {
            ad[q] = R::add(ad[q], t[9]);
            s[q] = R::sub(R::add(s[q], t[3 * q]), t[3 * q + 1]);
        }
        break;
    default:
        break;
    }
}

// One thread per cell, incidences in order. (One thread per incidence with
// the terms staged in shared memory and one warp folding them measured
// slower: 4.2-5.0 ms against 2.3 ms at 256^3.)
#ifndef UVW_CELL_MINB
#define UVW_CELL_MINB 2  // resident 256-thread blocks per SM asked of the register allocator (118 registers:
                         // the own-cell values held for the whole cell; 3 blocks at 80 spill them)
#endif
// The L2-prefetch launches run 64-thread blocks, four per 256-cell tile, at
// the same registers and warps per SM: a block's slot frees when its two
// warps end instead of its slowest of eight (2.007 -> 1.941 ms at 256^3;
// 128-thread blocks 1.964, 32-thread 1.954).
#ifndef UVW_PF_BLOCK
#define UVW_PF_BLOCK 64
#endif
#ifndef UVW_CHUNK
#define UVW_CHUNK 6      // incidence entries loaded ahead (a hexahedral cell in one chunk)
#endif
template <class T>
__device__ __forceinline__ void uvw_cell(const UvwArgs<T> &a, int c) {
    int wdt;
    const int2 *e = cell_entries(a.sv, c, wdt);
    T s[3] = {a.su[c], a.sv_[c], a.sw[c]}, ad[3] = {a.au[c], a.av[c], a.aw[c]};
    const UvwOwn<T> own = uvw_own(a, c);
    // the chunk's entries first (independent loads), then incidence by incidence
    for (int k0 = 0; k0 < wdt; k0 += UVW_CHUNK) {
        int2 en[UVW_CHUNK];
        load_entries<UVW_CHUNK>(e, k0, wdt, en);
        for (int j = 0; j < UVW_CHUNK; j++) {
            if (en[j].x < 0) break;
            T t[10];
            int kind = uvw_terms(a, c, own, en[j], t);
            uvw_fold(kind, t, s, ad);
        }
    }
    a.su[c] = s[0]; a.sv_[c] = s[1]; a.sw[c] = s[2];
    a.au[c] = ad[0]; a.av[c] = ad[1]; a.aw[c] = ad[2];
}

// The same with the L2 prefetch of the tile one wave of this kernel's
// resident blocks ahead (prefetch.cuh): its entries, face records and mass
// fluxes, and its cells' entries in the twenty cell arrays the loop reads.
// Needs the owner-sorted face order and 16-byte aligned arrays; launched as
// UVW_PF_BLOCK-thread blocks, TILE_CELLS / UVW_PF_BLOCK per tile (the last
// block of a tile prefetches for the tile).
template <class T>
__device__ __forceinline__ void uvw_cell_pf(const UvwArgs<T> &a, const PrefetchArgs &pf) {
    constexpr int TC = TILE_CELLS;
    const TileBlock<UVW_PF_BLOCK> tb(pf);
    const int c = tb.c, tp = tb.tp;
    const bool lead = tb.lead;
    __shared__ int4 s_rng;
    if (lead) fetch_ranges_async(&s_rng, pf.desc + tp);
    if (c < a.nC) uvw_cell(a, c);
    if (lead) {
        const int64_t L = a.ldg;
        const void *const cellSrc[20] = {a.u, a.v, a.w, a.visC, a.su, a.sv_, a.sw, a.au, a.av, a.aw,
                                         a.grads, a.grads + L, a.grads + 2 * L, a.grads + 3 * L, a.grads + 4 * L,
                                         a.grads + 5 * L, a.grads + 6 * L, a.grads + 7 * L, a.grads + 8 * L, a.cc};
        int cellBytes[20];
#pragma unroll
        for (int i = 0; i < 19; i++) cellBytes[i] = TC * (int) sizeof(T);
        cellBytes[19] = TC * (int) sizeof(typename UvwReal<T>::V4);
        prefetch_tile<20>(pf, tp, ranges_ready(&s_rng), a.fg, (int) sizeof(typename UvwReal<T>::V4),
                          (const T *) a.massFlux, cellSrc, cellBytes);
    }
}

// FP64 (the reference's T = double): plain and L2-prefetch launches.
// At 256^3 on one box: 2.15 ms with the own-cell values held at two blocks
// per SM, against 2.22 ms reloading them at three; 2.01 ms with the weights
// selected once per incidence instead of each value.
__global__ void __launch_bounds__(256, UVW_CELL_MINB) k_uvw_f64(const __grid_constant__ UvwArgs<double> a) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < a.nC) uvw_cell(a, c);
}
__global__ void __launch_bounds__(UVW_PF_BLOCK, UVW_CELL_MINB *TILE_CELLS / UVW_PF_BLOCK) k_uvw_f64_pf(const __grid_constant__ UvwArgs<double> a,
                                                                          PrefetchArgs pf) {
    uvw_cell_pf(a, pf);
}
// The reference's T = float instantiation.
__global__ void __launch_bounds__(256, UVW_CELL_MINB) k_uvw_f32ref(const __grid_constant__ UvwArgs<float> a) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < a.nC) uvw_cell(a, c);
}
__global__ void __launch_bounds__(UVW_PF_BLOCK, UVW_CELL_MINB *TILE_CELLS / UVW_PF_BLOCK) k_uvw_f32ref_pf(const __grid_constant__ UvwArgs<float> a,
                                                                             PrefetchArgs pf) {
    uvw_cell_pf(a, pf);
}

// ---------------------------------------------------------------------------
// Carried-value sources: exclusive prefix maxima over reference face ids of
// "face g sets uFace" (inlet, outlet) and "face g sets visFace" (interior,
// inlet, outlet), in three passes over blocks of CARRY_T faces.
// ---------------------------------------------------------------------------
constexpr int CARRY_T = 1024;

struct CarryIn {
    int nF;
    const int *faceO2N;  // reference face -> internal face
    const int2 *fcells;
    const int *bndRegion, *regionType;
};

// Face f's (uFace setter, visFace setter) values: f where it sets, else -1.
__device__ __forceinline__ int2 carry_vals(const CarryIn &a, int f) {
    if (f >= a.nF) return make_int2(-1, -1);
    int2 pn = a.fcells[a.faceO2N[f]];
    if (pn.y >= 0) return make_int2(-1, f);
    int t = a.regionType[a.bndRegion[-1 - pn.y]];
    bool s = t == CUPCFD_RTYPE_INLET || t == CUPCFD_RTYPE_OUTLET;
    return make_int2(s ? f : -1, s ? f : -1);
}

// Inclusive prefix maximum of (x, y) over the block's threads.
__device__ __forceinline__ int2 block_incl_max(int2 v, int2 *warpTot) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int x = __shfl_up_sync(0xffffffffu, v.x, o), y = __shfl_up_sync(0xffffffffu, v.y, o);
        if (lane >= o) { v.x = max(v.x, x); v.y = max(v.y, y); }
    }
    if (lane == 31) warpTot[wid] = v;
    __syncthreads();
    if (wid == 0) {
        int2 t = lane < (int) (blockDim.x >> 5) ? warpTot[lane] : make_int2(-1, -1);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int x = __shfl_up_sync(0xffffffffu, t.x, o), y = __shfl_up_sync(0xffffffffu, t.y, o);
            if (lane >= o) { t.x = max(t.x, x); t.y = max(t.y, y); }
        }
        warpTot[lane] = t;
    }
    __syncthreads();
    if (wid > 0) {
        int2 p = warpTot[wid - 1];
        v.x = max(v.x, p.x); v.y = max(v.y, p.y);
    }
    return v;
}

// pass 1: each block's maxima
__global__ void __launch_bounds__(CARRY_T) k_carry_reduce(CarryIn a, int2 *__restrict__ blockMax) {
    __shared__ int2 wt[32];
    int2 v = carry_vals(a, blockIdx.x * CARRY_T + threadIdx.x);
    v = block_incl_max(v, wt);
    if (threadIdx.x == CARRY_T - 1) blockMax[blockIdx.x] = v;
}

// pass 2 (one block): exclusive prefix maxima of the block maxima, in place
__global__ void __launch_bounds__(CARRY_T) k_carry_scan(int nBlocks, int2 *__restrict__ blockMax) {
    __shared__ int2 wt[32];
    __shared__ int2 carryIn;
    if (threadIdx.x == 0) carryIn = make_int2(-1, -1);
    __syncthreads();
    for (int b0 = 0; b0 < nBlocks; b0 += CARRY_T) {
        int b = b0 + threadIdx.x;
        int2 v = b < nBlocks ? blockMax[b] : make_int2(-1, -1);
        int2 incl = block_incl_max(v, wt);
        int2 base = carryIn;
        int2 prev = make_int2(__shfl_up_sync(0xffffffffu, incl.x, 1), __shfl_up_sync(0xffffffffu, incl.y, 1));
        __shared__ int2 lastOfWarp[32];
        if ((threadIdx.x & 31) == 31) lastOfWarp[threadIdx.x >> 5] = incl;
        __syncthreads();
        if ((threadIdx.x & 31) == 0) prev = threadIdx.x == 0 ? make_int2(-1, -1) : lastOfWarp[(threadIdx.x >> 5) - 1];
        int2 ex = make_int2(max(base.x, prev.x), max(base.y, prev.y));
        if (b < nBlocks) blockMax[b] = ex;
        __syncthreads();
        if (threadIdx.x == CARRY_T - 1) carryIn = make_int2(max(base.x, incl.x), max(base.y, incl.y));
        __syncthreads();
    }
}

// pass 3: each face's exclusive prefix maxima, encoded into carry[internal f]
__global__ void __launch_bounds__(CARRY_T) k_carry_apply(CarryIn a, const int2 *__restrict__ blockPrefix,
                                                        int *__restrict__ carry) {
    __shared__ int2 wt[32];
    __shared__ int2 lastOfWarp[32];
    const int f = blockIdx.x * CARRY_T + threadIdx.x;
    int2 incl = block_incl_max(carry_vals(a, f), wt);
    if ((threadIdx.x & 31) == 31) lastOfWarp[threadIdx.x >> 5] = incl;
    __syncthreads();
    int2 prev = make_int2(__shfl_up_sync(0xffffffffu, incl.x, 1), __shfl_up_sync(0xffffffffu, incl.y, 1));
    if ((threadIdx.x & 31) == 0) prev = threadIdx.x == 0 ? make_int2(-1, -1) : lastOfWarp[(threadIdx.x >> 5) - 1];
    const int2 base = blockPrefix[blockIdx.x];
    const int gUV = max(base.x, prev.x), gVis = max(base.y, prev.y);
    if (f >= a.nF) return;
    const int fi = a.faceO2N[f];
    const int2 pn = a.fcells[fi];
    int code = -1;
    if (pn.y >= 0) {
        if (gUV >= 0) {
            const int2 pg = a.fcells[a.faceO2N[gUV]];
            const int rg = a.bndRegion[-1 - pg.y];
            code = a.regionType[rg] == CUPCFD_RTYPE_OUTLET ? pg.x : -2 - rg;
        }
    } else if (a.regionType[a.bndRegion[-1 - pn.y]] == CUPCFD_RTYPE_SYMP) {
        code = gVis >= 0 ? a.faceO2N[gVis] : -1;
    }
    carry[fi] = code;
}

}  // namespace cupcfd_gpu
