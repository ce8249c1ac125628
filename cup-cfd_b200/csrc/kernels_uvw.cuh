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

// std::min / std::max of <algorithm>: min(a,b) = b < a ? b : a,
// max(a,b) = a < b ? b : a (the first argument wins ties and NaN compares).
__device__ __forceinline__ double std_min(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double std_max(double a, double b) { return (a < b) ? b : a; }

// EuclideanVector::dotProduct (EuclideanVector.cpp:83-90): accumulated from 0.
__device__ __forceinline__ double dot0(double a0, double a1, double a2, double b0, double b1, double b2) {
    double d = 0.0;
    d = da(d, dm(a0, b0));
    d = da(d, dm(a1, b1));
    d = da(d, dm(a2, b2));
    return d;
}

// EuclideanVector::normalise (EuclideanVector.cpp:100-109)
__device__ __forceinline__ void normalise(double &x, double &y, double &z) {
    double L = __dsqrt_rn(dot0(x, y, z, x, y, z));
    if (L != 0.0) {
        double sc = dvd(1.0, L);
        x = dm(x, sc); y = dm(y, sc); z = dm(z, sc);
    }
}

struct UvwArgs {
    int nC;
    SellView sv;
    const int2 *fcells;
    const double4 *fg, *fc, *cc;           // {S, lambda}, {x_f, area}, {x_c, 0}
    const int *bndRegion, *regionType;
    const double *regionUVW;
    const double *rlencos;                 // [nF] internal, null = zero
    const double *bndDist;                 // [nB], null = zero
    const int *carry;                      // [nF] internal; null when no region is an inlet, outlet or symmetry
    double gammaBlend, small;
    const double *u, *v, *w, *visC;        // [nC] internal
    const double *visB;                    // [nB]
    const double *grads;                   // 9 blocks [ldg]: dudx xyz, dvdx xyz, dwdx xyz
    int64_t ldg;
    double *uB, *vB, *wB;                  // [nB]
    double *massFlux, *rFace;              // [nF], [2 nF] internal
    double *shear;                         // [3 nB]
    double *su, *sv_, *sw, *au, *av, *aw;  // [nC] internal
};

// visFace that face g leaves behind (interior, inlet and outlet faces set it,
// UVWKernels.ipp:160, 274, 335).
__device__ __forceinline__ double vis_face_of(const UvwArgs &a, int g) {
    int2 pn = a.fcells[g];
    double rl = a.rlencos ? a.rlencos[g] : 0.0;
    double visac;
    if (pn.y >= 0) {
        double facn = a.fg[g].w, facp = ds(1.0, facn);
        visac = da(dm(a.visC[pn.y], facn), dm(a.visC[pn.x], facp));
    } else {
        int ib = -1 - pn.y;
        visac = a.regionType[a.bndRegion[ib]] == CUPCFD_RTYPE_INLET ? a.visB[ib] : a.visC[pn.x];
    }
    return dm(visac, rl);
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
__device__ __forceinline__ int uvw_terms(const UvwArgs &a, int c, int2 en, double (&t)[10]) {
    const int64_t L = a.ldg;
    auto gr = [&](int q, int cell) { return a.grads[q * L + cell]; };
    const int f = en.x >> 1;
    const bool owner = (en.x & 1) == 0;
    const double4 G = a.fg[f];
    const double rl = a.rlencos ? a.rlencos[f] : 0.0;
    if (en.y >= 0) {
        // interior face (UVWKernels.ipp:145-228)
        const int ip = owner ? c : en.y, in = owner ? en.y : c;
        const double facn = G.w, facp = ds(1.0, facn);
        double du[3], dv[3], dw[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            du[d] = da(dm(gr(d, in), facn), dm(gr(d, ip), facp));
            dv[d] = da(dm(gr(3 + d, in), facn), dm(gr(3 + d, ip), facp));
            dw[d] = da(dm(gr(6 + d, in), facn), dm(gr(6 + d, ip), facp));
        }
        const double visac = da(dm(a.visC[in], facn), dm(a.visC[ip], facp));
        const double4 Cn = a.cc[in], Cp = a.cc[ip];
        const double x0 = ds(Cn.x, Cp.x), x1 = ds(Cn.y, Cp.y), x2 = ds(Cn.z, Cp.z);
        const double visFace = dm(visac, rl);
        double uF = 0.0, vF = 0.0, wF = 0.0;
        const int cr = a.carry ? a.carry[f] : -1;
        if (cr >= 0) {
            uF = a.u[cr]; vF = a.v[cr]; wF = a.w[cr];
        } else if (cr <= -2) {
            const double *r = a.regionUVW + 3 * (-2 - cr);
            uF = r[0]; vF = r[1]; wF = r[2];
        }
        const double mf = a.massFlux[f];
        const double fmin = std_min(mf, 0.0), fmax = std_max(mf, 0.0);
        const double fuci = da(dm(fmin, a.u[in]), dm(fmax, a.u[ip]));
        const double fvci = da(dm(fmin, a.v[in]), dm(fmax, a.v[ip]));
        const double fwci = da(dm(fmin, a.w[in]), dm(fmax, a.w[ip]));
        t[0] = dm(a.gammaBlend, ds(dm(mf, uF), fuci));
        t[3] = dm(a.gammaBlend, ds(dm(mf, vF), fvci));
        t[6] = dm(a.gammaBlend, ds(dm(mf, wF), fwci));
        t[1] = dm(visac, da(da(dm(da(du[0], du[0]), G.x), dm(da(du[1], dv[0]), G.y)), dm(da(du[2], dw[0]), G.z)));
        t[4] = dm(visac, da(da(dm(da(du[1], dv[0]), G.x), dm(da(dv[1], dv[1]), G.y)), dm(da(dv[2], dw[1]), G.z)));
        t[7] = dm(visac, da(da(dm(da(du[2], dw[0]), G.x), dm(da(dw[1], dv[2]), G.y)), dm(da(dw[2], dw[2]), G.z)));
        t[2] = dm(visFace, dot0(du[0], du[1], du[2], x0, x1, x2));
        t[5] = dm(visFace, dot0(dv[0], dv[1], dv[2], x0, x1, x2));
        t[8] = dm(visFace, dot0(dw[0], dw[1], dw[2], x0, x1, x2));
        if (owner) {
            a.rFace[2 * (int64_t) f] = ds(-visFace, std_max(mf, 0.0));
            a.rFace[2 * (int64_t) f + 1] = da(-visFace, std_min(mf, 0.0));
        }
        return owner ? UVW_OWNER : UVW_NEIGH;
    }
    // boundary face: c is its owner
    const int ib = -1 - en.y;
    const int ir = a.bndRegion[ib];
    const int it = a.regionType[ir];
    if (it == CUPCFD_RTYPE_DEFAULT) return UVW_NONE;
    const double4 X = a.fc[f], Cp = a.cc[c];
    const double x0 = ds(X.x, Cp.x), x1 = ds(X.y, Cp.y), x2 = ds(X.z, Cp.z);
    const double uc = a.u[c], vc = a.v[c], wc = a.w[c];
    const double du0 = gr(0, c), du1 = gr(1, c), du2 = gr(2, c);
    const double dv0 = gr(3, c), dv1 = gr(4, c), dv2 = gr(5, c);
    const double dw0 = gr(6, c), dw1 = gr(7, c), dw2 = gr(8, c);
    if (it == CUPCFD_RTYPE_INLET || it == CUPCFD_RTYPE_OUTLET) {
        // UVWKernels.ipp:259-382 (outlet: operands of two sums swapped,
        // which IEEE addition does not see)
        double uF, vF, wF, visac;
        if (it == CUPCFD_RTYPE_INLET) {
            const double *r = a.regionUVW + 3 * ir;
            uF = r[0]; vF = r[1]; wF = r[2];
            visac = a.visB[ib];
        } else {
            uF = uc; vF = vc; wF = wc;
            visac = a.visC[c];
        }
        const double visFace = dm(visac, rl);
        double mf = a.massFlux[f];
        if (it == CUPCFD_RTYPE_OUTLET && mf < 0.0) {
            mf = a.small;
            a.massFlux[f] = mf;
        }
        const double fl = da(-visFace, std_min(mf, 0.0));
        t[0] = dm(fl, uF); t[3] = dm(fl, vF); t[6] = dm(fl, wF);
        t[1] = dm(visac, da(da(dm(da(du0, du0), G.x), dm(da(du1, dv0), G.y)), dm(da(du2, dw0), G.z)));
        t[4] = dm(visac, da(da(dm(da(du1, dv0), G.x), dm(da(dv1, dv1), G.y)), dm(da(dv2, dw1), G.z)));
        t[7] = dm(visac, da(da(dm(da(du2, dw0), G.x), dm(da(dw1, dv2), G.y)), dm(da(dw2, dw2), G.z)));
        t[2] = dm(visFace, dot0(du0, du1, du2, x0, x1, x2));
        t[5] = dm(visFace, dot0(dv0, dv1, dv2, x0, x1, x2));
        t[8] = dm(visFace, dot0(dw0, dw1, dw2, x0, x1, x2));
        t[9] = fl;
        a.uB[ib] = uF; a.vB[ib] = vF; a.wB[ib] = wF;
        return UVW_INOUT;
    }
    const double area = X.w;
    double Xc, f0 = 0.0, f1 = 0.0, f2 = 0.0;
    if (it == CUPCFD_RTYPE_SYMP) {
        // UVWKernels.ipp:383-436; visFace carried from an earlier face
        const int g = a.carry ? a.carry[f] : -1;
        Xc = g >= 0 ? vis_face_of(a, g) : 0.0;
        const double visac = a.visC[c];
        const double us0 = da(uc, dot0(du0, du1, du2, x0, x1, x2));
        const double us1 = da(vc, dot0(dv0, dv1, dv2, x0, x1, x2));
        const double us2 = da(wc, dot0(dw0, dw1, dw2, x0, x1, x2));
        double n0 = ds(0.0, G.x), n1 = ds(0.0, G.y), n2 = ds(0.0, G.z);
        normalise(n0, n1, n2);
        const double dp = dot0(us0, us1, us2, n0, n1, n2);
        const double dn = a.bndDist ? a.bndDist[ib] : 0.0;
        const double tv = dm(2.0, visac);
        f0 = dm(dvd(dm(tv, dm(dp, n0)), dn), area);
        f1 = dm(dvd(dm(tv, dm(dp, n1)), dn), area);
        f2 = dm(dvd(dm(tv, dm(dp, n2)), dn), area);
        a.uB[ib] = us0; a.vB[ib] = us1; a.wB[ib] = us2;
    } else {
        // wall, UVWKernels.ipp:437-510
        const double *uw = a.regionUVW + 3 * ir;
        const double visac = a.visB[ib];
        Xc = dvd(dm(visac, area), __dsqrt_rn(dot0(x0, x1, x2, x0, x1, x2)));
        double n0 = G.x, n1 = G.y, n2 = G.z;
        normalise(n0, n1, n2);
        const double up0 = ds(uc, uw[0]), up1 = ds(vc, uw[1]), up2 = ds(wc, uw[2]);
        const double dp = dot0(up0, up1, up2, n0, n1, n2);
        const double ut0 = ds(up0, dm(dp, n0)), ut1 = ds(up1, dm(dp, n1)), ut2 = ds(up2, dm(dp, n2));
        const double uvel = da(da(fabs(ut0), fabs(ut1)), fabs(ut2));
        if (uvel > a.small) {
            const double dn = a.bndDist ? a.bndDist[ib] : 0.0;
            f0 = dm(dvd(dm(visac, ut0), dn), area);
            f1 = dm(dvd(dm(visac, ut1), dn), area);
            f2 = dm(dvd(dm(visac, ut2), dn), area);
        }
        a.shear[3 * (int64_t) ib] = f0;
        a.shear[3 * (int64_t) ib + 1] = f1;
        a.shear[3 * (int64_t) ib + 2] = f2;
        a.uB[ib] = uw[0]; a.vB[ib] = uw[1]; a.wB[ib] = uw[2];
    }
    t[0] = dm(Xc, uc); t[3] = dm(Xc, vc); t[6] = dm(Xc, wc);
    t[1] = f0; t[4] = f1; t[7] = f2;
    t[9] = Xc;
    return UVW_WALLSYM;
}

// Applies one incidence's terms to the cell's running su/sv/sw (s) and
// au/av/aw (ad).
__device__ __forceinline__ void uvw_fold(int kind, const double (&t)[10], double (&s)[3], double (&ad)[3]) {
    switch (kind) {
    case UVW_OWNER:
#pragma unroll
        for (int q = 0; q < 3; q++) s[q] = ds(da(ds(s[q], t[3 * q]), t[3 * q + 1]), t[3 * q + 2]);
        break;
    case UVW_NEIGH:
#pragma unroll
        for (int q = 0; q < 3; q++) s[q] = da(ds(da(s[q], t[3 * q]), t[3 * q + 1]), t[3 * q + 2]);
        break;
    case UVW_INOUT:
#pragma unroll
        for (int q = 0; q < 3; q++) {
            ad[q] = ds(ad[q], t[9]);
            s[q] = ds(da(ds(s[q], t[3 * q]), t[3 * q + 1]), t[3 * q + 2]);
        }
        break;
    case UVW_WALLSYM:
#pragma unroll
        for (int q = 0; q < 3; q++) {
            ad[q] = da(ad[q], t[9]);
            s[q] = ds(da(s[q], t[3 * q]), t[3 * q + 1]);
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
#define UVW_CELL_MINB 3  // resident 256-thread blocks per SM asked of the register allocator (80 registers)
#endif
#ifndef UVW_CHUNK
#define UVW_CHUNK 6      // incidence entries loaded ahead (a hexahedral cell in one chunk)
#endif
__device__ __forceinline__ void uvw_cell(const UvwArgs &a, int c) {
    int wdt;
    const int2 *e = cell_entries(a.sv, c, wdt);
    double s[3] = {a.su[c], a.sv_[c], a.sw[c]}, ad[3] = {a.au[c], a.av[c], a.aw[c]};
    // the chunk's entries first (independent loads), then incidence by incidence
    for (int k0 = 0; k0 < wdt; k0 += UVW_CHUNK) {
        int2 en[UVW_CHUNK];
        load_entries<UVW_CHUNK>(e, k0, wdt, en);
        for (int j = 0; j < UVW_CHUNK; j++) {
            if (en[j].x < 0) break;
            double t[10];
            int kind = uvw_terms(a, c, en[j], t);
            uvw_fold(kind, t, s, ad);
        }
    }
    a.su[c] = s[0]; a.sv_[c] = s[1]; a.sw[c] = s[2];
    a.au[c] = ad[0]; a.av[c] = ad[1]; a.aw[c] = ad[2];
}

__global__ void __launch_bounds__(256, UVW_CELL_MINB) k_uvw_f64(const __grid_constant__ UvwArgs a) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < a.nC) uvw_cell(a, c);
}

// The same with the L2 prefetch of the tile one wave of this kernel's
// resident blocks ahead (prefetch.cuh): its entries, face records and mass
// fluxes, and its cells' entries in the twenty cell arrays the loop reads.
// Needs the owner-sorted face order, 256-thread blocks and 16-byte aligned
// arrays. 2.13 ms at 256^3 against 2.21 ms without the prefetch.
__global__ void __launch_bounds__(TILE_CELLS, UVW_CELL_MINB) k_uvw_f64_pf(const __grid_constant__ UvwArgs a,
                                                                          PrefetchArgs pf) {
    constexpr int T = TILE_CELLS;
    const int c = blockIdx.x * T + threadIdx.x;
    const int tp = blockIdx.x + pf.dist;
    const bool lead = threadIdx.x == T - 32 && tp < pf.nTiles;
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
        for (int i = 0; i < 19; i++) cellBytes[i] = T * 8;
        cellBytes[19] = T * 32;
        prefetch_tile<20>(pf, tp, ranges_ready(&s_rng), a.fg, 32, (const double *) a.massFlux, cellSrc, cellBytes);
    }
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
