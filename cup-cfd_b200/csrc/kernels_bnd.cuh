// Boundary / region loops of the mass-flux step, reference arithmetic
// (FluxMassDolfynBoundaryLoop1-5, FluxMassDolfynRegionLoop; MassKernels.ipp:311-554).
//
// The reference walks boundaries ib = 0 .. nB-1 and adds into scalars (and,
// in loop 2, per-region sums) one boundary at a time; reproducing its
// rounding means adding in that order (ordered_sum.cuh: the selected
// boundaries gathered in parallel, then one chain of additions per sum). The per-boundary updates
// (loops 4 and 5) are independent and run one thread per boundary. Loop 5's
// su[cell1] -= massFlux applies, per cell, its outlet boundaries in
// ascending boundary id: one thread per cell over the boundaries sorted by
// (cell, id) at mesh creation.
//
// Face data is reached through a boundary -> face map, either to reference
// face ids (host-buffer calls, arrays in the reference's numbering) or to
// internal ones (device-resident calls); cells likewise.
//
// F32: the arithmetic of the reference's T = float instantiation, every
// operation rounded to float, on values held in double arrays (which hold
// float values exactly; a float mesh's FP64 geometry holds its float
// geometry exactly). The loops have no double literals in their arithmetic.
#pragma once

#include "arith.cuh"
#include "internal.cuh"
#include "ordered_sum.cuh"

namespace cupcfd_gpu {

// One IEEE operation in double, or in float on float values held in double.
template <bool F32>
struct BndOps {
    static __device__ __forceinline__ double mul(double a, double b) {
        return F32 ? (double) __fmul_rn((float) a, (float) b) : __dmul_rn(a, b);
    }
    static __device__ __forceinline__ double add(double a, double b) {
        return F32 ? (double) __fadd_rn((float) a, (float) b) : __dadd_rn(a, b);
    }
    static __device__ __forceinline__ double sub(double a, double b) {
        return F32 ? (double) __fsub_rn((float) a, (float) b) : __dsub_rn(a, b);
    }
    static __device__ __forceinline__ double div(double a, double b) {
        return F32 ? (double) __fdiv_rn((float) a, (float) b) : __ddiv_rn(a, b);
    }
    static __device__ __forceinline__ double sqrt_(double a) {
        return F32 ? (double) __fsqrt_rn((float) a) : __dsqrt_rn(a);
    }
};

// Loop 3's last line: *ratearea = -flowin / areaout (MassKernels.ipp:390).
template <bool F32>
__global__ void k_bl_ratearea(const double *__restrict__ flowin, const double *__restrict__ areaout,
                              double *__restrict__ ratearea) {
    *ratearea = BndOps<F32>::div(-*flowin, *areaout);
}

// Loop 4 per outlet boundary (MassKernels.ipp:437-451): massFlux from the
// area rate, the unit normal, the outlet velocities.
template <bool F32>
__global__ void k_bl4_update(int nB, const int *__restrict__ bndRegion, const int *__restrict__ regionType,
                             const double *__restrict__ splvl, const int *__restrict__ mapMF,
                             const int *__restrict__ bndFaceInt, const double4 *__restrict__ fg64,
                             const double4 *__restrict__ fc64, double *__restrict__ massFlux, double *__restrict__ uB,
                             double *__restrict__ vB, double *__restrict__ wB, const double *__restrict__ denB,
                             const double *__restrict__ ratearea) {
    using O = BndOps<F32>;
    int ib = blockIdx.x * blockDim.x + threadIdx.x;
    if (ib >= nB) return;
    int ir = bndRegion[ib];
    if (regionType[ir] != CUPCFD_RTYPE_OUTLET) return;
    int i = mapMF[ib], fi = bndFaceInt[ib];
    double area = fc64[fi].w;
    double m = O::mul(O::mul(*ratearea, area), splvl[ir]);
    massFlux[i] = m;
    double faceFlux = O::div(O::div(m, denB[ib]), area);
    // EuclideanVector::normalise (EuclideanVector.cpp:100-109), length from a
    // dot product accumulated from 0 (EuclideanVector.cpp:83-98)
    double4 S = fg64[fi];
    double n0 = S.x, n1 = S.y, n2 = S.z;
    double d = 0.0;
    d = O::add(d, O::mul(n0, n0));
    d = O::add(d, O::mul(n1, n1));
    d = O::add(d, O::mul(n2, n2));
    double L = O::sqrt_(d);
    if (L != 0.0) {
        double sc = O::div(1.0, L);
        n0 = O::mul(n0, sc); n1 = O::mul(n1, sc); n2 = O::mul(n2, sc);
    }
    uB[ib] = O::mul(faceFlux, n0);
    vB[ib] = O::mul(faceFlux, n1);
    wB[ib] = O::mul(faceFlux, n2);
}

// Loop 5 per outlet boundary (MassKernels.ipp:495-508): massFlux scaled by
// its region's factor, optional velocity scaling.
template <bool F32>
__global__ void k_bl5_update(int nB, const int *__restrict__ bndRegion, const int *__restrict__ regionType,
                             const int *__restrict__ mapMF, double *__restrict__ massFlux,
                             const double *__restrict__ flowFact, double *__restrict__ uB, double *__restrict__ vB,
                             double *__restrict__ wB, double fact, int solveU, int solveV, int solveW) {
    int ib = blockIdx.x * blockDim.x + threadIdx.x;
    if (ib >= nB) return;
    int ir = bndRegion[ib];
    if (regionType[ir] != CUPCFD_RTYPE_OUTLET) return;
    using O = BndOps<F32>;
    int i = mapMF[ib];
    massFlux[i] = O::mul(massFlux[i], flowFact[ir]);
    if (solveU) uB[ib] = O::mul(uB[ib], fact);
    if (solveV) vB[ib] = O::mul(vB[ib], fact);
    if (solveW) wB[ib] = O::mul(wB[ib], fact);
}

// Loop 5's su[cell1] -= massFlux (MassKernels.ipp:510-516), per cell in
// ascending boundary id: sortedBnd lists the boundaries by (cell, id) and
// sortedCell their cells in the caller's numbering.
template <bool F32>
__global__ void k_bl5_su(int nB, const int *__restrict__ sortedBnd, const int *__restrict__ sortedCell,
                         const int *__restrict__ bndRegion, const int *__restrict__ regionType,
                         const int *__restrict__ mapMF, const double *__restrict__ massFlux, double *__restrict__ su) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nB) return;
    int c = sortedCell[k];
    if (k > 0 && sortedCell[k - 1] == c) return;  // not the first boundary of its cell
    double acc = su[c];
    bool any = false;
    for (int j = k; j < nB && sortedCell[j] == c; j++) {
        int ib = sortedBnd[j];
        if (regionType[bndRegion[ib]] != CUPCFD_RTYPE_OUTLET) continue;
        acc = BndOps<F32>::sub(acc, massFlux[mapMF[ib]]);
        any = true;
    }
    if (any) su[c] = acc;
}

// FluxMassDolfynRegionLoop (MassKernels.ipp:532-551).
template <bool F32>
__global__ void k_region_loop(int nR, const int *__restrict__ regionType, const double *__restrict__ splvl,
                              const double *__restrict__ flowRegion, const double *__restrict__ flowIn,
                              double *__restrict__ flowFact) {
    int ir = blockIdx.x * blockDim.x + threadIdx.x;
    if (ir >= nR) return;
    using O = BndOps<F32>;
    flowFact[ir] = regionType[ir] == CUPCFD_RTYPE_OUTLET ? O::div(-O::mul(splvl[ir], *flowIn), flowRegion[ir]) : 0.0;
}

}  // namespace cupcfd_gpu
