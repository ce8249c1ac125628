// Boundary / region loops of the mass-flux step, FP64, reference arithmetic
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
#pragma once

#include "arith.cuh"
#include "internal.cuh"
#include "ordered_sum.cuh"

namespace cupcfd_gpu {

// Loop 3's last line: *ratearea = -flowin / areaout (MassKernels.ipp:390).
__global__ void k_bl_ratearea(const double *__restrict__ flowin, const double *__restrict__ areaout,
                              double *__restrict__ ratearea) {
    *ratearea = __ddiv_rn(-*flowin, *areaout);
}

// Loop 4 per outlet boundary (MassKernels.ipp:437-451): massFlux from the
// area rate, the unit normal, the outlet velocities.
__global__ void k_bl4_update(int nB, const int *__restrict__ bndRegion, const int *__restrict__ regionType,
                             const double *__restrict__ splvl, const int *__restrict__ mapMF,
                             const int *__restrict__ bndFaceInt, const double4 *__restrict__ fg64,
                             const double4 *__restrict__ fc64, double *__restrict__ massFlux, double *__restrict__ uB,
                             double *__restrict__ vB, double *__restrict__ wB, const double *__restrict__ denB,
                             const double *__restrict__ ratearea) {
    int ib = blockIdx.x * blockDim.x + threadIdx.x;
    if (ib >= nB) return;
    int ir = bndRegion[ib];
    if (regionType[ir] != CUPCFD_RTYPE_OUTLET) return;
    int i = mapMF[ib], fi = bndFaceInt[ib];
    double area = fc64[fi].w;
    double m = dm(dm(*ratearea, area), splvl[ir]);
    massFlux[i] = m;
    double faceFlux = dvd(dvd(m, denB[ib]), area);
    // EuclideanVector::normalise (EuclideanVector.cpp:100-109), length from a
    // dot product accumulated from 0 (EuclideanVector.cpp:83-98)
    double4 S = fg64[fi];
    double n0 = S.x, n1 = S.y, n2 = S.z;
    double d = 0.0;
    d = da(d, dm(n0, n0));
    d = da(d, dm(n1, n1));
    d = da(d, dm(n2, n2));
    double L = __dsqrt_rn(d);
    if (L != 0.0) {
        double sc = dvd(1.0, L);
        n0 = dm(n0, sc); n1 = dm(n1, sc); n2 = dm(n2, sc);
    }
    uB[ib] = dm(faceFlux, n0);
    vB[ib] = dm(faceFlux, n1);
    wB[ib] = dm(faceFlux, n2);
}

// Loop 5 per outlet boundary (MassKernels.ipp:495-508): massFlux scaled by
// its region's factor, optional velocity scaling.
__global__ void k_bl5_update(int nB, const int *__restrict__ bndRegion, const int *__restrict__ regionType,
                             const int *__restrict__ mapMF, double *__restrict__ massFlux,
                             const double *__restrict__ flowFact, double *__restrict__ uB, double *__restrict__ vB,
                             double *__restrict__ wB, double fact, int solveU, int solveV, int solveW) {
    int ib = blockIdx.x * blockDim.x + threadIdx.x;
    if (ib >= nB) return;
    int ir = bndRegion[ib];
    if (regionType[ir] != CUPCFD_RTYPE_OUTLET) return;
    int i = mapMF[ib];
    massFlux[i] = dm(massFlux[i], flowFact[ir]);
    if (solveU) uB[ib] = dm(uB[ib], fact);
    if (solveV) vB[ib] = dm(vB[ib], fact);
    if (solveW) wB[ib] = dm(wB[ib], fact);
}

// Loop 5's su[cell1] -= massFlux (MassKernels.ipp:510-516), per cell in
// ascending boundary id: sortedBnd lists the boundaries by (cell, id) and
// sortedCell their cells in the caller's numbering.
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
        acc = ds(acc, massFlux[mapMF[ib]]);
        any = true;
    }
    if (any) su[c] = acc;
}

// FluxMassDolfynRegionLoop (MassKernels.ipp:532-551).
__global__ void k_region_loop(int nR, const int *__restrict__ regionType, const double *__restrict__ splvl,
                              const double *__restrict__ flowRegion, const double *__restrict__ flowIn,
                              double *__restrict__ flowFact) {
    int ir = blockIdx.x * blockDim.x + threadIdx.x;
    if (ir >= nR) return;
    flowFact[ir] = regionType[ir] == CUPCFD_RTYPE_OUTLET ? dvd(-dm(splvl[ir], *flowIn), flowRegion[ir]) : 0.0;
}

}  // namespace cupcfd_gpu
