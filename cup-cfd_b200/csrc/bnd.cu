// C ABI of the boundary / region loops of the mass-flux step
// (FluxMassDolfynBoundaryLoop1-5, FluxMassDolfynRegionLoop;
// MassKernels.ipp:311-554): reference-facing calls on host buffers in the
// reference's numbering, and device-resident calls in the mesh's internal
// numbering. Kernels in kernels_bnd.cuh; the arithmetic of the reference's
// T = double instantiation, and of its T = float one in the _f32 calls (float
// host arrays, widened on the device into the double scratch arrays, which
// hold float values exactly, and narrowed back exactly).
#include <algorithm>
#include <type_traits>

#include "kernels_bnd.cuh"
#include "perm.cuh"

using namespace cupcfd_gpu;

namespace {

constexpr int BT = 256;
// scratch slots of the host-buffer calls (kept across calls)
enum BndSlot { B_MF = 40, B_SU, B_U, B_V, B_W, B_DEN, B_REG, B_REG2, B_SCAL, B_SELC, B_SELV, B_SELR, B_STAGE };

// Boundary -> face and sorted-boundary -> cell maps for the caller's numbering.
struct Maps {
    const int *face, *cell;
};
inline Maps maps_for(const cupcfd_gpu_mesh *m, bool internal) {
    return internal ? Maps{m->bndFaceInt, m->bndSortedCellInt} : Maps{m->bndFaceRef, m->bndSortedCellRef};
}

int check_mesh(const cupcfd_gpu_mesh *m, bool needGeometry) {
    CG_RETURN_IF(!m, CUPCFD_E_NULL_PTR, "boundary loop: null mesh");
    CG_RETURN_IF(!m->bndMapsOk, CUPCFD_E_INVALID_INDEX,
                 "boundary loop: the mesh's boundary ids are not a permutation of 0 .. nBoundaries-1");
    CG_RETURN_IF(needGeometry && !(m->precisions & (1 << CUPCFD_PREC_F64)), CUPCFD_E_CONFIG_INVALID_VALUE,
                 "boundary loop: the mesh was created without FP64 geometry");
    return make_device_current(m->device);
}

template <class T>
int slot(cupcfd_gpu_mesh *m, int s, size_t n, T **p) {
    void *v;
    CG_TRY(m->scratchBuf(s, std::max<size_t>(n, 1) * sizeof(T), &v));
    *p = (T *) v;
    return CUPCFD_E_SUCCESS;
}

int up(void *d, const void *h, size_t bytes, cudaStream_t st) {
    if (bytes) CG_CHECK_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st));
    return CUPCFD_E_SUCCESS;
}
int down(void *h, const void *d, size_t bytes, cudaStream_t st) {
    if (bytes) CG_CHECK_CUDA(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, st));
    return CUPCFD_E_SUCCESS;
}

// Float host arrays go through one float staging buffer, sized once per call
// for its longest array (the copies and conversions are stream-ordered, so
// every array of a call can use it in turn).
template <class H>
int reserve_stage(cupcfd_gpu_mesh *m, size_t n, float **stage) {
    *stage = nullptr;
    return std::is_same<H, float>::value ? slot(m, B_STAGE, n, stage) : CUPCFD_E_SUCCESS;
}

// Host array of the real type H -> double device array d, and back.
template <class H>
int up_real(float *stage, double *d, const H *h, size_t n, cudaStream_t st) {
    if (std::is_same<H, double>::value || n == 0) return up(d, h, sizeof(H) * n, st);
    CG_TRY(up(stage, h, sizeof(float) * n, st));
    k_convert<float, double><<<grid_for((int64_t) n, BT), BT, 0, st>>>((int64_t) n, stage, d);
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}
template <class H>
int down_real(float *stage, H *h, const double *d, size_t n, cudaStream_t st) {
    if (std::is_same<H, double>::value || n == 0) return down(h, d, sizeof(H) * n, st);
    k_convert<double, float><<<grid_for((int64_t) n, BT), BT, 0, st>>>((int64_t) n, d, stage);
    CG_LAUNCHED();
    return down(h, stage, sizeof(float) * n, st);
}

// The sum over the boundaries of region type `type`, in boundary order, of
// base[map[ib] * stride + offset], from *init (or initValue) into *out, and
// into regionAcc[region] (may be null) in the same order.
template <bool F32>
int ordered_sum(cupcfd_gpu_mesh *m, int type, const double *base, int stride, int offset, const int *map,
                const double *init, double initValue, double *out, double *regionAcc, cudaStream_t st) {
    int *cnt, *regs;
    double *vals;
    CG_TRY(slot(m, B_SELC, (size_t) m->nB / SEL_T + 2, &cnt));
    CG_TRY(slot(m, B_SELV, (size_t) m->nB, &vals));
    CG_TRY(slot(m, B_SELR, (size_t) m->nB, &regs));
    return launch_ordered_sum<1, F32>(SelArgs{m->nB, m->bndRegion, m->regionType, type}, base, stride, offset, map, init,
                                 initValue, out, regionAcc, m->nR, cnt, vals, regs, st);
}

// ---- the loops on device arrays (face arrays indexed through mp.face, cell
// arrays through mp.cell); every scalar in device memory ----
template <bool F32>
int run_loop1(cupcfd_gpu_mesh *m, Maps mp, const double *mf, double *flowin, cudaStream_t st) {
    return ordered_sum<F32>(m, CUPCFD_RTYPE_INLET, mf, 1, 0, mp.face, nullptr, 0.0, flowin, nullptr, st);
}

template <bool F32>
int run_loop2(cupcfd_gpu_mesh *m, Maps mp, const double *mf, double *flowRegion, double *flowout, cudaStream_t st) {
    return ordered_sum<F32>(m, CUPCFD_RTYPE_OUTLET, mf, 1, 0, mp.face, nullptr, 0.0, flowout, flowRegion, st);
}

template <bool F32>
int run_loop3(cupcfd_gpu_mesh *m, const double *flowin, double *ratearea, double *areaout, cudaStream_t st) {
    // face areas from the internal {xf, yf, zf, area} records
    CG_TRY(ordered_sum<F32>(m, CUPCFD_RTYPE_OUTLET, (const double *) m->fc64, 4, 3, m->bndFaceInt, nullptr, 0.0, areaout,
                       nullptr, st));
    k_bl_ratearea<F32><<<1, 1, 0, st>>>(flowin, areaout, ratearea);
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}

template <bool F32>
int run_loop4(cupcfd_gpu_mesh *m, Maps mp, double *mf, double *uB, double *vB, double *wB, const double *denB,
              const double *ratearea, double *flowout, cudaStream_t st) {
    if (m->nB > 0) {
        k_bl4_update<F32><<<grid_for(m->nB, BT), BT, 0, st>>>(m->nB, m->bndRegion, m->regionType, m->regionSplvl, mp.face,
                                                         m->bndFaceInt, m->fg64, m->fc64, mf, uB, vB, wB, denB, ratearea);
        CG_LAUNCHED();
    }
    return ordered_sum<F32>(m, CUPCFD_RTYPE_OUTLET, mf, 1, 0, mp.face, nullptr, 0.0, flowout, nullptr, st);
}

template <bool F32>
int run_loop5(cupcfd_gpu_mesh *m, Maps mp, double *mf, double *su, double *uB, double *vB, double *wB, double fact,
              int solveU, int solveV, int solveW, const double *flowFact, double *flowout2, cudaStream_t st) {
    if (m->nB > 0) {
        k_bl5_update<F32><<<grid_for(m->nB, BT), BT, 0, st>>>(m->nB, m->bndRegion, m->regionType, mp.face, mf, flowFact, uB,
                                                         vB, wB, fact, solveU, solveV, solveW);
        CG_LAUNCHED();
        k_bl5_su<F32><<<grid_for(m->nB, BT), BT, 0, st>>>(m->nB, m->bndSorted, mp.cell, m->bndRegion, m->regionType, mp.face,
                                                     mf, su);
        CG_LAUNCHED();
    }
    // *flowout2 is not reset (MassKernels.ipp:457-521): the sum starts from its value
    return ordered_sum<F32>(m, CUPCFD_RTYPE_OUTLET, mf, 1, 0, mp.face, flowout2, 0.0, flowout2, nullptr, st);
}

template <bool F32>
int run_region_loop(cupcfd_gpu_mesh *m, double *flowFact, const double *flowRegion, const double *flowIn,
                    cudaStream_t st) {
    k_region_loop<F32><<<grid_for(m->nR, BT), BT, 0, st>>>(m->nR, m->regionType, m->regionSplvl, flowRegion, flowIn,
                                                     flowFact);
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}

inline cudaStream_t as_stream(void *s) { return (cudaStream_t) s; }

}  // namespace

// ---------------------------------------------------------------------------
// region split levels
// ---------------------------------------------------------------------------
extern "C" int cupcfd_gpu_mesh_set_region_split(cupcfd_gpu_mesh *m, int32_t nRegions, const double *splvl) {
    clear_error();
    CG_RETURN_IF(!m || !splvl, CUPCFD_E_NULL_PTR, "set_region_split: null argument");
    CG_RETURN_IF(nRegions != m->nR, CUPCFD_E_ARRAY_SIZE_MISMATCH, "set_region_split: nRegions differs from the mesh's");
    CG_TRY(make_device_current(m->device));
    CG_CHECK_CUDA(cudaMemcpyAsync(m->regionSplvl, splvl, sizeof(double) * nRegions, cudaMemcpyHostToDevice, m->stream));
    CG_CHECK_CUDA(cudaStreamSynchronize(m->stream));
    return CUPCFD_E_SUCCESS;
}

// ---------------------------------------------------------------------------
// reference-facing calls: host buffers, reference numbering. Arrays shorter
// than the mesh needs return E_INVALID_INDEX, as the reference's DEBUG build
// does (MassKernels.ipp:326-330, 354-361, 420-436, 477-493, 511-515, 535-542).
// ---------------------------------------------------------------------------
namespace {

// The host-buffer calls for host arrays of the real type H; F32 when H is
// float (the reference's T = float instantiation).
template <class H>
int host_loop1(cupcfd_gpu_mesh *m, const H *massFlux, int32_t nMassFlux, H *flowin) {
    constexpr bool F32 = std::is_same<H, float>::value;
    clear_error();
    CG_TRY(check_mesh(m, false));
    CG_RETURN_IF(!massFlux || !flowin, CUPCFD_E_NULL_PTR, "boundary_loop1: null argument");
    CG_RETURN_IF(nMassFlux < m->nF, CUPCFD_E_INVALID_INDEX, "boundary_loop1: massFlux shorter than nFaces");
    cudaStream_t st = m->stream;
    double *mf, *sc;
    float *stage;
    CG_TRY(slot(m, B_MF, m->nF, &mf));
    CG_TRY(slot(m, B_SCAL, 4, &sc));
    CG_TRY(reserve_stage<H>(m, m->nF, &stage));
    CG_TRY(up_real(stage, mf, massFlux, m->nF, st));
    CG_TRY(run_loop1<F32>(m, maps_for(m, false), mf, sc, st));
    double r;
    CG_TRY(down(&r, sc, sizeof(double), st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    *flowin = (H) r;
    return CUPCFD_E_SUCCESS;
}

template <class H>
int host_loop2(cupcfd_gpu_mesh *m, const H *massFlux, int32_t nMassFlux, H *flowRegion, int32_t nFlowRegion,
               H *flowout) {
    constexpr bool F32 = std::is_same<H, float>::value;
    clear_error();
    CG_TRY(check_mesh(m, false));
    CG_RETURN_IF(!massFlux || !flowRegion || !flowout, CUPCFD_E_NULL_PTR, "boundary_loop2: null argument");
    CG_RETURN_IF(nMassFlux < m->nF || nFlowRegion < m->nR, CUPCFD_E_INVALID_INDEX, "boundary_loop2: array too short");
    cudaStream_t st = m->stream;
    double *mf, *fr, *sc;
    float *stage;
    CG_TRY(slot(m, B_MF, m->nF, &mf));
    CG_TRY(slot(m, B_REG, m->nR, &fr));
    CG_TRY(slot(m, B_SCAL, 4, &sc));
    CG_TRY(reserve_stage<H>(m, std::max(m->nF, m->nR), &stage));
    CG_TRY(up_real(stage, mf, massFlux, m->nF, st));
    CG_TRY(up_real(stage, fr, flowRegion, m->nR, st));
    CG_TRY(run_loop2<F32>(m, maps_for(m, false), mf, fr, sc, st));
    CG_TRY(down_real(stage, flowRegion, fr, m->nR, st));
    double r;
    CG_TRY(down(&r, sc, sizeof(double), st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    *flowout = (H) r;
    return CUPCFD_E_SUCCESS;
}

template <class H>
int host_loop3(cupcfd_gpu_mesh *m, H flowin, H *ratearea) {
    constexpr bool F32 = std::is_same<H, float>::value;
    clear_error();
    CG_TRY(check_mesh(m, true));
    CG_RETURN_IF(!ratearea, CUPCFD_E_NULL_PTR, "boundary_loop3: null argument");
    cudaStream_t st = m->stream;
    double *sc;
    CG_TRY(slot(m, B_SCAL, 4, &sc));
    const double fin = (double) flowin;
    CG_TRY(up(sc, &fin, sizeof(double), st));
    CG_TRY(run_loop3<F32>(m, sc, sc + 1, sc + 2, st));
    double r;
    CG_TRY(down(&r, sc + 1, sizeof(double), st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    *ratearea = (H) r;
    return CUPCFD_E_SUCCESS;
}

template <class H>
int host_loop4(cupcfd_gpu_mesh *m, H *massFlux, int32_t nMassFlux, H *uBoundary, int32_t nUBoundary, H *vBoundary,
               int32_t nVBoundary, H *wBoundary, int32_t nWBoundary, const H *denBoundary, int32_t nDenBoundary,
               H ratearea, H *flowout) {
    constexpr bool F32 = std::is_same<H, float>::value;
    clear_error();
    CG_TRY(check_mesh(m, true));
    CG_RETURN_IF(!massFlux || !uBoundary || !vBoundary || !wBoundary || !denBoundary || !flowout, CUPCFD_E_NULL_PTR,
                 "boundary_loop4: null argument");
    CG_RETURN_IF(nMassFlux < m->nF || nUBoundary < m->nB || nVBoundary < m->nB || nWBoundary < m->nB ||
                     nDenBoundary < m->nB,
                 CUPCFD_E_INVALID_INDEX, "boundary_loop4: array too short");
    cudaStream_t st = m->stream;
    const size_t nb = m->nB;
    double *mf, *u, *v, *w, *den, *sc;
    float *stage;
    CG_TRY(slot(m, B_MF, m->nF, &mf));
    CG_TRY(slot(m, B_U, nb, &u));
    CG_TRY(slot(m, B_V, nb, &v));
    CG_TRY(slot(m, B_W, nb, &w));
    CG_TRY(slot(m, B_DEN, nb, &den));
    CG_TRY(slot(m, B_SCAL, 4, &sc));
    CG_TRY(reserve_stage<H>(m, std::max((size_t) m->nF, nb), &stage));
    CG_TRY(up_real(stage, mf, massFlux, m->nF, st));
    CG_TRY(up_real(stage, u, uBoundary, nb, st));
    CG_TRY(up_real(stage, v, vBoundary, nb, st));
    CG_TRY(up_real(stage, w, wBoundary, nb, st));
    CG_TRY(up_real(stage, den, denBoundary, nb, st));
    const double ra = (double) ratearea;
    CG_TRY(up(sc, &ra, sizeof(double), st));
    CG_TRY(run_loop4<F32>(m, maps_for(m, false), mf, u, v, w, den, sc, sc + 1, st));
    CG_TRY(down_real(stage, massFlux, mf, m->nF, st));
    CG_TRY(down_real(stage, uBoundary, u, nb, st));
    CG_TRY(down_real(stage, vBoundary, v, nb, st));
    CG_TRY(down_real(stage, wBoundary, w, nb, st));
    double r;
    CG_TRY(down(&r, sc + 1, sizeof(double), st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    *flowout = (H) r;
    return CUPCFD_E_SUCCESS;
}

template <class H>
int host_loop5(cupcfd_gpu_mesh *m, H *massFlux, int32_t nMassFlux, H *su, int32_t nSu, H *uBoundary,
               int32_t nUBoundary, H *vBoundary, int32_t nVBoundary, H *wBoundary, int32_t nWBoundary, H fact,
               int32_t solveU, int32_t solveV, int32_t solveW, const H *flowFact, int32_t nFlowFact, H *flowout2) {
    constexpr bool F32 = std::is_same<H, float>::value;
    clear_error();
    CG_TRY(check_mesh(m, false));
    CG_RETURN_IF(!massFlux || !su || !uBoundary || !vBoundary || !wBoundary || !flowFact || !flowout2,
                 CUPCFD_E_NULL_PTR, "boundary_loop5: null argument");
    CG_RETURN_IF(nMassFlux < m->nF || nSu < m->nC || nUBoundary < m->nB || nVBoundary < m->nB || nWBoundary < m->nB ||
                     nFlowFact < m->nR,
                 CUPCFD_E_INVALID_INDEX, "boundary_loop5: array too short");
    cudaStream_t st = m->stream;
    const size_t nb = m->nB;
    double *mf, *suD, *u, *v, *w, *ff, *sc;
    float *stage;
    CG_TRY(slot(m, B_MF, m->nF, &mf));
    CG_TRY(slot(m, B_SU, m->nC, &suD));
    CG_TRY(slot(m, B_U, nb, &u));
    CG_TRY(slot(m, B_V, nb, &v));
    CG_TRY(slot(m, B_W, nb, &w));
    CG_TRY(slot(m, B_REG, m->nR, &ff));
    CG_TRY(slot(m, B_SCAL, 4, &sc));
    CG_TRY(reserve_stage<H>(m, std::max({(size_t) m->nF, (size_t) m->nC, nb, (size_t) m->nR}), &stage));
    CG_TRY(up_real(stage, mf, massFlux, m->nF, st));
    CG_TRY(up_real(stage, suD, su, m->nC, st));
    CG_TRY(up_real(stage, u, uBoundary, nb, st));
    CG_TRY(up_real(stage, v, vBoundary, nb, st));
    CG_TRY(up_real(stage, w, wBoundary, nb, st));
    CG_TRY(up_real(stage, ff, flowFact, m->nR, st));
    const double f2 = (double) *flowout2;
    CG_TRY(up(sc, &f2, sizeof(double), st));
    CG_TRY(run_loop5<F32>(m, maps_for(m, false), mf, suD, u, v, w, (double) fact, solveU != 0, solveV != 0,
                          solveW != 0, ff, sc, st));
    CG_TRY(down_real(stage, massFlux, mf, m->nF, st));
    CG_TRY(down_real(stage, su, suD, m->nC, st));
    CG_TRY(down_real(stage, uBoundary, u, nb, st));
    CG_TRY(down_real(stage, vBoundary, v, nb, st));
    CG_TRY(down_real(stage, wBoundary, w, nb, st));
    double r;
    CG_TRY(down(&r, sc, sizeof(double), st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    *flowout2 = (H) r;
    return CUPCFD_E_SUCCESS;
}

template <class H>
int host_region_loop(cupcfd_gpu_mesh *m, H *flowFact, int32_t nFlowFact, const H *flowRegion, int32_t nFlowRegion,
                     H flowIn) {
    constexpr bool F32 = std::is_same<H, float>::value;
    clear_error();
    CG_TRY(check_mesh(m, false));
    CG_RETURN_IF(!flowFact || !flowRegion, CUPCFD_E_NULL_PTR, "region_loop: null argument");
    CG_RETURN_IF(nFlowFact < m->nR || nFlowRegion < m->nR, CUPCFD_E_INVALID_INDEX, "region_loop: array too short");
    cudaStream_t st = m->stream;
    double *ff, *fr, *sc;
    float *stage;
    CG_TRY(slot(m, B_REG, m->nR, &ff));
    CG_TRY(slot(m, B_REG2, m->nR, &fr));
    CG_TRY(slot(m, B_SCAL, 4, &sc));
    CG_TRY(reserve_stage<H>(m, m->nR, &stage));
    CG_TRY(up_real(stage, fr, flowRegion, m->nR, st));
    const double fin = (double) flowIn;
    CG_TRY(up(sc, &fin, sizeof(double), st));
    CG_TRY(run_region_loop<F32>(m, ff, fr, sc, st));
    CG_TRY(down_real(stage, flowFact, ff, m->nR, st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    return CUPCFD_E_SUCCESS;
}

}  // namespace

#define CG_BND_HOST_ENTRIES(H, SUFFIX)                                                                                  \
    extern "C" int cupcfd_gpu_flux_mass_dolfyn_boundary_loop1##SUFFIX(cupcfd_gpu_mesh *m, const H *massFlux,           \
                                                                      int32_t nMassFlux, H *flowin) {                  \
        return host_loop1<H>(m, massFlux, nMassFlux, flowin);                                                          \
    }                                                                                                                  \
    extern "C" int cupcfd_gpu_flux_mass_dolfyn_boundary_loop2##SUFFIX(cupcfd_gpu_mesh *m, const H *massFlux,           \
                                                                      int32_t nMassFlux, H *flowRegion,                \
                                                                      int32_t nFlowRegion, H *flowout) {               \
        return host_loop2<H>(m, massFlux, nMassFlux, flowRegion, nFlowRegion, flowout);                                \
    }                                                                                                                  \
    extern "C" int cupcfd_gpu_flux_mass_dolfyn_boundary_loop3##SUFFIX(cupcfd_gpu_mesh *m, H flowin, H *ratearea) {     \
        return host_loop3<H>(m, flowin, ratearea);                                                                     \
    }                                                                                                                  \
    extern "C" int cupcfd_gpu_flux_mass_dolfyn_boundary_loop4##SUFFIX(                                                 \
        cupcfd_gpu_mesh *m, H *massFlux, int32_t nMassFlux, H *uBoundary, int32_t nUBoundary, H *vBoundary,            \
        int32_t nVBoundary, H *wBoundary, int32_t nWBoundary, const H *denBoundary, int32_t nDenBoundary, H ratearea,  \
        H *flowout) {                                                                                                  \
        return host_loop4<H>(m, massFlux, nMassFlux, uBoundary, nUBoundary, vBoundary, nVBoundary, wBoundary,          \
                             nWBoundary, denBoundary, nDenBoundary, ratearea, flowout);                                \
    }                                                                                                                  \
    extern "C" int cupcfd_gpu_flux_mass_dolfyn_boundary_loop5##SUFFIX(                                                 \
        cupcfd_gpu_mesh *m, H *massFlux, int32_t nMassFlux, H *su, int32_t nSu, H *uBoundary, int32_t nUBoundary,      \
        H *vBoundary, int32_t nVBoundary, H *wBoundary, int32_t nWBoundary, H fact, int32_t solveU, int32_t solveV,    \
        int32_t solveW, const H *flowFact, int32_t nFlowFact, H *flowout2) {                                           \
        return host_loop5<H>(m, massFlux, nMassFlux, su, nSu, uBoundary, nUBoundary, vBoundary, nVBoundary, wBoundary, \
                             nWBoundary, fact, solveU, solveV, solveW, flowFact, nFlowFact, flowout2);                 \
    }                                                                                                                  \
    extern "C" int cupcfd_gpu_flux_mass_dolfyn_region_loop##SUFFIX(cupcfd_gpu_mesh *m, H *flowFact, int32_t nFlowFact, \
                                                                   const H *flowRegion, int32_t nFlowRegion,           \
                                                                   H flowIn) {                                         \
        return host_region_loop<H>(m, flowFact, nFlowFact, flowRegion, nFlowRegion, flowIn);                           \
    }

CG_BND_HOST_ENTRIES(double, )
CG_BND_HOST_ENTRIES(float, _f32)
#undef CG_BND_HOST_ENTRIES

// ---------------------------------------------------------------------------
// device-resident calls: device pointers, internal face and cell numbering,
// boundary and region arrays by reference id, scalars in device memory,
// stream-ordered (no synchronisation)
// ---------------------------------------------------------------------------
extern "C" int cupcfd_gpu_dev_boundary_loop1(cupcfd_gpu_mesh *m, const double *massFlux, double *flowin, void *stream) {
    clear_error();
    CG_TRY(check_mesh(m, false));
    CG_RETURN_IF(!massFlux || !flowin, CUPCFD_E_NULL_PTR, "dev_boundary_loop1: null argument");
    return run_loop1<false>(m, maps_for(m, true), massFlux, flowin, as_stream(stream));
}

extern "C" int cupcfd_gpu_dev_boundary_loop2(cupcfd_gpu_mesh *m, const double *massFlux, double *flowRegion,
                                             double *flowout, void *stream) {
    clear_error();
    CG_TRY(check_mesh(m, false));
    CG_RETURN_IF(!massFlux || !flowRegion || !flowout, CUPCFD_E_NULL_PTR, "dev_boundary_loop2: null argument");
    return run_loop2<false>(m, maps_for(m, true), massFlux, flowRegion, flowout, as_stream(stream));
}

extern "C" int cupcfd_gpu_dev_boundary_loop3(cupcfd_gpu_mesh *m, const double *flowin, double *ratearea, void *stream) {
    clear_error();
    CG_TRY(check_mesh(m, true));
    CG_RETURN_IF(!flowin || !ratearea, CUPCFD_E_NULL_PTR, "dev_boundary_loop3: null argument");
    double *sc;
    CG_TRY(slot(m, B_SCAL + 1, 1, &sc));  // the outlet area
    return run_loop3<false>(m, flowin, ratearea, sc, as_stream(stream));
}

extern "C" int cupcfd_gpu_dev_boundary_loop4(cupcfd_gpu_mesh *m, double *massFlux, double *uBoundary,
                                             double *vBoundary, double *wBoundary, const double *denBoundary,
                                             const double *ratearea, double *flowout, void *stream) {
    clear_error();
    CG_TRY(check_mesh(m, true));
    CG_RETURN_IF(!massFlux || !uBoundary || !vBoundary || !wBoundary || !denBoundary || !ratearea || !flowout,
                 CUPCFD_E_NULL_PTR, "dev_boundary_loop4: null argument");
    return run_loop4<false>(m, maps_for(m, true), massFlux, uBoundary, vBoundary, wBoundary, denBoundary, ratearea, flowout,
                     as_stream(stream));
}

extern "C" int cupcfd_gpu_dev_boundary_loop5(cupcfd_gpu_mesh *m, double *massFlux, double *su, double *uBoundary,
                                             double *vBoundary, double *wBoundary, double fact, int32_t solveU,
                                             int32_t solveV, int32_t solveW, const double *flowFact, double *flowout2,
                                             void *stream) {
    clear_error();
    CG_TRY(check_mesh(m, false));
    CG_RETURN_IF(!massFlux || !su || !uBoundary || !vBoundary || !wBoundary || !flowFact || !flowout2,
                 CUPCFD_E_NULL_PTR, "dev_boundary_loop5: null argument");
    return run_loop5<false>(m, maps_for(m, true), massFlux, su, uBoundary, vBoundary, wBoundary, fact, solveU != 0,
                     solveV != 0, solveW != 0, flowFact, flowout2, as_stream(stream));
}

extern "C" int cupcfd_gpu_dev_region_loop(cupcfd_gpu_mesh *m, double *flowFact, const double *flowRegion,
                                          const double *flowIn, void *stream) {
    clear_error();
    CG_TRY(check_mesh(m, false));
    CG_RETURN_IF(!flowFact || !flowRegion || !flowIn, CUPCFD_E_NULL_PTR, "dev_region_loop: null argument");
    return run_region_loop<false>(m, flowFact, flowRegion, flowIn, as_stream(stream));
}
