// cupcfd_gpu/fvm.hpp - C++ drop-in for CUP-CFD's face-loop kernels on B200.
//
// Same names and parameter lists as the reference's templates
//   cupcfd::fvm::GradientPhiGaussDolfyn  (include/fvm/implementation/component/GradientKernels.h:48-54)
//   cupcfd::fvm::FluxMassDolfynFaceLoop  (include/fvm/implementation/component/MassKernels.h:48-81),
//                                        for T = double and T = float meshes
//   cupcfd::fvm::FluxMassDolfynBoundaryLoop1-5, FluxMassDolfynRegionLoop (MassKernels.h:90-171),
//                                        for T = double and T = float
//   cupcfd::fvm::FluxUVWDolfynFaceLoop1, FluxUVWDolfynRegionLoop1, FluxUVWDolfynBndsLoop1
//                                        (include/fvm/implementation/component/UVWKernels.h:45-92),
//                                        face loop for T = double and T = float
// in namespace cupcfd::fvm::gpu, so a call site switches by namespace only:
//
//   status = cupcfd::fvm::gpu::GradientPhiGaussDolfyn(mesh, nGradient, phiCell, nPhiCell,
//                                                     phiBoundary, nPhiBoundary,
//                                                     dPhidxCell, nDPhidxCell, dPhidxoCell, nDPhidxoCell);
//
// The mesh is any object with the reference mesh getters (a CupCfdSoAMesh,
// a CupCfdAoSMesh or the UnstructuredMeshInterface<M,I,T,L> they derive
// from). On the first call for a mesh object its arrays are read through
// those getters once and uploaded (cupcfd_gpu_mesh_create); later calls
// reuse the device mesh. Call release(mesh) before the host mesh changes or
// goes away. Field arrays are the caller's host arrays, as in the
// reference; the vptr-carrying EuclideanVector<T,3> arrays are passed as
// strided views and only their components are written.
//
// Return type: cupcfd::error::eCodes when the reference's Error.h has been
// included first, else int with the same values.
#pragma once

#include <cstddef>
#include <cstdint>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "cupcfd_gpu.h"

namespace cupcfd {
namespace fvm {
namespace gpu {

#ifdef CUPCFD_ERROR_INCLUDE_H
using ecode_t = cupcfd::error::eCodes;
#else
using ecode_t = int;
#endif

// Precision and numbering used for meshes attached implicitly. Change before
// the first call on a mesh (or release it and attach again).
struct Settings {
    int precision = CUPCFD_PREC_F64;  // bit-identical to the reference for T = double (and, for the
                                      // gradient with T = float, taken as CUPCFD_PREC_F32REF: the
                                      // float instantiation's own arithmetic)
    int sign_mode = CUPCFD_SIGN_REFERENCE;
    int order = CUPCFD_ORDER_MORTON;
    int device = -1;
};
inline Settings &settings() {
    static Settings s;
    return s;
}

namespace detail {

template <class V>
inline cupcfd_vec3_view view_of(const V *a) {
    // component 0 of element 0 relative to the element start: the vptr slot
    // (8 bytes) for the reference's EuclideanVector/EuclideanPoint
    cupcfd_vec3_view v;
    v.base = a;
    v.stride = (int32_t) sizeof(V);
    v.offset = a ? (int32_t) ((const char *) &a->cmp[0] - (const char *) a) : 0;
    return v;
}

struct Registry {
    std::mutex mu;
    std::unordered_map<const void *, cupcfd_gpu_mesh *> meshes;
    static Registry &get() {
        static Registry r;
        return r;
    }
};

// Reads a mesh through its getters into packed arrays and uploads it.
template <class Mesh>
int upload(Mesh &mesh, cupcfd_gpu_mesh **out) {
    using T = decltype(mesh.getFaceLambda(0));
    const int nF = (int) mesh.properties.lFaces;
    const int nC = (int) mesh.properties.lTCells;
    const int nB = (int) mesh.properties.lBoundaries;
    const int nR = (int) mesh.properties.lRegions;
    std::vector<int32_t> c1(nF), c2(nF), bnd(nF);
    std::vector<T> lam(nF), area(nF), S(3 * (size_t) nF), xf(3 * (size_t) nF), xp(3 * (size_t) nF),
        xn(3 * (size_t) nF), cc(3 * (size_t) nC), vol(nC);
    bool xzero = true;
    for (int f = 0; f < nF; f++) {
        c1[f] = (int32_t) mesh.getFaceCell1ID(f);
        c2[f] = (int32_t) mesh.getFaceCell2ID(f);
        bool isB = mesh.getFaceIsBoundary(f);
        bnd[f] = isB ? (int32_t) mesh.getFaceBoundaryID(f) : -1;
        lam[f] = mesh.getFaceLambda(f);
        area[f] = mesh.getFaceArea(f);
        auto n = mesh.getFaceNorm(f);
        auto x = mesh.getFaceCenter(f);
        auto a = mesh.getFaceXpac(f);
        auto b = mesh.getFaceXnac(f);
        for (int d = 0; d < 3; d++) {
            S[3 * f + d] = n.cmp[d];
            xf[3 * f + d] = x.cmp[d];
            xp[3 * f + d] = a.cmp[d];
            xn[3 * f + d] = b.cmp[d];
            xzero = xzero && a.cmp[d] == T(0) && b.cmp[d] == T(0);
        }
    }
    for (int c = 0; c < nC; c++) {
        auto x = mesh.getCellCenter(c);
        for (int d = 0; d < 3; d++) cc[3 * c + d] = x.cmp[d];
        vol[c] = mesh.getCellVolume(c);
    }
    cupcfd_mesh_view v;
    v.nCells = nC;
    v.nFaces = nF;
    v.nBoundaries = nB;
    v.real_size = (int32_t) sizeof(T);
    v.faceCell1 = c1.data();
    v.faceCell2 = c2.data();
    v.faceBnd = bnd.data();
    v.faceLambda = lam.data();
    v.faceArea = area.data();
    v.faceNorm = {S.data(), (int32_t) (3 * sizeof(T)), 0};
    v.faceCenter = {xf.data(), (int32_t) (3 * sizeof(T)), 0};
    v.faceXpac = {xzero ? nullptr : xp.data(), (int32_t) (3 * sizeof(T)), 0};
    v.faceXnac = {xzero ? nullptr : xn.data(), (int32_t) (3 * sizeof(T)), 0};
    v.cellCenter = {cc.data(), (int32_t) (3 * sizeof(T)), 0};
    v.cellVolume = vol.data();
    cupcfd_mesh_options o;
    o.order = settings().order;
    o.precisions = (1 << CUPCFD_PREC_F64) | (1 << CUPCFD_PREC_F32C);
    o.device = settings().device;
    int rc = cupcfd_gpu_mesh_create(&v, &o, out);
    if (rc != CUPCFD_E_SUCCESS) return rc;
    // boundary regions (UnstructuredMeshInterface.h:1306-1949)
    if (nR > 0) {
        std::vector<int32_t> rt(nR), br(nB);
        std::vector<double> uvw(3 * (size_t) nR), den(nR);
        for (int r = 0; r < nR; r++) {
            rt[r] = (int32_t) mesh.getRegionType(r);
            auto u = mesh.getRegionUVW(r);
            for (int d = 0; d < 3; d++) uvw[3 * r + d] = (double) u.cmp[d];
            den[r] = (double) mesh.getRegionDen(r);
        }
        for (int b = 0; b < nB; b++) br[b] = (int32_t) mesh.getBoundaryRegionID(b);
        rc = cupcfd_gpu_mesh_set_regions(*out, nR, rt.data(), uvw.data(), den.data(), br.data(), nB);
        if (rc == CUPCFD_E_SUCCESS) {
            // split levels (getRegionSplvl), read by the outlet boundary loops
            std::vector<double> sp(nR);
            for (int r = 0; r < nR; r++) sp[r] = (double) mesh.getRegionSplvl(r);
            rc = cupcfd_gpu_mesh_set_region_split(*out, nR, sp.data());
        }
    }
    // momentum-loop geometry (getFaceRLencos, getBoundaryDistance); zero on
    // every MeshSource-built mesh, uploaded only when some entry is not
    if (rc == CUPCFD_E_SUCCESS) {
        std::vector<double> rl(nF), bd(nB);
        bool rlAny = false, bdAny = false;
        for (int f = 0; f < nF; f++) rlAny |= (rl[f] = (double) mesh.getFaceRLencos(f)) != 0.0;
        for (int b = 0; b < nB; b++) bdAny |= (bd[b] = (double) mesh.getBoundaryDistance(b)) != 0.0;
        if (rlAny) rc = cupcfd_gpu_mesh_set_face_rlencos(*out, rl.data(), nF);
        if (rc == CUPCFD_E_SUCCESS && bdAny) rc = cupcfd_gpu_mesh_set_boundary_distance(*out, bd.data(), nB);
    }
    if (rc != CUPCFD_E_SUCCESS && *out) {
        cupcfd_gpu_mesh_destroy(*out);
        *out = nullptr;
    }
    return rc;
}

// Boundary shears and region force tangents between the host mesh (the
// reference's state, get/setBoundaryShear, get/setRegionForceTangent) and the
// device mesh. toHost: only boundaries of `onlyType` (-1: all) are written.
template <class Mesh>
int sync_shear(Mesh &mesh, cupcfd_gpu_mesh *m, bool toHost, int onlyType) {
    const int nB = (int) mesh.properties.lBoundaries;
    std::vector<double> sh(3 * (size_t) nB);
    if (!toHost)
        for (int b = 0; b < nB; b++) {
            auto v = mesh.getBoundaryShear(b);
            for (int d = 0; d < 3; d++) sh[3 * b + d] = (double) v.cmp[d];
        }
    int rc = cupcfd_gpu_mesh_boundary_shear(m, toHost ? nullptr : sh.data(), toHost ? sh.data() : nullptr, nB);
    if (rc != CUPCFD_E_SUCCESS || !toHost) return rc;
    for (int b = 0; b < nB; b++) {
        if (onlyType >= 0 && (int) mesh.getRegionType(mesh.getBoundaryRegionID(b)) != onlyType) continue;
        auto v = mesh.getBoundaryShear(b);
        for (int d = 0; d < 3; d++) v.cmp[d] = sh[3 * b + d];
        mesh.setBoundaryShear(b, v);
    }
    return rc;
}

template <class Mesh>
int sync_force_tangent(Mesh &mesh, cupcfd_gpu_mesh *m, bool toHost) {
    const int nR = (int) mesh.properties.lRegions;
    std::vector<double> ft(3 * (size_t) nR);
    if (!toHost)
        for (int r = 0; r < nR; r++) {
            auto v = mesh.getRegionForceTangent(r);
            for (int d = 0; d < 3; d++) ft[3 * r + d] = (double) v.cmp[d];
        }
    int rc = cupcfd_gpu_mesh_region_force_tangent(m, toHost ? nullptr : ft.data(), toHost ? ft.data() : nullptr, nR);
    if (rc != CUPCFD_E_SUCCESS || !toHost) return rc;
    for (int r = 0; r < nR; r++) {
        auto v = mesh.getRegionForceTangent(r);
        for (int d = 0; d < 3; d++) v.cmp[d] = ft[3 * r + d];
        mesh.setRegionForceTangent(r, v);
    }
    return rc;
}

}  // namespace detail

// Device mesh of a host mesh object (uploaded on first use).
template <class Mesh>
int attach(Mesh &mesh, cupcfd_gpu_mesh **out) {
    auto &r = detail::Registry::get();
    std::lock_guard<std::mutex> g(r.mu);
    auto it = r.meshes.find(&mesh);
    if (it != r.meshes.end()) {
        *out = it->second;
        return CUPCFD_E_SUCCESS;
    }
    int rc = detail::upload(mesh, out);
    if (rc == CUPCFD_E_SUCCESS) r.meshes[&mesh] = *out;
    return rc;
}

// Frees the device copy of a host mesh (no-op if none).
template <class Mesh>
void release(Mesh &mesh) {
    auto &r = detail::Registry::get();
    std::lock_guard<std::mutex> g(r.mu);
    auto it = r.meshes.find(&mesh);
    if (it != r.meshes.end()) {
        cupcfd_gpu_mesh_destroy(it->second);
        r.meshes.erase(it);
    }
}

// GradientPhiGaussDolfyn (GradientKernels.h:48-54)
template <class Mesh, class I, class T, class Vec>
ecode_t GradientPhiGaussDolfyn(Mesh &mesh, I nGradient, T *phiCell, I nPhiCell, T *phiBoundary, I nPhiBoundary,
                               Vec *dPhidxCell, I nDPhidxCell, Vec *dPhidxoCell, I nDPhidxoCell) {
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    cupcfd_vec3_view v = detail::view_of(dPhidxCell), vo = detail::view_of(dPhidxoCell);
    rc = cupcfd_gpu_gradient_phi_gauss_dolfyn(m, (int32_t) nGradient, phiCell, (int32_t) nPhiCell, phiBoundary,
                                              (int32_t) nPhiBoundary, dPhidxCell, (int32_t) nDPhidxCell, v.stride,
                                              v.offset, dPhidxoCell, (int32_t) nDPhidxoCell, vo.stride, vo.offset,
                                              (int32_t) sizeof(T),
                                              sizeof(T) == 4 && settings().precision == CUPCFD_PREC_F64
                                                  ? CUPCFD_PREC_F32REF
                                                  : settings().precision,
                                              settings().sign_mode);
    return (ecode_t) rc;
}

// FluxMassDolfynFaceLoop (MassKernels.h:48-81), T = double
template <class Mesh, class I, class Vec>
ecode_t FluxMassDolfynFaceLoop(Mesh &mesh, Vec *dudx, I nDudx, Vec *dvdx, I nDvdx, Vec *dwdx, I nDwdx, Vec *dpdx,
                               I nDpdx, double *denCell, I nDenCell, double *denBoundary, I nDenBoundary,
                               double *uCell, I nUCell, double *vCell, I nVCell, double *wCell, I nWCell,
                               double *massFlux, I nMassFlux, double *p, I nP, double *ar, I nAr, double *su, I nSu,
                               double *rface, I nRFace, double small, I *icinl, I *icout, I *icsym, I *icwal,
                               bool solveTurbEnergy, bool solveTurbDiss, bool solveVisc, bool solveEnthalpy,
                               double *teCell, I nTeCell, double *teBoundary, I nTeBoundary, double *edCell,
                               I nEdCell, double *edBoundary, I nEdBoundary, double *viseffCell, I nViseffCell,
                               double *viseffBoundary, I nViseffBoundary, double *tCell, I nTCell, double *tBoundary,
                               I nTBoundary) {
    static_assert(sizeof(I) == 4, "int32 indices");
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    rc = cupcfd_gpu_flux_mass_dolfyn_face_loop(
        m, detail::view_of(dudx), nDudx, detail::view_of(dvdx), nDvdx, detail::view_of(dwdx), nDwdx,
        detail::view_of(dpdx), nDpdx, denCell, nDenCell, denBoundary, nDenBoundary, uCell, nUCell, vCell, nVCell,
        wCell, nWCell, massFlux, nMassFlux, p, nP, ar, nAr, su, nSu, rface, nRFace, small, (int32_t *) icinl,
        (int32_t *) icout, (int32_t *) icsym, (int32_t *) icwal, solveTurbEnergy, solveTurbDiss, solveVisc,
        solveEnthalpy, teCell, nTeCell, teBoundary, nTeBoundary, edCell, nEdCell, edBoundary, nEdBoundary,
        viseffCell, nViseffCell, viseffBoundary, nViseffBoundary, tCell, nTCell, tBoundary, nTBoundary);
    return (ecode_t) rc;
}

// FluxMassDolfynFaceLoop, T = float: the reference's float instantiation
// (BenchmarkKernels.cpp:1134-1138) on a CupCfdSoAMesh<int,float,int>, with
// its arithmetic (cupcfd_gpu_flux_mass_dolfyn_face_loop_f32)
template <class Mesh, class I, class Vec>
ecode_t FluxMassDolfynFaceLoop(Mesh &mesh, Vec *dudx, I nDudx, Vec *dvdx, I nDvdx, Vec *dwdx, I nDwdx, Vec *dpdx,
                               I nDpdx, float *denCell, I nDenCell, float *denBoundary, I nDenBoundary,
                               float *uCell, I nUCell, float *vCell, I nVCell, float *wCell, I nWCell,
                               float *massFlux, I nMassFlux, float *p, I nP, float *ar, I nAr, float *su, I nSu,
                               float *rface, I nRFace, float small, I *icinl, I *icout, I *icsym, I *icwal,
                               bool solveTurbEnergy, bool solveTurbDiss, bool solveVisc, bool solveEnthalpy,
                               float *teCell, I nTeCell, float *teBoundary, I nTeBoundary, float *edCell,
                               I nEdCell, float *edBoundary, I nEdBoundary, float *viseffCell, I nViseffCell,
                               float *viseffBoundary, I nViseffBoundary, float *tCell, I nTCell, float *tBoundary,
                               I nTBoundary) {
    static_assert(sizeof(I) == 4, "int32 indices");
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    rc = cupcfd_gpu_flux_mass_dolfyn_face_loop_f32(
        m, detail::view_of(dudx), nDudx, detail::view_of(dvdx), nDvdx, detail::view_of(dwdx), nDwdx,
        detail::view_of(dpdx), nDpdx, denCell, nDenCell, denBoundary, nDenBoundary, uCell, nUCell, vCell, nVCell,
        wCell, nWCell, massFlux, nMassFlux, p, nP, ar, nAr, su, nSu, rface, nRFace, small, (int32_t *) icinl,
        (int32_t *) icout, (int32_t *) icsym, (int32_t *) icwal, solveTurbEnergy, solveTurbDiss, solveVisc,
        solveEnthalpy, teCell, nTeCell, teBoundary, nTeBoundary, edCell, nEdCell, edBoundary, nEdBoundary,
        viseffCell, nViseffCell, viseffBoundary, nViseffBoundary, tCell, nTCell, tBoundary, nTBoundary);
    return (ecode_t) rc;
}

// FluxMassDolfynBoundaryLoop1-5 and FluxMassDolfynRegionLoop (MassKernels.h:90-171), T = double.
// Region types and split levels are those read when the mesh was attached.
template <class Mesh, class I>
ecode_t FluxMassDolfynBoundaryLoop1(Mesh &mesh, double *massFlux, I nMassFlux, double *flowin) {
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    return (ecode_t) cupcfd_gpu_flux_mass_dolfyn_boundary_loop1(m, massFlux, (int32_t) nMassFlux, flowin);
}

template <class Mesh, class I>
ecode_t FluxMassDolfynBoundaryLoop2(Mesh &mesh, double *massFlux, I nMassFlux, double *flowRegion, I nFlowRegion,
                                    double *flowout) {
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    return (ecode_t) cupcfd_gpu_flux_mass_dolfyn_boundary_loop2(m, massFlux, (int32_t) nMassFlux, flowRegion,
                                                                (int32_t) nFlowRegion, flowout);
}

template <class Mesh>
ecode_t FluxMassDolfynBoundaryLoop3(Mesh &mesh, double flowin, double *ratearea) {
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    return (ecode_t) cupcfd_gpu_flux_mass_dolfyn_boundary_loop3(m, flowin, ratearea);
}

template <class Mesh, class I>
ecode_t FluxMassDolfynBoundaryLoop4(Mesh &mesh, double *massFlux, I nMassFlux, double *uBoundary, I nUBoundary,
                                    double *vBoundary, I nVboundary, double *wBoundary, I nWBoundary,
                                    double *denBoundary, I nDenBoundary, double ratearea, double *flowout) {
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    return (ecode_t) cupcfd_gpu_flux_mass_dolfyn_boundary_loop4(
        m, massFlux, (int32_t) nMassFlux, uBoundary, (int32_t) nUBoundary, vBoundary, (int32_t) nVboundary, wBoundary,
        (int32_t) nWBoundary, denBoundary, (int32_t) nDenBoundary, ratearea, flowout);
}

template <class Mesh, class I>
ecode_t FluxMassDolfynBoundaryLoop5(Mesh &mesh, double *massFlux, I nMassFlux, double *su, I nSu, double *uBoundary,
                                    I nUBoundary, double *vBoundary, I nVBoundary, double *wBoundary, I nWBoundary,
                                    double fact, bool solveU, bool solveV, bool solveW, double *flowFact,
                                    I nFlowFact, double *flowout2) {
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    return (ecode_t) cupcfd_gpu_flux_mass_dolfyn_boundary_loop5(
        m, massFlux, (int32_t) nMassFlux, su, (int32_t) nSu, uBoundary, (int32_t) nUBoundary, vBoundary,
        (int32_t) nVBoundary, wBoundary, (int32_t) nWBoundary, fact, solveU, solveV, solveW, flowFact,
        (int32_t) nFlowFact, flowout2);
}

template <class Mesh, class I>
ecode_t FluxMassDolfynRegionLoop(Mesh &mesh, double *flowFact, I nFlowFact, double *flowRegion, I nFlowRegion,
                                 double flowIn) {
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    return (ecode_t) cupcfd_gpu_flux_mass_dolfyn_region_loop(m, flowFact, (int32_t) nFlowFact, flowRegion,
                                                            (int32_t) nFlowRegion, flowIn);
}

// The same loops, T = float: the reference's float instantiation on a
// CupCfdSoAMesh<int,float,int> (float arithmetic in the reference's order).
template <class Mesh, class I>
ecode_t FluxMassDolfynBoundaryLoop1(Mesh &mesh, float *massFlux, I nMassFlux, float *flowin) {
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    return (ecode_t) cupcfd_gpu_flux_mass_dolfyn_boundary_loop1_f32(m, massFlux, (int32_t) nMassFlux, flowin);
}

template <class Mesh, class I>
ecode_t FluxMassDolfynBoundaryLoop2(Mesh &mesh, float *massFlux, I nMassFlux, float *flowRegion, I nFlowRegion,
                                    float *flowout) {
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    return (ecode_t) cupcfd_gpu_flux_mass_dolfyn_boundary_loop2_f32(m, massFlux, (int32_t) nMassFlux, flowRegion,
                                                                    (int32_t) nFlowRegion, flowout);
}

template <class Mesh>
ecode_t FluxMassDolfynBoundaryLoop3(Mesh &mesh, float flowin, float *ratearea) {
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    return (ecode_t) cupcfd_gpu_flux_mass_dolfyn_boundary_loop3_f32(m, flowin, ratearea);
}

template <class Mesh, class I>
ecode_t FluxMassDolfynBoundaryLoop4(Mesh &mesh, float *massFlux, I nMassFlux, float *uBoundary, I nUBoundary,
                                    float *vBoundary, I nVboundary, float *wBoundary, I nWBoundary,
                                    float *denBoundary, I nDenBoundary, float ratearea, float *flowout) {
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    return (ecode_t) cupcfd_gpu_flux_mass_dolfyn_boundary_loop4_f32(
        m, massFlux, (int32_t) nMassFlux, uBoundary, (int32_t) nUBoundary, vBoundary, (int32_t) nVboundary, wBoundary,
        (int32_t) nWBoundary, denBoundary, (int32_t) nDenBoundary, ratearea, flowout);
}

template <class Mesh, class I>
ecode_t FluxMassDolfynBoundaryLoop5(Mesh &mesh, float *massFlux, I nMassFlux, float *su, I nSu, float *uBoundary,
                                    I nUBoundary, float *vBoundary, I nVBoundary, float *wBoundary, I nWBoundary,
                                    float fact, bool solveU, bool solveV, bool solveW, float *flowFact,
                                    I nFlowFact, float *flowout2) {
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    return (ecode_t) cupcfd_gpu_flux_mass_dolfyn_boundary_loop5_f32(
        m, massFlux, (int32_t) nMassFlux, su, (int32_t) nSu, uBoundary, (int32_t) nUBoundary, vBoundary,
        (int32_t) nVBoundary, wBoundary, (int32_t) nWBoundary, fact, solveU, solveV, solveW, flowFact,
        (int32_t) nFlowFact, flowout2);
}

template <class Mesh, class I>
ecode_t FluxMassDolfynRegionLoop(Mesh &mesh, float *flowFact, I nFlowFact, float *flowRegion, I nFlowRegion,
                                 float flowIn) {
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    return (ecode_t) cupcfd_gpu_flux_mass_dolfyn_region_loop_f32(m, flowFact, (int32_t) nFlowFact, flowRegion,
                                                                (int32_t) nFlowRegion, flowIn);
}

// FluxUVWDolfynFaceLoop1 (UVWKernels.h:45-67), T = double. rlencos and the
// boundary distances are those read when the mesh was attached; the wall
// shears the loop computes are written back through setBoundaryShear.
template <class Mesh, class I, class Vec>
ecode_t FluxUVWDolfynFaceLoop1(Mesh &mesh, double gammaBlend, double small, double *uCell, I nUCell, double *vCell,
                               I nVCell, double *wCell, I nWCell, double *uBoundary, I nUBoundary, double *vBoundary,
                               I nVBoundary, double *wBoundary, I nWBoundary, double *visEffCell, I nVisEffCell,
                               double *visEffBoundary, I nVisEffBoundary, double *massFlux, I nMassFlux, Vec *dudx,
                               I nDudx, Vec *dvdx, I nDvdx, Vec *dwdx, I nDwdx, double *rFace, I nRFace, double *su,
                               I nSu, double *sv, I nSv, double *sw, I nSw, double *au, I nAu, double *av, I nAv,
                               double *aw, I nAw) {
    static_assert(sizeof(I) == 4, "int32 indices");
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    rc = cupcfd_gpu_flux_uvw_dolfyn_face_loop1(
        m, gammaBlend, small, uCell, nUCell, vCell, nVCell, wCell, nWCell, uBoundary, nUBoundary, vBoundary,
        nVBoundary, wBoundary, nWBoundary, visEffCell, nVisEffCell, visEffBoundary, nVisEffBoundary, massFlux,
        nMassFlux, detail::view_of(dudx), nDudx, detail::view_of(dvdx), nDvdx, detail::view_of(dwdx), nDwdx, rFace,
        nRFace, su, nSu, sv, nSv, sw, nSw, au, nAu, av, nAv, aw, nAw);
    if (rc == CUPCFD_E_SUCCESS) rc = detail::sync_shear(mesh, m, true, CUPCFD_RTYPE_WALL);
    return (ecode_t) rc;
}

// FluxUVWDolfynFaceLoop1, T = float: the reference's float instantiation
// (cupcfd_gpu_flux_uvw_dolfyn_face_loop1_f32). rlencos and the
// boundary distances are those read when the mesh was attached; the wall
// shears the loop computes are written back through setBoundaryShear.
template <class Mesh, class I, class Vec>
ecode_t FluxUVWDolfynFaceLoop1(Mesh &mesh, float gammaBlend, float small, float *uCell, I nUCell, float *vCell,
                               I nVCell, float *wCell, I nWCell, float *uBoundary, I nUBoundary, float *vBoundary,
                               I nVBoundary, float *wBoundary, I nWBoundary, float *visEffCell, I nVisEffCell,
                               float *visEffBoundary, I nVisEffBoundary, float *massFlux, I nMassFlux, Vec *dudx,
                               I nDudx, Vec *dvdx, I nDvdx, Vec *dwdx, I nDwdx, float *rFace, I nRFace, float *su,
                               I nSu, float *sv, I nSv, float *sw, I nSw, float *au, I nAu, float *av, I nAv,
                               float *aw, I nAw) {
    static_assert(sizeof(I) == 4, "int32 indices");
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc != CUPCFD_E_SUCCESS) return (ecode_t) rc;
    rc = cupcfd_gpu_flux_uvw_dolfyn_face_loop1_f32(
        m, gammaBlend, small, uCell, nUCell, vCell, nVCell, wCell, nWCell, uBoundary, nUBoundary, vBoundary,
        nVBoundary, wBoundary, nWBoundary, visEffCell, nVisEffCell, visEffBoundary, nVisEffBoundary, massFlux,
        nMassFlux, detail::view_of(dudx), nDudx, detail::view_of(dvdx), nDvdx, detail::view_of(dwdx), nDwdx, rFace,
        nRFace, su, nSu, sv, nSv, sw, nSw, au, nAu, av, nAv, aw, nAw);
    if (rc == CUPCFD_E_SUCCESS) rc = detail::sync_shear(mesh, m, true, CUPCFD_RTYPE_WALL);
    return (ecode_t) rc;
}

// FluxUVWDolfynRegionLoop1 / FluxUVWDolfynBndsLoop1 (UVWKernels.h:72-92) on
// the host mesh's force tangents and shears (read, computed on the GPU,
// written back). The reference's return void; these return the status.
template <class Mesh>
ecode_t FluxUVWDolfynRegionLoop1(Mesh &mesh) {
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc == CUPCFD_E_SUCCESS) rc = cupcfd_gpu_flux_uvw_dolfyn_region_loop1(m);
    if (rc == CUPCFD_E_SUCCESS) rc = detail::sync_force_tangent(mesh, m, true);
    return (ecode_t) rc;
}

template <class Mesh>
ecode_t FluxUVWDolfynBndsLoop1(Mesh &mesh) {
    cupcfd_gpu_mesh *m = nullptr;
    int rc = attach(mesh, &m);
    if (rc == CUPCFD_E_SUCCESS) rc = detail::sync_shear(mesh, m, false, -1);
    if (rc == CUPCFD_E_SUCCESS) rc = detail::sync_force_tangent(mesh, m, false);
    if (rc == CUPCFD_E_SUCCESS) rc = cupcfd_gpu_flux_uvw_dolfyn_bnds_loop1(m);
    if (rc == CUPCFD_E_SUCCESS) rc = detail::sync_force_tangent(mesh, m, true);
    return (ecode_t) rc;
}

}  // namespace gpu
}  // namespace fvm
}  // namespace cupcfd
