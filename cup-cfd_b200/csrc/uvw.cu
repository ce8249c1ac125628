// C ABI of the momentum face loop (FluxUVWDolfynFaceLoop1, RegionLoop1,
// BndsLoop1; UVWKernels.ipp:38-544) and the mesh state it reads and writes
// (getFaceRLencos, getBoundaryDistance, get/setBoundaryShear,
// get/setRegionForceTangent). Reference-facing calls on host buffers in the
// reference's numbering, and device-resident calls in the mesh's internal
// numbering. Kernels in kernels_uvw.cuh; FP64 arithmetic of the reference.
#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>

#include "kernels_uvw.cuh"
#include "ordered_sum.cuh"
#include "strided.cuh"
#include "perm.cuh"

using namespace cupcfd_gpu;

namespace {

constexpr int BT = 256;
// scratch slots of the host-buffer call (kept across calls)
enum UvwSlot { U_CELLS = 60, U_GRADS, U_VEC, U_TMP, U_MF, U_RF, U_BND, U_BLK, U_SELC, U_SELV, U_SELR, U_SPAN };

template <class T>
int slot(cupcfd_gpu_mesh *m, int s, size_t n, T **p) {
    void *v;
    CG_TRY(m->scratchBuf(s, std::max<size_t>(n, 1) * sizeof(T), &v));
    *p = (T *) v;
    return CUPCFD_E_SUCCESS;
}

int check_mesh(const cupcfd_gpu_mesh *m) {
    CG_RETURN_IF(!m, CUPCFD_E_NULL_PTR, "momentum loop: null mesh");
    CG_RETURN_IF(!(m->precisions & (1 << CUPCFD_PREC_F64)), CUPCFD_E_CONFIG_INVALID_VALUE,
                 "momentum loop: the mesh was created without FP64 geometry");
    CG_RETURN_IF(!m->bndMapsOk, CUPCFD_E_INVALID_INDEX,
                 "momentum loop: the mesh's boundary ids are not a permutation of 0 .. nBoundaries-1");
    return make_device_current(m->device);
}

// Boundary shear, region force tangents and the carried-value sources, on
// first use and after the regions change. Synchronises `st` when it builds
// the sources, so later calls on any stream see them.
int ensure_state(cupcfd_gpu_mesh *m, cudaStream_t st) {
    if (!m->bndShear) {
        CG_TRY(m->alloc(&m->bndShear, 3 * (size_t) std::max(m->nB, 1)));
        CG_CHECK_CUDA(cudaMemsetAsync(m->bndShear, 0, sizeof(double) * 3 * std::max(m->nB, 1), st));
    }
    if (m->regionFTcap < m->nR) {
        CG_TRY(m->alloc(&m->regionFT, 3 * (size_t) m->nR));
        CG_CHECK_CUDA(cudaMemsetAsync(m->regionFT, 0, sizeof(double) * 3 * m->nR, st));
        m->regionFTcap = m->nR;
    }
    if (!m->uvwCarry) CG_TRY(m->alloc(&m->uvwCarry, (size_t) m->nF));
    if (!m->uvwCarryValid) {
        int nBlk = (int) grid_for(m->nF, CARRY_T);
        int2 *blk;
        CG_TRY(slot(m, U_BLK, (size_t) nBlk, &blk));
        CarryIn ci{m->nF, m->faceO2N, m->faceCells, m->bndRegion, m->regionType};
        k_carry_reduce<<<nBlk, CARRY_T, 0, st>>>(ci, blk);
        CG_LAUNCHED();
        k_carry_scan<<<1, CARRY_T, 0, st>>>(nBlk, blk);
        CG_LAUNCHED();
        k_carry_apply<<<nBlk, CARRY_T, 0, st>>>(ci, blk, m->uvwCarry);
        CG_LAUNCHED();
        CG_CHECK_CUDA(cudaStreamSynchronize(st));
        m->uvwCarryValid = true;
    }
    return CUPCFD_E_SUCCESS;
}

// CUPCFD_UVW_PREFETCH=0 runs the plain kernel (for comparisons).
bool prefetch_disabled() {
    static const bool off = [] {
        const char *e = std::getenv("CUPCFD_UVW_PREFETCH");
        return e && e[0] == '0';
    }();
    return off;
}

// Prefetch distance of k_uvw_f64_pf: one wave of its resident blocks
// (SMs x blocks per SM), the measured optimum (2.13 ms at 256^3 against
// 2.35-2.39 ms for 1/3 to 4/3 of a wave; CUPCFD_PREFETCH_DIST overrides).
int prefetch_wave(int device) {
    static std::mutex mu;
    static std::map<int, int> wave;
    std::lock_guard<std::mutex> g(mu);
    auto it = wave.find(device);
    if (it != wave.end()) return it->second;
    int sms = 148, blocks = UVW_CELL_MINB;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_uvw_f64_pf, TILE_CELLS, 0);
    int d = std::max(1, sms * std::max(1, blocks));
    if (const char *e = std::getenv("CUPCFD_PREFETCH_DIST")) if (*e) d = std::max(1, std::atoi(e));
    wave[device] = d;
    return d;
}

int run_face_loop(cupcfd_gpu_mesh *m, double gammaBlend, double small, const double *u, const double *v,
                  const double *w, double *uB, double *vB, double *wB, const double *visC, const double *visB,
                  double *massFlux, const double *grads, int64_t ldg, double *rFace, double *su, double *sv, double *sw,
                  double *au, double *av, double *aw, cudaStream_t st) {
    CG_TRY(ensure_state(m, st));
    UvwArgs a;
    a.nC = m->nC;
    a.sv = SellView{m->sell.slicePtr, m->sell.inc, m->sell.width};
    a.fcells = m->faceCells;
    a.fg = m->fg64; a.fc = m->fc64; a.cc = m->cc64;
    a.bndRegion = m->bndRegion; a.regionType = m->regionType; a.regionUVW = m->regionUVW;
    // the carried values matter only with an inlet, outlet or symmetry region
    bool carried = false;
    for (int t : m->hRegionType)
        carried |= t == CUPCFD_RTYPE_INLET || t == CUPCFD_RTYPE_OUTLET || t == CUPCFD_RTYPE_SYMP;
    a.rlencos = m->rlencos; a.bndDist = m->bndDist; a.carry = carried ? m->uvwCarry : nullptr;
    a.gammaBlend = gammaBlend; a.small = small;
    a.u = u; a.v = v; a.w = w; a.visC = visC; a.visB = visB;
    a.grads = grads; a.ldg = ldg;
    a.uB = uB; a.vB = vB; a.wB = wB;
    a.massFlux = massFlux; a.rFace = rFace; a.shear = m->bndShear;
    a.su = su; a.sv_ = sv; a.sw = sw; a.au = au; a.av = av; a.aw = aw;
    if (m->nC == 0) return CUPCFD_E_SUCCESS;
    // the L2-prefetch form when the mesh has tile ranges and every streamed
    // array starts on a 16-byte boundary (same arithmetic, same bits)
    auto a16 = [](const void *p) { return ((uintptr_t) p & 15u) == 0; };
    const bool pfOk = m->tiles && m->tileDesc && a16(u) && a16(v) && a16(w) && a16(visC) &&
                      a16(su) && a16(sv) && a16(sw) && a16(au) && a16(av) && a16(aw) && a16(grads) &&
                      (ldg % 2) == 0 && a16(massFlux) && !prefetch_disabled();
    if (pfOk) {
        PrefetchArgs pf;
        pf.desc = (const TileDesc *) m->tileDesc;
        pf.inc = m->sell.inc;
        pf.nC = m->nC;
        pf.nF = m->nF;
        pf.nTiles = m->nTiles;
        pf.dist = prefetch_wave(m->device);
        k_uvw_f64_pf<<<grid_for(m->nC, TILE_CELLS), TILE_CELLS, 0, st>>>(a, pf);
    } else {
        k_uvw_f64<<<grid_for(m->nC, BT), BT, 0, st>>>(a);
    }
    CG_LAUNCHED();
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

// reference-numbered [n] double array (3 per element when vec) on the host
// -> device, then to internal order
int cells_in(cupcfd_gpu_mesh *m, const double *h, double *dst, double *tmp, cudaStream_t st) {
    CG_TRY(up(tmp, h, sizeof(double) * m->nC, st));
    k_gather<double, double><<<grid_for(m->nC, BT), BT, 0, st>>>(m->nC, 1, m->cellN2O, tmp, 0, dst, 0);
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}
int cells_out(cupcfd_gpu_mesh *m, const double *src, double *h, double *tmp, cudaStream_t st) {
    k_gather<double, double><<<grid_for(m->nC, BT), BT, 0, st>>>(m->nC, 1, m->cellO2N, src, 0, tmp, 0);
    CG_LAUNCHED();
    return down(h, tmp, sizeof(double) * m->nC, st);
}

int vec3_in(cupcfd_gpu_mesh *m, const cupcfd_vec3_view &v, double *dst, int64_t ld, double *tmp, cudaStream_t st) {
    CG_RETURN_IF(!v.base, CUPCFD_E_NULL_PTR, "momentum loop: null vector array");
    CG_RETURN_IF(v.stride < 24 || v.offset < 0 || v.offset + 24 > v.stride, CUPCFD_E_CONFIG_INVALID_VALUE,
                 "momentum loop: bad vector stride/offset");
    char *span = nullptr;
    if (v.stride != 24) CG_TRY(slot(m, U_SPAN, vec3_span_bytes(m->nC, v.stride, v.offset, 8), &span));
    CG_TRY(upload_vec3_span(v.base, v.stride, v.offset, m->nC, 8, span, tmp, st));
    k_aos_to_blocks<double, double><<<grid_for(m->nC, BT), BT, 0, st>>>(m->nC, 3, m->cellN2O, tmp, dst, ld);
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}

}  // namespace

// ===========================================================================
// mesh state
// ===========================================================================
extern "C" int cupcfd_gpu_mesh_set_face_rlencos(cupcfd_gpu_mesh *m, const double *rlencos, int32_t nFaces) {
    clear_error();
    CG_RETURN_IF(!m, CUPCFD_E_NULL_PTR, "set_face_rlencos: null mesh");
    CG_TRY(make_device_current(m->device));
    if (!rlencos) {  // back to all zero
        m->rlencos = nullptr;
        return CUPCFD_E_SUCCESS;
    }
    CG_RETURN_IF(nFaces != m->nF, CUPCFD_E_ARRAY_SIZE_MISMATCH, "set_face_rlencos: nFaces differs from the mesh");
    cudaStream_t st = m->stream;
    if (!m->rlencosBuf) CG_TRY(m->alloc(&m->rlencosBuf, (size_t) m->nF));
    double *d = m->rlencosBuf, *tmp;
    CG_TRY(slot(m, U_TMP, (size_t) m->nF, &tmp));
    CG_TRY(up(tmp, rlencos, sizeof(double) * m->nF, st));
    k_gather<double, double><<<grid_for(m->nF, BT), BT, 0, st>>>(m->nF, 1, m->faceN2O, tmp, 0, d, 0);
    CG_LAUNCHED();
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    m->rlencos = d;
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_mesh_set_boundary_distance(cupcfd_gpu_mesh *m, const double *dist, int32_t nBoundaries) {
    clear_error();
    CG_RETURN_IF(!m, CUPCFD_E_NULL_PTR, "set_boundary_distance: null mesh");
    CG_TRY(make_device_current(m->device));
    if (!dist) {
        m->bndDist = nullptr;
        return CUPCFD_E_SUCCESS;
    }
    CG_RETURN_IF(nBoundaries != m->nB, CUPCFD_E_ARRAY_SIZE_MISMATCH, "set_boundary_distance: nBoundaries differs from the mesh");
    if (!m->bndDistBuf) CG_TRY(m->alloc(&m->bndDistBuf, (size_t) std::max(m->nB, 1)));
    double *d = m->bndDistBuf;
    CG_TRY(up(d, dist, sizeof(double) * m->nB, m->stream));
    CG_CHECK_CUDA(cudaStreamSynchronize(m->stream));
    m->bndDist = d;
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_mesh_boundary_shear(cupcfd_gpu_mesh *m, const double *in, double *out, int32_t nBoundaries) {
    clear_error();
    CG_TRY(check_mesh(m));
    CG_RETURN_IF(nBoundaries != m->nB, CUPCFD_E_ARRAY_SIZE_MISMATCH, "boundary_shear: nBoundaries differs from the mesh");
    CG_TRY(ensure_state(m, m->stream));
    if (in) CG_TRY(up(m->bndShear, in, sizeof(double) * 3 * m->nB, m->stream));
    if (out) CG_TRY(down(out, m->bndShear, sizeof(double) * 3 * m->nB, m->stream));
    CG_CHECK_CUDA(cudaStreamSynchronize(m->stream));
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_mesh_region_force_tangent(cupcfd_gpu_mesh *m, const double *in, double *out, int32_t nRegions) {
    clear_error();
    CG_TRY(check_mesh(m));
    CG_RETURN_IF(nRegions != m->nR, CUPCFD_E_ARRAY_SIZE_MISMATCH, "region_force_tangent: nRegions differs from the mesh");
    CG_TRY(ensure_state(m, m->stream));
    if (in) CG_TRY(up(m->regionFT, in, sizeof(double) * 3 * m->nR, m->stream));
    if (out) CG_TRY(down(out, m->regionFT, sizeof(double) * 3 * m->nR, m->stream));
    CG_CHECK_CUDA(cudaStreamSynchronize(m->stream));
    return CUPCFD_E_SUCCESS;
}

// ===========================================================================
// FluxUVWDolfynFaceLoop1 on host buffers
// ===========================================================================
extern "C" int cupcfd_gpu_flux_uvw_dolfyn_face_loop1(
    cupcfd_gpu_mesh *m, double gammaBlend, double small, const double *u, int32_t nU, const double *v, int32_t nV,
    const double *w, int32_t nW, double *uB, int32_t nUB, double *vB, int32_t nVB, double *wB, int32_t nWB,
    const double *visC, int32_t nVisC, const double *visB, int32_t nVisB, double *massFlux, int32_t nMassFlux,
    cupcfd_vec3_view dudx, int32_t nDudx, cupcfd_vec3_view dvdx, int32_t nDvdx, cupcfd_vec3_view dwdx, int32_t nDwdx,
    double *rFace, int32_t nRFace, double *su, int32_t nSu, double *sv, int32_t nSv, double *sw, int32_t nSw,
    double *au, int32_t nAu, double *av, int32_t nAv, double *aw, int32_t nAw) {
    clear_error();
    CG_RETURN_IF(!m || !u || !v || !w || !visC || !massFlux || !rFace || !su || !sv || !sw || !au || !av || !aw ||
                     (m->nB > 0 && (!uB || !vB || !wB || !visB)),
                 CUPCFD_E_NULL_PTR, "FluxUVWDolfynFaceLoop1: null argument");
    const int nC = m->nC, nF = m->nF, nB = m->nB;
    // the reference's DEBUG index checks (UVWKernels.ipp:99-142, 204-208, 237-257)
    CG_RETURN_IF(nU < nC || nV < nC || nW < nC || nVisC < nC || nDudx < nC || nDvdx < nC || nDwdx < nC || nSu < nC ||
                     nSv < nC || nSw < nC || nAu < nC || nAv < nC || nAw < nC || nMassFlux < nF || nRFace < 2 * nF ||
                     nUB < nB || nVB < nB || nWB < nB || nVisB < nB,
                 CUPCFD_E_INVALID_INDEX, "FluxUVWDolfynFaceLoop1: array shorter than the mesh needs");
    CG_TRY(check_mesh(m));
    cudaStream_t st = m->stream;
    const int64_t ld = nC;
    double *cells, *grads, *vec, *tmp, *mf, *rf, *bnd;
    CG_TRY(slot(m, U_CELLS, 10 * (size_t) nC, &cells));
    CG_TRY(slot(m, U_GRADS, 9 * (size_t) nC, &grads));
    CG_TRY(slot(m, U_VEC, 3 * (size_t) nC, &vec));
    CG_TRY(slot(m, U_TMP, std::max<size_t>(nC, 2 * (size_t) nF), &tmp));
    CG_TRY(slot(m, U_MF, (size_t) nF, &mf));
    CG_TRY(slot(m, U_RF, 2 * (size_t) nF, &rf));
    CG_TRY(slot(m, U_BND, 4 * (size_t) nB, &bnd));
    // cells: u v w visC su sv sw au av aw
    const double *cin[10] = {u, v, w, visC, su, sv, sw, au, av, aw};
    for (int q = 0; q < 10; q++) CG_TRY(cells_in(m, cin[q], cells + q * ld, tmp, st));
    const cupcfd_vec3_view vv[3] = {dudx, dvdx, dwdx};
    for (int q = 0; q < 3; q++) CG_TRY(vec3_in(m, vv[q], grads + 3 * q * ld, ld, vec, st));
    // faces: massFlux, rFace pairs
    CG_TRY(up(tmp, massFlux, sizeof(double) * nF, st));
    k_gather<double, double><<<grid_for(nF, BT), BT, 0, st>>>(nF, 1, m->faceN2O, tmp, 0, mf, 0);
    CG_LAUNCHED();
    CG_TRY(up(tmp, rFace, sizeof(double) * 2 * nF, st));
    k_gather_pairs<double><<<grid_for(nF, BT), BT, 0, st>>>(nF, m->faceN2O, tmp, rf);
    CG_LAUNCHED();
    // boundaries (same ids on both sides): uB vB wB visB
    double *hb[4] = {uB, vB, wB, const_cast<double *>(visB)};
    for (int q = 0; q < 4; q++) CG_TRY(up(bnd + (size_t) q * nB, hb[q], sizeof(double) * nB, st));
    double *c = cells;
    CG_TRY(run_face_loop(m, gammaBlend, small, c, c + ld, c + 2 * ld, bnd, bnd + nB, bnd + 2 * (size_t) nB, c + 3 * ld,
                         bnd + 3 * (size_t) nB, mf, grads, ld, rf, c + 4 * ld, c + 5 * ld, c + 6 * ld, c + 7 * ld,
                         c + 8 * ld, c + 9 * ld, st));
    // back to the reference's numbering; one staging buffer, reused in
    // stream order (each copy out finishes before the next gather runs)
    k_gather<double, double><<<grid_for(nF, BT), BT, 0, st>>>(nF, 1, m->faceO2N, mf, 0, tmp, 0);
    CG_LAUNCHED();
    CG_TRY(down(massFlux, tmp, sizeof(double) * nF, st));
    k_gather_pairs<double><<<grid_for(nF, BT), BT, 0, st>>>(nF, m->faceO2N, rf, tmp);
    CG_LAUNCHED();
    CG_TRY(down(rFace, tmp, sizeof(double) * 2 * nF, st));
    double *cout_[6] = {su, sv, sw, au, av, aw};
    for (int q = 0; q < 6; q++) CG_TRY(cells_out(m, c + (4 + q) * ld, cout_[q], tmp, st));
    for (int q = 0; q < 3; q++) CG_TRY(down(hb[q], bnd + (size_t) q * nB, sizeof(double) * nB, st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    return CUPCFD_E_SUCCESS;
}

// ===========================================================================
// device-resident calls (internal numbering, caller stream)
// ===========================================================================
extern "C" int cupcfd_gpu_dev_uvw_face_loop1(cupcfd_gpu_mesh *m, double gammaBlend, double small, const double *u,
                                             const double *v, const double *w, double *uB, double *vB, double *wB,
                                             const double *visC, const double *visB, double *massFlux,
                                             const double *grads, int64_t ldg, double *rFace, double *su, double *sv,
                                             double *sw, double *au, double *av, double *aw, void *stream) {
    clear_error();
    CG_RETURN_IF(!m || !u || !v || !w || !visC || !massFlux || !grads || !rFace || !su || !sv || !sw || !au || !av ||
                     !aw || (m->nB > 0 && (!uB || !vB || !wB || !visB)),
                 CUPCFD_E_NULL_PTR, "dev_uvw_face_loop1: null argument");
    CG_RETURN_IF(ldg < m->nC, CUPCFD_E_INVALID_INDEX, "dev_uvw_face_loop1: gradient leading dimension below nCells");
    CG_TRY(check_mesh(m));
    return run_face_loop(m, gammaBlend, small, u, v, w, uB, vB, wB, visC, visB, massFlux, grads, ldg, rFace, su, sv, sw,
                         au, av, aw, (cudaStream_t) stream);
}

extern "C" int cupcfd_gpu_dev_uvw_region_loop1(cupcfd_gpu_mesh *m, void *stream) {
    clear_error();
    CG_TRY(check_mesh(m));
    cudaStream_t st = (cudaStream_t) stream;
    CG_TRY(ensure_state(m, st));
    CG_CHECK_CUDA(cudaMemsetAsync(m->regionFT, 0, sizeof(double) * 3 * m->nR, st));
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_dev_uvw_bnds_loop1(cupcfd_gpu_mesh *m, void *stream) {
    clear_error();
    CG_TRY(check_mesh(m));
    cudaStream_t st = (cudaStream_t) stream;
    CG_TRY(ensure_state(m, st));
    if (m->nB > 0) {
        // wall boundaries add their shear onto their region's force tangent
        // in boundary order (UVWKernels.ipp:527-544)
        int *cnt, *regs;
        double *vals;
        CG_TRY(slot(m, U_SELC, (size_t) m->nB / SEL_T + 2, &cnt));
        CG_TRY(slot(m, U_SELV, 3 * (size_t) m->nB, &vals));
        CG_TRY(slot(m, U_SELR, (size_t) m->nB, &regs));
        CG_TRY(launch_ordered_sum<3>(SelArgs{m->nB, m->bndRegion, m->regionType, CUPCFD_RTYPE_WALL}, m->bndShear, 3, 0,
                                     nullptr, nullptr, 0.0, nullptr, m->regionFT, m->nR, cnt, vals, regs, st));
    }
    return CUPCFD_E_SUCCESS;
}

// host-synchronous forms (the reference's calls take only the mesh)
extern "C" int cupcfd_gpu_flux_uvw_dolfyn_region_loop1(cupcfd_gpu_mesh *m) {
    CG_TRY(cupcfd_gpu_dev_uvw_region_loop1(m, m ? m->stream : nullptr));
    CG_CHECK_CUDA(cudaStreamSynchronize(m->stream));
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_flux_uvw_dolfyn_bnds_loop1(cupcfd_gpu_mesh *m) {
    CG_TRY(cupcfd_gpu_dev_uvw_bnds_loop1(m, m ? m->stream : nullptr));
    CG_CHECK_CUDA(cudaStreamSynchronize(m->stream));
    return CUPCFD_E_SUCCESS;
}
