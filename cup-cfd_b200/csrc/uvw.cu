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

// geomPrec: the geometry the call reads (FP64 for T = double, FP32 for the
// float instantiation)
int check_mesh(const cupcfd_gpu_mesh *m, int geomPrec = CUPCFD_PREC_F64) {
    CG_RETURN_IF(!m, CUPCFD_E_NULL_PTR, "momentum loop: null mesh");
    CG_RETURN_IF(!(m->precisions & (1 << geomPrec)), CUPCFD_E_CONFIG_INVALID_VALUE,
                 geomPrec == CUPCFD_PREC_F64 ? "momentum loop: the mesh was created without FP64 geometry"
                                             : "momentum loop: the mesh was created without FP32 geometry");
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

// Prefetch distance of the L2-prefetch kernel `kern`, in tiles: 1.25 waves
// of its resident blocks (SMs x tiles' worth of blocks per SM): with
// 64-thread blocks 1.87 ms at 256^3 against 1.94 at 1 wave, 1.95 at 1.5,
// 2.08 at 0.75, 2.21 at 2. In 256-thread blocks one wave was the measured
// optimum for
// k_uvw_f64_pf (2.13 ms at 256^3 against 2.35-2.39 ms for 1/3 to 4/3 of a
// wave; CUPCFD_PREFETCH_DIST overrides).
int prefetch_wave(int device, const void *kern) {
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, int> wave;
    std::lock_guard<std::mutex> g(mu);
    auto it = wave.find({device, kern});
    if (it != wave.end()) return it->second;
    int sms = 148, blocks = UVW_CELL_MINB * TILE_CELLS / UVW_PF_BLOCK;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, UVW_PF_BLOCK, 0);
    int d = std::max(1, sms * std::max(1, blocks * UVW_PF_BLOCK / TILE_CELLS) * 5 / 4);  // in tiles
    if (const char *e = std::getenv("CUPCFD_PREFETCH_DIST")) if (*e) d = std::max(1, std::atoi(e));
    wave[{device, kern}] = d;
    return d;
}

template <class T>
int run_face_loop(cupcfd_gpu_mesh *m, T gammaBlend, T small, const T *u, const T *v, const T *w, T *uB, T *vB, T *wB,
                  const T *visC, const T *visB, T *massFlux, const T *grads, int64_t ldg, T *rFace, T *su, T *sv,
                  T *sw, T *au, T *av, T *aw, cudaStream_t st) {
    constexpr bool F64 = sizeof(T) == 8;
    CG_TRY(ensure_state(m, st));
    UvwArgs<T> a;
    a.nC = m->nC;
    a.sv = SellView{m->sell.slicePtr, m->sell.inc, m->sell.width};
    a.fcells = m->faceCells;
    if constexpr (F64) {
        a.fg = m->fg64; a.fc = m->fc64; a.cc = m->cc64;
    } else {
        a.fg = m->fg32; a.fc = m->fc32; a.cc = m->cc32;
    }
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
                      (ldg * (int64_t) sizeof(T)) % 16 == 0 && a16(massFlux) && !prefetch_disabled();
    if (pfOk) {
        PrefetchArgs pf;
        pf.desc = (const TileDesc *) m->tileDesc;
        pf.inc = m->sell.inc;
        pf.nC = m->nC;
        pf.nF = m->nF;
        pf.nTiles = m->nTiles;
        if constexpr (F64) {
            pf.dist = prefetch_wave(m->device, (const void *) k_uvw_f64_pf);
            k_uvw_f64_pf<<<grid_for(m->nC, TILE_CELLS) * (TILE_CELLS / UVW_PF_BLOCK), UVW_PF_BLOCK, 0, st>>>(a, pf);
        } else {
            pf.dist = prefetch_wave(m->device, (const void *) k_uvw_f32ref_pf);
            k_uvw_f32ref_pf<<<grid_for(m->nC, TILE_CELLS) * (TILE_CELLS / UVW_PF_BLOCK), UVW_PF_BLOCK, 0, st>>>(a, pf);
        }
    } else {
        if constexpr (F64)
            k_uvw_f64<<<grid_for(m->nC, BT), BT, 0, st>>>(a);
        else
            k_uvw_f32ref<<<grid_for(m->nC, BT), BT, 0, st>>>(a);
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

// reference-numbered [n] array of T (3 per element when vec) on the host
// -> device, then to internal order
template <class T>
int cells_in(cupcfd_gpu_mesh *m, const T *h, T *dst, T *tmp, cudaStream_t st) {
    CG_TRY(up(tmp, h, sizeof(T) * m->nC, st));
    k_gather<T, T><<<grid_for(m->nC, BT), BT, 0, st>>>(m->nC, 1, m->cellN2O, tmp, 0, dst, 0);
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}
template <class T>
int cells_out(cupcfd_gpu_mesh *m, const T *src, T *h, T *tmp, cudaStream_t st) {
    k_gather<T, T><<<grid_for(m->nC, BT), BT, 0, st>>>(m->nC, 1, m->cellO2N, src, 0, tmp, 0);
    CG_LAUNCHED();
    return down(h, tmp, sizeof(T) * m->nC, st);
}

template <class T>
int vec3_in(cupcfd_gpu_mesh *m, const cupcfd_vec3_view &v, T *dst, int64_t ld, T *tmp, cudaStream_t st) {
    constexpr int RS = (int) sizeof(T);
    CG_RETURN_IF(!v.base, CUPCFD_E_NULL_PTR, "momentum loop: null vector array");
    CG_RETURN_IF(v.stride < 3 * RS || v.offset < 0 || v.offset + 3 * RS > v.stride, CUPCFD_E_CONFIG_INVALID_VALUE,
                 "momentum loop: bad vector stride/offset");
    char *span = nullptr;
    if (v.stride != 3 * RS) CG_TRY(slot(m, U_SPAN, vec3_span_bytes(m->nC, v.stride, v.offset, RS), &span));
    CG_TRY(upload_vec3_span(v.base, v.stride, v.offset, m->nC, RS, span, tmp, st));
    k_aos_to_blocks<T, T><<<grid_for(m->nC, BT), BT, 0, st>>>(m->nC, 3, m->cellN2O, tmp, dst, ld);
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
namespace {
template <class T>
int uvw_face_loop1_t(cupcfd_gpu_mesh *m, T gammaBlend, T small, const T *u, int32_t nU, const T *v, int32_t nV,
                     const T *w, int32_t nW, T *uB, int32_t nUB, T *vB, int32_t nVB, T *wB, int32_t nWB,
                     const T *visC, int32_t nVisC, const T *visB, int32_t nVisB, T *massFlux, int32_t nMassFlux,
                     cupcfd_vec3_view dudx, int32_t nDudx, cupcfd_vec3_view dvdx, int32_t nDvdx, cupcfd_vec3_view dwdx,
                     int32_t nDwdx, T *rFace, int32_t nRFace, T *su, int32_t nSu, T *sv, int32_t nSv, T *sw,
                     int32_t nSw, T *au, int32_t nAu, T *av, int32_t nAv, T *aw, int32_t nAw) {
    CG_RETURN_IF(!m || !u || !v || !w || !visC || !massFlux || !rFace || !su || !sv || !sw || !au || !av || !aw ||
                     (m->nB > 0 && (!uB || !vB || !wB || !visB)),
                 CUPCFD_E_NULL_PTR, "FluxUVWDolfynFaceLoop1: null argument");
    const int nC = m->nC, nF = m->nF, nB = m->nB;
    // the reference's DEBUG index checks (UVWKernels.ipp:99-142, 204-208, 237-257)
    CG_RETURN_IF(nU < nC || nV < nC || nW < nC || nVisC < nC || nDudx < nC || nDvdx < nC || nDwdx < nC || nSu < nC ||
                     nSv < nC || nSw < nC || nAu < nC || nAv < nC || nAw < nC || nMassFlux < nF || nRFace < 2 * nF ||
                     nUB < nB || nVB < nB || nWB < nB || nVisB < nB,
                 CUPCFD_E_INVALID_INDEX, "FluxUVWDolfynFaceLoop1: array shorter than the mesh needs");
    CG_TRY(check_mesh(m, sizeof(T) == 8 ? CUPCFD_PREC_F64 : CUPCFD_PREC_F32C));
    cudaStream_t st = m->stream;
    const int64_t ld = nC;
    T *cells, *grads, *vec, *tmp, *mf, *rf, *bnd;
    CG_TRY(slot(m, U_CELLS, 10 * (size_t) nC, &cells));
    CG_TRY(slot(m, U_GRADS, 9 * (size_t) nC, &grads));
    CG_TRY(slot(m, U_VEC, 3 * (size_t) nC, &vec));
    CG_TRY(slot(m, U_TMP, std::max<size_t>(nC, 2 * (size_t) nF), &tmp));
    CG_TRY(slot(m, U_MF, (size_t) nF, &mf));
    CG_TRY(slot(m, U_RF, 2 * (size_t) nF, &rf));
    CG_TRY(slot(m, U_BND, 4 * (size_t) nB, &bnd));
    // cells: u v w visC su sv sw au av aw
    const T *cin[10] = {u, v, w, visC, su, sv, sw, au, av, aw};
    for (int q = 0; q < 10; q++) CG_TRY(cells_in(m, cin[q], cells + q * ld, tmp, st));
    const cupcfd_vec3_view vv[3] = {dudx, dvdx, dwdx};
    for (int q = 0; q < 3; q++) CG_TRY(vec3_in(m, vv[q], grads + 3 * q * ld, ld, vec, st));
    // faces: massFlux, rFace pairs
    CG_TRY(up(tmp, massFlux, sizeof(T) * nF, st));
    k_gather<T, T><<<grid_for(nF, BT), BT, 0, st>>>(nF, 1, m->faceN2O, tmp, 0, mf, 0);
    CG_LAUNCHED();
    CG_TRY(up(tmp, rFace, sizeof(T) * 2 * nF, st));
    k_gather_pairs<T><<<grid_for(nF, BT), BT, 0, st>>>(nF, m->faceN2O, tmp, rf);
    CG_LAUNCHED();
    // boundaries (same ids on both sides): uB vB wB visB
    T *hb[4] = {uB, vB, wB, const_cast<T *>(visB)};
    for (int q = 0; q < 4; q++) CG_TRY(up(bnd + (size_t) q * nB, hb[q], sizeof(T) * nB, st));
    T *c = cells;
    CG_TRY(run_face_loop(m, gammaBlend, small, c, c + ld, c + 2 * ld, bnd, bnd + nB, bnd + 2 * (size_t) nB, c + 3 * ld,
                         bnd + 3 * (size_t) nB, mf, grads, ld, rf, c + 4 * ld, c + 5 * ld, c + 6 * ld, c + 7 * ld,
                         c + 8 * ld, c + 9 * ld, st));
    // back to the reference's numbering; one staging buffer, reused in
    // stream order (each copy out finishes before the next gather runs)
    k_gather<T, T><<<grid_for(nF, BT), BT, 0, st>>>(nF, 1, m->faceO2N, mf, 0, tmp, 0);
    CG_LAUNCHED();
    CG_TRY(down(massFlux, tmp, sizeof(T) * nF, st));
    k_gather_pairs<T><<<grid_for(nF, BT), BT, 0, st>>>(nF, m->faceO2N, rf, tmp);
    CG_LAUNCHED();
    CG_TRY(down(rFace, tmp, sizeof(T) * 2 * nF, st));
    T *cout_[6] = {su, sv, sw, au, av, aw};
    for (int q = 0; q < 6; q++) CG_TRY(cells_out(m, c + (4 + q) * ld, cout_[q], tmp, st));
    for (int q = 0; q < 3; q++) CG_TRY(down(hb[q], bnd + (size_t) q * nB, sizeof(T) * nB, st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    return CUPCFD_E_SUCCESS;
}

}  // namespace

extern "C" int cupcfd_gpu_flux_uvw_dolfyn_face_loop1(
    cupcfd_gpu_mesh *m, double gammaBlend, double small, const double *u, int32_t nU, const double *v, int32_t nV,
    const double *w, int32_t nW, double *uB, int32_t nUB, double *vB, int32_t nVB, double *wB, int32_t nWB,
    const double *visC, int32_t nVisC, const double *visB, int32_t nVisB, double *massFlux, int32_t nMassFlux,
    cupcfd_vec3_view dudx, int32_t nDudx, cupcfd_vec3_view dvdx, int32_t nDvdx, cupcfd_vec3_view dwdx, int32_t nDwdx,
    double *rFace, int32_t nRFace, double *su, int32_t nSu, double *sv, int32_t nSv, double *sw, int32_t nSw,
    double *au, int32_t nAu, double *av, int32_t nAv, double *aw, int32_t nAw) {
    clear_error();
    return uvw_face_loop1_t<double>(m, gammaBlend, small, u, nU, v, nV, w, nW, uB, nUB, vB, nVB, wB, nWB, visC, nVisC,
                                    visB, nVisB, massFlux, nMassFlux, dudx, nDudx, dvdx, nDvdx, dwdx, nDwdx, rFace,
                                    nRFace, su, nSu, sv, nSv, sw, nSw, au, nAu, av, nAv, aw, nAw);
}

extern "C" int cupcfd_gpu_flux_uvw_dolfyn_face_loop1_f32(
    cupcfd_gpu_mesh *m, float gammaBlend, float small, const float *u, int32_t nU, const float *v, int32_t nV,
    const float *w, int32_t nW, float *uB, int32_t nUB, float *vB, int32_t nVB, float *wB, int32_t nWB,
    const float *visC, int32_t nVisC, const float *visB, int32_t nVisB, float *massFlux, int32_t nMassFlux,
    cupcfd_vec3_view dudx, int32_t nDudx, cupcfd_vec3_view dvdx, int32_t nDvdx, cupcfd_vec3_view dwdx, int32_t nDwdx,
    float *rFace, int32_t nRFace, float *su, int32_t nSu, float *sv, int32_t nSv, float *sw, int32_t nSw,
    float *au, int32_t nAu, float *av, int32_t nAv, float *aw, int32_t nAw) {
    clear_error();
    return uvw_face_loop1_t<float>(m, gammaBlend, small, u, nU, v, nV, w, nW, uB, nUB, vB, nVB, wB, nWB, visC, nVisC,
                                   visB, nVisB, massFlux, nMassFlux, dudx, nDudx, dvdx, nDvdx, dwdx, nDwdx, rFace,
                                   nRFace, su, nSu, sv, nSv, sw, nSw, au, nAu, av, nAv, aw, nAw);
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
    return run_face_loop<double>(m, gammaBlend, small, u, v, w, uB, vB, wB, visC, visB, massFlux, grads, ldg, rFace, su,
                                 sv, sw, au, av, aw, (cudaStream_t) stream);
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
        // (in float on a mesh of the reference's T = float instantiation)
        const SelArgs sa{m->nB, m->bndRegion, m->regionType, CUPCFD_RTYPE_WALL};
        const int rc = m->realSize == 4
                           ? launch_ordered_sum<3, true>(sa, m->bndShear, 3, 0, nullptr, nullptr, 0.0, nullptr,
                                                         m->regionFT, m->nR, cnt, vals, regs, st)
                           : launch_ordered_sum<3>(sa, m->bndShear, 3, 0, nullptr, nullptr, 0.0, nullptr, m->regionFT,
                                                   m->nR, cnt, vals, regs, st);
        CG_TRY(rc);
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
