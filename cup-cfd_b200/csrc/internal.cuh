// Internal definitions shared by the CUDA translation units of libcupcfd_gpu.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>
#include <atomic>

#include "cupcfd_gpu.h"

namespace cupcfd_gpu {

// ---------------------------------------------------------------------------
// error plumbing: every ABI entry point returns an eCodes value; CUDA errors
// become CUPCFD_E_ERROR with the message kept per thread.
// ---------------------------------------------------------------------------
void set_error(const std::string &msg);
void clear_error();
extern std::atomic<int64_t> g_launches;

#define CG_CHECK_CUDA(expr)                                                                         \
    do {                                                                                            \
        cudaError_t e_ = (expr);                                                                    \
        if (e_ != cudaSuccess) {                                                                    \
            ::cupcfd_gpu::set_error(std::string(#expr) + ": " + cudaGetErrorString(e_) + " at " +   \
                                    __FILE__ + ":" + std::to_string(__LINE__));                     \
            return CUPCFD_E_ERROR;                                                                  \
        }                                                                                           \
    } while (0)

#define CG_RETURN_IF(cond, code, msg)          \
    do {                                       \
        if (cond) {                            \
            ::cupcfd_gpu::set_error(msg);      \
            return (code);                     \
        }                                      \
    } while (0)

#define CG_TRY(expr)                           \
    do {                                       \
        int s_ = (expr);                       \
        if (s_ != CUPCFD_E_SUCCESS) return s_; \
    } while (0)

// Counts one kernel launch and checks the launch status.
#define CG_LAUNCHED()                                                                      \
    do {                                                                                   \
        ::cupcfd_gpu::g_launches.fetch_add(1, std::memory_order_relaxed);                   \
        CG_CHECK_CUDA(cudaGetLastError());                                                 \
    } while (0)

inline unsigned grid_for(int64_t n, int block) { return (unsigned) ((n + block - 1) / block); }

// ---------------------------------------------------------------------------
// device buffer owned by a mesh
// ---------------------------------------------------------------------------
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

// Cell-incidence lists in SELL-32 layout: the cells of slice s (internal ids
// 32s .. 32s+31) own entries [slicePtr[s], slicePtr[s+1]); entry k of lane l
// sits at slicePtr[s] + 32k + l, so entry k of a warp's 32 cells is one
// coalesced 256-byte load. An entry is {code, other}: code = (internal face
// id << 1) | role, role 0 when the cell is the face's cell1 (owner, P) and 1
// when it is cell2 (neighbour, N); other = the face's other cell, or
// -1 - boundaryId on a boundary face. Padding entries are {-1, -1} and come
// after a cell's real ones. Within a cell, entries are in ascending
// REFERENCE face id: the order the reference's face loop adds contributions
// into that cell (GradientKernels.ipp:73-116).
struct Sell {
    int nSlices = 0;
    int *slicePtr = nullptr;
    int2 *inc = nullptr;
    int64_t nEntries = 0;
    int width = 0;  // the common width when every slice has it (then slice s starts at 32 * width * s), else 0
};

}  // namespace cupcfd_gpu

struct cupcfd_gpu_mesh {
    int device = 0;
    cudaStream_t stream = nullptr;  // used by the host-buffer calls
    // the host forward+adjoint's copies back run on outStream after pipeEv[i],
    // its copies in on inStream, each input set's arrival inEv[i]
    // (created on first use)
    cudaStream_t outStream = nullptr, inStream = nullptr;
    cudaEvent_t pipeEv[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t inEv[3] = {nullptr, nullptr, nullptr};
    int nC = 0, nF = 0, nB = 0, nFi = 0, nR = 0;
    int nInc = 0, maxDeg = 0;
    int order = 0, precisions = 0;
    int realSize = 8;           // bytes of the real type the source arrays held (4: a T = float mesh)
    int fullWidth = 0;          // 6: every cell has six incidences, the prefetch kernels' specialisation
    bool xpacZero = true;       // all xpac = xnac = 0 (meshes built through a MeshSource)
    bool allDefaultRegions = true;

    // numbering (internal <-> reference)
    int *cellN2O = nullptr, *cellO2N = nullptr, *faceN2O = nullptr, *faceO2N = nullptr;
    // connectivity, internal numbering: {P, N} or {P, -1 - boundaryId}
    int2 *faceCells = nullptr;
    cupcfd_gpu::Sell sell;
    // cell -> face CSR in reference numbering (CupCfdSoAMesh::cellFaceMapCSR*)
    int *refXadj = nullptr, *refAdj = nullptr;

    // FP64 geometry (internal numbering)
    double4 *fg64 = nullptr;   // {Sx, Sy, Sz, lambda}
    double4 *fc64 = nullptr;   // {xf, yf, zf, area}
    double4 *fxp64 = nullptr;  // {xpac, 0}; null when xpacZero
    double4 *fxn64 = nullptr;  // {xnac, 0}; null when xpacZero
    double4 *cc64 = nullptr;   // {xc, yc, zc, 0}
    double *vol = nullptr;     // FP64 in both precisions
    // FP32 geometry
    float4 *fg32 = nullptr;
    float4 *fc32 = nullptr;
    float4 *cc32 = nullptr;

    // boundary regions (boundary ids in reference numbering)
    int *bndRegion = nullptr, *regionType = nullptr;
    double *regionUVW = nullptr, *regionDen = nullptr;
    double *regionSplvl = nullptr;  // getRegionSplvl, zeros until cupcfd_gpu_mesh_set_region_split
    // boundary loops: each boundary's face (reference and internal ids), and
    // the boundaries sorted by (owner cell, id) with those cells in internal
    // and reference numbering; bndMapsOk false if the boundary ids were not
    // a permutation of 0 .. nB-1
    int *bndFaceRef = nullptr, *bndFaceInt = nullptr;
    int *bndSorted = nullptr, *bndSortedCellInt = nullptr, *bndSortedCellRef = nullptr;
    bool bndMapsOk = false;
    std::vector<int> hRegionType;
    // momentum loops (FluxUVWDolfyn*): getFaceRLencos per internal face and
    // getBoundaryDistance per boundary (null = all zero until set), boundary
    // shear [3 nB] and region force tangents [3 nR] (zero until written), and
    // per internal face the source of its carried face value (kernels_uvw.cuh),
    // rebuilt after the regions change
    double *rlencos = nullptr, *bndDist = nullptr, *bndShear = nullptr, *regionFT = nullptr;
    double *rlencosBuf = nullptr, *bndDistBuf = nullptr;  // storage behind rlencos / bndDist once set
    int regionFTcap = 0;
    int *uvwCarry = nullptr;
    bool uvwCarryValid = false;
    int bandwidth = 0;            // numbering bandwidth: largest |c - neighbour|
    // L2-prefetch face loops: per-tile ranges (TileDesc[nTiles], 256-cell
    // tiles); tiles false when the faces are not numbered by owner tile
    void *tileDesc = nullptr;
    int nTiles = 0;
    bool tiles = false;
    int prefetchDist = 0;         // tiles ahead for the L2 prefetch
    int prefetchWave[8] = {};  // per prefetch kernel (PfKernel in api.cu): one wave of its blocks, in tiles

    std::vector<cupcfd_gpu::DevBuf> owned;  // everything above, freed by destroy
    std::vector<cupcfd_gpu::DevBuf> scratch; // reusable buffers for host-buffer calls
    std::vector<char> hostStage;             // host staging of strided copies back (strided.cuh)
    int64_t bytes = 0;

    template <class T>
    int alloc(T **out, size_t n) {
        *out = nullptr;
        if (n == 0) n = 1;
        void *p = nullptr;
        cudaError_t e = cudaMalloc(&p, n * sizeof(T));
        if (e != cudaSuccess) {
            cupcfd_gpu::set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
            return CUPCFD_E_ERROR;
        }
        owned.push_back({p, n * sizeof(T)});
        bytes += (int64_t) (n * sizeof(T));
        *out = (T *) p;
        return CUPCFD_E_SUCCESS;
    }
    // Scratch slot `slot` grown to at least `bytes` (kept across calls).
    int scratchBuf(int slot, size_t nbytes, void **out);
};

namespace cupcfd_gpu {
// mesh build from device source arrays in reference numbering (mesh.cu)
struct Source {
    int nC, nF, nB;
    int *c1, *c2, *bnd;                 // [nF]
    double *lam, *area;                 // [nF]
    double *S, *xf, *xpac, *xnac;       // [3*nF] xyz-interleaved; xpac/xnac may be null (zero)
    double *cc, *vol;                   // [3*nC], [nC]
};
int build_mesh_from_source(cupcfd_gpu_mesh *m, const Source &src, const cupcfd_mesh_options *opt);
// bandwidth of the numbering and the fused pipeline's device state (api.cu)
int mesh_post_build(cupcfd_gpu_mesh *m, cudaStream_t st);
int make_device_current(int device);
}  // namespace cupcfd_gpu
