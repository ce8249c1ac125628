// C ABI: reference-facing host-buffer calls and device-resident calls.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <initializer_list>
#include <map>
#include <mutex>

#include "kernels_pf.cuh"
#include "strided.cuh"
#include "perm.cuh"

using namespace cupcfd_gpu;

namespace {

constexpr int BLK = 256;

// the L2-prefetch kernels, indexing cupcfd_gpu_mesh::prefetchWave
enum PfKernel { PF_FWD_F32 = 0, PF_ADJ_F32, PF_FWD_F64, PF_ADJ_F64, PF_FWD_MADJ, PF_GADJ, PF_MADJ, PF_COUNT };

// scratch slots of a mesh (each grows on demand and is reused across calls)
enum Slot {
    S_ERR = 0, S_GEOM = 1, S_IN0, S_IN1, S_IN2, S_IN3, S_IN4, S_IN5, S_IN6, S_IN7,
    S_OUT0, S_OUT1, S_OUT2, S_OUT3, S_OUT4, S_GO, S_LOSS, S_CNT, S_NORM, S_SPAN
};

template <class T>
int scratch(cupcfd_gpu_mesh *m, int slot, size_t n, T **p) {
    void *v;
    CG_TRY(m->scratchBuf(slot, n * sizeof(T), &v));
    *p = (T *) v;
    return CUPCFD_E_SUCCESS;
}

inline cudaStream_t as_stream(void *s) { return (cudaStream_t) s; }

// The mesh's second and third streams and their events (created on first
// use): the host forward+adjoint's copy-back and copy-in streams, and the
// loss reduction beside the gradient adjoint in the device forward+adjoint.
// The stream has the device's highest priority, so that the loss
// reduction's one block is placed as soon as an SM has room for it, not
// after the gradient adjoint's blocks.
#ifndef CUPCFD_AUX_PRIORITY
#define CUPCFD_AUX_PRIORITY 1
#endif
int pipe_init(cupcfd_gpu_mesh *m) {
    if (m->outStream) return CUPCFD_E_SUCCESS;
    for (cudaEvent_t &e : m->pipeEv)
        if (!e) CG_CHECK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (cudaEvent_t &e : m->inEv)
        if (!e) CG_CHECK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    if (!m->inStream) CG_CHECK_CUDA(cudaStreamCreateWithFlags(&m->inStream, cudaStreamNonBlocking));
    int lo = 0, hi = 0;
    CG_CHECK_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    CG_CHECK_CUDA(cudaStreamCreateWithPriority(&m->outStream, cudaStreamNonBlocking, CUPCFD_AUX_PRIORITY ? hi : lo));
    return CUPCFD_E_SUCCESS;
}

inline SellView sell(const cupcfd_gpu_mesh *m) { return SellView{m->sell.slicePtr, m->sell.inc, m->sell.width}; }

// The width the L2-prefetch kernels are specialised for (kernels_pf.cuh:
// WF), set by tiles_setup: 6 when every cell has exactly six incidences
// (all hexahedral meshes), else 0 (the general kernels).
inline int full_width(const cupcfd_gpu_mesh *m) { return m->fullWidth; }
// launches the L2-prefetch kernel template K at the mesh's full width
#define CG_LAUNCH_PF_BLOCK(m, K, grid, block, st, ...)                          \
    do {                                                                        \
        if (full_width(m) == 6) K<6><<<(grid), (block), 0, (st)>>>(__VA_ARGS__); \
        else K<0><<<(grid), (block), 0, (st)>>>(__VA_ARGS__);                   \
    } while (0)
#define CG_LAUNCH_PF(m, K, grid, st, ...) CG_LAUNCH_PF_BLOCK(m, K, grid, BLK, st, __VA_ARGS__)

// ---------------------------------------------------------------------------
// device timers (cupcfd_gpu_timing_*): a KTIMER scope records one event
// before and one after the launch it encloses, on the launch's stream
// ---------------------------------------------------------------------------
struct TimerRec {
    const char *name;
    int device;
    cudaEvent_t a, b;
};
std::mutex g_timer_mu;
std::atomic<bool> g_timer_on{false};
std::vector<TimerRec> g_timer_recs;

class KernelTimer {
  public:
    KernelTimer(const char *name, cudaStream_t st) : name_(name), st_(st) {
        if (!g_timer_on.load(std::memory_order_relaxed)) return;
        if (cudaEventCreate(&a_) != cudaSuccess || cudaEventRecord(a_, st_) != cudaSuccess) a_ = nullptr;
    }
    void set_name(const char *name) { name_ = name; }
    ~KernelTimer() {
        if (!a_) return;
        cudaEvent_t b = nullptr;
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaEventCreate(&b) != cudaSuccess || cudaEventRecord(b, st_) != cudaSuccess) {
            cudaEventDestroy(a_);
            if (b) cudaEventDestroy(b);
            return;
        }
        std::lock_guard<std::mutex> lk(g_timer_mu);
        g_timer_recs.push_back({name_, dev, a_, b});
    }
  private:
    const char *name_;
    cudaStream_t st_;
    cudaEvent_t a_ = nullptr;
};
#define KTIMER(name, stream) KernelTimer ktimer_(name, stream)

inline bool aligned16(const void *p) { return ((uintptr_t) p & 15u) == 0; }

// Builds the per-tile ranges the L2-prefetch kernels of both precisions read
// and the prefetch distance of each kernel; leaves m->tiles false (plain
// kernels only) when the faces are not numbered by owner tile (the native
// numbering keeps the reference's face order) or a slice is too wide.
int tiles_setup(cupcfd_gpu_mesh *m, cudaStream_t st) {
    m->tiles = false;
    if (m->nF < 1 || m->nC < 1) return CUPCFD_E_SUCCESS;
    m->nTiles = (int) grid_for(m->nC, TILE_CELLS);
    TileDesc *desc;
    CG_TRY(m->alloc(&desc, (size_t) m->nTiles));
    m->tileDesc = desc;
    int *start, *aux;  // aux: [0..2] maxima, [3] order flag
    CG_TRY(m->alloc(&start, (size_t) m->nTiles + 1));
    CG_TRY(m->alloc(&aux, 4));
    CG_CHECK_CUDA(cudaMemsetAsync(aux, 0, 4 * sizeof(int), st));
    k_tile_face_start<<<grid_for(m->nF, BLK), BLK, 0, st>>>(m->nF, m->nTiles, m->faceCells, start, aux + 3);
    CG_LAUNCHED();
    k_tile_desc<<<grid_for(m->nTiles, BLK), BLK, 0, st>>>(m->nTiles, m->sell.nSlices, m->sell.slicePtr, start, desc, aux);
    CG_LAUNCHED();
    int h[4];
    CG_CHECK_CUDA(cudaMemcpyAsync(h, aux, sizeof(h), cudaMemcpyDeviceToHost, st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    if (h[3] != 0 || h[2] > 255) return CUPCFD_E_SUCCESS;  // faces not by owner tile, or too wide a slice
    int dev = 0, sms = 0;
    CG_CHECK_CUDA(cudaGetDevice(&dev));
    CG_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // prefetch one wave of resident blocks ahead (the block that will take
    // this block's place), the best distance measured; each kernel's own
    // wave (the gradient adjoint holds more blocks per SM than the forward:
    // 0.345 ms at its 740-tile wave against 0.359 ms at the forward's 592 at
    // 256^3)
    // CUPCFD_FULL_WIDTH=0 keeps the general kernels on hexahedral meshes
    // (identical results), for comparisons
    const char *fw = std::getenv("CUPCFD_FULL_WIDTH");
    m->fullWidth = m->sell.width == 6 && (int64_t) m->nInc == 6 * (int64_t) m->nC &&
                   !(fw && std::strcmp(fw, "0") == 0) ? 6 : 0;
    const bool w6 = full_width(m) == 6;
    const void *pfKern[] = {
        w6 ? (const void *) k_fwd_f32_pf<6> : (const void *) k_fwd_f32_pf<0>,
        w6 ? (const void *) k_adj_f32_pf<6> : (const void *) k_adj_f32_pf<0>,
        w6 ? (const void *) k_fwd_f64_pf<6> : (const void *) k_fwd_f64_pf<0>,
        w6 ? (const void *) k_adj_f64_pf<6> : (const void *) k_adj_f64_pf<0>,
        w6 ? (const void *) k_fwd_madj_f32_pf<6> : (const void *) k_fwd_madj_f32_pf<0>,
        w6 ? (const void *) k_gadj_f32_pf<6> : (const void *) k_gadj_f32_pf<0>,
        w6 ? (const void *) k_madj_f32_pf<6> : (const void *) k_madj_f32_pf<0>};
    static_assert(sizeof(pfKern) / sizeof(pfKern[0]) == PF_COUNT, "one kernel per PfKernel");
    static_assert(PF_COUNT <= (int) (sizeof(m->prefetchWave) / sizeof(m->prefetchWave[0])), "room for every wave");
    // block sizes: 64 threads (TileBlock) for the forward kernels and the
    // FP32 adjoint, 256 (one tile) for the FP64 adjoint and the adjoint parts
    const int pfBlock[PF_COUNT] = {CUPCFD_FWD_BLOCK,      CUPCFD_FWD_BLOCK, CUPCFD_FWD_BLOCK, TILE_CELLS,
                                   CUPCFD_FWD_MADJ_BLOCK, TILE_CELLS,       TILE_CELLS};
    // prefetch distance in waves, in quarters, measured at 256^3 (same box):
    // 1.25 waves for the forward+mass adjoint (0.538 ms against 0.546 at 1
    // wave, 0.541 at 1.5, 0.581 at 0.75), the separate FP32 forward and
    // adjoint (0.491 / 0.528 against 0.492 / 0.531), the FP64 forward (0.706
    // against 0.720) and the mass-only adjoint; 1 wave for the gradient
    // adjoint (equal) and the FP64 adjoint (0.84 against 0.81 ms)
    int pfQuarters[PF_COUNT] = {5, 5, 5, 4, 5, 4, 5};
    // CUPCFD_PREFETCH_QUARTERS=q sets every kernel's distance to q/4 waves
    if (const char *e = std::getenv("CUPCFD_PREFETCH_QUARTERS"))
        if (*e)
            for (int &q : pfQuarters) q = std::max(1, std::atoi(e));
    for (int i = 0; i < PF_COUNT; i++) {
        int nb = 0;
        CG_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, pfKern[i], pfBlock[i], 0));
        m->prefetchWave[i] = sms * std::max(1, nb * pfBlock[i] / TILE_CELLS) * pfQuarters[i] / 4;  // in tiles
    }
    m->prefetchDist = m->prefetchWave[PF_FWD_F32];
    if (const char *e = std::getenv("CUPCFD_PREFETCH_DIST"))
        if (*e) {
            m->prefetchDist = std::max(1, std::atoi(e));
            for (int &w : m->prefetchWave) w = m->prefetchDist;
        }
    // CUPCFD_TILE_MODE=0 keeps the plain kernels (identical results), for comparisons
    const char *e = std::getenv("CUPCFD_TILE_MODE");
    m->tiles = !(e && std::strcmp(e, "0") == 0);
    return CUPCFD_E_SUCCESS;
}

PrefetchArgs prefetch_args(const cupcfd_gpu_mesh *m, int kernel = -1) {
    PrefetchArgs p;
    p.desc = (const TileDesc *) m->tileDesc;
    p.inc = m->sell.inc;
    p.nC = m->nC;
    p.nF = m->nF;
    p.nTiles = m->nTiles;
    p.dist = kernel >= 0 && m->prefetchWave[kernel] > 0 ? m->prefetchWave[kernel] : m->prefetchDist;
    return p;
}


// allowRef: the gradient calls also take CUPCFD_PREC_F32REF (FP32 geometry)
int check_prec(const cupcfd_gpu_mesh *m, int precision, bool allowRef = false) {
    CG_RETURN_IF(precision != CUPCFD_PREC_F64 && precision != CUPCFD_PREC_F32C &&
                     !(allowRef && precision == CUPCFD_PREC_F32REF),
                 CUPCFD_E_CONFIG_INVALID_VALUE, "unknown precision");
    const int geom = precision == CUPCFD_PREC_F32REF ? CUPCFD_PREC_F32C : precision;
    CG_RETURN_IF(!(m->precisions & (1 << geom)), CUPCFD_E_CONFIG_INVALID_VALUE,
                 "the mesh was created without this precision's geometry");
    return CUPCFD_E_SUCCESS;
}

// Device arrays must be aligned to their element: T for scalars and vector
// blocks, 16 bytes for the F32C float4 state (8 for the F64 state blocks).
int check_align(int precision, std::initializer_list<const void *> arrays, std::initializer_list<const void *> states) {
    uintptr_t a = precision == CUPCFD_PREC_F64 ? 8 : 4, sa = precision == CUPCFD_PREC_F64 ? 8 : 16;
    for (const void *p : arrays)
        CG_RETURN_IF(((uintptr_t) p) % a != 0, CUPCFD_E_CONFIG_INVALID_VALUE,
                     "device array not aligned to its element size");
    for (const void *p : states)
        CG_RETURN_IF(((uintptr_t) p) % sa != 0, CUPCFD_E_CONFIG_INVALID_VALUE,
                     precision == CUPCFD_PREC_F64 ? "state array not 8-byte aligned"
                                                  : "F32C state (float4 records) not 16-byte aligned");
    return CUPCFD_E_SUCCESS;
}

// ---------------------------------------------------------------------------
// one gradient iteration (device, internal numbering). corr: add the
// non-orthogonal correction of the previous iterate `prev` (which must not
// alias `grad`); gcopy (optional) receives a copy of the result.
// ---------------------------------------------------------------------------
int launch_grad_once(cupcfd_gpu_mesh *m, int precision, bool corr, bool sgn, const void *phi, const void *phiB,
                     const void *prev, void *grad, void *gcopy, cudaStream_t st) {
    int64_t ldc = m->nC;
    unsigned grid = grid_for(m->nC, BLK);
    if (precision == CUPCFD_PREC_F64) {
        const double *pp = (const double *) phi, *pb = (const double *) phiB, *go = (const double *) prev;
        double *g = (double *) grad, *gc = (double *) gcopy;
        if (!corr && !sgn) k_grad_f64<false, false><<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg64, m->fc64, m->cc64, pp, pb, m->vol, go, g, gc, ldc);
        else if (!corr && sgn) k_grad_f64<false, true><<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg64, m->fc64, m->cc64, pp, pb, m->vol, go, g, gc, ldc);
        else if (corr && !sgn) k_grad_f64<true, false><<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg64, m->fc64, m->cc64, pp, pb, m->vol, go, g, gc, ldc);
        else k_grad_f64<true, true><<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg64, m->fc64, m->cc64, pp, pb, m->vol, go, g, gc, ldc);
    } else if (precision == CUPCFD_PREC_F32REF) {
        const float *pp = (const float *) phi, *pb = (const float *) phiB, *go = (const float *) prev;
        float *g = (float *) grad, *gc = (float *) gcopy;
        if (!corr && !sgn) k_grad_f32ref<false, false><<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg32, m->fc32, m->cc32, pp, pb, m->vol, go, g, gc, ldc);
        else if (!corr && sgn) k_grad_f32ref<false, true><<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg32, m->fc32, m->cc32, pp, pb, m->vol, go, g, gc, ldc);
        else if (corr && !sgn) k_grad_f32ref<true, false><<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg32, m->fc32, m->cc32, pp, pb, m->vol, go, g, gc, ldc);
        else k_grad_f32ref<true, true><<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg32, m->fc32, m->cc32, pp, pb, m->vol, go, g, gc, ldc);
    } else {
        const float *pp = (const float *) phi, *pb = (const float *) phiB, *go = (const float *) prev;
        float *g = (float *) grad, *gc = (float *) gcopy;
        if (!corr && !sgn) k_grad_f32<false, false><<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg32, m->fc32, m->cc32, pp, pb, m->vol, go, g, gc, ldc);
        else if (!corr && sgn) k_grad_f32<false, true><<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg32, m->fc32, m->cc32, pp, pb, m->vol, go, g, gc, ldc);
        else if (corr && !sgn) k_grad_f32<true, false><<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg32, m->fc32, m->cc32, pp, pb, m->vol, go, g, gc, ldc);
        else k_grad_f32<true, true><<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg32, m->fc32, m->cc32, pp, pb, m->vol, go, g, gc, ldc);
    }
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}

}  // namespace

namespace cupcfd_gpu {
int mesh_post_build(cupcfd_gpu_mesh *m, cudaStream_t st) {
    int nC = m->nC;
    int *bw;
    CG_TRY(scratch(m, S_ERR, 1, &bw));
    CG_CHECK_CUDA(cudaMemsetAsync(bw, 0, sizeof(int), st));
    k_bandwidth<<<grid_for(nC, BLK), BLK, 0, st>>>(nC, sell(m), bw);
    CG_LAUNCHED();
    CG_CHECK_CUDA(cudaMemcpyAsync(&m->bandwidth, bw, sizeof(int), cudaMemcpyDeviceToHost, st));
    CG_TRY(tiles_setup(m, st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    return CUPCFD_E_SUCCESS;
}
}  // namespace cupcfd_gpu

extern "C" int cupcfd_gpu_mesh_check_status(cupcfd_gpu_mesh *m, void *stream) {
    clear_error();
    CG_RETURN_IF(!m, CUPCFD_E_NULL_PTR, "check_status: null mesh");
    CG_TRY(make_device_current(m->device));
    CG_CHECK_CUDA(cudaStreamSynchronize(as_stream(stream)));
    CG_CHECK_CUDA(cudaGetLastError());
    return CUPCFD_E_SUCCESS;
}

// ===========================================================================
// device-resident calls
// ===========================================================================
extern "C" int cupcfd_gpu_dev_permute_cells(const cupcfd_gpu_mesh *m, int32_t to_internal, int32_t ncomp, const void *src,
                                            int32_t src_size, int64_t src_cs, void *dst, int32_t dst_size, int64_t dst_cs,
                                            void *stream) {
    clear_error();
    CG_RETURN_IF(!m || !src || !dst, CUPCFD_E_NULL_PTR, "permute_cells: null argument");
    CG_RETURN_IF((src_size != 4 && src_size != 8) || (dst_size != 4 && dst_size != 8) || ncomp <= 0,
                 CUPCFD_E_CONFIG_INVALID_VALUE, "permute_cells: element size must be 4 or 8");
    CG_RETURN_IF(src == dst, CUPCFD_E_CONFIG_INVALID_VALUE, "permute_cells: in-place permutation is not supported");
    int64_t ss = src_cs ? src_cs / src_size : m->nC, dsd = dst_cs ? dst_cs / dst_size : m->nC;
    const int *map = to_internal ? m->cellN2O : m->cellO2N;
    cudaStream_t st = as_stream(stream);
    unsigned grid = grid_for(m->nC, BLK);
    if (src_size == 8 && dst_size == 8) k_gather<double, double><<<grid, BLK, 0, st>>>(m->nC, ncomp, map, (const double *) src, ss, (double *) dst, dsd);
    else if (src_size == 8) k_gather<double, float><<<grid, BLK, 0, st>>>(m->nC, ncomp, map, (const double *) src, ss, (float *) dst, dsd);
    else if (dst_size == 8) k_gather<float, double><<<grid, BLK, 0, st>>>(m->nC, ncomp, map, (const float *) src, ss, (double *) dst, dsd);
    else k_gather<float, float><<<grid, BLK, 0, st>>>(m->nC, ncomp, map, (const float *) src, ss, (float *) dst, dsd);
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_dev_permute_faces(const cupcfd_gpu_mesh *m, int32_t to_internal, const void *src, int32_t src_size,
                                            void *dst, int32_t dst_size, void *stream) {
    clear_error();
    CG_RETURN_IF(!m || !src || !dst, CUPCFD_E_NULL_PTR, "permute_faces: null argument");
    CG_RETURN_IF((src_size != 4 && src_size != 8) || (dst_size != 4 && dst_size != 8), CUPCFD_E_CONFIG_INVALID_VALUE,
                 "permute_faces: element size must be 4 or 8");
    CG_RETURN_IF(src == dst, CUPCFD_E_CONFIG_INVALID_VALUE, "permute_faces: in-place permutation is not supported");
    const int *map = to_internal ? m->faceN2O : m->faceO2N;
    cudaStream_t st = as_stream(stream);
    unsigned grid = grid_for(m->nF, BLK);
    if (src_size == 8 && dst_size == 8) k_gather<double, double><<<grid, BLK, 0, st>>>(m->nF, 1, map, (const double *) src, 0, (double *) dst, 0);
    else if (src_size == 8) k_gather<double, float><<<grid, BLK, 0, st>>>(m->nF, 1, map, (const double *) src, 0, (float *) dst, 0);
    else if (dst_size == 8) k_gather<float, double><<<grid, BLK, 0, st>>>(m->nF, 1, map, (const float *) src, 0, (double *) dst, 0);
    else k_gather<float, float><<<grid, BLK, 0, st>>>(m->nF, 1, map, (const float *) src, 0, (float *) dst, 0);
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_dev_gradient(cupcfd_gpu_mesh *m, int32_t precision, int32_t nGradient, int32_t sign_mode,
                                       const void *phi, const void *phiB, void *grad, void *grad_o, void *stream) {
    clear_error();
    CG_RETURN_IF(!m, CUPCFD_E_NULL_PTR, "dev_gradient: null mesh");
    CG_TRY(check_prec(m, precision, true));
    CG_RETURN_IF(sign_mode != CUPCFD_SIGN_REFERENCE && sign_mode != CUPCFD_SIGN_SIGNED, CUPCFD_E_CONFIG_INVALID_VALUE,
                 "unknown sign_mode");
    CG_RETURN_IF(!phi || !grad || (m->nB > 0 && !phiB), CUPCFD_E_NULL_PTR, "dev_gradient: null device pointer");
    CG_TRY(check_align(precision, {phi, phiB, grad, grad_o}, {}));
    cudaStream_t st = as_stream(stream);
    size_t es = precision == CUPCFD_PREC_F64 ? 8 : 4;
    size_t bytes = 3 * (size_t) m->nC * es;
    bool sgn = sign_mode == CUPCFD_SIGN_SIGNED;
    if (nGradient <= 0) {
        // GradientKernels.ipp:57-61: the previous-iterate array is zeroed, the gradient untouched
        if (grad_o) CG_CHECK_CUDA(cudaMemsetAsync(grad_o, 0, bytes, st));
        return CUPCFD_E_SUCCESS;
    }
    // first iteration: the previous iterate is zero, so the correction is exactly +0 and skipped
    CG_TRY(launch_grad_once(m, precision, false, sgn, phi, phiB, nullptr, grad, nGradient == 1 ? grad_o : nullptr, st));
    if (nGradient > 1) {
        // later iterations read the previous iterate from a separate copy so
        // no launch reads the buffer it writes
        char *prev;
        CG_TRY(scratch(m, S_GO, bytes, &prev));
        for (int it = 1; it < nGradient; it++) {
            CG_CHECK_CUDA(cudaMemcpyAsync(prev, grad, bytes, cudaMemcpyDeviceToDevice, st));
            CG_TRY(launch_grad_once(m, precision, true, sgn, phi, phiB, prev, grad, nullptr, st));
        }
        if (grad_o) CG_CHECK_CUDA(cudaMemcpyAsync(grad_o, grad, bytes, cudaMemcpyDeviceToDevice, st));
    }
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_dev_mass_plain(cupcfd_gpu_mesh *m, int32_t precision, const void *state, void *massFlux, void *stream) {
    clear_error();
    CG_RETURN_IF(!m || !state || !massFlux, CUPCFD_E_NULL_PTR, "dev_mass_plain: null argument");
    CG_TRY(check_prec(m, precision));
    CG_TRY(check_align(precision, {massFlux}, {state}));
    cudaStream_t st = as_stream(stream);
    if (precision == CUPCFD_PREC_F64)
        k_mass_plain_f64<<<grid_for(m->nF, BLK), BLK, 0, st>>>(m->nF, m->faceCells, m->fg64, (const double *) state, m->nC, (double *) massFlux);
    else
        k_mass_plain_f32<<<grid_for(m->nF, BLK), BLK, 0, st>>>(m->nF, m->faceCells, m->fg32, (const float4 *) state, (float *) massFlux);
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_dev_gradient_adjoint(cupcfd_gpu_mesh *m, int32_t precision, int32_t sign_mode, const void *gbar,
                                               void *phiBar, void *phiBBar, void *stream) {
    clear_error();
    CG_RETURN_IF(!m || !gbar || !phiBar || (m->nB > 0 && !phiBBar), CUPCFD_E_NULL_PTR, "dev_gradient_adjoint: null argument");
    CG_TRY(check_prec(m, precision));
    CG_TRY(check_align(precision, {gbar, phiBar, phiBBar}, {}));
    CG_RETURN_IF(sign_mode != CUPCFD_SIGN_REFERENCE && sign_mode != CUPCFD_SIGN_SIGNED, CUPCFD_E_CONFIG_INVALID_VALUE,
                 "unknown sign_mode");
    cudaStream_t st = as_stream(stream);
    unsigned grid = grid_for(m->nC, BLK);
    bool sgn = sign_mode == CUPCFD_SIGN_SIGNED;
    if (precision == CUPCFD_PREC_F64) {
        if (sgn) k_grad_adj_general<true, double><<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg64, nullptr, m->vol, (const double *) gbar, (double *) phiBar, (double *) phiBBar, m->nC);
        else k_grad_adj_general<false, double><<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg64, nullptr, m->vol, (const double *) gbar, (double *) phiBar, (double *) phiBBar, m->nC);
    } else {
        if (sgn) k_grad_adj_general<true, float><<<grid, BLK, 0, st>>>(m->nC, sell(m), nullptr, m->fg32, m->vol, (const float *) gbar, (float *) phiBar, (float *) phiBBar, m->nC);
        else k_grad_adj_general<false, float><<<grid, BLK, 0, st>>>(m->nC, sell(m), nullptr, m->fg32, m->vol, (const float *) gbar, (float *) phiBar, (float *) phiBBar, m->nC);
    }
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_dev_mass_plain_adjoint(cupcfd_gpu_mesh *m, int32_t precision, const void *state, const void *mbar,
                                                 void *stateBar, void *stream) {
    clear_error();
    CG_RETURN_IF(!m || !state || !mbar || !stateBar, CUPCFD_E_NULL_PTR, "dev_mass_plain_adjoint: null argument");
    CG_TRY(check_prec(m, precision));
    CG_TRY(check_align(precision, {mbar}, {state, stateBar}));
    cudaStream_t st = as_stream(stream);
    unsigned grid = grid_for(m->nC, BLK);
    if (precision == CUPCFD_PREC_F64)
        k_adj_f64<<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg64, nullptr, 0.0, (const double *) state,
                                        (const double *) mbar, nullptr, nullptr, (double *) stateBar, m->nC);
    else
        k_adj_f32<<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg32, nullptr, 0.f, (const float4 *) state,
                                        (const float *) mbar, nullptr, nullptr, (float4 *) stateBar, m->nC);
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}

namespace {
// FP32 forward: the L2-prefetch kernel when the mesh has tile ranges and the
// arrays start on 16-byte boundaries, else the plain one (identical results).
// One launch either way; the caller checks it. part: the loss partials, or
// null: one per warp (TILE_CELLS / 32 per tile, warp-major; *group set to
// that) from the L2-prefetch kernel, one per 256-cell tile (*group 1) from
// the plain one; room for TILE_CELLS / 32 per tile either way.
const char *launch_fwd_f32(const cupcfd_gpu_mesh *m, const void *phi, const void *phiB, const void *state,
                           const void *gface, void *grad, void *massFlux, double *part, cudaStream_t st,
                           int *group) {
    *group = 1;
    if (m->tiles && aligned16(phi) && aligned16(state) && (!gface || aligned16(gface))) {
        CG_LAUNCH_PF_BLOCK(m, k_fwd_f32_pf, grid_for(m->nC, BLK) * (TILE_CELLS / CUPCFD_FWD_BLOCK), CUPCFD_FWD_BLOCK,
                           st, m->nC, sell(m), m->fg32, (const float *) phi, (const float *) phiB, m->vol,
                           (const float4 *) state, (const float *) gface, (float *) grad, (float *) massFlux, part,
                           m->nC, prefetch_args(m, PF_FWD_F32));
        *group = TILE_CELLS / 32;
        return "k_fwd_f32_pf";
    }
    k_fwd_f32<BLK><<<grid_for(m->nC, BLK), BLK, 0, st>>>(m->nC, sell(m), m->fg32, (const float *) phi,
                                                         (const float *) phiB, m->vol, (const float4 *) state,
                                                         (const float *) gface, (float *) grad, (float *) massFlux,
                                                         part, m->nC);
    return "k_fwd_f32";
}

// FP64 forward: the L2-prefetch kernel when the tile ranges exist and the
// arrays allow whole 16-byte ranges (state blocks of an even cell count),
// else the plain one. Identical results.
const char *launch_fwd_f64(const cupcfd_gpu_mesh *m, const void *phi, const void *phiB, const void *state,
                           const void *gface, void *grad, void *massFlux, double *part, cudaStream_t st,
                           int *group) {
    *group = 1;
    if (m->tiles && aligned16(phi) && aligned16(state) && (!gface || aligned16(gface)) &&
        m->nC % 2 == 0) {
        CG_LAUNCH_PF_BLOCK(m, k_fwd_f64_pf, grid_for(m->nC, BLK) * (TILE_CELLS / CUPCFD_FWD_BLOCK), CUPCFD_FWD_BLOCK,
                           st, m->nC, sell(m), m->fg64, (const double *) phi, (const double *) phiB, m->vol,
                           (const double *) state, (const double *) gface, (double *) grad, (double *) massFlux,
                           part, m->nC, prefetch_args(m, PF_FWD_F64));
        *group = TILE_CELLS / 32;
        return "k_fwd_f64_pf";
    }
    k_fwd_f64<BLK><<<grid_for(m->nC, BLK), BLK, 0, st>>>(m->nC, sell(m), m->fg64, (const double *) phi,
                                                         (const double *) phiB, m->vol, (const double *) state,
                                                         (const double *) gface, (double *) grad, (double *) massFlux,
                                                         part, m->nC);
    return "k_fwd_f64";
}
}  // namespace

extern "C" int cupcfd_gpu_dev_forward(cupcfd_gpu_mesh *m, int32_t precision, const void *phi, const void *phiB,
                                      const void *state, const void *gface, void *grad, void *massFlux, double *loss,
                                      void *stream) {
    clear_error();
    CG_RETURN_IF(!m || !phi || !state || !grad || !massFlux || (m->nB > 0 && !phiB), CUPCFD_E_NULL_PTR,
                 "dev_forward: null argument");
    CG_RETURN_IF((gface == nullptr) != (loss == nullptr), CUPCFD_E_NULL_PTR, "dev_forward: gface and loss go together");
    CG_TRY(check_prec(m, precision));
    CG_TRY(check_align(precision, {phi, phiB, gface, grad, massFlux}, {state}));
    CG_RETURN_IF(((uintptr_t) loss) % 8 != 0, CUPCFD_E_CONFIG_INVALID_VALUE, "dev_forward: loss not 8-byte aligned");
    cudaStream_t st = as_stream(stream);
    unsigned grid = grid_for(m->nC, BLK);
    double *part = nullptr;
    if (loss) CG_TRY(scratch(m, S_LOSS, (size_t) grid * (TILE_CELLS / 32), &part));
    int group = 1;
    {
        KernelTimer kt(nullptr, st);
        kt.set_name(precision == CUPCFD_PREC_F64
                        ? launch_fwd_f64(m, phi, phiB, state, gface, grad, massFlux, part, st, &group)
                        : launch_fwd_f32(m, phi, phiB, state, gface, grad, massFlux, part, st, &group));
        CG_LAUNCHED();
    }
    if (loss) {
        // per-warp partials: each tile's value first (many blocks), then the
        // fixed-order sum over tiles; the same bits as per-tile partials
        if (group > 1) {
            KTIMER("k_group_partials", st);
            k_group_partials<TILE_CELLS / 32><<<grid_for(grid, BLK), BLK, 0, st>>>((int) grid, part);
            CG_LAUNCHED();
        }
        KTIMER("k_reduce_partials", st);
        k_reduce_partials<<<1, 1024, 0, st>>>((int) grid, part, loss);
        CG_LAUNCHED();
    }
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_dev_adjoint(cupcfd_gpu_mesh *m, int32_t precision, const void *grad, const void *state,
                                      const void *gface, void *phiBar, void *phiBBar, void *stateBar, void *stream) {
    clear_error();
    CG_RETURN_IF(!m || !grad || !state || !gface || !phiBar || !stateBar || (m->nB > 0 && !phiBBar), CUPCFD_E_NULL_PTR,
                 "dev_adjoint: null argument");
    CG_TRY(check_prec(m, precision));
    CG_TRY(check_align(precision, {grad, gface, phiBar, phiBBar}, {state, stateBar}));
    cudaStream_t st = as_stream(stream);
    unsigned grid = grid_for(m->nC, BLK);
    KernelTimer kt(nullptr, st);
    if (precision == CUPCFD_PREC_F64 && m->tiles && aligned16(grad) && aligned16(state) &&
        aligned16(gface) && m->nC % 2 == 0) {
        kt.set_name("k_adj_f64_pf");
        CG_LAUNCH_PF(m, k_adj_f64_pf, grid, st, m->nC, sell(m), m->fg64, (const double *) grad, 2.0,
                     (const double *) state, (const double *) gface, (double *) phiBar, (double *) phiBBar,
                     (double *) stateBar, m->nC, prefetch_args(m, PF_ADJ_F64));
    } else if (precision == CUPCFD_PREC_F64) {
        kt.set_name("k_adj_f64");
        k_adj_f64<<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg64, (const double *) grad, 2.0, (const double *) state,
                                        (const double *) gface, (double *) phiBar, (double *) phiBBar, (double *) stateBar, m->nC);
    } else if (m->tiles && aligned16(grad) && aligned16(state) && aligned16(gface) && m->nC % 4 == 0) {
        kt.set_name("k_adj_f32_pf");
        CG_LAUNCH_PF_BLOCK(m, k_adj_f32_pf, grid * (TILE_CELLS / CUPCFD_FWD_BLOCK), CUPCFD_FWD_BLOCK, st, m->nC,
                           sell(m), m->fg32, (const float *) grad, 2.f, (const float4 *) state, (const float *) gface,
                           (float *) phiBar, (float *) phiBBar, (float4 *) stateBar, m->nC,
                           prefetch_args(m, PF_ADJ_F32));
    } else {
        kt.set_name("k_adj_f32");
        k_adj_f32<<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg32, (const float *) grad, 2.f, (const float4 *) state,
                                        (const float *) gface, (float *) phiBar, (float *) phiBBar, (float4 *) stateBar, m->nC);
    }
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_dev_forward_adjoint(cupcfd_gpu_mesh *m, int32_t precision, const void *phi, const void *phiB,
                                              const void *state, const void *gface, void *grad, void *massFlux,
                                              void *phiBar, void *phiBBar, void *stateBar, double *loss, void *stream) {
    clear_error();
    CG_RETURN_IF(!m || !gface, CUPCFD_E_NULL_PTR, "dev_forward_adjoint: null argument");
    double *lp = loss;
    if (!lp) CG_TRY(scratch(m, S_NORM, 1, &lp));
    CG_TRY(check_prec(m, precision));
    if (precision == CUPCFD_PREC_F32C && m->tiles && aligned16(phi) && aligned16(state) &&
        aligned16(gface) && aligned16(grad) && aligned16(stateBar) && m->nC % 4 == 0) {
        // forward with the mass-flux adjoint, then the gradient adjoint: the
        // state and gface stream through one pass only
        CG_RETURN_IF(!phi || !state || !grad || !massFlux || !phiBar || !stateBar || (m->nB > 0 && (!phiB || !phiBBar)),
                     CUPCFD_E_NULL_PTR, "dev_forward_adjoint: null argument");
        CG_TRY(check_align(precision, {phi, phiB, gface, grad, massFlux, phiBar, phiBBar}, {state, stateBar}));
        CG_RETURN_IF(((uintptr_t) lp) % 8 != 0, CUPCFD_E_CONFIG_INVALID_VALUE, "dev_forward_adjoint: loss not 8-byte aligned");
        cudaStream_t st = as_stream(stream);
        unsigned grid = grid_for(m->nC, BLK);
        // one loss partial per warp: TILE_CELLS / 32 per tile
        constexpr int WPT = TILE_CELLS / 32;
        double *part;
        CG_TRY(scratch(m, S_LOSS, (size_t) grid * WPT, &part));
        CG_TRY(pipe_init(m));
        PrefetchArgs pf = prefetch_args(m, PF_FWD_MADJ), pfg = prefetch_args(m, PF_GADJ);
        {
            KTIMER("k_fwd_madj_f32_pf", st);
            CG_LAUNCH_PF_BLOCK(m, k_fwd_madj_f32_pf, grid * (TILE_CELLS / CUPCFD_FWD_MADJ_BLOCK), CUPCFD_FWD_MADJ_BLOCK,
                         st, m->nC, sell(m), m->fg32, (const float *) phi,
                         (const float *) phiB, m->vol, (const float4 *) state, (const float *) gface, (float *) grad,
                         (float *) massFlux, (float4 *) stateBar, part, m->nC, pf);
            CG_LAUNCHED();
        }
        {
            // the FP64 loss reduction (one block) runs on the mesh's second
            // stream beside the gradient adjoint, which does not need it;
            // the caller's stream waits for both
            cudaStream_t so = m->outStream;
            CG_CHECK_CUDA(cudaEventRecord(m->pipeEv[0], st));
            CG_CHECK_CUDA(cudaStreamWaitEvent(so, m->pipeEv[0], 0));
            KTIMER("k_reduce_partials", so);
            k_reduce_partials<WPT><<<1, 1024, 0, so>>>((int) grid, part, lp);
            CG_LAUNCHED();
        }
        CG_CHECK_CUDA(cudaEventRecord(m->pipeEv[1], m->outStream));
        {
            KTIMER("k_gadj_f32_pf", st);
            CG_LAUNCH_PF(m, k_gadj_f32_pf, grid, st, m->nC, sell(m), m->fg32, (const float *) grad, 2.f,
                         (float *) phiBar, (float *) phiBBar, m->nC, pfg);
            CG_LAUNCHED();
        }
        CG_CHECK_CUDA(cudaStreamWaitEvent(st, m->pipeEv[1], 0));
        return CUPCFD_E_SUCCESS;
    }
    CG_TRY(cupcfd_gpu_dev_forward(m, precision, phi, phiB, state, gface, grad, massFlux, lp, stream));
    return cupcfd_gpu_dev_adjoint(m, precision, grad, state, gface, phiBar, phiBBar, stateBar, stream);
}

// ---------------------------------------------------------------------------
// error norms (FP64)
// ---------------------------------------------------------------------------
namespace {
template <class TA, class TB>
__global__ void k_norms(int64_t n, const TA *__restrict__ a, const TB *__restrict__ b, double floor, double *__restrict__ part) {
    __shared__ double sh[5][256 / 32];
    double mx = 0, mb = 0, s2 = 0, b2 = 0, mr = 0;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
        double x = (double) a[i], y = (double) b[i], d = fabs(x - y);
        mx = fmax(mx, d);
        mb = fmax(mb, fabs(y));
        s2 += d * d;
        b2 += y * y;
        mr = fmax(mr, d / fmax(fabs(y), floor));
    }
    for (int k = 16; k > 0; k >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, k));
        mb = fmax(mb, __shfl_xor_sync(0xffffffffu, mb, k));
        s2 += __shfl_xor_sync(0xffffffffu, s2, k);
        b2 += __shfl_xor_sync(0xffffffffu, b2, k);
        mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, k));
    }
    int wq = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { sh[0][wq] = mx; sh[1][wq] = mb; sh[2][wq] = s2; sh[3][wq] = b2; sh[4][wq] = mr; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r[5] = {0, 0, 0, 0, 0};
        for (int i = 0; i < (int) blockDim.x / 32; i++) {
            r[0] = fmax(r[0], sh[0][i]); r[1] = fmax(r[1], sh[1][i]);
            r[2] += sh[2][i]; r[3] += sh[3][i]; r[4] = fmax(r[4], sh[4][i]);
        }
        for (int k = 0; k < 5; k++) part[5 * blockIdx.x + k] = r[k];
    }
}
}  // namespace

extern "C" int cupcfd_gpu_dev_error_norms(const void *a, int32_t as, const void *b, int32_t bs, int64_t n, double floor,
                                          double *out, void *stream) {
    clear_error();
    CG_RETURN_IF(!a || !b || !out, CUPCFD_E_NULL_PTR, "error_norms: null argument");
    CG_RETURN_IF((as != 4 && as != 8) || (bs != 4 && bs != 8), CUPCFD_E_CONFIG_INVALID_VALUE, "error_norms: size 4 or 8");
    cudaStream_t st = as_stream(stream);
    const int blocks = 592;
    double *part;
    CG_CHECK_CUDA(cudaMallocAsync((void **) &part, sizeof(double) * 5 * blocks, st));
    if (as == 8 && bs == 8) k_norms<double, double><<<blocks, 256, 0, st>>>(n, (const double *) a, (const double *) b, floor, part);
    else if (as == 8) k_norms<double, float><<<blocks, 256, 0, st>>>(n, (const double *) a, (const float *) b, floor, part);
    else if (bs == 8) k_norms<float, double><<<blocks, 256, 0, st>>>(n, (const float *) a, (const double *) b, floor, part);
    else k_norms<float, float><<<blocks, 256, 0, st>>>(n, (const float *) a, (const float *) b, floor, part);
    CG_LAUNCHED();
    std::vector<double> h(5 * blocks);
    CG_CHECK_CUDA(cudaMemcpyAsync(h.data(), part, sizeof(double) * 5 * blocks, cudaMemcpyDeviceToHost, st));
    CG_CHECK_CUDA(cudaFreeAsync(part, st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    double r[5] = {0, 0, 0, 0, 0};
    for (int i = 0; i < blocks; i++) {
        r[0] = std::max(r[0], h[5 * i]); r[1] = std::max(r[1], h[5 * i + 1]);
        r[2] += h[5 * i + 2]; r[3] += h[5 * i + 3]; r[4] = std::max(r[4], h[5 * i + 4]);
    }
    for (int k = 0; k < 5; k++) out[k] = r[k];
    return CUPCFD_E_SUCCESS;
}

// ===========================================================================
// reference-facing calls (host buffers)
// ===========================================================================
namespace {

int h2d_real(cupcfd_gpu_mesh *m, int slot, const void *h, int64_t n, int rs, void **dptr) {
    void *d;
    CG_TRY(m->scratchBuf(slot, (size_t) std::max<int64_t>(n, 1) * rs, &d));
    if (n > 0) CG_CHECK_CUDA(cudaMemcpyAsync(d, h, (size_t) n * rs, cudaMemcpyHostToDevice, m->stream));
    *dptr = d;
    return CUPCFD_E_SUCCESS;
}

// strided host vec3 view -> packed device [3n] of rs bytes (strided.cuh)
int h2d_vec3(cupcfd_gpu_mesh *m, int slot, const cupcfd_vec3_view &v, int64_t n, int rs, void **dptr) {
    CG_RETURN_IF(!v.base, CUPCFD_E_NULL_PTR, "null vector array");
    CG_RETURN_IF(v.stride < 3 * rs || v.offset < 0 || v.offset + 3 * rs > v.stride, CUPCFD_E_CONFIG_INVALID_VALUE,
                 "vector view: bad stride/offset");
    void *d, *span = nullptr;
    CG_TRY(m->scratchBuf(slot, (size_t) std::max<int64_t>(n, 1) * 3 * rs, &d));
    if (v.stride != 3 * rs) CG_TRY(m->scratchBuf(S_SPAN, std::max<size_t>(vec3_span_bytes(n, v.stride, v.offset, rs), 1), &span));
    CG_TRY(upload_vec3_span(v.base, v.stride, v.offset, n, rs, span, d, m->stream));
    *dptr = d;
    return CUPCFD_E_SUCCESS;
}

// packed device [3n] of rs bytes -> strided host vec3 view (strided.cuh;
// returns once the host records are written unless they are packed)
int d2h_vec3(cupcfd_gpu_mesh *m, const void *d, void *base, int stride, int offset, int64_t n, int rs) {
    return download_vec3_span(d, base, stride, offset, n, rs, m->hostStage, m->stream);
}

void zero_vec3_tail(void *base, int stride, int offset, int from, int to, int rs) {
    for (int i = from; i < to; i++) std::memset((char *) base + (size_t) i * stride + offset, 0, 3 * rs);
}

}  // namespace

extern "C" int cupcfd_gpu_gradient_phi_gauss_dolfyn(cupcfd_gpu_mesh *m, int32_t nGradient, const void *phiCell, int32_t nPhiCell,
                                                    const void *phiBoundary, int32_t nPhiBoundary, void *dPhidxCell,
                                                    int32_t nDPhidxCell, int32_t stride, int32_t offset, void *dPhidxoCell,
                                                    int32_t nDPhidxoCell, int32_t strideo, int32_t offseto,
                                                    int32_t rs, int32_t precision, int32_t sign_mode) {
    clear_error();
    CG_RETURN_IF(!m || !phiCell || !dPhidxCell || !dPhidxoCell || (m->nB > 0 && !phiBoundary), CUPCFD_E_NULL_PTR,
                 "GradientPhiGaussDolfyn: null argument");
    CG_RETURN_IF(rs != 4 && rs != 8, CUPCFD_E_CONFIG_INVALID_VALUE, "GradientPhiGaussDolfyn: real_size must be 4 or 8");
    CG_RETURN_IF(stride < 3 * rs || strideo < 3 * rs || offset < 0 || offseto < 0 || offset + 3 * rs > stride ||
                     offseto + 3 * rs > strideo,
                 CUPCFD_E_CONFIG_INVALID_VALUE, "GradientPhiGaussDolfyn: bad vector stride/offset");
    CG_TRY(check_prec(m, precision, true));
    // the reference reads phiCell[ip/in], phiBoundary[ib] and updates dPhidxCell[0..lTCells)
    // (GradientKernels.ipp:90-95,107-111,122-126); short arrays are index errors
    CG_RETURN_IF(nPhiCell < m->nC || nPhiBoundary < m->nB || nDPhidxCell < m->nC || nDPhidxoCell < 0 ||
                     nDPhidxoCell > nDPhidxCell,
                 CUPCFD_E_INVALID_INDEX, "GradientPhiGaussDolfyn: array shorter than the mesh needs");
    CG_TRY(make_device_current(m->device));
    cudaStream_t st = m->stream;
    int nC = m->nC;
    if (nGradient <= 0) {
        // dPhidxoCell zeroed, dPhidxCell untouched (GradientKernels.ipp:57-61)
        zero_vec3_tail(dPhidxoCell, strideo, offseto, 0, nDPhidxoCell, rs);
        return CUPCFD_E_SUCCESS;
    }
    size_t es = precision == CUPCFD_PREC_F64 ? 8 : 4;
    void *dphiRef, *dphibRef;
    CG_TRY(h2d_real(m, S_IN0, phiCell, nC, rs, &dphiRef));
    CG_TRY(h2d_real(m, S_IN1, phiBoundary, m->nB, rs, &dphibRef));
    void *phi, *phib, *grad, *out;
    CG_TRY(m->scratchBuf(S_IN2, (size_t) nC * es, &phi));
    CG_TRY(m->scratchBuf(S_IN3, (size_t) std::max(m->nB, 1) * es, &phib));
    CG_TRY(m->scratchBuf(S_OUT0, 3 * (size_t) nC * es, &grad));
    CG_TRY(m->scratchBuf(S_OUT1, 3 * (size_t) nC * rs, &out));
    CG_TRY(cupcfd_gpu_dev_permute_cells(m, 1, 1, dphiRef, rs, 0, phi, (int) es, 0, st));
    if (m->nB > 0) {
        if ((size_t) rs == es) CG_CHECK_CUDA(cudaMemcpyAsync(phib, dphibRef, (size_t) m->nB * es, cudaMemcpyDeviceToDevice, st));
        else if (rs == 8) { k_convert<double, float><<<grid_for(m->nB, BLK), BLK, 0, st>>>(m->nB, (const double *) dphibRef, (float *) phib); CG_LAUNCHED(); }
        else { k_convert<float, double><<<grid_for(m->nB, BLK), BLK, 0, st>>>(m->nB, (const float *) dphibRef, (double *) phib); CG_LAUNCHED(); }
    }
    CG_TRY(cupcfd_gpu_dev_gradient(m, precision, nGradient, sign_mode, phi, phib, grad, nullptr, st));
    unsigned grid = grid_for(nC, BLK);
    if (es == 8 && rs == 8) k_blocks_to_aos<double, double><<<grid, BLK, 0, st>>>(nC, 3, m->cellO2N, (const double *) grad, nC, (double *) out);
    else if (es == 8) k_blocks_to_aos<double, float><<<grid, BLK, 0, st>>>(nC, 3, m->cellO2N, (const double *) grad, nC, (float *) out);
    else if (rs == 8) k_blocks_to_aos<float, double><<<grid, BLK, 0, st>>>(nC, 3, m->cellO2N, (const float *) grad, nC, (double *) out);
    else k_blocks_to_aos<float, float><<<grid, BLK, 0, st>>>(nC, 3, m->cellO2N, (const float *) grad, nC, (float *) out);
    CG_LAUNCHED();
    CG_TRY(d2h_vec3(m, out, dPhidxCell, stride, offset, nC, rs));
    if (stride != 3 * rs)  // the packed values are in host staging already: one copy back serves both arrays
        scatter_vec3_host(m->hostStage.data(), dPhidxoCell, strideo, offseto, std::min(nC, nDPhidxoCell), rs);
    else
        CG_TRY(d2h_vec3(m, out, dPhidxoCell, strideo, offseto, std::min(nC, nDPhidxoCell), rs));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    // entries past lTCells: zeroed by the reset loop, copied into dPhidxoCell (:66-70, :129-131)
    zero_vec3_tail(dPhidxCell, stride, offset, nC, nDPhidxCell, rs);
    zero_vec3_tail(dPhidxoCell, strideo, offseto, nC, nDPhidxoCell, rs);
    return CUPCFD_E_SUCCESS;
}

namespace {
// FluxMassDolfynFaceLoop over host arrays of the reference's real type T
// (double: FP64 geometry, bit-identical to T = double; float: the mesh's FP32
// geometry and the float instantiation's arithmetic, k_mass_full_f32ref).
template <class T>
int flux_mass_face_loop_t(
    cupcfd_gpu_mesh *m, cupcfd_vec3_view dudx, int32_t nDudx, cupcfd_vec3_view dvdx, int32_t nDvdx, cupcfd_vec3_view dwdx,
    int32_t nDwdx, cupcfd_vec3_view dpdx, int32_t nDpdx, const T *den, int32_t nDen, T *denB, int32_t nDenB,
    const T *u, int32_t nU, const T *v, int32_t nV, const T *w, int32_t nW, T *massFlux,
    int32_t nMassFlux, const T *p, int32_t nP, const T *ar, int32_t nAr, T *su, int32_t nSu, T *rface,
    int32_t nRFace, T small, int32_t *icinl, int32_t *icout, int32_t *icsym, int32_t *icwal, int32_t solveTurbEnergy,
    int32_t solveTurbDiss, int32_t solveVisc, int32_t solveEnthalpy, const T *teC, int32_t nTeC, T *teB,
    int32_t nTeB, const T *edC, int32_t nEdC, T *edB, int32_t nEdB, const T *visC, int32_t nVisC,
    T *visB, int32_t nVisB, const T *tC, int32_t nTC, T *tB, int32_t nTB) {
    constexpr bool F64 = sizeof(T) == 8;
    CG_RETURN_IF(!m || !den || !u || !v || !w || !massFlux || !p || !ar || !su || !rface || !icinl || !icout || !icsym ||
                     !icwal,
                 CUPCFD_E_NULL_PTR, "FluxMassDolfynFaceLoop: null argument");
    CG_TRY(check_prec(m, F64 ? CUPCFD_PREC_F64 : CUPCFD_PREC_F32C));
    int nC = m->nC, nF = m->nF, nB = m->nB;
    // index checks of the reference's DEBUG build (MassKernels.ipp:101-138, 203-245)
    CG_RETURN_IF(nDudx < nC || nDvdx < nC || nDwdx < nC || nDpdx < nC || nDen < nC || nU < nC || nV < nC || nW < nC ||
                     nP < nC || nAr < nC || nSu < nC || nMassFlux < nF || nRFace < 2 * nF || nDenB < nB,
                 CUPCFD_E_INVALID_INDEX, "FluxMassDolfynFaceLoop: array shorter than the mesh needs");
    bool anyOutlet = false, anyInlet = false;
    for (int t : m->hRegionType) { anyOutlet |= t == CUPCFD_RTYPE_OUTLET; anyInlet |= t == CUPCFD_RTYPE_INLET; }
    const T *bcI[4] = {teC, edC, visC, tC};
    T *bcO[4] = {teB, edB, visB, tB};
    int nbcI[4] = {nTeC, nEdC, nVisC, nTC}, nbcO[4] = {nTeB, nEdB, nVisB, nTB};
    int flags = (solveTurbEnergy ? 1 : 0) | (solveTurbDiss ? 2 : 0) | (solveVisc ? 4 : 0) | (solveEnthalpy ? 8 : 0);
    if (anyOutlet)
        for (int q = 0; q < 4; q++)
            if (flags & (1 << q)) {
                CG_RETURN_IF(!bcI[q] || !bcO[q], CUPCFD_E_NULL_PTR, "FluxMassDolfynFaceLoop: null boundary-copy array");
                CG_RETURN_IF(nbcI[q] < nC || nbcO[q] < nB, CUPCFD_E_INVALID_INDEX, "FluxMassDolfynFaceLoop: boundary-copy array too short");
            }
    CG_TRY(make_device_current(m->device));
    cudaStream_t st = m->stream;
    int64_t ldc = nC;
    unsigned gC = grid_for(nC, BLK), gF = grid_for(nF, BLK);
    // gradients: four packed [3nC] reference arrays -> 12 internal blocks
    T *grads, *cs, *mf, *rf, *suD, *tmp, *bcIn = nullptr, *bcOut = nullptr, *denBD;
    int *cnt;
    CG_TRY(scratch(m, S_IN0, 12 * (size_t) nC, &grads));
    CG_TRY(scratch(m, S_IN1, 6 * (size_t) nC, &cs));
    CG_TRY(scratch(m, S_IN2, 3 * (size_t) std::max(nC, 2 * nF), &tmp));
    CG_TRY(scratch(m, S_OUT0, (size_t) nF, &mf));
    CG_TRY(scratch(m, S_OUT1, 2 * (size_t) nF, &rf));
    CG_TRY(scratch(m, S_OUT2, (size_t) nC, &suD));
    CG_TRY(scratch(m, S_OUT3, (size_t) std::max(nB, 1), &denBD));
    CG_TRY(scratch(m, S_CNT, 4, &cnt));
    cupcfd_vec3_view vv[4] = {dudx, dvdx, dwdx, dpdx};
    for (int q = 0; q < 4; q++) {
        void *d;
        CG_TRY(h2d_vec3(m, S_IN3, vv[q], nC, (int) sizeof(T), &d));
        k_aos_to_blocks<T, T><<<gC, BLK, 0, st>>>(nC, 3, m->cellN2O, (const T *) d, grads + 3 * q * ldc, ldc);
        CG_LAUNCHED();
    }
    const T *cin[6] = {den, u, v, w, p, ar};
    for (int q = 0; q < 6; q++) {
        CG_CHECK_CUDA(cudaMemcpyAsync(tmp, cin[q], sizeof(T) * nC, cudaMemcpyHostToDevice, st));
        k_gather<T, T><<<gC, BLK, 0, st>>>(nC, 1, m->cellN2O, tmp, 0, cs + q * ldc, 0);
        CG_LAUNCHED();
    }
    // in/out arrays: massFlux, rface (faces), su (cells), denB (boundaries)
    CG_CHECK_CUDA(cudaMemcpyAsync(tmp, massFlux, sizeof(T) * nF, cudaMemcpyHostToDevice, st));
    k_gather<T, T><<<gF, BLK, 0, st>>>(nF, 1, m->faceN2O, tmp, 0, mf, 0);
    CG_LAUNCHED();
    CG_CHECK_CUDA(cudaMemcpyAsync(tmp, rface, sizeof(T) * 2 * nF, cudaMemcpyHostToDevice, st));
    k_gather_pairs<T><<<gF, BLK, 0, st>>>(nF, m->faceN2O, tmp, rf);
    CG_LAUNCHED();
    if (anyInlet) {
        CG_CHECK_CUDA(cudaMemcpyAsync(tmp, su, sizeof(T) * nC, cudaMemcpyHostToDevice, st));
        k_gather<T, T><<<gC, BLK, 0, st>>>(nC, 1, m->cellN2O, tmp, 0, suD, 0);
        CG_LAUNCHED();
    }
    if (anyOutlet && nB > 0) {
        CG_CHECK_CUDA(cudaMemcpyAsync(denBD, denB, sizeof(T) * nB, cudaMemcpyHostToDevice, st));
        if (flags) {
            CG_TRY(scratch(m, S_IN4, 4 * (size_t) nC, &bcIn));
            CG_TRY(scratch(m, S_OUT4, 4 * (size_t) nB, &bcOut));
            for (int q = 0; q < 4; q++) {
                if (!(flags & (1 << q))) continue;
                CG_CHECK_CUDA(cudaMemcpyAsync(tmp, bcI[q], sizeof(T) * nC, cudaMemcpyHostToDevice, st));
                k_gather<T, T><<<gC, BLK, 0, st>>>(nC, 1, m->cellN2O, tmp, 0, bcIn + q * ldc, 0);
                CG_LAUNCHED();
                CG_CHECK_CUDA(cudaMemcpyAsync(bcOut + (size_t) q * nB, bcO[q], sizeof(T) * nB, cudaMemcpyHostToDevice, st));
            }
        }
    }
    CG_CHECK_CUDA(cudaMemsetAsync(cnt, 0, 4 * sizeof(int), st));
    if constexpr (F64)
        k_mass_full_f64<<<gF, BLK, 0, st>>>(nF, m->faceCells, m->fg64, m->fc64, m->fxp64, m->fxn64, m->cc64, m->vol, grads, cs,
                                            ldc, m->bndRegion, m->regionType, m->regionUVW, m->regionDen, small, flags, mf, rf,
                                            denBD, bcIn, bcOut, nB, cnt);
    else
        k_mass_full_f32ref<<<gF, BLK, 0, st>>>(nF, m->faceCells, m->fg32, m->fc32, m->fxp64, m->fxn64, m->cc32, m->vol, grads,
                                               cs, ldc, m->bndRegion, m->regionType, m->regionUVW, m->regionDen, small, flags,
                                               mf, rf, denBD, bcIn, bcOut, nB, cnt);
    CG_LAUNCHED();
    if (anyInlet) {
        k_inlet_su<T><<<gC, BLK, 0, st>>>(nC, sell(m), m->bndRegion, m->regionType, mf, suD);
        CG_LAUNCHED();
    }
    // back to reference numbering and to the host
    T *hmf, *hrf;
    CG_TRY(scratch(m, S_IN5, (size_t) nF, &hmf));
    CG_TRY(scratch(m, S_IN6, 2 * (size_t) nF, &hrf));
    k_gather<T, T><<<gF, BLK, 0, st>>>(nF, 1, m->faceO2N, mf, 0, hmf, 0);
    CG_LAUNCHED();
    k_gather_pairs<T><<<gF, BLK, 0, st>>>(nF, m->faceO2N, rf, hrf);
    CG_LAUNCHED();
    CG_CHECK_CUDA(cudaMemcpyAsync(massFlux, hmf, sizeof(T) * nF, cudaMemcpyDeviceToHost, st));
    CG_CHECK_CUDA(cudaMemcpyAsync(rface, hrf, sizeof(T) * 2 * nF, cudaMemcpyDeviceToHost, st));
    if (anyInlet) {
        k_gather<T, T><<<gC, BLK, 0, st>>>(nC, 1, m->cellO2N, suD, 0, tmp, 0);
        CG_LAUNCHED();
        CG_CHECK_CUDA(cudaMemcpyAsync(su, tmp, sizeof(T) * nC, cudaMemcpyDeviceToHost, st));
    }
    if (anyOutlet && nB > 0) {
        CG_CHECK_CUDA(cudaMemcpyAsync(denB, denBD, sizeof(T) * nB, cudaMemcpyDeviceToHost, st));
        for (int q = 0; q < 4; q++)
            if (flags & (1 << q))
                CG_CHECK_CUDA(cudaMemcpyAsync(bcO[q], bcOut + (size_t) q * nB, sizeof(T) * nB, cudaMemcpyDeviceToHost, st));
    }
    int hc[4];
    CG_CHECK_CUDA(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    *icinl += hc[0]; *icout += hc[1]; *icsym += hc[2]; *icwal += hc[3];
    return CUPCFD_E_SUCCESS;
}

}  // namespace

extern "C" int cupcfd_gpu_flux_mass_dolfyn_face_loop(
    cupcfd_gpu_mesh *m, cupcfd_vec3_view dudx, int32_t nDudx, cupcfd_vec3_view dvdx, int32_t nDvdx, cupcfd_vec3_view dwdx,
    int32_t nDwdx, cupcfd_vec3_view dpdx, int32_t nDpdx, const double *den, int32_t nDen, double *denB, int32_t nDenB,
    const double *u, int32_t nU, const double *v, int32_t nV, const double *w, int32_t nW, double *massFlux,
    int32_t nMassFlux, const double *p, int32_t nP, const double *ar, int32_t nAr, double *su, int32_t nSu, double *rface,
    int32_t nRFace, double small, int32_t *icinl, int32_t *icout, int32_t *icsym, int32_t *icwal, int32_t solveTurbEnergy,
    int32_t solveTurbDiss, int32_t solveVisc, int32_t solveEnthalpy, const double *teC, int32_t nTeC, double *teB,
    int32_t nTeB, const double *edC, int32_t nEdC, double *edB, int32_t nEdB, const double *visC, int32_t nVisC,
    double *visB, int32_t nVisB, const double *tC, int32_t nTC, double *tB, int32_t nTB) {
    clear_error();
    return flux_mass_face_loop_t<double>(m, dudx, nDudx, dvdx, nDvdx, dwdx, nDwdx, dpdx, nDpdx, den, nDen, denB, nDenB, u,
                                         nU, v, nV, w, nW, massFlux, nMassFlux, p, nP, ar, nAr, su, nSu, rface, nRFace, small,
                                         icinl, icout, icsym, icwal, solveTurbEnergy, solveTurbDiss, solveVisc, solveEnthalpy,
                                         teC, nTeC, teB, nTeB, edC, nEdC, edB, nEdB, visC, nVisC, visB, nVisB, tC, nTC, tB, nTB);
}

extern "C" int cupcfd_gpu_flux_mass_dolfyn_face_loop_f32(
    cupcfd_gpu_mesh *m, cupcfd_vec3_view dudx, int32_t nDudx, cupcfd_vec3_view dvdx, int32_t nDvdx, cupcfd_vec3_view dwdx,
    int32_t nDwdx, cupcfd_vec3_view dpdx, int32_t nDpdx, const float *den, int32_t nDen, float *denB, int32_t nDenB,
    const float *u, int32_t nU, const float *v, int32_t nV, const float *w, int32_t nW, float *massFlux,
    int32_t nMassFlux, const float *p, int32_t nP, const float *ar, int32_t nAr, float *su, int32_t nSu, float *rface,
    int32_t nRFace, float small, int32_t *icinl, int32_t *icout, int32_t *icsym, int32_t *icwal, int32_t solveTurbEnergy,
    int32_t solveTurbDiss, int32_t solveVisc, int32_t solveEnthalpy, const float *teC, int32_t nTeC, float *teB,
    int32_t nTeB, const float *edC, int32_t nEdC, float *edB, int32_t nEdB, const float *visC, int32_t nVisC,
    float *visB, int32_t nVisB, const float *tC, int32_t nTC, float *tB, int32_t nTB) {
    clear_error();
    return flux_mass_face_loop_t<float>(m, dudx, nDudx, dvdx, nDvdx, dwdx, nDwdx, dpdx, nDpdx, den, nDen, denB, nDenB, u,
                                        nU, v, nV, w, nW, massFlux, nMassFlux, p, nP, ar, nAr, su, nSu, rface, nRFace, small,
                                        icinl, icout, icsym, icwal, solveTurbEnergy, solveTurbDiss, solveVisc, solveEnthalpy,
                                        teC, nTeC, teB, nTeB, edC, nEdC, edB, nEdB, visC, nVisC, visB, nVisB, tC, nTC, tB, nTB);
}


namespace {
// One part of the benchmark adjoint: the gradient part (phibar, phibBar from
// g, hscale 2) when state and gface are null, the mass part (stateBar) when g
// is null and hscale 0. FP32 on tiled meshes with 16-byte aligned arrays: the
// L2-prefetch kernels of each part (k_gadj_f32_pf, k_madj_f32_pf); else the
// plain adjoint kernels. Each output's sum is the one the combined kernels
// form, so the results are theirs.
int launch_adj_part(const cupcfd_gpu_mesh *m, bool f64, const void *g, double hscale, const void *state,
                    const void *gface, void *phiBar, void *phiBBar, void *stateBar, cudaStream_t st) {
    unsigned grid = grid_for(m->nC, BLK);
    const bool gradPart = gface == nullptr;
    KernelTimer kt(nullptr, st);
    if (!f64 && m->tiles && m->nC % 4 == 0 &&
        (gradPart ? hscale == 2.0 && aligned16(g) : hscale == 0.0 && !g && aligned16(state) && aligned16(gface))) {
        kt.set_name(gradPart ? "k_gadj_f32_pf" : "k_madj_f32_pf");
        if (gradPart)
            CG_LAUNCH_PF(m, k_gadj_f32_pf, grid, st, m->nC, sell(m), m->fg32, (const float *) g, 2.f,
                         (float *) phiBar, (float *) phiBBar, m->nC, prefetch_args(m, PF_GADJ));
        else
            CG_LAUNCH_PF(m, k_madj_f32_pf, grid, st, m->nC, sell(m), m->fg32, (const float4 *) state,
                         (const float *) gface, (float4 *) stateBar, m->nC, prefetch_args(m, PF_MADJ));
        CG_LAUNCHED();
        return CUPCFD_E_SUCCESS;
    }
    kt.set_name(f64 ? "k_adj_f64" : "k_adj_f32");
    if (f64)
        k_adj_f64<<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg64, (const double *) g, hscale, (const double *) state,
                                        (const double *) gface, (double *) phiBar, (double *) phiBBar,
                                        (double *) stateBar, m->nC);
    else
        k_adj_f32<<<grid, BLK, 0, st>>>(m->nC, sell(m), m->fg32, (const float *) g, (float) hscale,
                                        (const float4 *) state, (const float *) gface, (float *) phiBar,
                                        (float *) phiBBar, (float4 *) stateBar, m->nC);
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}
}  // namespace

// Host-buffer forward+adjoint. The host link carries about 1.1 GB in and
// 1.5 GB out per call at 256^3, against about 1 ms of kernels, so the call is
// ordered for the link rather than the kernels: each result goes back as soon
// as it exists, while the next inputs still come in (the link carries both
// directions at once).
//   mesh stream:  phi in -> gradient -> gradient adjoint -> [e0] -> state in
//                 -> mass flux -> [e1] -> gface in -> loss -> mass adjoint -> [e2]
//   copy stream:  after e0 the gradient and phiBar out (while the state comes
//                 in), after e1 the mass fluxes (while gface comes in), after
//                 e2 the state adjoint and the loss
// The kernels are the device calls' (gradient, mass flux, the two parts of
// the adjoint, and the loss from the stored gradient and mass fluxes), whose
// results equal cupcfd_gpu_dev_forward_adjoint's bit for bit.
namespace {
// The host-buffer forward+adjoint over host arrays of type H (double: the
// reference's T = double arrays; float: T = float arrays, half the bytes on
// the host link). The compute precision is `precision` either way.
template <class H>
int forward_adjoint_t(cupcfd_gpu_mesh *m, int32_t precision, const H *phi, const H *phiB, const H *den, const H *u,
                      const H *v, const H *w, const H *gface, H *grad, H *massFlux, H *phiBar, H *phiBBar, H *denBar,
                      H *uBar, H *vBar, H *wBar, double *loss) {
    constexpr size_t HS = sizeof(H);
    CG_RETURN_IF(!m || !phi || !den || !u || !v || !w || !gface || (m->nB > 0 && !phiB), CUPCFD_E_NULL_PTR,
                 "forward_adjoint: null input");
    CG_TRY(check_prec(m, precision));
    CG_TRY(make_device_current(m->device));
    cudaStream_t st = m->stream;
    int nC = m->nC, nF = m->nF, nB = m->nB;
    int64_t ldc = nC;
    unsigned gC = grid_for(nC, BLK), gF = grid_for(nF, BLK);
    bool f64 = precision == CUPCFD_PREC_F64;
    size_t es = f64 ? 8 : 4;
    CG_TRY(pipe_init(m));
    cudaStream_t so = m->outStream;
    // host -> device staging (reference numbering, host type)
    H *in;
    void *phiI, *phibI, *stI, *gI, *gradI, *mfI, *pbI, *pbbI, *sbI;
    CG_TRY(scratch(m, S_IN0, 5 * (size_t) nC + nB + nF, &in));
    H *hPhi = in, *hR = in + nC, *hU = in + 2 * (size_t) nC, *hV = in + 3 * (size_t) nC, *hW = in + 4 * (size_t) nC;
    H *hPb = in + 5 * (size_t) nC, *hG = hPb + nB;
    // internal numbering, compute precision
    CG_TRY(m->scratchBuf(S_IN1, (size_t) nC * es, &phiI));
    CG_TRY(m->scratchBuf(S_IN2, (size_t) std::max(nB, 1) * es, &phibI));
    CG_TRY(m->scratchBuf(S_IN3, 4 * (size_t) nC * es, &stI));
    CG_TRY(m->scratchBuf(S_IN4, (size_t) nF * es, &gI));
    CG_TRY(m->scratchBuf(S_OUT0, 3 * (size_t) nC * es, &gradI));
    CG_TRY(m->scratchBuf(S_OUT1, (size_t) nF * es, &mfI));
    CG_TRY(m->scratchBuf(S_OUT2, (size_t) nC * es, &pbI));
    CG_TRY(m->scratchBuf(S_OUT3, (size_t) std::max(nB, 1) * es, &pbbI));
    CG_TRY(m->scratchBuf(S_OUT4, 4 * (size_t) nC * es, &sbI));
    double *dloss, *part;
    H *out;
    CG_TRY(scratch(m, S_NORM, 1, &dloss));
    CG_TRY(scratch(m, S_LOSS, gC, &part));
    CG_TRY(scratch(m, S_IN5, 8 * (size_t) nC + nF + nB, &out));
    H *oG = out, *oMf = out + 3 * (size_t) nC, *oPb = oMf + nF, *oR = oPb + nC, *oU = oR + nC, *oV = oU + nC,
           *oW = oV + nC, *oPbb = oW + nC;

    // The inputs go in on the copy-in stream, each set's arrival an event the
    // computation waits for, so the copy engine carries the next set while the
    // GPU computes on the last (issued in this order, so that host staging of
    // pageable arrays still overlaps the computation).
    cudaStream_t si = m->inStream;
    // phi in, gradient
    CG_CHECK_CUDA(cudaMemcpyAsync(hPhi, phi, HS * (size_t) nC, cudaMemcpyHostToDevice, si));
    if (nB > 0) CG_CHECK_CUDA(cudaMemcpyAsync(hPb, phiB, HS * (size_t) nB, cudaMemcpyHostToDevice, si));
    CG_CHECK_CUDA(cudaEventRecord(m->inEv[0], si));
    CG_CHECK_CUDA(cudaStreamWaitEvent(st, m->inEv[0], 0));
    if (f64) {
        k_gather<H, double><<<gC, BLK, 0, st>>>(nC, 1, m->cellN2O, hPhi, 0, (double *) phiI, 0);
        if (nB > 0) {
            k_convert<H, double><<<grid_for(nB, BLK), BLK, 0, st>>>(nB, hPb, (double *) phibI);
            g_launches.fetch_add(1, std::memory_order_relaxed);
        }
    } else {
        k_gather<H, float><<<gC, BLK, 0, st>>>(nC, 1, m->cellN2O, hPhi, 0, (float *) phiI, 0);
        if (nB > 0) {
            k_convert<H, float><<<grid_for(nB, BLK), BLK, 0, st>>>(nB, hPb, (float *) phibI);
            g_launches.fetch_add(1, std::memory_order_relaxed);
        }
    }
    CG_LAUNCHED();
    CG_TRY(launch_grad_once(m, precision, false, false, phiI, phibI, nullptr, gradI, nullptr, st));
    CG_TRY(launch_adj_part(m, f64, gradI, 2.0, nullptr, nullptr, pbI, pbbI, nullptr, st));
    // Each result goes back to reference numbering (host type) on the mesh
    // stream right after the kernel that makes it, so the copy stream only
    // copies: its engine does not wait for a conversion between two copies.
    if (f64) {
        k_blocks_to_aos<double, H><<<gC, BLK, 0, st>>>(nC, 3, m->cellO2N, (const double *) gradI, ldc, oG);
        k_gather<double, H><<<gC, BLK, 0, st>>>(nC, 1, m->cellO2N, (const double *) pbI, 0, oPb, 0);
        if (nB > 0) {
            k_convert<double, H><<<grid_for(nB, BLK), BLK, 0, st>>>(nB, (const double *) pbbI, oPbb);
            g_launches.fetch_add(1, std::memory_order_relaxed);
        }
    } else {
        k_blocks_to_aos<float, H><<<gC, BLK, 0, st>>>(nC, 3, m->cellO2N, (const float *) gradI, ldc, oG);
        k_gather<float, H><<<gC, BLK, 0, st>>>(nC, 1, m->cellO2N, (const float *) pbI, 0, oPb, 0);
        if (nB > 0) {
            k_convert<float, H><<<grid_for(nB, BLK), BLK, 0, st>>>(nB, (const float *) pbbI, oPbb);
            g_launches.fetch_add(1, std::memory_order_relaxed);
        }
    }
    g_launches.fetch_add(1, std::memory_order_relaxed);
    CG_LAUNCHED();
    CG_CHECK_CUDA(cudaEventRecord(m->pipeEv[0], st));
    // state in, mass flux
    CG_CHECK_CUDA(cudaMemcpyAsync(hR, den, HS * (size_t) nC, cudaMemcpyHostToDevice, si));
    CG_CHECK_CUDA(cudaMemcpyAsync(hU, u, HS * (size_t) nC, cudaMemcpyHostToDevice, si));
    CG_CHECK_CUDA(cudaMemcpyAsync(hV, v, HS * (size_t) nC, cudaMemcpyHostToDevice, si));
    CG_CHECK_CUDA(cudaMemcpyAsync(hW, w, HS * (size_t) nC, cudaMemcpyHostToDevice, si));
    CG_CHECK_CUDA(cudaEventRecord(m->inEv[1], si));
    CG_CHECK_CUDA(cudaStreamWaitEvent(st, m->inEv[1], 0));
    if (f64) k_gather<H, double><<<gC, BLK, 0, st>>>(nC, 4, m->cellN2O, hR, nC, (double *) stI, ldc);
    else k_state_to_f4<H><<<gC, BLK, 0, st>>>(nC, m->cellN2O, hR, hU, hV, hW, (float4 *) stI);
    CG_LAUNCHED();
    CG_TRY(cupcfd_gpu_dev_mass_plain(m, precision, stI, mfI, st));
    if (f64) k_faces_to_ref<double, H><<<gF, BLK, 0, st>>>(nF, m->faceO2N, m->faceCells, (const double *) mfI, oMf, 1);
    else k_faces_to_ref<float, H><<<gF, BLK, 0, st>>>(nF, m->faceO2N, m->faceCells, (const float *) mfI, oMf, 1);
    CG_LAUNCHED();
    CG_CHECK_CUDA(cudaEventRecord(m->pipeEv[1], st));
    // gface in, loss and adjoint
    CG_CHECK_CUDA(cudaMemcpyAsync(hG, gface, HS * (size_t) nF, cudaMemcpyHostToDevice, si));
    CG_CHECK_CUDA(cudaEventRecord(m->inEv[2], si));
    CG_CHECK_CUDA(cudaStreamWaitEvent(st, m->inEv[2], 0));
    if (f64) k_gather<H, double><<<gF, BLK, 0, st>>>(nF, 1, m->faceN2O, hG, 0, (double *) gI, 0);
    else k_gather<H, float><<<gF, BLK, 0, st>>>(nF, 1, m->faceN2O, hG, 0, (float *) gI, 0);
    CG_LAUNCHED();
    // the mass part of the adjoint first: its results are the last large set
    // to go out; the loss (8 bytes) follows it
    CG_TRY(launch_adj_part(m, f64, nullptr, 0.0, stI, gI, nullptr, nullptr, sbI, st));
    if (f64) k_gather<double, H><<<gC, BLK, 0, st>>>(nC, 4, m->cellO2N, (const double *) sbI, ldc, oR, nC);
    else k_f4_to_ref<H><<<gC, BLK, 0, st>>>(nC, m->cellO2N, (const float4 *) sbI, oR, oU, oV, oW);
    CG_LAUNCHED();
    CG_CHECK_CUDA(cudaEventRecord(m->pipeEv[2], st));
    if (f64)
        k_loss<double><<<gC, 256, 0, st>>>(nC, sell(m), (const double *) gI, (const double *) mfI,
                                           (const double *) gradI, m->vol, part, ldc);
    else
        k_loss<float><<<gC, 256, 0, st>>>(nC, sell(m), (const float *) gI, (const float *) mfI,
                                          (const float *) gradI, m->vol, part, ldc);
    CG_LAUNCHED();
    k_reduce_partials<<<1, 1024, 0, st>>>((int) gC, part, dloss);
    CG_LAUNCHED();

    // to the host, on the copy stream, each set once it exists
    CG_CHECK_CUDA(cudaStreamWaitEvent(so, m->pipeEv[0], 0));
    if (grad) CG_CHECK_CUDA(cudaMemcpyAsync(grad, oG, 3 * HS * (size_t) nC, cudaMemcpyDeviceToHost, so));
    if (phiBar) CG_CHECK_CUDA(cudaMemcpyAsync(phiBar, oPb, HS * (size_t) nC, cudaMemcpyDeviceToHost, so));
    if (phiBBar && nB > 0) CG_CHECK_CUDA(cudaMemcpyAsync(phiBBar, oPbb, HS * (size_t) nB, cudaMemcpyDeviceToHost, so));
    CG_CHECK_CUDA(cudaStreamWaitEvent(so, m->pipeEv[1], 0));
    if (massFlux) CG_CHECK_CUDA(cudaMemcpyAsync(massFlux, oMf, HS * (size_t) nF, cudaMemcpyDeviceToHost, so));
    CG_CHECK_CUDA(cudaStreamWaitEvent(so, m->pipeEv[2], 0));
    if (denBar) CG_CHECK_CUDA(cudaMemcpyAsync(denBar, oR, HS * (size_t) nC, cudaMemcpyDeviceToHost, so));
    if (uBar) CG_CHECK_CUDA(cudaMemcpyAsync(uBar, oU, HS * (size_t) nC, cudaMemcpyDeviceToHost, so));
    if (vBar) CG_CHECK_CUDA(cudaMemcpyAsync(vBar, oV, HS * (size_t) nC, cudaMemcpyDeviceToHost, so));
    if (wBar) CG_CHECK_CUDA(cudaMemcpyAsync(wBar, oW, HS * (size_t) nC, cudaMemcpyDeviceToHost, so));
    if (loss) CG_CHECK_CUDA(cudaMemcpyAsync(loss, dloss, 8, cudaMemcpyDeviceToHost, st));
    CG_CHECK_CUDA(cudaStreamSynchronize(so));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    return CUPCFD_E_SUCCESS;
}

}  // namespace

extern "C" int cupcfd_gpu_forward_adjoint(cupcfd_gpu_mesh *m, int32_t precision, const double *phi, const double *phiB,
                                          const double *den, const double *u, const double *v, const double *w,
                                          const double *gface, double *grad, double *massFlux, double *phiBar,
                                          double *phiBBar, double *denBar, double *uBar, double *vBar, double *wBar,
                                          double *loss) {
    clear_error();
    return forward_adjoint_t<double>(m, precision, phi, phiB, den, u, v, w, gface, grad, massFlux, phiBar, phiBBar,
                                     denBar, uBar, vBar, wBar, loss);
}

extern "C" int cupcfd_gpu_forward_adjoint_f32(cupcfd_gpu_mesh *m, int32_t precision, const float *phi, const float *phiB,
                                              const float *den, const float *u, const float *v, const float *w,
                                              const float *gface, float *grad, float *massFlux, float *phiBar,
                                              float *phiBBar, float *denBar, float *uBar, float *vBar, float *wBar,
                                              double *loss) {
    clear_error();
    return forward_adjoint_t<float>(m, precision, phi, phiB, den, u, v, w, gface, grad, massFlux, phiBar, phiBBar,
                                    denBar, uBar, vBar, wBar, loss);
}

// ===========================================================================
// Forward without any allocation (no counterpart in the reference)
// ===========================================================================
// cupcfd_gpu_dev_forward takes the per-block loss partials from the mesh's
// scratch pool, which grows with cudaMalloc on first use. Some callers
// cannot allocate at the point where they run the forward: a solver that
// reserves its whole device-memory budget at start-up and treats any later
// allocation as a failure, or a caller running inside another runtime that
// owns the device's allocator and must not see a foreign cudaMalloc/cudaFree
// (which also synchronises the device). This variant runs the same kernels
// with the partials in a fixed array compiled into the library instead.
//
// Limits: the array holds NOALLOC_MAX_PARTIALS doubles (4 MiB: one per warp,
// eight per 256-cell tile, for NOALLOC_MAX_TILES tiles), so a loss can be
// reduced for meshes of up to 16,777,216 cells; larger meshes are rejected
// with CUPCFD_E_ARRAY_SIZE_MISMATCH before anything runs. Every GPU that loads the library holds the array until the
// process exits. All calls share it: each call writes every slot it reads
// before reading it (nothing needs clearing), but calls whose kernels
// overlap on the GPU (different streams, no ordering between them) race on
// it. The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current; make that first call
// before any stream capture. No error message is recorded (recording one
// allocates host memory); the status code says what failed.
namespace {
constexpr int NOALLOC_MAX_TILES = 65536;
constexpr int NOALLOC_MAX_PARTIALS = NOALLOC_MAX_TILES * (TILE_CELLS / 32);
constexpr int NOALLOC_MAX_DEVICES = 64;
static __device__ __align__(256) double g_noalloc_partials[NOALLOC_MAX_PARTIALS];
// Per device, the array's device address once looked up (null until then).
// The pointer is its own ready flag: threads that race on a device's first
// call may each look the address up, and they store the same value.
static std::atomic<double *> g_noalloc_ptr[NOALLOC_MAX_DEVICES];

// Makes `dev` current for the lifetime of the guard and gives the caller's
// device back afterwards (cudaGetDevice / cudaSetDevice allocate nothing).
struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) return;
        ok = prev == dev || cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard() {
        if (ok && prev >= 0) cudaSetDevice(prev);
    }
};
}  // namespace

extern "C" int cupcfd_gpu_dev_forward_noalloc(cupcfd_gpu_mesh *m, int32_t precision, const void *phi,
                                              const void *phiB, const void *state, const void *gface, void *grad,
                                              void *massFlux, double *loss, void *stream) {
    if (!m || !phi || !state || !grad || !massFlux || (m->nB > 0 && !phiB)) return CUPCFD_E_NULL_PTR;
    if ((gface == nullptr) != (loss == nullptr)) return CUPCFD_E_NULL_PTR;
    if ((precision != CUPCFD_PREC_F64 && precision != CUPCFD_PREC_F32C) || !(m->precisions & (1 << precision)))
        return CUPCFD_E_CONFIG_INVALID_VALUE;
    {
        uintptr_t a = precision == CUPCFD_PREC_F64 ? 8 : 4, sa = precision == CUPCFD_PREC_F64 ? 8 : 16;
        for (const void *p : {phi, phiB, gface, (const void *) grad, (const void *) massFlux})
            if (((uintptr_t) p) % a != 0) return CUPCFD_E_CONFIG_INVALID_VALUE;
        if (((uintptr_t) state) % sa != 0 || ((uintptr_t) loss) % 8 != 0) return CUPCFD_E_CONFIG_INVALID_VALUE;
    }
    unsigned grid = grid_for(m->nC, BLK);
    if (loss && grid > (unsigned) NOALLOC_MAX_TILES) return CUPCFD_E_ARRAY_SIZE_MISMATCH;
    int dev = m->device;
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return CUPCFD_E_NOT_IMPLEMENTED;
    DeviceGuard guard(dev);
    if (!guard.ok) return CUPCFD_E_ERROR;
    double *part = nullptr;
    if (loss) {
        // one-time set-up per device, with that device current
        part = g_noalloc_ptr[dev].load(std::memory_order_acquire);
        if (!part) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess) return CUPCFD_E_ERROR;
            part = (double *) p;
            g_noalloc_ptr[dev].store(part, std::memory_order_release);
        }
    }
    cudaStream_t st = as_stream(stream);
    int group = 1;
    if (precision == CUPCFD_PREC_F64)
        launch_fwd_f64(m, phi, phiB, state, gface, grad, massFlux, part, st, &group);
    else
        launch_fwd_f32(m, phi, phiB, state, gface, grad, massFlux, part, st, &group);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (cudaGetLastError() != cudaSuccess) return CUPCFD_E_ERROR;
    if (loss) {
        if (group > 1) {
            k_group_partials<TILE_CELLS / 32><<<grid_for(grid, BLK), BLK, 0, st>>>((int) grid, part);
            g_launches.fetch_add(1, std::memory_order_relaxed);
            if (cudaGetLastError() != cudaSuccess) return CUPCFD_E_ERROR;
        }
        k_reduce_partials<<<1, 1024, 0, st>>>((int) grid, part, loss);
        g_launches.fetch_add(1, std::memory_order_relaxed);
        if (cudaGetLastError() != cudaSuccess) return CUPCFD_E_ERROR;
    }
    return CUPCFD_E_SUCCESS;
}

// ---------------------------------------------------------------------------
// device timers
// ---------------------------------------------------------------------------
extern "C" int cupcfd_gpu_timing_enable(int32_t on) {
    clear_error();
    g_timer_on.store(on != 0);
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_timing_read(int32_t capacity, char *names, int64_t *launches, double *ms, int32_t *count) {
    clear_error();
    CG_RETURN_IF(!count || (capacity > 0 && (!names || !launches || !ms)), CUPCFD_E_NULL_PTR, "timing_read: null argument");
    std::vector<TimerRec> recs;
    {
        std::lock_guard<std::mutex> lk(g_timer_mu);
        recs.swap(g_timer_recs);
    }
    std::map<std::string, std::pair<int64_t, double>> acc;
    std::vector<std::string> order;
    int dev0 = 0;
    cudaGetDevice(&dev0);
    int failed = 0;
    for (const TimerRec &r : recs) {
        float t = 0.f;
        cudaSetDevice(r.device);
        if (cudaEventSynchronize(r.b) != cudaSuccess || cudaEventElapsedTime(&t, r.a, r.b) != cudaSuccess) failed++;
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
        std::string nm = r.name ? r.name : "?";
        if (!acc.count(nm)) order.push_back(nm);
        acc[nm].first += 1;
        acc[nm].second += t;
    }
    cudaSetDevice(dev0);
    CG_RETURN_IF(failed, CUPCFD_E_ERROR, "timing_read: a recorded event could not be timed");
    int n = 0;
    for (const std::string &nm : order) {
        if (n < capacity) {
            std::snprintf(names + 64 * (size_t) n, 64, "%s", nm.c_str());
            launches[n] = acc[nm].first;
            ms[n] = acc[nm].second;
        }
        n++;
    }
    *count = n;
    return CUPCFD_E_SUCCESS;
}
