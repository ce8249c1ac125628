// Device mesh construction: validation, the reference cell->face CSR,
// renumbering and the device layout the face-loop kernels read.
//
// One-time integer work. Sorting and prefix sums use CUB (part of the CUDA
// toolkit); everything else is hand-written here.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "strided.cuh"
#include "internal.cuh"

namespace cupcfd_gpu {

static thread_local std::string t_last_error;
std::atomic<int64_t> g_launches{0};

void set_error(const std::string &msg) { t_last_error = msg; }
void clear_error() { t_last_error.clear(); }

int make_device_current(int device) {
    if (device >= 0) CG_CHECK_CUDA(cudaSetDevice(device));
    return CUPCFD_E_SUCCESS;
}

// ---------------------------------------------------------------------------
// validation
// ---------------------------------------------------------------------------
// err bits: 1 cell1 out of range, 2 cell2 out of range / equals cell1,
// 4 boundary id out of range or inconsistent with cell2, 8 boundary id used twice
__global__ void k_validate(int nF, int nC, int nB, const int *__restrict__ c1, const int *__restrict__ c2,
                           const int *__restrict__ bnd, int *__restrict__ bcount, int *__restrict__ err) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    int a = c1[f], b = c2[f], r = bnd[f];
    int e = 0;
    if (a < 0 || a >= nC) e |= 1;
    if (r > -1) {
        if (b != -1 || r >= nB) e |= 4;
        else if (atomicAdd(&bcount[r], 1) != 0) e |= 8;
    } else {
        if (b < 0 || b >= nC || b == a) e |= 2;
    }
    if (e) atomicOr(err, e);
}

__global__ void k_degree(int nF, const int *__restrict__ c1, const int *__restrict__ c2, int *__restrict__ deg) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    atomicAdd(&deg[c1[f]], 1);
    int b = c2[f];
    if (b > -1) atomicAdd(&deg[b], 1);
}

// Slot order is arbitrary here; k_sort_lists makes each cell's list ascending,
// which is the order CupCfdSoAMesh::updateCellFaceMap produces
// (ascending-face fill plus per-cell merge_sort, CupCfdSoAMesh.cpp:576-621).
__global__ void k_fill_csr(int nF, const int *__restrict__ c1, const int *__restrict__ c2, int *__restrict__ cursor,
                           int *__restrict__ adj) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    adj[atomicAdd(&cursor[c1[f]], 1)] = f;
    int b = c2[f];
    if (b > -1) adj[atomicAdd(&cursor[b], 1)] = f;
}

__global__ void k_sort_lists(int nC, const int *__restrict__ xadj, int *__restrict__ adj) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    int b = xadj[c], e = xadj[c + 1];
    for (int i = b + 1; i < e; i++) {
        int v = adj[i], j = i - 1;
        while (j >= b && adj[j] > v) { adj[j + 1] = adj[j]; j--; }
        adj[j + 1] = v;
    }
}

// ---------------------------------------------------------------------------
// renumbering
// ---------------------------------------------------------------------------
__global__ void k_iota(int n, int *__restrict__ a) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

__global__ void k_invert(int n, const int *__restrict__ n2o, int *__restrict__ o2n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) o2n[n2o[i]] = i;
}

__device__ __forceinline__ uint64_t spread3(uint64_t x) {
    x &= 0x1fffff;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}

// bbox[0..2] = min, bbox[3..5] = max of the cell centres
__global__ void k_morton_keys(int nC, const double *__restrict__ cc, const double *__restrict__ bbox,
                              uint64_t *__restrict__ key) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    uint64_t q[3];
    for (int d = 0; d < 3; d++) {
        double lo = bbox[d], hi = bbox[3 + d];
        double t = hi > lo ? (cc[3 * c + d] - lo) / (hi - lo) : 0.0;
        t = fmin(fmax(t, 0.0), 1.0);
        q[d] = (uint64_t) (t * 2097151.0);
    }
    key[c] = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
}

__global__ void k_bbox(int nC, const double *__restrict__ cc, unsigned long long *__restrict__ bb) {
    // order-preserving integer encoding of doubles so atomicMin/Max work
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    for (int d = 0; d < 3; d++) {
        long long v = __double_as_longlong(cc[3 * c + d]);
        unsigned long long u = v < 0 ? ~(unsigned long long) v : ((unsigned long long) v | 0x8000000000000000ULL);
        atomicMin(&bb[d], u);
        atomicMax(&bb[3 + d], u);
    }
}

__global__ void k_bbox_decode(const unsigned long long *__restrict__ bb, double *__restrict__ out) {
    int d = threadIdx.x;
    if (d >= 6) return;
    unsigned long long u = bb[d];
    long long v = (u & 0x8000000000000000ULL) ? (long long) (u & 0x7fffffffffffffffULL) : (long long) ~u;
    out[d] = __longlong_as_double(v);
}

__global__ void k_face_owner_keys(int nF, const int *__restrict__ c1, const int *__restrict__ cellO2N,
                                  uint64_t *__restrict__ key) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    key[f] = ((uint64_t) (uint32_t) cellO2N[c1[f]] << 32) | (uint32_t) f;
}

// j = rank of face f among its owner's faces (ascending reference face id),
// for every face (one thread per reference cell). err bit set if j >= 32.
__global__ void k_owned_rank(int nC, const int *__restrict__ xadj, const int *__restrict__ adj,
                             const int *__restrict__ c1, int *__restrict__ rank, int *__restrict__ err) {
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nC) return;
    int j = 0;
    for (int k = xadj[o]; k < xadj[o + 1]; k++) {
        int f = adj[k];
        if (c1[f] == o) rank[f] = j++;
    }
    if (j > 32) atomicOr(err, 1);
}

// Face key (owner slice, owned-face rank, owner lane): entry k of a warp's 32
// cells then reads consecutive face records (a SELL layout for faces).
__global__ void k_face_slice_keys(int nF, const int *__restrict__ c1, const int *__restrict__ cellO2N,
                                  const int *__restrict__ rank, uint64_t *__restrict__ key) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    uint64_t P = (uint64_t) (uint32_t) cellO2N[c1[f]];
    key[f] = ((P >> 5) << 10) | ((uint64_t) rank[f] << 5) | (P & 31);
}

__global__ void k_low32(int n, const uint64_t *__restrict__ key, int *__restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (int) (uint32_t) key[i];
}

// ---------------------------------------------------------------------------
// internal layout
// ---------------------------------------------------------------------------
__global__ void k_layout_faces(int nF, const int *__restrict__ faceN2O, const int *__restrict__ cellO2N,
                               const int *__restrict__ c1, const int *__restrict__ c2, const int *__restrict__ bnd,
                               const double *__restrict__ lam, const double *__restrict__ area,
                               const double *__restrict__ S, const double *__restrict__ xf,
                               const double *__restrict__ xpac, const double *__restrict__ xnac,
                               int2 *__restrict__ fcells, double4 *__restrict__ fg64, double4 *__restrict__ fc64,
                               double4 *__restrict__ fxp64, double4 *__restrict__ fxn64, float4 *__restrict__ fg32,
                               float4 *__restrict__ fc32) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    int o = faceN2O[f];
    int b = bnd[o];
    fcells[f] = make_int2(cellO2N[c1[o]], b > -1 ? -1 - b : cellO2N[c2[o]]);
    double4 g = make_double4(S[3 * o], S[3 * o + 1], S[3 * o + 2], lam[o]);
    double4 c = make_double4(xf[3 * o], xf[3 * o + 1], xf[3 * o + 2], area[o]);
    if (fg64) { fg64[f] = g; fc64[f] = c; }
    if (fxp64) {
        fxp64[f] = make_double4(xpac[3 * o], xpac[3 * o + 1], xpac[3 * o + 2], 0.0);
        fxn64[f] = make_double4(xnac[3 * o], xnac[3 * o + 1], xnac[3 * o + 2], 0.0);
    }
    if (fg32) {
        fg32[f] = make_float4((float) g.x, (float) g.y, (float) g.z, (float) g.w);
        fc32[f] = make_float4((float) c.x, (float) c.y, (float) c.z, (float) c.w);
    }
}

__global__ void k_layout_cells(int nC, const int *__restrict__ cellN2O, const double *__restrict__ cc,
                               const double *__restrict__ vol, double4 *__restrict__ cc64, float4 *__restrict__ cc32,
                               double *__restrict__ vout) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    int o = cellN2O[c];
    double4 p = make_double4(cc[3 * o], cc[3 * o + 1], cc[3 * o + 2], 0.0);
    if (cc64) cc64[c] = p;
    if (cc32) cc32[c] = make_float4((float) p.x, (float) p.y, (float) p.z, 0.f);
    vout[c] = vol[o];
}

// one warp per slice: width = max degree over the slice's cells
__global__ void k_slice_width(int nC, int nSlices, const int *__restrict__ cellN2O, const int *__restrict__ xadj,
                              int *__restrict__ words) {
    int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (s >= nSlices) return;
    int c = s * 32 + lane;
    int d = 0;
    if (c < nC) {
        int o = cellN2O[c];
        d = xadj[o + 1] - xadj[o];
    }
    for (int k = 16; k > 0; k >>= 1) d = max(d, __shfl_xor_sync(0xffffffffu, d, k));
    if (lane == 0) words[s] = d > INT_MAX / 32 ? INT_MAX : 32 * d;  // an overfull slice is refused by the host
}

__global__ void k_fill_sell(int nC, const int *__restrict__ cellN2O, const int *__restrict__ cellO2N,
                            const int *__restrict__ xadj, const int *__restrict__ adj, const int *__restrict__ c1,
                            const int *__restrict__ c2, const int *__restrict__ bnd, const int *__restrict__ faceO2N,
                            const int *__restrict__ slicePtr, int2 *__restrict__ inc) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    int s = c >> 5, lane = c & 31;
    if (s * 32 >= nC) return;
    int width = (slicePtr[s + 1] - slicePtr[s]) >> 5;
    int base = slicePtr[s] + lane;
    int k = 0;
    if (c < nC) {
        int o = cellN2O[c];
        for (int j = xadj[o]; j < xadj[o + 1]; j++, k++) {
            int fo = adj[j];
            int role = (c1[fo] == o) ? 0 : 1;
            int other = role ? cellO2N[c1[fo]] : (bnd[fo] > -1 ? -1 - bnd[fo] : cellO2N[c2[fo]]);
            inc[base + 32 * k] = make_int2((faceO2N[fo] << 1) | role, other);
        }
    }
    for (; k < width; k++) inc[base + 32 * k] = make_int2(-1, -1);
}

// Boundary -> face maps and the (owner cell, boundary id) sort keys; a
// boundary id out of range or met twice sets err.
__global__ void k_bnd_maps(int nF, int nB, const int *__restrict__ faceN2O, const int *__restrict__ bndRef,
                           const int2 *__restrict__ fcells, int *__restrict__ bndFaceRef, int *__restrict__ bndFaceInt,
                           unsigned long long *__restrict__ keys, int *__restrict__ err) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    int fo = faceN2O[f], b = bndRef[fo];
    if (b < 0) return;
    if (b >= nB || atomicCAS(bndFaceRef + b, -1, fo) != -1) {
        atomicOr(err, 1);
        return;
    }
    bndFaceInt[b] = f;
    keys[b] = ((unsigned long long) (unsigned) fcells[f].x << 32) | (unsigned) b;
}

__global__ void k_bnd_unkey(int nB, const unsigned long long *__restrict__ keys, const int *__restrict__ cellN2O,
                            const int *__restrict__ bndFaceRef, int *__restrict__ sorted, int *__restrict__ cellInt,
                            int *__restrict__ cellRef, int *__restrict__ err) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nB) return;
    if (bndFaceRef[k] < 0) atomicOr(err, 1);  // a boundary id no face carries
    int c = (int) (keys[k] >> 32);
    sorted[k] = (int) (unsigned) keys[k];
    cellInt[k] = c;
    cellRef[k] = cellN2O[c];
}

__global__ void k_any_nonzero(int64_t n, const double *__restrict__ a, int *__restrict__ flag) {
    int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && a[i] != 0.0) *flag = 1;
}

}  // namespace cupcfd_gpu

using namespace cupcfd_gpu;

int cupcfd_gpu_mesh::scratchBuf(int slot, size_t nbytes, void **out) {
    if ((int) scratch.size() <= slot) scratch.resize(slot + 1);
    DevBuf &b = scratch[slot];
    if (b.bytes < nbytes) {
        if (b.p) cudaFree(b.p);
        b.p = nullptr;
        b.bytes = 0;
        cudaError_t e = cudaMalloc(&b.p, nbytes);
        if (e != cudaSuccess) {
            set_error(std::string("cudaMalloc (scratch): ") + cudaGetErrorString(e));
            return CUPCFD_E_ERROR;
        }
        b.bytes = nbytes;
    }
    *out = b.p;
    return CUPCFD_E_SUCCESS;
}

namespace {

// RAII temporary device buffer for the build
struct Tmp {
    void *p = nullptr;
    ~Tmp() { if (p) cudaFree(p); }
    template <class T>
    int get(T **out, size_t n) {
        if (n == 0) n = 1;
        cudaError_t e = cudaMalloc(&p, n * sizeof(T));
        if (e != cudaSuccess) {
            set_error(std::string("cudaMalloc (build): ") + cudaGetErrorString(e));
            return CUPCFD_E_ERROR;
        }
        *out = (T *) p;
        return CUPCFD_E_SUCCESS;
    }
};

int exclusive_scan(const int *in, int *out, int n, cudaStream_t st) {
    size_t tb = 0;
    CG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, n, st));
    Tmp t;
    void *tp;
    CG_TRY(t.get((char **) &tp, tb));
    CG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(tp, tb, in, out, n, st));
    g_launches.fetch_add(1);
    return CUPCFD_E_SUCCESS;
}

int sort_keys(uint64_t *keys, uint64_t *keysOut, int n, int endBit, cudaStream_t st) {
    size_t tb = 0;
    CG_CHECK_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys, keysOut, n, 0, endBit, st));
    Tmp t;
    void *tp;
    CG_TRY(t.get((char **) &tp, tb));
    CG_CHECK_CUDA(cub::DeviceRadixSort::SortKeys(tp, tb, keys, keysOut, n, 0, endBit, st));
    g_launches.fetch_add(1);
    return CUPCFD_E_SUCCESS;
}

int sort_pairs(uint64_t *keys, uint64_t *keysOut, int *vals, int *valsOut, int n, int endBit, cudaStream_t st) {
    size_t tb = 0;
    CG_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keysOut, vals, valsOut, n, 0, endBit, st));
    Tmp t;
    void *tp;
    CG_TRY(t.get((char **) &tp, tb));
    CG_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(tp, tb, keys, keysOut, vals, valsOut, n, 0, endBit, st));
    g_launches.fetch_add(1);
    return CUPCFD_E_SUCCESS;
}

int bits_for(uint64_t v) {
    int b = 0;
    while (b < 64 && (v >> b) != 0) b++;
    return b;
}

}  // namespace

namespace cupcfd_gpu {

// Reverse Cuthill-McKee numbering of the cell graph (host). Each connected
// component starts from a pseudo-peripheral cell (repeated breadth-first
// search from a minimum-degree cell until the eccentricity stops growing);
// neighbours are visited in ascending degree, ties by reference id; the
// final order is reversed. cellN2O[new] = reference id.
static int rcm_numbering(cupcfd_gpu_mesh *m, const Source &s, cudaStream_t st) {
    int nC = s.nC, nF = s.nF;
    std::vector<int> xadj(nC + 1), adj(m->nInc), c1(nF), c2(nF);
    CG_CHECK_CUDA(cudaMemcpyAsync(xadj.data(), m->refXadj, sizeof(int) * (nC + 1), cudaMemcpyDeviceToHost, st));
    CG_CHECK_CUDA(cudaMemcpyAsync(adj.data(), m->refAdj, sizeof(int) * (size_t) m->nInc, cudaMemcpyDeviceToHost, st));
    CG_CHECK_CUDA(cudaMemcpyAsync(c1.data(), s.c1, sizeof(int) * nF, cudaMemcpyDeviceToHost, st));
    CG_CHECK_CUDA(cudaMemcpyAsync(c2.data(), s.c2, sizeof(int) * nF, cudaMemcpyDeviceToHost, st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    // cell adjacency (interior faces only)
    std::vector<int> nx(nC + 1, 0);
    for (int c = 0; c < nC; c++) {
        int d = 0;
        for (int k = xadj[c]; k < xadj[c + 1]; k++) d += (c2[adj[k]] >= 0);
        nx[c + 1] = nx[c] + d;
    }
    std::vector<int> nb(nx[nC]);
    for (int c = 0; c < nC; c++) {
        int p = nx[c];
        for (int k = xadj[c]; k < xadj[c + 1]; k++) {
            int f = adj[k];
            if (c2[f] < 0) continue;
            nb[p++] = c1[f] == c ? c2[f] : c1[f];
        }
    }
    auto deg = [&](int c) { return nx[c + 1] - nx[c]; };
    std::vector<int> level(nC, -1), order;
    order.reserve(nC);
    std::vector<char> done(nC, 0);
    std::vector<int> q;
    q.reserve(nC);
    auto bfs_last = [&](int start, int &ecc) {
        // returns a minimum-degree cell of the last level
        q.clear();
        q.push_back(start);
        level[start] = 0;
        size_t h = 0;
        int last = start;
        while (h < q.size()) {
            int c = q[h++];
            for (int k = nx[c]; k < nx[c + 1]; k++) {
                int o = nb[k];
                if (level[o] < 0) { level[o] = level[c] + 1; q.push_back(o); }
            }
        }
        ecc = level[q.back()];
        for (int c : q)
            if (level[c] == ecc && (deg(c) < deg(last) || level[last] != ecc)) last = c;
        for (int c : q) level[c] = -1;
        return last;
    };
    std::vector<int> byDeg(nC);
    for (int i = 0; i < nC; i++) byDeg[i] = i;
    std::stable_sort(byDeg.begin(), byDeg.end(), [&](int a, int b) { return deg(a) < deg(b); });
    for (int seed : byDeg) {
        if (done[seed]) continue;
        int ecc = 0, e2 = 0;
        int start = bfs_last(seed, ecc);
        for (int it = 0; it < 4; it++) {
            int cand = bfs_last(start, e2);
            if (e2 <= ecc) break;
            ecc = e2;
            start = cand;
        }
        size_t h = order.size();
        order.push_back(start);
        done[start] = 1;
        std::vector<int> tmp;
        while (h < order.size()) {
            int c = order[h++];
            tmp.clear();
            for (int k = nx[c]; k < nx[c + 1]; k++)
                if (!done[nb[k]]) { done[nb[k]] = 1; tmp.push_back(nb[k]); }
            std::sort(tmp.begin(), tmp.end(), [&](int a, int b) { return deg(a) != deg(b) ? deg(a) < deg(b) : a < b; });
            order.insert(order.end(), tmp.begin(), tmp.end());
        }
    }
    std::reverse(order.begin(), order.end());
    CG_CHECK_CUDA(cudaMemcpyAsync(m->cellN2O, order.data(), sizeof(int) * nC, cudaMemcpyHostToDevice, st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    return CUPCFD_E_SUCCESS;
}

int build_mesh_from_source(cupcfd_gpu_mesh *m, const Source &s, const cupcfd_mesh_options *opt) {
    cudaStream_t st = m->stream;
    const int B = 256;
    int nC = s.nC, nF = s.nF, nB = s.nB;
    CG_RETURN_IF(nC <= 0 || nF <= 0 || nB < 0, CUPCFD_E_ARRAY_SIZE_MISMATCH, "mesh: empty or negative sizes");
    CG_RETURN_IF(nF >= (1 << 30), CUPCFD_E_NOT_IMPLEMENTED, "mesh: more than 2^30 faces");
    m->nC = nC; m->nF = nF; m->nB = nB;
    m->order = opt ? opt->order : CUPCFD_ORDER_MORTON;
    m->precisions = opt ? opt->precisions : ((1 << CUPCFD_PREC_F64) | (1 << CUPCFD_PREC_F32C));
    CG_RETURN_IF(m->order < 0 || m->order > 3, CUPCFD_E_CONFIG_INVALID_VALUE, "mesh: unknown order");
    CG_RETURN_IF((m->precisions & 3) == 0, CUPCFD_E_CONFIG_INVALID_VALUE, "mesh: no precision selected");

    // --- validation
    int *err, *bcount;
    Tmp tErr, tBc;
    CG_TRY(tErr.get(&err, 1));
    CG_TRY(tBc.get(&bcount, (size_t) nB));
    CG_CHECK_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    CG_CHECK_CUDA(cudaMemsetAsync(bcount, 0, sizeof(int) * (size_t) std::max(nB, 1), st));
    k_validate<<<grid_for(nF, B), B, 0, st>>>(nF, nC, nB, s.c1, s.c2, s.bnd, bcount, err);
    CG_LAUNCHED();
    int herr = 0;
    CG_CHECK_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    if (herr) {
        set_error("mesh: invalid connectivity (flags " + std::to_string(herr) +
                  ": 1 cell1 out of range, 2 cell2 out of range or equal to cell1, 4 boundary id out of range or "
                  "on an interior face, 8 boundary id on two faces)");
        return CUPCFD_E_INVALID_INDEX;
    }

    // --- reference CSR (updateCellFaceMap)
    int *deg;
    Tmp tDeg;
    CG_TRY(tDeg.get(&deg, (size_t) nC + 1));
    CG_CHECK_CUDA(cudaMemsetAsync(deg, 0, sizeof(int) * ((size_t) nC + 1), st));
    k_degree<<<grid_for(nF, B), B, 0, st>>>(nF, s.c1, s.c2, deg);
    CG_LAUNCHED();
    CG_TRY(m->alloc(&m->refXadj, (size_t) nC + 1));
    CG_TRY(exclusive_scan(deg, m->refXadj, nC + 1, st));
    int nInc = 0;
    CG_CHECK_CUDA(cudaMemcpyAsync(&nInc, m->refXadj + nC, sizeof(int), cudaMemcpyDeviceToHost, st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    m->nInc = nInc;
    m->nFi = nInc - nF;  // each interior face appears twice, each boundary face once
    CG_TRY(m->alloc(&m->refAdj, (size_t) nInc));
    {
        int *cursor;
        Tmp tc;
        CG_TRY(tc.get(&cursor, (size_t) nC + 1));
        CG_CHECK_CUDA(cudaMemcpyAsync(cursor, m->refXadj, sizeof(int) * ((size_t) nC + 1), cudaMemcpyDeviceToDevice, st));
        k_fill_csr<<<grid_for(nF, B), B, 0, st>>>(nF, s.c1, s.c2, cursor, m->refAdj);
        CG_LAUNCHED();
        k_sort_lists<<<grid_for(nC, B), B, 0, st>>>(nC, m->refXadj, m->refAdj);
        CG_LAUNCHED();
    }

    // --- cell numbering
    CG_TRY(m->alloc(&m->cellN2O, (size_t) nC));
    CG_TRY(m->alloc(&m->cellO2N, (size_t) nC));
    if (m->order == CUPCFD_ORDER_MORTON) {
        unsigned long long *bb;
        double *bbox;
        uint64_t *keys, *keysOut;
        int *vals;
        Tmp t1, t2, t3, t4, t5;
        CG_TRY(t1.get(&bb, 6));
        CG_TRY(t2.get(&bbox, 6));
        CG_TRY(t3.get(&keys, (size_t) nC));
        CG_TRY(t4.get(&keysOut, (size_t) nC));
        CG_TRY(t5.get(&vals, (size_t) nC));
        unsigned long long init[6] = {~0ULL, ~0ULL, ~0ULL, 0ULL, 0ULL, 0ULL};
        CG_CHECK_CUDA(cudaMemcpyAsync(bb, init, sizeof(init), cudaMemcpyHostToDevice, st));
        k_bbox<<<grid_for(nC, B), B, 0, st>>>(nC, s.cc, bb);
        CG_LAUNCHED();
        k_bbox_decode<<<1, 32, 0, st>>>(bb, bbox);
        CG_LAUNCHED();
        k_morton_keys<<<grid_for(nC, B), B, 0, st>>>(nC, s.cc, bbox, keys);
        CG_LAUNCHED();
        k_iota<<<grid_for(nC, B), B, 0, st>>>(nC, vals);
        CG_LAUNCHED();
        // stable LSD radix sort: equal keys keep ascending reference id
        CG_TRY(sort_pairs(keys, keysOut, vals, m->cellN2O, nC, 63, st));
        CG_CHECK_CUDA(cudaStreamSynchronize(st));
    } else if (m->order == CUPCFD_ORDER_RCM) {
        CG_TRY(rcm_numbering(m, s, st));
    } else {
        k_iota<<<grid_for(nC, B), B, 0, st>>>(nC, m->cellN2O);
        CG_LAUNCHED();
    }
    k_invert<<<grid_for(nC, B), B, 0, st>>>(nC, m->cellN2O, m->cellO2N);
    CG_LAUNCHED();

    // --- face numbering
    CG_TRY(m->alloc(&m->faceN2O, (size_t) nF));
    CG_TRY(m->alloc(&m->faceO2N, (size_t) nF));
    if (m->order == CUPCFD_ORDER_NATIVE) {
        k_iota<<<grid_for(nF, B), B, 0, st>>>(nF, m->faceN2O);
        CG_LAUNCHED();
    } else {
        // faces by (owner slice, owned-face rank, owner lane); falls back to
        // (owner, reference id) if some cell owns more than 32 faces
        uint64_t *keys, *keysOut;
        int *rank, *err2, *vals;
        Tmp t1, t2, t3, t4, t5;
        CG_TRY(t1.get(&keys, (size_t) nF));
        CG_TRY(t2.get(&keysOut, (size_t) nF));
        CG_TRY(t3.get(&rank, (size_t) nF));
        CG_TRY(t4.get(&err2, 1));
        CG_TRY(t5.get(&vals, (size_t) nF));
        CG_CHECK_CUDA(cudaMemsetAsync(err2, 0, sizeof(int), st));
        k_owned_rank<<<grid_for(nC, B), B, 0, st>>>(nC, m->refXadj, m->refAdj, s.c1, rank, err2);
        CG_LAUNCHED();
        int herr2 = 0;
        CG_CHECK_CUDA(cudaMemcpyAsync(&herr2, err2, sizeof(int), cudaMemcpyDeviceToHost, st));
        CG_CHECK_CUDA(cudaStreamSynchronize(st));
        if (!herr2) {
            k_face_slice_keys<<<grid_for(nF, B), B, 0, st>>>(nF, s.c1, m->cellO2N, rank, keys);
            CG_LAUNCHED();
            k_iota<<<grid_for(nF, B), B, 0, st>>>(nF, vals);
            CG_LAUNCHED();
            CG_TRY(sort_pairs(keys, keysOut, vals, m->faceN2O, nF, 10 + bits_for((uint64_t) (nC >> 5) + 1), st));
        } else {
            k_face_owner_keys<<<grid_for(nF, B), B, 0, st>>>(nF, s.c1, m->cellO2N, keys);
            CG_LAUNCHED();
            CG_TRY(sort_keys(keys, keysOut, nF, 32 + bits_for((uint64_t) nC), st));
            k_low32<<<grid_for(nF, B), B, 0, st>>>(nF, keysOut, m->faceN2O);
            CG_LAUNCHED();
        }
        CG_CHECK_CUDA(cudaStreamSynchronize(st));
    }
    k_invert<<<grid_for(nF, B), B, 0, st>>>(nF, m->faceN2O, m->faceO2N);
    CG_LAUNCHED();

    // --- xpac / xnac present?
    m->xpacZero = true;
    if (s.xpac && s.xnac) {
        int *flag;
        Tmp tf;
        CG_TRY(tf.get(&flag, 1));
        CG_CHECK_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), st));
        k_any_nonzero<<<grid_for(3 * (int64_t) nF, B), B, 0, st>>>(3 * (int64_t) nF, s.xpac, flag);
        CG_LAUNCHED();
        k_any_nonzero<<<grid_for(3 * (int64_t) nF, B), B, 0, st>>>(3 * (int64_t) nF, s.xnac, flag);
        CG_LAUNCHED();
        int h = 0;
        CG_CHECK_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
        CG_CHECK_CUDA(cudaStreamSynchronize(st));
        m->xpacZero = (h == 0);
    }

    // --- device layout
    bool f64 = m->precisions & (1 << CUPCFD_PREC_F64);
    bool f32 = m->precisions & (1 << CUPCFD_PREC_F32C);
    CG_TRY(m->alloc(&m->faceCells, (size_t) nF));
    if (f64) {
        CG_TRY(m->alloc(&m->fg64, (size_t) nF));
        CG_TRY(m->alloc(&m->fc64, (size_t) nF));
        CG_TRY(m->alloc(&m->cc64, (size_t) nC));
        if (!m->xpacZero) {
            CG_TRY(m->alloc(&m->fxp64, (size_t) nF));
            CG_TRY(m->alloc(&m->fxn64, (size_t) nF));
        }
    }
    if (f32) {
        CG_TRY(m->alloc(&m->fg32, (size_t) nF));
        CG_TRY(m->alloc(&m->fc32, (size_t) nF));
        CG_TRY(m->alloc(&m->cc32, (size_t) nC));
    }
    CG_TRY(m->alloc(&m->vol, (size_t) nC));
    k_layout_faces<<<grid_for(nF, B), B, 0, st>>>(nF, m->faceN2O, m->cellO2N, s.c1, s.c2, s.bnd, s.lam, s.area, s.S,
                                                 s.xf, s.xpac, s.xnac, m->faceCells, m->fg64, m->fc64, m->fxp64,
                                                 m->fxn64, m->fg32, m->fc32);
    CG_LAUNCHED();
    k_layout_cells<<<grid_for(nC, B), B, 0, st>>>(nC, m->cellN2O, s.cc, s.vol, m->cc64, m->cc32, m->vol);
    CG_LAUNCHED();

    // --- SELL-32 incidence lists
    int nSlices = (nC + 31) / 32;
    m->sell.nSlices = nSlices;
    {
        int *words;
        Tmp tw;
        CG_TRY(tw.get(&words, (size_t) nSlices + 1));
        CG_CHECK_CUDA(cudaMemsetAsync(words + nSlices, 0, sizeof(int), st));
        k_slice_width<<<grid_for((int64_t) nSlices * 32, B), B, 0, st>>>(nC, nSlices, m->cellN2O, m->refXadj, words);
        CG_LAUNCHED();
        {
            // The slice pointers are int: padded slices of wide cells can hold
            // more entries in all than an int counts even below 2^30 faces, so
            // the total is summed in 64 bits first and such meshes are refused.
            std::vector<int> hw((size_t) nSlices);
            CG_CHECK_CUDA(cudaMemcpyAsync(hw.data(), words, sizeof(int) * (size_t) nSlices, cudaMemcpyDeviceToHost, st));
            CG_CHECK_CUDA(cudaStreamSynchronize(st));
            int64_t total64 = 0;
            for (int w : hw) total64 += w;
            CG_RETURN_IF(total64 > (int64_t) INT_MAX, CUPCFD_E_NOT_IMPLEMENTED,
                         "mesh: padded incidence lists exceed 2^31 - 1 entries");
        }
        CG_TRY(m->alloc(&m->sell.slicePtr, (size_t) nSlices + 1));
        CG_TRY(exclusive_scan(words, m->sell.slicePtr, nSlices + 1, st));
        int total = 0;
        CG_CHECK_CUDA(cudaMemcpyAsync(&total, m->sell.slicePtr + nSlices, sizeof(int), cudaMemcpyDeviceToHost, st));
        CG_CHECK_CUDA(cudaStreamSynchronize(st));
        m->sell.nEntries = total;
        CG_TRY(m->alloc(&m->sell.inc, (size_t) total));
        k_fill_sell<<<grid_for((int64_t) nSlices * 32, B), B, 0, st>>>(nC, m->cellN2O, m->cellO2N, m->refXadj, m->refAdj,
                                                                      s.c1, s.c2, s.bnd, m->faceO2N, m->sell.slicePtr,
                                                                      m->sell.inc);
        CG_LAUNCHED();
    }
    {
        // max degree
        int *mx;
        Tmp tm;
        CG_TRY(tm.get(&mx, 1));
        size_t tb = 0;
        CG_CHECK_CUDA(cub::DeviceReduce::Max(nullptr, tb, deg, mx, nC, st));
        Tmp tt;
        void *tp;
        CG_TRY(tt.get((char **) &tp, tb));
        CG_CHECK_CUDA(cub::DeviceReduce::Max(tp, tb, deg, mx, nC, st));
        g_launches.fetch_add(1);
        CG_CHECK_CUDA(cudaMemcpyAsync(&m->maxDeg, mx, sizeof(int), cudaMemcpyDeviceToHost, st));
        CG_CHECK_CUDA(cudaStreamSynchronize(st));
        // every slice is maxDeg wide exactly when the entries fill 32 * maxDeg per slice
        // (CUPCFD_UNIFORM_SELL=0 keeps the slice-pointer lookup, for comparisons)
        const char *e = std::getenv("CUPCFD_UNIFORM_SELL");
        bool allow = !(e && std::strcmp(e, "0") == 0);
        m->sell.width = (allow && m->sell.nEntries == (int64_t) 32 * nSlices * m->maxDeg) ? m->maxDeg : 0;
    }

    // --- boundary maps for the boundary loops
    if (nB > 0) {
        CG_TRY(m->alloc(&m->bndFaceRef, (size_t) nB));
        CG_TRY(m->alloc(&m->bndFaceInt, (size_t) nB));
        CG_TRY(m->alloc(&m->bndSorted, (size_t) nB));
        CG_TRY(m->alloc(&m->bndSortedCellInt, (size_t) nB));
        CG_TRY(m->alloc(&m->bndSortedCellRef, (size_t) nB));
        uint64_t *keys, *keysOut;
        int *berr;
        Tmp tk1, tk2, tk3;
        CG_TRY(tk1.get(&keys, (size_t) nB));
        CG_TRY(tk2.get(&keysOut, (size_t) nB));
        CG_TRY(tk3.get(&berr, 1));
        CG_CHECK_CUDA(cudaMemsetAsync(m->bndFaceRef, 0xFF, sizeof(int) * (size_t) nB, st));
        CG_CHECK_CUDA(cudaMemsetAsync(keys, 0xFF, sizeof(uint64_t) * (size_t) nB, st));
        CG_CHECK_CUDA(cudaMemsetAsync(berr, 0, sizeof(int), st));
        k_bnd_maps<<<grid_for(nF, B), B, 0, st>>>(nF, nB, m->faceN2O, s.bnd, m->faceCells, m->bndFaceRef, m->bndFaceInt,
                                                  (unsigned long long *) keys, berr);
        CG_LAUNCHED();
        int hb = 0;
        CG_CHECK_CUDA(cudaMemcpyAsync(&hb, berr, sizeof(int), cudaMemcpyDeviceToHost, st));
        CG_CHECK_CUDA(cudaStreamSynchronize(st));
        if (hb == 0) {
            CG_TRY(sort_keys(keys, keysOut, nB, 64, st));
            k_bnd_unkey<<<grid_for(nB, B), B, 0, st>>>(nB, (const unsigned long long *) keysOut, m->cellN2O,
                                                       m->bndFaceRef, m->bndSorted, m->bndSortedCellInt,
                                                       m->bndSortedCellRef, berr);
            CG_LAUNCHED();
            CG_CHECK_CUDA(cudaMemcpyAsync(&hb, berr, sizeof(int), cudaMemcpyDeviceToHost, st));
            CG_CHECK_CUDA(cudaStreamSynchronize(st));
        }
        m->bndMapsOk = hb == 0;
    } else {
        m->bndMapsOk = true;
    }

    // --- numbering bandwidth and the fused pipeline's control words (api.cu)
    CG_TRY(mesh_post_build(m, st));

    // --- one default region
    m->nR = 1;
    CG_TRY(m->alloc(&m->bndRegion, (size_t) std::max(nB, 1)));
    CG_TRY(m->alloc(&m->regionType, 1));
    CG_TRY(m->alloc(&m->regionUVW, 3));
    CG_TRY(m->alloc(&m->regionDen, 1));
    CG_TRY(m->alloc(&m->regionSplvl, 1));
    CG_CHECK_CUDA(cudaMemsetAsync(m->regionSplvl, 0, sizeof(double), st));
    CG_CHECK_CUDA(cudaMemsetAsync(m->bndRegion, 0, sizeof(int) * (size_t) std::max(nB, 1), st));
    CG_CHECK_CUDA(cudaMemsetAsync(m->regionType, 0, sizeof(int), st));
    CG_CHECK_CUDA(cudaMemsetAsync(m->regionUVW, 0, 3 * sizeof(double), st));
    CG_CHECK_CUDA(cudaMemsetAsync(m->regionDen, 0, sizeof(double), st));
    m->hRegionType.assign(1, CUPCFD_RTYPE_DEFAULT);
    m->allDefaultRegions = true;
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    return CUPCFD_E_SUCCESS;
}

}  // namespace cupcfd_gpu

// ===========================================================================
// ABI: mesh
// ===========================================================================
extern "C" const char *cupcfd_gpu_last_error(void) { return t_last_error.c_str(); }
extern "C" const char *cupcfd_gpu_version(void) { return "cupcfd_gpu 0.1 (sm_100a)"; }
extern "C" int64_t cupcfd_gpu_launch_count(void) { return g_launches.load(); }

namespace {

__global__ void k_f32_to_f64(int64_t n, const float *__restrict__ a, double *__restrict__ b) {
    int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (double) a[i];
}

int upload_real(const void *h, int64_t n, int rs, double *dst, float *stage, cudaStream_t st) {
    if (rs == 8) {
        CG_CHECK_CUDA(cudaMemcpyAsync(dst, h, (size_t) n * 8, cudaMemcpyHostToDevice, st));
    } else {
        CG_CHECK_CUDA(cudaMemcpyAsync(stage, h, (size_t) n * 4, cudaMemcpyHostToDevice, st));
        k_f32_to_f64<<<grid_for(n, 256), 256, 0, st>>>(n, stage, dst);
        CG_LAUNCHED();
    }
    return CUPCFD_E_SUCCESS;
}

// span: device staging of the view's span (strided.cuh)
int upload_vec3(const cupcfd_vec3_view &v, int64_t n, int rs, double *dst, float *stage, void *span, cudaStream_t st) {
    CG_RETURN_IF(v.stride < 3 * rs || v.offset < 0 || v.offset + 3 * rs > v.stride, CUPCFD_E_CONFIG_INVALID_VALUE,
                 "vec3 view: bad stride/offset");
    if (rs == 8) {
        CG_TRY(upload_vec3_span(v.base, v.stride, v.offset, n, 8, span, dst, st));
    } else {
        CG_TRY(upload_vec3_span(v.base, v.stride, v.offset, n, 4, span, stage, st));
        k_f32_to_f64<<<grid_for(3 * n, 256), 256, 0, st>>>(3 * n, stage, dst);
        CG_LAUNCHED();
    }
    return CUPCFD_E_SUCCESS;
}

struct Bufs {
    std::vector<void *> p;
    ~Bufs() { for (void *q : p) cudaFree(q); }
    template <class T>
    T *get(size_t n) {
        void *q = nullptr;
        if (cudaMalloc(&q, (n ? n : 1) * sizeof(T)) != cudaSuccess) return nullptr;
        p.push_back(q);
        return (T *) q;
    }
};

int new_mesh(const cupcfd_mesh_options *opt, cupcfd_gpu_mesh **out) {
    CG_RETURN_IF(!out, CUPCFD_E_NULL_PTR, "mesh: null output pointer");
    *out = nullptr;
    int dev = opt ? opt->device : -1;
    CG_TRY(make_device_current(dev));
    cupcfd_gpu_mesh *m = new cupcfd_gpu_mesh();
    CG_CHECK_CUDA(cudaGetDevice(&m->device));
    cudaError_t e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete m;
        set_error(std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
        return CUPCFD_E_ERROR;
    }
    *out = m;
    return CUPCFD_E_SUCCESS;
}

}  // namespace

extern "C" int cupcfd_gpu_mesh_destroy(cupcfd_gpu_mesh *m) {
    if (!m) return CUPCFD_E_NULL_PTR;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    if (m->outStream) cudaStreamSynchronize(m->outStream);
    if (m->inStream) cudaStreamSynchronize(m->inStream);
    for (auto &b : m->owned) cudaFree(b.p);
    for (auto &b : m->scratch)
        if (b.p) cudaFree(b.p);
    for (cudaEvent_t e : m->pipeEv)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : m->inEv)
        if (e) cudaEventDestroy(e);
    if (m->outStream) cudaStreamDestroy(m->outStream);
    if (m->inStream) cudaStreamDestroy(m->inStream);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_mesh_create(const cupcfd_mesh_view *v, const cupcfd_mesh_options *opt, cupcfd_gpu_mesh **out) {
    clear_error();
    CG_RETURN_IF(!v || !out, CUPCFD_E_NULL_PTR, "mesh_create: null view or output");
    CG_RETURN_IF(v->real_size != 4 && v->real_size != 8, CUPCFD_E_CONFIG_INVALID_VALUE, "mesh_create: real_size must be 4 or 8");
    CG_RETURN_IF(!v->faceCell1 || !v->faceCell2 || !v->faceBnd || !v->faceLambda || !v->faceArea || !v->faceNorm.base ||
                     !v->faceCenter.base || !v->cellCenter.base || !v->cellVolume,
                 CUPCFD_E_NULL_PTR, "mesh_create: a required array is null");
    CG_RETURN_IF(v->nCells <= 0 || v->nFaces <= 0 || v->nBoundaries < 0, CUPCFD_E_ARRAY_SIZE_MISMATCH,
                 "mesh_create: sizes must be positive");
    cupcfd_gpu_mesh *m;
    CG_TRY(new_mesh(opt, &m));
    int nC = v->nCells, nF = v->nFaces, rs = v->real_size;
    cudaStream_t st = m->stream;
    // staging for the source in reference numbering
    Bufs b;
    Source s{};
    s.nC = nC; s.nF = nF; s.nB = v->nBoundaries;
    s.c1 = b.get<int>(nF); s.c2 = b.get<int>(nF); s.bnd = b.get<int>(nF);
    s.lam = b.get<double>(nF); s.area = b.get<double>(nF);
    s.S = b.get<double>(3 * (size_t) nF); s.xf = b.get<double>(3 * (size_t) nF);
    s.cc = b.get<double>(3 * (size_t) nC); s.vol = b.get<double>(nC);
    bool hasX = v->faceXpac.base && v->faceXnac.base;
    if (hasX) { s.xpac = b.get<double>(3 * (size_t) nF); s.xnac = b.get<double>(3 * (size_t) nF); }
    float *stage = rs == 4 ? b.get<float>(3 * (size_t) std::max(nF, nC)) : nullptr;
    size_t spanBytes = 1;
    for (const cupcfd_vec3_view *w : {&v->faceNorm, &v->faceCenter, &v->cellCenter, &v->faceXpac, &v->faceXnac})
        if (w->base && w->stride != 3 * rs)
            spanBytes = std::max(spanBytes, vec3_span_bytes(w == &v->cellCenter ? nC : nF, w->stride, w->offset, rs));
    void *span = b.get<char>(spanBytes);
    int rc = CUPCFD_E_SUCCESS;
    if (!s.c1 || !s.c2 || !s.bnd || !s.lam || !s.area || !s.S || !s.xf || !s.cc || !s.vol || (hasX && (!s.xpac || !s.xnac)) ||
        (rs == 4 && !stage) || !span) {
        set_error("mesh_create: out of device memory for the source arrays");
        rc = CUPCFD_E_ERROR;
    }
#define TRYRC(x) if (rc == CUPCFD_E_SUCCESS) rc = (x)
    TRYRC(cudaMemcpyAsync(s.c1, v->faceCell1, 4 * (size_t) nF, cudaMemcpyHostToDevice, st) == cudaSuccess ? 0 + CUPCFD_E_SUCCESS : CUPCFD_E_ERROR);
    TRYRC(cudaMemcpyAsync(s.c2, v->faceCell2, 4 * (size_t) nF, cudaMemcpyHostToDevice, st) == cudaSuccess ? 0 + CUPCFD_E_SUCCESS : CUPCFD_E_ERROR);
    TRYRC(cudaMemcpyAsync(s.bnd, v->faceBnd, 4 * (size_t) nF, cudaMemcpyHostToDevice, st) == cudaSuccess ? 0 + CUPCFD_E_SUCCESS : CUPCFD_E_ERROR);
    TRYRC(upload_real(v->faceLambda, nF, rs, s.lam, stage, st));
    TRYRC(upload_real(v->faceArea, nF, rs, s.area, stage, st));
    TRYRC(upload_real(v->cellVolume, nC, rs, s.vol, stage, st));
    TRYRC(upload_vec3(v->faceNorm, nF, rs, s.S, stage, span, st));
    TRYRC(upload_vec3(v->faceCenter, nF, rs, s.xf, stage, span, st));
    TRYRC(upload_vec3(v->cellCenter, nC, rs, s.cc, stage, span, st));
    if (hasX) {
        TRYRC(upload_vec3(v->faceXpac, nF, rs, s.xpac, stage, span, st));
        TRYRC(upload_vec3(v->faceXnac, nF, rs, s.xnac, stage, span, st));
    }
    if (rc == CUPCFD_E_SUCCESS && cudaStreamSynchronize(st) != cudaSuccess) {
        set_error("mesh_create: upload failed");
        rc = CUPCFD_E_ERROR;
    }
    TRYRC(build_mesh_from_source(m, s, opt));
#undef TRYRC
    if (rc != CUPCFD_E_SUCCESS) {
        std::string e = t_last_error;
        cupcfd_gpu_mesh_destroy(m);
        set_error(e);
        return rc;
    }
    m->realSize = rs;
    *out = m;
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_mesh_get_info(const cupcfd_gpu_mesh *m, cupcfd_mesh_info *info) {
    CG_RETURN_IF(!m || !info, CUPCFD_E_NULL_PTR, "mesh_get_info: null argument");
    info->nCells = m->nC;
    info->nFaces = m->nF;
    info->nInteriorFaces = m->nFi;
    info->nBoundaries = m->nB;
    info->nRegions = m->nR;
    info->nIncidences = m->nInc;
    info->maxCellFaces = m->maxDeg;
    info->order = m->order;
    info->precisions = m->precisions;
    info->bandwidth = m->bandwidth;
    info->deviceBytes = m->bytes;
    info->tiles = m->tiles ? 1 : 0;
    info->fullWidth = m->tiles ? m->fullWidth : 0;
    return CUPCFD_E_SUCCESS;
}

namespace {
__global__ void k_check_regions(int nB, int nR, const int *__restrict__ br, int *__restrict__ err) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nB && (br[i] < 0 || br[i] >= nR)) atomicOr(err, 1);
}
}  // namespace

extern "C" int cupcfd_gpu_mesh_set_regions(cupcfd_gpu_mesh *m, int32_t nR, const int32_t *type, const double *uvw,
                                           const double *den, const int32_t *bndRegion, int32_t nB) {
    clear_error();
    CG_RETURN_IF(!m || !type || !uvw || !den || (!bndRegion && nB > 0), CUPCFD_E_NULL_PTR, "set_regions: null argument");
    CG_RETURN_IF(nR <= 0, CUPCFD_E_ARRAY_SIZE_MISMATCH, "set_regions: nRegions must be positive");
    CG_RETURN_IF(nB != m->nB, CUPCFD_E_ARRAY_SIZE_MISMATCH, "set_regions: nBoundaries differs from the mesh");
    for (int r = 0; r < nR; r++)
        CG_RETURN_IF(type[r] < CUPCFD_RTYPE_DEFAULT || type[r] > CUPCFD_RTYPE_WALL, CUPCFD_E_CONFIG_INVALID_VALUE,
                     "set_regions: unknown region type");
    CG_TRY(make_device_current(m->device));
    cudaStream_t st = m->stream;
    if (nR > m->nR) {
        CG_TRY(m->alloc(&m->regionType, (size_t) nR));
        CG_TRY(m->alloc(&m->regionUVW, 3 * (size_t) nR));
        CG_TRY(m->alloc(&m->regionDen, (size_t) nR));
        CG_TRY(m->alloc(&m->regionSplvl, (size_t) nR));
    }
    CG_CHECK_CUDA(cudaMemsetAsync(m->regionSplvl, 0, sizeof(double) * nR, st));
    CG_CHECK_CUDA(cudaMemcpyAsync(m->regionType, type, sizeof(int) * nR, cudaMemcpyHostToDevice, st));
    CG_CHECK_CUDA(cudaMemcpyAsync(m->regionUVW, uvw, sizeof(double) * 3 * nR, cudaMemcpyHostToDevice, st));
    CG_CHECK_CUDA(cudaMemcpyAsync(m->regionDen, den, sizeof(double) * nR, cudaMemcpyHostToDevice, st));
    if (nB > 0) {
        int *err;
        void *ev;
        CG_TRY(m->scratchBuf(0, sizeof(int), &ev));
        err = (int *) ev;
        CG_CHECK_CUDA(cudaMemcpyAsync(m->bndRegion, bndRegion, sizeof(int) * nB, cudaMemcpyHostToDevice, st));
        CG_CHECK_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
        k_check_regions<<<grid_for(nB, 256), 256, 0, st>>>(nB, nR, m->bndRegion, err);
        CG_LAUNCHED();
        int h = 0;
        CG_CHECK_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st));
        CG_CHECK_CUDA(cudaStreamSynchronize(st));
        CG_RETURN_IF(h != 0, CUPCFD_E_INVALID_INDEX, "set_regions: a boundary's region id is out of range");
    }
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    m->nR = nR;
    m->hRegionType.assign(type, type + nR);
    m->uvwCarryValid = false;  // the carried-value sources depend on the region types
    if (m->regionFT && nR <= m->regionFTcap) {
        CG_CHECK_CUDA(cudaMemsetAsync(m->regionFT, 0, sizeof(double) * 3 * nR, st));
        CG_CHECK_CUDA(cudaStreamSynchronize(st));
    } else {
        m->regionFTcap = 0;  // reallocated (zeroed) by the next momentum loop
    }
    m->allDefaultRegions = true;
    for (int r = 0; r < nR; r++)
        if (type[r] != CUPCFD_RTYPE_DEFAULT) m->allDefaultRegions = false;
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_mesh_get_cell_face_csr(const cupcfd_gpu_mesh *m, int32_t *xadj, int32_t nXAdj, int32_t *adj,
                                                 int32_t nAdj) {
    clear_error();
    CG_RETURN_IF(!m || !xadj || !adj, CUPCFD_E_NULL_PTR, "get_cell_face_csr: null argument");
    CG_RETURN_IF(nXAdj != m->nC + 1 || nAdj != m->nInc, CUPCFD_E_ARRAY_SIZE_MISMATCH, "get_cell_face_csr: size mismatch");
    CG_TRY(make_device_current(m->device));
    CG_CHECK_CUDA(cudaMemcpyAsync(xadj, m->refXadj, sizeof(int) * nXAdj, cudaMemcpyDeviceToHost, m->stream));
    CG_CHECK_CUDA(cudaMemcpyAsync(adj, m->refAdj, sizeof(int) * (size_t) nAdj, cudaMemcpyDeviceToHost, m->stream));
    CG_CHECK_CUDA(cudaStreamSynchronize(m->stream));
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_mesh_get_incidences(const cupcfd_gpu_mesh *m, int32_t *xadj, int32_t nXAdj, int32_t *face,
                                              int32_t *other, int32_t nInc) {
    clear_error();
    CG_RETURN_IF(!m || !xadj || !face || !other, CUPCFD_E_NULL_PTR, "get_incidences: null argument");
    CG_RETURN_IF(nXAdj != m->nC + 1 || nInc != m->nInc, CUPCFD_E_ARRAY_SIZE_MISMATCH, "get_incidences: size mismatch");
    CG_TRY(make_device_current(m->device));
    const int nS = m->sell.nSlices;
    std::vector<int> sp((size_t) nS + 1);
    std::vector<int2> inc((size_t) m->sell.nEntries);
    CG_CHECK_CUDA(cudaMemcpyAsync(sp.data(), m->sell.slicePtr, sizeof(int) * sp.size(), cudaMemcpyDeviceToHost, m->stream));
    CG_CHECK_CUDA(cudaMemcpyAsync(inc.data(), m->sell.inc, sizeof(int2) * inc.size(), cudaMemcpyDeviceToHost, m->stream));
    CG_CHECK_CUDA(cudaStreamSynchronize(m->stream));
    int64_t k = 0;
    xadj[0] = 0;
    for (int c = 0; c < m->nC; c++) {
        const int s = c >> 5, lane = c & 31, w = (sp[s + 1] - sp[s]) >> 5;
        for (int j = 0; j < w; j++) {
            const int2 e = inc[(size_t) sp[s] + 32 * (size_t) j + lane];
            if (e.x < 0) break;  // padding follows a cell's real entries
            CG_RETURN_IF(k >= nInc, CUPCFD_E_ERROR, "get_incidences: more entries than incidences");
            face[k] = e.x;
            other[k] = e.y;
            k++;
        }
        xadj[c + 1] = (int32_t) k;
    }
    CG_RETURN_IF(k != nInc, CUPCFD_E_ERROR, "get_incidences: fewer entries than incidences");
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_mesh_get_numbering(const cupcfd_gpu_mesh *m, int32_t *cellN2O, int32_t *faceN2O) {
    clear_error();
    CG_RETURN_IF(!m, CUPCFD_E_NULL_PTR, "get_numbering: null mesh");
    CG_TRY(make_device_current(m->device));
    if (cellN2O) CG_CHECK_CUDA(cudaMemcpyAsync(cellN2O, m->cellN2O, sizeof(int) * (size_t) m->nC, cudaMemcpyDeviceToHost, m->stream));
    if (faceN2O) CG_CHECK_CUDA(cudaMemcpyAsync(faceN2O, m->faceN2O, sizeof(int) * (size_t) m->nF, cudaMemcpyDeviceToHost, m->stream));
    CG_CHECK_CUDA(cudaStreamSynchronize(m->stream));
    return CUPCFD_E_SUCCESS;
}

namespace {
__global__ void k_geom_to_ref(int nF, int nC, const int *__restrict__ faceN2O, const int *__restrict__ cellN2O,
                              const int2 *__restrict__ fcells, const double4 *__restrict__ fg, const double4 *__restrict__ fc,
                              const double4 *__restrict__ cc, const double *__restrict__ vol, int *c1, int *c2, int *bnd,
                              double *lam, double *area, double *S, double *xf, double *ccOut, double *volOut) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nF) {
        int o = faceN2O[i];
        int2 pc = fcells[i];
        c1[o] = cellN2O[pc.x];
        c2[o] = pc.y >= 0 ? cellN2O[pc.y] : -1;
        bnd[o] = pc.y >= 0 ? -1 : -1 - pc.y;
        double4 g = fg[i], c = fc[i];
        lam[o] = g.w; area[o] = c.w;
        S[3 * o] = g.x; S[3 * o + 1] = g.y; S[3 * o + 2] = g.z;
        xf[3 * o] = c.x; xf[3 * o + 1] = c.y; xf[3 * o + 2] = c.z;
    }
    if (i < nC) {
        int o = cellN2O[i];
        double4 p = cc[i];
        ccOut[3 * o] = p.x; ccOut[3 * o + 1] = p.y; ccOut[3 * o + 2] = p.z;
        volOut[o] = vol[i];
    }
}
}  // namespace

extern "C" int cupcfd_gpu_mesh_get_geometry(const cupcfd_gpu_mesh *mc, int32_t *faceCell1, int32_t *faceCell2,
                                            int32_t *faceBnd, double *faceLambda, double *faceArea, double *faceNorm,
                                            double *faceCenter, double *cellCenter, double *cellVolume) {
    clear_error();
    cupcfd_gpu_mesh *m = const_cast<cupcfd_gpu_mesh *>(mc);
    CG_RETURN_IF(!m, CUPCFD_E_NULL_PTR, "get_geometry: null mesh");
    CG_RETURN_IF(!m->fg64, CUPCFD_E_NOT_IMPLEMENTED, "get_geometry: mesh holds no FP64 geometry");
    CG_TRY(make_device_current(m->device));
    size_t nF = m->nF, nC = m->nC;
    size_t off[10], tot = 0;
    size_t sz[10] = {4 * nF, 4 * nF, 4 * nF, 8 * nF, 8 * nF, 24 * nF, 24 * nF, 24 * nC, 8 * nC, 0};
    for (int k = 0; k < 9; k++) { off[k] = tot; tot += (sz[k] + 255) / 256 * 256; }
    void *buf;
    CG_TRY(m->scratchBuf(1, tot, &buf));
    char *b = (char *) buf;
    int n = (int) std::max(nF, nC);
    k_geom_to_ref<<<grid_for(n, 256), 256, 0, m->stream>>>(
        m->nF, m->nC, m->faceN2O, m->cellN2O, m->faceCells, m->fg64, m->fc64, m->cc64, m->vol, (int *) (b + off[0]),
        (int *) (b + off[1]), (int *) (b + off[2]), (double *) (b + off[3]), (double *) (b + off[4]),
        (double *) (b + off[5]), (double *) (b + off[6]), (double *) (b + off[7]), (double *) (b + off[8]));
    CG_LAUNCHED();
    void *outs[9] = {faceCell1, faceCell2, faceBnd, faceLambda, faceArea, faceNorm, faceCenter, cellCenter, cellVolume};
    for (int k = 0; k < 9; k++)
        if (outs[k]) CG_CHECK_CUDA(cudaMemcpyAsync(outs[k], b + off[k], sz[k], cudaMemcpyDeviceToHost, m->stream));
    CG_CHECK_CUDA(cudaStreamSynchronize(m->stream));
    return CUPCFD_E_SUCCESS;
}

// Generators (structgen / jittered) live in generators.cu and call back here.
namespace cupcfd_gpu {
int mesh_new(const cupcfd_mesh_options *opt, cupcfd_gpu_mesh **out) { return new_mesh(opt, out); }
}  // namespace cupcfd_gpu
