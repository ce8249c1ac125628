// Numbering conversions between the reference's arrays and the mesh's
// internal numbering (gathers and their inverses), used by the host-buffer
// calls of several translation units. The kernels sit in an unnamed
// namespace: each translation unit that includes this header gets its own
// copies, so no kernel symbol is defined twice.
#pragma once

#include <cstdint>

namespace {

// ---------------------------------------------------------------------------
// permutation kernels (gathers): dst[c][i] = src[c][map[i]]
// ---------------------------------------------------------------------------
template <class TS, class TD>
__global__ void k_gather(int n, int ncomp, const int *__restrict__ map, const TS *__restrict__ src, int64_t ss,
                         TD *__restrict__ dst, int64_t dsd) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int j = map ? map[i] : i;
    for (int c = 0; c < ncomp; c++) dst[c * dsd + i] = (TD) src[c * ss + j];
}

// reference-order AoS [n][ncomp] (packed) -> internal component blocks
template <class TS, class TD>
__global__ void k_aos_to_blocks(int n, int ncomp, const int *__restrict__ n2o, const TS *__restrict__ src,
                                TD *__restrict__ dst, int64_t ld) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int o = n2o[i];
    for (int c = 0; c < ncomp; c++) dst[c * ld + i] = (TD) src[(int64_t) o * ncomp + c];
}

// internal component blocks -> reference-order AoS [n][ncomp]
template <class TS, class TD>
__global__ void k_blocks_to_aos(int n, int ncomp, const int *__restrict__ o2n, const TS *__restrict__ src, int64_t ld,
                                TD *__restrict__ dst) {
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    int i = o2n[o];
    for (int c = 0; c < ncomp; c++) dst[(int64_t) o * ncomp + c] = (TD) src[c * ld + i];
}

// float4 state <-> blocks
template <class TS>
__global__ void k_state_to_f4(int n, const int *__restrict__ n2o, const TS *__restrict__ r, const TS *__restrict__ u,
                              const TS *__restrict__ v, const TS *__restrict__ w, float4 *__restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int o = n2o[i];
    out[i] = make_float4((float) r[o], (float) u[o], (float) v[o], (float) w[o]);
}

template <class TD>
__global__ void k_f4_to_ref(int n, const int *__restrict__ o2n, const float4 *__restrict__ in, TD *__restrict__ r,
                            TD *__restrict__ u, TD *__restrict__ v, TD *__restrict__ w) {
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    float4 s = in[o2n[o]];
    r[o] = s.x; u[o] = s.y; v[o] = s.z; w[o] = s.w;
}

// face data internal -> reference (boundary entries zero when zeroBnd)
template <class TS, class TD = double>
__global__ void k_faces_to_ref(int nF, const int *__restrict__ o2n, const int2 *__restrict__ fcells, const TS *__restrict__ src,
                               TD *__restrict__ dst, int zeroBnd) {
    int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nF) return;
    int i = o2n[o];
    dst[o] = (zeroBnd && fcells[i].y < 0) ? TD(0) : (TD) src[i];
}

template <class TS, class TD>
__global__ void k_convert(int64_t n, const TS *__restrict__ a, TD *__restrict__ b) {
    int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (TD) a[i];
}

// rface pairs: dst[2i], dst[2i+1] = src[2 map[i]], src[2 map[i]+1]
template <class T>
__global__ void k_gather_pairs(int n, const int *__restrict__ map, const T *__restrict__ src, T *__restrict__ dst) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int j = map[i];
    dst[2 * (int64_t) i] = src[2 * (int64_t) j];
    dst[2 * (int64_t) i + 1] = src[2 * (int64_t) j + 1];
}

}  // namespace
