// Strided host vector arrays (the reference's EuclideanVector arrays: per
// record a vptr, then three components; cupcfd_vec3_view {base, stride,
// offset}) moved between host and device as whole spans. A strided
// cudaMemcpy2D over records of 24 bytes ran at a few hundred nanoseconds a
// record on B200 (6.3 M records from pageable memory: 0.9 s host to device,
// 1.7 s back, against 20 ms and 11 ms for one plain copy of the span).
//   in:  one copy of the records' whole span into device staging, then a
//        kernel picks the components out;
//   out: one copy of the packed components into host staging, then the host
//        writes each record's component bytes (the bytes in between, the
//        vptr, are left as they are).
// Kernels and helpers sit in an unnamed namespace (at file scope, as in
// perm.cuh): each translation unit that includes this header gets its own
// copies.
#pragma once

#include <cstdint>
#include <cstring>
#include <vector>

#include "internal.cuh"

namespace {

// dst[3 i + q] = component q of record i in the span (T-aligned records)
template <class T>
__global__ void k_unstride3(int64_t n, int stride, int offset, const char *__restrict__ span, T *__restrict__ dst) {
    const int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
    if (i >= n) return;
    const T *p = reinterpret_cast<const T *>(span + i * stride + offset);
    dst[3 * i] = p[0];
    dst[3 * i + 1] = p[1];
    dst[3 * i + 2] = p[2];
}

// the same byte by byte, for records that are not T-aligned
__global__ void k_unstride3_bytes(int64_t n, int stride, int offset, int bytes, const char *__restrict__ span,
                                  char *__restrict__ dst) {
    const int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int b = 0; b < bytes; b++) dst[i * bytes + b] = span[i * stride + offset + b];
}

// Bytes from the first record's start to the last record's last component.
inline size_t vec3_span_bytes(int64_t n, int stride, int offset, int rs) {
    return n > 0 ? (size_t) (n - 1) * stride + offset + 3 * (size_t) rs : 0;
}

// n records of three rs-byte components at base (stride, offset) -> packed
// device [3n]. stage: device scratch of vec3_span_bytes() bytes (unused when
// the records are packed already). Stream-ordered.
inline int upload_vec3_span(const void *base, int stride, int offset, int64_t n, int rs, void *stage, void *dst,
                            cudaStream_t st) {
    if (n <= 0) return CUPCFD_E_SUCCESS;
    const char *b = static_cast<const char *>(base);
    if (stride == 3 * rs) {
        CG_CHECK_CUDA(cudaMemcpyAsync(dst, b + offset, (size_t) n * 3 * rs, cudaMemcpyHostToDevice, st));
        return CUPCFD_E_SUCCESS;
    }
    CG_CHECK_CUDA(cudaMemcpyAsync(stage, b, vec3_span_bytes(n, stride, offset, rs), cudaMemcpyHostToDevice, st));
    const unsigned grid = (unsigned) ((n + 255) / 256);
    const char *sp = static_cast<const char *>(stage);
    if (stride % rs == 0 && offset % rs == 0) {
        if (rs == 8) k_unstride3<double><<<grid, 256, 0, st>>>(n, stride, offset, sp, static_cast<double *>(dst));
        else k_unstride3<float><<<grid, 256, 0, st>>>(n, stride, offset, sp, static_cast<float *>(dst));
    } else {
        k_unstride3_bytes<<<grid, 256, 0, st>>>(n, stride, offset, 3 * rs, sp, static_cast<char *>(dst));
    }
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}

// packed components [3n] in host memory -> the component bytes of n host
// records (stride, offset)
inline void scatter_vec3_host(const char *packed, void *base, int stride, int offset, int64_t n, int rs) {
    char *b = static_cast<char *>(base) + offset;
    const size_t rec = 3 * (size_t) rs;
    for (int64_t i = 0; i < n; i++) std::memcpy(b + (size_t) i * stride, packed + (size_t) i * rec, rec);
}

// packed device [3n] -> the component bytes of n host records (stride,
// offset). A packed destination is copied into directly (stream-ordered);
// otherwise the copy goes through host staging and the call returns once the
// records are written.
inline int download_vec3_span(const void *src, void *base, int stride, int offset, int64_t n, int rs,
                              std::vector<char> &hstage, cudaStream_t st) {
    if (n <= 0) return CUPCFD_E_SUCCESS;
    char *b = static_cast<char *>(base) + offset;
    const size_t rec = 3 * (size_t) rs;
    if (stride == 3 * rs) {
        CG_CHECK_CUDA(cudaMemcpyAsync(b, src, (size_t) n * rec, cudaMemcpyDeviceToHost, st));
        return CUPCFD_E_SUCCESS;
    }
    if (hstage.size() < (size_t) n * rec) hstage.resize((size_t) n * rec);
    CG_CHECK_CUDA(cudaMemcpyAsync(hstage.data(), src, (size_t) n * rec, cudaMemcpyDeviceToHost, st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));
    scatter_vec3_host(hstage.data(), base, stride, offset, n, rs);
    return CUPCFD_E_SUCCESS;
}

}  // namespace
