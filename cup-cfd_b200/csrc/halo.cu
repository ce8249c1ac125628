// Halo exchange support for meshes split across ranks: packing the owned
// cells the peers need into one contiguous send buffer (peer after peer, the
// CSR layout of the reference's send lists), and unpacking a received
// buffer into this rank's ghost cells. Replaces the pack / unpack halves of
// the reference's ExchangePatternTwoSidedNonBlocking
// (src/comm/implementation/component/ExchangePatternTwoSidedNonBlocking.cpp:
// packSendBuffer :129, unpackRecvBuffer :150); the transfer itself is left
// to the caller's communicator (NCCL send / recv through torch.distributed).
//
//   pack:   dst[i * ncomp + c]   = src[c * ld + idx[i]]   (i < n, c < ncomp)
//   unpack: dst[c * ld + idx[i]] = src[i * ncomp + c]
// (element-major buffers, so each peer's part of a buffer is contiguous)
//
// Element sizes 4, 8 and 16 bytes (a float4 state record is one element).
// Indices are in the mesh's internal numbering, on the device.
#include <cstdint>

#include "internal.cuh"

using namespace cupcfd_gpu;

namespace {

constexpr int HB = 256;

template <class T>
__global__ void k_pack(int n, int ncomp, int64_t ld, const int *__restrict__ idx, const T *__restrict__ src,
                       T *__restrict__ dst) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t j = idx[i];
    for (int c = 0; c < ncomp; c++) dst[(int64_t) i * ncomp + c] = src[c * ld + j];
}

template <class T>
__global__ void k_unpack(int n, int ncomp, int64_t ld, const int *__restrict__ idx, const T *__restrict__ src,
                         T *__restrict__ dst) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t j = idx[i];
    for (int c = 0; c < ncomp; c++) dst[c * ld + j] = src[(int64_t) i * ncomp + c];
}

int launch(bool pack, int elemSize, int n, int ncomp, int64_t ld, const int *idx, const void *src, void *dst,
           cudaStream_t st) {
    unsigned grid = grid_for(n, HB);
    switch (elemSize) {
    case 4:
        if (pack) k_pack<float><<<grid, HB, 0, st>>>(n, ncomp, ld, idx, (const float *) src, (float *) dst);
        else k_unpack<float><<<grid, HB, 0, st>>>(n, ncomp, ld, idx, (const float *) src, (float *) dst);
        break;
    case 8:
        if (pack) k_pack<double><<<grid, HB, 0, st>>>(n, ncomp, ld, idx, (const double *) src, (double *) dst);
        else k_unpack<double><<<grid, HB, 0, st>>>(n, ncomp, ld, idx, (const double *) src, (double *) dst);
        break;
    default:
        if (pack) k_pack<float4><<<grid, HB, 0, st>>>(n, ncomp, ld, idx, (const float4 *) src, (float4 *) dst);
        else k_unpack<float4><<<grid, HB, 0, st>>>(n, ncomp, ld, idx, (const float4 *) src, (float4 *) dst);
        break;
    }
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}

int check(int elemSize, int n, int ncomp, int64_t ld, const void *idx, const void *src, void *dst) {
    CG_RETURN_IF(n < 0 || ncomp <= 0 || (n > 0 && (!idx || !src || !dst)), CUPCFD_E_NULL_PTR, "halo: null argument");
    CG_RETURN_IF(elemSize != 4 && elemSize != 8 && elemSize != 16, CUPCFD_E_CONFIG_INVALID_VALUE,
                 "halo: element size must be 4, 8 or 16");
    CG_RETURN_IF(ncomp > 1 && ld <= 0, CUPCFD_E_CONFIG_INVALID_VALUE, "halo: component stride must be positive");
    CG_RETURN_IF(((uintptr_t) src | (uintptr_t) dst) % elemSize != 0, CUPCFD_E_CONFIG_INVALID_VALUE,
                 "halo: arrays must be aligned to their element");
    return CUPCFD_E_SUCCESS;
}

// Several fields in one launch: blockIdx.y is the field.
constexpr int HALO_MAX_FIELDS = 8;
struct FieldSet {
    cupcfd_halo_field f[HALO_MAX_FIELDS];
};

template <class T>
__device__ __forceinline__ void move(bool pack, int i, int ncomp, int64_t ld, int64_t j, const cupcfd_halo_field &f) {
    T *field = static_cast<T *>(f.field), *buf = static_cast<T *>(f.buffer);
    for (int c = 0; c < ncomp; c++) {
        if (pack) buf[(int64_t) i * ncomp + c] = field[c * ld + j];
        else field[c * ld + j] = buf[(int64_t) i * ncomp + c];
    }
}

__global__ void k_halo_fields(bool pack, int n, const int *__restrict__ idx, const __grid_constant__ FieldSet fs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const cupcfd_halo_field &f = fs.f[blockIdx.y];
    const int64_t j = idx[i];
    switch (f.elemSize) {
    case 4: move<float>(pack, i, f.ncomp, f.ld, j, f); break;
    case 8: move<double>(pack, i, f.ncomp, f.ld, j, f); break;
    default: move<float4>(pack, i, f.ncomp, f.ld, j, f); break;
    }
}

int launch_fields(bool pack, const cupcfd_halo_field *fields, int nFields, const int32_t *idx, int32_t n,
                  cudaStream_t st) {
    CG_RETURN_IF(!fields || nFields < 0 || nFields > HALO_MAX_FIELDS, CUPCFD_E_CONFIG_INVALID_VALUE,
                 "halo: 0 to 8 fields per call");
    FieldSet fs{};
    for (int k = 0; k < nFields; k++) {
        const cupcfd_halo_field &f = fields[k];
        CG_TRY(check(f.elemSize, n, f.ncomp, f.ld, idx, f.field, f.buffer));
        fs.f[k] = f;
    }
    if (n == 0 || nFields == 0) return CUPCFD_E_SUCCESS;
    k_halo_fields<<<dim3(grid_for(n, HB), nFields), HB, 0, st>>>(pack, n, idx, fs);
    CG_LAUNCHED();
    return CUPCFD_E_SUCCESS;
}

}  // namespace

extern "C" int cupcfd_gpu_dev_halo_pack_fields(const cupcfd_halo_field *fields, int32_t nFields, const int32_t *idx,
                                               int32_t n, void *stream) {
    clear_error();
    return launch_fields(true, fields, nFields, idx, n, (cudaStream_t) stream);
}

extern "C" int cupcfd_gpu_dev_halo_unpack_fields(const cupcfd_halo_field *fields, int32_t nFields, const int32_t *idx,
                                                 int32_t n, void *stream) {
    clear_error();
    return launch_fields(false, fields, nFields, idx, n, (cudaStream_t) stream);
}

extern "C" int cupcfd_gpu_dev_halo_pack(const void *src, int32_t elemSize, int32_t ncomp, int64_t ld, const int32_t *idx,
                                        int32_t n, void *dst, void *stream) {
    clear_error();
    CG_TRY(check(elemSize, n, ncomp, ld, idx, src, dst));
    if (n == 0) return CUPCFD_E_SUCCESS;
    return launch(true, elemSize, n, ncomp, ld, idx, src, dst, (cudaStream_t) stream);
}

extern "C" int cupcfd_gpu_dev_halo_unpack(const void *src, int32_t elemSize, int32_t ncomp, int32_t n, const int32_t *idx,
                                          void *dst, int64_t ld, void *stream) {
    clear_error();
    CG_TRY(check(elemSize, n, ncomp, ld, idx, src, dst));
    if (n == 0) return CUPCFD_E_SUCCESS;
    return launch(false, elemSize, n, ncomp, ld, idx, src, dst, (cudaStream_t) stream);
}
