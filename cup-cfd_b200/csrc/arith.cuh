// FP64 operations with explicit round-to-nearest, one IEEE rounding each and
// no contraction: the reference's arithmetic, operator by operator.
#pragma once

namespace cupcfd_gpu {

__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

}  // namespace cupcfd_gpu
