// sw_storage.cuh -- conversions of the 16-bit storage form (sw_config.storage
// = SW_STORE_BF16 or SW_STORE_F16; no reference counterpart): FP32 values to
// bfloat16 or IEEE half with round-to-nearest-even, and back.  The kernels of
// that form are in sw_s16.cuh.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "sw_common.cuh"

namespace swb {

template <class S16>
__device__ __forceinline__ S16 to16(float x);
template <>
__device__ __forceinline__ __nv_bfloat16 to16<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }
template <>
__device__ __forceinline__ __half to16<__half>(float x) { return __float2half_rn(x); }
__device__ __forceinline__ float from16(__nv_bfloat16 x) { return __bfloat162float(x); }
__device__ __forceinline__ float from16(__half x) { return __half2float(x); }

}  // namespace swb
