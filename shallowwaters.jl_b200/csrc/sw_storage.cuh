// sw_storage.cuh -- the 16-bit storage form of the prognostic state
// (sw_config.storage = SW_STORE_BF16 or SW_STORE_F16; no reference counterpart).
//
// Between time steps every value of u, v and eta is held as a compensated
// pair of 16-bit numbers, hi + lo: hi = round16(s*x) and lo = round16(s*x - hi),
// where s is a power of two (sw_config.storage_scale_uv for u and v, 1 for
// eta).  lo keeps the rounding error of hi, as the compensation term of Kahan
// summation does, so increments far below one unit in the last place of hi
// still accumulate from step to step.  The tracer is held as one 16-bit number.
// Tendencies and the RK stages are computed in FP32; after each step the new
// state is rounded to this form in place (store_round_kernel), so the FP32
// buffers always hold exactly the values the 16-bit form represents.
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

// x -> the value of its compensated 16-bit pair at scale s (s, 1/s powers of two)
template <class S16>
__device__ __forceinline__ float round_pair(float x, float s, float inv_s) {
    const float y = x * s;
    const S16 hi = to16<S16>(y);
    const float r = y - from16(hi);          // exact: hi is y rounded to fewer bits
    const S16 lo = to16<S16>(r);
    return (from16(hi) + from16(lo)) * inv_s;
}

// Rounds n elements of u, v (scale s_uv), eta (scale 1) to compensated pairs
// and sst to single 16-bit values, in place.  Padding cells are zero and stay
// zero; halo cells are rounded like the cells they copy, so ghost copies stay
// consistent.
template <class S16>
__global__ void __launch_bounds__(256)
store_round_kernel(float* u, float* v, float* e, float* sst, long long n, float s_uv, float inv_s_uv) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        u[k] = round_pair<S16>(u[k], s_uv, inv_s_uv);
        v[k] = round_pair<S16>(v[k], s_uv, inv_s_uv);
        e[k] = round_pair<S16>(e[k], 1.f, 1.f);
        sst[k] = from16(to16<S16>(sst[k]));
    }
}

}  // namespace swb
