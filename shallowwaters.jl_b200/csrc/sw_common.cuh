// sw_common.cuh -- device layout and shared helpers of libswb200.
//
// Device layout.  Every field lives in a padded 2-D buffer of pitch P
// elements (P a multiple of 32) and R rows.  A point with physical x index X
// and y index Y is stored at  (Y + ROW0) * P + (X + COL0)  with COL0 = 4,
// ROW0 = 2, where
//   u at face F (x = F*Δ), row b      -> X = F, Y = b
//   v at column a, face G (y = G*Δ)   -> X = a, Y = G
//   eta, h, sst, H at T-cell (a, b)   -> X = a, Y = b
// The reference's Julia indices map as (src/grid.jl:26-66,
// src/initial_conditions.jl:18-21):
//   u[i,j]  : F = i - 2 - ep, b = j - 3      v[i,j] : a = i - 3, G = j - 2
//   eta[i,j]: a = i - 2,      b = j - 2      sst[i,j]: a = i - 2, b = j - 1
// so that interior u is F in [1-ep, N-1], v is G in [1, M-1], eta/sst a in
// [0, N-1], b in [0, M-1].  Buffers are zero-initialised; padding is never
// written.
#pragma once
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "swb200.h"

// unroll factor of the row-streaming loops
#ifndef SWB_UNROLL
#define SWB_UNROLL 2
#endif
#define SWB_PRAGMA(x) _Pragma(#x)
#define SWB_UNROLL_PRAGMA(n) SWB_PRAGMA(unroll n)
#define SWB_ROW_UNROLL SWB_UNROLL_PRAGMA(SWB_UNROLL)

namespace swb {

constexpr int COL0 = 4;
constexpr int ROW0 = 2;

struct Geom {
    int N, M;      // nx, ny
    int ep;        // 1 periodic, 0 nonperiodic
    int P;         // pitch (elements)
    int R;         // rows
    __host__ __device__ inline int idx(int x, int y) const {
        return (y + ROW0) * P + (x + COL0);
    }
    // interior ranges (inclusive lower, exclusive upper)
    __host__ __device__ inline int u_x0() const { return 1 - ep; }
    __host__ __device__ inline bool u_in(int F, int b) const { return F >= 1 - ep && F < N && b >= 0 && b < M; }
    __host__ __device__ inline bool v_in(int a, int G) const { return a >= 0 && a < N && G >= 1 && G < M; }
    __host__ __device__ inline bool e_in(int a, int b) const { return a >= 0 && a < N && b >= 0 && b < M; }
};

// A static field (f_q, Fx, Fy, H, ...) with strides that are 0 along the
// axes on which it is constant, so structured inputs are broadcast reads.
template <class T>
struct SField {
    const T* p;
    int sx, sy;    // element strides along x and y
    __device__ __forceinline__ T at(int x, int y) const { return p[(y + ROW0) * sy + (x + COL0) * sx]; }
};

// Julia's Float16 as a compute type: every +, -, *, / and sqrt is evaluated in
// Float32 and rounded once to binary16 (what Julia does for Float16 values);
// conversions from Float32 and Float64 round directly, ties to even.
struct jf16 {
    __half h;
    jf16() = default;
    __host__ __device__ explicit jf16(float x) : h(__float2half_rn(x)) {}
    __host__ __device__ explicit jf16(double x) : h(__double2half(x)) {}
    __host__ __device__ explicit jf16(int x) : h(__double2half((double)x)) {}
    __host__ __device__ explicit operator float() const { return __half2float(h); }
    __host__ __device__ explicit operator double() const { return (double)__half2float(h); }
    __host__ __device__ explicit operator int() const { return (int)__half2float(h); }
    // found by argument-dependent lookup only, so float and double calls are untouched
    friend __device__ inline jf16 sqrt(jf16 a) { return jf16(sqrtf(float(a))); }
    friend __device__ inline jf16 floor(jf16 a) { return jf16(floorf(float(a))); }
    friend __device__ inline jf16 fabs(jf16 a) { return jf16(fabsf(float(a))); }
};
static_assert(sizeof(jf16) == 2, "jf16 must have the layout of binary16");
__host__ __device__ inline jf16 operator+(jf16 a, jf16 b) { return jf16(float(a) + float(b)); }
__host__ __device__ inline jf16 operator-(jf16 a, jf16 b) { return jf16(float(a) - float(b)); }
__host__ __device__ inline jf16 operator*(jf16 a, jf16 b) { return jf16(float(a) * float(b)); }
__host__ __device__ inline jf16 operator/(jf16 a, jf16 b) { return jf16(float(a) / float(b)); }
__host__ __device__ inline jf16 operator-(jf16 a) { return jf16(-float(a)); }
__host__ __device__ inline jf16& operator+=(jf16& a, jf16 b) { return a = a + b; }
__host__ __device__ inline jf16& operator-=(jf16& a, jf16 b) { return a = a - b; }
__host__ __device__ inline jf16& operator*=(jf16& a, jf16 b) { return a = a * b; }
__host__ __device__ inline bool operator<(jf16 a, jf16 b) { return float(a) < float(b); }
__host__ __device__ inline bool operator>(jf16 a, jf16 b) { return float(a) > float(b); }
__host__ __device__ inline bool operator<=(jf16 a, jf16 b) { return float(a) <= float(b); }
__host__ __device__ inline bool operator>=(jf16 a, jf16 b) { return float(a) >= float(b); }
__host__ __device__ inline bool operator==(jf16 a, jf16 b) { return float(a) == float(b); }
__host__ __device__ inline bool operator!=(jf16 a, jf16 b) { return float(a) != float(b); }

// number conversion (Julia's T(x))
template <class To, class From>
__host__ __device__ inline To cvt(From x) { return static_cast<To>(x); }
template <> __host__ __device__ inline float cvt<float, __half>(__half x) { return __half2float(x); }
template <> __host__ __device__ inline double cvt<double, __half>(__half x) { return (double)__half2float(x); }
template <> __host__ __device__ inline __half cvt<__half, float>(float x) { return __float2half_rn(x); }
template <> __host__ __device__ inline __half cvt<__half, double>(double x) { return __double2half(x); }
template <> __host__ __device__ inline __half cvt<__half, __half>(__half x) { return x; }

// T(Tcomm(x)) for the periodic ghost copies (src/ghost_points.jl:65-68)
template <class T>
__device__ inline T via_comm(int Tcomm, T x) {
    if (Tcomm == SW_FLOAT16) return cvt<T>(__half2float(__double2half((double)cvt<double>(x))));
    if (Tcomm == SW_FLOAT32) return cvt<T>((float)cvt<double>(x));
    return x;
}

// Identifier of the calling thread's current CUDA context (cuCtxGetId), or 0
// if there is none or it cannot be read.  Host-side caches of device
// addresses are keyed by it, so a context that is destroyed and created again
// (cudaDeviceReset, or the primary context released and retained) never
// receives addresses that belonged to the old one.
inline unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static const GetCurrent get_current = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        return (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
                q == cudaDriverEntryPointSuccess) ? reinterpret_cast<GetCurrent>(p) : (GetCurrent) nullptr;
    }();
    static const GetId get_id = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        return (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
                q == cudaDriverEntryPointSuccess) ? reinterpret_cast<GetId>(p) : (GetId) nullptr;
    }();
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device status shared by all kernels of a context.
struct DevStatus {
    int stop;             // set once a NaN check fails: later kernels return at once
    int error;            // sw_error of a kernel-detected failure (e.g. departure)
    long long nan_step;   // step of the failed NaN check
    unsigned long long nan_count;
    long long step;       // completed steps (advanced by the last kernel of a step)
};

}  // namespace swb
