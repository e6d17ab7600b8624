// sw_tracer.cuh -- semi-Lagrangian tracer advection and small helper kernels.
//
// tracer_kernel does, per T-cell, what tracer! does per array
// (src/tracer_advection.jl:1-275): departure! (Ix!/Iy! to the T-grid,
// backtraj! at half step, interp_uv! of the mid-point velocity with clip/wrap
// and bilin, backtraj! at full step), adv_sst!, tracer_consumption! and
// ghost_points_sst!, writing the new tracer out of place.  Index arithmetic
// is kept in the reference's 1-based Julia indices and mapped to device
// storage at the loads:
//   um[k,l]  -> (F = k-2-ep, b = l-3)   vm[k,l] -> (a = k-3, G = l-2)
//   sst[k,l] -> (a = k-2,   b = l-1)
// A departure index the reference could not take (Int(floor(NaN)), or a
// wrapped index outside the array, which throws in Julia) sets
// DevStatus.error = SW_ERR_DEPARTURE and the access is clamped.
#pragma once
#include "sw_common.cuh"
#include "sw_ghost.cuh"

namespace swb {

template <class T, class Tp>
struct TracerArgs {
    Geom g;
    const Tp* u; const Tp* v;       // u0, v0 after the tail (converted to T on load)
    const T* um; const T* vm;       // mid-point velocities (T); may alias u, v (see um_is_u)
    const Tp* sst; Tp* sst_o;
    T dtadvu, dtadvv, half_dtadvu, half_dtadvv;
    T jSST, SSTmin;
    GhostRule<Tp> gr;
    DevStatus* st;
};

// Julia's Int(floor(x)); NaN, Inf and indices no array can take are flagged.
// Within the range the conversion rounds toward -inf in one instruction.
__device__ __forceinline__ int floor_to_int(float x) { return __float2int_rd(x); }
__device__ __forceinline__ int floor_to_int(double x) { return __double2int_rd(x); }
__device__ __forceinline__ int floor_to_int(jf16 x) { return (int)floorf(float(x)); }
template <class T>
__device__ __forceinline__ int ifloor(T x, int& bad) {
    if (!(fabs(x) < T(1.0e9))) { bad = 1; return 0; }
    return floor_to_int(x);
}

// bilin (src/tracer_advection.jl:243-246)
template <class T>
__device__ __forceinline__ T bilin(T f00, T f10, T f01, T f11, T x, T y) {
    const T one = T(1);
    return f00 * (one - x) * (one - y) + f10 * x * (one - y) + f01 * (one - x) * y + f11 * x * y;
}

// Lower-left index and relative coordinate along one axis.  clip and wrap
// (src/tracer_advection.jl:211-240) written for an offset k0 = xi + i (the
// departure cell relative to the arrival cell i): the reference's index is
// in range for k0 in [lo, hi]; clip pins to lo/hi with coordinate 0/1, wrap
// shifts by n (one period) and keeps xy - xi.
template <class T, bool WRAP>
__device__ __forceinline__ int axis(int k0, int xi, T xy, int lo, int hi, int n, T& x0) {
    if (WRAP) {
        x0 = xy - (T)xi;
        if (k0 < lo) return k0 + n;
        if (k0 > hi) return k0 - n;
        return k0;
    } else {
        if (k0 < lo) { x0 = T(0); return lo; }
        if (k0 > hi) { x0 = T(1); return hi; }
        x0 = xy - (T)xi;
        return k0;
    }
}

// How the tracer reads u, v and sst and writes sst.  TracerIONative: arrays of
// Tprog.  The 16-bit storage form reads and writes scaled 16-bit numbers
// (sw_s16.cuh); its pointers travel in TracerArgs as Tprog pointers.
template <class T, class Tp>
struct TracerIONative {
    using EU = Tp;                       // element type of u, v
    using ES = Tp;                       // element type of sst
    __device__ __forceinline__ T u(EU x) const { return cvt<T>(x); }
    __device__ __forceinline__ T s(ES x) const { return cvt<T>(x); }
    __device__ __forceinline__ ES operator()(Tp x) const { return x; }   // Tprog value -> sst element
};

// 2-D launch: x over columns, y over rows (grid-stride in y)
// The tracer for column block bx and rows by, by + gy, ... (128 threads).
template <class T, class Tp, bool PER, bool UM_IS_U, bool CONS, class IO = TracerIONative<T, Tp>>
__device__ __forceinline__ void tracer_body(const TracerArgs<T, Tp>& A, int bx, int by, int gy, const IO& io = IO()) {
    using EU = typename IO::EU;
    using ES = typename IO::ES;
    if (A.st->stop) return;
    const Geom& g = A.g;
    const int N = g.N, M = g.M;
    const int a = bx * 128 + threadIdx.x;
    if (a >= N) return;
    const T half = T(0.5);
    int bad = 0;
    const int P = g.P;
    const bool gx = a == 0 || a == N - 1;
    // element (x, y) of a field sits at (y + ROW0) * P + x + COL0
    auto at = [&](int x, int y) { return (y + ROW0) * P + x + COL0; };
    // the output never aliases the inputs: loads of later rows may be issued early
    const EU* __restrict__ pu = reinterpret_cast<const EU*>(A.u);
    const EU* __restrict__ pv = reinterpret_cast<const EU*>(A.v);
    const T* __restrict__ pum = A.um;
    const T* __restrict__ pvm = A.vm;
    const ES* __restrict__ psst = reinterpret_cast<const ES*>(A.sst);
    ES* __restrict__ psst_o = reinterpret_cast<ES*>(A.sst_o);
    for (int b = by; b < M; b += gy) {
        // departure!: u_T = Ix!(u), v_T = Iy!(v); backtraj! at half step (:75-76, :96-124)
        const int o = at(a, b);
        const T uT = half * (io.u(pu[o + 1]) + io.u(pu[o]));
        const T vT = half * (io.u(pv[o + P]) + io.u(pv[o]));
        T xd = (-A.half_dtadvu) * uT;
        T yd = (-A.half_dtadvv) * vT;
        int xi = ifloor(xd, bad), yi = ifloor(yd, bad);
        T ui, vi;
        {   // interp_uv!(uinterp, um_T, ...): um_T at T-cell F0 is ½(um(F0+1) + um(F0)) (:130-176)
            T x0, y0;
            int F0 = axis<T, PER>(xi + a, xi, xd, 0, N - 1, N, x0);
            const int b0 = axis<T, false>(yi + b, yi, yd, 0, M, 0, y0);
            if (F0 < -2 || F0 > N - 1) { bad = 1; F0 = 0; }
            const int k = at(F0, b0);
            T m00, m10, m20, m01, m11, m21;
            if (UM_IS_U) {
                m00 = io.u(pu[k]); m10 = io.u(pu[k + 1]); m20 = io.u(pu[k + 2]);
                m01 = io.u(pu[k + P]); m11 = io.u(pu[k + P + 1]); m21 = io.u(pu[k + P + 2]);
            } else {
                m00 = pum[k]; m10 = pum[k + 1]; m20 = pum[k + 2];
                m01 = pum[k + P]; m11 = pum[k + P + 1]; m21 = pum[k + P + 2];
            }
            ui = bilin(half * (m10 + m00), half * (m20 + m10), half * (m11 + m01), half * (m21 + m11), x0, y0);
        }
        {   // interp_uv!(vinterp, vm_T, ...): vm_T at T-row G0 is ½(vm(G0+1) + vm(G0))
            T x0, y0;
            int a0 = axis<T, PER>(xi + a, xi, xd, 0, N, N, x0);
            const int G0 = axis<T, false>(yi + b, yi, yd, 0, M - 1, 0, y0);
            if (a0 < -2 || a0 > N) { bad = 1; a0 = 0; }
            const int k = at(a0, G0);
            T m00, m01, m02, m10, m11, m12;
            if (UM_IS_U) {
                m00 = io.u(pv[k]); m01 = io.u(pv[k + P]); m02 = io.u(pv[k + 2 * P]);
                m10 = io.u(pv[k + 1]); m11 = io.u(pv[k + P + 1]); m12 = io.u(pv[k + 2 * P + 1]);
            } else {
                m00 = pvm[k]; m01 = pvm[k + P]; m02 = pvm[k + 2 * P];
                m10 = pvm[k + 1]; m11 = pvm[k + P + 1]; m12 = pvm[k + 2 * P + 1];
            }
            vi = bilin(half * (m01 + m00), half * (m11 + m10), half * (m02 + m01), half * (m12 + m11), x0, y0);
        }
        // backtraj! at full step (:83-84)
        xd = (-A.dtadvu) * ui;
        yd = (-A.dtadvv) * vi;
        xi = ifloor(xd, bad);
        yi = ifloor(yd, bad);
        T s;
        {   // adv_sst! (:179-206)
            T x0, y0;
            int a0 = axis<T, PER>(xi + a, xi, xd, 0, N - 1, N, x0);
            const int b0 = axis<T, false>(yi + b, yi, yd, 0, M - 2, 0, y0);
            if (a0 < -1 || a0 > N - 1) { bad = 1; a0 = 0; }
            const int k = at(a0, b0);
            s = bilin(io.s(psst[k]), io.s(psst[k + 1]), io.s(psst[k + P]), io.s(psst[k + P + 1]), x0, y0);
        }
        if (CONS) s += A.jSST * (A.SSTmin - s);              // tracer_consumption! (:262-275)
        const Tp out = cvt<Tp>(s);
        psst_o[o] = io(out);
        if (gx) A.gr.sst(psst_o, g, a, b, out, io);             // ghost_points_sst! (:40)
    }
    if (bad) {   // the reference throws here; halt the device-side loop
        atomicCAS(&A.st->error, 0, (int)SW_ERR_DEPARTURE);
        atomicExch(&A.st->stop, 1);
    }
}

template <class T, class Tp, bool PER, bool UM_IS_U, bool CONS>
__global__ void __launch_bounds__(128)
tracer_kernel(const __grid_constant__ TracerArgs<T, Tp> A) {
    tracer_body<T, Tp, PER, UM_IS_U, CONS>(A, (int)blockIdx.x, (int)blockIdx.y, (int)gridDim.y);
}

// um, vm = u0, v0 converted to T (src/tracer_advection.jl:12-17), over whole buffers
template <class T, class Tp>
__global__ void copy_convert_kernel(const Tp* __restrict__ u, const Tp* __restrict__ v, T* __restrict__ um,
                                    T* __restrict__ vm, long long n, const DevStatus* st) {
    if (st->stop) return;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        um[k] = cvt<T>(u[k]);
        vm[k] = cvt<T>(v[k]);
    }
}

// nan_detection! (src/feedback.jl:61-72) over the reference's array extents of
// u, v, eta (state before the step) and sst (after it); on NaNs it stops the
// run like `break` in src/time_integration.jl:235-237.
template <class Tp>
__device__ inline bool is_nan_(Tp x) { return isnan((double)x); }

template <class Tp>
__global__ void nan_check_kernel(Geom g, const Tp* u, const Tp* v, const Tp* e, const Tp* sst, long long step,
                                 DevStatus* st) {
    if (st->stop) return;
    const int N = g.N, M = g.M, ep = g.ep;
    const int uw = (ep ? N : N - 1) + 4;
    // extents as (x range, y range, base x, base y)
    struct Ext { int w, h, x0, y0; const Tp* p; };
    Ext ex[4] = {{uw, M + 4, ep ? -2 : -1, -2, u}, {N + 4, M + 3, -2, -1, v}, {N + 2, M + 2, -1, -1, e},
                 {N + 2, M, -1, 0, sst}};
    unsigned long long cnt = 0;
    for (int f = 0; f < 4; f++) {
        long long tot = (long long)ex[f].w * ex[f].h;
        for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < tot; k += (long long)gridDim.x * blockDim.x) {
            int x = ex[f].x0 + (int)(k % ex[f].w), y = ex[f].y0 + (int)(k / ex[f].w);
            cnt += is_nan_(ex[f].p[g.idx(x, y)]) ? 1 : 0;
        }
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) {
        atomicAdd(&st->nan_count, cnt);
        atomicCAS(&st->stop, 0, 1);
        // every block that saw NaNs writes the same step
        st->nan_step = step;
    }
}

}  // namespace swb
