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
    int um_is_u;                    // nadvstep == 1: um, vm are u, v of this step
    const Tp* sst; Tp* sst_o;
    T dtadvu, dtadvv, half_dtadvu, half_dtadvv;
    int consumption;
    T jSST, SSTmin;
    GhostRule<Tp> gr;
    DevStatus* st;
};

struct Clip { long long k; };

template <class T>
__device__ inline long long jfloor(T x, int& bad) {
    double d = (double)x;
    if (!(fabs(d) < 9.2e18)) { bad = 1; return 0; }
    return (long long)floor(d);
}

// clip (src/tracer_advection.jl:211-223) and wrap (:227-240)
template <class T>
__device__ inline long long clip_idx(long long xyi, long long ij, T xy, long long mn, long long h1, T& x0) {
    long long xyis = xyi + ij + h1;
    if (xyis < 1 + h1) { x0 = T(0); return 1 + h1; }
    if (xyis > mn - 1) { x0 = T(1); return mn - 1; }
    x0 = xy - (T)(double)xyi;
    return xyis;
}
template <class T>
__device__ inline long long wrap_idx(long long xyi, long long ij, T xy, long long mn, long long h1, long long h2, T& x0) {
    long long xyis = xyi + ij + h1;
    x0 = xy - (T)(double)xyi;
    if (xyis < 1 + h1) return xyis + mn - h1 - h2;
    if (xyis > mn - 1) return xyis - mn + h1 + h2;
    return xyis;
}
// bilin (src/tracer_advection.jl:243-246)
template <class T>
__device__ inline T bilin(T f00, T f10, T f01, T f11, T x, T y) {
    const T one = T(1);
    return f00 * (one - x) * (one - y) + f10 * x * (one - y) + f01 * (one - x) * y + f11 * x * y;
}

template <class T, class Tp>
__global__ void tracer_kernel(TracerArgs<T, Tp> A) {
    if (A.st->stop) return;
    const Geom& g = A.g;
    const int N = g.N, M = g.M, ep = g.ep;
    const int nux = ep ? N : N - 1;
    int bad = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)N * M;
         t += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(t % N), b = (int)(t / N);
        const long long i = a + 1, j = b + 1;            // Julia indices of xd[i,j]
        const T half = T(0.5);
        auto U = [&](int F, int bb) { return cvt<T>(A.u[g.idx(F, bb)]); };
        auto V = [&](int aa, int G) { return cvt<T>(A.v[g.idx(aa, G)]); };
        auto UM = [&](int F, int bb) { return A.um_is_u ? cvt<T>(A.u[g.idx(F, bb)]) : A.um[g.idx(F, bb)]; };
        auto VM = [&](int aa, int G) { return A.um_is_u ? cvt<T>(A.v[g.idx(aa, G)]) : A.vm[g.idx(aa, G)]; };

        // u_T = Ix!(u), v_T = Iy!(v) at the T-cell; backtraj! at half step (:75-76, :96-124)
        T uT = half * (U(a + 1, b) + U(a, b));
        T vT = half * (V(a, b + 1) + V(a, b));
        T xd = (-A.half_dtadvu) * uT;
        T yd = (-A.half_dtadvv) * vT;

        // interp_uv!(uinterp, um_T, xd, yd): u case, muv = nux+3, nuv = M+4 (:130-176)
        T ui, vi;
        {
            long long xi = jfloor(xd, bad), yi = jfloor(yd, bad);
            T x0, y0;
            long long muv = nux + 3, nuv = M + 4;
            long long k = ep ? wrap_idx(xi, i, xd, muv, 1 + ep, 1, x0) : clip_idx(xi, i, xd, muv, 1 + ep, x0);
            long long l = clip_idx(yi, j, yd, nuv, 2, y0);
            if (k < 1 || k + 1 > muv || l < 1 || l + 1 > nuv) { bad = 1; k = min(max(k, 1LL), muv - 1); l = min(max(l, 1LL), nuv - 1); }
            // um_T[k,l] = 0.5*(um[k+1,l] + um[k,l]), um[k,l] at (F = k-2-ep, b = l-3)
            auto umT = [&](long long kk, long long ll) {
                int F = (int)kk - 2 - ep, bb = (int)ll - 3;
                return half * (UM(F + 1, bb) + UM(F, bb));
            };
            ui = bilin(umT(k, l), umT(k + 1, l), umT(k, l + 1), umT(k + 1, l + 1), x0, y0);
        }
        {
            long long xi = jfloor(xd, bad), yi = jfloor(yd, bad);
            T x0, y0;
            long long muv = N + 4, nuv = M + 2;
            long long k = ep ? wrap_idx(xi, i, xd, muv, 2, 2, x0) : clip_idx(xi, i, xd, muv, 2, x0);
            long long l = clip_idx(yi, j, yd, nuv, 1, y0);
            if (k < 1 || k + 1 > muv || l < 1 || l + 1 > nuv) { bad = 1; k = min(max(k, 1LL), muv - 1); l = min(max(l, 1LL), nuv - 1); }
            // vm_T[k,l] = 0.5*(vm[k,l+1] + vm[k,l]), vm[k,l] at (a = k-3, G = l-2)
            auto vmT = [&](long long kk, long long ll) {
                int aa = (int)kk - 3, G = (int)ll - 2;
                return half * (VM(aa, G + 1) + VM(aa, G));
            };
            vi = bilin(vmT(k, l), vmT(k + 1, l), vmT(k, l + 1), vmT(k + 1, l + 1), x0, y0);
        }
        // backtraj! at full step (:83-84)
        xd = (-A.dtadvu) * ui;
        yd = (-A.dtadvv) * vi;

        // adv_sst! (:179-206): m = N+2, n = M, halo 1 in x, 0 in y
        T s;
        {
            long long xi = jfloor(xd, bad), yi = jfloor(yd, bad);
            T x0, y0;
            long long m = N + 2, n = M;
            long long k = ep ? wrap_idx(xi, i, xd, m, 1, 1, x0) : clip_idx(xi, i, xd, m, 1, x0);
            long long l = clip_idx(yi, j, yd, n, 0, y0);
            if (k < 1 || k + 1 > m || l < 1 || l + 1 > n) { bad = 1; k = min(max(k, 1LL), m - 1); l = min(max(l, 1LL), n - 1); }
            auto S = [&](long long kk, long long ll) { return cvt<T>(A.sst[g.idx((int)kk - 2, (int)ll - 1)]); };
            s = bilin(S(k, l), S(k + 1, l), S(k, l + 1), S(k + 1, l + 1), x0, y0);
        }
        if (A.consumption) s += A.jSST * (A.SSTmin - s);   // tracer_consumption! (:262-275)
        Tp out = cvt<Tp>(s);
        A.sst_o[g.idx(a, b)] = out;
        A.gr.sst(A.sst_o, g, a, b, out);                   // ghost_points_sst! (:40)
    }
    if (bad) {   // the reference throws here; halt the device-side loop
        atomicCAS(&A.st->error, 0, (int)SW_ERR_DEPARTURE);
        atomicExch(&A.st->stop, 1);
    }
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
