// sw_ghost.cuh -- ghost points fused into the kernels' write-back.
//
// ghost_points! (src/ghost_points.jl:46-241) fills halo cells from interior
// cells.  Here the thread that writes a source cell also writes every halo
// cell that the reference would copy from it, so no separate ghost pass is
// needed.  Halo cells the reference never writes ("untouched": the periodic
// y-halo of u and v, the nonperiodic x-halo of u) keep the value of the
// point-wise update with a zero tendency; they are written by "ring" threads.
#pragma once
#include "sw_common.cuh"

namespace swb {

template <class Tp>
struct GhostRule {
    int ep, N, M, Tcomm;
    Tp oma;   // one_minus_α (src/constants.jl:86)

    __device__ __forceinline__ Tp comm(Tp val) const {
        return (Tcomm == SW_FLOAT16 || (Tcomm == SW_FLOAT32 && sizeof(Tp) == 8)) ? via_comm(Tcomm, val) : val;
    }
    // Is (x, y) a source of a ghost copy?  Cheap tests for the hot loops.
    __device__ __forceinline__ bool u_src(int F, int b) const {
        return ep ? (F <= 1 || F >= N - 2) : (b <= 1 || b >= M - 2);
    }
    __device__ __forceinline__ bool v_src(int a) const { return a <= 1 || a >= N - 2; }
    __device__ __forceinline__ bool eta_src(int a, int b) const { return a == 0 || a == N - 1 || b == 0 || b == M - 1; }

    // u at (F, b) was set to val: write the halo cells copied from it.
    // periodic  u[1]=u[end-3], u[2]=u[end-2], u[end-1]=u[3], u[end]=u[4]  (:64-69)
    // nonperiodic u[:,1]=(1-α)u[:,4], u[:,2]=(1-α)u[:,3], u[:,end-1]=(1-α)u[:,end-2],
    //             u[:,end]=(1-α)u[:,end-3]                                 (:51-56)
    // Each rule has a form for arrays of another element type D: put(x)
    // converts the Tp value written there (the 16-bit storage form).
    template <class D, class Put>
    __device__ __forceinline__ void u(D* __restrict__ dst, const Geom& g, int F, int b, Tp val, Put put) const {
        if (ep) {
            Tp c = comm(val);
            if (F == 0 || F == 1) dst[g.idx(F + N, b)] = put(c);
            if (F == N - 2 || F == N - 1) dst[g.idx(F - N, b)] = put(c);
        } else {
            Tp c = oma * val;
            if (b == 0) dst[g.idx(F, -1)] = put(c);
            if (b == 1) dst[g.idx(F, -2)] = put(c);
            if (b == M - 1) dst[g.idx(F, M)] = put(c);
            if (b == M - 2) dst[g.idx(F, M + 1)] = put(c);
        }
    }
    __device__ __forceinline__ void u(Tp* __restrict__ dst, const Geom& g, int F, int b, Tp val) const {
        u(dst, g, F, b, val, Same{});
    }
    // v at (a, G): periodic x copies (:93-98); nonperiodic (1-α) mirror in x (:80-85)
    template <class D, class Put>
    __device__ __forceinline__ void v(D* __restrict__ dst, const Geom& g, int a, int G, Tp val, Put put) const {
        if (ep) {
            Tp c = comm(val);
            if (a == 0 || a == 1) dst[g.idx(a + N, G)] = put(c);
            if (a == N - 2 || a == N - 1) dst[g.idx(a - N, G)] = put(c);
        } else {
            Tp c = oma * val;
            if (a == 0) dst[g.idx(-1, G)] = put(c);
            if (a == 1) dst[g.idx(-2, G)] = put(c);
            if (a == N - 1) dst[g.idx(N, G)] = put(c);
            if (a == N - 2) dst[g.idx(N + 1, G)] = put(c);
        }
    }
    __device__ __forceinline__ void v(Tp* __restrict__ dst, const Geom& g, int a, int G, Tp val) const {
        v(dst, g, a, G, val, Same{});
    }
    // eta at (a, b): columns first, then rows over all columns, so the corners
    // take the column-copied value (src/ghost_points.jl:102-133)
    template <class D, class Put>
    __device__ __forceinline__ void eta(D* __restrict__ dst, const Geom& g, int a, int b, Tp val, Put put) const {
        // the (at most two) ghost columns copied from column a; NONE if there is none
        constexpr int NONE = -1000000;
        int xa = NONE, xb = NONE;
        Tp cx = ep ? comm(val) : val;
        if (ep) {
            if (a == N - 1) xa = -1;
            if (a == 0) xb = N;
        } else {
            if (a == 0) xa = -1;
            if (a == N - 1) xb = N;
        }
        if (xa != NONE) dst[g.idx(xa, b)] = put(cx);
        if (xb != NONE) dst[g.idx(xb, b)] = put(cx);
        if (b == 0 || b == M - 1) {
            int yt = (b == 0) ? -1 : M;
            dst[g.idx(a, yt)] = put(val);
            if (xa != NONE) dst[g.idx(xa, yt)] = put(cx);
            if (xb != NONE) dst[g.idx(xb, yt)] = put(cx);
            if (b == 0 && b == M - 1) {   // M == 1: both rows
                dst[g.idx(a, M)] = put(val);
                if (xa != NONE) dst[g.idx(xa, M)] = put(cx);
                if (xb != NONE) dst[g.idx(xb, M)] = put(cx);
            }
        }
    }
    __device__ __forceinline__ void eta(Tp* __restrict__ dst, const Geom& g, int a, int b, Tp val) const {
        eta(dst, g, a, b, val, Same{});
    }
    // sst at (a, b): periodic / zero-gradient copies in x (src/ghost_points.jl:136-179)
    template <class D, class Put>
    __device__ __forceinline__ void sst(D* __restrict__ dst, const Geom& g, int a, int b, Tp val, Put put) const {
        if (ep) {
            Tp c = comm(val);
            if (a == N - 1) dst[g.idx(-1, b)] = put(c);
            if (a == 0) dst[g.idx(N, b)] = put(c);
        } else {
            if (a == 0) dst[g.idx(-1, b)] = put(val);
            if (a == N - 1) dst[g.idx(N, b)] = put(val);
        }
    }
    __device__ __forceinline__ void sst(Tp* __restrict__ dst, const Geom& g, int a, int b, Tp val) const {
        sst(dst, g, a, b, val, Same{});
    }
    struct Same {
        __device__ __forceinline__ Tp operator()(Tp x) const { return x; }
    };
};

// The untouched halo cells of u and v, enumerated 0..count-1.
//   u periodic:    rows b in {-2,-1,M,M+1}, F in [0,N)
//   u nonperiodic: cols F in {-1,0,N,N+1}, b in [0,M)
//   v:             rows G in {-1,0,M,M+1}, a in [0,N)
struct Ring {
    __host__ __device__ static inline int u_count(int ep, int N, int M) { return ep ? 4 * N : 4 * M; }
    __host__ __device__ static inline int v_count(int N) { return 4 * N; }
    __device__ static inline void u_at(int k, int ep, int N, int M, int& F, int& b) {
        if (ep) {
            int r = k / N;
            F = k % N;
            b = (r == 0) ? -2 : (r == 1) ? -1 : (r == 2) ? M : M + 1;
        } else {
            int r = k / M;
            b = k % M;
            F = (r == 0) ? -1 : (r == 1) ? 0 : (r == 2) ? N : N + 1;
        }
    }
    __device__ static inline void v_at(int k, int N, int M, int& a, int& G) {
        int r = k / N;
        a = k % N;
        G = (r == 0) ? -1 : (r == 1) ? 0 : (r == 2) ? M : M + 1;
    }
};

}  // namespace swb
