// sw_linear.cuh -- linear dynamics (dynamics = "linear"): rhs_linear!
// (src/rhs.jl:59-86) with fv!/fu! (src/rhs.jl:183-215), momentum_u!/_v!
// (src/rhs.jl:218-274).
//
//   du(F, b) = (Tp(f_u*Ixy(v)) - Tp(dx(g*eta))) + Tp(Fxt*Fx)
//   dv(a, G) = -(Tp(f_v*Ixy(u)) + Tp(dy(g*eta))) + Tp(Fyt*Fy)
// with Ixy = 1/4 (a + b) + 1/4 (c + d) over the four neighbours
// (src/interpolations.jl:33-45) and g*eta rounded before it is differenced.
//
// rhs_linear! does not call UVfluxes!, and for time_scheme = "RK" neither does
// continuity! (src/continuity.jl:80-85): U and V keep the zeros they were
// allocated with, so deta is -(0 + 0) plus any relaxation/forcing term, and
// eta changes only through those terms.  The SSP schemes recompute U, V from
// the new u, v in continuity! and use ssp_continuity_kernel unchanged.
//
// These are point-wise kernels (one thread per T-cell, direct loads): linear
// dynamics is an option branch, not the measured configuration.
#pragma once
#include "sw_ssp.cuh"

namespace swb {

// du at the u-point (F, b) and dv at the v-point (a, G); inputs in Tprog, rhs in T
template <class T, class Tp>
struct LinearRhs {
    Geom g;
    const Tp* u; const Tp* v; const Tp* e;
    SField<T> fu, fv, Fx, Fy;
    T g_, Fxt, Fyt;

    __device__ T uat(int x, int y) const { return cvt<T>(u[g.idx(x, y)]); }
    __device__ T vat(int x, int y) const { return cvt<T>(v[g.idx(x, y)]); }
    __device__ T geta(int x, int y) const { return g_ * cvt<T>(e[g.idx(x, y)]); }

    __device__ Tp du(int F, int b) const {
        const T q4 = T(0.25);
        const T v_u = q4 * (vat(F - 1, b) + vat(F, b)) + q4 * (vat(F - 1, b + 1) + vat(F, b + 1));
        const T qhv = fu.at(F, b) * v_u;                                // fv! (src/rhs.jl:183-198)
        const T dpdx = geta(F, b) - geta(F - 1, b);
        return (cvt<Tp>(qhv) - cvt<Tp>(dpdx)) + cvt<Tp>(Fxt * Fx.at(F, b));
    }
    __device__ Tp dv(int a, int G) const {
        const T q4 = T(0.25);
        const T u_v = q4 * (uat(a, G - 1) + uat(a + 1, G - 1)) + q4 * (uat(a, G) + uat(a + 1, G));
        const T qhu = fv.at(a, G) * u_v;                                // fu! (src/rhs.jl:201-215)
        const T dpdy = geta(a, G) - geta(a, G - 1);
        return -(cvt<Tp>(qhu) + cvt<Tp>(dpdy)) + cvt<Tp>(Fyt * Fy.at(a, G));
    }
};

// One RK stage with linear dynamics: the update and ghost rules of
// rk_stage_kernel, one thread per T-cell; blocks past the cells do the ring.
template <class T, class Tp, bool PER, bool FIRST, bool LAST>
__global__ void __launch_bounds__(256)
lin_rk_stage_kernel(StageArgs<T, Tp> A, LinearRhs<T, Tp> L, int ncell_blocks) {
    if (A.st->stop) return;
    if ((int)blockIdx.x >= ncell_blocks) {
        stage_ring(A, FIRST, LAST, ((int)blockIdx.x - ncell_blocks) * 256 + threadIdx.x, A.nring_blocks * 256);
        return;
    }
    const Geom& g = A.g;
    const int N = g.N, M = g.M;
    const long long k = (long long)blockIdx.x * 256 + threadIdx.x;
    if (k >= (long long)N * M) return;
    const int c = (int)(k % N), r = (int)(k / N);
    const int o = g.idx(c, r);
    if (c >= (PER ? 0 : 1)) {
        const Tp du = L.du(c, r);
        const Tp X = A.uX[o];
        const bool gs = (PER && (c <= 1 || c >= N - 2)) || (!PER && (r <= 1 || r >= M - 2));
        if (!LAST) {
            const Tp x1 = X + A.b * du;
            A.u1o[o] = x1;
            if (gs) A.gr.u(A.u1o, g, c, r, x1);
        }
        const Tp x0 = (FIRST ? X : A.u0i[o]) + A.a * du;
        A.u0o[o] = x0;
        if (LAST && gs) A.gr.u(A.u0o, g, c, r, x0);
    }
    if (r >= 1) {
        const Tp dv = L.dv(c, r);
        const Tp X = A.vX[o];
        const bool gs = c <= 1 || c >= N - 2;
        if (!LAST) {
            const Tp x1 = X + A.b * dv;
            A.v1o[o] = x1;
            if (gs) A.gr.v(A.v1o, g, c, r, x1);
        }
        const Tp x0 = (FIRST ? X : A.v0i[o]) + A.a * dv;
        A.v0o[o] = x0;
        if (LAST && gs) A.gr.v(A.v0o, g, c, r, x0);
    }
    {
        // stale U = V = 0: dUdx = dVdy = 0 (src/continuity.jl:80-97)
        const T eta = cvt<T>(A.e1[o]);
        const Tp de = deta_of<T, Tp>(A.cont, T(0) - T(0), T(0) - T(0), eta, A.eref, A.Feta, A.gamma, A.Fetat, c, r);
        const Tp X = A.eX[o];
        const bool gs = c == 0 || c == N - 1 || r == 0 || r == M - 1;
        if (!LAST) {
            const Tp x1 = X + A.b * de;
            A.e1o[o] = x1;
            if (gs) A.gr.eta(A.e1o, g, c, r, x1);
        }
        const Tp x0 = (FIRST ? X : A.e0i[o]) + A.a * de;
        A.e0o[o] = x0;
        if (LAST && gs) A.gr.eta(A.e0o, g, c, r, x0);
    }
}

// The momentum half of an SSP stage with linear dynamics (the continuity half
// is ssp_continuity_kernel).
template <class T, class Tp, bool PER, int MODE, bool COMBO>
__global__ void __launch_bounds__(256)
lin_ssp_momentum_kernel(SspArgs<T, Tp> A, LinearRhs<T, Tp> L, int ncell_blocks) {
    if (A.st->stop) return;
    if ((int)blockIdx.x >= ncell_blocks) {
        ssp_ring<MODE, COMBO>(A, ((int)blockIdx.x - ncell_blocks) * 256 + threadIdx.x, A.nring_blocks * 256);
        return;
    }
    const Geom& g = A.g;
    const int N = g.N, M = g.M;
    const long long k = (long long)blockIdx.x * 256 + threadIdx.x;
    if (k >= (long long)N * M) return;
    const int c = (int)(k % N), r = (int)(k / N);
    const int o = g.idx(c, r);
    if (c >= (PER ? 0 : 1)) {
        const Tp du = L.du(c, r);
        const Tp z = (MODE == SSP_KN) ? A.uZ[o] : Tp(0);
        const Tp x1 = ssp_update<MODE>(A.k, A.u1[o], z, du);
        const bool gs = (PER && (c <= 1 || c >= N - 2)) || (!PER && (r <= 1 || r >= M - 2));
        A.u1o[o] = x1;
        if (gs) A.gr.u(A.u1o, g, c, r, x1);
        if (COMBO) {
            const Tp f = A.k.fa * A.uS[o] + A.k.fb * x1;
            A.ufo[o] = f;
            if (gs) A.gr.u(A.ufo, g, c, r, f);
        }
    }
    if (r >= 1) {
        const Tp dv = L.dv(c, r);
        const Tp z = (MODE == SSP_KN) ? A.vZ[o] : Tp(0);
        const Tp x1 = ssp_update<MODE>(A.k, A.v1[o], z, dv);
        const bool gs = c <= 1 || c >= N - 2;
        A.v1o[o] = x1;
        if (gs) A.gr.v(A.v1o, g, c, r, x1);
        if (COMBO) {
            const Tp f = A.k.fa * A.vS[o] + A.k.fb * x1;
            A.vfo[o] = f;
            if (gs) A.gr.v(A.vfo, g, c, r, f);
        }
    }
}

}  // namespace swb
