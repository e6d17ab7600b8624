// sw_advcor.cuh -- advection/Coriolis terms refreshed every nstep_advcor
// steps (nstep_advcor > 0 with nonlinear dynamics).
//
// With nstep_advcor > 0, rhs_nonlinear! skips advection_coriolis!
// (src/rhs.jl:30-35): the stages reuse q (and the Arakawa-Hsu or Sadourny
// combinations formed from it) and the kinetic energies KEu, KEv of the last
// refresh.  A refresh happens in the prologue of time_integration
// (src/time_integration.jl:20-36, from the initial state) and after the stages
// of every nstep_advcor-th step, from the new u0, v0, eta0
// (src/time_integration.jl:208-211).  bottom_drag_quadratic! recomputes KEu,
// KEv from u0 into the same arrays (src/bottom_drag.jl:38-48), so after a
// quadratic-drag tail the stages see that drag's KE: a KE-only refresh from u0
// reproduces it.
//
// Stored per point of the device layout (type T):
//   q(F, G)  PV at the corner, PV! (src/PV_advection.jl:2-18); for periodic
//            bcs column F = -1 holds q(N, G), the q[end] that AHβ!/AHγ! read
//            at i = 1 (src/PV_advection.jl:110,126), exactly what the stage
//            kernels' wrap lane computes;
//   KEu(a, b) = ½(u(a+1,b)² + u(a,b)²),  KEv(a, b) = ½(v(a,b+1)² + v(a,b)²).
// The stage kernels form the combinations from stored q with the same
// operations as from freshly computed q, so the results are those of the
// reference's stored qα..qδ / q_u, q_v.
#pragma once
#include "sw_stage.cuh"

namespace swb {

// One thread per point, x in [-2, N+2), y in [-1, M+1): every column and row
// the stage kernels read (their halo lanes included) lies inside.
template <class T, class Tp, bool PER, bool KE_ONLY>
__global__ void __launch_bounds__(256)
advcor_refresh_kernel(Geom g, const Tp* __restrict__ u, const Tp* __restrict__ v, const Tp* __restrict__ e,
                      SField<T> H, SField<T> fq, T* __restrict__ q, T* __restrict__ KEu, T* __restrict__ KEv) {
    const int x = (int)(blockIdx.x * blockDim.x + threadIdx.x) - 2;
    const int y = (int)blockIdx.y - 1;
    if (x >= g.N + 2) return;
    const T half = T(0.5);
    auto U = [&](int a, int b) { return cvt<T>(u[g.idx(a, b)]); };
    auto V = [&](int a, int b) { return cvt<T>(v[g.idx(a, b)]); };
    const int o = g.idx(x, y);
    // speed!, Ix!, Iy! (src/rhs.jl:142-159, src/interpolations.jl:3-30)
    {
        const T ur = U(x + 1, y), uc = U(x, y);
        const T vt = V(x, y + 1), vc = V(x, y);
        KEu[o] = half * (ur * ur + uc * uc);
        KEv[o] = half * (vt * vt + vc * vc);
    }
    if (KE_ONLY) return;
    const int c = (PER && x == -1) ? g.N : x;     // q[end] at the periodic wrap column
    auto h = [&](int a, int b) { return cvt<T>(e[g.idx(a, b)]) + H.at(a, b); };
    q[o] = pv_q<T>(fq.at(c, y), V(c, y), V(c - 1, y), U(c, y), U(c, y - 1), h(c - 1, y - 1), h(c, y - 1),
                   h(c - 1, y), h(c, y));
}

}  // namespace swb
