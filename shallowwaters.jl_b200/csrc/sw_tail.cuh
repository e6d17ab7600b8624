// sw_tail.cuh -- the dissipative step tail, fused into one launch.
//
// From X0 = (u0, v0, eta0) after ghost_points! it computes
//   bottom_drag!               (src/bottom_drag.jl:2-119: quadratic/linear/none)
//   diffusion!                 (src/diffusion.jl:2-218: Smagorinsky or constant,
//                               biharmonic ∇·ν∇∇²u)
//   add_drag_diff_tendencies!  (src/diffusion.jl:221-251)
//   ghost_points_uv!           (src/ghost_points.jl:202-216)
// writing u, v out of place.  Intermediates follow the reference's arrays and
// operation order; positions in T-cell/face coordinates:
//   Lu(F,b) = ∇²u at u-points, Lv(a,G) at v-points           (src/gradients.jl:29-42)
//   DSq(F,G) = (dudy + dvdx)² at corners; DT(a,b) = (dudx + dvdy)² at T-cells
//   ν(a,b) = cSmag·sqrt(Ixy(DSq) + DT); νq = Ixy(ν) at corners (src/diffusion.jl:68-111)
//   S11(a,b) = ν·∂xLu, S22(a,b) = ν·∂yLv, S12(F,G) = νq·∂yLu, S21(F,G) = νq·∂xLv
//   LLu1 = ∂xS11, LLu2 = ∂yS12, LLv1 = ∂xS21, LLv2 = ∂yS22
// Tile TX x TY with a 2-cell halo: device columns [x0, x0+TX+8), rows
// [y0, y0+TY+4), local (lx, ly) = (x - x0 + 4, y - y0 + 2).
#pragma once
#include "sw_common.cuh"
#include "sw_ghost.cuh"

namespace swb {

template <class T, class Tp>
struct TailArgs {
    Geom g;
    int ntx, nty;
    const Tp* u0; const Tp* v0; const Tp* e0;   // X0 after ghost points
    Tp* uo; Tp* vo;                             // new u, v
    SField<T> H;
    int drag;        // enum sw_bottom_drag
    int smag;        // 1 Smagorinsky, 0 constant
    T cD, rD, cSmag, nuB;
    Tp Dt_diff;
    GhostRule<Tp> gr;
    DevStatus* st;
};

template <class T, class Tp, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT)
tail_kernel(TailArgs<T, Tp> A) {
    if (A.st->stop) return;
    const Geom& g = A.g;
    const int ntiles = A.ntx * A.nty;

    // untouched halo cells keep u0 (and so do their ghost copies)
    if ((int)blockIdx.x >= ntiles) {
        const int nu = Ring::u_count(g.ep, g.N, g.M), nv = Ring::v_count(g.N);
        for (int k = ((int)blockIdx.x - ntiles) * NT + threadIdx.x; k < nu + nv;
             k += ((int)gridDim.x - ntiles) * NT) {
            if (k < nu) {
                int F, b;
                Ring::u_at(k, g.ep, g.N, g.M, F, b);
                Tp x = A.u0[g.idx(F, b)];
                A.uo[g.idx(F, b)] = x;
                A.gr.u(A.uo, g, F, b, x);
            } else {
                int a, G;
                Ring::v_at(k - nu, g.N, g.M, a, G);
                Tp x = A.v0[g.idx(a, G)];
                A.vo[g.idx(a, G)] = x;
                A.gr.v(A.vo, g, a, G, x);
            }
        }
        return;
    }

    constexpr int SW = TX + 8, SH = TY + 4, SZ = SW * SH;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* su = reinterpret_cast<T*>(smem_raw);
    T* sv = su + SZ;
    T* sh = sv + SZ;       // h = eta0 + H
    T* sLu = sh + SZ;
    T* sLv = sLu + SZ;
    T* sDSq = sLv + SZ;
    T* sNu = sDSq + SZ;    // DT, then ν in place
    T* sKE = sNu + SZ;     // sqrtKE
    T* sS11 = sKE + SZ;
    T* sS22 = sS11 + SZ;
    T* sS12 = sS22 + SZ;
    T* sS21 = sS12 + SZ;
#define S_(arr, lx, ly) arr[(ly) * SW + (lx)]

    const int x0 = ((int)blockIdx.x % A.ntx) * TX;
    const int y0 = ((int)blockIdx.x / A.ntx) * TY;
    const int tid = threadIdx.x;
    const T half = T(0.5), q4 = T(0.25);

    for (int k = tid; k < SZ; k += NT) {
        int ly = k / SW, lx = k - ly * SW;
        int row = y0 + ly, col = x0 + lx;
        T uu = T(0), vv = T(0), hh = T(0);
        if (row < g.R && col < g.P) {
            long gi = (long)row * g.P + col;
            uu = cvt<T>(A.u0[gi]);
            vv = cvt<T>(A.v0[gi]);
            if (A.drag == SW_DRAG_QUADRATIC) hh = cvt<T>(A.e0[gi]) + A.H.at(col - COL0, row - ROW0);
        }
        su[k] = uu; sv[k] = vv; sh[k] = hh;
    }
    __syncthreads();

    // Lu, Lv over lx in [3,TX+4], ly in [1,TY+2]; DT over the same T-cells;
    // DSq over corners lx in [3,TX+5], ly in [1,TY+3]; sqrtKE over lx in [3,TX+3], ly in [1,TY+1]
    {
        constexpr int W1 = TX + 2, H1 = TY + 2;
        for (int k = tid; k < W1 * H1; k += NT) {
            int ly = 1 + k / W1, lx = 3 + k % W1;
            T c = S_(su, lx, ly);
            S_(sLu, lx, ly) = ((S_(su, lx - 1, ly) - c) + (S_(su, lx + 1, ly) - c)) +
                              ((S_(su, lx, ly - 1) - c) + (S_(su, lx, ly + 1) - c));
            c = S_(sv, lx, ly);
            S_(sLv, lx, ly) = ((S_(sv, lx - 1, ly) - c) + (S_(sv, lx + 1, ly) - c)) +
                              ((S_(sv, lx, ly - 1) - c) + (S_(sv, lx, ly + 1) - c));
            if (A.smag) {
                T dudx = S_(su, lx + 1, ly) - S_(su, lx, ly);      // ∂x!(dudx, u) at T-cell
                T dvdy = S_(sv, lx, ly + 1) - S_(sv, lx, ly);      // ∂y!(dvdy, v) at T-cell
                T s = dudx + dvdy;
                S_(sNu, lx, ly) = s * s;                          // DT
            }
        }
        if (A.smag) {
            constexpr int W2 = TX + 3, H2 = TY + 3;
            for (int k = tid; k < W2 * H2; k += NT) {
                int ly = 1 + k / W2, lx = 3 + k % W2;
                T dudy = S_(su, lx, ly) - S_(su, lx, ly - 1);
                T dvdx = S_(sv, lx, ly) - S_(sv, lx - 1, ly);
                T s = dudy + dvdx;
                S_(sDSq, lx, ly) = s * s;                         // DS_q
            }
        }
        if (A.drag == SW_DRAG_QUADRATIC) {
            constexpr int W3 = TX + 1, H3 = TY + 1;
            for (int k = tid; k < W3 * H3; k += NT) {
                int ly = 1 + k / W3, lx = 3 + k % W3;
                T uR = S_(su, lx + 1, ly), uL = S_(su, lx, ly);
                T vT = S_(sv, lx, ly + 1), vB = S_(sv, lx, ly);
                T KEu = half * (uR * uR + uL * uL);
                T KEv = half * (vT * vT + vB * vB);
                S_(sKE, lx, ly) = sqrt(KEu + KEv);                // src/bottom_drag.jl:46-50
            }
        }
    }
    __syncthreads();

    // ν = cSmag·sqrt(DS + DT) with DS = Ixy(DS_q), over lx in [3,TX+4], ly in [1,TY+2]
    if (A.smag) {
        constexpr int W1 = TX + 2, H1 = TY + 2;
        for (int k = tid; k < W1 * H1; k += NT) {
            int ly = 1 + k / W1, lx = 3 + k % W1;
            T DS = q4 * (S_(sDSq, lx, ly) + S_(sDSq, lx + 1, ly)) + q4 * (S_(sDSq, lx, ly + 1) + S_(sDSq, lx + 1, ly + 1));
            S_(sNu, lx, ly) = A.cSmag * sqrt(DS + S_(sNu, lx, ly));
        }
        __syncthreads();
    }

    // S11(a,b): lx in [3,TX+3], ly in [2,TY+2);  S22(a,b): lx in [4,TX+4), ly in [1,TY+2)
    // S12(F,G): lx in [4,TX+4), ly in [2,TY+2];  S21(F,G): lx in [4,TX+4], ly in [2,TY+2)
    {
        constexpr int W = TX + 1, Hh = TY + 1;
        for (int k = tid; k < W * Hh; k += NT) {
            int ly = 1 + k / W, lx = 3 + k % W;       // lx in [3,TX+3], ly in [1,TY+1]
            // S11 at T-cell (lx, ly+1): ν(a,b)·(Lu(a+1,b) - Lu(a,b))
            {
                int l2 = ly + 1;
                T d = S_(sLu, lx + 1, l2) - S_(sLu, lx, l2);
                S_(sS11, lx, l2) = (A.smag ? S_(sNu, lx, l2) : A.nuB) * d;
            }
            // S22 at T-cell (lx+1, ly): ν(a,b)·(Lv(a,b+1) - Lv(a,b))
            if (lx < TX + 3) {
                int l1 = lx + 1;
                T d = S_(sLv, l1, ly + 1) - S_(sLv, l1, ly);
                S_(sS22, l1, ly) = (A.smag ? S_(sNu, l1, ly) : A.nuB) * d;
            }
            // corners (lx+1, ly+1): νq = Ixy(ν)
            int cx = lx + 1, cy = ly + 1;
            T nq = A.nuB;
            if (A.smag)
                nq = q4 * (S_(sNu, cx - 1, cy - 1) + S_(sNu, cx, cy - 1)) + q4 * (S_(sNu, cx - 1, cy) + S_(sNu, cx, cy));
            if (cx < TX + 4) S_(sS12, cx, cy) = nq * (S_(sLu, cx, cy) - S_(sLu, cx, cy - 1));
            if (cy < TY + 2) S_(sS21, cx, cy) = nq * (S_(sLv, cx, cy) - S_(sLv, cx - 1, cy));
        }
    }
    __syncthreads();

    for (int k = tid; k < TX * TY; k += NT) {
        int ly = 2 + k / TX, lx = 4 + k % TX;
        int x = x0 + lx - 4, y = y0 + ly - 2;
        if (g.u_in(x, y)) {
            T Bu;
            if (A.drag == SW_DRAG_QUADRATIC) {
                T ke = half * (S_(sKE, lx, ly) + S_(sKE, lx - 1, ly));      // sqrtKE_u = Ix!(sqrtKE)
                T hu = half * (S_(sh, lx, ly) + S_(sh, lx - 1, ly));        // h_u = Ix!(h)
                Bu = A.cD * ke * S_(su, lx, ly) / hu;                       // src/bottom_drag.jl:60-64
            } else if (A.drag == SW_DRAG_LINEAR) {
                Bu = A.rD * S_(su, lx, ly);
            } else {
                Bu = T(0);
            }
            T LLu1 = S_(sS11, lx, ly) - S_(sS11, lx - 1, ly);
            T LLu2 = S_(sS12, lx, ly + 1) - S_(sS12, lx, ly);
            long gi = g.idx(x, y);
            Tp nu_ = A.u0[gi] + A.Dt_diff * (cvt<Tp>(Bu) + cvt<Tp>(LLu1) + cvt<Tp>(LLu2));
            A.uo[gi] = nu_;
            A.gr.u(A.uo, g, x, y, nu_);
        }
        if (g.v_in(x, y)) {
            T Bv;
            if (A.drag == SW_DRAG_QUADRATIC) {
                T ke = half * (S_(sKE, lx, ly) + S_(sKE, lx, ly - 1));      // sqrtKE_v = Iy!(sqrtKE)
                T hv = half * (S_(sh, lx, ly) + S_(sh, lx, ly - 1));
                Bv = A.cD * ke * S_(sv, lx, ly) / hv;                       // src/bottom_drag.jl:71-75
            } else if (A.drag == SW_DRAG_LINEAR) {
                Bv = A.rD * S_(sv, lx, ly);
            } else {
                Bv = T(0);
            }
            T LLv1 = S_(sS21, lx + 1, ly) - S_(sS21, lx, ly);
            T LLv2 = S_(sS22, lx, ly) - S_(sS22, lx, ly - 1);
            long gi = g.idx(x, y);
            Tp nv_ = A.v0[gi] + A.Dt_diff * (cvt<Tp>(Bv) + cvt<Tp>(LLv1) + cvt<Tp>(LLv2));
            A.vo[gi] = nv_;
            A.gr.v(A.vo, g, x, y, nv_);
        }
    }
#undef S_
}

}  // namespace swb
