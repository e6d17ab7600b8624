// sw_stage.cuh -- one fused Runge-Kutta stage of the nonlinear model.
//
// One launch computes, for a stage input X1 = (u1, v1, eta1) whose ghost
// points are valid, the tendencies of
//   rhs_nonlinear!  (src/rhs.jl:24-51: UVfluxes!, advection_coriolis!, PV!,
//                    PV_ArakawaHsu!, bernoulli!, momentum_u!, momentum_v!)
//   continuity!     (src/continuity.jl:72-97, explicit form for "RK")
// and applies the stage combination of src/time_integration.jl:55-78,
//   X1' = X + b*d  (caxb!),  X0 += a*d  (axb!)
// including ghost_points! on X1' (and on X0 after the last stage).
// Every intermediate is formed at the reference's index with the reference's
// operation order, so results are bit-identical to the Julia arrays when
// built without FMA contraction (--fmad=false).
//
// Tile: TX x TY T-cells at (x0, y0).  The block stages u, v, eta and
// h = eta + H over device columns [x0, x0+TX+8) and rows [y0, y0+TY+3) in
// shared memory, i.e. local (lx, ly) = (x - x0 + 4, y - y0 + 2):
//   q(F,G)  at lx in [3,TX+4], ly in [1,TY+2]   (PV! on the q-grid)
//   p(a,b)  at lx in [3,TX+3], ly in [1,TY+1]   (bernoulli!)
//   U(F,b)  at lx in [4,TX+4], ly in [1,TY+1]   (Uflux!)
//   V(a,G)  at lx in [3,TX+3], ly in [2,TY+2]   (Vflux!)
// then du, dv, deta for the TX x TY outputs.
#pragma once
#include "sw_common.cuh"
#include "sw_ghost.cuh"

namespace swb {

template <class T, class Tp>
struct StageArgs {
    Geom g;
    int ntx, nty;                       // interior tiles; blocks beyond do the ring
    const Tp* u1; const Tp* v1; const Tp* e1;    // stage input (ghosts valid)
    const Tp* uX; const Tp* vX; const Tp* eX;    // step-start state X
    const Tp* u0i; const Tp* v0i; const Tp* e0i; // accumulator in (unused on the first stage)
    Tp* u1o; Tp* v1o; Tp* e1o;                   // X1' (nullptr on the last stage)
    Tp* u0o; Tp* v0o; Tp* e0o;                   // accumulator out
    SField<T> H, fq, Fx, Fy;
    Tp a, b;                            // RKaΔt[k], RKbΔt[k] (Tprog)
    T g_;                               // gravity (T)
    T Fxt, Fyt;                         // seasonal factors (1 if off)
    GhostRule<Tp> gr;
    int first, last;
    DevStatus* st;
};

template <class T>
struct StageSmem {
    static constexpr int NARR = 8;
};

// q at the corner (F, G) from values: PV! (src/PV_advection.jl:2-18) with
// h_q = Ixy!(h) (src/interpolations.jl:33-45), dvdx = ∂x!(v), dudy = ∂y!(u)
template <class T>
__device__ inline T pv_q(T fq, T vR, T vL, T uT, T uB, T hLB, T hRB, T hLT, T hRT) {
    const T q4 = T(0.25);
    T hq = q4 * (hLB + hRB) + q4 * (hLT + hRT);
    T dvdx = vR - vL;
    T dudy = uT - uB;
    return (fq + dvdx - dudy) / hq;
}

template <class T, class Tp, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT)
rk_stage_kernel(StageArgs<T, Tp> A) {
    if (A.st->stop) return;
    const Geom& g = A.g;
    const int ntiles = A.ntx * A.nty;

    // ---------------------------------------------------------------- ring
    if ((int)blockIdx.x >= ntiles) {
        const int nu = Ring::u_count(g.ep, g.N, g.M), nv = Ring::v_count(g.N);
        for (int k = ((int)blockIdx.x - ntiles) * NT + threadIdx.x; k < nu + nv;
             k += ((int)gridDim.x - ntiles) * NT) {
            const Tp zero = Tp(0);
            if (k < nu) {
                int F, b;
                Ring::u_at(k, g.ep, g.N, g.M, F, b);
                long gi = g.idx(F, b);
                Tp x = A.uX[gi];
                if (!A.last) {
                    Tp v1 = x + A.b * zero;
                    A.u1o[gi] = v1;
                    A.gr.u(A.u1o, g, F, b, v1);
                }
                Tp x0 = (A.first ? x : A.u0i[gi]) + A.a * zero;
                A.u0o[gi] = x0;
                if (A.last) A.gr.u(A.u0o, g, F, b, x0);
            } else {
                int a, G;
                Ring::v_at(k - nu, g.N, g.M, a, G);
                long gi = g.idx(a, G);
                Tp x = A.vX[gi];
                if (!A.last) {
                    Tp v1 = x + A.b * zero;
                    A.v1o[gi] = v1;
                    A.gr.v(A.v1o, g, a, G, v1);
                }
                Tp x0 = (A.first ? x : A.v0i[gi]) + A.a * zero;
                A.v0o[gi] = x0;
                if (A.last) A.gr.v(A.v0o, g, a, G, x0);
            }
        }
        return;
    }

    constexpr int SW = TX + 8, SH = TY + 3, SZ = SW * SH;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* su = reinterpret_cast<T*>(smem_raw);
    T* sv = su + SZ;
    T* se = sv + SZ;
    T* sh = se + SZ;
    T* sq = sh + SZ;
    T* sp = sq + SZ;
    T* sU = sp + SZ;
    T* sV = sU + SZ;
#define S_(arr, lx, ly) arr[(ly) * SW + (lx)]

    const int x0 = ((int)blockIdx.x % A.ntx) * TX;
    const int y0 = ((int)blockIdx.x / A.ntx) * TY;
    const int tid = threadIdx.x;

    // ---------------------------------------------- load X1 and h = eta + H
    for (int k = tid; k < SZ; k += NT) {
        int ly = k / SW, lx = k - ly * SW;
        int row = y0 + ly, col = x0 + lx;
        T uu = T(0), vv = T(0), ee = T(0), hh = T(0);
        if (row < g.R && col < g.P) {
            long gi = (long)row * g.P + col;
            uu = cvt<T>(A.u1[gi]);
            vv = cvt<T>(A.v1[gi]);
            ee = cvt<T>(A.e1[gi]);
            hh = ee + A.H.at(col - COL0, row - ROW0);       // thickness! (src/rhs.jl:131-139)
        }
        su[k] = uu; sv[k] = vv; se[k] = ee; sh[k] = hh;
    }
    __syncthreads();

    // ---------------------------------------------------- q, p, U, V
    {
        const T half = T(0.5);
        // q over lx in [3,TX+4], ly in [1,TY+2]
        constexpr int QW = TX + 2, QH = TY + 2;
        for (int k = tid; k < QW * QH; k += NT) {
            int ly = 1 + k / QW, lx = 3 + k % QW;
            int F = x0 + lx - 4, G = y0 + ly - 2;
            T qv;
            if (g.ep && F == -1) {
                // AHβ!/AHγ! wrap onto q[end] = q at F = N (src/PV_advection.jl:110,126):
                // evaluate that column from global memory
                int FN = g.N;
                auto U1 = [&](int x, int y) { return cvt<T>(A.u1[g.idx(x, y)]); };
                auto V1 = [&](int x, int y) { return cvt<T>(A.v1[g.idx(x, y)]); };
                auto H1 = [&](int x, int y) { return cvt<T>(A.e1[g.idx(x, y)]) + A.H.at(x, y); };
                qv = (G >= -1 && G <= g.M + 1)
                         ? pv_q<T>(A.fq.at(FN, G), V1(FN, G), V1(FN - 1, G), U1(FN, G), U1(FN, G - 1),
                                   H1(FN - 1, G - 1), H1(FN, G - 1), H1(FN - 1, G), H1(FN, G))
                         : T(0);
            } else {
                qv = pv_q<T>(A.fq.at(F, G), S_(sv, lx, ly), S_(sv, lx - 1, ly), S_(su, lx, ly), S_(su, lx, ly - 1),
                             S_(sh, lx - 1, ly - 1), S_(sh, lx, ly - 1), S_(sh, lx - 1, ly), S_(sh, lx, ly));
            }
            S_(sq, lx, ly) = qv;
        }
        // p over lx in [3,TX+3], ly in [1,TY+1]: bernoulli! (src/rhs.jl:162-180)
        constexpr int PW = TX + 1, PH = TY + 1;
        for (int k = tid; k < PW * PH; k += NT) {
            int ly = 1 + k / PW, lx = 3 + k % PW;
            T uR = S_(su, lx + 1, ly), uL = S_(su, lx, ly);
            T vT = S_(sv, lx, ly + 1), vB = S_(sv, lx, ly);
            T KEu = half * (uR * uR + uL * uL);     // Ix!(KEu, u²)
            T KEv = half * (vT * vT + vB * vB);     // Iy!(KEv, v²)
            S_(sp, lx, ly) = half * (KEu + KEv) + A.g_ * S_(se, lx, ly);
        }
        // U over lx in [4,TX+4], ly in [1,TY+1]: Uflux! with h_u = Ix!(h)
        for (int k = tid; k < PW * PH; k += NT) {
            int ly = 1 + k / PW, lx = 4 + k % PW;
            T hu = half * (S_(sh, lx, ly) + S_(sh, lx - 1, ly));
            S_(sU, lx, ly) = S_(su, lx, ly) * hu;
        }
        // V over lx in [3,TX+3], ly in [2,TY+2]: Vflux! with h_v = Iy!(h)
        for (int k = tid; k < PW * PH; k += NT) {
            int ly = 2 + k / PW, lx = 3 + k % PW;
            T hv = half * (S_(sh, lx, ly) + S_(sh, lx, ly - 1));
            S_(sV, lx, ly) = S_(sv, lx, ly) * hv;
        }
    }
    __syncthreads();

    // ------------------------------------------------ tendencies and RK update
    const T o12 = T(1.0 / 12.0);
    for (int k = tid; k < TX * TY; k += NT) {
        int ly = 2 + k / TX, lx = 4 + k % TX;
        int x = x0 + lx - 4, y = y0 + ly - 2;

        if (g.u_in(x, y)) {
            // Arakawa-Hsu combinations at the u-point (F=x, b=y) (src/PV_advection.jl:63-146)
            T q00 = S_(sq, lx, ly), q01 = S_(sq, lx, ly + 1);
            T qa = o12 * (q00 + q01 + S_(sq, lx + 1, ly + 1));
            T qb = o12 * (q00 + q01 + S_(sq, lx - 1, ly + 1));
            T qc = (x == 0) ? o12 * (q00 + q01 + S_(sq, lx - 1, ly))      // γ[1,j] order (:126)
                            : o12 * (q00 + S_(sq, lx - 1, ly) + q01);
            T qd = o12 * (q00 + q01 + S_(sq, lx + 1, ly));
            T qhv = qa * S_(sV, lx, ly + 1) + qb * S_(sV, lx - 1, ly + 1) + qc * S_(sV, lx - 1, ly) +
                    qd * S_(sV, lx, ly);
            T dpdx = S_(sp, lx, ly) - S_(sp, lx - 1, ly);
            // momentum_u! (src/rhs.jl:218-245)
            Tp du = (cvt<Tp>(qhv) - cvt<Tp>(dpdx)) + cvt<Tp>(A.Fxt * A.Fx.at(x, y));
            long gi = g.idx(x, y);
            Tp X = A.uX[gi];
            if (!A.last) {
                Tp v1 = X + A.b * du;                                     // caxb!
                A.u1o[gi] = v1;
                A.gr.u(A.u1o, g, x, y, v1);
            }
            Tp x0v = (A.first ? X : A.u0i[gi]) + A.a * du;               // axb!
            A.u0o[gi] = x0v;
            if (A.last) A.gr.u(A.u0o, g, x, y, x0v);
        }
        if (g.v_in(x, y)) {
            T q00 = S_(sq, lx, ly);
            T qa = o12 * (S_(sq, lx, ly - 1) + q00 + S_(sq, lx + 1, ly));
            T qb = o12 * (S_(sq, lx + 1, ly - 1) + S_(sq, lx + 1, ly) + q00);
            T qc = o12 * (S_(sq, lx + 1, ly) + q00 + S_(sq, lx + 1, ly + 1));
            T qd = o12 * (q00 + S_(sq, lx, ly + 1) + S_(sq, lx + 1, ly));
            T qhu = qa * S_(sU, lx, ly - 1) + qb * S_(sU, lx + 1, ly - 1) + qc * S_(sU, lx + 1, ly) +
                    qd * S_(sU, lx, ly);
            T dpdy = S_(sp, lx, ly) - S_(sp, lx, ly - 1);
            // momentum_v! (src/rhs.jl:248-274)
            Tp dv = -(cvt<Tp>(qhu) + cvt<Tp>(dpdy)) + cvt<Tp>(A.Fyt * A.Fy.at(x, y));
            long gi = g.idx(x, y);
            Tp X = A.vX[gi];
            if (!A.last) {
                Tp v1 = X + A.b * dv;
                A.v1o[gi] = v1;
                A.gr.v(A.v1o, g, x, y, v1);
            }
            Tp x0v = (A.first ? X : A.v0i[gi]) + A.a * dv;
            A.v0o[gi] = x0v;
            if (A.last) A.gr.v(A.v0o, g, x, y, x0v);
        }
        if (g.e_in(x, y)) {
            // continuity_itself! (src/continuity.jl:52-68)
            T dUdx = S_(sU, lx + 1, ly) - S_(sU, lx, ly);
            T dVdy = S_(sV, lx, ly + 1) - S_(sV, lx, ly);
            Tp de = -(cvt<Tp>(dUdx) + cvt<Tp>(dVdy));
            long gi = g.idx(x, y);
            Tp X = A.eX[gi];
            if (!A.last) {
                Tp v1 = X + A.b * de;
                A.e1o[gi] = v1;
                A.gr.eta(A.e1o, g, x, y, v1);
            }
            Tp x0v = (A.first ? X : A.e0i[gi]) + A.a * de;
            A.e0o[gi] = x0v;
            if (A.last) A.gr.eta(A.e0o, g, x, y, x0v);
        }
    }
#undef S_
}

}  // namespace swb
