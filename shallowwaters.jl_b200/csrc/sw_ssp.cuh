// sw_ssp.cuh -- stages of the strong-stability-preserving schemes SSPRK2,
// SSPRK3 and 4SSPRK3 (src/time_integration.jl:80-196).
//
// Unlike RK, every stage of these schemes is semi-implicit: the momentum
// update u1 <- f(u1, du) comes first, ghost_points_uv! follows, and only then
// is continuity! evaluated with the NEW u1, v1 and the old eta1
// (src/time_integration.jl:91-100; UVfluxes! inside continuity!,
// src/continuity.jl:80-85).  A stage is therefore two launches:
//   ssp_momentum_kernel   rhs_nonlinear! (du, dv) + the scheme's u/v update,
//                         with ghost points fused into the write-back and the
//                         untouched halo cells updated by ring blocks;
//   ssp_continuity_kernel U, V from the new u, v; deta; the eta update.
// Where a scheme combines u1 with the state after continuity! has used it
// (SSPRK2's final cxayb!, 4SSPRK3's stage-3 cxayb!), the kernels write that
// combination fa*u + fb*u1 as a second output (COMBO) next to u1.
// The per-cell updates follow the reference's whole-array helpers
// (src/time_integration.jl:253-326) operation for operation:
//   axb!     a += x*b                     caxb!   c = a + x*b
//   cxab!    c = x*(a + b)                cxayb!  c = x*a + y*b
//   dxaybzc! d = x*a + y*b + z*c
// Halo cells that ghost_points! never writes go through the same update with
// a zero tendency, exactly as the whole-array helpers treat them.
#pragma once
#include "sw_stage.cuh"

namespace swb {

// What a stage does to u1 (and, in the continuity kernel, to eta1).
enum SspMode : int {
    SSP_AXB = 0,    // u1 += x*du                        SSPRK2; SSPRK3 ordinary stages
    SSP_KN = 1,     // u1 = kna*u1 + knb*u0 + z*du       SSPRK3 stage kn (dxaybzc!)
    SSP_4 = 2,      // u0 = u1 + x*du; u1 = ½(u1 + u0)   4SSPRK3 (caxb!, cxab!)
};

template <class Tp>
struct SspCoef {
    Tp x;            // Δt_Δs, Δt_Δn, Δt_Δnc or Δt_Δ
    Tp kna, knb;     // SSPRK3 kn-stage weights
    Tp half;         // Tp(0.5)
    Tp fa, fb;       // COMBO weights: Tp(1/RKs), Tp((RKs-1)/RKs) or Tp(2/3), Tp(1/3)
};

// the stage update of one value; z is the snapshot u0 (SSP_KN)
template <int MODE, class Tp>
__device__ __forceinline__ Tp ssp_update(const SspCoef<Tp>& k, Tp u1, Tp z, Tp d) {
    if (MODE == SSP_AXB) return u1 + k.x * d;
    if (MODE == SSP_KN) return k.kna * u1 + k.knb * z + k.x * d;
    const Tp u0 = u1 + k.x * d;          // caxb!(u0, u1, Δt_Δ, du)
    return k.half * (u1 + u0);           // cxab!(u1, 1/2, u1, u0)
}

template <class T, class Tp>
struct SspArgs {
    Geom g;
    int nsx, nsy, nring_blocks;
    const Tp* u1; const Tp* v1; const Tp* e1;   // stage input (ghosts valid)
    const Tp* uS; const Tp* vS; const Tp* eS;   // state u at the step start (COMBO)
    const Tp* uZ; const Tp* vZ; const Tp* eZ;   // snapshot u0 (SSP_KN)
    Tp* u1o; Tp* v1o; Tp* e1o;                   // updated u1 (always written)
    Tp* ufo; Tp* vfo; Tp* efo;                   // combination fa*u + fb*u1 (COMBO only)
    SField<T> H, fq, Fx, Fy;
    T g_, Fxt, Fyt;
    int cont;                                    // continuity! variant, as StageArgs::cont
    int sadourny;                                // PV_Sadourny!, as StageArgs::sadourny
    const T* qS; const T* KEuS; const T* KEvS;   // stored advection/Coriolis terms, as StageArgs
    SField<T> eref, Feta;
    T gamma, Fetat;
    SspCoef<Tp> k;
    GhostRule<Tp> gr;
    DevStatus* st;
};

// untouched halo cells of u1 (and of the final combination)
template <int MODE, bool COMBO, class T, class Tp>
__device__ void ssp_ring(const SspArgs<T, Tp>& A, int k0, int kstride) {
    const Geom& g = A.g;
    const int nu = Ring::u_count(g.ep, g.N, g.M), nv = Ring::v_count(g.N);
    const Tp zero = Tp(0);
    for (int k = k0; k < nu + nv; k += kstride) {
        int x, y;
        const bool isu = k < nu;
        if (isu) Ring::u_at(k, g.ep, g.N, g.M, x, y);
        else Ring::v_at(k - nu, g.N, g.M, x, y);
        const int gi = g.idx(x, y);
        const Tp* in = isu ? A.u1 : A.v1;
        const Tp* zs = isu ? A.uZ : A.vZ;
        const Tp* ss = isu ? A.uS : A.vS;
        const Tp z = (MODE == SSP_KN) ? zs[gi] : zero;
        const Tp s = COMBO ? ss[gi] : zero;
        const Tp r = ssp_update<MODE>(A.k, in[gi], z, zero);
        Tp* out = isu ? A.u1o : A.v1o;
        out[gi] = r;
        if (isu) A.gr.u(out, g, x, y, r); else A.gr.v(out, g, x, y, r);
        if (COMBO) {
            const Tp f = A.k.fa * s + A.k.fb * r;
            Tp* fo = isu ? A.ufo : A.vfo;
            fo[gi] = f;
            if (isu) A.gr.u(fo, g, x, y, f); else A.gr.v(fo, g, x, y, f);
        }
    }
}

// rhs_nonlinear! (src/rhs.jl:24-51) for du, dv at the stage input, then the
// stage update of u1, v1.  Same row recurrence as rk_stage_kernel.
template <class T, class Tp, bool PER, int MODE, bool COMBO, int TY>
__global__ void __launch_bounds__(128)
ssp_momentum_kernel(const __grid_constant__ SspArgs<T, Tp> A) {
    if (A.st->stop) return;
    const Geom& g = A.g;
    const int nstrips = A.nsx * A.nsy;
    const int nstrip_blocks = (nstrips + 3) / 4;
    if ((int)blockIdx.x >= nstrip_blocks) {
        ssp_ring<MODE, COMBO>(A, ((int)blockIdx.x - nstrip_blocks) * 128 + threadIdx.x, A.nring_blocks * 128);
        return;
    }
    const int w = (int)blockIdx.x * 4 + (int)(threadIdx.x >> 5);
    if (w >= nstrips) return;
    const int lane = threadIdx.x & 31;
    const int sx = w % A.nsx, sy = w / A.nsx;
    const int c = sx * STRIP + lane - 2;
    const int y0 = sy * TY;
    const int N = g.N, M = g.M, P = g.P;
    const bool out_lane = lane >= 2 && lane < 2 + STRIP;
    const bool col_u = out_lane && c >= (PER ? 0 : 1) && c < N;
    const bool col_a = out_lane && c >= 0 && c < N;
    const bool gx_u = PER && (c <= 1 || c >= N - 2);
    const bool gx_v = c <= 1 || c >= N - 2;
    const bool wrap = PER && c == -1;     // q[end] for the AHβ!/AHγ! wrap (src/PV_advection.jl:110,126)
    const T half = T(0.5), o12 = T(1.0 / 12.0);

    const int cb = c + COL0;
    const Tp* __restrict__ pu = A.u1 + cb;
    const Tp* __restrict__ pv = A.v1 + cb;
    const Tp* __restrict__ pe = A.e1 + cb;
    auto row = [&](int y) { return (y + ROW0) * P; };

    int r = y0 - 2;
    T u_r = cvt<T>(pu[row(r)]), v_r = cvt<T>(pv[row(r)]), e_r = cvt<T>(pe[row(r)]);
    T h_r = e_r + A.H.at(c, r);
    T hl_r = shup(h_r), ur_r = shdn(u_r);
    T U_r = u_r * (half * (h_r + hl_r));
    T Ur_r = shdn(U_r);
    T V_r = T(0), Vl_r = T(0), q_r = T(0), ql_r = T(0), qr_r = T(0);
    T p_rm1 = T(0), qhu_part = T(0), sad_part = T(0);
    T uN_r = T(0), hN_r = T(0), hNm1_r = T(0);
    if (wrap) {
        uN_r = cvt<T>(A.u1[g.idx(N, r)]);
        hN_r = cvt<T>(A.e1[g.idx(N, r)]) + A.H.at(N, r);
        hNm1_r = cvt<T>(A.e1[g.idx(N - 1, r)]) + A.H.at(N - 1, r);
    }

    for (; r < y0 + TY; r++) {
        const int o1 = row(r + 1);
        const T u_r1 = cvt<T>(pu[o1]), v_r1 = cvt<T>(pv[o1]), e_r1 = cvt<T>(pe[o1]);
        const T h_r1 = e_r1 + A.H.at(c, r + 1);                    // thickness! (src/rhs.jl:131-139)
        const T hl_r1 = shup(h_r1), vl_r1 = shup(v_r1), ur_r1 = shdn(u_r1);

        T q_r1;                                                     // PV! (src/PV_advection.jl:2-18)
        const T fq = A.fq.at(c, r + 1);
        T uN_r1 = T(0), hN_r1 = T(0), hNm1_r1 = T(0);
        if (A.qS) {
            q_r1 = A.qS[g.idx(c, r + 1)];                          // stored at the last refresh
        } else if (wrap) {
            uN_r1 = cvt<T>(A.u1[g.idx(N, r + 1)]);
            hN_r1 = cvt<T>(A.e1[g.idx(N, r + 1)]) + A.H.at(N, r + 1);
            hNm1_r1 = cvt<T>(A.e1[g.idx(N - 1, r + 1)]) + A.H.at(N - 1, r + 1);
            T vN = cvt<T>(A.v1[g.idx(N, r + 1)]), vNm1 = cvt<T>(A.v1[g.idx(N - 1, r + 1)]);
            q_r1 = pv_q<T>(fq, vN, vNm1, uN_r1, uN_r, hNm1_r, hN_r, hNm1_r1, hN_r1);
        } else {
            q_r1 = pv_q<T>(fq, v_r1, vl_r1, u_r1, u_r, hl_r, h_r, hl_r1, h_r1);
        }
        const T ql_r1 = shup(q_r1), qr_r1 = shdn(q_r1);
        const T U_r1 = u_r1 * (half * (h_r1 + hl_r1));              // Uflux!/Vflux! (src/rhs.jl:277-304)
        const T V_r1 = v_r1 * (half * (h_r1 + h_r));
        const T Ur_r1 = shdn(U_r1), Vl_r1 = shup(V_r1);
        const T KEu = A.qS ? A.KEuS[g.idx(c, r)] : half * (ur_r * ur_r + u_r * u_r);             // bernoulli! (src/rhs.jl:162-180)
        const T KEv = A.qS ? A.KEvS[g.idx(c, r)] : half * (v_r1 * v_r1 + v_r * v_r);
        const T p_r = half * (KEu + KEv) + A.g_ * e_r;
        const T pl_r = shup(p_r);
        const T s = q_r + q_r1;                                     // AHα..δ (src/PV_advection.jl:88-146)
        const T qa = o12 * (s + qr_r1);
        const T qb = o12 * (s + ql_r1);
        const T qc = (PER && c == 0) ? o12 * (s + ql_r) : o12 * (q_r + ql_r + q_r1);
        const T qd = o12 * (s + qr_r);
        const T qbr = shdn(qb), qcr = shdn(qc);

        if (r >= y0 && r < M) {
            const int o = row(r) + cb;
            if (col_u) {                                            // momentum_u! (src/rhs.jl:218-245)
                const T qhv = A.sadourny ? sadourny_qhv(q_r, q_r1, V_r, Vl_r, V_r1, Vl_r1)
                                         : qa * V_r1 + qb * Vl_r1 + qc * Vl_r + qd * V_r;
                const T dpdx = p_r - pl_r;
                const Tp du = (cvt<Tp>(qhv) - cvt<Tp>(dpdx)) + cvt<Tp>(A.Fxt * A.Fx.at(c, r));
                const Tp z = (MODE == SSP_KN) ? A.uZ[o] : Tp(0);
                const Tp st = COMBO ? A.uS[o] : Tp(0);
                const Tp x1 = ssp_update<MODE>(A.k, A.u1[o], z, du);
                const bool gs = gx_u || (!PER && (r <= 1 || r >= M - 2));
                A.u1o[o] = x1;
                if (gs) A.gr.u(A.u1o, g, c, r, x1);
                if (COMBO) {
                    const Tp f = A.k.fa * st + A.k.fb * x1;        // cxayb! (src/time_integration.jl:107-109,186-191)
                    A.ufo[o] = f;
                    if (gs) A.gr.u(A.ufo, g, c, r, f);
                }
            }
            if (col_a && r >= 1) {                                  // momentum_v! (src/rhs.jl:248-274)
                const T qhu = A.sadourny ? (half * (qr_r + q_r)) * (sad_part + T(0.25) * (U_r + Ur_r))
                                             : qhu_part + qcr * Ur_r + qd * U_r;
                const T dpdy = p_r - p_rm1;
                const Tp dv = -(cvt<Tp>(qhu) + cvt<Tp>(dpdy)) + cvt<Tp>(A.Fyt * A.Fy.at(c, r));
                const Tp z = (MODE == SSP_KN) ? A.vZ[o] : Tp(0);
                const Tp st = COMBO ? A.vS[o] : Tp(0);
                const Tp x1 = ssp_update<MODE>(A.k, A.v1[o], z, dv);
                A.v1o[o] = x1;
                if (gx_v) A.gr.v(A.v1o, g, c, r, x1);
                if (COMBO) {
                    const Tp f = A.k.fa * st + A.k.fb * x1;
                    A.vfo[o] = f;
                    if (gx_v) A.gr.v(A.vfo, g, c, r, f);
                }
            }
        }

        qhu_part = qa * U_r + qbr * Ur_r;
        sad_part = T(0.25) * (U_r + Ur_r);
        u_r = u_r1; v_r = v_r1; e_r = e_r1; h_r = h_r1; hl_r = hl_r1; ur_r = ur_r1;
        q_r = q_r1; ql_r = ql_r1; qr_r = qr_r1;
        U_r = U_r1; Ur_r = Ur_r1;
        V_r = V_r1; Vl_r = Vl_r1;
        p_rm1 = p_r;
        uN_r = uN_r1; hN_r = hN_r1; hNm1_r = hNm1_r1;
    }
}

// continuity! with UVfluxes! of the new u, v (src/continuity.jl:72-97,
// src/rhs.jl:307-324): U = u*Ix(h), V = v*Iy(h), h = eta1 + H, then
// deta = -(dUdx + dVdy) and the eta update.  One thread per T-cell.
template <class T, class Tp, int MODE, bool COMBO>
__global__ void __launch_bounds__(256)
ssp_continuity_kernel(const __grid_constant__ SspArgs<T, Tp> A) {
    if (A.st->stop) return;
    const Geom& g = A.g;
    const int a = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int b = (int)blockIdx.y;
    if (a >= g.N) return;
    const T half = T(0.5);
    auto h = [&](int x, int y) { return cvt<T>(A.e1[g.idx(x, y)]) + A.H.at(x, y); };
    const T hc = h(a, b);
    const T Ua = cvt<T>(A.u1o[g.idx(a, b)]) * (half * (hc + h(a - 1, b)));
    const T Ua1 = cvt<T>(A.u1o[g.idx(a + 1, b)]) * (half * (h(a + 1, b) + hc));
    const T Vb = cvt<T>(A.v1o[g.idx(a, b)]) * (half * (hc + h(a, b - 1)));
    const T Vb1 = cvt<T>(A.v1o[g.idx(a, b + 1)]) * (half * (h(a, b + 1) + hc));
    const T dUdx = Ua1 - Ua;
    const T dVdy = Vb1 - Vb;
    const Tp de = deta_of<T, Tp>(A.cont, dUdx, dVdy, cvt<T>(A.e1[g.idx(a, b)]), A.eref, A.Feta, A.gamma, A.Fetat,
                                 a, b);                              // src/continuity.jl:3-68
    const int o = g.idx(a, b);
    const Tp z = (MODE == SSP_KN) ? A.eZ[o] : Tp(0);
    const Tp st = COMBO ? A.eS[o] : Tp(0);
    const Tp x1 = ssp_update<MODE>(A.k, A.e1[o], z, de);
    const bool gs = a == 0 || a == g.N - 1 || b == 0 || b == g.M - 1;
    if (!COMBO) {
        A.e1o[o] = x1;
        if (gs) A.gr.eta(A.e1o, g, a, b, x1);
    } else {
        const Tp f = A.k.fa * st + A.k.fb * x1;                   // cxayb! on eta
        A.efo[o] = f;
        if (gs) A.gr.eta(A.efo, g, a, b, f);
    }
}

}  // namespace swb
