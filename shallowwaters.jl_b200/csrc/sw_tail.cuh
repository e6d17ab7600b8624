// sw_tail.cuh -- the dissipative step tail, fused into one launch.
//
// From X0 = (u0, v0, eta0) after ghost_points! it computes
//   bottom_drag!               (src/bottom_drag.jl:2-119: quadratic/linear/none)
//   diffusion!                 (src/diffusion.jl:2-218: Smagorinsky or constant,
//                               biharmonic ∇·ν∇∇²u)
//   add_drag_diff_tendencies!  (src/diffusion.jl:221-251)
//   ghost_points_uv!           (src/ghost_points.jl:202-216)
// writing u, v out of place.  Intermediates follow the reference's arrays and
// operation order, at T-cell (a,b), u-point (F,b), v-point (a,G), corner (F,G):
//   Lu(F,b) = ∇²u, Lv(a,G) = ∇²v                          (src/gradients.jl:29-42)
//   DSq(F,G) = (dudy + dvdx)², DT(a,b) = (dudx + dvdy)²    (src/diffusion.jl:68-111)
//   ν(a,b) = cSmag·sqrt(Ixy(DSq) + DT),  νq(F,G) = Ixy(ν)
//   S11(a,b) = ν·∂xLu, S22(a,b) = ν·∂yLv, S12(F,G) = νq·∂yLu, S21(F,G) = νq·∂xLv
//   LLu1 = ∂xS11, LLu2 = ∂yS12, LLv1 = ∂xS21, LLv2 = ∂yS22  (src/diffusion.jl:126-183)
//   Bu = cD·Ix(sqrtKE)·u / Ix(h), Bv = cD·Iy(sqrtKE)·v / Iy(h) (src/bottom_drag.jl:20-76)
// Execution as in sw_stage.cuh: one warp per 28-column strip, lanes 2..29
// produce output, rows streamed bottom-up with a register window; iteration r
// consumes input row r+2 and writes output row r.
#pragma once
#include "sw_common.cuh"
#include "sw_ghost.cuh"
#include "sw_stage.cuh"

namespace swb {

template <class T, class Tp>
struct TailArgs {
    Geom g;
    int nsx, nsy, nring_blocks;
    const Tp* u0; const Tp* v0; const Tp* e0;   // X0 after ghost points
    Tp* uo; Tp* vo;                             // new u, v
    SField<T> H;
    T cD, rD, cSmag, nuB;
    Tp Dt_diff;
    GhostRule<Tp> gr;
    DevStatus* st;
};

// Where the tail's new u, v go.  TailStoreNative: into A.uo, A.vo (Tprog),
// with their ghost copies when gs.  The 16-bit storage form stores pairs
// instead (sw_s16.cuh).
template <class Tp>
struct TailStoreNative {
    template <class Args>
    __device__ __forceinline__ void u(const Args& A, const Geom& g, int F, int b, int o, Tp val, bool gs) const {
        A.uo[o] = val;
        if (gs) A.gr.u(A.uo, g, F, b, val);
    }
    template <class Args>
    __device__ __forceinline__ void v(const Args& A, const Geom& g, int a, int G, int o, Tp val, bool gs) const {
        A.vo[o] = val;
        if (gs) A.gr.v(A.vo, g, a, G, val);
    }
};

// untouched halo cells keep u0 (and so do their ghost copies)
template <class T, class Tp, class ST = TailStoreNative<Tp>>
__device__ void tail_ring(const TailArgs<T, Tp>& A, int k0, int kstride, const ST& out = ST()) {
    const Geom& g = A.g;
    const int nu = Ring::u_count(g.ep, g.N, g.M), nv = Ring::v_count(g.N);
    for (int k = k0; k < nu + nv; k += kstride) {
        if (k < nu) {
            int F, b;
            Ring::u_at(k, g.ep, g.N, g.M, F, b);
            Tp x = A.u0[g.idx(F, b)];
            out.u(A, g, F, b, g.idx(F, b), x, true);
        } else {
            int a, G;
            Ring::v_at(k - nu, g.N, g.M, a, G);
            Tp x = A.v0[g.idx(a, G)];
            out.v(A, g, a, G, g.idx(a, G), x, true);
        }
    }
}

#ifndef SWB_TAIL_MINB
#define SWB_TAIL_MINB 1    // resident blocks per SM the register budget is sized for
#endif
#ifndef SWB_TAIL_PF
#define SWB_TAIL_PF 2      // input rows in flight ahead of the one consumed (4 and 6 measured slower)
#endif
constexpr int TAIL_PF = SWB_TAIL_PF;
// DRAG: enum sw_bottom_drag; SMAG: Smagorinsky (else constant νB)
// The streaming tail for block bx of its grid (strip blocks, then ring blocks).
template <class T, class Tp, bool PER, int DRAG, bool SMAG, int TY, class ST = TailStoreNative<Tp>>
__device__ __forceinline__ void tail_body(const TailArgs<T, Tp>& A, int bx, const ST& out = ST()) {
    if (A.st->stop) return;
    const Geom& g = A.g;
    const int nstrips = A.nsx * A.nsy;
    const int nstrip_blocks = (nstrips + 3) / 4;
    if (bx >= nstrip_blocks) {
        tail_ring(A, (bx - nstrip_blocks) * 128 + threadIdx.x, A.nring_blocks * 128, out);
        return;
    }
    const int w = bx * 4 + (int)(threadIdx.x >> 5);
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
    constexpr bool QUAD = (DRAG == SW_DRAG_QUADRATIC);
    const T half = T(0.5), q4 = T(0.25);
    const int cb = c + COL0;
    auto ofs = [&](int y) { return (y + ROW0) * P + cb; };

    // window: index 0 = row r, 1 = r+1, 2 = r+2 (inputs); older rows kept explicitly
    auto ldrow = [&](int y, T& uu, T& vv, T& hh) {
        uu = cvt<T>(A.u0[ofs(y)]);
        vv = cvt<T>(A.v0[ofs(y)]);
        if (QUAD) hh = cvt<T>(A.e0[ofs(y)]) + A.H.at(c, y);
        else hh = T(0);
    };
    int r = y0 - 3;
    const int ra = max(r, -2), rb = max(r + 1, -2);
    T u_r, v_r, h_r, u_r1, v_r1, h_r1;
    ldrow(ra, u_r, v_r, h_r);
    ldrow(rb, u_r1, v_r1, h_r1);
    T ul_r1 = shup(u_r1), ur_r1 = shdn(u_r1), vl_r1 = shup(v_r1), vr_r1 = shdn(v_r1), hl_r1 = shup(h_r1);
    T hl_r = shup(h_r);
    T h_rm1 = T(0);
    // derived windows
    T DSq_r1 = T(0), DSqR_r1 = T(0);
    T nu_r = T(0), nul_r = T(0);
    T Lu_r = T(0), Lv_r = T(0);
    T S11_r = T(0), S11l_r = T(0), S12_r = T(0), S21_r = T(0), S21r_r = T(0), S22_rm1 = T(0);
    T sKE_rm1 = T(0), sKE_r = T(0), sKEl_r = T(0);

    // software pipeline: at iteration r, row r+2 is consumed while rows r+3 ..
    // r+2+TAIL_PF are in flight
    T u_r2 = cvt<T>(A.u0[ofs(r + 2)]), v_r2 = cvt<T>(A.v0[ofs(r + 2)]);
    T h_r2 = QUAD ? cvt<T>(A.e0[ofs(r + 2)]) + A.H.at(c, r + 2) : T(0);
    Tp pu[TAIL_PF], pv[TAIL_PF], pe[TAIL_PF];
    T pH[TAIL_PF];
#pragma unroll
    for (int k = 0; k < TAIL_PF; k++) {
        pu[k] = A.u0[ofs(r + 3 + k)];
        pv[k] = A.v0[ofs(r + 3 + k)];
        pe[k] = QUAD ? A.e0[ofs(r + 3 + k)] : Tp(0);
        pH[k] = QUAD ? A.H.at(c, r + 3 + k) : T(0);
    }

SWB_ROW_UNROLL
    for (; r < y0 + TY; r++) {
        if (r > y0 - 3) {
            u_r2 = cvt<T>(pu[0]); v_r2 = cvt<T>(pv[0]);
            h_r2 = QUAD ? cvt<T>(pe[0]) + pH[0] : T(0);
#pragma unroll
            for (int k = 0; k + 1 < TAIL_PF; k++) {
                pu[k] = pu[k + 1]; pv[k] = pv[k + 1]; pe[k] = pe[k + 1]; pH[k] = pH[k + 1];
            }
            const int on = ofs(r + 2 + TAIL_PF);
            pu[TAIL_PF - 1] = A.u0[on]; pv[TAIL_PF - 1] = A.v0[on];
            if (QUAD) { pe[TAIL_PF - 1] = A.e0[on]; pH[TAIL_PF - 1] = A.H.at(c, r + 2 + TAIL_PF); }
        }
        const T ul_r2 = shup(u_r2), ur_r2 = shdn(u_r2), vl_r2 = shup(v_r2), vr_r2 = shdn(v_r2);
        const T hl_r2 = QUAD ? shup(h_r2) : T(0);
        const bool out_row = r >= y0 && r < M;
        Tp U0 = Tp(0), V0 = Tp(0);
        if (std::is_same<T, Tp>::value) { U0 = cvt<Tp>(u_r); V0 = cvt<Tp>(v_r); }
        else if (out_row && out_lane) { U0 = A.u0[ofs(r)]; V0 = A.v0[ofs(r)]; }

        // ∇² at row r+1 (∇²!: ((u[i,j+1]-c)+(u[i+2,j+1]-c)) + ((u[i+1,j]-c)+(u[i+1,j+2]-c)))
        T Lu_r1, Lv_r1;
        {
            T cc = u_r1;
            Lu_r1 = ((ul_r1 - cc) + (ur_r1 - cc)) + ((u_r - cc) + (u_r2 - cc));
            cc = v_r1;
            Lv_r1 = ((vl_r1 - cc) + (vr_r1 - cc)) + ((v_r - cc) + (v_r2 - cc));
        }
        const T Lur_r1 = shdn(Lu_r1), Lvl_r1 = shup(Lv_r1);

        // viscosity ν at T-row r+1 and νq at corner row r+1
        T nu_r1, nuq_r1;
        if (SMAG) {
            T s = (u_r2 - u_r1) + (v_r2 - vl_r2);          // dudy + dvdx at corner (c, r+2)
            const T DSq_r2 = s * s;
            const T DSqR_r2 = shdn(DSq_r2);
            const T DS = q4 * (DSq_r1 + DSqR_r1) + q4 * (DSq_r2 + DSqR_r2);
            s = (ur_r1 - u_r1) + (v_r2 - v_r1);            // dudx + dvdy at T-cell (c, r+1)
            const T DT = s * s;
            nu_r1 = A.cSmag * sqrt(DS + DT);
            const T nul_r1 = shup(nu_r1);
            nuq_r1 = q4 * (nul_r + nu_r) + q4 * (nul_r1 + nu_r1);
            DSq_r1 = DSq_r2; DSqR_r1 = DSqR_r2;
            nul_r = nul_r1;
        } else {
            nu_r1 = A.nuB;
            nuq_r1 = A.nuB;
        }
        const T S11_r1 = nu_r1 * (Lur_r1 - Lu_r1);       // at T-cell (c, r+1)
        const T S11l_r1 = shup(S11_r1);
        const T S12_r1 = nuq_r1 * (Lu_r1 - Lu_r);         // at corner (c, r+1)
        const T S21_r1 = nuq_r1 * (Lv_r1 - Lvl_r1);       // at corner (c, r+1)
        const T S21r_r1 = shdn(S21_r1);
        const T S22_r = nu_r * (Lv_r1 - Lv_r);            // at T-cell (c, r)

        T sKE_r1 = T(0), sKEl_r1 = T(0);
        if (QUAD) {
            const T KEu = half * (ur_r1 * ur_r1 + u_r1 * u_r1);
            const T KEv = half * (v_r2 * v_r2 + v_r1 * v_r1);
            sKE_r1 = sqrt(KEu + KEv);
            sKEl_r1 = shup(sKE_r1);
        }

        if (out_row) {
            if (col_u) {
                T Bu;
                if (QUAD) {
                    T ke = half * (sKE_r + sKEl_r);
                    T hu = half * (h_r + hl_r);
                    Bu = A.cD * ke * u_r / hu;
                } else if (DRAG == SW_DRAG_LINEAR) {
                    Bu = A.rD * u_r;
                } else {
                    Bu = T(0);
                }
                const T LLu1 = S11_r - S11l_r;
                const T LLu2 = S12_r1 - S12_r;
                Tp val = U0 + A.Dt_diff * (cvt<Tp>(Bu) + cvt<Tp>(LLu1) + cvt<Tp>(LLu2));
                out.u(A, g, c, r, ofs(r), val, gx_u || (!PER && (r <= 1 || r >= M - 2)));
            }
            if (col_a && r >= 1) {
                T Bv;
                if (QUAD) {
                    T ke = half * (sKE_r + sKE_rm1);
                    T hv = half * (h_r + h_rm1);
                    Bv = A.cD * ke * v_r / hv;
                } else if (DRAG == SW_DRAG_LINEAR) {
                    Bv = A.rD * v_r;
                } else {
                    Bv = T(0);
                }
                const T LLv1 = S21r_r - S21_r;
                const T LLv2 = S22_r - S22_rm1;
                Tp val = V0 + A.Dt_diff * (cvt<Tp>(Bv) + cvt<Tp>(LLv1) + cvt<Tp>(LLv2));
                out.v(A, g, c, r, ofs(r), val, gx_v);
            }
        }

        // slide
        h_rm1 = h_r;
        u_r = u_r1; v_r = v_r1; h_r = h_r1; hl_r = hl_r1;
        u_r1 = u_r2; v_r1 = v_r2; h_r1 = h_r2; hl_r1 = hl_r2;
        ul_r1 = ul_r2; ur_r1 = ur_r2; vl_r1 = vl_r2; vr_r1 = vr_r2;
        nu_r = nu_r1;
        Lu_r = Lu_r1; Lv_r = Lv_r1;
        S11_r = S11_r1; S11l_r = S11l_r1; S12_r = S12_r1; S21_r = S21_r1; S21r_r = S21r_r1;
        S22_rm1 = S22_r;
        sKE_rm1 = sKE_r; sKE_r = sKE_r1; sKEl_r = sKEl_r1;
    }
}


template <class T, class Tp, bool PER, int DRAG, bool SMAG, int TY>
__global__ void __launch_bounds__(128, SWB_TAIL_MINB)
tail_kernel(const __grid_constant__ TailArgs<T, Tp> A) {
    tail_body<T, Tp, PER, DRAG, SMAG, TY>(A, (int)blockIdx.x);
}

}  // namespace swb
