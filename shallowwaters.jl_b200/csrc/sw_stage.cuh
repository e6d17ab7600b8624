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
// Execution: register streaming.  Each warp owns a strip of 28 columns
// (lanes 2..29 produce output; lanes 0,1 and 30,31 are halo) and TY rows.  It
// walks up the rows holding a sliding window of every intermediate in
// registers; x-neighbours come from warp shuffles, so there is no shared
// memory and no block barrier.  Column of lane L: c = 28*strip + L - 2, used
// as the face index F for u/U/q and as the T-cell index a for v/V/h/p.
// Iteration r (from y0-2 to y0+TY-1) consumes input row r+1 and forms
//   q(c, G=r+1), U(c, b=r+1), V(c, G=r+1), p(c, b=r), AH combos at (c, b=r)
// and the outputs du(c, r), dv(c, G=r), deta(c, r).
#pragma once
#include <type_traits>

#include "sw_common.cuh"
#include "sw_ghost.cuh"
#include "sw_tma.cuh"

namespace swb {

constexpr int STRIP = 28;   // output columns per warp

template <class T, class Tp>
struct StageArgs {
    Geom g;
    int nsx, nsy;                       // strips in x and y; warps beyond do the ring
    int nring_blocks;
    const Tp* u1; const Tp* v1; const Tp* e1;    // stage input (ghosts valid)
    const Tp* uX; const Tp* vX; const Tp* eX;    // step-start state X
    const Tp* u0i; const Tp* v0i; const Tp* e0i; // accumulator in (unused on the first stage)
    Tp* u1o; Tp* v1o; Tp* e1o;                   // X1' (unused on the last stage)
    Tp* u0o; Tp* v0o; Tp* e0o;                   // accumulator out
    SField<T> H, fq, Fx, Fy;
    Tp a, b;                            // RKaΔt[k], RKbΔt[k] (Tprog)
    T g_;                               // gravity (T)
    T Fxt, Fyt;                         // seasonal factors (1 if off)
    // continuity! variant (src/continuity.jl:3-49): 0 plain, 1 surface
    // relaxation gamma*(eta_ref - eta), 2 surface forcing Fetat*Feta.  Only the
    // streaming kernel implements 1 and 2.
    int cont;
    SField<T> eref, Feta;
    T gamma, Fetat;
    int sadourny;                       // 1: PV_Sadourny! instead of PV_ArakawaHsu! (streaming kernel only)
    // nstep_advcor > 0: q and KEu, KEv of the last refresh (sw_advcor.cuh),
    // null otherwise (streaming kernel only)
    const T* qS; const T* KEuS; const T* KEvS;
    GhostRule<Tp> gr;
    DevStatus* st;
    // bounded waits of the TMA kernel: polls per wait, and (test only, -1
    // otherwise) a chunk of block 0's first tile that the producer leaves out,
    // so that its consumers' wait runs out
    uint32_t spin_limit;
    int skip_chunk;
};

// deta at the T-cell (c, r) from the flux divergences: continuity_itself!,
// continuity_surf_relax!, continuity_forcing! (src/continuity.jl:3-68)
template <class T, class Tp>
__device__ __forceinline__ Tp deta_of(int cont, T dUdx, T dVdy, T eta, const SField<T>& eref, const SField<T>& Feta,
                                      T gamma, T Fetat, int c, int r) {
    const Tp de = -(cvt<Tp>(dUdx) + cvt<Tp>(dVdy));
    if (cont == 1) return de + cvt<Tp>(gamma * (eref.at(c, r) - eta));
    if (cont == 2) return de + cvt<Tp>(Fetat * Feta.at(c, r));
    return de;
}

// PV_Sadourny! at the u-point (F, b) (src/PV_advection.jl:31-59):
// Iy!(q) * Ixy!(V) with q at the corners (F, b), (F, b+1) and V at
// (F-1, b), (F, b), (F-1, b+1), (F, b+1).  The v-point form Ix!(q) * Ixy!(U)
// is written inline where its lower half, carried from the previous row, is.
template <class T>
__device__ __forceinline__ T sadourny_qhv(T q_b, T q_b1, T V_b, T Vl_b, T V_b1, T Vl_b1) {
    const T half = T(0.5), q4 = T(0.25);
    return (half * (q_b1 + q_b)) * (q4 * (Vl_b + V_b) + q4 * (Vl_b1 + V_b1));
}

// q at the corner (F, G): PV! (src/PV_advection.jl:2-18) with h_q = Ixy!(h)
// (src/interpolations.jl:33-45), dvdx = ∂x!(v), dudy = ∂y!(u)
template <class T>
__device__ __forceinline__ T pv_q(T fq, T vR, T vL, T uT, T uB, T hLB, T hRB, T hLT, T hRT) {
    const T q4 = T(0.25);
    T hq = q4 * (hLB + hRB) + q4 * (hLT + hRT);
    T dvdx = vR - vL;
    T dudy = uT - uB;
    return (fq + dvdx - dudy) / hq;
}

template <class T>
__device__ __forceinline__ T shup(T x) { return __shfl_up_sync(0xffffffffu, x, 1); }
template <class T>
__device__ __forceinline__ T shdn(T x) { return __shfl_down_sync(0xffffffffu, x, 1); }
__device__ __forceinline__ jf16 shup(jf16 x) { jf16 r; r.h = __shfl_up_sync(0xffffffffu, x.h, 1); return r; }
__device__ __forceinline__ jf16 shdn(jf16 x) { jf16 r; r.h = __shfl_down_sync(0xffffffffu, x.h, 1); return r; }

// Ring: untouched halo cells of X1' / X0 (see sw_ghost.cuh)
template <class T, class Tp>
__device__ void stage_ring(const StageArgs<T, Tp>& A, bool first, bool last, int k0, int kstride) {
    const Geom& g = A.g;
    const int nu = Ring::u_count(g.ep, g.N, g.M), nv = Ring::v_count(g.N);
    const Tp zero = Tp(0);
    for (int k = k0; k < nu + nv; k += kstride) {
        if (k < nu) {
            int F, b;
            Ring::u_at(k, g.ep, g.N, g.M, F, b);
            int gi = g.idx(F, b);
            Tp x = A.uX[gi];
            if (!last) {
                Tp v1 = x + A.b * zero;
                A.u1o[gi] = v1;
                A.gr.u(A.u1o, g, F, b, v1);
            }
            Tp x0 = (first ? x : A.u0i[gi]) + A.a * zero;
            A.u0o[gi] = x0;
            if (last) A.gr.u(A.u0o, g, F, b, x0);
        } else {
            int a, G;
            Ring::v_at(k - nu, g.N, g.M, a, G);
            int gi = g.idx(a, G);
            Tp x = A.vX[gi];
            if (!last) {
                Tp v1 = x + A.b * zero;
                A.v1o[gi] = v1;
                A.gr.v(A.v1o, g, a, G, v1);
            }
            Tp x0 = (first ? x : A.v0i[gi]) + A.a * zero;
            A.v0o[gi] = x0;
            if (last) A.gr.v(A.v0o, g, a, G, x0);
        }
    }
}

// The streaming stage for block bx of its grid (strip blocks, then ring blocks).
template <class T, class Tp, bool PER, bool FIRST, bool LAST, int TY>
__device__ __forceinline__ void rk_stage_body(const StageArgs<T, Tp>& A, int bx) {
    if (A.st->stop) return;
    const Geom& g = A.g;
    const int nstrips = A.nsx * A.nsy;
    const int nstrip_blocks = (nstrips + 3) / 4;
    if (bx >= nstrip_blocks) {
        stage_ring(A, FIRST, LAST, (bx - nstrip_blocks) * 128 + threadIdx.x, A.nring_blocks * 128);
        return;
    }
    const int w = bx * 4 + (int)(threadIdx.x >> 5);
    if (w >= nstrips) return;                 // whole warp leaves together
    const int lane = threadIdx.x & 31;
    const int sx = w % A.nsx, sy = w / A.nsx;
    const int c = sx * STRIP + lane - 2;
    const int y0 = sy * TY;
    const int N = g.N, M = g.M, P = g.P;
    const bool out_lane = lane >= 2 && lane < 2 + STRIP;
    const bool col_u = out_lane && c >= (PER ? 0 : 1) && c < N;
    const bool col_a = out_lane && c >= 0 && c < N;
    // ghost sources that depend on the column only
    const bool gx_u = PER && (c <= 1 || c >= N - 2);
    const bool gx_v = c <= 1 || c >= N - 2;
    const bool gx_e = c == 0 || c == N - 1;
    // the lane whose q feeds the AHβ!/AHγ! wrap at F = 0 evaluates q at F = N
    // (q[end], src/PV_advection.jl:110,126) instead of at its own column -1
    const bool wrap = PER && c == -1;
    const T half = T(0.5), o12 = T(1.0 / 12.0);
    constexpr bool SAME = std::is_same<T, Tp>::value;

    // lane base pointers; row y is at offset (y + ROW0) * P
    const int cb = c + COL0;
    const Tp* __restrict__ pu = A.u1 + cb;
    const Tp* __restrict__ pv = A.v1 + cb;
    const Tp* __restrict__ pe = A.e1 + cb;
    const int Hsx = A.H.sx, Hsy = A.H.sy;
    const T* __restrict__ pH = A.H.p + cb * Hsx;
    const T* __restrict__ pfq = A.fq.p + cb * A.fq.sx;
    const int fqsy = A.fq.sy;
    auto row = [&](int y) { return (y + ROW0) * P; };

    // ---- preload row y0-2
    int r = y0 - 2;
    T u_r = cvt<T>(pu[row(r)]), v_r = cvt<T>(pv[row(r)]), e_r = cvt<T>(pe[row(r)]);
    T h_r = e_r + pH[(r + ROW0) * Hsy];
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
    // software pipeline: inputs one row ahead, X/X0 one row ahead
    Tp pu1 = pu[row(r + 1)], pv1 = pv[row(r + 1)], pe1 = pe[row(r + 1)];
    T pH1 = pH[(r + 1 + ROW0) * Hsy];
    Tp xu = Tp(0), xv = Tp(0), xe = Tp(0), x0u = Tp(0), x0v = Tp(0), x0e = Tp(0);
    auto load_x = [&](int y, Tp& a_, Tp& b_, Tp& c_, Tp& d_, Tp& e_, Tp& f_) {
        if (y >= y0 && out_lane) {
            const int oy = row(y) + cb;
            if (FIRST) {
                // X is the stage input; re-read only if converting to T lost bits
                if (!SAME) { a_ = A.uX[oy]; b_ = A.vX[oy]; c_ = A.eX[oy]; }
            } else {
                if (!LAST) { a_ = A.uX[oy]; b_ = A.vX[oy]; c_ = A.eX[oy]; }
                d_ = A.u0i[oy]; e_ = A.v0i[oy]; f_ = A.e0i[oy];
            }
        }
    };
    load_x(r, xu, xv, xe, x0u, x0v, x0e);

SWB_ROW_UNROLL
    for (; r < y0 + TY; r++) {
        // ---- row r+1 from the pipeline; issue row r+2
        const T u_r1 = cvt<T>(pu1), v_r1 = cvt<T>(pv1), e_r1 = cvt<T>(pe1);
        const T h_r1 = e_r1 + pH1;                              // thickness! (src/rhs.jl:131-139)
        {
            const int o2 = row(r + 2);
            pu1 = pu[o2]; pv1 = pv[o2]; pe1 = pe[o2];
            pH1 = pH[(r + 2 + ROW0) * Hsy];
        }
        const int o = row(r) + cb;
        // X and X0 at the output row r (issued one iteration earlier); issue row r+1
        const Tp Xu_ = xu, Xv_ = xv, Xe_ = xe, X0u = x0u, X0v = x0v, X0e = x0e;
        load_x(r + 1, xu, xv, xe, x0u, x0v, x0e);
        const T hl_r1 = shup(h_r1), vl_r1 = shup(v_r1), ur_r1 = shdn(u_r1);

        // ---- q(c, G=r+1)
        T q_r1;
        const T fq = pfq[(r + 1 + ROW0) * fqsy];
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

        // ---- U(c, r+1) = u·Ix!(h), V(c, r+1) = v·Iy!(h)   (Uflux!/Vflux!, src/rhs.jl:277-304)
        const T U_r1 = u_r1 * (half * (h_r1 + hl_r1));
        const T V_r1 = v_r1 * (half * (h_r1 + h_r));
        const T Ur_r1 = shdn(U_r1), Vl_r1 = shup(V_r1);

        // ---- p(c, r) = ½(KEu + KEv) + gη   (bernoulli!, src/rhs.jl:162-180)
        const T KEu = A.qS ? A.KEuS[g.idx(c, r)] : half * (ur_r * ur_r + u_r * u_r);
        const T KEv = A.qS ? A.KEvS[g.idx(c, r)] : half * (v_r1 * v_r1 + v_r * v_r);
        const T p_r = half * (KEu + KEv) + A.g_ * e_r;
        const T pl_r = shup(p_r);

        // ---- Arakawa-Hsu combinations at the u-point (c, r)  (src/PV_advection.jl:88-146)
        const T s = q_r + q_r1;
        const T qa = o12 * (s + qr_r1);
        const T qb = o12 * (s + ql_r1);
        const T qc = (PER && c == 0) ? o12 * (s + ql_r) : o12 * (q_r + ql_r + q_r1);
        const T qd = o12 * (s + qr_r);
        const T qbr = shdn(qb), qcr = shdn(qc);

        if (r >= y0 && r < M) {
            // du at (F=c, b=r): momentum_u! (src/rhs.jl:218-245) with qhv (PV_ArakawaHsu!, :63-75)
            if (col_u) {
                const T qhv = A.sadourny ? sadourny_qhv(q_r, q_r1, V_r, Vl_r, V_r1, Vl_r1)
                                         : qa * V_r1 + qb * Vl_r1 + qc * Vl_r + qd * V_r;
                const T dpdx = p_r - pl_r;
                const Tp du = (cvt<Tp>(qhv) - cvt<Tp>(dpdx)) + cvt<Tp>(A.Fxt * A.Fx.at(c, r));
                const Tp X = (FIRST && SAME) ? cvt<Tp>(u_r) : Xu_;
                const bool gs = gx_u || (!PER && (r <= 1 || r >= M - 2));
                if (!LAST) {
                    const Tp x1 = X + A.b * du;                     // caxb!
                    A.u1o[o] = x1;
                    if (gs) A.gr.u(A.u1o, g, c, r, x1);
                }
                const Tp x0 = (FIRST ? X : X0u) + A.a * du;         // axb!
                A.u0o[o] = x0;
                if (LAST && gs) A.gr.u(A.u0o, g, c, r, x0);
            }
            if (col_a) {
                // dv at (a=c, G=r): momentum_v! (:248-274) with qhu (:77-83)
                if (r >= 1) {
                    const T qhu = A.sadourny ? (half * (qr_r + q_r)) * (sad_part + T(0.25) * (U_r + Ur_r))
                                             : qhu_part + qcr * Ur_r + qd * U_r;
                    const T dpdy = p_r - p_rm1;
                    const Tp dv = -(cvt<Tp>(qhu) + cvt<Tp>(dpdy)) + cvt<Tp>(A.Fyt * A.Fy.at(c, r));
                    const Tp X = (FIRST && SAME) ? cvt<Tp>(v_r) : Xv_;
                    if (!LAST) {
                        const Tp x1 = X + A.b * dv;
                        A.v1o[o] = x1;
                        if (gx_v) A.gr.v(A.v1o, g, c, r, x1);
                    }
                    const Tp x0 = (FIRST ? X : X0v) + A.a * dv;
                    A.v0o[o] = x0;
                    if (LAST && gx_v) A.gr.v(A.v0o, g, c, r, x0);
                }
                // deta at (a=c, b=r): continuity_itself! (src/continuity.jl:52-68)
                const T dUdx = Ur_r - U_r;
                const T dVdy = V_r1 - V_r;
                const Tp de = deta_of<T, Tp>(A.cont, dUdx, dVdy, e_r, A.eref, A.Feta, A.gamma, A.Fetat, c, r);
                const Tp X = (FIRST && SAME) ? cvt<Tp>(e_r) : Xe_;
                const bool gs = gx_e || r == 0 || r == M - 1;
                if (!LAST) {
                    const Tp x1 = X + A.b * de;
                    A.e1o[o] = x1;
                    if (gs) A.gr.eta(A.e1o, g, c, r, x1);
                }
                const Tp x0 = (FIRST ? X : X0e) + A.a * de;
                A.e0o[o] = x0;
                if (LAST && gs) A.gr.eta(A.e0o, g, c, r, x0);
            }
        }

        // ---- slide the window; the first two products of qhu at G = r+1
        // (qα(c,r)·U(c,r) + qβ(c+1,r)·U(c+1,r)) are formed now, in the same order
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


template <class T, class Tp, bool PER, bool FIRST, bool LAST, int TY>
__global__ void __launch_bounds__(128)
rk_stage_kernel(const __grid_constant__ StageArgs<T, Tp> A) {
    rk_stage_body<T, Tp, PER, FIRST, LAST, TY>(A, (int)blockIdx.x);
}

// ===========================================================================
// TMA-fed variant.  Persistent blocks of 4 consumer warps (one 28-column strip
// each: a 112-column band) and 1 producer warp.  The producer takes tiles
// (band x TY rows) from a global counter and copies, for every K-row chunk of
// a tile, the stage input (120 columns: the band plus a 4-column halo on each
// side, from device column cx0) and the point-wise operands X, X0 (the band's
// 112 columns) into a ring of S shared-memory slots, with the tile number in
// the slot's metadata; consumers run the same row recurrence as
// rk_stage_kernel reading their column from the slot.  Chunk j of a tile
// holds rows y0-2+jK .. y0-2+jK+K-1 of every field; iteration r = y0-2+i
// reads input row r+1 (index i+1) and X/X0 row r (index i).
constexpr int BAND = 4 * STRIP;      // output columns per block
constexpr int BOXW_IN = BAND + 8;    // input box width
constexpr int BOXW_X = BAND;         // X/X0 box width

struct StageMaps {
    CUtensorMap in_u, in_v, in_e;    // stage input X1, box BOXW_IN x K
    CUtensorMap x_u, x_v, x_e;       // state X, box BOXW_X x K
    CUtensorMap a_u, a_v, a_e;       // accumulator X0, box BOXW_X x K
};

// tile scheduler shared by the stage launches of a context (reset by the last
// producer of each launch)
struct TileSched {
    int next;
    int done;
};

template <class Tp, bool FIRST, bool LAST, int K>
struct StageSlot {
    static constexpr bool LOAD_X = !FIRST && !LAST;   // X read for the b update
    static constexpr bool LOAD_A = !FIRST;            // X0 read for the a update
    // each box region starts on a 128-byte boundary; the copies fill K rows of
    // the box width densely and the rest of a region is padding
    static constexpr int ALIGN = int(128 / sizeof(Tp));
    static constexpr int IN = (K * BOXW_IN + ALIGN - 1) / ALIGN * ALIGN;    // region strides (elements)
    static constexpr int XE = (K * BOXW_X + ALIGN - 1) / ALIGN * ALIGN;
    static constexpr int NX = (LOAD_X ? 3 : 0) + (LOAD_A ? 3 : 0);
    static constexpr int ELEMS = 3 * IN + NX * XE;                          // slot stride (elements)
    static constexpr uint32_t BYTES = ELEMS * sizeof(Tp);                   // slot size
    static constexpr uint32_t TX_BYTES = (3 * K * BOXW_IN + NX * K * BOXW_X) * sizeof(Tp);   // bytes copied
    static constexpr int U = 0, V = IN, E = 2 * IN;
    static constexpr int XU = 3 * IN, XV = XU + XE, XW = XV + XE;
    static constexpr int AU = 3 * IN + (LOAD_X ? 3 * XE : 0), AV = AU + XE, AW = AV + XE;
    static_assert((IN * sizeof(Tp)) % 128 == 0 && (XE * sizeof(Tp)) % 128 == 0, "TMA destinations need 128-B alignment");
};

template <class T, class Tp, bool FIRST, bool LAST, int K, int S>
__host__ __device__ constexpr int stage_tma_smem() {
    return S * StageSlot<Tp, FIRST, LAST, K>::BYTES + 2 * S * 8 + S * 4;
}

#ifndef SWB_TMA_UNROLL
#define SWB_TMA_UNROLL 2        // row-loop unroll of interior warps (code size vs. scheduling)
#endif
#ifndef SWB_TMA_UNROLL_EDGE
#define SWB_TMA_UNROLL_EDGE 1   // edge warps are few: keep their code small
#endif
constexpr int TMA_UNROLL = SWB_TMA_UNROLL, TMA_UNROLL_EDGE = SWB_TMA_UNROLL_EDGE;
// One tile (band x TY rows) of the consumer warps of rk_stage_tma.  EDGE is
// false for warps none of whose output cells is near a boundary: then every
// output lane writes, nothing is a ghost source and the row loop is unrolled.
// Returns false if a wait timed out.
template <class T, class Tp, bool PER, bool FIRST, bool LAST, int TY, int K, int S, bool EDGE, bool ROWF>
__device__ __forceinline__ bool stage_tile(const StageArgs<T, Tp>& A, const Tp* ring, uint64_t* full, uint64_t* empty,
                                           uint32_t gbase, int cx0, int y0, int warp, int lane) {
    using SL = StageSlot<Tp, FIRST, LAST, K>;
    constexpr int NCH = (TY + 3 + K - 1) / K;
    const Geom& g = A.g;
    const int N = g.N, M = g.M;
    const T half = T(0.5), o12 = T(1.0 / 12.0);
    const int P = g.P;
    const int sc_in = warp * STRIP + lane + 2;     // column inside the input box
    const int sc_x = warp * STRIP + lane - 2;      // column inside the X/X0 box (output lanes)
    const bool out_lane = lane >= 2 && lane < 2 + STRIP;
    const int Hsy = A.H.sy, fqsy = A.fq.sy, Fxsy = A.Fx.sy, Fysy = A.Fy.sy;
    const int c = cx0 + warp * STRIP + lane - 2;
    const bool col_u = EDGE ? out_lane && c >= (PER ? 0 : 1) && c < N : out_lane;
    const bool col_a = EDGE ? out_lane && c >= 0 && c < N : out_lane;
    const bool gx_u = EDGE && PER && (c <= 1 || c >= N - 2);
    const bool gx_v = EDGE && (c <= 1 || c >= N - 2);
    const bool gx_e = EDGE && (c == 0 || c == N - 1);
    const bool wrap = EDGE && PER && c == -1;
    const bool qc_wrap = EDGE && PER && c == 0;
    const int cb = c + COL0;

    auto slot_ptr = [&](int j) { return ring + ((gbase + j) % S) * SL::ELEMS; };
    auto wait_chunk = [&](int j) { return mbar_wait(&full[(gbase + j) % S], ((gbase + j) / S) & 1, A.st, A.spin_limit); };
    auto release = [&](int j) {
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[(gbase + j) % S]);
    };

    // static fields.  ROWF (all four constant along x): lane k holds row
    // y0-2+k of each, broadcast to the row being computed by warp shuffles.
    // Otherwise lane pointers at the row of first use, one row ahead in registers.
    int r = y0 - 2;
    static_assert(TY + 3 <= 32, "a tile's static rows must fit in one warp");
    T tH = T(0), tfq = T(0), tFx = T(0), tFy = T(0);
    if (ROWF) {
        const int ry = y0 - 2 + (lane < TY + 3 ? lane : TY + 2) + ROW0;
        tH = A.H.p[ry * Hsy]; tfq = A.fq.p[ry * fqsy]; tFx = A.Fx.p[ry * Fxsy]; tFy = A.Fy.p[ry * Fysy];
    }
    const T* __restrict__ pH = A.H.p + (r + 1 + ROW0) * Hsy + cb * A.H.sx;
    const T* __restrict__ pfq = A.fq.p + (r + 1 + ROW0) * fqsy + cb * A.fq.sx;
    const T* __restrict__ pFx = A.Fx.p + (r + ROW0) * Fxsy + cb * A.Fx.sx;
    const T* __restrict__ pFy = A.Fy.p + (r + ROW0) * Fysy + cb * A.Fy.sx;
    T nH = T(0), nfq = T(0), nFx = T(0), nFy = T(0);
    if (!ROWF) { nH = *pH; nfq = *pfq; nFx = *pFx; nFy = *pFy; }

    const Tp* pin = slot_ptr(0) + sc_in;        // input row 0 of the tile
    T u_r = cvt<T>(pin[SL::U]), v_r = cvt<T>(pin[SL::V]), e_r = cvt<T>(pin[SL::E]);
    Tp Xu_r = pin[SL::U], Xv_r = pin[SL::V], Xe_r = pin[SL::E];   // raw row r (X of the first stage)
    T h_r = e_r + (ROWF ? __shfl_sync(0xffffffffu, tH, 0) : A.H.at(c, r));
    T hl_r = shup(h_r), ur_r = shdn(u_r);
    T U_r = u_r * (half * (h_r + hl_r));
    T Ur_r = shdn(U_r);
    T V_r = T(0), Vl_r = T(0), q_r = T(0), ql_r = T(0), qr_r = T(0);
    T p_rm1 = T(0), qhu_part = T(0);
    T uN_r = T(0), hN_r = T(0), hNm1_r = T(0);
    if (wrap) {
        uN_r = cvt<T>(A.u1[g.idx(N, r)]);
        hN_r = cvt<T>(A.e1[g.idx(N, r)]) + A.H.at(N, r);
        hNm1_r = cvt<T>(A.e1[g.idx(N - 1, r)]) + A.H.at(N - 1, r);
    }
    const Tp* px = slot_ptr(0) + sc_x;          // X/X0 row 0 of the tile
    int nrel = 0;

#pragma unroll (EDGE ? TMA_UNROLL_EDGE : TMA_UNROLL)
    for (int i = 0; i < TY + 2; i++, r++) {
        // next input row (index i+1): new slot at a chunk boundary
        const int kin = i + 1;
        if (kin % K == 0) {
            if (!wait_chunk(kin / K)) return false;
            pin = slot_ptr(kin / K) + sc_in;
        } else {
            pin += BOXW_IN;
        }
        const Tp rawu = pin[SL::U], rawv = pin[SL::V], rawe = pin[SL::E];
        T fq, H1, Fxr, Fyr;
        if (ROWF) {          // rows r+1 (H, f_q) and r (Fx, Fy) of the tile's lane table
            fq = __shfl_sync(0xffffffffu, tfq, i + 1); H1 = __shfl_sync(0xffffffffu, tH, i + 1);
            Fxr = __shfl_sync(0xffffffffu, tFx, i); Fyr = __shfl_sync(0xffffffffu, tFy, i);
        } else {
            fq = nfq; H1 = nH; Fxr = nFx; Fyr = nFy;
            pH += Hsy; pfq += fqsy; pFx += Fxsy; pFy += Fysy;
            nH = *pH; nfq = *pfq; nFx = *pFx; nFy = *pFy;
        }
        // X/X0 row (index i)
        if (i > 0) {
            if (i % K == 0) px = slot_ptr(i / K) + sc_x;
            else px += BOXW_X;
        }

        const T u_r1 = cvt<T>(rawu), v_r1 = cvt<T>(rawv), e_r1 = cvt<T>(rawe);
        const T h_r1 = e_r1 + H1;                                 // thickness! (src/rhs.jl:131-139)
        const T hl_r1 = shup(h_r1), vl_r1 = shup(v_r1), ur_r1 = shdn(u_r1);

        T q_r1;
        T uN_r1 = T(0), hN_r1 = T(0), hNm1_r1 = T(0);
        if (wrap) {
            uN_r1 = cvt<T>(A.u1[g.idx(N, r + 1)]);
            hN_r1 = cvt<T>(A.e1[g.idx(N, r + 1)]) + A.H.at(N, r + 1);
            hNm1_r1 = cvt<T>(A.e1[g.idx(N - 1, r + 1)]) + A.H.at(N - 1, r + 1);
            const T vN = cvt<T>(A.v1[g.idx(N, r + 1)]), vNm1 = cvt<T>(A.v1[g.idx(N - 1, r + 1)]);
            q_r1 = pv_q<T>(fq, vN, vNm1, uN_r1, uN_r, hNm1_r, hN_r, hNm1_r1, hN_r1);
        } else {
            q_r1 = pv_q<T>(fq, v_r1, vl_r1, u_r1, u_r, hl_r, h_r, hl_r1, h_r1);
        }
        const T ql_r1 = shup(q_r1), qr_r1 = shdn(q_r1);
        const T U_r1 = u_r1 * (half * (h_r1 + hl_r1));
        const T V_r1 = v_r1 * (half * (h_r1 + h_r));
        const T Ur_r1 = shdn(U_r1), Vl_r1 = shup(V_r1);
        const T KEu = half * (ur_r * ur_r + u_r * u_r);
        const T KEv = half * (v_r1 * v_r1 + v_r * v_r);
        const T p_r = half * (KEu + KEv) + A.g_ * e_r;
        const T pl_r = shup(p_r);
        const T s = q_r + q_r1;
        const T qa = o12 * (s + qr_r1);
        const T qb = o12 * (s + ql_r1);
        const T qc = qc_wrap ? o12 * (s + ql_r) : o12 * (q_r + ql_r + q_r1);
        const T qd = o12 * (s + qr_r);
        const T qbr = shdn(qb), qcr = shdn(qc);

        if (i >= 2 && (!EDGE || r < M)) {
            const int o = (r + ROW0) * P + cb;
            if (col_u) {
                const T qhv = qa * V_r1 + qb * Vl_r1 + qc * Vl_r + qd * V_r;
                const T dpdx = p_r - pl_r;
                const Tp du = (cvt<Tp>(qhv) - cvt<Tp>(dpdx)) + cvt<Tp>(A.Fxt * Fxr);
                const Tp X = FIRST ? Xu_r : (SL::LOAD_X ? px[SL::XU] : Tp(0));
                const bool gs = EDGE && (gx_u || (!PER && (r <= 1 || r >= M - 2)));
                if (!LAST) {
                    const Tp x1 = X + A.b * du;
                    A.u1o[o] = x1;
                    if (gs) A.gr.u(A.u1o, g, c, r, x1);
                }
                const Tp x0 = (FIRST ? X : px[SL::AU]) + A.a * du;
                A.u0o[o] = x0;
                if (LAST && gs) A.gr.u(A.u0o, g, c, r, x0);
            }
            if (col_a) {
                if (!EDGE || r >= 1) {
                    const T qhu = qhu_part + qcr * Ur_r + qd * U_r;
                    const T dpdy = p_r - p_rm1;
                    const Tp dv = -(cvt<Tp>(qhu) + cvt<Tp>(dpdy)) + cvt<Tp>(A.Fyt * Fyr);
                    const Tp X = FIRST ? Xv_r : (SL::LOAD_X ? px[SL::XV] : Tp(0));
                    if (!LAST) {
                        const Tp x1 = X + A.b * dv;
                        A.v1o[o] = x1;
                        if (gx_v) A.gr.v(A.v1o, g, c, r, x1);
                    }
                    const Tp x0 = (FIRST ? X : px[SL::AV]) + A.a * dv;
                    A.v0o[o] = x0;
                    if (LAST && gx_v) A.gr.v(A.v0o, g, c, r, x0);
                }
                const T dUdx = Ur_r - U_r;
                const T dVdy = V_r1 - V_r;
                const Tp de = -(cvt<Tp>(dUdx) + cvt<Tp>(dVdy));
                const Tp X = FIRST ? Xe_r : (SL::LOAD_X ? px[SL::XW] : Tp(0));
                const bool gs = EDGE && (gx_e || r == 0 || r == M - 1);
                if (!LAST) {
                    const Tp x1 = X + A.b * de;
                    A.e1o[o] = x1;
                    if (gs) A.gr.eta(A.e1o, g, c, r, x1);
                }
                const Tp x0 = (FIRST ? X : px[SL::AW]) + A.a * de;
                A.e0o[o] = x0;
                if (LAST && gs) A.gr.eta(A.e0o, g, c, r, x0);
            }
        }
        // chunk i/K is done once its last X row (and so all its input rows) was used
        if (i % K == K - 1) { release(i / K); nrel++; }

        qhu_part = qa * U_r + qbr * Ur_r;
        u_r = u_r1; v_r = v_r1; e_r = e_r1; h_r = h_r1; hl_r = hl_r1; ur_r = ur_r1;
        q_r = q_r1; ql_r = ql_r1; qr_r = qr_r1;
        U_r = U_r1; Ur_r = Ur_r1;
        V_r = V_r1; Vl_r = Vl_r1;
        p_rm1 = p_r;
        uN_r = uN_r1; hN_r = hN_r1; hNm1_r = hNm1_r1;
        Xu_r = rawu; Xv_r = rawv; Xe_r = rawe;
    }
    for (int j = nrel; j < NCH; j++) release(j);
    return true;
}

#ifndef SWB_TMA_MINB
#define SWB_TMA_MINB 6     // resident blocks per SM the register budget is sized for
#endif
template <class T, class Tp, bool PER, bool FIRST, bool LAST, int TY, int K, int S, bool ROWF>
__global__ void __launch_bounds__(160, SWB_TMA_MINB)
rk_stage_tma(const __grid_constant__ StageArgs<T, Tp> A, const __grid_constant__ StageMaps MP, int npersist,
             TileSched* sched) {
    using SL = StageSlot<Tp, FIRST, LAST, K>;
    if ((int)blockIdx.x >= npersist) {
        if (A.st->stop) return;
        const int rb = (int)blockIdx.x - npersist;
        stage_ring(A, FIRST, LAST, rb * 160 + threadIdx.x, ((int)gridDim.x - npersist) * 160);
        return;
    }
    extern __shared__ __align__(128) unsigned char smem_raw[];
    Tp* ring = reinterpret_cast<Tp*>(smem_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + S * SL::BYTES);
    uint64_t* empty = full + S;
    int* slot_tile = reinterpret_cast<int*>(empty + S);

    const Geom& g = A.g;
    const int N = g.N, M = g.M;
    const int nbx = (N + BAND - 1) / BAND, nby = (M + TY - 1) / TY, ntiles = nbx * nby;
    constexpr int NCH = (TY + 3 + K - 1) / K;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    __shared__ int stop_flag;
    if (threadIdx.x == 0) {
        stop_flag = A.st->stop;
        for (int s = 0; s < S; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 4);
        }
        fence_mbar_init();
    }
    __syncthreads();
    if (stop_flag) return;      // block-uniform

    if (warp == 4) {
        // ------------------------------------------------------------ producer
        if (lane != 0) return;
        uint32_t gc = 0;
        bool ok = true;
        auto acquire = [&](int slot) {
            return gc < (uint32_t)S || mbar_wait(&empty[slot], ((gc / S) - 1) & 1, A.st, A.spin_limit);
        };
        bool first_tile = true;
        for (;;) {
            const int t = atomicAdd(&sched->next, 1);
            const int slot0 = gc % S;
            if (t >= ntiles) {
                // end marker: a slot with tile -1 and no copies
                if (acquire(slot0)) {
                    slot_tile[slot0] = -1;
                    mbar_arrive(&full[slot0]);
                    gc++;
                } else {
                    ok = false;
                }
                break;
            }
            const int cx0 = (t % nbx) * BAND, y0 = (t / nbx) * TY;
            for (int j = 0; j < NCH; j++, gc++) {
                const int slot = gc % S;
                if (!acquire(slot)) { ok = false; break; }
                if (first_tile && j == A.skip_chunk && blockIdx.x == 0) continue;   // test only: never filled
                slot_tile[slot] = t;
                mbar_arrive_expect_tx(&full[slot], SL::TX_BYTES);
                Tp* b = ring + slot * SL::ELEMS;
                const int yd = y0 - 2 + j * K + ROW0;
                tma_load_2d(b + SL::U, &MP.in_u, cx0, yd, &full[slot]);
                tma_load_2d(b + SL::V, &MP.in_v, cx0, yd, &full[slot]);
                tma_load_2d(b + SL::E, &MP.in_e, cx0, yd, &full[slot]);
                if (SL::LOAD_X) {
                    tma_load_2d(b + SL::XU, &MP.x_u, cx0 + COL0, yd, &full[slot]);
                    tma_load_2d(b + SL::XV, &MP.x_v, cx0 + COL0, yd, &full[slot]);
                    tma_load_2d(b + SL::XW, &MP.x_e, cx0 + COL0, yd, &full[slot]);
                }
                if (SL::LOAD_A) {
                    tma_load_2d(b + SL::AU, &MP.a_u, cx0 + COL0, yd, &full[slot]);
                    tma_load_2d(b + SL::AV, &MP.a_v, cx0 + COL0, yd, &full[slot]);
                    tma_load_2d(b + SL::AW, &MP.a_e, cx0 + COL0, yd, &full[slot]);
                }
            }
            if (!ok) break;
            first_tile = false;
        }
        // all issued copies must land before the block may exit
        for (uint32_t q = (gc >= (uint32_t)S ? gc - S : 0); q < gc; q++)
            mbar_wait(&full[q % S], (q / S) & 1, A.st, A.spin_limit);
        // the last producer of the launch resets the scheduler for the next one
        if (atomicAdd(&sched->done, 1) == npersist - 1) {
            sched->next = 0;
            sched->done = 0;
        }
        (void)ok;
        return;
    }

    // -------------------------------------------------------------- consumers
    for (uint32_t gbase = 0;; gbase += NCH) {
        if (!mbar_wait(&full[gbase % S], (gbase / S) & 1, A.st, A.spin_limit)) return;
        const int t = slot_tile[gbase % S];
        if (t < 0) return;
        const int cx0 = (t % nbx) * BAND, y0 = (t / nbx) * TY;
        // Warp-uniform: does any output cell of this warp need edge handling
        // (ghost sources, the periodic q wrap, columns beyond N, rows near the
        // y boundaries)?  Interior warps run without any of those tests.
        const int cw = cx0 + warp * STRIP;               // column of output lane 2
        const bool edge = cw <= 1 || cw + STRIP - 1 >= N - 2 || y0 <= 1 || y0 + TY - 1 >= M - 2;
        const bool ok = edge ? stage_tile<T, Tp, PER, FIRST, LAST, TY, K, S, true, ROWF>(A, ring, full, empty, gbase, cx0, y0, warp, lane)
                             : stage_tile<T, Tp, PER, FIRST, LAST, TY, K, S, false, ROWF>(A, ring, full, empty, gbase, cx0, y0, warp, lane);
        if (!ok) return;
    }
}

}  // namespace swb
