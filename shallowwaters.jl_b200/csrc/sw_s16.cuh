// sw_s16.cuh -- the 16-bit storage form of the time loop (sw_config.storage =
// SW_STORE_BF16 or SW_STORE_F16; no counterpart in the reference, whose own
// storage/compute split is the T/Tprog conversion of
// src/time_integration.jl:330-347).
//
// Every array the time loop keeps in HBM holds 16-bit numbers (bfloat16 or
// IEEE half) scaled by a power of two s (sw_config.storage_scale_uv, for u,
// v and eta alike; the tracer is unscaled):
//   state   u, v, eta as compensated pairs hi + lo: hi = round16(s*x),
//           lo = round16(s*x - hi).  lo is the Kahan compensation term: it
//           keeps the rounding error of hi, so increments far below one unit
//           in the last place of hi still accumulate from step to step.
//   δ       the stage increment b_k*dt*d_k: the input of stage k+1 is
//           X1 = (hi + lo) + δ, formed in FP32 (the increment is small against
//           the state, so its 16 bits cost the stage input almost nothing)
//   D       the RK increment accumulated so far, sum of a_k*dt*d_k
//   sst     one 16-bit number
// Tendencies, the stage combination and the tail are computed in FP32 from
// those values.  The last stage forms X0 = (hi + lo) + (D + a_4*dt*d_4) in
// FP32: u and v (and eta, for the depth of the quadratic drag) go to FP32
// buffers that the tail reads once and turns into the new pairs; eta goes to
// its new pair directly.  Bytes per cell and step (RK4, tail and tracer every
// step, static fields counted as full FP32 fields like in the FP32 count):
//   stage 1  32   stages 2, 3  44 each   stage 4  48   tail 24   tracer 8
// 200 bytes against the 264 of plain Float32.
//
// Execution follows the streaming stage kernel of sw_stage.cuh (one warp per
// 28-column strip, rows streamed upward with a register window and warp
// shuffles for x-neighbours), in the reference's operation order, with
// Arakawa-Hsu PV advection and the plain continuity equation.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "sw_common.cuh"
#include "sw_ghost.cuh"
#include "sw_stage.cuh"
#include "sw_storage.cuh"
#include "sw_tail.cuh"
#include "sw_tracer.cuh"

namespace swb {

// value <-> scaled 16-bit number
template <class S16>
struct Put16 {
    float s;
    __device__ __forceinline__ S16 operator()(float x) const { return to16<S16>(x * s); }
};
// the compensation half of a pair: round16(s*x - round16(s*x))
template <class S16>
struct PutLo16 {
    float s;
    __device__ __forceinline__ S16 operator()(float x) const {
        const float y = x * s;
        return to16<S16>(y - from16(to16<S16>(y)));
    }
};

template <class S16>
struct S16StageArgs {
    Geom g;
    int nsx, nsy, nring_blocks;
    const S16* uh; const S16* vh; const S16* eh;   // state hi
    const S16* ul; const S16* vl; const S16* el;   // state lo
    const S16* ud; const S16* vd; const S16* ed;   // stage increment δ in (not read by the first stage)
    const S16* uD; const S16* vD; const S16* eD;   // accumulated increment D in (not read by the first stage)
    S16* udo; S16* vdo; S16* edo;                  // δ out, with ghost copies (not the last stage)
    S16* uDo; S16* vDo; S16* eDo;                  // D out (not the last stage)
    float* u0o; float* v0o; float* e0o;            // last stage: X0 in FP32, with ghost copies
    S16* eho; S16* elo;                            // last stage: the new eta pair, with ghost copies
    SField<float> H, fq, Fx, Fy;
    float a, b;                                    // RKaΔt[k], RKbΔt[k]
    float g_, Fxt, Fyt;
    float s, inv_s;
    GhostRule<float> gr;
    DevStatus* st;
};

template <class S16>
__device__ __forceinline__ float ld16(const S16* p, int k, float inv_s) { return from16(p[k]) * inv_s; }

// untouched halo cells of u and v: δ' = 0 (X1 = X), D' = D, X0 = X + D
template <class S16, bool FIRST, bool LAST>
__device__ void s16_stage_ring(const S16StageArgs<S16>& A, int k0, int kstride) {
    const Geom& g = A.g;
    const int nu = Ring::u_count(g.ep, g.N, g.M), nv = Ring::v_count(g.N);
    const Put16<S16> put{A.s};
    for (int k = k0; k < nu + nv; k += kstride) {
        const bool isu = k < nu;
        int x, y;
        if (isu) Ring::u_at(k, g.ep, g.N, g.M, x, y);
        else Ring::v_at(k - nu, g.N, g.M, x, y);
        const int gi = g.idx(x, y);
        if (!LAST) {
            S16* od = isu ? A.udo : A.vdo;
            S16* oD = isu ? A.uDo : A.vDo;
            od[gi] = to16<S16>(0.f);
            oD[gi] = FIRST ? to16<S16>(0.f) : (isu ? A.uD : A.vD)[gi];
            if (isu) A.gr.u(od, g, x, y, 0.f, put);
            else A.gr.v(od, g, x, y, 0.f, put);
        } else {
            const S16* ph = isu ? A.uh : A.vh;
            const S16* pl = isu ? A.ul : A.vl;
            const S16* pD = isu ? A.uD : A.vD;
            const float x0 = (from16(ph[gi]) + from16(pl[gi])) * A.inv_s + from16(pD[gi]) * A.inv_s;
            float* o0 = isu ? A.u0o : A.v0o;
            o0[gi] = x0;
            if (isu) A.gr.u(o0, g, x, y, x0);
            else A.gr.v(o0, g, x, y, x0);
        }
    }
}

// One RK stage of the 16-bit form (nonlinear, Arakawa-Hsu, plain continuity),
// block bx of (nsx * nsy + 3) / 4 strip blocks and nring_blocks ring blocks.
template <class S16, bool PER, bool FIRST, bool LAST, int TY>
__device__ __forceinline__ void s16_stage_body(const S16StageArgs<S16>& A, int bx) {
    if (A.st->stop) return;
    const Geom& g = A.g;
    const int nstrips = A.nsx * A.nsy;
    const int nstrip_blocks = (nstrips + 3) / 4;
    if (bx >= nstrip_blocks) {
        s16_stage_ring<S16, FIRST, LAST>(A, (bx - nstrip_blocks) * 128 + threadIdx.x, A.nring_blocks * 128);
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
    const bool gx_e = c == 0 || c == N - 1;
    const bool wrap = PER && c == -1;
    const float half = 0.5f, o12 = float(1.0 / 12.0), inv = A.inv_s;
    const Put16<S16> put{A.s};
    const PutLo16<S16> putlo{A.s};

    const int cb = c + COL0;
    const S16* __restrict__ ph[3] = {A.uh + cb, A.vh + cb, A.eh + cb};
    const S16* __restrict__ pl[3] = {A.ul + cb, A.vl + cb, A.el + cb};
    const S16* __restrict__ pd[3] = {A.ud + cb, A.vd + cb, A.ed + cb};
    const S16* __restrict__ pD[3] = {A.uD + cb, A.vD + cb, A.eD + cb};
    const int Hsy = A.H.sy;
    const float* __restrict__ pH = A.H.p + cb * A.H.sx;
    const float* __restrict__ pfq = A.fq.p + cb * A.fq.sx;
    const int fqsy = A.fq.sy;
    auto row = [&](int y) { return (y + ROW0) * P; };
    // the state (hi + lo) and the stage input X1 = state + δ of field f at offset k
    struct In { S16 h, l, d; };
    auto fetch = [&](int f, int k) {
        In v;
        v.h = ph[f][k];
        v.l = pl[f][k];
        v.d = FIRST ? to16<S16>(0.f) : pd[f][k];
        return v;
    };
    auto state = [&](const In& v) { return (from16(v.h) + from16(v.l)) * inv; };
    auto stage_in = [&](const In& v) { return FIRST ? state(v) : state(v) + from16(v.d) * inv; };
    // the same at a column of its own (the periodic q wrap)
    auto at_col = [&](int f, int x, int y) {
        const S16* hh = f == 0 ? A.uh : f == 1 ? A.vh : A.eh;
        const S16* ll = f == 0 ? A.ul : f == 1 ? A.vl : A.el;
        const S16* dd = f == 0 ? A.ud : f == 1 ? A.vd : A.ed;
        const int k = g.idx(x, y);
        const float xs = (from16(hh[k]) + from16(ll[k])) * inv;
        return FIRST ? xs : xs + from16(dd[k]) * inv;
    };

    int r = y0 - 2;
    In cu = fetch(0, row(r)), cv = fetch(1, row(r)), ce = fetch(2, row(r));
    float u_r = stage_in(cu), v_r = stage_in(cv), e_r = stage_in(ce);
    float us_r = state(cu), vs_r = state(cv), es_r = state(ce);     // the state itself (last stage's X0)
    float h_r = e_r + pH[(r + ROW0) * Hsy];
    float hl_r = shup(h_r), ur_r = shdn(u_r);
    float U_r = u_r * (half * (h_r + hl_r));
    float Ur_r = shdn(U_r);
    float V_r = 0.f, Vl_r = 0.f, q_r = 0.f, ql_r = 0.f, qr_r = 0.f;
    float p_rm1 = 0.f, qhu_part = 0.f;
    float uN_r = 0.f, hN_r = 0.f, hNm1_r = 0.f;
    if (wrap) {
        uN_r = at_col(0, N, r);
        hN_r = at_col(2, N, r) + A.H.at(N, r);
        hNm1_r = at_col(2, N - 1, r) + A.H.at(N - 1, r);
    }
    // software pipeline: the next input row one iteration ahead, and the
    // output row's accumulated increment D
    In nu = fetch(0, row(r + 1)), nv = fetch(1, row(r + 1)), ne = fetch(2, row(r + 1));
    float nH = pH[(r + 1 + ROW0) * Hsy];
    S16 nD[3];
#pragma unroll
    for (int f = 0; f < 3; f++) nD[f] = to16<S16>(0.f);
    auto load_D = [&](int y) {
        if constexpr (!FIRST) {
            if (y >= y0 && out_lane) {
#pragma unroll
                for (int f = 0; f < 3; f++) nD[f] = pD[f][row(y)];
            }
        }
    };
    load_D(r);

    for (; r < y0 + TY; r++) {
        const float u_r1 = stage_in(nu), v_r1 = stage_in(nv), e_r1 = stage_in(ne);
        const float us_r1 = LAST ? state(nu) : 0.f, vs_r1 = LAST ? state(nv) : 0.f, es_r1 = LAST ? state(ne) : 0.f;
        const float h_r1 = e_r1 + nH;
        {
            const int o2 = row(r + 2);
            nu = fetch(0, o2); nv = fetch(1, o2); ne = fetch(2, o2);
            nH = pH[(r + 2 + ROW0) * Hsy];
        }
        S16 cD[3];
#pragma unroll
        for (int f = 0; f < 3; f++) cD[f] = nD[f];
        load_D(r + 1);
        const float hl_r1 = shup(h_r1), vl_r1 = shup(v_r1), ur_r1 = shdn(u_r1);
        float q_r1;
        const float fq = pfq[(r + 1 + ROW0) * fqsy];
        float uN_r1 = 0.f, hN_r1 = 0.f, hNm1_r1 = 0.f;
        if (wrap) {
            uN_r1 = at_col(0, N, r + 1);
            hN_r1 = at_col(2, N, r + 1) + A.H.at(N, r + 1);
            hNm1_r1 = at_col(2, N - 1, r + 1) + A.H.at(N - 1, r + 1);
            const float vN = at_col(1, N, r + 1), vNm1 = at_col(1, N - 1, r + 1);
            q_r1 = pv_q<float>(fq, vN, vNm1, uN_r1, uN_r, hNm1_r, hN_r, hNm1_r1, hN_r1);
        } else {
            q_r1 = pv_q<float>(fq, v_r1, vl_r1, u_r1, u_r, hl_r, h_r, hl_r1, h_r1);
        }
        const float ql_r1 = shup(q_r1), qr_r1 = shdn(q_r1);
        const float U_r1 = u_r1 * (half * (h_r1 + hl_r1));
        const float V_r1 = v_r1 * (half * (h_r1 + h_r));
        const float Ur_r1 = shdn(U_r1), Vl_r1 = shup(V_r1);
        const float KEu = half * (ur_r * ur_r + u_r * u_r);
        const float KEv = half * (v_r1 * v_r1 + v_r * v_r);
        const float p_r = half * (KEu + KEv) + A.g_ * e_r;
        const float pl_r = shup(p_r);
        const float s = q_r + q_r1;
        const float qa = o12 * (s + qr_r1);
        const float qb = o12 * (s + ql_r1);
        const float qc = (PER && c == 0) ? o12 * (s + ql_r) : o12 * (q_r + ql_r + q_r1);
        const float qd = o12 * (s + qr_r);
        const float qbr = shdn(qb), qcr = shdn(qc);

        if (r >= y0 && r < M) {
            const int o = row(r) + cb;
            // D' = D + a d (the first stage starts from 0); the last stage's X0 = state + D'
            auto incr = [&](int f, float d) { return (FIRST ? 0.f : from16(cD[f]) * inv) + A.a * d; };
            if (col_u) {
                const float qhv = qa * V_r1 + qb * Vl_r1 + qc * Vl_r + qd * V_r;
                const float dpdx = p_r - pl_r;
                const float du = (qhv - dpdx) + A.Fxt * A.Fx.at(c, r);
                const bool gs = gx_u || (!PER && (r <= 1 || r >= M - 2));
                const float dD = incr(0, du);
                if (!LAST) {
                    const float dl = A.b * du;                   // δ' : X1' = X + b d
                    A.udo[o] = put(dl);
                    if (gs) A.gr.u(A.udo, g, c, r, dl, put);
                    A.uDo[o] = put(dD);
                } else {
                    const float x0 = us_r + dD;
                    A.u0o[o] = x0;
                    if (gs) A.gr.u(A.u0o, g, c, r, x0);
                }
            }
            if (col_a) {
                if (r >= 1) {
                    const float qhu = qhu_part + qcr * Ur_r + qd * U_r;
                    const float dpdy = p_r - p_rm1;
                    const float dv = -(qhu + dpdy) + A.Fyt * A.Fy.at(c, r);
                    const float dD = incr(1, dv);
                    if (!LAST) {
                        const float dl = A.b * dv;
                        A.vdo[o] = put(dl);
                        if (gx_v) A.gr.v(A.vdo, g, c, r, dl, put);
                        A.vDo[o] = put(dD);
                    } else {
                        const float x0 = vs_r + dD;
                        A.v0o[o] = x0;
                        if (gx_v) A.gr.v(A.v0o, g, c, r, x0);
                    }
                }
                const float dUdx = Ur_r - U_r;
                const float dVdy = V_r1 - V_r;
                const float de = -(dUdx + dVdy);
                const bool gs = gx_e || r == 0 || r == M - 1;
                const float dD = incr(2, de);
                if (!LAST) {
                    const float dl = A.b * de;
                    A.edo[o] = put(dl);
                    if (gs) A.gr.eta(A.edo, g, c, r, dl, put);
                    A.eDo[o] = put(dD);
                } else {
                    const float x0 = es_r + dD;
                    A.e0o[o] = x0;
                    A.eho[o] = put(x0);
                    A.elo[o] = putlo(x0);
                    if (gs) {
                        A.gr.eta(A.e0o, g, c, r, x0);
                        A.gr.eta(A.eho, g, c, r, x0, put);
                        A.gr.eta(A.elo, g, c, r, x0, putlo);
                    }
                }
            }
        }
        qhu_part = qa * U_r + qbr * Ur_r;
        u_r = u_r1; v_r = v_r1; e_r = e_r1; h_r = h_r1; hl_r = hl_r1; ur_r = ur_r1;
        us_r = us_r1; vs_r = vs_r1; es_r = es_r1;
        q_r = q_r1; ql_r = ql_r1; qr_r = qr_r1;
        U_r = U_r1; Ur_r = Ur_r1;
        V_r = V_r1; Vl_r = Vl_r1;
        p_rm1 = p_r;
        uN_r = uN_r1; hN_r = hN_r1; hNm1_r = hNm1_r1;
    }
}

template <class S16, bool PER, bool FIRST, bool LAST, int TY>
__global__ void __launch_bounds__(128)
s16_stage_kernel(const __grid_constant__ S16StageArgs<S16> A) {
    s16_stage_body<S16, PER, FIRST, LAST, TY>(A, (int)blockIdx.x);
}

// The tail's new u, v as pairs (hi, lo), with the ghost copies of both.
template <class S16>
struct TailStorePair {
    S16* uh; S16* ul; S16* vh; S16* vl;
    float s;
    template <class Args>
    __device__ __forceinline__ void u(const Args& A, const Geom& g, int F, int b, int o, float val, bool gs) const {
        const Put16<S16> hi{s};
        const PutLo16<S16> lo{s};
        uh[o] = hi(val);
        ul[o] = lo(val);
        if (gs) {
            A.gr.u(uh, g, F, b, val, hi);
            A.gr.u(ul, g, F, b, val, lo);
        }
    }
    template <class Args>
    __device__ __forceinline__ void v(const Args& A, const Geom& g, int a, int G, int o, float val, bool gs) const {
        const Put16<S16> hi{s};
        const PutLo16<S16> lo{s};
        vh[o] = hi(val);
        vl[o] = lo(val);
        if (gs) {
            A.gr.v(vh, g, a, G, val, hi);
            A.gr.v(vl, g, a, G, val, lo);
        }
    }
};

template <class S16, bool PER, int DRAG, bool SMAG, int TY>
__global__ void __launch_bounds__(128)
s16_tail_kernel(const __grid_constant__ TailArgs<float, float> A, const __grid_constant__ TailStorePair<S16> out) {
    tail_body<float, float, PER, DRAG, SMAG, TY>(A, (int)blockIdx.x, out);
}

// The tracer reading u, v (hi) and sst as scaled 16-bit numbers.
template <class S16>
struct TracerIO16 {
    using EU = S16;
    using ES = S16;
    float inv_s;
    __device__ __forceinline__ float u(EU x) const { return from16(x) * inv_s; }
    __device__ __forceinline__ float s(ES x) const { return from16(x); }
    __device__ __forceinline__ ES operator()(float x) const { return to16<S16>(x); }
};

template <class S16, bool PER, bool UM_IS_U, bool CONS>
__global__ void __launch_bounds__(128)
s16_tracer_kernel(const __grid_constant__ TracerArgs<float, float> A, const __grid_constant__ TracerIO16<S16> io) {
    tracer_body<float, float, PER, UM_IS_U, CONS>(A, (int)blockIdx.x, (int)blockIdx.y, (int)gridDim.y, io);
}

// Whole buffers: FP32 state -> pairs (u, v, eta) and 16-bit sst.
template <class S16>
__global__ void __launch_bounds__(256)
s16_pack_kernel(const float* u, const float* v, const float* e, const float* sst, S16* uh, S16* ul, S16* vh, S16* vl,
                S16* eh, S16* el, S16* so, long long n, float s) {
    const Put16<S16> hi{s};
    const PutLo16<S16> lo{s};
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        uh[k] = hi(u[k]); ul[k] = lo(u[k]);
        vh[k] = hi(v[k]); vl[k] = lo(v[k]);
        eh[k] = hi(e[k]); el[k] = lo(e[k]);
        so[k] = to16<S16>(sst[k]);
    }
}

// Whole buffers: pairs and 16-bit sst -> FP32 (the value each pair holds).
template <class S16>
__global__ void __launch_bounds__(256)
s16_unpack_kernel(const S16* uh, const S16* ul, const S16* vh, const S16* vl, const S16* eh, const S16* el,
                  const S16* si, float* u, float* v, float* e, float* sst, long long n, float inv_s) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        u[k] = (from16(uh[k]) + from16(ul[k])) * inv_s;
        v[k] = (from16(vh[k]) + from16(vl[k])) * inv_s;
        e[k] = (from16(eh[k]) + from16(el[k])) * inv_s;
        sst[k] = from16(si[k]);
    }
}

// X0 (FP32 u, v after the last stage) -> the new state's pairs, on steps
// without the tail (nstep_diff > 1); ghost copies are already in X0.
template <class S16>
__global__ void __launch_bounds__(256)
s16_pack_uv_kernel(const float* u, const float* v, S16* uh, S16* ul, S16* vh, S16* vl, long long n, float s,
                   const DevStatus* st) {
    if (st->stop) return;
    const Put16<S16> hi{s};
    const PutLo16<S16> lo{s};
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        uh[k] = hi(u[k]); ul[k] = lo(u[k]);
        vh[k] = hi(v[k]); vl[k] = lo(v[k]);
    }
}

// um, vm = u, v (hi) in FP32 for the tracer's mid-point velocity (nadvstep > 1)
template <class S16>
__global__ void __launch_bounds__(256)
s16_copy_uv_kernel(const S16* uh, const S16* vh, float* um, float* vm, long long n, float inv_s, const DevStatus* st) {
    if (st->stop) return;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        um[k] = from16(uh[k]) * inv_s;
        vm[k] = from16(vh[k]) * inv_s;
    }
}

// nan_detection! (src/feedback.jl:61-72) on the his of u, v, eta (before the
// step) and on sst (after it): a pair is NaN exactly when its hi is
template <class S16>
__global__ void s16_nan_check_kernel(Geom g, const S16* u, const S16* v, const S16* e, const S16* sst, long long step,
                                     DevStatus* st) {
    if (st->stop) return;
    const int N = g.N, M = g.M, ep = g.ep;
    const int uw = (ep ? N : N - 1) + 4;
    struct Ext { int w, h, x0, y0; const S16* p; };
    Ext ex[4] = {{uw, M + 4, ep ? -2 : -1, -2, u}, {N + 4, M + 3, -2, -1, v}, {N + 2, M + 2, -1, -1, e},
                 {N + 2, M, -1, 0, sst}};
    unsigned long long cnt = 0;
    for (int f = 0; f < 4; f++) {
        const long long tot = (long long)ex[f].w * ex[f].h;
        for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < tot; k += (long long)gridDim.x * blockDim.x) {
            const int x = ex[f].x0 + (int)(k % ex[f].w), y = ex[f].y0 + (int)(k / ex[f].w);
            const float val = from16(ex[f].p[g.idx(x, y)]);
            cnt += (val != val) ? 1 : 0;
        }
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) {
        atomicAdd(&st->nan_count, cnt);
        atomicCAS(&st->stop, 0, 1);
        st->nan_step = step;
    }
}

}  // namespace swb
