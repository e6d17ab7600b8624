// sw_stage2.cuh -- the RK stage for T = Tprog = Float32 with two columns per
// lane and packed FP32x2 arithmetic (sm_100).
//
// Same mathematics, operation order and results as rk_stage_tma in
// sw_stage.cuh (each packed __fadd2_rn/__fmul2_rn rounds both elements exactly
// like the scalar operation; a - b is formed as a + (-b), which IEEE defines
// to be the same).  Lane L of a warp owns columns c0 = base + 2L - 2 and
// c1 = c0 + 1; lanes 1..30 produce output, so a warp covers 60 columns and a
// block of 4 consumer warps a 240-column band.  A neighbour column is either
// the lane's other column or one shuffle away:
//   left(x)  = (shfl_up(x.y), x.x)      right(x) = (x.y, shfl_down(x.x))
// Input rows arrive through the TMA ring of rk_stage_tma (box 248 columns from
// device column bx0, i.e. columns bx0-4 .. bx0+243); X and X0 through a 240
// column box from device column bx0+4.
#pragma once
#include "sw_stage.cuh"

namespace swb {

constexpr int STRIP2 = 60;                 // output columns per warp
constexpr int BAND2 = 4 * STRIP2;          // output columns per block
constexpr int BOXW_IN2 = BAND2 + 16;       // 256: input box width (16-column pad keeps boxes 128-B aligned)
constexpr int BOXW_X2 = BAND2;             // 240

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 lft(float2 x) { return f2(__shfl_up_sync(0xffffffffu, x.y, 1), x.x); }
__device__ __forceinline__ float2 rgt(float2 x) { return f2(x.y, __shfl_down_sync(0xffffffffu, x.x, 1)); }

template <bool FIRST, bool LAST, int K>
struct StageSlot2 {
    static constexpr bool LOAD_X = !FIRST && !LAST;
    static constexpr bool LOAD_A = !FIRST;
    static constexpr int IN = K * BOXW_IN2;
    static constexpr int XE = K * BOXW_X2;
    static constexpr int NX = (LOAD_X ? 3 : 0) + (LOAD_A ? 3 : 0);
    static constexpr int ELEMS = 3 * IN + NX * XE;
    static constexpr uint32_t BYTES = ELEMS * 4;
    static constexpr int U = 0, V = IN, E = 2 * IN;
    static constexpr int XU = 3 * IN, XV = XU + XE, XW = XV + XE;
    static constexpr int AU = 3 * IN + (LOAD_X ? 3 * XE : 0), AV = AU + XE, AW = AV + XE;
    static_assert((IN * 4) % 128 == 0 && (XE * 4) % 128 == 0, "TMA destinations need 128-B alignment");
};

template <bool FIRST, bool LAST, int K, int S>
__host__ __device__ constexpr int stage2_smem() {
    return S * StageSlot2<FIRST, LAST, K>::BYTES + 2 * S * 8 + S * 4;
}

struct StageMaps2 {
    CUtensorMap in_u, in_v, in_e;    // box BOXW_IN2 x K
    CUtensorMap x_u, x_v, x_e;       // box BOXW_X2 x K
    CUtensorMap a_u, a_v, a_e;
};

template <bool PER, bool FIRST, bool LAST, int TY, int K, int S>
__global__ void __launch_bounds__(160)
rk_stage_f2(const __grid_constant__ StageArgs<float, float> A, const __grid_constant__ StageMaps2 MP, int npersist,
            TileSched* sched) {
    using SL = StageSlot2<FIRST, LAST, K>;
    using T = float;
    if ((int)blockIdx.x >= npersist) {
        if (A.st->stop) return;
        const int rb = (int)blockIdx.x - npersist;
        stage_ring(A, FIRST, LAST, rb * 160 + threadIdx.x, ((int)gridDim.x - npersist) * 160);
        return;
    }
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float* ring = reinterpret_cast<float*>(smem_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + S * SL::BYTES);
    uint64_t* empty = full + S;
    int* slot_tile = reinterpret_cast<int*>(empty + S);

    const Geom& g = A.g;
    const int N = g.N, M = g.M;
    const int nbx = (N + BAND2 - 1) / BAND2, nby = (M + TY - 1) / TY, ntiles = nbx * nby;
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
    if (stop_flag) return;

    if (warp == 4) {
        // ------------------------------------------------------------ producer
        if (lane != 0) return;
        uint32_t gc = 0;
        auto acquire = [&](int slot) {
            return gc < (uint32_t)S || mbar_wait(&empty[slot], ((gc / S) - 1) & 1, A.st);
        };
        bool ok = true;
        for (;;) {
            const int t = atomicAdd(&sched->next, 1);
            if (t >= ntiles) {
                const int slot0 = gc % S;
                if (acquire(slot0)) {
                    slot_tile[slot0] = -1;
                    mbar_arrive(&full[slot0]);
                    gc++;
                }
                break;
            }
            const int bx0 = (t % nbx) * BAND2, y0 = (t / nbx) * TY;
            for (int j = 0; j < NCH; j++, gc++) {
                const int slot = gc % S;
                if (!acquire(slot)) { ok = false; break; }
                slot_tile[slot] = t;
                mbar_arrive_expect_tx(&full[slot], SL::BYTES);
                float* b = ring + slot * SL::ELEMS;
                const int yd = y0 - 2 + j * K + ROW0;
                tma_load_2d(b + SL::U, &MP.in_u, bx0, yd, &full[slot]);
                tma_load_2d(b + SL::V, &MP.in_v, bx0, yd, &full[slot]);
                tma_load_2d(b + SL::E, &MP.in_e, bx0, yd, &full[slot]);
                if (SL::LOAD_X) {
                    tma_load_2d(b + SL::XU, &MP.x_u, bx0 + COL0, yd, &full[slot]);
                    tma_load_2d(b + SL::XV, &MP.x_v, bx0 + COL0, yd, &full[slot]);
                    tma_load_2d(b + SL::XW, &MP.x_e, bx0 + COL0, yd, &full[slot]);
                }
                if (SL::LOAD_A) {
                    tma_load_2d(b + SL::AU, &MP.a_u, bx0 + COL0, yd, &full[slot]);
                    tma_load_2d(b + SL::AV, &MP.a_v, bx0 + COL0, yd, &full[slot]);
                    tma_load_2d(b + SL::AW, &MP.a_e, bx0 + COL0, yd, &full[slot]);
                }
            }
            if (!ok) break;
        }
        for (uint32_t q = (gc >= (uint32_t)S ? gc - S : 0); q < gc; q++) mbar_wait(&full[q % S], (q / S) & 1, A.st);
        if (atomicAdd(&sched->done, 1) == npersist - 1) {
            sched->next = 0;
            sched->done = 0;
        }
        return;
    }

    // -------------------------------------------------------------- consumers
    const float2 half = bc2(0.5f), o12 = bc2(1.0f / 12.0f);
    const float2 q4 = bc2(0.25f);
    const int P = g.P;
    const int sc_in = warp * STRIP2 + 2 * lane + 2;   // even: float2-aligned
    const int sc_x = warp * STRIP2 + 2 * lane - 2;
    const bool out_lane = lane >= 1 && lane <= 30;
    const int Hsy = A.H.sy, fqsy = A.fq.sy, Fxsy = A.Fx.sy, Fysy = A.Fy.sy;
    const float2 ga = bc2(A.g_), Fxt = bc2(A.Fxt), Fyt = bc2(A.Fyt);
    const float2 ca = bc2(A.a), cbv = bc2(A.b);
    uint32_t gbase = 0;

    for (;; gbase += NCH) {
        if (!mbar_wait(&full[gbase % S], (gbase / S) & 1, A.st)) return;
        const int t = slot_tile[gbase % S];
        if (t < 0) return;
        const int bx0 = (t % nbx) * BAND2, y0 = (t / nbx) * TY;
        const int c0 = bx0 + warp * STRIP2 + 2 * lane - 2, c1 = c0 + 1;
        const int ulo = PER ? 0 : 1;
        const bool u0ok = out_lane && c0 >= ulo && c0 < N, u1ok = out_lane && c1 >= ulo && c1 < N;
        const bool a0ok = out_lane && c0 >= 0 && c0 < N, a1ok = out_lane && c1 >= 0 && c1 < N;
        // ghost sources touched by this lane's columns (rare: domain edges)
        const bool gx = (PER && (c0 <= 1 || c1 >= N - 2)) || c0 <= 1 || c1 >= N - 2;
        const bool wrap = PER && c1 == -1;            // q at c1 is q[end] (F = N)
        const bool qc_wrap0 = PER && c0 == 0;         // qγ at F = 0 sums in another order
        const int cb = c0 + COL0;

        auto slot_ptr = [&](int j) { return ring + ((gbase + j) % S) * SL::ELEMS; };
        auto wait_chunk = [&](int j) { return mbar_wait(&full[(gbase + j) % S], ((gbase + j) / S) & 1, A.st); };
        auto release = [&](int j) {
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[(gbase + j) % S]);
        };
        auto ld2 = [&](const float* p) { return *reinterpret_cast<const float2*>(p); };
        auto sfield2 = [&](const SField<T>& F, const T* p) {   // (F(c0), F(c1)) at the row of p
            return F.sx ? ld2(p) : bc2(*p);
        };

        int r = y0 - 2;
        const T* pH = A.H.p + (r + 1 + ROW0) * Hsy + cb * A.H.sx;
        const T* pfq = A.fq.p + (r + 1 + ROW0) * fqsy + cb * A.fq.sx;
        const T* pFx = A.Fx.p + (r + ROW0) * Fxsy + cb * A.Fx.sx;
        const T* pFy = A.Fy.p + (r + ROW0) * Fysy + cb * A.Fy.sx;
        float2 nH = sfield2(A.H, pH), nfq = sfield2(A.fq, pfq), nFx = sfield2(A.Fx, pFx), nFy = sfield2(A.Fy, pFy);

        const float* pin = slot_ptr(0) + sc_in;
        float2 u_r = ld2(pin + SL::U), v_r = ld2(pin + SL::V), e_r = ld2(pin + SL::E);
        float2 h_r = add2(e_r, f2(A.H.at(c0, r), A.H.at(c1, r)));
        float2 hl_r = lft(h_r), ur_r = rgt(u_r);
        float2 U_r = mul2(u_r, mul2(half, add2(h_r, hl_r)));
        float2 Ur_r = rgt(U_r);
        float2 V_r = bc2(0.f), Vl_r = bc2(0.f), q_r = bc2(0.f), ql_r = bc2(0.f), qr_r = bc2(0.f);
        float2 p_rm1 = bc2(0.f), qhu_part = bc2(0.f);
        float uN_r = 0.f, hN_r = 0.f, hNm1_r = 0.f;
        if (wrap) {
            uN_r = A.u1[g.idx(N, r)];
            hN_r = A.e1[g.idx(N, r)] + A.H.at(N, r);
            hNm1_r = A.e1[g.idx(N - 1, r)] + A.H.at(N - 1, r);
        }
        const float* px = slot_ptr(0) + sc_x;
        int nrel = 0;

        for (int i = 0; i < TY + 2; i++, r++) {
            const int kin = i + 1;
            if (kin % K == 0) {
                if (!wait_chunk(kin / K)) return;
                pin = slot_ptr(kin / K) + sc_in;
            } else {
                pin += BOXW_IN2;
            }
            const float2 u_r1 = ld2(pin + SL::U), v_r1 = ld2(pin + SL::V), e_r1 = ld2(pin + SL::E);
            const float2 fq = nfq, H1 = nH, Fxr = nFx, Fyr = nFy;
            pH += Hsy; pfq += fqsy; pFx += Fxsy; pFy += Fysy;
            nH = sfield2(A.H, pH); nfq = sfield2(A.fq, pfq); nFx = sfield2(A.Fx, pFx); nFy = sfield2(A.Fy, pFy);
            if (i > 0) {
                if (i % K == 0) px = slot_ptr(i / K) + sc_x;
                else px += BOXW_X2;
            }

            const float2 h_r1 = add2(e_r1, H1);                      // thickness!
            const float2 hl_r1 = lft(h_r1), vl_r1 = lft(v_r1), ur_r1 = rgt(u_r1);

            // q(c, G=r+1): PV! with h_q = Ixy!(h)
            const float2 hq = add2(mul2(q4, add2(hl_r, h_r)), mul2(q4, add2(hl_r1, h_r1)));
            const float2 num = sub2(add2(fq, sub2(v_r1, vl_r1)), sub2(u_r1, u_r));
            float2 q_r1 = f2(num.x / hq.x, num.y / hq.y);
            float uN_r1 = 0.f, hN_r1 = 0.f, hNm1_r1 = 0.f;
            if (wrap) {
                uN_r1 = A.u1[g.idx(N, r + 1)];
                hN_r1 = A.e1[g.idx(N, r + 1)] + A.H.at(N, r + 1);
                hNm1_r1 = A.e1[g.idx(N - 1, r + 1)] + A.H.at(N - 1, r + 1);
                const float vN = A.v1[g.idx(N, r + 1)], vNm1 = A.v1[g.idx(N - 1, r + 1)];
                q_r1.y = pv_q<float>(fq.y, vN, vNm1, uN_r1, uN_r, hNm1_r, hN_r, hNm1_r1, hN_r1);
            }
            const float2 ql_r1 = lft(q_r1), qr_r1 = rgt(q_r1);
            const float2 U_r1 = mul2(u_r1, mul2(half, add2(h_r1, hl_r1)));
            const float2 V_r1 = mul2(v_r1, mul2(half, add2(h_r1, h_r)));
            const float2 Ur_r1 = rgt(U_r1), Vl_r1 = lft(V_r1);
            const float2 KEu = mul2(half, add2(mul2(ur_r, ur_r), mul2(u_r, u_r)));
            const float2 KEv = mul2(half, add2(mul2(v_r1, v_r1), mul2(v_r, v_r)));
            const float2 p_r = add2(mul2(half, add2(KEu, KEv)), mul2(ga, e_r));
            const float2 pl_r = lft(p_r);
            const float2 s = add2(q_r, q_r1);
            const float2 qa = mul2(o12, add2(s, qr_r1));
            const float2 qb = mul2(o12, add2(s, ql_r1));
            float2 qc = mul2(o12, add2(add2(q_r, ql_r), q_r1));
            if (qc_wrap0) qc.x = (1.0f / 12.0f) * (s.x + ql_r.x);  // γ[1,j] order (src/PV_advection.jl:126)
            const float2 qd = mul2(o12, add2(s, qr_r));
            const float2 qbr = rgt(qb), qcr = rgt(qc);

            if (i >= 2 && r < M) {
                const int o = (r + ROW0) * P + cb;
                // momentum_u! with qhv
                const float2 qhv = add2(add2(add2(mul2(qa, V_r1), mul2(qb, Vl_r1)), mul2(qc, Vl_r)), mul2(qd, V_r));
                const float2 du = add2(sub2(qhv, sub2(p_r, pl_r)), mul2(Fxt, Fxr));
                // momentum_v! with qhu (its first two products formed last iteration)
                const float2 qhu = add2(add2(qhu_part, mul2(qcr, Ur_r)), mul2(qd, U_r));
                const float2 dv = add2(neg2(add2(qhu, sub2(p_r, p_rm1))), mul2(Fyt, Fyr));
                // continuity_itself!
                const float2 de = neg2(add2(sub2(Ur_r, U_r), sub2(V_r1, V_r)));
                const float2 Xu = FIRST ? u_r : (SL::LOAD_X ? ld2(px + SL::XU) : bc2(0.f));
                const float2 Xv = FIRST ? v_r : (SL::LOAD_X ? ld2(px + SL::XV) : bc2(0.f));
                const float2 Xe = FIRST ? e_r : (SL::LOAD_X ? ld2(px + SL::XW) : bc2(0.f));
                const float2 x0u = add2(FIRST ? Xu : ld2(px + SL::AU), mul2(ca, du));
                const float2 x0v = add2(FIRST ? Xv : ld2(px + SL::AV), mul2(ca, dv));
                const float2 x0e = add2(FIRST ? Xe : ld2(px + SL::AW), mul2(ca, de));
                float2 x1u = bc2(0.f), x1v = bc2(0.f), x1e = bc2(0.f);
                if (!LAST) {
                    x1u = add2(Xu, mul2(cbv, du));
                    x1v = add2(Xv, mul2(cbv, dv));
                    x1e = add2(Xe, mul2(cbv, de));
                }
                const bool vrow = r >= 1;
                float* du1 = A.u1o + o; float* dv1 = A.v1o + o; float* de1 = A.e1o + o;
                float* du0 = A.u0o + o; float* dv0 = A.v0o + o; float* de0 = A.e0o + o;
                if (u0ok && u1ok && a0ok && a1ok && vrow) {
                    if (!LAST) {
                        *reinterpret_cast<float2*>(du1) = x1u;
                        *reinterpret_cast<float2*>(dv1) = x1v;
                        *reinterpret_cast<float2*>(de1) = x1e;
                    }
                    *reinterpret_cast<float2*>(du0) = x0u;
                    *reinterpret_cast<float2*>(dv0) = x0v;
                    *reinterpret_cast<float2*>(de0) = x0e;
                } else {
                    if (u0ok) { if (!LAST) du1[0] = x1u.x; du0[0] = x0u.x; }
                    if (u1ok) { if (!LAST) du1[1] = x1u.y; du0[1] = x0u.y; }
                    if (vrow && a0ok) { if (!LAST) dv1[0] = x1v.x; dv0[0] = x0v.x; }
                    if (vrow && a1ok) { if (!LAST) dv1[1] = x1v.y; dv0[1] = x0v.y; }
                    if (a0ok) { if (!LAST) de1[0] = x1e.x; de0[0] = x0e.x; }
                    if (a1ok) { if (!LAST) de1[1] = x1e.y; de0[1] = x0e.y; }
                }
                // ghost points (domain edges only)
                const bool gy = r <= 1 || r >= M - 2;
                if (gx || gy) {
                    float* tu = LAST ? A.u0o : A.u1o;
                    float* tv = LAST ? A.v0o : A.v1o;
                    float* te = LAST ? A.e0o : A.e1o;
                    const float2 wu = LAST ? x0u : x1u, wv = LAST ? x0v : x1v, we = LAST ? x0e : x1e;
                    if (u0ok && A.gr.u_src(c0, r)) A.gr.u(tu, g, c0, r, wu.x);
                    if (u1ok && A.gr.u_src(c1, r)) A.gr.u(tu, g, c1, r, wu.y);
                    if (vrow && a0ok && A.gr.v_src(c0)) A.gr.v(tv, g, c0, r, wv.x);
                    if (vrow && a1ok && A.gr.v_src(c1)) A.gr.v(tv, g, c1, r, wv.y);
                    if (a0ok && A.gr.eta_src(c0, r)) A.gr.eta(te, g, c0, r, we.x);
                    if (a1ok && A.gr.eta_src(c1, r)) A.gr.eta(te, g, c1, r, we.y);
                }
            }
            if (i % K == K - 1) { release(i / K); nrel++; }

            qhu_part = add2(mul2(qa, U_r), mul2(qbr, Ur_r));
            u_r = u_r1; v_r = v_r1; e_r = e_r1; h_r = h_r1; hl_r = hl_r1; ur_r = ur_r1;
            q_r = q_r1; ql_r = ql_r1; qr_r = qr_r1;
            U_r = U_r1; Ur_r = Ur_r1;
            V_r = V_r1; Vl_r = Vl_r1;
            p_rm1 = p_r;
            uN_r = uN_r1; hN_r = hN_r1; hNm1_r = hNm1_r1;
        }
        for (int j = nrel; j < NCH; j++) release(j);
    }
}

}  // namespace swb
