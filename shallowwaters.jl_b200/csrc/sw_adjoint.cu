// sw_adjoint.cu -- reverse-mode gradient of an eta misfit through the time loop.
//
//   J = sum over the interior of (eta after nsteps - eta_obs)^2
//
// differentiated with respect to the initial state (u, v, eta with their
// halos) and the wind forcing Fx.  The forward model is the RK, SSPRK2, SSPRK3
// or 4SSPRK3 branch of time_integration (src/time_integration.jl:45-196, the
// SSP ones with their semi-implicit continuity, and the tail :204-233) with
// nonlinear (Arakawa-Hsu or Sadourny PV advection) or linear dynamics,
// quadratic / linear / no bottom drag and Smagorinsky / constant biharmonic
// diffusion, periodic or nonperiodic boundaries.  The tracer is passive (it never feeds back into
// u, v, eta), so it plays no part in J.
//
// Layout: every field is kept in the reference's own array shape (Julia
// (i, j), x fastest, 1-based, no padding), one device array per reference
// array, so each kernel below is the reference pass it cites and its adjoint.
// Forward passes recompute the reference's intermediate arrays exactly (same
// operation order; built with --fmad=false), so the recomputed forward state
// is bit-identical with the time loop's.  Each reverse pass is the transpose
// of one forward pass written in scatter form: for every output point it adds
// (output adjoint) x (partial derivative) into the adjoints of the inputs it
// read, with atomicAdd where several outputs share an input.  The summation
// order of those atomics is not fixed, so gradients agree between runs to
// rounding, not bit for bit.
//
// sqrt at zero (quadratic drag sqrt(KEu + KEv), src/bottom_drag.jl:48, and
// the Smagorinsky coefficient sqrt(DS + DT), src/diffusion.jl:106): the
// derivative is taken as 0 there, which is the derivative of the |u|u forms
// at rest.
//
// Time window: the step states are kept in device memory at checkpoints;
// with fewer checkpoint slots than steps, the reverse sweep recomputes the
// missing states from the nearest checkpoint with the binomial schedule
// (Griewank and Walther, "Algorithm 799: Revolve", ACM TOMS 26 (2000)).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "swb200.h"

namespace swa {

#ifdef SWA_HOST_CHECK
#define SWA_BOUNDS
#endif
#ifdef SWA_BOUNDS
// host check build: every array access outside its reference shape is counted
// (and redirected to a scratch element) instead of being performed
extern long long swa_bounds_failures;
#endif

template <class T>
struct A2 {
    T* d = nullptr;
    int m = 0, n = 0;
    __host__ __device__ __forceinline__ T& operator()(int i, int j) const {
#if defined(SWA_BOUNDS) && !defined(__CUDA_ARCH__)
        if (i < 1 || i > m || j < 1 || j > n || !d) {
            static T scratch;
            if (swa_bounds_failures++ < 8) fprintf(stderr, "swa: (%d, %d) outside %d x %d\n", i, j, m, n);
            return scratch;
        }
#endif
        return d[(i - 1) + (long long)(j - 1) * m];
    }
    size_t size() const { return (size_t)m * (size_t)n; }
};

template <class T>
__host__ __device__ __forceinline__ void add(T& r, T x) {
#ifdef __CUDA_ARCH__
    atomicAdd(&r, x);
#else
    r += x;
#endif
}

template <class T>
__host__ __device__ __forceinline__ T sqrt_(T x) {
#ifdef __CUDA_ARCH__
    return sqrt(x);
#else
    return std::sqrt(x);
#endif
}

// Programmatic dependent launch: a pass launched with programmatic stream
// serialization may start while its predecessor runs; griddepcontrol.wait
// holds its threads until the predecessor has completed and its writes are
// visible, and launch_dependents then lets the next pass be scheduled.  The
// passes of a step are short at the sizes the adjoint runs on, so hiding each
// launch behind the previous pass shortens the chain.  Without the launch
// attribute both instructions do nothing.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// one thread per point (i, j) of an m x n range, 1-based
template <class F>
__global__ void __launch_bounds__(256) for2d(int m, int n, F f) {
    pdl_enter();
    const int i = (int)(blockIdx.x * 32 + threadIdx.x) + 1;
    const int j = (int)(blockIdx.y * 8 + threadIdx.y) + 1;
    if (i <= m && j <= n) f(i, j);
}

template <class F>
__global__ void __launch_bounds__(256) for1d(long long n, F f) {
    pdl_enter();
    for (long long k = blockIdx.x * 256LL + threadIdx.x; k < n; k += (long long)gridDim.x * 256LL) f(k);
}

// Issues the passes on a stream (or, in the host check build, runs them in
// loops on the host).
struct Launcher {
    cudaStream_t s;
    bool host = false;
    int launches = 0;
    bool pdl = false;          // launch with programmatic stream serialization (see pdl_enter)
    template <class K, class... Args>
    void launch(K kern, dim3 g, dim3 b, Args... args) {
        if (!pdl) {
            kern<<<g, b, 0, s>>>(args...);
            return;
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = g;
        cfg.blockDim = b;
        cfg.dynamicSmemBytes = 0;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, kern, args...);
    }
    template <class F>
    void d2(int m, int n, F f) {
        if (host) {
            for (int j = 1; j <= n; j++)
                for (int i = 1; i <= m; i++) f(i, j);
        } else {
            dim3 g((unsigned)((m + 31) / 32), (unsigned)((n + 7) / 8)), b(32, 8);
            launch(for2d<F>, g, b, m, n, f);
        }
        launches++;
    }
    template <class F>
    void d1(long long n, F f) {
        if (host) {
            for (long long k = 0; k < n; k++) f(k);
        } else {
            const long long nb = std::min<long long>((n + 255) / 256, 148LL * 16);
            launch(for1d<F>, dim3((unsigned)std::max<long long>(nb, 1)), dim3(256), n, f);
        }
        launches++;
    }
    void zero(void* p, size_t bytes) {
        if (host) std::memset(p, 0, bytes);
        else cudaMemsetAsync(p, 0, bytes, s);
    }
    void copy(void* dst, const void* src, size_t bytes) {
        if (host) std::memcpy(dst, src, bytes);
        else cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s);
    }
};

// qhv at u-point (i, j) and qhu at v-point (i, j) of the PV advection, from
// the Arakawa-Hsu coefficients (src/PV_advection.jl:63-84) or the Sadourny
// averages (src/PV_advection.jl:31-59)
template <class T>
struct PVterms {
    A2<T> qa, qb, qc, qd, qu, qv, Vu, Uv, U, V;
    bool sad;
    int ep;
    __host__ __device__ __forceinline__ T qhv(int i, int j) const {
        const int c = 1 - ep + i;
        if (sad) return qu(c, j) * Vu(c, j);
        return qa(c, j) * V(c + 1, j + 1) + qb(c, j) * V(c, j + 1) + qc(c, j) * V(c, j) + qd(c, j) * V(c + 1, j);
    }
    __host__ __device__ __forceinline__ T qhu(int i, int j) const {
        if (sad) return qv(i, j + 1) * Uv(i, j + 1);
        return qa(i, j) * U(i, j + 1) + qb(i + 1, j) * U(i + 1, j + 1) + qc(i + 1, j + 1) * U(i + 1, j + 2) + qd(i, j + 1) * U(i, j + 2);
    }
};

// the three prognostic fields of one state, contiguous in one block
template <class T>
struct State {
    A2<T> u, v, e;
    T* base = nullptr;
    size_t elems = 0;
};

template <class T>
struct Work {
    int nx, ny, nux, nuy, nvx, nvy, ep, rko;
    bool ssp = false;           // SSPRK2 (src/time_integration.jl:80-104) or 4SSPRK3 (:150-196) instead of RK
    bool four = false;          // 4SSPRK3: averaged updates, full ghost points, the third sub-stage's mix
    // SSPRK3 (:112-156): s = n^2 sub-stages of Δt_Δn updates; sub-stage rki = kn mixes the snapshot u0
    // (kna*u1 + knb*u0 + Δt_Δnc*du, dxaybzc!); the snapshot is the state after sub-stage rki = mn
    // (or the step's start when mn = 1), eta ghosted in place there and at the last sub-stage
    bool ssp3 = false;
    int s3_kn = 0, s3_mn = 0;
    T s3_cnc, s3_kna, s3_knb;
    int rks = 0, nst = 0;       // SSPRK2 sub-stages; stage states kept per step
    T cssp, ssp_a, ssp_b;       // Δt_Δs, 1/RKs, (RKs-1)/RKs (Tprog)
    T g, cD, rD, cSmag, nuB, Dt_diff, oma;   // oma = 1 - alpha (Tprog = T)
    T RKa[4], RKb[3];
    int drag, diff;
    bool sadourny = false;      // PV_Sadourny! (src/PV_advection.jl:31-59) instead of Arakawa-Hsu
    bool linear = false;        // rhs_linear! (src/rhs.jl:59-86)
    // static fields
    A2<T> H, f_q, Fx, Fy, eta_ref, Feta, f_u, f_v;
    // time-dependent forcing: the step's Fxt, Fyt (seasonal wind, src/rhs.jl:233-238,
    // 262-267) and Fetat (continuity_forcing!, src/continuity.jl:27-49) are read
    // from force[0..2], which the host sets before each step's replay
    bool timedep = false, forcing = false;
    T* force = nullptr;
    bool relax = false;         // continuity_surf_relax! (src/continuity.jl:3-24)
    T gamma = T(0);
    // states
    State<T> X;                 // the state being advanced (in / out of a step)
    // stage states.  RK: Ys[k-1] = input of stage k after its ghost points
    // (Ys[0] = ghosted start state).  SSP schemes: Ys[0] = ghosted start state,
    // Ys[2k-1] = sub-stage k's input after ghost_points_eta!, Ys[2k] = its
    // state after the momentum update and ghost_points_uv!, Ys[2 RKs + 1] =
    // the state after the last sub-stage.
    State<T> Ys[20];
    State<T> Z;                 // RK result after ghost points = the tail's input
    T* stage_block = nullptr;   // Ys[0..nst-1] and Z, contiguous in this order
    size_t stage_block_elems = 0;
    size_t tail_inter_elems = 0;   // the tail intermediates, right after Z in the same block
    bool tail_kept = false;     // records keep the tail intermediates: a stored reverse step does not recompute them
    State<T> Xb, acc, Yb[2];    // adjoints: of the step output / input, of the stage inputs
    // stage intermediates (src/preallocate.jl:70-152, 227-254)
    A2<T> hu, hv, hq, U, V, q, qa, qb, qc, qd, p;
    A2<T> qu, qv, Vu, Uv;       // Sadourny: Iy(q), Ix(q), Ixy(V), Ixy(U)
    // their adjoints
    A2<T> bU, bV, bp, bqa, bqb, bqc, bqd, bq, bqu, bqv, bVu, bUv;
    // tail intermediates (src/preallocate.jl:193-222, 259-338)
    A2<T> thu, thv, sKE, sKEu, sKEv, Bu, Bv, Lu, Lv, dLudx, dLudy, dLvdx, dLvdy, sDT, sDS, DSq, rS, nuS, nuSq, S11,
        S12, S21, S22;
    A2<T> bBu, bBv, bS11, bS12, bS21, bS22, bnuS, bLu, bLv, bsKE, bDSq;
    A2<T> bFx;                  // gradient with respect to Fx
    T* stage_adj = nullptr; size_t stage_adj_elems = 0;   // bU..bq, one block (zeroed per stage)
    bool clear_stage_adj = true;  // stage_rev clears bU..bq first (not when they were cleared beforehand)
    T* tail_adj = nullptr; size_t tail_adj_elems = 0;     // bBu..bDSq, one block (zeroed per step)
};

// rhs_linear! tendencies at u-point (i, j) and v-point (i, j) of state y
// (src/rhs.jl:59-86, fv! :183-198, fu! :201-215): Coriolis on Ixy! of the other
// velocity and the gradient of g*eta, before the forcing term
template <class T>
struct LinTerms {
    A2<T> f_u, f_v;
    T g;
    int ep;
    __host__ __device__ __forceinline__ T du(const A2<T>& u, const A2<T>& v, const A2<T>& e, int i, int j) const {
        const T quarter = T(0.25);
        const int I = i + 2 - ep, J = j + 1;   // v_u(i+2-ep, j+1) = Ixy(v)
        const T vu = quarter * (v(I, J) + v(I + 1, J)) + quarter * (v(I, J + 1) + v(I + 1, J + 1));
        const T qhv = f_u(i, j) * vu;
        const T dpdx = g * e(i + 2 - ep, j + 1) - g * e(i + 1 - ep, j + 1);
        (void)u;
        return qhv - dpdx;
    }
    __host__ __device__ __forceinline__ T dv_part(const A2<T>& u, const A2<T>& e, int i, int j, T& dpdy) const {
        const T quarter = T(0.25);
        const int I = i + 1 + ep, J = j + 2;   // u_v(i+1+ep, j+2) = Ixy(u)
        const T uv = quarter * (u(I, J) + u(I + 1, J)) + quarter * (u(I, J + 1) + u(I + 1, J + 1));
        dpdy = g * e(i + 1, j + 2) - g * e(i + 1, j + 1);
        return f_v(i, j) * uv;   // qhu
    }
};

template <class T>
PVterms<T> pvterms(const Work<T>& w) {
    return PVterms<T>{w.qa, w.qb, w.qc, w.qd, w.qu, w.qv, w.Vu, w.Uv, w.U, w.V, w.sadourny, w.ep};
}

// ------------------------------------------------------------ ghost points
// ghost_points! (src/ghost_points.jl:182-199) on u, v (and eta); with uv_only
// only ghost_points_uv! (:202-216).  One launch, one thread per halo copy
// (row or column t, copy q of four).  eta's y-halo rows copy row 2 and row
// n-1 after its x-halo columns were set (src/ghost_points.jl:119-133), so the
// corner of row 1 (or n) takes the x-halo source of row 2 (or n-1) directly:
// etasrc(i) is that column.
template <class T>
__host__ __device__ __forceinline__ int etasrc(int i, int m, int ep) {
    if (i == 1) return ep ? m - 1 : 2;
    if (i == m) return ep ? 2 : m - 1;
    return i;
}

// ghost() / ghostT() modes: all fields, u and v only (ghost_points_uv!), eta
// only (ghost_points_eta!, src/ghost_points.jl:219-229)
constexpr int GH_ALL = 0, GH_UV = 1, GH_ETA = 2;

template <class T>
void ghost(Launcher& L, const Work<T>& w, const State<T>& s, int mode) {
    const bool uv_only = mode == GH_UV, eta_only = mode == GH_ETA;
    const A2<T> u = s.u, v = s.v, e = s.e;
    const int ep = w.ep;
    const T c = w.oma;
    const int nmax = std::max(std::max(u.m, u.n), std::max(std::max(v.m, v.n), std::max(e.m, e.n)));
    L.d1(4LL * nmax, [=] __host__ __device__(long long k) {
        const int t = (int)(k >> 2) + 1, q = (int)(k & 3);
        if (eta_only) {
        } else if (ep) {   // x-halo columns 1, 2, m-1, m from m-3, m-2, 3, 4
            if (t <= u.n) { const int m = u.m, d[4] = {1, 2, m - 1, m}, sx[4] = {m - 3, m - 2, 3, 4}; u(d[q], t) = u(sx[q], t); }
            if (t <= v.n) { const int m = v.m, d[4] = {1, 2, m - 1, m}, sx[4] = {m - 3, m - 2, 3, 4}; v(d[q], t) = v(sx[q], t); }
        } else {    // u: y-halo rows 1, 2, n-1, n from 4, 3, n-2, n-3; v: x-halo columns likewise
            if (t <= u.m) { const int n = u.n, d[4] = {1, 2, n - 1, n}, sy[4] = {4, 3, n - 2, n - 3}; u(t, d[q]) = c * u(t, sy[q]); }
            if (t <= v.n) { const int m = v.m, d[4] = {1, 2, m - 1, m}, sx[4] = {4, 3, m - 2, m - 3}; v(d[q], t) = c * v(sx[q], t); }
        }
        if (uv_only) return;
        const int m = e.m, n = e.n;
        if (q < 2) {   // x-halo columns of rows 2..n-1
            if (t >= 2 && t <= n - 1) {
                if (q == 0) e(1, t) = e(etasrc<T>(1, m, ep), t);
                else e(m, t) = e(etasrc<T>(m, m, ep), t);
            }
        } else if (t <= m) {   // y-halo rows 1 and n, corners included
            if (q == 2) e(t, 1) = e(etasrc<T>(t, m, ep), 2);
            else e(t, n) = e(etasrc<T>(t, m, ep), n - 1);
        }
    });
}

// transpose of ghost(): each halo adjoint is added onto its source and cleared
template <class T>
void ghostT(Launcher& L, const Work<T>& w, const State<T>& s, int mode) {
    const bool uv_only = mode == GH_UV, eta_only = mode == GH_ETA;
    const A2<T> u = s.u, v = s.v, e = s.e;
    const int ep = w.ep;
    const T c = w.oma;
    const T zero = T(0);
    const int nmax = std::max(std::max(u.m, u.n), std::max(std::max(v.m, v.n), std::max(e.m, e.n)));
    L.d1(4LL * nmax, [=] __host__ __device__(long long k) {
        const int t = (int)(k >> 2) + 1, q = (int)(k & 3);
        if (eta_only) {
        } else if (ep) {
            if (t <= u.n) {
                const int m = u.m, d[4] = {1, 2, m - 1, m}, sx[4] = {m - 3, m - 2, 3, 4};
                u(sx[q], t) += u(d[q], t); u(d[q], t) = zero;
            }
            if (t <= v.n) {
                const int m = v.m, d[4] = {1, 2, m - 1, m}, sx[4] = {m - 3, m - 2, 3, 4};
                v(sx[q], t) += v(d[q], t); v(d[q], t) = zero;
            }
        } else {
            if (t <= u.m) {
                const int n = u.n, d[4] = {1, 2, n - 1, n}, sy[4] = {4, 3, n - 2, n - 3};
                u(t, sy[q]) += c * u(t, d[q]); u(t, d[q]) = zero;
            }
            if (t <= v.n) {
                const int m = v.m, d[4] = {1, 2, m - 1, m}, sx[4] = {4, 3, m - 2, m - 3};
                v(sx[q], t) += c * v(d[q], t); v(d[q], t) = zero;
            }
        }
        if (uv_only) return;
        // eta: sources of rows 2 and n-1 are shared by the x-halo and y-halo
        // copies, so those sums are atomic; every halo cell is read and
        // cleared by one thread only
        const int m = e.m, n = e.n;
        if (q < 2) {
            if (t >= 2 && t <= n - 1) {
                const int d = q == 0 ? 1 : m;
                add(e(etasrc<T>(d, m, ep), t), e(d, t));
                e(d, t) = zero;
            }
        } else if (t <= m) {
            const int r = q == 2 ? 1 : n, rs = q == 2 ? 2 : n - 1;
            add(e(etasrc<T>(t, m, ep), rs), e(t, r));
            e(t, r) = zero;
        }
    });
}

// ------------------------------------------------------------ RK stage, forward
// rhs_nonlinear! without the momentum write (src/rhs.jl:24-51): thickness!,
// Ix!/Iy!/Ixy! of h, UVfluxes! (:307-324), PV! (src/PV_advection.jl:2-18),
// AHα..δ! (src/PV_advection.jl:88-146) and bernoulli! (src/rhs.jl:162-180).
template <class T>
void stage_fwd(Launcher& L, const Work<T>& w, const State<T>& Y) {
    const A2<T> u = Y.u, v = Y.v, e = Y.e, H = w.H, f_q = w.f_q;
    const A2<T> hu = w.hu, hv = w.hv, hq = w.hq, U = w.U, V = w.V, q = w.q;
    const int nx = w.nx, ny = w.ny, ep = w.ep;
    L.d2(nx + 2, ny + 2, [=] __host__ __device__(int i, int j) {
        const T half = T(0.5), quarter = T(0.25);
        auto h = [&](int a, int b) { return e(a, b) + H(a, b); };
        if (i <= nx + 1) {
            const T hu_ = half * (h(i + 1, j) + h(i, j));
            hu(i, j) = hu_;
            U(i, j) = u(1 + ep + i, 1 + j) * hu_;
        }
        if (j <= ny + 1) {
            const T hv_ = half * (h(i, j + 1) + h(i, j));
            hv(i, j) = hv_;
            V(i, j) = v(i + 1, j + 1) * hv_;
        }
        if (i <= nx + 1 && j <= ny + 1) {
            const T hq_ = quarter * (h(i, j) + h(i + 1, j)) + quarter * (h(i, j + 1) + h(i + 1, j + 1));
            hq(i, j) = hq_;
            const T dvdx = v(i + 2, j + 1) - v(i + 1, j + 1);
            const T dudy = u(i + 1 + ep, j + 2) - u(i + 1 + ep, j + 1);
            q(i, j) = (f_q(i, j) + dvdx - dudy) / hq_;
        }
    });
    if (w.linear) return;   // rhs_linear! needs none of the PV and Bernoulli terms
    const A2<T> qa = w.qa, qb = w.qb, qc = w.qc, qd = w.qd, p = w.p;
    const A2<T> qu = w.qu, qv = w.qv, Vu = w.Vu, Uv = w.Uv;
    const bool sad = w.sadourny;
    const T g = w.g;
    L.d2(nx + 2, ny + 2, [=] __host__ __device__(int i, int j) {
        const T o12 = T(1.0 / 12.0), half = T(0.5), quarter = T(0.25);
        const int qend = q.m;
        if (sad) {   // Iy!(q_u, q), Ix!(q_v, q), Ixy!(V_u, V), Ixy!(U_v, U)
            if (i <= nx + 1 && j <= ny) {
                qu(i, j) = half * (q(i, j + 1) + q(i, j));
                Vu(i, j) = quarter * (V(i, j) + V(i + 1, j)) + quarter * (V(i, j + 1) + V(i + 1, j + 1));
            }
            if (i <= nx && j <= ny + 1) {
                qv(i, j) = half * (q(i + 1, j) + q(i, j));
                Uv(i, j) = quarter * (U(i, j) + U(i + 1, j)) + quarter * (U(i, j + 1) + U(i + 1, j + 1));
            }
        } else if (i <= nx && j <= ny) {
            qa(i, j) = o12 * (q(i, j) + q(i, j + 1) + q(i + 1, j + 1));
            qd(i, j) = o12 * (q(i, j) + q(i, j + 1) + q(i + 1, j));
        }
        if (!sad && i <= nx + 1 && j <= ny) {
            if (i == 1) {
                qb(1, j) = o12 * (q(1, j) + q(1, j + 1) + q(qend, j + 1));
                qc(1, j) = o12 * (q(1, j) + q(1, j + 1) + q(qend, j));
            } else {
                qb(i, j) = o12 * (q(i, j) + q(i, j + 1) + q(i - 1, j + 1));
                qc(i, j) = o12 * (q(i, j) + q(i - 1, j) + q(i, j + 1));
            }
        }
        const int a = i + ep, b = j + 1;   // KEu(a, b) = Ix(u^2), KEv(i+1, j) = Iy(v^2)
        const T KEu = half * (u(a + 1, b) * u(a + 1, b) + u(a, b) * u(a, b));
        const T KEv = half * (v(i + 1, j + 1) * v(i + 1, j + 1) + v(i + 1, j) * v(i + 1, j));
        p(i, j) = half * (KEu + KEv) + g * e(i, j);
    });
}

// momentum_u!/v! (src/rhs.jl:218-274), continuity_itself! (src/continuity.jl:52-68)
// and the RK combination (src/time_integration.jl:64-72): Y1 = Xt + b*d (k < RKo),
// X0 += a*d.  d is zero on the halo, so halo points keep Xt / X0.
template <class T>
void stage_update(Launcher& L, const Work<T>& w, int k, const State<T>& Y, const State<T>& Xt, const State<T>* Y1,
                  const State<T>& X0) {
    const A2<T> p = w.p, Fx = w.Fx, Fy = w.Fy, U = w.U, V = w.V;
    const PVterms<T> pv = pvterms(w);
    const int nx = w.nx, ny = w.ny, nux = w.nux, nuy = w.nuy, nvx = w.nvx, nvy = w.nvy, ep = w.ep;
    const T a = w.RKa[k - 1], b = k < w.rko ? w.RKb[k - 1] : T(0);
    const bool next = Y1 != nullptr;
    const State<T> xt = Xt, x0 = X0, y1 = next ? *Y1 : Xt;
    const A2<T> eta_ref = w.eta_ref, ye = Y.e, Feta = w.Feta, yu = Y.u, yv = Y.v;
    const bool relax = w.relax, timedep = w.timedep, forcing = w.forcing, linear = w.linear;
    const T gamma = w.gamma;
    const T* force = w.force;
    const LinTerms<T> lt{w.f_u, w.f_v, w.g, w.ep};
    L.d2(nx + 4, ny + 4, [=] __host__ __device__(int I, int J) {
        const T zero = T(0);
        if (I <= xt.u.m && J <= xt.u.n) {
            T d = zero;
            if (I >= 3 && I <= nux + 2 && J >= 3 && J <= nuy + 2) {
                const int i = I - 2, j = J - 2;
                T m;
                if (linear) {
                    m = lt.du(yu, yv, ye, i, j);
                } else {
                    const T qhv = pv.qhv(i, j);
                    const T dpdx = p(i + 2 - ep, j + 1) - p(i + 1 - ep, j + 1);
                    m = qhv - dpdx;
                }
                d = timedep ? m + force[0] * Fx(i, j) : m + Fx(i, j);
            }
            if (next) y1.u(I, J) = xt.u(I, J) + b * d;
            x0.u(I, J) += a * d;
        }
        if (I <= xt.v.m && J <= xt.v.n) {
            T d = zero;
            if (I >= 3 && I <= nvx + 2 && J >= 3 && J <= nvy + 2) {
                const int i = I - 2, j = J - 2;
                T qhu, dpdy;
                if (linear) {
                    qhu = lt.dv_part(yu, ye, i, j, dpdy);
                } else {
                    qhu = pv.qhu(i, j);
                    dpdy = p(i + 1, j + 2) - p(i + 1, j + 1);
                }
                d = timedep ? -(qhu + dpdy) + force[1] * Fy(i, j) : -(qhu + dpdy) + Fy(i, j);
            }
            if (next) y1.v(I, J) = xt.v(I, J) + b * d;
            x0.v(I, J) += a * d;
        }
        if (I <= xt.e.m && J <= xt.e.n) {
            T d = zero;
            if (I >= 2 && I <= nx + 1 && J >= 2 && J <= ny + 1) {
                const int i = I - 1, j = J - 1;
                // with linear dynamics the RK continuity reads U, V that rhs_linear!
                // never forms, i.e. zeros (src/time_integration.jl:71, src/continuity.jl:72-97)
                const T dUdx = linear ? zero - zero : U(i + 1, j + 1) - U(i, j + 1);
                const T dVdy = linear ? zero - zero : V(i + 1, j + 1) - V(i + 1, j);
                d = -(dUdx + dVdy);
                if (relax) d = d + gamma * (eta_ref(i, j) - ye(i + 1, j + 1));
                else if (forcing) d = d + force[2] * Feta(i, j);
            }
            if (next) y1.e(I, J) = xt.e(I, J) + b * d;
            x0.e(I, J) += a * d;
        }
    });
}

// ------------------------------------------------------------ RK stage, reverse
// Given the stage's tendency adjoint  dbar = a*Xb0 + b*Wb  (interior points),
// adds the adjoint of the stage input Y into Yb.  Transposes, in reverse
// order, the passes of stage_fwd and stage_update.
// transpose of a linear-dynamics stage (rhs_linear!, src/rhs.jl:59-86, and
// the RK continuity, whose only state dependence is the relaxation term).
// Two passes: the tendency adjoints into scratch (bqa at u-points, bqd at
// v-points, with the sign of dv), then their scatter onto the state adjoint,
// so Yb may be Xb0 itself.
template <class T>
void stage_rev_linear(Launcher& L, const Work<T>& w, int k, const State<T>& Xb0, const State<T>* Wb, const State<T>& Yb,
                      bool mom_only, T coef) {
    const A2<T> gu = w.bqa, gv = w.bqd, bFx = w.bFx, f_u = w.f_u, f_v = w.f_v;
    const int nx = w.nx, ny = w.ny, nux = w.nux, nuy = w.nuy, nvx = w.nvx, nvy = w.nvy, ep = w.ep;
    const T a = mom_only ? coef : w.RKa[k - 1], b = (Wb && !mom_only) ? w.RKb[k - 1] : T(0);
    const State<T> x0 = Xb0, wb = Wb ? *Wb : Xb0, yb = Yb;
    const bool has_w = Wb != nullptr && !mom_only, relax = w.relax, timedep = w.timedep;
    const T gamma = w.gamma, g = w.g;
    const T* force = w.force;
    L.d2(nx, ny, [=] __host__ __device__(int i, int j) {
        if (i <= nux && j <= nuy) {
            T t = a * x0.u(i + 2, j + 2);
            if (has_w) t += b * wb.u(i + 2, j + 2);
            gu(i, j) = t;
            bFx(i, j) += timedep ? force[0] * t : t;
        }
        if (i <= nvx && j <= nvy) {
            T t = a * x0.v(i + 2, j + 2);
            if (has_w) t += b * wb.v(i + 2, j + 2);
            gv(i, j) = -t;
        }
        if (!mom_only && relax) {
            T t = a * x0.e(i + 1, j + 1);
            if (has_w) t += b * wb.e(i + 1, j + 1);
            add(yb.e(i + 1, j + 1), -(gamma * t));
        }
    });
    L.d2(nx, ny, [=] __host__ __device__(int i, int j) {
        const T quarter = T(0.25);
        if (i <= nux && j <= nuy) {   // du = (f_u*Ixy(v) - (g*eta(i+2-ep) - g*eta(i+1-ep))) + ...
            const T t = gu(i, j);
            const int I = i + 2 - ep, J = j + 1;
            const T s = quarter * (f_u(i, j) * t);
            add(yb.v(I, J), s); add(yb.v(I + 1, J), s); add(yb.v(I, J + 1), s); add(yb.v(I + 1, J + 1), s);
            add(yb.e(i + 2 - ep, j + 1), -(g * t)); add(yb.e(i + 1 - ep, j + 1), g * t);
        }
        if (i <= nvx && j <= nvy) {   // dv = -(f_v*Ixy(u) + (g*eta(j+2) - g*eta(j+1))) + ...
            const T m = gv(i, j);
            const int I = i + 1 + ep, J = j + 2;
            const T s = quarter * (f_v(i, j) * m);
            add(yb.u(I, J), s); add(yb.u(I + 1, J), s); add(yb.u(I, J + 1), s); add(yb.u(I + 1, J + 1), s);
            add(yb.e(i + 1, j + 2), g * m); add(yb.e(i + 1, j + 1), -(g * m));
        }
    });
}

template <class T>
void stage_rev(Launcher& L, const Work<T>& w, int k, const State<T>& Y, const State<T>& Xb0, const State<T>* Wb,
               const State<T>& Yb, bool mom_only = false, T coef = T(0)) {
    if (w.linear) { stage_rev_linear(L, w, k, Xb0, Wb, Yb, mom_only, coef); return; }
    const A2<T> u = Y.u, v = Y.v;
    const A2<T> hu = w.hu, hv = w.hv, hq = w.hq, U = w.U, V = w.V, q = w.q, qa = w.qa, qb = w.qb, qc = w.qc, qd = w.qd;
    const A2<T> bU = w.bU, bV = w.bV, bp = w.bp, bqa = w.bqa, bqb = w.bqb, bqc = w.bqc, bqd = w.bqd, bq = w.bq,
                bFx = w.bFx;
    const A2<T> qu = w.qu, qv = w.qv, Vu = w.Vu, Uv = w.Uv, bqu = w.bqu, bqv = w.bqv, bVu = w.bVu, bUv = w.bUv;
    const bool sad = w.sadourny, relax = w.relax, timedep = w.timedep;
    const T gamma = w.gamma;
    const T* force = w.force;
    const int nx = w.nx, ny = w.ny, nux = w.nux, nuy = w.nuy, nvx = w.nvx, nvy = w.nvy, ep = w.ep;
    // RK: dbar = RKa*Xb0 + RKb*Wb.  Momentum only (SSPRK2): dbar = coef*Xb0 for
    // u and v, no continuity part (Yb may then be Xb0 itself: this first pass
    // reads Xb0 and writes no state adjoint)
    const T a = mom_only ? coef : w.RKa[k - 1], b = (Wb && !mom_only) ? w.RKb[k - 1] : T(0);
    const State<T> x0 = Xb0, wb = Wb ? *Wb : Xb0, yb = Yb;
    const bool has_w = Wb != nullptr && !mom_only;
    // (clearing the scratch where the passes read it instead of this memset
    // measured 50 % slower: 491 against 335 ms for 2000 reverse steps)
    if (w.clear_stage_adj) L.zero(w.stage_adj, w.stage_adj_elems * sizeof(T));
    // momentum_u^T, momentum_v^T (with PV_ArakawaHsu^T), continuity^T
    L.d2(nx, ny, [=] __host__ __device__(int i, int j) {
        if (i <= nux && j <= nuy) {
            T g = a * x0.u(i + 2, j + 2);
            if (has_w) g += b * wb.u(i + 2, j + 2);
            bFx(i, j) += timedep ? force[0] * g : g;
            add(bp(i + 2 - ep, j + 1), -g);
            add(bp(i + 1 - ep, j + 1), g);
            const int c = 1 - ep + i;      // qhv (src/PV_advection.jl:73, Sadourny :49)
            if (sad) {
                add(bqu(c, j), g * Vu(c, j)); add(bVu(c, j), g * qu(c, j));
            } else {
                add(bqa(c, j), g * V(c + 1, j + 1)); add(bV(c + 1, j + 1), g * qa(c, j));
                add(bqb(c, j), g * V(c, j + 1));     add(bV(c, j + 1), g * qb(c, j));
                add(bqc(c, j), g * V(c, j));         add(bV(c, j), g * qc(c, j));
                add(bqd(c, j), g * V(c + 1, j));     add(bV(c + 1, j), g * qd(c, j));
            }
        }
        if (i <= nvx && j <= nvy) {
            T g = a * x0.v(i + 2, j + 2);
            if (has_w) g += b * wb.v(i + 2, j + 2);
            const T m = -g;                 // dv = -(qhu + dpdy) + Fy
            add(bp(i + 1, j + 2), m);
            add(bp(i + 1, j + 1), -m);
            if (sad) {                      // qhu = q_v(i, j+1) * U_v(i, j+1)
                add(bqv(i, j + 1), m * Uv(i, j + 1)); add(bUv(i, j + 1), m * qv(i, j + 1));
            } else {
                add(bqa(i, j), m * U(i, j + 1));             add(bU(i, j + 1), m * qa(i, j));
                add(bqb(i + 1, j), m * U(i + 1, j + 1));     add(bU(i + 1, j + 1), m * qb(i + 1, j));
                add(bqc(i + 1, j + 1), m * U(i + 1, j + 2)); add(bU(i + 1, j + 2), m * qc(i + 1, j + 1));
                add(bqd(i, j + 1), m * U(i, j + 2));         add(bU(i, j + 2), m * qd(i, j + 1));
            }
        }
        if (!mom_only) {
            T g = a * x0.e(i + 1, j + 1);
            if (has_w) g += b * wb.e(i + 1, j + 1);
            add(bU(i + 1, j + 1), -g); add(bU(i, j + 1), g);
            add(bV(i + 1, j + 1), -g); add(bV(i + 1, j), g);
            if (relax) add(yb.e(i + 1, j + 1), -(gamma * g));   // gamma*(eta_ref - eta); yb is not x0 here
        }
    });
    // bernoulli^T (through KEu = Ix(u^2), KEv = Iy(v^2)) and AHα..δ^T
    const T g = w.g;
    L.d2(nx + 2, ny + 2, [=] __host__ __device__(int i, int j) {
        const T half = T(0.5), o12 = T(1.0 / 12.0);
        const T wp = bp(i, j);
        add(yb.e(i, j), g * wp);
        const T hw = half * wp;
        const int a2 = i + ep, b2 = j + 1;
        add(yb.u(a2 + 1, b2), hw * u(a2 + 1, b2));
        add(yb.u(a2, b2), hw * u(a2, b2));
        add(yb.v(i + 1, j + 1), hw * v(i + 1, j + 1));
        add(yb.v(i + 1, j), hw * v(i + 1, j));
        const int qend = q.m;
        if (sad) {   // Iy^T, Ix^T of q; Ixy^T of V and U (their U, V adjoints are read in the next pass)
            const T quarter = T(0.25);
            if (i <= nx + 1 && j <= ny) {
                const T t = half * bqu(i, j);
                add(bq(i, j + 1), t); add(bq(i, j), t);
                const T s = quarter * bVu(i, j);
                add(bV(i, j), s); add(bV(i + 1, j), s); add(bV(i, j + 1), s); add(bV(i + 1, j + 1), s);
            }
            if (i <= nx && j <= ny + 1) {
                const T t = half * bqv(i, j);
                add(bq(i + 1, j), t); add(bq(i, j), t);
                const T s = quarter * bUv(i, j);
                add(bU(i, j), s); add(bU(i + 1, j), s); add(bU(i, j + 1), s); add(bU(i + 1, j + 1), s);
            }
        } else if (i <= nx && j <= ny) {
            const T ta = o12 * bqa(i, j), td = o12 * bqd(i, j);
            add(bq(i, j), ta + td); add(bq(i, j + 1), ta + td);
            add(bq(i + 1, j + 1), ta); add(bq(i + 1, j), td);
        }
        if (!sad && i <= nx + 1 && j <= ny) {
            const T tb = o12 * bqb(i, j), tc = o12 * bqc(i, j);
            add(bq(i, j), tb + tc); add(bq(i, j + 1), tb + tc);
            if (i == 1) { add(bq(qend, j + 1), tb); add(bq(qend, j), tc); }
            else { add(bq(i - 1, j + 1), tb); add(bq(i - 1, j), tc); }
        }
    });
    // PV^T, Uflux^T, Vflux^T, each followed at once by the Ixy^T, Ix^T, Iy^T of
    // h = eta + H that its h_q, h_u, h_v adjoint (formed here alone) feeds
    L.d2(nx + 2, ny + 2, [=] __host__ __device__(int i, int j) {
        const T half = T(0.5), quarter = T(0.25);
        if (i <= nx + 1 && j <= ny + 1) {
            const T n = bq(i, j) / hq(i, j);
            add(yb.v(i + 2, j + 1), n); add(yb.v(i + 1, j + 1), -n);
            add(yb.u(i + 1 + ep, j + 2), -n); add(yb.u(i + 1 + ep, j + 1), n);
            const T t = quarter * -(n * q(i, j));
            add(yb.e(i, j), t); add(yb.e(i + 1, j), t); add(yb.e(i, j + 1), t); add(yb.e(i + 1, j + 1), t);
        }
        if (i <= nx + 1) {
            const T wU = bU(i, j);
            add(yb.u(1 + ep + i, 1 + j), wU * hu(i, j));
            const T t = half * (wU * u(1 + ep + i, 1 + j));
            add(yb.e(i + 1, j), t); add(yb.e(i, j), t);
        }
        if (j <= ny + 1) {
            const T wV = bV(i, j);
            add(yb.v(i + 1, j + 1), wV * hv(i, j));
            const T t = half * (wV * v(i + 1, j + 1));
            add(yb.e(i, j + 1), t); add(yb.e(i, j), t);
        }
    });
}

// ------------------------------------------------------------ SSPRK2 sub-stage
// src/time_integration.jl:80-104: u1 += Δt_Δs*du, v1 += Δt_Δs*dv (axb!, whole
// arrays, du zero on the halo) after rhs! at the sub-stage input Yp (whose
// stage_fwd intermediates are current); eta is carried over.
template <class T>
void ssp_mom(Launcher& L, const Work<T>& w, const State<T>& Yp, const State<T>& Ym, const State<T>* Zs = nullptr) {
    const A2<T> p = w.p, Fx = w.Fx, Fy = w.Fy;
    const PVterms<T> pv = pvterms(w);
    const LinTerms<T> lt{w.f_u, w.f_v, w.g, w.ep};
    const bool linear = w.linear, four = w.four;
    const int nx = w.nx, ny = w.ny, nux = w.nux, nuy = w.nuy, nvx = w.nvx, nvy = w.nvy, ep = w.ep;
    const T c = w.cssp;
    const bool timedep = w.timedep;
    const T* force = w.force;
    const State<T> yp = Yp, ym = Ym;
    const bool kn = Zs != nullptr;   // SSPRK3's stage kn: kna*u1 + knb*u0 + Δt_Δnc*du (dxaybzc!)
    const State<T> zs = kn ? *Zs : Yp;
    const T kna = w.s3_kna, knb = w.s3_knb, cnc = w.s3_cnc;
    L.d2(nx + 4, ny + 4, [=] __host__ __device__(int I, int J) {
        const T zero = T(0);
        if (I <= yp.u.m && J <= yp.u.n) {
            T d = zero;
            if (I >= 3 && I <= nux + 2 && J >= 3 && J <= nuy + 2) {
                const int i = I - 2, j = J - 2;
                T m;
                if (linear) {
                    m = lt.du(yp.u, yp.v, yp.e, i, j);
                } else {
                    const T qhv = pv.qhv(i, j);
                    const T dpdx = p(i + 2 - ep, j + 1) - p(i + 1 - ep, j + 1);
                    m = qhv - dpdx;
                }
                d = timedep ? m + force[0] * Fx(i, j) : m + Fx(i, j);
            }
            if (four) {   // u0 = u1 + Δt_Δ*du; u1 = 0.5*(u1 + u0) (caxb!, cxab!)
                const T t = yp.u(I, J) + c * d;
                ym.u(I, J) = T(0.5) * (yp.u(I, J) + t);
            } else if (kn) {
                ym.u(I, J) = kna * yp.u(I, J) + knb * zs.u(I, J) + cnc * d;
            } else {
                ym.u(I, J) = yp.u(I, J) + c * d;
            }
        }
        if (I <= yp.v.m && J <= yp.v.n) {
            T d = zero;
            if (I >= 3 && I <= nvx + 2 && J >= 3 && J <= nvy + 2) {
                const int i = I - 2, j = J - 2;
                T qhu, dpdy;
                if (linear) {
                    qhu = lt.dv_part(yp.u, yp.e, i, j, dpdy);
                } else {
                    qhu = pv.qhu(i, j);
                    dpdy = p(i + 1, j + 2) - p(i + 1, j + 1);
                }
                d = timedep ? -(qhu + dpdy) + force[1] * Fy(i, j) : -(qhu + dpdy) + Fy(i, j);
            }
            if (four) {
                const T t = yp.v(I, J) + c * d;
                ym.v(I, J) = T(0.5) * (yp.v(I, J) + t);
            } else if (kn) {
                ym.v(I, J) = kna * yp.v(I, J) + knb * zs.v(I, J) + cnc * d;
            } else {
                ym.v(I, J) = yp.v(I, J) + c * d;
            }
        }
        if (I <= yp.e.m && J <= yp.e.n) ym.e(I, J) = yp.e(I, J);
    });
}

// the semi-implicit continuity (src/continuity.jl:72-97 with UVfluxes! of the
// updated u1, v1 and the sub-stage's eta1, whose h_u, h_v stage_fwd formed)
// and eta1 += Δt_Δs*deta; u1, v1 carried over into Yn
template <class T>
void ssp_cont(Launcher& L, const Work<T>& w, const State<T>& Ym, const State<T>& Yn, const State<T>* Zs = nullptr) {
    const A2<T> hu = w.hu, hv = w.hv;
    const int nx = w.nx, ny = w.ny, ep = w.ep;
    const T c = w.cssp;
    const State<T> ym = Ym, yn = Yn;
    const A2<T> eta_ref = w.eta_ref, Feta = w.Feta;
    const bool relax = w.relax, forcing = w.forcing, four = w.four;
    const T gamma = w.gamma;
    const T* force = w.force;
    const bool kn = Zs != nullptr;   // SSPRK3's stage kn: kna*eta1 + knb*eta0 + Δt_Δnc*deta
    const State<T> zs = kn ? *Zs : Ym;
    const T kna = w.s3_kna, knb = w.s3_knb, cnc = w.s3_cnc;
    L.d2(nx + 4, ny + 4, [=] __host__ __device__(int I, int J) {
        if (I <= ym.u.m && J <= ym.u.n) yn.u(I, J) = ym.u(I, J);
        if (I <= ym.v.m && J <= ym.v.n) yn.v(I, J) = ym.v(I, J);
        if (I <= ym.e.m && J <= ym.e.n) {
            T d = T(0);
            if (I >= 2 && I <= nx + 1 && J >= 2 && J <= ny + 1) {
                const int i = I - 1, j = J - 1;
                auto Uf = [&](int a, int b) { return ym.u(1 + ep + a, 1 + b) * hu(a, b); };
                auto Vf = [&](int a, int b) { return ym.v(a + 1, b + 1) * hv(a, b); };
                const T dUdx = Uf(i + 1, j + 1) - Uf(i, j + 1);
                const T dVdy = Vf(i + 1, j + 1) - Vf(i + 1, j);
                d = -(dUdx + dVdy);
                if (relax) d = d + gamma * (eta_ref(i, j) - ym.e(i + 1, j + 1));
                else if (forcing) d = d + force[2] * Feta(i, j);
            }
            if (four) {   // eta0 = eta1 + Δt_Δ*deta; eta1 = 0.5*(eta1 + eta0)
                const T t = ym.e(I, J) + c * d;
                yn.e(I, J) = T(0.5) * (ym.e(I, J) + t);
            } else if (kn) {
                yn.e(I, J) = kna * ym.e(I, J) + knb * zs.e(I, J) + cnc * d;
            } else {
                yn.e(I, J) = ym.e(I, J) + c * d;
            }
        }
    });
}

// transpose of ssp_cont on the adjoint Yb of Yn (in place: Yb becomes the
// adjoint of Ym).  Two passes: the flux adjoints in gather form (they read
// Yb's eta), then their scatter onto u, v and, through h_u, h_v, eta.
template <class T>
void ssp_cont_rev(Launcher& L, const Work<T>& w, const State<T>& Ym, const State<T>& Yb, T coef) {
    const A2<T> hu = w.hu, hv = w.hv, bU = w.bU, bV = w.bV, bp = w.bp;
    const bool relax = w.relax;
    const T gamma = w.gamma;
    const int nx = w.nx, ny = w.ny, ep = w.ep;
    const T c = coef;   // d(new eta)/d(deta): Δt_Δs (SSPRK2) or Δt_Δ/2 (4SSPRK3)
    const State<T> ym = Ym, yb = Yb;
    L.d2(nx + 2, ny + 2, [=] __host__ __device__(int I, int J) {
        auto g = [&](int i, int j) {   // deta adjoint at T-point (i, j), zero off the interior
            return (i >= 1 && i <= nx && j >= 1 && j <= ny) ? c * yb.e(i + 1, j + 1) : T(0);
        };
        if (I <= nx + 1) bU(I, J) = g(I, J - 1) - g(I - 1, J - 1);        // dUdx(i, j+1) = U(i+1, j+1) - U(i, j+1)
        if (J <= ny + 1) bV(I, J) = g(I - 1, J) - g(I - 1, J - 1);        // dVdy(i+1, j) = V(i+1, j+1) - V(i+1, j)
        if (relax && I <= nx && J <= ny) bp(I, J) = g(I, J);              // for the relaxation term, next pass
    });
    L.d2(nx + 2, ny + 2, [=] __host__ __device__(int I, int J) {
        const T half = T(0.5);
        if (relax && I <= nx && J <= ny) add(yb.e(I + 1, J + 1), -(gamma * bp(I, J)));   // gamma*(eta_ref - eta)
        if (I <= nx + 1) {   // U = u1(1+ep+I, 1+J) * h_u(I, J), h_u = Ix(eta + H)
            const T b = bU(I, J);
            add(yb.u(1 + ep + I, 1 + J), b * hu(I, J));
            const T t = half * (b * ym.u(1 + ep + I, 1 + J));
            add(yb.e(I + 1, J), t); add(yb.e(I, J), t);
        }
        if (J <= ny + 1) {   // V = v1(I+1, J+1) * h_v(I, J), h_v = Iy(eta + H)
            const T b = bV(I, J);
            add(yb.v(I + 1, J + 1), b * hv(I, J));
            const T t = half * (b * ym.v(I + 1, J + 1));
            add(yb.e(I, J + 1), t); add(yb.e(I, J), t);
        }
    });
}

// d += a*x on one field, and x *= a
template <class T>
void field_axpy(Launcher& L, const A2<T>& d, T a, const A2<T>& x) {
    T* dp = d.d;
    const T* xp = x.d;
    L.d1((long long)d.size(), [=] __host__ __device__(long long i) { dp[i] += a * xp[i]; });
}
template <class T>
void field_scale(Launcher& L, const A2<T>& x, T a) {
    T* xp = x.d;
    L.d1((long long)x.size(), [=] __host__ __device__(long long i) { xp[i] = a * xp[i]; });
}

// d = x*a + y*b over whole states (cxayb!, src/time_integration.jl:293-305)
template <class T>
void combine(Launcher& L, const State<T>& d, T x, const State<T>& a, T y, const State<T>& b) {
    T* dp = d.base;
    const T* ap = a.base;
    const T* bp = b.base;
    L.d1((long long)d.elems, [=] __host__ __device__(long long i) { dp[i] = x * ap[i] + y * bp[i]; });
}

// ------------------------------------------------------------ tail, forward
// bottom_drag! (src/bottom_drag.jl:2-119), diffusion! (src/diffusion.jl:2-218)
// and add_drag_diff_tendencies! (src/diffusion.jl:221-251) on Z; the result
// goes to *Xs (eta copied), then ghost_points_uv! (src/time_integration.jl:231).
// With Xs null only the intermediates the reverse tail reads are formed.
template <class T>
void tail_fwd(Launcher& L, const Work<T>& w, const State<T>& Zs, const State<T>* Xs) {
    const A2<T> u = Zs.u, v = Zs.v, e = Zs.e, H = w.H;
    const A2<T> thu = w.thu, thv = w.thv, sKE = w.sKE, Lu = w.Lu, Lv = w.Lv, sDT = w.sDT, sDS = w.sDS, DSq = w.DSq;
    const int nx = w.nx, ny = w.ny, ep = w.ep, drag = w.drag;
    const bool smag = w.diff == SW_DIFF_SMAGORINSKY;
    L.d2(nx + 4, ny + 4, [=] __host__ __device__(int i, int j) {
        const T half = T(0.5);
        auto h = [&](int a, int b) { return e(a, b) + H(a, b); };
        if (drag == SW_DRAG_QUADRATIC) {
            if (i <= nx + 1 && j <= ny + 2) thu(i, j) = half * (h(i + 1, j) + h(i, j));
            if (i <= nx + 2 && j <= ny + 1) thv(i, j) = half * (h(i, j + 1) + h(i, j));
            if (i <= nx + 2 && j <= ny + 2) {
                const int a = i + ep, b = j + 1;
                const T KEu = half * (u(a + 1, b) * u(a + 1, b) + u(a, b) * u(a, b));
                const T KEv = half * (v(i + 1, j + 1) * v(i + 1, j + 1) + v(i + 1, j) * v(i + 1, j));
                sKE(i, j) = sqrt_(KEu + KEv);
            }
        }
        if (i <= Lu.m && j <= Lu.n) {   // ∇² (src/gradients.jl:39)
            const T c = u(i + 1, j + 1);
            Lu(i, j) = ((u(i, j + 1) - c) + (u(i + 2, j + 1) - c)) + ((u(i + 1, j) - c) + (u(i + 1, j + 2) - c));
        }
        if (i <= Lv.m && j <= Lv.n) {
            const T c = v(i + 1, j + 1);
            Lv(i, j) = ((v(i, j + 1) - c) + (v(i + 2, j + 1) - c)) + ((v(i + 1, j) - c) + (v(i + 1, j + 2) - c));
        }
        if (smag) {
            if (i <= nx + 2 && j <= ny + 2) {      // DT (src/diffusion.jl:88-97)
                const T s = (u(i + ep + 1, j + 1) - u(i + ep, j + 1)) + (v(i + 1, j + 1) - v(i + 1, j));
                sDT(i, j) = s;
            }
            if (i <= nx + 3 && j <= ny + 3) {      // DS_q (src/diffusion.jl:72-80)
                const T s = (u(i + ep, j + 1) - u(i + ep, j)) + (v(i + 1, j) - v(i, j));
                sDS(i, j) = s;
                DSq(i, j) = s * s;
            }
        }
    });
    const A2<T> dLudx = w.dLudx, dLudy = w.dLudy, dLvdx = w.dLvdx, dLvdy = w.dLvdy, sKEu = w.sKEu, sKEv = w.sKEv,
                rS = w.rS, nuS = w.nuS;
    const T cSmag = w.cSmag;
    L.d2(nx + 4, ny + 4, [=] __host__ __device__(int i, int j) {
        const T half = T(0.5), quarter = T(0.25);
        if (i <= dLudx.m && j <= dLudx.n) dLudx(i, j) = Lu(i + 1, j) - Lu(i, j);
        if (i <= dLudy.m && j <= dLudy.n) dLudy(i, j) = Lu(i, j + 1) - Lu(i, j);
        if (i <= dLvdx.m && j <= dLvdx.n) dLvdx(i, j) = Lv(i + 1, j) - Lv(i, j);
        if (i <= dLvdy.m && j <= dLvdy.n) dLvdy(i, j) = Lv(i, j + 1) - Lv(i, j);
        if (drag == SW_DRAG_QUADRATIC) {
            if (i <= nx + 1 && j <= ny + 2) sKEu(i, j) = half * (sKE(i + 1, j) + sKE(i, j));
            if (i <= nx + 2 && j <= ny + 1) sKEv(i, j) = half * (sKE(i, j + 1) + sKE(i, j));
        }
        if (smag && i <= nx + 2 && j <= ny + 2) {
            const T DS = quarter * (DSq(i, j) + DSq(i + 1, j)) + quarter * (DSq(i, j + 1) + DSq(i + 1, j + 1));
            const T DT = sDT(i, j) * sDT(i, j);
            const T r = sqrt_(DS + DT);
            rS(i, j) = r;
            nuS(i, j) = cSmag * r;
        }
    });
    const A2<T> Bu = w.Bu, Bv = w.Bv, nuSq = w.nuSq, S11 = w.S11, S12 = w.S12, S21 = w.S21, S22 = w.S22;
    const T cD = w.cD, rD = w.rD, nuB = w.nuB;
    L.d2(nx + 2, ny + 2, [=] __host__ __device__(int i, int j) {
        const T quarter = T(0.25);
        if (i <= nx + 1 && j <= ny + 2) {
            if (drag == SW_DRAG_QUADRATIC) Bu(i, j) = cD * sKEu(i, j) * u(i + 1 + ep, j + 1) / thu(i, j);
            else if (drag == SW_DRAG_LINEAR) Bu(i, j) = rD * u(i + 1 + ep, j + 1);
            else Bu(i, j) = T(0);
        }
        if (i <= nx + 2 && j <= ny + 1) {
            if (drag == SW_DRAG_QUADRATIC) Bv(i, j) = cD * sKEv(i, j) * v(i + 1, j + 1) / thv(i, j);
            else if (drag == SW_DRAG_LINEAR) Bv(i, j) = rD * v(i + 1, j + 1);
            else Bv(i, j) = T(0);
        }
        T nq = T(0);   // nuSmag_q at (i, j), used by S12 and S21 at the same point
        if (smag && i <= nx + 1 && j <= ny + 1) {
            nq = quarter * (nuS(i, j) + nuS(i + 1, j)) + quarter * (nuS(i, j + 1) + nuS(i + 1, j + 1));
            nuSq(i, j) = nq;
        }
        // viscous tensor (src/diffusion.jl:126-218)
        if (i <= S11.m && j <= S11.n) S11(i, j) = smag ? nuS(i + 1 - ep, j) * dLudx(i, j) : nuB * dLudx(i, j);
        if (i <= S12.m && j <= S12.n) S12(i, j) = smag ? nq * dLudy(i + ep, j) : nuB * dLudy(i + ep, j);
        if (i <= S21.m && j <= S21.n) S21(i, j) = smag ? nq * dLvdx(i, j) : nuB * dLvdx(i, j);
        if (i <= S22.m && j <= S22.n) S22(i, j) = smag ? nuS(i, j + 1) * dLvdy(i, j) : nuB * dLvdy(i, j);
    });
    if (!Xs) return;
    const int nux = w.nux, nuy = w.nuy, nvx = w.nvx, nvy = w.nvy;
    const T Dt = w.Dt_diff;
    const A2<T> xu = Xs->u, xv = Xs->v, xe = Xs->e;
    L.d2(nx + 4, ny + 4, [=] __host__ __device__(int I, int J) {
        if (I <= u.m && J <= u.n) {
            T r = u(I, J);
            if (I >= 3 && I <= nux + 2 && J >= 3 && J <= nuy + 2) {
                const int i = I - 2, j = J - 2;
                const T LLu1 = S11(i + 1, j + 1) - S11(i, j + 1);
                const T LLu2 = S12(i + 1 - ep, j + 1) - S12(i + 1 - ep, j);
                r += Dt * (Bu(i + 1 - ep, j + 1) + LLu1 + LLu2);
            }
            xu(I, J) = r;
        }
        if (I <= v.m && J <= v.n) {
            T r = v(I, J);
            if (I >= 3 && I <= nvx + 2 && J >= 3 && J <= nvy + 2) {
                const int i = I - 2, j = J - 2;
                const T LLv1 = S21(i + 1, j + 1) - S21(i, j + 1);
                const T LLv2 = S22(i + 1, j + 1) - S22(i + 1, j);
                r += Dt * (Bv(i + 1, j + 1) + LLv1 + LLv2);
            }
            xv(I, J) = r;
        }
        if (I <= e.m && J <= e.n) xe(I, J) = e(I, J);
    });
    ghost(L, w, *Xs, true);
}

// ------------------------------------------------------------ tail, reverse
// On entry Xb holds the adjoint of the tail's output before ghost_points_uv!
// (already transposed); on return it holds the adjoint of Z.
template <class T>
void tail_rev(Launcher& L, const Work<T>& w, const State<T>& Zs, const State<T>& Xb) {
    const A2<T> u = Zs.u, v = Zs.v;
    const State<T> zb = Xb;
    const int nx = w.nx, ny = w.ny, nux = w.nux, nuy = w.nuy, nvx = w.nvx, nvy = w.nvy, ep = w.ep, drag = w.drag;
    const bool smag = w.diff == SW_DIFF_SMAGORINSKY;
    const T Dt = w.Dt_diff;
    const A2<T> bBu = w.bBu, bBv = w.bBv, bS11 = w.bS11, bS12 = w.bS12, bS21 = w.bS21, bS22 = w.bS22;
    L.zero(w.tail_adj, w.tail_adj_elems * sizeof(T));
    // add_drag_diff_tendencies^T and dx/dy^T of the stress tensor
    L.d2(nx, ny, [=] __host__ __device__(int i, int j) {
        if (i <= nux && j <= nuy) {
            const T t = Dt * zb.u(i + 2, j + 2);
            bBu(i + 1 - ep, j + 1) += t;
            add(bS11(i + 1, j + 1), t); add(bS11(i, j + 1), -t);
            add(bS12(i + 1 - ep, j + 1), t); add(bS12(i + 1 - ep, j), -t);
        }
        if (i <= nvx && j <= nvy) {
            const T t = Dt * zb.v(i + 2, j + 2);
            bBv(i + 1, j + 1) += t;
            add(bS21(i + 1, j + 1), t); add(bS21(i, j + 1), -t);
            add(bS22(i + 1, j + 1), t); add(bS22(i + 1, j), -t);
        }
    });
    const A2<T> nuS = w.nuS, nuSq = w.nuSq, dLudx = w.dLudx, dLudy = w.dLudy, dLvdx = w.dLvdx, dLvdy = w.dLvdy;
    const A2<T> thu = w.thu, thv = w.thv, sKEu = w.sKEu, sKEv = w.sKEv, Bu = w.Bu, Bv = w.Bv;
    const A2<T> bnuS = w.bnuS, bLu = w.bLu, bLv = w.bLv, bsKE = w.bsKE;
    const T cD = w.cD, rD = w.rD, nuB = w.nuB;
    // viscous tensor^T and bottom drag^T; the adjoints these form alone (of the
    // Laplacians' gradients, nuSmag_q, sqrtKE_u/v and h_u/h_v at this point) go
    // straight through their dx/dy^T, Ixy^T, Ix/Iy^T
    L.d2(nx + 2, ny + 2, [=] __host__ __device__(int i, int j) {
        const T half = T(0.5), quarter = T(0.25);
        T nq = T(0);   // adjoint of nuSmag_q(i, j)
        if (i <= bS11.m && j <= bS11.n) {
            const T s = bS11(i, j);
            T t;
            if (smag) { add(bnuS(i + 1 - ep, j), s * dLudx(i, j)); t = s * nuS(i + 1 - ep, j); }
            else t = s * nuB;
            add(bLu(i + 1, j), t); add(bLu(i, j), -t);            // dLudx = dx(Lu)
        }
        if (i <= bS12.m && j <= bS12.n) {
            const T s = bS12(i, j);
            T t;
            if (smag) { nq += s * dLudy(i + ep, j); t = s * nuSq(i, j); }
            else t = s * nuB;
            add(bLu(i + ep, j + 1), t); add(bLu(i + ep, j), -t);  // dLudy = dy(Lu)
        }
        if (i <= bS21.m && j <= bS21.n) {
            const T s = bS21(i, j);
            T t;
            if (smag) { nq += s * dLvdx(i, j); t = s * nuSq(i, j); }
            else t = s * nuB;
            add(bLv(i + 1, j), t); add(bLv(i, j), -t);            // dLvdx = dx(Lv)
        }
        if (i <= bS22.m && j <= bS22.n) {
            const T s = bS22(i, j);
            T t;
            if (smag) { add(bnuS(i, j + 1), s * dLvdy(i, j)); t = s * nuS(i, j + 1); }
            else t = s * nuB;
            add(bLv(i, j + 1), t); add(bLv(i, j), -t);            // dLvdy = dy(Lv)
        }
        if (smag && i <= nx + 1 && j <= ny + 1) {                // nuSmag_q = Ixy(nuSmag)
            const T t = quarter * nq;
            add(bnuS(i, j), t); add(bnuS(i + 1, j), t); add(bnuS(i, j + 1), t); add(bnuS(i + 1, j + 1), t);
        }
        if (i <= nx + 1 && j <= ny + 2) {
            const T bb = bBu(i, j);
            const T uu = u(i + 1 + ep, j + 1);
            if (drag == SW_DRAG_QUADRATIC) {     // Bu = cD*s*u/h
                const T hh = thu(i, j);
                const T ts = half * (bb * (cD * uu / hh));        // sqrtKE_u = Ix(sqrtKE)
                add(bsKE(i + 1, j), ts); add(bsKE(i, j), ts);
                add(zb.u(i + 1 + ep, j + 1), bb * (cD * sKEu(i, j) / hh));
                const T th = half * -(bb * Bu(i, j) / hh);        // h_u = Ix(eta + H)
                add(zb.e(i + 1, j), th); add(zb.e(i, j), th);
            } else if (drag == SW_DRAG_LINEAR) {
                add(zb.u(i + 1 + ep, j + 1), bb * rD);
            }
        }
        if (i <= nx + 2 && j <= ny + 1) {
            const T bb = bBv(i, j);
            const T vv = v(i + 1, j + 1);
            if (drag == SW_DRAG_QUADRATIC) {
                const T hh = thv(i, j);
                const T ts = half * (bb * (cD * vv / hh));        // sqrtKE_v = Iy(sqrtKE)
                add(bsKE(i, j + 1), ts); add(bsKE(i, j), ts);
                add(zb.v(i + 1, j + 1), bb * (cD * sKEv(i, j) / hh));
                const T th = half * -(bb * Bv(i, j) / hh);        // h_v = Iy(eta + H)
                add(zb.e(i, j + 1), th); add(zb.e(i, j), th);
            } else if (drag == SW_DRAG_LINEAR) {
                add(zb.v(i + 1, j + 1), bb * rD);
            }
        }
    });
    const A2<T> rS = w.rS, sKE = w.sKE, sDT = w.sDT, sDS = w.sDS, bDSq = w.bDSq;
    const T cSmag = w.cSmag;
    const A2<T> Lu = w.Lu, Lv = w.Lv;
    // sqrt^T (Smagorinsky coefficient, then DT^T and Ixy^T of DS at the same
    // point; sqrtKE through KE = Ix(u^2) + Iy(v^2)) and ∇²^T
    L.d2(nx + 4, ny + 4, [=] __host__ __device__(int i, int j) {
        const T zero = T(0), two = T(2), quarter = T(0.25);
        if (smag && i <= nx + 2 && j <= ny + 2) {
            const T r = rS(i, j);
            const T d = r > zero ? bnuS(i, j) * cSmag / (two * r) : zero;   // adjoint of DS and of DT
            const T t = two * sDT(i, j) * d;                                 // DT = s^2, s = dudx + dvdy
            add(zb.u(i + ep + 1, j + 1), t); add(zb.u(i + ep, j + 1), -t);
            add(zb.v(i + 1, j + 1), t); add(zb.v(i + 1, j), -t);
            const T q4 = quarter * d;                                        // DS = Ixy(DS_q)
            add(bDSq(i, j), q4); add(bDSq(i + 1, j), q4); add(bDSq(i, j + 1), q4); add(bDSq(i + 1, j + 1), q4);
        }
        if (drag == SW_DRAG_QUADRATIC && i <= nx + 2 && j <= ny + 2) {
            const T r = sKE(i, j);
            const T k = r > zero ? bsKE(i, j) / (two * r) : zero;
            const int a = i + ep, b = j + 1;    // d/du of half*(u(a+1)^2 + u(a)^2) is u
            add(zb.u(a + 1, b), k * u(a + 1, b)); add(zb.u(a, b), k * u(a, b));
            add(zb.v(i + 1, j + 1), k * v(i + 1, j + 1)); add(zb.v(i + 1, j), k * v(i + 1, j));
        }
        if (i <= Lu.m && j <= Lu.n) {
            const T t = bLu(i, j);
            add(zb.u(i, j + 1), t); add(zb.u(i + 2, j + 1), t); add(zb.u(i + 1, j), t); add(zb.u(i + 1, j + 2), t);
            add(zb.u(i + 1, j + 1), -(T(4) * t));
        }
        if (i <= Lv.m && j <= Lv.n) {
            const T t = bLv(i, j);
            add(zb.v(i, j + 1), t); add(zb.v(i + 2, j + 1), t); add(zb.v(i + 1, j), t); add(zb.v(i + 1, j + 2), t);
            add(zb.v(i + 1, j + 1), -(T(4) * t));
        }
    });
    if (!smag) return;
    // DS_q^T (s^2 with s = dudy + dvdx)
    L.d2(nx + 3, ny + 3, [=] __host__ __device__(int i, int j) {
        const T t = T(2) * sDS(i, j) * bDSq(i, j);
        add(zb.u(i + ep, j + 1), t); add(zb.u(i + ep, j), -t);
        add(zb.v(i + 1, j), t); add(zb.v(i, j), -t);
    });
}

// ------------------------------------------------------------ whole steps
template <class T>
void copy_state(Launcher& L, const State<T>& dst, const State<T>& src) {
    L.copy(dst.base, src.base, src.elems * sizeof(T));
}

// one time step X -> X (src/time_integration.jl:45-243, RK branch); leaves the
// stage inputs in Ys, the tail input in Z and the last stage's intermediates.
template <class T>
void fwd_step_ssp(Launcher& L, const Work<T>& w, bool tail);

// the end of a step (src/time_integration.jl:204-233): after ghost_points! of
// the RK sum, drag and diffusion on steps i with i % nstep_diff == 0 (tail),
// else the ghosted sum is the new state
template <class T>
void step_end(Launcher& L, const Work<T>& w, bool tail) {
    ghost(L, w, w.Z, GH_ALL);
    if (tail) tail_fwd(L, w, w.Z, &w.X);
    else copy_state(L, w.X, w.Z);
}

template <class T>
void fwd_step(Launcher& L, const Work<T>& w, bool tail = true) {
    if (w.ssp) { fwd_step_ssp(L, w, tail); return; }
    copy_state(L, w.Ys[0], w.X);
    ghost(L, w, w.Ys[0], false);
    copy_state(L, w.Z, w.Ys[0]);
    for (int k = 1; k <= w.rko; k++) {
        if (k > 1) ghost(L, w, w.Ys[k - 1], false);
        stage_fwd(L, w, w.Ys[k - 1]);
        stage_update(L, w, k, w.Ys[k - 1], w.Ys[0], k < w.rko ? &w.Ys[k] : nullptr, w.Z);
    }
    step_end(L, w, tail);
}

// adjoint of one step: on entry Xb holds the adjoint of the step's output and
// either X its input state (stored = false: the step is recomputed) or Ys and
// Z its stage inputs and tail input as the forward sweep kept them (stored =
// true: only the passes' intermediates are recomputed).  On return Xb holds
// the adjoint of the input, and bFx has this step's forcing adjoint added.
// SSPRK3's snapshot u0 at its stage kn: the state after sub-stage rki = mn
// (sub-stage k = mn - 1), or the step's start when mn = 1
template <class T>
const State<T>& ssp3_snapshot(const Work<T>& w) {
    return w.s3_mn <= 1 ? w.Ys[0] : w.Ys[2 * (w.s3_mn - 1) + 1];
}

// one SSPRK2, SSPRK3 or 4SSPRK3 time step X -> X (src/time_integration.jl:80-196, 204-243)
template <class T>
void fwd_step_ssp(Launcher& L, const Work<T>& w, bool tail) {
    copy_state(L, w.Ys[0], w.X);
    ghost(L, w, w.Ys[0], GH_ALL);
    copy_state(L, w.Ys[1], w.Ys[0]);
    for (int k = 1; k <= w.rks; k++) {
        const State<T>&yp = w.Ys[2 * k - 1], &ym = w.Ys[2 * k], &yn = w.Ys[2 * k + 1];
        if (k > 1) ghost(L, w, yp, w.four ? GH_ALL : GH_ETA);
        stage_fwd(L, w, yp);
        const State<T>* zs = (w.ssp3 && k + 1 == w.s3_kn) ? &ssp3_snapshot(w) : nullptr;
        ssp_mom(L, w, yp, ym, zs);
        ghost(L, w, ym, GH_UV);
        ssp_cont(L, w, ym, yn, zs);
        if (w.four && k == 3) combine(L, yn, w.ssp_a, w.Ys[0], w.ssp_b, yn);   // 2/3 X + 1/3 X1 (cxayb!)
        // SSPRK3: ghost_points_eta! before the snapshot copy and the final copy (:148-152)
        if (w.ssp3 && (k + 1 == w.s3_mn || k == w.rks)) ghost(L, w, yn, GH_ETA);
    }
    if (w.four || w.ssp3) copy_state(L, w.Z, w.Ys[2 * w.rks + 1]);
    else combine(L, w.Z, w.ssp_a, w.Ys[0], w.ssp_b, w.Ys[2 * w.rks + 1]);
    step_end(L, w, tail);
}

template <class T>
void adj_step_ssp(Launcher& L, const Work<T>& w, bool stored, bool tail) {
    if (!stored) fwd_step_ssp(L, w, tail);
    else if (tail && !w.tail_kept) tail_fwd(L, w, w.Z, (const State<T>*)nullptr);
    if (tail) {
        ghostT(L, w, w.Xb, GH_UV);
        tail_rev(L, w, w.Z, w.Xb);
    }
    ghostT(L, w, w.Xb, GH_ALL);    // Xb: adjoint of X0 = a*Ys[0] + b*Ys[2 RKs + 1]
    const State<T>& Yb = w.Yb[0];
    const State<T>& Zb = w.Yb[1];  // SSPRK3: adjoint of the snapshot u0
    if (w.four || w.ssp3) {   // X0 is the last sub-stage's result
        copy_state(L, Yb, w.Xb);
        L.zero(w.acc.base, w.acc.elems * sizeof(T));
        if (w.ssp3) {
            L.zero(Zb.base, Zb.elems * sizeof(T));
            ghostT(L, w, Yb, GH_ETA);   // the last sub-stage's ghost_points_eta!
        }
    } else {        // X0 = a*Ys[0] + b*Ys[2 RKs + 1]
        combine(L, w.acc, w.ssp_a, w.Xb, T(0), w.Xb);
        combine(L, Yb, w.ssp_b, w.Xb, T(0), w.Xb);
    }
    // d(new state)/d(tendency): Δt_Δs or Δt_Δn, or Δt_Δ/2 for the averaged 4SSPRK3 update
    const T coef = w.four ? T(0.5) * w.cssp : w.cssp;
    for (int k = w.rks; k >= 1; k--) {
        const State<T>&yp = w.Ys[2 * k - 1], &ym = w.Ys[2 * k];
        if (w.four && k == 3) {   // Yn = 2/3 X + 1/3 Yn
            combine(L, w.acc, T(1), w.acc, w.ssp_a, Yb);
            combine(L, Yb, w.ssp_b, Yb, T(0), Yb);
        }
        if (w.ssp3 && k + 1 == w.s3_mn && k < w.rks) {
            // the state after this sub-stage was eta-ghosted in place and copied
            // to the snapshot: its adjoint gathers the snapshot's
            combine(L, Yb, T(1), Yb, T(1), Zb);
            L.zero(Zb.base, Zb.elems * sizeof(T));
            ghostT(L, w, Yb, GH_ETA);
        }
        // stage kn: new = kna*old + knb*snapshot + Δt_Δnc*d; the old value's
        // adjoint is scaled by kna first, so the tendency's coefficient becomes
        // Δt_Δnc/kna on the scaled adjoint
        const bool kn = w.ssp3 && k + 1 == w.s3_kn;
        const T ck = kn ? w.s3_cnc / w.s3_kna : coef;
        stage_fwd(L, w, yp);                              // h_u, h_v and the rhs intermediates of sub-stage k
        if (kn) {
            field_axpy(L, Zb.e, w.s3_knb, Yb.e);
            field_scale(L, Yb.e, w.s3_kna);
        }
        ssp_cont_rev(L, w, ym, Yb, ck);                   // Yb: adjoint of Ym
        ghostT(L, w, Yb, GH_UV);
        if (kn) {
            field_axpy(L, Zb.u, w.s3_knb, Yb.u);
            field_axpy(L, Zb.v, w.s3_knb, Yb.v);
            field_scale(L, Yb.u, w.s3_kna);
            field_scale(L, Yb.v, w.s3_kna);
        }
        stage_rev(L, w, 1, yp, Yb, (const State<T>*)nullptr, Yb, true, ck);   // adjoint of Yp
        if (k > 1) ghostT(L, w, Yb, w.four ? GH_ALL : GH_ETA);
    }
    if (w.ssp3 && w.s3_mn <= 1) combine(L, w.acc, T(1), w.acc, T(1), Zb);   // the snapshot was the start state
    const T* src = Yb.base;
    T* dst = w.acc.base;
    L.d1((long long)Yb.elems, [=] __host__ __device__(long long i) { dst[i] += src[i]; });
    ghostT(L, w, w.acc, GH_ALL);
    copy_state(L, w.Xb, w.acc);
}

template <class T>
void adj_step(Launcher& L, const Work<T>& w, bool stored, bool tail = true) {
    if (w.ssp) { adj_step_ssp(L, w, stored, tail); return; }
    if (!stored) fwd_step(L, w, tail);
    else if (tail && !w.tail_kept) tail_fwd(L, w, w.Z, (const State<T>*)nullptr);
    if (tail) {
        ghostT(L, w, w.Xb, GH_UV);
        tail_rev(L, w, w.Z, w.Xb);
    }
    ghostT(L, w, w.Xb, false);     // Xb is now the adjoint of the RK sum X0
    copy_state(L, w.acc, w.Xb);  // X0 starts as the ghosted input
    const State<T>* Wb = nullptr;
    for (int k = w.rko; k >= 1; k--) {
        const State<T>& Yb = w.Yb[k % 2];
        L.zero(Yb.base, Yb.elems * sizeof(T));
        if (stored || k < w.rko) stage_fwd(L, w, w.Ys[k - 1]);   // after fwd_step the last stage's are in place
        stage_rev(L, w, k, w.Ys[k - 1], w.Xb, Wb, Yb);
        if (k > 1) ghostT(L, w, Yb, false);             // Ys[k-1] = ghost(Y1)
        const T* src = Yb.base;
        T* dst = w.acc.base;
        L.d1((long long)Yb.elems, [=] __host__ __device__(long long i) { dst[i] += src[i]; });
        Wb = &Yb;
    }
    ghostT(L, w, w.acc, false);    // the step starts with ghost_points!
    copy_state(L, w.Xb, w.acc);
}

// The adjoint of an RK step from its kept stage inputs, with every stage's
// intermediates in a buffer set of its own (ws[k-1] for stage k: copies of w
// with their own hu .. Uv): stage_fwd of all stages runs on a side branch
// (`side`, forked and joined with the events evf, evj) while the main branch
// transposes the tail; the stage transposes then read them.  acc and the two
// stage adjoints are set by one pass, the next stage adjoint is cleared by
// the accumulation that frees it, and the last accumulation writes Xb.  Each
// stage has its own scratch adjoints too (one block, ws_adj, cleared at the
// fork).  The sums are those of adj_step, in the same order.
template <class T>
void adj_step_split(Launcher& L, Launcher* side, cudaEvent_t evf, cudaEvent_t evj, const Work<T>& w,
                    const Work<T>* ws, T* ws_adj, size_t ws_adj_elems, bool tail) {
    const bool fork = !L.host && side != nullptr;
    if (fork) {
        cudaEventRecord(evf, L.s);
        cudaStreamWaitEvent(side->s, evf, 0);
    }
    Launcher& S = fork ? *side : L;
    S.zero(ws_adj, ws_adj_elems * sizeof(T));   // every stage's scratch adjoints bU .. bUv
    for (int k = 1; k <= w.rko; k++) stage_fwd(S, ws[k - 1], w.Ys[k - 1]);
    if (fork) cudaEventRecord(evj, side->s);
    if (tail) {
        if (!w.tail_kept) tail_fwd(L, w, w.Z, (const State<T>*)nullptr);
        ghostT(L, w, w.Xb, GH_UV);
        tail_rev(L, w, w.Z, w.Xb);
    }
    ghostT(L, w, w.Xb, GH_ALL);    // Xb is now the adjoint of the RK sum X0
    {
        T* acc = w.acc.base; T* y0 = w.Yb[0].base; T* y1 = w.Yb[1].base;
        const T* xb = w.Xb.base;
        L.d1((long long)w.Xb.elems, [=] __host__ __device__(long long i) {
            acc[i] = xb[i];
            y0[i] = T(0);
            y1[i] = T(0);
        });
    }
    if (fork) cudaStreamWaitEvent(L.s, evj, 0);
    const State<T>* Wb = nullptr;
    for (int k = w.rko; k >= 1; k--) {
        const State<T>& Yb = w.Yb[k % 2];
        stage_rev(L, ws[k - 1], k, w.Ys[k - 1], w.Xb, Wb, Yb);
        T* acc = w.acc.base;
        const T* yb = Yb.base;
        if (k > 1) {
            ghostT(L, w, Yb, GH_ALL);            // Ys[k-1] = ghost(Y1)
            T* nxt = w.Yb[(k + 1) % 2].base;     // Wb of this stage, the next stage's adjoint
            L.d1((long long)Yb.elems, [=] __host__ __device__(long long i) {
                acc[i] += yb[i];
                nxt[i] = T(0);
            });
        } else {
            T* xb = w.Xb.base;
            L.d1((long long)Yb.elems, [=] __host__ __device__(long long i) { xb[i] = acc[i] + yb[i]; });
        }
        Wb = &Yb;
    }
    ghostT(L, w, w.Xb, GH_ALL);    // the step starts with ghost_points!
}

// J = sum (eta - obs)^2 over the interior, the differences and squares in
// FP64, as row sums (out[j-1]); and the seed eb = dJ/deta = 2 (eta - obs) on
// the interior, rounded once to T
template <class T>
void cost_seed(Launcher& L, const A2<T>& ef, const A2<T>& obs, const A2<T>& eb, double* out) {
    const A2<T> e = ef, o = obs, b = eb;
    const int nx = obs.m;
    L.d1(obs.n, [=] __host__ __device__(long long jj) {
        const int j = (int)jj + 1;
        double acc = 0.0;
        for (int i = 1; i <= nx; i++) {
            const double d = (double)e(i + 1, j + 1) - (double)o(i, j);
            acc += d * d;
            b(i + 1, j + 1) = (T)(2.0 * d);
        }
        out[jj] = acc;
    });
}

}  // namespace swa

// ================================================================ host side
namespace {

using namespace swa;

struct AdjCfgError {
    int code;
    const char* why;
};

AdjCfgError adjoint_check(const sw_config& c) {
    if (c.abi_version != SWB200_ABI_VERSION) return {SW_ERR_ARG, "abi_version"};
    if (c.halo != 2 || c.haloeta != 1 || c.halosstx != 1 || c.halossty != 0) return {SW_ERR_ARG, "halo sizes"};
    if (c.nx < 8 || c.ny < 8) return {SW_ERR_ARG, "grid smaller than 8 x 8"};
    if (c.T != c.Tprog || (c.T != SW_FLOAT32 && c.T != SW_FLOAT64) || c.Tcomm != c.T)
        return {SW_ERR_UNSUPPORTED, "the adjoint computes in T = Tprog = Tcomm, Float32 or Float64"};
    if (!((c.time_scheme == SW_RK && c.RKo >= 2 && c.RKo <= 4) || (c.time_scheme == SW_SSPRK2 && c.RKs >= 2 && c.RKs <= 4) ||
          (c.time_scheme == SW_SSPRK3 && c.ssp_n >= 2 && c.ssp_n <= 3) || c.time_scheme == SW_4SSPRK3))
        return {SW_ERR_UNSUPPORTED, "the adjoint follows RK2/3/4, SSPRK2 with 2-4 sub-stages, SSPRK3 with n = 2 or 3 and 4SSPRK3"};
    if (c.dynamics == SW_NONLINEAR && c.nstep_advcor != 0)
        return {SW_ERR_UNSUPPORTED, "the adjoint follows nonlinear dynamics with nstep_advcor = 0"};
    if (c.nstep_diff < 1) return {SW_ERR_ARG, "nstep_diff"};
    if (c.surface_forcing && c.surface_relax) return {SW_ERR_ARG, "surface relaxation and forcing together"};
    if (c.storage != SW_STORE_NATIVE) return {SW_ERR_UNSUPPORTED, "the adjoint keeps the native storage"};
    return {SW_OK, nullptr};
}

// The work buffers, the checkpoint slots, the two captured step graphs
// (forward step, adjoint step) and the checkpoint schedule.  With host = true
// (the host check build only) the same passes run in host loops on host
// memory.
template <class T>
struct Adjoint {
    Work<T> w;
    // Two-level schedule, overlapped: a second forward worker (its own state,
    // stage states, intermediates and forcing multipliers; the static fields
    // are shared) recomputes segment j - 1 on stream s2 while s reverses
    // segment j, each segment's records in one of two halves of `records`
    Work<T> wf;
    bool overlap = false;
    // RK adjoint steps from kept stage inputs (adj_step_split): one set of
    // stage intermediates per stage (ws[k-1]), computed on the side stream s3
    // of the step graph's capture
    Work<T> ws[4];
    T* ws_adj = nullptr;        // the stages' scratch adjoints, one block
    size_t ws_adj_elems = 0;
    bool split = false;
    cudaStream_t s3 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool host = false;
    std::vector<void*> blocks;
    cudaStream_t s = nullptr, s2 = nullptr;
    // step graphs, by whether the step ends with drag and diffusion ([1]) or not ([0])
    cudaGraphExec_t g_fwd[2] = {}, g_adj[2] = {}, g_adj_st[2] = {}, g_fwd2[2] = {};
    int nstep_diff = 1;
    T* step_force = nullptr;    // per step k: Fxt, Fyt, Fetat at t = k*dtint (pinned host memory)
    T* records = nullptr;       // per step: Ys[0..nst-1] and Z as the forward sweep left them (and the tail intermediates)
    size_t rec_elems = 0;       // elements of a record
    bool stored = false;
    std::vector<State<T>> slots;
    long long fwd_steps = 0, adj_steps = 0;
    int launches_fwd = 0, launches_adj = 0;
    std::string err;

    ~Adjoint() {
        if (s) cudaStreamSynchronize(s);
        if (s2) cudaStreamSynchronize(s2);
        if (step_force) { if (host) std::free(step_force); else cudaFreeHost(step_force); }
        for (int t = 0; t < 2; t++)
            for (cudaGraphExec_t g : {g_fwd[t], g_adj[t], g_adj_st[t], g_fwd2[t]})
                if (g) cudaGraphExecDestroy(g);
        for (void* p : blocks) {
            if (host) std::free(p); else cudaFree(p);
        }
        if (s) cudaStreamDestroy(s);
        if (s2) cudaStreamDestroy(s2);
        if (s3) cudaStreamDestroy(s3);
        for (cudaEvent_t x : {ev_fork, ev_join})
            if (x) cudaEventDestroy(x);
    }

    bool pdl = false;           // programmatic dependent launch of the passes (SWB200_ADJ_PDL=0: off)
    Launcher launcher() { Launcher L{s}; L.host = host; L.pdl = pdl; return L; }

    T* alloc(size_t elems) {
        const size_t bytes = std::max<size_t>(elems, 1) * sizeof(T);
        void* p = nullptr;
        if (host) p = std::calloc(1, bytes);
        else if (cudaMalloc(&p, bytes) != cudaSuccess) { p = nullptr; (void)cudaGetLastError(); }
        if (!p) return nullptr;
        blocks.push_back(p);
        return static_cast<T*>(p);
    }
    cudaError_t upload(void* dst, const void* src, size_t bytes) {
        if (host) { std::memcpy(dst, src, bytes); return cudaSuccess; }
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
    }
    cudaError_t download(void* dst, const void* src, size_t bytes) {
        if (host) { std::memcpy(dst, src, bytes); return cudaSuccess; }
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
    }
    cudaError_t zero(void* p, size_t bytes) {
        if (host) { std::memset(p, 0, bytes); return cudaSuccess; }
        return cudaMemsetAsync(p, 0, bytes, s);
    }
    void copy(const State<T>& dst, const State<T>& src) {
        Launcher L = launcher();
        copy_state(L, dst, src);
    }

    // arrays carved from one block, in declaration order (each padded to 32 elements)
    struct Carver {
        std::vector<std::pair<A2<T>*, std::pair<int, int>>> list;
        void add(A2<T>& a, int m, int n) { list.push_back({&a, {m, n}}); }
        static size_t padded(int m, int n) { return ((size_t)m * (size_t)n + 31) & ~(size_t)31; }
        size_t total() const {
            size_t t = 0;
            for (auto& x : list) t += padded(x.second.first, x.second.second);
            return t;
        }
        void place(T* base) {
            size_t o = 0;
            for (auto& x : list) {
                x.first->d = base + o;
                x.first->m = x.second.first;
                x.first->n = x.second.second;
                o += padded(x.second.first, x.second.second);
            }
        }
    };

    bool carve(Carver& cv, T** base = nullptr, size_t* elems = nullptr) {
        const size_t n = cv.total();
        T* b = alloc(n);
        if (!b) return false;
        cv.place(b);
        if (base) *base = b;
        if (elems) *elems = n;
        return zero(b, n * sizeof(T)) == cudaSuccess;
    }

    // n state slots in one block; on allocation failure n is halved (to 1)
    bool make_slots(int n) {
        for (; n >= 1; n /= 2) {
            std::vector<State<T>> sl(n);
            Carver cv;
            for (auto& x : sl) {
                cv.add(x.u, w.nux + 4, w.nuy + 4);
                cv.add(x.v, w.nvx + 4, w.nvy + 4);
                cv.add(x.e, w.nx + 2, w.ny + 2);
            }
            const size_t total = cv.total();
            void* p = nullptr;
            if (host) p = std::calloc(total, sizeof(T));
            else if (cudaMalloc(&p, total * sizeof(T)) != cudaSuccess) { p = nullptr; cudaGetLastError(); }
            if (!p) continue;
            blocks.push_back(p);
            cv.place(static_cast<T*>(p));
            for (auto& x : sl) {
                x.base = x.u.d;
                x.elems = Carver::padded(x.u.m, x.u.n) + Carver::padded(x.v.m, x.v.n) + Carver::padded(x.e.m, x.e.n);
            }
            slots = std::move(sl);
            return true;
        }
        return false;
    }

    bool make_state(State<T>& st) {
        Carver c;
        c.add(st.u, w.nux + 4, w.nuy + 4);
        c.add(st.v, w.nvx + 4, w.nvy + 4);
        c.add(st.e, w.nx + 2, w.ny + 2);
        return carve(c, &st.base, &st.elems);
    }

    static void add_stage_adj(Carver& cv, Work<T>& x) {
        const int nx = x.nx, ny = x.ny;
        cv.add(x.bU, nx + 1, ny + 2); cv.add(x.bV, nx + 2, ny + 1); cv.add(x.bp, nx + 2, ny + 2);
        cv.add(x.bqa, nx, ny); cv.add(x.bqb, nx + 1, ny); cv.add(x.bqc, nx + 1, ny); cv.add(x.bqd, nx, ny);
        cv.add(x.bq, nx + 1, ny + 1);
        cv.add(x.bqu, nx + 1, ny); cv.add(x.bqv, nx, ny + 1); cv.add(x.bVu, nx + 1, ny); cv.add(x.bUv, nx, ny + 1);
    }
    static void add_stage_inter(Carver& cv, Work<T>& x) {
        const int nx = x.nx, ny = x.ny;
        cv.add(x.hu, nx + 1, ny + 2); cv.add(x.hv, nx + 2, ny + 1); cv.add(x.hq, nx + 1, ny + 1);
        cv.add(x.U, nx + 1, ny + 2); cv.add(x.V, nx + 2, ny + 1); cv.add(x.q, nx + 1, ny + 1);
        cv.add(x.qa, nx, ny); cv.add(x.qb, nx + 1, ny); cv.add(x.qc, nx + 1, ny); cv.add(x.qd, nx, ny);
        cv.add(x.p, nx + 2, ny + 2);
        cv.add(x.qu, nx + 1, ny); cv.add(x.qv, nx, ny + 1); cv.add(x.Vu, nx + 1, ny); cv.add(x.Uv, nx, ny + 1);
    }

    // what a forward step writes: the state X, the stage states Ys and the
    // tail input Z and, right after them, the tail intermediates (one block:
    // one copy keeps a step's record), and the stage intermediates
    bool make_forward(Work<T>& x) {
        if (!make_state(x.X)) return false;
        const int nx = x.nx, ny = x.ny, nux = x.nux, nuy = x.nuy, nvx = x.nvx, nvy = x.nvy;
        {
            Carver cv;   // the stage states Ys[0..nst-1] and the tail input Z
            std::vector<State<T>*> st;
            for (int k = 0; k < x.nst; k++) st.push_back(&x.Ys[k]);
            st.push_back(&x.Z);
            for (State<T>* y : st) {
                cv.add(y->u, nux + 4, nuy + 4);
                cv.add(y->v, nvx + 4, nvy + 4);
                cv.add(y->e, nx + 2, ny + 2);
            }
            const size_t states = cv.total();
            // tail intermediates
            cv.add(x.thu, nx + 1, ny + 2); cv.add(x.thv, nx + 2, ny + 1); cv.add(x.sKE, nx + 2, ny + 2);
            cv.add(x.sKEu, nx + 1, ny + 2); cv.add(x.sKEv, nx + 2, ny + 1);
            cv.add(x.Bu, nx + 1, ny + 2); cv.add(x.Bv, nx + 2, ny + 1);
            cv.add(x.Lu, nux + 2, nuy + 2); cv.add(x.Lv, nvx + 2, nvy + 2);
            cv.add(x.dLudx, nux + 1, nuy + 2); cv.add(x.dLudy, nux + 2, nuy + 1);
            cv.add(x.dLvdx, nvx + 1, nvy + 2); cv.add(x.dLvdy, nvx + 2, nvy + 1);
            cv.add(x.sDT, nx + 2, ny + 2); cv.add(x.sDS, nvx + 3, nvy + 4); cv.add(x.DSq, nvx + 3, nvy + 4);
            cv.add(x.rS, nx + 2, ny + 2); cv.add(x.nuS, nx + 2, ny + 2); cv.add(x.nuSq, nx + 1, ny + 1);
            cv.add(x.S11, nux + 1, nuy + 2); cv.add(x.S12, nx + 1, ny + 1); cv.add(x.S21, nx + 1, ny + 1);
            cv.add(x.S22, nvx + 2, nvy + 1);
            size_t all = 0;
            if (!carve(cv, &x.stage_block, &all)) return false;
            x.stage_block_elems = states;
            x.tail_inter_elems = all - states;
            for (State<T>* y : st) {
                y->base = y->u.d;
                y->elems = Carver::padded(y->u.m, y->u.n) + Carver::padded(y->v.m, y->v.n) + Carver::padded(y->e.m, y->e.n);
            }
        }
        {
            Carver cv;   // stage intermediates
            add_stage_inter(cv, x);
            if (!carve(cv)) return false;
        }
        return true;
    }

    // want_store: keep nrecords steps' stage inputs (all steps, or one
    // segment); want_overlap: two segments' records and the second forward
    // worker (falls back to one segment's records without it)
    int setup(const sw_config& c, const sw_static& stt, bool want_store, long long nrecords, bool want_overlap) {
        if (!host && cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return SW_ERR_CUDA;
        const char* env_pdl = getenv("SWB200_ADJ_PDL");
        pdl = !host && !(env_pdl && env_pdl[0] == '0');
        w.nx = c.nx; w.ny = c.ny; w.ep = c.periodic ? 1 : 0;
        w.nux = w.ep ? c.nx : c.nx - 1; w.nuy = c.ny; w.nvx = c.nx; w.nvy = c.ny - 1;
        w.rko = c.RKo;
        w.four = c.time_scheme == SW_4SSPRK3;
        w.ssp3 = c.time_scheme == SW_SSPRK3;
        w.ssp = c.time_scheme == SW_SSPRK2 || w.four || w.ssp3;
        w.rks = w.four ? 4 : w.ssp3 ? c.ssp_s : c.RKs;
        w.cssp = (T)(w.four ? c.Dt_D : w.ssp3 ? c.ssp_Dt_Dn : c.Dt_Ds);
        w.s3_kn = c.ssp_kn; w.s3_mn = c.ssp_mn;
        w.s3_cnc = (T)c.ssp_Dt_Dnc; w.s3_kna = (T)c.ssp_kna; w.s3_knb = (T)c.ssp_knb;
        w.ssp_a = (T)(w.four ? 2.0 / 3.0 : 1.0 / c.RKs);
        w.ssp_b = (T)(w.four ? 1.0 / 3.0 : (double)(c.RKs - 1) / c.RKs);
        w.nst = w.ssp ? 2 * w.rks + 2 : w.rko;
        w.g = (T)c.g; w.cD = (T)c.cD; w.rD = (T)c.rD; w.cSmag = (T)c.cSmag; w.nuB = (T)c.nuB;
        w.Dt_diff = (T)c.Dt_diff; w.oma = (T)c.one_minus_alpha;
        for (int k = 0; k < 4; k++) w.RKa[k] = (T)c.RKaDt[k];
        for (int k = 0; k < 3; k++) w.RKb[k] = (T)c.RKbDt[k];
        w.drag = c.bottom_drag; w.diff = c.diffusion;
        w.sadourny = c.adv_scheme == SW_SADOURNY;
        w.linear = c.dynamics == SW_LINEAR;
        nstep_diff = c.nstep_diff;
        w.relax = c.surface_relax != 0;
        w.gamma = (T)c.gamma;
        w.forcing = c.surface_forcing != 0;
        w.timedep = c.seasonal_wind_x || c.seasonal_wind_y || w.forcing;
        const int nx = w.nx, ny = w.ny, nux = w.nux, nuy = w.nuy, nvx = w.nvx, nvy = w.nvy;
        {
            Carver cv;   // static fields and the forcing adjoint
            cv.add(w.H, nx + 2, ny + 2); cv.add(w.f_q, nx + 1, ny + 1); cv.add(w.Fx, nux, nuy); cv.add(w.Fy, nvx, nvy);
            cv.add(w.eta_ref, nx, ny); cv.add(w.Feta, nx, ny); cv.add(w.f_u, nux, nuy); cv.add(w.f_v, nvx, nvy);
            cv.add(w.bFx, nux, nuy);
            A2<T> fv;
            cv.add(fv, 4, 1);
            if (!carve(cv)) return SW_ERR_NOMEM;
            w.force = fv.d;
            const void* src[8] = {stt.H, stt.f_q, stt.Fx, stt.Fy, stt.eta_ref, stt.Feta, stt.f_u, stt.f_v};
            A2<T>* dst[8] = {&w.H, &w.f_q, &w.Fx, &w.Fy, &w.eta_ref, &w.Feta, &w.f_u, &w.f_v};
            for (int k = 0; k < 8; k++) {
                if ((k == 4 && !w.relax) || (k == 5 && !w.forcing) || (k >= 6 && !w.linear)) continue;
                if (!src[k]) return SW_ERR_ARG;
                if (upload(dst[k]->d, src[k], dst[k]->size() * sizeof(T)) != cudaSuccess) return SW_ERR_CUDA;
            }
        }
        if (!make_forward(w) || !make_state(w.Xb) || !make_state(w.acc) || !make_state(w.Yb[0]) || !make_state(w.Yb[1]))
            return SW_ERR_NOMEM;
        {
            Carver cv;   // stage adjoints (zeroed per stage)
            add_stage_adj(cv, w);
            if (!carve(cv, &w.stage_adj, &w.stage_adj_elems)) return SW_ERR_NOMEM;
        }
        {
            Carver cv;   // tail adjoints (zeroed per step)
            cv.add(w.bBu, nx + 1, ny + 2); cv.add(w.bBv, nx + 2, ny + 1);
            cv.add(w.bS11, nux + 1, nuy + 2); cv.add(w.bS12, nx + 1, ny + 1); cv.add(w.bS21, nx + 1, ny + 1);
            cv.add(w.bS22, nvx + 2, nvy + 1); cv.add(w.bnuS, nx + 2, ny + 2);
            cv.add(w.bLu, nux + 2, nuy + 2); cv.add(w.bLv, nvx + 2, nvy + 2);
            cv.add(w.bsKE, nx + 2, ny + 2); cv.add(w.bDSq, nvx + 3, nvy + 4);
            if (!carve(cv, &w.tail_adj, &w.tail_adj_elems)) return SW_ERR_NOMEM;
        }
        if (want_store) {   // one record per step; without the memory the steps are recomputed instead
            bool two = want_overlap && !host;
            if (two) {
                wf = w;    // shares the static fields; gets its own forward buffers and multipliers
                Carver cv;
                A2<T> fv;
                cv.add(fv, 4, 1);
                two = make_forward(wf) && carve(cv);
                wf.force = fv.d;
                two = two && cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking) == cudaSuccess;
            }
            // a record is the stage states and Z, and also the tail
            // intermediates when they fit, except for the overlapped segments
            // (measured: the f32 reverse sweep of 2000 steps at 512x256 with
            // every step kept in 253 against 275 ms; overlapped, where the
            // recomputation copies them too, no faster)
            const int tr_max = want_overlap ? 0 : 1;
            for (int nb = two ? 2 : 1; nb >= 1 && !stored; nb--)
                for (int tr = tr_max; tr >= 0 && !stored; tr--) {
                    const size_t re = w.stage_block_elems + (tr ? w.tail_inter_elems : 0);
                    const size_t n = (size_t)nb * (size_t)nrecords * re;
                    void* p = nullptr;
                    if (host) p = std::calloc(n, sizeof(T));
                    else if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) { p = nullptr; (void)cudaGetLastError(); }
                    if (p) {
                        blocks.push_back(p);
                        records = static_cast<T*>(p);
                        stored = true;
                        overlap = nb == 2;
                        rec_elems = re;
                        w.tail_kept = tr == 1;
                    }
                }
        }
        const char* env_split = getenv("SWB200_ADJ_SPLIT");
        const char* env_fork = getenv("SWB200_ADJ_FORK");
        if (stored && !w.ssp && !w.linear && !(env_split && env_split[0] == '0')) {   // per-stage intermediates
            split = true;
            Carver ca;   // the stages' scratch adjoints, one block
            for (int k = 0; k < w.rko && split; k++) {
                ws[k] = w;
                ws[k].clear_stage_adj = false;
                Carver cv;
                add_stage_inter(cv, ws[k]);
                split = carve(cv);
                add_stage_adj(ca, ws[k]);
            }
            split = split && carve(ca, &ws_adj, &ws_adj_elems);
            if (split && !host && !(env_fork && env_fork[0] == '0'))
                split = cudaStreamCreateWithFlags(&s3, cudaStreamNonBlocking) == cudaSuccess &&
                        cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming) == cudaSuccess &&
                        cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming) == cudaSuccess;
        }
        return host ? SW_OK : capture();
    }

    int capture() {
        for (int t = (nstep_diff > 1 ? 0 : 1); t < 2; t++)
            for (int k = 0; k < 3; k++) {
                if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return SW_ERR_CUDA;
                Launcher L = launcher();
                Launcher side{s3};
                side.pdl = pdl;
                if (k == 0) fwd_step(L, w, t == 1);
                else if (k == 2 && split) adj_step_split(L, s3 ? &side : nullptr, ev_fork, ev_join, w, ws, ws_adj, ws_adj_elems, t == 1);
                else adj_step(L, w, k == 2, t == 1);
                if (k == 2 && split) L.launches += side.launches;
                cudaError_t e = cudaGetLastError();
                cudaGraph_t graph = nullptr;
                const cudaError_t ec = cudaStreamEndCapture(s, &graph);
                if (e == cudaSuccess) e = ec;
                if (e == cudaSuccess) e = cudaGraphInstantiate(k == 0 ? &g_fwd[t] : (k == 1 ? &g_adj[t] : &g_adj_st[t]), graph, 0);
                if (graph) cudaGraphDestroy(graph);
                if (e != cudaSuccess) {
                    err = std::string("adjoint graph: ") + cudaGetErrorString(e);
                    return SW_ERR_CUDA;
                }
                if (t == 1 && k == 0) launches_fwd = L.launches;
                else if (t == 1 && k == (stored ? 2 : 1)) launches_adj = L.launches;
            }
        if (!overlap) return SW_OK;
        for (int t = (nstep_diff > 1 ? 0 : 1); t < 2; t++) {   // the second worker's forward steps, on s2
            if (cudaStreamBeginCapture(s2, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return SW_ERR_CUDA;
            Launcher L{s2};
            L.pdl = pdl;
            fwd_step(L, wf, t == 1);
            cudaError_t e = cudaGetLastError();
            cudaGraph_t graph = nullptr;
            const cudaError_t ec = cudaStreamEndCapture(s2, &graph);
            if (e == cudaSuccess) e = ec;
            if (e == cudaSuccess) e = cudaGraphInstantiate(&g_fwd2[t], graph, 0);
            if (graph) cudaGraphDestroy(graph);
            if (e != cudaSuccess) {
                err = std::string("adjoint graph: ") + cudaGetErrorString(e);
                return SW_ERR_CUDA;
            }
        }
        return SW_OK;
    }

    // the time-dependent multipliers of every step (src/rhs.jl:233-238, 262-267,
    // src/continuity.jl:27-49 with t = k*dtint, the model time at step k's start)
    int make_forcing(const sw_config& c, long long nsteps) {
        if (!w.timedep) return SW_OK;
        const size_t bytes = (size_t)nsteps * 3 * sizeof(T);
        if (host) step_force = static_cast<T*>(std::malloc(bytes));
        else if (cudaMallocHost(&step_force, bytes) != cudaSuccess) step_force = nullptr;
        if (!step_force) return SW_ERR_NOMEM;
        for (long long k = 0; k < nsteps; k++) {
            const double t = (double)(k * (long long)c.dtint);
            step_force[3 * k] = c.seasonal_wind_x ? (T)std::sin(c.omegaFx * t) : T(1);
            step_force[3 * k + 1] = c.seasonal_wind_y ? (T)std::sin(c.omegaFy * t) : T(1);
            step_force[3 * k + 2] = c.surface_forcing ? (T)std::sin(c.omegaFeta * t) : T(0);
        }
        return SW_OK;
    }
    // before the replay of the step that starts at state k (on worker w, or
    // the second forward worker on s2)
    void set_force(long long k, bool second = false) {
        if (!w.timedep) return;
        T* dst = second ? wf.force : w.force;
        if (host) std::memcpy(dst, step_force + 3 * k, 3 * sizeof(T));
        else cudaMemcpyAsync(dst, step_force + 3 * k, 3 * sizeof(T), cudaMemcpyHostToDevice, second ? s2 : s);
    }

    // the step i = k + 1 that starts at state k ends with drag and diffusion?
    bool tail_of(long long k) const { return ((k + 1) % nstep_diff) == 0; }

    // X: state `from` -> state `from + n`
    cudaError_t advance(long long from, long long n) {
        cudaError_t e = cudaSuccess;
        for (long long k = from; k < from + n && e == cudaSuccess; k++) {
            const int t = tail_of(k) ? 1 : 0;
            set_force(k);
            if (host) { Launcher L = launcher(); fwd_step(L, w, t == 1); }
            else e = cudaGraphLaunch(g_fwd[t], s);
        }
        fwd_steps += n;
        return e;
    }
    // the second worker: its X from state `from` to state `from + n`, on s2
    cudaError_t advance2(long long from, long long n) {
        cudaError_t e = cudaSuccess;
        for (long long k = from; k < from + n && e == cudaSuccess; k++) {
            set_force(k, true);
            e = cudaGraphLaunch(g_fwd2[tail_of(k) ? 1 : 0], s2);
        }
        fwd_steps += n;
        return e;
    }
    cudaError_t adjoint_here(long long k) {   // Xb <- adjoint of the step that starts at state k (in X)
        adj_steps++;
        const int t = tail_of(k) ? 1 : 0;
        set_force(k);
        if (host) { Launcher L = launcher(); adj_step(L, w, false, t == 1); return cudaSuccess; }
        return cudaGraphLaunch(g_adj[t], s);
    }
    // Xb <- adjoint of the step from state k, from its stage states kept in record rec
    cudaError_t adjoint_stored(long long k, long long rec) {
        Launcher L = launcher();
        L.copy(w.stage_block, records + (size_t)rec * rec_elems, rec_elems * sizeof(T));
        adj_steps++;
        const int t = tail_of(k) ? 1 : 0;
        set_force(k);
        if (host) {
            if (split) adj_step_split(L, (Launcher*)nullptr, nullptr, nullptr, w, ws, ws_adj, ws_adj_elems, t == 1);
            else adj_step(L, w, true, t == 1);
            return cudaSuccess;
        }
        return cudaGraphLaunch(g_adj_st[t], s);
    }
    cudaError_t adjoint_of(const State<T>& state, long long k) {
        copy(w.X, state);
        return adjoint_here(k);
    }

    // binomial reversal of steps [a, b): the state of step a is in slot `slot`;
    // slots above `slot` are free; Xb holds the adjoint of step b's state.
    cudaError_t reverse(long long a, long long b, int slot) {
        cudaError_t e = cudaSuccess;
        while (b > a && e == cudaSuccess) {
            const long long t = b - a;
            const int free_slots = (int)slots.size() - 1 - slot;
            if (t == 1) return adjoint_of(slots[slot], a);
            if (free_slots <= 0) {   // no slot left: recompute the state of step b - 1 from a
                copy(w.X, slots[slot]);
                e = advance(a, t - 1);
                if (e == cudaSuccess) e = adjoint_here(b - 1);
                b--;
                continue;
            }
            // r: fewest repetitions with C(free + r, free) >= t; the left part gets C(free + r - 1, free) steps
            auto binom = [](long long nn, long long kk) {
                double x = 1.0;
                for (long long q = 1; q <= kk; q++) x = x * (double)(nn - kk + q) / (double)q;
                return x;
            };
            long long r = 0;
            while (binom(free_slots + r, free_slots) < (double)t) r++;
            long long left = r >= 1 ? (long long)binom(free_slots + r - 1, free_slots) : 1;
            left = std::max(1LL, std::min(left, t - 1));
            const long long m = a + left;
            copy(w.X, slots[slot]);
            e = advance(a, m - a);
            if (e != cudaSuccess) return e;
            copy(slots[slot + 1], w.X);
            e = reverse(m, b, slot + 1);
            b = m;       // then reverse [a, m) with the same slot
        }
        return e;
    }
};

// The reverse sweep of the two-level schedule with the recomputation one
// segment ahead: segment j's records (its steps' stage inputs) go to half
// j % 2 of the records; the second worker recomputes segment j - 1 on s2
// while s reverses segment j.  Events order the halves: the reverse of j
// waits for the recomputation of j, the recomputation of j - 1 for the
// reverse of j + 1 (the previous user of its half).  Every step is computed
// as in the sequential order, on the same graphs' passes.
template <class T>
cudaError_t reverse_overlapped(Adjoint<T>& A, int nslots, long long seg, long long nsteps) {
    Work<T>& w = A.w;
    cudaEvent_t ev_start = nullptr, ev_rec[2] = {}, ev_rev[2] = {};
    cudaError_t e = cudaSuccess;
    for (cudaEvent_t* x : {&ev_start, &ev_rec[0], &ev_rec[1], &ev_rev[0], &ev_rev[1]})
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(x, cudaEventDisableTiming);
    auto range = [&](long long j, long long& a, long long& b) {
        a = j * seg;
        b = std::min<long long>(nsteps, a + seg);
    };
    auto rec_of = [&](long long j, long long k) { return (j % 2) * seg + (k - j * seg); };
    auto recompute = [&](long long j) {
        long long a, b;
        range(j, a, b);
        Launcher L{A.s2};
        copy_state(L, A.wf.X, A.slots[j]);
        for (long long k = a; k < b && e == cudaSuccess; k++) {
            e = A.advance2(k, 1);
            L.copy(A.records + (size_t)rec_of(j, k) * A.rec_elems, A.wf.stage_block, A.rec_elems * sizeof(T));
        }
        if (e == cudaSuccess) e = cudaEventRecord(ev_rec[j % 2], A.s2);
    };
    // the slots were written by the forward sweep on s
    if (e == cudaSuccess) e = cudaEventRecord(ev_start, A.s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(A.s2, ev_start, 0);
    const long long last = nslots - 1;
    if (e == cudaSuccess) recompute(last);
    for (long long j = last; j >= 0 && e == cudaSuccess; j--) {
        if (j >= 1) {
            if (j + 1 <= last) e = cudaStreamWaitEvent(A.s2, ev_rev[(j + 1) % 2], 0);
            if (e == cudaSuccess) recompute(j - 1);
        }
        if (e == cudaSuccess) e = cudaStreamWaitEvent(A.s, ev_rec[j % 2], 0);
        long long a, b;
        range(j, a, b);
        for (long long k = b - 1; k >= a && e == cudaSuccess; k--) e = A.adjoint_stored(k, rec_of(j, k));
        if (e == cudaSuccess) e = cudaEventRecord(ev_rev[j % 2], A.s);
    }
    // nothing on s2 is left unwaited: the last reverse waited for the last recomputation
    for (cudaEvent_t x : {ev_start, ev_rec[0], ev_rec[1], ev_rev[0], ev_rev[1]})
        if (x) cudaEventDestroy(x);
    return e;
}

template <class T>
int adjoint_run(bool host, const sw_config& c, const sw_static& st, const void* u, const void* v, const void* eta,
                const void* eta_obs, int64_t nsteps, int32_t ncheckpoints, double* J, void* g_u, void* g_v,
                void* g_eta, void* g_Fx, void* eta_final, sw_adjoint_stats* stats) {
    Adjoint<T> A;
    A.host = host;
    // Keeping every step's stage inputs (rko + 1 states a step) spares the
    // reverse sweep the recomputation of the forward step; it needs a slot per
    // step and is off with SWB200_ADJ_STORE=0.  With fewer checkpoints than
    // steps the default schedule is two-level: a state slot at the start of
    // each segment of seg = ceil(nsteps / ncheckpoints) steps, and the reverse
    // sweep recomputes one segment at a time, keeping its steps' stage inputs
    // (seg records), so every step is recomputed once.  When those records do
    // not fit, or with SWB200_ADJ_SCHEDULE=binomial, the binomial schedule
    // runs instead on the state slots alone.
    // The segments' recomputation runs on a second stream, one segment ahead
    // of the reverse steps (SWB200_ADJ_OVERLAP=0: one after the other).
    const char* env = getenv("SWB200_ADJ_STORE");
    const char* envs = getenv("SWB200_ADJ_SCHEDULE");
    const char* envo = getenv("SWB200_ADJ_OVERLAP");
    const bool store_ok = !(env && env[0] == '0');
    const bool all_steps = ncheckpoints >= nsteps;
    const bool want_segments = !all_steps && store_ok && !(envs && std::string(envs) == "binomial");
    const long long seg = want_segments ? (nsteps + ncheckpoints - 1) / std::max<long long>(1, ncheckpoints) : 0;
    int rc = A.setup(c, st, store_ok && (all_steps || want_segments), all_steps ? nsteps : seg,
                     want_segments && !(envo && envo[0] == '0'));
    if (!rc) rc = A.make_forcing(c, nsteps);
    if (rc) {
        if (!A.err.empty()) fprintf(stderr, "swb200: %s\n", A.err.c_str());
        return rc;
    }
    Work<T>& w = A.w;
    const size_t bytes_u = w.X.u.size() * sizeof(T), bytes_v = w.X.v.size() * sizeof(T), bytes_e = w.X.e.size() * sizeof(T);
    // ncheckpoints is an upper bound: when that many state slots do not fit in
    // device memory, half as many are tried (down to one), and the binomial
    // schedule recomputes what the missing slots would have kept
    // the J row sums are allocated before the checkpoint slots, which take the
    // largest block that fits and would otherwise leave no room for them
    double* rowsum = host ? static_cast<double*>(std::calloc(w.ny, sizeof(double))) : nullptr;
    if (!host && cudaMalloc(&rowsum, w.ny * sizeof(double)) != cudaSuccess) {
        (void)cudaGetLastError();
        return SW_ERR_NOMEM;
    }
    auto free_rowsum = [&] {
        if (host) std::free(rowsum);
        else if (rowsum) cudaFree(rowsum);
        rowsum = nullptr;
    };
    const bool segments = want_segments && A.stored;      // the segment's records fit
    const bool stored_all = all_steps && A.stored;
    int nslots = stored_all ? 1
               : segments ? (int)((nsteps + seg - 1) / seg)
                          : (int)std::max<long long>(1, std::min<long long>(ncheckpoints, nsteps));
    if (!A.make_slots(nslots)) {
        free_rowsum();
        return SW_ERR_NOMEM;
    }
    if (segments && (int)A.slots.size() < nslots) {
        // fewer slots than segments: no room for the two-level schedule
        free_rowsum();
        return SW_ERR_NOMEM;
    }
    nslots = (int)A.slots.size();
    cudaEvent_t ev[3] = {};
    auto destroy_events = [&] {
        for (auto& x : ev)
            if (x) cudaEventDestroy(x);
    };
    if (!host)
        for (auto& x : ev)
            if (cudaEventCreate(&x) != cudaSuccess) {
                x = nullptr;
                destroy_events();
                free_rowsum();
                return SW_ERR_CUDA;
            }
    auto record = [&](int k) { if (!host) cudaEventRecord(ev[k], A.s); };
    cudaError_t e = A.upload(A.slots[0].u.d, u, bytes_u);
    if (e == cudaSuccess) e = A.upload(A.slots[0].v.d, v, bytes_v);
    if (e == cudaSuccess) e = A.upload(A.slots[0].e.d, eta, bytes_e);
    // eta_obs (nx x ny) is kept in Yb[0]'s eta block until J is formed; the
    // reverse sweep clears that block before its first use
    A2<T> obs{w.Yb[0].e.d, w.nx, w.ny};
    if (e == cudaSuccess) e = A.upload(obs.d, eta_obs, obs.size() * sizeof(T));
    record(0);
    // forward sweep: with a slot per step every state is kept, otherwise only the first
    A.copy(w.X, A.slots[0]);
    const bool keep_all = !A.stored && nslots >= nsteps;
    for (long long k = 1; k <= nsteps && e == cudaSuccess; k++) {
        e = A.advance(k - 1, 1);
        if (keep_all && k < nsteps) A.copy(A.slots[k], w.X);
        if (segments && k % seg == 0 && k < nsteps) A.copy(A.slots[k / seg], w.X);
        if (stored_all) {
            Launcher L = A.launcher();
            L.copy(A.records + (size_t)(k - 1) * A.rec_elems, w.stage_block, A.rec_elems * sizeof(T));
        }
    }
    record(1);
    // J (FP64 row sums, added on the host in a fixed order) and the seed Xb = dJ/d(state at nsteps)
    std::vector<double> rows(w.ny);
    if (e == cudaSuccess) e = A.zero(w.Xb.base, w.Xb.elems * sizeof(T));
    if (e == cudaSuccess) {
        Launcher L = A.launcher();
        cost_seed(L, w.X.e, obs, w.Xb.e, rowsum);
        if (!host) e = cudaGetLastError();
    }
    if (e == cudaSuccess && eta_final) e = A.download(eta_final, w.X.e.d, bytes_e);
    if (e == cudaSuccess) e = A.download(rows.data(), rowsum, w.ny * sizeof(double));
    if (e == cudaSuccess) e = A.zero(w.bFx.d, w.bFx.size() * sizeof(T));
    // reverse sweep
    if (e == cudaSuccess) {
        if (stored_all) {
            for (long long k = nsteps - 1; k >= 0 && e == cudaSuccess; k--) e = A.adjoint_stored(k, k);
        } else if (segments && A.overlap) {
            e = reverse_overlapped(A, nslots, seg, nsteps);
        } else if (segments) {
            for (long long j = nslots - 1; j >= 0 && e == cudaSuccess; j--) {
                const long long a = j * seg, b = std::min<long long>(nsteps, a + seg);
                A.copy(w.X, A.slots[j]);
                for (long long k = a; k < b && e == cudaSuccess; k++) {
                    e = A.advance(k, 1);
                    Launcher L = A.launcher();
                    L.copy(A.records + (size_t)(k - a) * A.rec_elems, w.stage_block, A.rec_elems * sizeof(T));
                }
                for (long long k = b - 1; k >= a && e == cudaSuccess; k--) e = A.adjoint_stored(k, k - a);
            }
        } else if (keep_all) {
            for (long long k = nsteps - 1; k >= 0 && e == cudaSuccess; k--) e = A.adjoint_of(A.slots[k], k);
        } else {
            e = A.reverse(0, nsteps, 0);
        }
    }
    record(2);
    if (e == cudaSuccess && g_u) e = A.download(g_u, w.Xb.u.d, bytes_u);
    if (e == cudaSuccess && g_v) e = A.download(g_v, w.Xb.v.d, bytes_v);
    if (e == cudaSuccess && g_eta) e = A.download(g_eta, w.Xb.e.d, bytes_e);
    if (e == cudaSuccess && g_Fx) e = A.download(g_Fx, w.bFx.d, w.bFx.size() * sizeof(T));
    if (e == cudaSuccess && !host) e = cudaStreamSynchronize(A.s);
    free_rowsum();
    float ms_f = 0.f, ms_r = 0.f;
    if (!host && e == cudaSuccess) {
        cudaEventElapsedTime(&ms_f, ev[0], ev[1]);
        cudaEventElapsedTime(&ms_r, ev[1], ev[2]);
    }
    destroy_events();
    if (e != cudaSuccess) {
        fprintf(stderr, "swb200: adjoint: %s\n", cudaGetErrorString(e));
        return SW_ERR_CUDA;
    }
    double Jv = 0.0;
    for (double r : rows) Jv += r;
    if (J) *J = Jv;
    if (stats) {
        stats->forward_ms = ms_f;
        stats->reverse_ms = ms_r;
        stats->forward_steps = A.fwd_steps;
        stats->adjoint_steps = A.adj_steps;
        stats->checkpoints = nslots;
        stats->launches_per_forward_step = A.launches_fwd;
        stats->launches_per_adjoint_step = A.launches_adj;
        stats->stored_stage_states = stored_all ? 1 : segments ? (A.overlap ? 3 : 2) : 0;
    }
    return SW_OK;
}

int adjoint_entry(bool host, const sw_config* cfg, const sw_static* st, const void* u, const void* v,
                  const void* eta, const void* eta_obs, int64_t nsteps, int32_t ncheckpoints, double* J, void* g_u,
                  void* g_v, void* g_eta, void* g_Fx, void* eta_final, sw_adjoint_stats* stats) {
    if (!cfg || !st || !u || !v || !eta || !eta_obs || nsteps < 1 || ncheckpoints < 1) return SW_ERR_ARG;
    const AdjCfgError ce = adjoint_check(*cfg);
    if (ce.code) {
        fprintf(stderr, "swb200: adjoint: %s\n", ce.why);
        return ce.code;
    }
    if (!host) {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return SW_ERR_NODEVICE;
    }
    if (cfg->T == SW_FLOAT64)
        return adjoint_run<double>(host, *cfg, *st, u, v, eta, eta_obs, nsteps, ncheckpoints, J, g_u, g_v, g_eta,
                                   g_Fx, eta_final, stats);
    return adjoint_run<float>(host, *cfg, *st, u, v, eta, eta_obs, nsteps, ncheckpoints, J, g_u, g_v, g_eta, g_Fx,
                              eta_final, stats);
}

}  // namespace

extern "C" int sw_adjoint_run(const sw_config* cfg, const sw_static* st, const void* u, const void* v,
                              const void* eta, const void* eta_obs, int64_t nsteps, int32_t ncheckpoints,
                              double* J, void* g_u, void* g_v, void* g_eta, void* g_Fx, void* eta_final,
                              sw_adjoint_stats* stats) {
    return adjoint_entry(false, cfg, st, u, v, eta, eta_obs, nsteps, ncheckpoints, J, g_u, g_v, g_eta, g_Fx,
                         eta_final, stats);
}

#ifdef SWA_HOST_CHECK
// Host check build (tests only, never part of libswb200.so): the same passes,
// checkpoint schedule and reductions executed in host loops with every array
// access checked against its reference shape.  Returns the number of accesses
// that fell outside in *bounds_failures.
namespace swa { long long swa_bounds_failures = 0; }
extern "C" int swa_host_check_run(const sw_config* cfg, const sw_static* st, const void* u, const void* v,
                                  const void* eta, const void* eta_obs, int64_t nsteps, int32_t ncheckpoints,
                                  double* J, void* g_u, void* g_v, void* g_eta, void* g_Fx, void* eta_final,
                                  long long* bounds_failures) {
    swa::swa_bounds_failures = 0;
    const int rc = adjoint_entry(true, cfg, st, u, v, eta, eta_obs, nsteps, ncheckpoints, J, g_u, g_v, g_eta, g_Fx,
                                 eta_final, nullptr);
    if (bounds_failures) *bounds_failures = swa::swa_bounds_failures;
    return rc;
}
#endif
