// sw_batch16.cuh -- batched ensembles of members in the 16-bit storage form.
//
// The same scheme as sw_batch.cuh (one launch per sub-step for all members of
// a group, per-member argument tables in device memory, the global step read
// from device memory), with the bodies of the single-model 16-bit kernels of
// sw_s16.cuh, so a member computes exactly what it computes alone:
//   stage    s16_stage_body on the member's pairs, increments and X0
//   tail     tail_body with the member's TailStorePair (new u, v pairs)
//   tracer   tracer_body reading u, v (hi) and sst as 16-bit numbers
//   copy     um, vm = hi of u, v in FP32 (tracer with nadvstep > 1)
//   NaN      on the his of u, v, eta and on the 16-bit sst
#pragma once
#include "sw_batch.cuh"
#include "sw_s16.cuh"

namespace swb {

template <class S16, bool PER, bool FIRST, bool LAST, int TY>
__global__ void __launch_bounds__(128)
s16_stage_batch(const S16StageArgs<S16>* __restrict__ args, const int* __restrict__ block0, int n,
                const BatchMember* __restrict__ mem, const long long* __restrict__ istep) {
    const long long i = *istep;
    __shared__ __align__(16) S16StageArgs<S16> A;
    const int m = batch_member(block0, n, (int)blockIdx.x);
    if (i > mem[m].nt) return;
    load_args(A, args + m);
    __syncthreads();
    s16_stage_body<S16, PER, FIRST, LAST, TY>(A, (int)blockIdx.x - block0[m]);
}

template <class S16>
struct S16TailBatchArgs {
    TailArgs<float, float> t;
    TailStorePair<S16> out;
};

template <class S16, bool PER, int DRAG, bool SMAG, int TY>
__global__ void __launch_bounds__(128)
s16_tail_batch(const S16TailBatchArgs<S16>* __restrict__ args, const int* __restrict__ block0, int n,
               const BatchMember* __restrict__ mem, const long long* __restrict__ istep) {
    const long long i = *istep;
    __shared__ __align__(16) S16TailBatchArgs<S16> A;
    const int m = batch_member(block0, n, (int)blockIdx.x);
    if (i > mem[m].nt) return;
    load_args(A, args + m);
    __syncthreads();
    tail_body<float, float, PER, DRAG, SMAG, TY>(A.t, (int)blockIdx.x - block0[m], A.out);
}

template <class S16>
struct S16TracerBatchArgs {
    TracerArgs<float, float> t;
    TracerIO16<S16> io;
};

// args: per member, k odd at [m], k even at [n + m], as tracer_batch
template <class S16, bool PER, bool UM_IS_U, bool CONS>
__global__ void __launch_bounds__(128)
s16_tracer_batch(const S16TracerBatchArgs<S16>* __restrict__ args, const int* __restrict__ block0,
                 const int* __restrict__ nbx, int n, const BatchMember* __restrict__ mem,
                 const long long* __restrict__ istep) {
    const long long i = *istep;
    __shared__ __align__(16) S16TracerBatchArgs<S16> A;
    const int m = batch_member(block0, n, (int)blockIdx.x);
    const BatchMember& me = mem[m];
    if (i > me.nt || !me.tracer || (i % me.nadvstep) != 0) return;
    const long long k = i / me.nadvstep;
    load_args(A, args + (k % 2 == 1 ? m : n + m));
    __syncthreads();
    const int b = (int)blockIdx.x - block0[m];
    const int gy = (block0[m + 1] - block0[m]) / nbx[m];
    tracer_body<float, float, PER, UM_IS_U, CONS>(A.t, b % nbx[m], b / nbx[m], gy, A.io);
}

template <class S16>
struct BatchCopy16 {   // um, vm = hi of u, v of a member, in FP32
    const S16* u; const S16* v; float* um; float* vm;
    long long n;
    float inv_s;
    const DevStatus* st;
};

template <class S16>
__global__ void __launch_bounds__(256)
s16_copy_batch(const BatchCopy16<S16>* __restrict__ args, const int* __restrict__ block0, int n,
               const BatchMember* __restrict__ mem, const long long* __restrict__ istep) {
    const long long i = *istep;
    const int m = batch_member(block0, n, (int)blockIdx.x);
    const BatchMember& me = mem[m];
    if (i > me.nt || !me.tracer || me.nadvstep <= 1 || ((i + me.nadvstep_half) % me.nadvstep) != 0) return;
    const BatchCopy16<S16>& a = args[m];
    if (a.st->stop) return;
    const int b = (int)blockIdx.x - block0[m], nb = block0[m + 1] - block0[m];
    for (long long k = b * 256LL + threadIdx.x; k < a.n; k += nb * 256LL) {
        a.um[k] = from16(a.u[k]) * a.inv_s;
        a.vm[k] = from16(a.v[k]) * a.inv_s;
    }
}

template <class S16>
struct BatchNan16 {
    Geom g;
    const S16* u; const S16* v; const S16* e; const S16* sst;
    DevStatus* st;
};

// args: per member, [m] for an even number of tracer steps so far, [n + m] for odd
template <class S16>
__global__ void __launch_bounds__(256)
s16_nan_batch(const BatchNan16<S16>* __restrict__ args, const int* __restrict__ block0, int n,
              const BatchMember* __restrict__ mem, const long long* __restrict__ istep) {
    const long long i = *istep;
    const int m = batch_member(block0, n, (int)blockIdx.x);
    const BatchMember& me = mem[m];
    if (i > me.nt || (i % me.nout) != 0) return;
    const long long k = me.tracer ? i / me.nadvstep : 0;
    const BatchNan16<S16>& a = args[k % 2 == 0 ? m : n + m];
    if (a.st->stop) return;
    const Geom& g = a.g;
    const int N = g.N, M = g.M, ep = g.ep;
    const int uw = (ep ? N : N - 1) + 4;
    struct Ext { int w, h, x0, y0; const S16* p; };
    const Ext ex[4] = {{uw, M + 4, ep ? -2 : -1, -2, a.u}, {N + 4, M + 3, -2, -1, a.v}, {N + 2, M + 2, -1, -1, a.e},
                       {N + 2, M, -1, 0, a.sst}};
    const int b = (int)blockIdx.x - block0[m], nb = block0[m + 1] - block0[m];
    unsigned long long cnt = 0;
    for (int f = 0; f < 4; f++) {
        const long long tot = (long long)ex[f].w * ex[f].h;
        for (long long k2 = b * 256LL + threadIdx.x; k2 < tot; k2 += nb * 256LL) {
            const int x = ex[f].x0 + (int)(k2 % ex[f].w), y = ex[f].y0 + (int)(k2 / ex[f].w);
            const float val = from16(ex[f].p[g.idx(x, y)]);
            cnt += (val != val) ? 1 : 0;
        }
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) {
        atomicAdd(&a.st->nan_count, cnt);
        atomicCAS(&a.st->stop, 0, 1);
        a.st->nan_step = i;
    }
}

}  // namespace swb
