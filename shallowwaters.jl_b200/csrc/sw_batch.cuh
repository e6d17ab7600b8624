// sw_batch.cuh -- one launch per sub-step for a whole ensemble of models.
//
// Members are independent runs (own grid size, parameters, step length and
// number of steps) that share the option set, so each kernel of a time step
// can serve all of them at once: the launch's blocks are the concatenation of
// every member's blocks, and a block finds its member from a table of block
// offsets.  The per-member kernel arguments live in device memory, one table
// per state parity (and tracer parity), built once when the batch is set up.
// All members advance in lockstep by global step i = 1, 2, ...; each member's
// own schedule follows from i and its constants:
//   finished      i > nt                  (the member's blocks return at once)
//   tracer due    i % nadvstep == 0, as the k = i / nadvstep-th tracer step,
//                 reading sst[(k-1) % 2] and writing sst[k % 2]
//   um/vm copy    (i + nadvstep_half) % nadvstep == 0
//   NaN check     i % nout == 0
// The bodies are those of the single-model kernels (rk_stage_body, tail_body,
// tracer_body), so every member computes exactly what it computes alone.  The
// kernels read i from device memory and batch_advance moves it on, so the
// launches of a step can be replayed from a CUDA graph.
#pragma once
#include "sw_stage.cuh"
#include "sw_tail.cuh"
#include "sw_tracer.cuh"

namespace swb {

struct BatchMember {
    long long nt;          // the member's number of steps
    int tracer;            // tracer_advection
    int nadvstep, nadvstep_half, nout;
    int cells;             // nx * ny (for the diagnostics of the runner)
};

// the member of block b: the largest m with block0[m] <= b (block0 has n+1 entries)
__device__ __forceinline__ int batch_member(const int* __restrict__ block0, int n, int b) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (block0[mid] <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// copies a member's argument struct into shared memory (word by word)
template <class Args>
__device__ __forceinline__ void load_args(Args& dst, const Args* __restrict__ src) {
    static_assert(sizeof(Args) % 4 == 0, "argument structs are word-sized");
    const unsigned* s = reinterpret_cast<const unsigned*>(src);
    unsigned* d = reinterpret_cast<unsigned*>(&dst);
    for (int k = threadIdx.x; k < (int)(sizeof(Args) / 4); k += blockDim.x) d[k] = s[k];
}

template <class T, class Tp, bool PER, bool FIRST, bool LAST, int TY>
__global__ void __launch_bounds__(128)
rk_stage_batch(const StageArgs<T, Tp>* __restrict__ args, const int* __restrict__ block0, int n,
               const BatchMember* __restrict__ mem, const long long* __restrict__ istep) {
    const long long i = *istep;
    __shared__ __align__(16) StageArgs<T, Tp> A;
    const int m = batch_member(block0, n, (int)blockIdx.x);
    if (i > mem[m].nt) return;
    load_args(A, args + m);
    __syncthreads();
    rk_stage_body<T, Tp, PER, FIRST, LAST, TY>(A, (int)blockIdx.x - block0[m]);
}

template <class T, class Tp, bool PER, int DRAG, bool SMAG, int TY>
__global__ void __launch_bounds__(128)
tail_batch(const TailArgs<T, Tp>* __restrict__ args, const int* __restrict__ block0, int n,
           const BatchMember* __restrict__ mem, const long long* __restrict__ istep) {
    const long long i = *istep;
    __shared__ __align__(16) TailArgs<T, Tp> A;
    const int m = batch_member(block0, n, (int)blockIdx.x);
    if (i > mem[m].nt) return;
    load_args(A, args + m);
    __syncthreads();
    tail_body<T, Tp, PER, DRAG, SMAG, TY>(A, (int)blockIdx.x - block0[m]);
}

// args holds, per member, the tracer arguments for k odd ([m]) and k even ([n + m]);
// member m owns nbx[m] * gy[m] blocks (column blocks x row blocks)
template <class T, class Tp, bool PER, bool UM_IS_U, bool CONS>
__global__ void __launch_bounds__(128)
tracer_batch(const TracerArgs<T, Tp>* __restrict__ args, const int* __restrict__ block0, const int* __restrict__ nbx,
             int n, const BatchMember* __restrict__ mem, const long long* __restrict__ istep) {
    const long long i = *istep;
    __shared__ __align__(16) TracerArgs<T, Tp> A;
    const int m = batch_member(block0, n, (int)blockIdx.x);
    const BatchMember& me = mem[m];
    if (i > me.nt || !me.tracer || (i % me.nadvstep) != 0) return;
    const long long k = i / me.nadvstep;
    load_args(A, args + (k % 2 == 1 ? m : n + m));
    __syncthreads();
    const int b = (int)blockIdx.x - block0[m];
    const int gy = (block0[m + 1] - block0[m]) / nbx[m];
    tracer_body<T, Tp, PER, UM_IS_U, CONS>(A, b % nbx[m], b / nbx[m], gy);
}

struct BatchCopy {     // um, vm = u0, v0 of a member (tracer with nadvstep > 1)
    const float* u; const float* v; float* um; float* vm;
    long long n;
    const DevStatus* st;
};

__global__ void __launch_bounds__(256)
copy_batch(const BatchCopy* __restrict__ args, const int* __restrict__ block0, int n,
           const BatchMember* __restrict__ mem, const long long* __restrict__ istep) {
    const long long i = *istep;
    const int m = batch_member(block0, n, (int)blockIdx.x);
    const BatchMember& me = mem[m];
    if (i > me.nt || !me.tracer || me.nadvstep <= 1 || ((i + me.nadvstep_half) % me.nadvstep) != 0) return;
    const BatchCopy& a = args[m];
    if (a.st->stop) return;
    const int b = (int)blockIdx.x - block0[m], nb = block0[m + 1] - block0[m];
    for (long long k = b * 256LL + threadIdx.x; k < a.n; k += nb * 256LL) {
        a.um[k] = a.u[k];
        a.vm[k] = a.v[k];
    }
}

struct BatchNan {      // nan_check_kernel's operands for one member and tracer parity
    Geom g;
    const float* u; const float* v; const float* e; const float* sst;
    DevStatus* st;
};

// args: per member, [m] for an even number of tracer steps so far, [n + m] for odd
__global__ void __launch_bounds__(256)
nan_batch(const BatchNan* __restrict__ args, const int* __restrict__ block0, int n,
          const BatchMember* __restrict__ mem, const long long* __restrict__ istep) {
    const long long i = *istep;
    const int m = batch_member(block0, n, (int)blockIdx.x);
    const BatchMember& me = mem[m];
    if (i > me.nt || (i % me.nout) != 0) return;
    const long long k = me.tracer ? i / me.nadvstep : 0;
    const BatchNan& a = args[k % 2 == 0 ? m : n + m];
    if (a.st->stop) return;
    const Geom& g = a.g;
    const int N = g.N, M = g.M, ep = g.ep;
    const int uw = (ep ? N : N - 1) + 4;
    struct Ext { int w, h, x0, y0; const float* p; };
    const Ext ex[4] = {{uw, M + 4, ep ? -2 : -1, -2, a.u}, {N + 4, M + 3, -2, -1, a.v}, {N + 2, M + 2, -1, -1, a.e},
                       {N + 2, M, -1, 0, a.sst}};
    const int b = (int)blockIdx.x - block0[m], nb = block0[m + 1] - block0[m];
    unsigned long long cnt = 0;
    for (int f = 0; f < 4; f++) {
        const long long tot = (long long)ex[f].w * ex[f].h;
        for (long long k2 = b * 256LL + threadIdx.x; k2 < tot; k2 += nb * 256LL) {
            const int x = ex[f].x0 + (int)(k2 % ex[f].w), y = ex[f].y0 + (int)(k2 / ex[f].w);
            const float val = ex[f].p[g.idx(x, y)];
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

// the global step i of the next replay
__global__ void batch_advance(long long* istep) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *istep += 1;
}

}  // namespace swb
