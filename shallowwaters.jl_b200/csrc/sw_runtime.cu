// sw_runtime.cu -- libswb200: contexts, device buffers, the time loop and the
// C ABI of include/swb200.h.
//
// Per time step (src/time_integration.jl:45-243) the RK scheme issues
//   RKo x rk_stage_kernel   (rhs! + continuity! + caxb!/axb! + ghost points)
//   tail_kernel             (every nstep_diff steps: drag + diffusion + add)
//   [copy_convert_kernel]   (mid-point velocity copy, nadvstep > 1)
//   tracer_kernel           (every nadvstep steps)
//   nan_check_kernel        (every nout steps)
// on one stream.  Buffers: two state sets S[0], S[1] (u, v, eta), two stage
// sets A, B, the accumulator Acc (u0, v0, eta0), two tracer buffers.  With
// state parity p, step i reads S[p] and leaves the new state in S[1-p]; S[p]
// survives the step, which gives the reference's NaN semantics (return the
// state from before the failing step).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <map>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "swb200.h"
#include "sw_common.cuh"
#include "sw_ghost.cuh"
#include "sw_stage.cuh"
#include "sw_ssp.cuh"
#include "sw_linear.cuh"
#include "sw_advcor.cuh"
#include "sw_storage.cuh"
#include "sw_s16.cuh"
#include "sw_batch.cuh"
#include "sw_batch16.cuh"
#include "sw_diag.cuh"
#include "sw_tail.cuh"
#include "sw_tracer.cuh"

using namespace swb;

namespace {

#ifndef SWB_STAGE_TY
#define SWB_STAGE_TY 32
#endif
#ifndef SWB_TAIL_TY
#define SWB_TAIL_TY 32
#endif
constexpr int STAGE_TY = SWB_STAGE_TY;  // rows per warp strip of the stage kernel
constexpr int TAIL_TY = SWB_TAIL_TY;
constexpr int PADX = 72, PADY = 44;     // column/row padding: strips read up to TY+6 rows and 30 columns past the edge
constexpr int RING_BLOCKS_MAX = 32;

const char* err_name(int c) {
    switch (c) {
        case SW_OK: return "ok";
        case SW_ERR_ARG: return "invalid argument";
        case SW_ERR_CUDA: return "CUDA error";
        case SW_NAN_DETECTED: return "NaNs detected";
        case SW_ERR_TIMEOUT: return "device wait timed out";
        case SW_ERR_UNSUPPORTED: return "option combination not supported";
        case SW_ERR_NOMEM: return "device allocation failed";
        case SW_ERR_DEPARTURE: return "tracer departure point outside the domain";
        case SW_ERR_NODEVICE: return "no CUDA device";
    }
    return "unknown error";
}

size_t fmt_size(int f) { return f == SW_FLOAT16 ? 2 : f == SW_FLOAT32 ? 4 : f == SW_FLOAT64 ? 8 : 0; }

struct Fields3 { void* u = nullptr; void* v = nullptr; void* e = nullptr; };

}  // namespace

// Device and pinned blocks released by sw_destroy are kept for reuse by later
// contexts of the same sizes: a drop-in call (create, run, destroy) then costs
// no cudaMalloc/cudaFree after the first, which are slow and, for cudaFree,
// erratic (milliseconds to a second).  At most CACHE_LIMIT bytes of device
// memory are held; sw_trim_memory returns them all.  Device blocks are keyed
// by the CUDA context that allocated them (current_context_id), so a block of
// a context that was destroyed meanwhile is never handed out again.
namespace {
struct DevKey {
    int device;
    unsigned long long context;
    size_t bytes;
    bool operator<(const DevKey& o) const {
        if (device != o.device) return device < o.device;
        if (context != o.context) return context < o.context;
        return bytes < o.bytes;
    }
};
struct BlockCache {
    std::mutex mu;
    std::multimap<DevKey, void*> dev;
    std::multimap<size_t, void*> pinned;
    size_t cached = 0;
};
BlockCache& block_cache() {
    static BlockCache* c = new BlockCache();   // never destroyed: may be used during process exit
    return *c;
}
constexpr size_t CACHE_LIMIT = size_t(16) << 30;

cudaError_t cached_malloc(void** p, size_t bytes) {
    int d = 0;
    cudaGetDevice(&d);
    const unsigned long long cid = current_context_id();
    if (cid) {
        BlockCache& c = block_cache();
        std::lock_guard<std::mutex> lock(c.mu);
        auto it = c.dev.find({d, cid, bytes});
        if (it != c.dev.end()) {
            *p = it->second;
            c.dev.erase(it);
            c.cached -= bytes;
            return cudaSuccess;
        }
    }
    return cudaMalloc(p, bytes);
}
void cached_free(void* p, size_t bytes) {
    int d = 0;
    cudaGetDevice(&d);
    const unsigned long long cid = current_context_id();
    if (cid) {
        BlockCache& c = block_cache();
        std::lock_guard<std::mutex> lock(c.mu);
        if (c.cached + bytes <= CACHE_LIMIT) {
            c.dev.insert({{d, cid, bytes}, p});
            c.cached += bytes;
            return;
        }
    }
    cudaFree(p);
}
cudaError_t cached_malloc_host(void** p, size_t bytes) {
    {
        BlockCache& c = block_cache();
        std::lock_guard<std::mutex> lock(c.mu);
        auto it = c.pinned.find(bytes);
        if (it != c.pinned.end()) {
            *p = it->second;
            c.pinned.erase(it);
            return cudaSuccess;
        }
    }
    return cudaMallocHost(p, bytes);
}
void cached_free_host(void* p, size_t bytes) {
    BlockCache& c = block_cache();
    std::lock_guard<std::mutex> lock(c.mu);
    c.pinned.insert({bytes, p});
}
}  // namespace

struct sw_ctx;
struct EngineBase {
    virtual ~EngineBase() = default;
    virtual int step(sw_ctx* ctx, long long i) = 0;          // one time step, without the NaN check
    virtual int nan_check(sw_ctx* ctx, long long i) = 0;     // the check of step i (state before it)
    virtual int diagnostics(sw_ctx* ctx, sw_diag* out) = 0;
    virtual int prologue(sw_ctx* ctx) = 0;                   // work of time_integration before its loop
    virtual int ghost_state(sw_ctx* ctx) = 0;
    // the storage form's own copy of the state: made from the FP32 buffers
    // S[p], sst[sp] after an upload, and written back into them before a
    // download or a diagnostics pass (no-ops for the native storage)
    virtual int state_uploaded(sw_ctx*) { return SW_OK; }
    virtual int state_to_fp32(sw_ctx*) { return SW_OK; }
};

struct sw_ctx {
    sw_config cfg;
    Geom g;
    size_t nelem = 0;          // elements per field buffer (P*R)
    size_t tsz = 0, tpsz = 0;  // sizeof(T), sizeof(Tprog)
    cudaStream_t stream = nullptr;
    int device = 0;
    std::vector<std::pair<void*, size_t>> allocs;   // device blocks and their sizes (cached_malloc)
    std::vector<std::pair<void*, size_t>> zeroed;   // the blocks that start at zero (state, stage, status)
    unsigned long long context_id = 0;              // CUDA context the blocks belong to
    std::string env;                                // the SWB200_* settings read at creation
    Fields3 S[2], A, B, Acc;
    Fields3 C;                 // third stage buffer of the SSP schemes
    void* qS = nullptr;        // nstep_advcor > 0: stored q, KEu, KEv (type T, sw_advcor.cuh)
    void* KEuS = nullptr;
    void* KEvS = nullptr;
    void* sst[2] = {nullptr, nullptr};
    void* um = nullptr; void* vm = nullptr;
    void* flush = nullptr; size_t flush_bytes = 0;
    // static fields (type T) and their strides
    struct SF { void* p = nullptr; int sx = 0, sy = 0; size_t bytes = 0; } H, fq, Fx, Fy, fu, fv, eref, Feta;
    std::vector<std::vector<unsigned char>> staging;   // host sources of uploads in flight
    // TMA descriptors per state buffer: input box (BOXW_IN x K) and point-wise box (BOXW_X x K)
    struct Maps { CUtensorMap in, x; };
    TileSched* sched = nullptr;   // device tile counter of the TMA stage kernel
    std::map<const void*, Maps> tmaps;
    bool use_tma = false;
    int stage_blocks_cap = 0;     // > 0: at most this many persistent blocks in rk_stage_tma
    uint32_t spin_limit = MBAR_SPIN_LIMIT;   // polls per bounded wait of rk_stage_tma
    int test_skip_chunk = -1;     // test only: a chunk rk_stage_tma's producer leaves out
    // CUDA graphs of one time step, keyed by the buffer parities and the
    // sub-steps that are due (see step_key); off with SWB200_GRAPHS=0
    bool use_graphs = true;
    struct StepGraph { cudaGraphExec_t exec = nullptr; long long launches = 0; bool flips_sp = false; Fields3 rhs_in; };
    // the buffers the last right-hand-side evaluation of the last step read
    // (the input of the last RK stage or SSP sub-stage); null before a step
    Fields3 rhs_in;
    std::map<unsigned, StepGraph> graphs;
    int nsm = 148;
    int tail_ty = TAIL_TY;        // rows per warp strip of the streaming tail (see pick_strip_ty)
    int stage_ty = STAGE_TY;      // rows per warp strip of the streaming stage and SSP momentum kernels
    DevStatus* dst = nullptr;     // device status
    DiagPartial* diag = nullptr;  // DIAG_BLOCKS partials + the result (allocated on first use)
    DevStatus* hst = nullptr;     // pinned host mirror
    int p = 0;                    // state parity
    int sp = 0;                   // tracer parity
    long long step = 0;           // completed steps
    long long t = 0;              // model time [s]
    long long launches = 0;
    std::string err;
    std::unique_ptr<EngineBase> eng;
    // profiling
    bool prof = false;
    std::vector<cudaEvent_t> evpool;
    size_t evnext = 0;
    struct Mark { int kind; cudaEvent_t a, b; };
    std::vector<Mark> marks;
    cudaEvent_t evget();
};

cudaEvent_t sw_ctx::evget() {
    if (evnext == evpool.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        evpool.push_back(e);
    }
    return evpool[evnext++];
}

namespace {

// Strip height of the streaming tail and stage kernels for Float32 / Float64
// contexts: the tallest of 32, 16, 8 rows whose strips still give four
// blocks (16 warps) per SM, else 8; where the kernel has them (short_ok), the
// tallest of 32 .. 2 rows with 16 strips per SM, else 1 (the values do not
// depend on it).  The environment variable `env` (SWB200_TAIL_TY,
// SWB200_STAGE_TY) forces one.  Other number types keep 32.
int pick_strip_ty(const sw_config& c, const Geom& g, int nsm, const char* envname, bool short_ok) {
    if (c.T != c.Tprog || (c.T != SW_FLOAT32 && c.T != SW_FLOAT64)) return 32;
    const char* env = getenv(envname);
    if (env) {
        const int want = atoi(env);
        if (want == 8 || want == 16 || want == 32) return want;
        if (short_ok && (want == 1 || want == 2 || want == 4)) return want;
    }
    const int nsx = (g.N + STRIP - 1) / STRIP;
    if (short_ok) {
        // down to one row: a strip's rows are a serial chain of dependent
        // loads and shuffles, which only enough warps per SM hide
        for (int ty : {32, 16, 8, 4, 2})
            if ((long long)nsx * ((g.M + ty - 1) / ty) >= 16LL * nsm) return ty;
        return 1;
    }
    for (int ty : {32, 16, 8}) {
        const long long blocks = ((long long)nsx * ((g.M + ty - 1) / ty) + 3) / 4;
        if (blocks >= 4LL * nsm) return ty;
    }
    return 8;
}

int fail(sw_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

#define CK(call)                                                                             \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? SW_ERR_NOMEM : SW_ERR_CUDA,   \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                 \
    } while (0)

// Rows per tile of the TMA stage kernel.  A tile of TY rows copies
// ceil((TY + 3) / K) chunks of K rows; 12 rows fill four chunks with one spare
// row (16 rows copied for 12 computed, against 12 for 8) and give 1634 tiles at
// 2048x1024, about 1.8 per persistent block: measured 37.9 us per stage against
// 39.3 for 8 rows (9, 10, 13 and 16 rows were slower than 12).
#ifndef SWB_TMA_TY
#define SWB_TMA_TY 12
#endif
#ifndef SWB_TMA_K
#define SWB_TMA_K 4
#endif
#ifndef SWB_TMA_S
#define SWB_TMA_S 2
#endif
constexpr int STAGE_TMA_TY = SWB_TMA_TY, STAGE_TMA_K = SWB_TMA_K, STAGE_TMA_S = SWB_TMA_S;

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    // looked up once, thread-safely (contexts may be created from several threads)
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    }();
    return fn;
}

// 2-D map over a P x R field buffer; boxes of boxw x boxh elements, zero fill
// outside the buffer
bool make_map(CUtensorMap* m, void* base, size_t elsize, int P, int R, int boxw, int boxh) {
    auto fn = encode_fn();
    if (!fn) return false;
    CUtensorMapDataType dt = elsize == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                           : elsize == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    cuuint64_t dims[2] = {(cuuint64_t)P, (cuuint64_t)R};
    cuuint64_t strides[1] = {(cuuint64_t)P * elsize};
    cuuint32_t box[2] = {(cuuint32_t)boxw, (cuuint32_t)boxh};
    cuuint32_t es[2] = {1, 1};
    CUresult r = fn(m, dt, 2, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

template <class T>
SField<T> sf(const sw_ctx::SF& s) { return SField<T>{static_cast<const T*>(s.p), s.sx, s.sy}; }

// kernel launch bracketed by profiling events when enabled
template <class F>
int launch(sw_ctx* ctx, int kind, F&& f) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (ctx->prof) {
        a = ctx->evget();
        b = ctx->evget();
        cudaEventRecord(a, ctx->stream);
    }
    f();
    ctx->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ctx, SW_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    if (ctx->prof) {
        cudaEventRecord(b, ctx->stream);
        ctx->marks.push_back({kind, a, b});
    }
    return SW_OK;
}

// ghost points of u, v, eta: the rule of every cell whose value some halo cell
// copies (the source cells of sw_ghost.cuh) and of the untouched ring cells,
// enumerated directly so the launch touches only the domain's edges
template <class Tp>
__global__ void ghost_state_kernel(Geom g, Tp* u, Tp* v, Tp* e, GhostRule<Tp> gr) {
    const int N = g.N, M = g.M, ep = g.ep;
    const int nux = ep ? N : N - 1;
    // u sources: periodic columns F in {0, 1, N-2, N-1}; nonperiodic rows b in {0, 1, M-2, M-1}
    const long long nus = ep ? 4LL * M : 4LL * nux;
    const long long nvs = 4LL * (M - 1);                   // v: columns a in {0, 1, N-2, N-1}, G in [1, M)
    const long long nes = 2LL * N + 2LL * (M - 2);         // eta: the perimeter of the T-cells
    const long long nur = Ring::u_count(ep, N, M), nvr = Ring::v_count(N);
    const long long tot = nus + nvs + nes + nur + nvr;
    auto edge4 = [](int k, int n) { return k < 2 ? k : n - 4 + k; };   // 0, 1, n-2, n-1
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < tot; k += (long long)gridDim.x * blockDim.x) {
        long long r = k;
        if (r < nus) {
            int F, b;
            if (ep) { F = edge4((int)(r / M), N); b = (int)(r % M); }
            else { b = edge4((int)(r / nux), M); F = (int)(r % nux) + 1; }
            gr.u(u, g, F, b, u[g.idx(F, b)]);
            continue;
        }
        r -= nus;
        if (r < nvs) {
            const int a = edge4((int)(r / (M - 1)), N), G = (int)(r % (M - 1)) + 1;
            gr.v(v, g, a, G, v[g.idx(a, G)]);
            continue;
        }
        r -= nvs;
        if (r < nes) {
            int a, b;
            if (r < 2LL * N) { a = (int)(r % N); b = r < N ? 0 : M - 1; }
            else { const int q = (int)(r - 2LL * N); a = q < M - 2 ? 0 : N - 1; b = q % (M - 2) + 1; }
            gr.eta(e, g, a, b, e[g.idx(a, b)]);
            continue;
        }
        r -= nes;
        if (r < nur) {
            int F, b;
            Ring::u_at((int)r, ep, N, M, F, b);
            gr.u(u, g, F, b, u[g.idx(F, b)]);
            continue;
        }
        r -= nur;
        int a, G;
        Ring::v_at((int)r, N, M, a, G);
        gr.v(v, g, a, G, v[g.idx(a, G)]);
    }
}

// The tracer's launch grid: 128 columns by one row per block row, one thread
// per cell (measured faster at 2048 x 1024 than several rows per thread, and
// than staging the tile's velocities and tracer in shared memory).
dim3 tracer_grid(const sw_ctx* ctx) {
    const Geom& g = ctx->g;
    return dim3((g.N + 127) / 128, std::min(g.M, 4096));
}

template <class T, class Tp>
struct Engine : EngineBase {
    int init(sw_ctx*) { return SW_OK; }

    // continuity! variant and its fields (src/continuity.jl:3-49); the forcing
    // factor Fetat = T(sin(omega_Feta*t)) at the step's model time
    template <class Args>
    void set_cont(sw_ctx* ctx, Args& a) const {
        const sw_config& c = ctx->cfg;
        a.cont = c.surface_relax ? 1 : c.surface_forcing ? 2 : 0;
        a.sadourny = c.adv_scheme == SW_SADOURNY;
        a.qS = (const T*)ctx->qS; a.KEuS = (const T*)ctx->KEuS; a.KEvS = (const T*)ctx->KEvS;
        a.eref = sf<T>(ctx->eref); a.Feta = sf<T>(ctx->Feta);
        a.gamma = (T)c.gamma;
        a.Fetat = c.surface_forcing ? (T)std::sin(c.omegaFeta * (double)ctx->t) : T(0);
    }

    GhostRule<Tp> rule(sw_ctx* ctx) const {
        GhostRule<Tp> r;
        r.ep = ctx->g.ep; r.N = ctx->g.N; r.M = ctx->g.M; r.Tcomm = ctx->cfg.Tcomm;
        r.oma = (Tp)ctx->cfg.one_minus_alpha;
        return r;
    }

    static int ring_blocks(const Geom& g, int nt) {
        int n = Ring::u_count(g.ep, g.N, g.M) + Ring::v_count(g.N);
        return std::min(RING_BLOCKS_MAX, (n + nt - 1) / nt);
    }

    static constexpr bool SAME_TY = std::is_same<T, Tp>::value &&
                                    (std::is_same<T, float>::value || std::is_same<T, double>::value);
    template <bool PER, bool FIRST, bool LAST>
    static void stage_launch(const StageArgs<T, Tp>& a, int nblk, cudaStream_t s, int ty) {
        if constexpr (SAME_TY) {
            if (ty == 1) { rk_stage_kernel<T, Tp, PER, FIRST, LAST, 1><<<nblk, 128, 0, s>>>(a); return; }
            if (ty == 2) { rk_stage_kernel<T, Tp, PER, FIRST, LAST, 2><<<nblk, 128, 0, s>>>(a); return; }
            if (ty == 4) { rk_stage_kernel<T, Tp, PER, FIRST, LAST, 4><<<nblk, 128, 0, s>>>(a); return; }
            if (ty == 8) { rk_stage_kernel<T, Tp, PER, FIRST, LAST, 8><<<nblk, 128, 0, s>>>(a); return; }
            if (ty == 16) { rk_stage_kernel<T, Tp, PER, FIRST, LAST, 16><<<nblk, 128, 0, s>>>(a); return; }
        }
        rk_stage_kernel<T, Tp, PER, FIRST, LAST, STAGE_TY><<<nblk, 128, 0, s>>>(a);
    }
    static void stage_dispatch(const StageArgs<T, Tp>& a, bool per, bool first, bool last, int nblk, cudaStream_t s,
                               int ty) {
        if (per) {
            if (first) stage_launch<true, true, false>(a, nblk, s, ty);
            else if (last) stage_launch<true, false, true>(a, nblk, s, ty);
            else stage_launch<true, false, false>(a, nblk, s, ty);
        } else {
            if (first) stage_launch<false, true, false>(a, nblk, s, ty);
            else if (last) stage_launch<false, false, true>(a, nblk, s, ty);
            else stage_launch<false, false, false>(a, nblk, s, ty);
        }
    }
    // the TMA stage kernel serves Float32/Float64 compute; Float16 compute runs streaming
    static constexpr bool TMA_TYPES = !std::is_same<T, jf16>::value && !std::is_same<Tp, jf16>::value;
    template <bool PER, bool FIRST, bool LAST, bool ROWF>
    static int stage_tma_launch(sw_ctx* ctx, const StageArgs<T, Tp>& a, const StageMaps& mp) {
      if constexpr (!TMA_TYPES) {
        return -1;
      } else {
        constexpr int TY = STAGE_TMA_TY, K = STAGE_TMA_K, S = STAGE_TMA_S;
        auto kern = rk_stage_tma<T, Tp, PER, FIRST, LAST, TY, K, S, ROWF>;
        constexpr int smem = stage_tma_smem<T, Tp, FIRST, LAST, K, S>();
        // per instantiation, set up once and thread-safely
        static const int occ = [&] {
            int o = -1;
            if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess ||
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, 160, smem) != cudaSuccess)
                o = -1;
            return o;
        }();
        if (occ < 1) return -1;
        const Geom& g = a.g;
        const int ntiles = ((g.N + BAND - 1) / BAND) * ((g.M + TY - 1) / TY);
        int npersist = std::min(ntiles, ctx->nsm * occ);
        if (ctx->stage_blocks_cap > 0) npersist = std::min(npersist, ctx->stage_blocks_cap);
        const int nring = std::min(RING_BLOCKS_MAX, (Ring::u_count(g.ep, g.N, g.M) + Ring::v_count(g.N) + 159) / 160);
        kern<<<npersist + nring, 160, smem, ctx->stream>>>(a, mp, npersist, ctx->sched);
        return 0;
      }
    }
    static int stage_tma_dispatch(sw_ctx* ctx, const StageArgs<T, Tp>& a, const StageMaps& mp, bool per, bool first,
                                  bool last) {
        // static fields constant along x (flat bottom, beta-plane f, zonal winds):
        // the kernel variant that broadcasts their rows by warp shuffles
        const bool rowf = a.H.sx == 0 && a.fq.sx == 0 && a.Fx.sx == 0 && a.Fy.sx == 0;
        if (rowf) return stage_tma_pick<true>(ctx, a, mp, per, first, last);
        return stage_tma_pick<false>(ctx, a, mp, per, first, last);
    }
    template <bool ROWF>
    static int stage_tma_pick(sw_ctx* ctx, const StageArgs<T, Tp>& a, const StageMaps& mp, bool per, bool first,
                              bool last) {
        if (per) {
            if (first) return stage_tma_launch<true, true, false, ROWF>(ctx, a, mp);
            if (last) return stage_tma_launch<true, false, true, ROWF>(ctx, a, mp);
            return stage_tma_launch<true, false, false, ROWF>(ctx, a, mp);
        }
        if (first) return stage_tma_launch<false, true, false, ROWF>(ctx, a, mp);
        if (last) return stage_tma_launch<false, false, true, ROWF>(ctx, a, mp);
        return stage_tma_launch<false, false, false, ROWF>(ctx, a, mp);
    }

    // Shorter strips for Float32 / Float64 grids too small to fill the GPU
    // with 32-row strips (the values do not depend on the strip height).
    template <bool PER, int DRAG, bool SMAG>
    static void tail_launch(const TailArgs<T, Tp>& a, int nblk, cudaStream_t s, int ty) {
        constexpr bool SAME = std::is_same<T, Tp>::value && (std::is_same<T, float>::value || std::is_same<T, double>::value);
        if constexpr (SAME) {
            if (ty == 1) { tail_kernel<T, Tp, PER, DRAG, SMAG, 1><<<nblk, 128, 0, s>>>(a); return; }
            if (ty == 2) { tail_kernel<T, Tp, PER, DRAG, SMAG, 2><<<nblk, 128, 0, s>>>(a); return; }
            if (ty == 4) { tail_kernel<T, Tp, PER, DRAG, SMAG, 4><<<nblk, 128, 0, s>>>(a); return; }
            if (ty == 8) { tail_kernel<T, Tp, PER, DRAG, SMAG, 8><<<nblk, 128, 0, s>>>(a); return; }
            if (ty == 16) { tail_kernel<T, Tp, PER, DRAG, SMAG, 16><<<nblk, 128, 0, s>>>(a); return; }
        }
        tail_kernel<T, Tp, PER, DRAG, SMAG, TAIL_TY><<<nblk, 128, 0, s>>>(a);
    }
    template <bool PER>
    static void tail_dispatch2(const TailArgs<T, Tp>& a, int drag, bool smag, int nblk, cudaStream_t s, int ty) {
        if (smag) {
            if (drag == SW_DRAG_QUADRATIC) tail_launch<PER, SW_DRAG_QUADRATIC, true>(a, nblk, s, ty);
            else if (drag == SW_DRAG_LINEAR) tail_launch<PER, SW_DRAG_LINEAR, true>(a, nblk, s, ty);
            else tail_launch<PER, SW_DRAG_NONE, true>(a, nblk, s, ty);
        } else {
            if (drag == SW_DRAG_QUADRATIC) tail_launch<PER, SW_DRAG_QUADRATIC, false>(a, nblk, s, ty);
            else if (drag == SW_DRAG_LINEAR) tail_launch<PER, SW_DRAG_LINEAR, false>(a, nblk, s, ty);
            else tail_launch<PER, SW_DRAG_NONE, false>(a, nblk, s, ty);
        }
    }
    template <bool PER>
    static void tracer_dispatch2(const TracerArgs<T, Tp>& a, bool um_is_u, bool cons, dim3 grid, cudaStream_t s) {
        if (um_is_u) {
            if (cons) tracer_kernel<T, Tp, PER, true, true><<<grid, 128, 0, s>>>(a);
            else tracer_kernel<T, Tp, PER, true, false><<<grid, 128, 0, s>>>(a);
        } else {
            if (cons) tracer_kernel<T, Tp, PER, false, true><<<grid, 128, 0, s>>>(a);
            else tracer_kernel<T, Tp, PER, false, false><<<grid, 128, 0, s>>>(a);
        }
    }

    int ghost_state(sw_ctx* ctx) override {
        const Geom& g = ctx->g;
        Fields3& X = ctx->S[ctx->p];
        return launch(ctx, 5, [&] {
            ghost_state_kernel<Tp><<<148, 256, 0, ctx->stream>>>(g, (Tp*)X.u, (Tp*)X.v, (Tp*)X.e, rule(ctx));
        });
    }

    // ---------------------------------------------- SSP schemes (:80-196)
    template <bool PER, int MODE, bool FINAL>
    static void ssp_launch(sw_ctx* ctx, const SspArgs<T, Tp>& a) {
        const Geom& g = a.g;
        if (ctx->cfg.dynamics == SW_LINEAR) {
            const int ncb = (int)(((long long)g.N * g.M + 255) / 256);
            const SspArgs<T, Tp> b = ring256(a);
            lin_ssp_momentum_kernel<T, Tp, PER, MODE, FINAL><<<ncb + b.nring_blocks, 256, 0, ctx->stream>>>(
                b, linear_rhs(ctx, a.u1, a.v1, a.e1, a.Fxt, a.Fyt), ncb);
            return;
        }
        const int nb = (a.nsx * a.nsy + 3) / 4 + a.nring_blocks;
        if constexpr (SAME_TY) {
            if (ctx->stage_ty == 1) { ssp_momentum_kernel<T, Tp, PER, MODE, FINAL, 1><<<nb, 128, 0, ctx->stream>>>(a); return; }
            if (ctx->stage_ty == 2) { ssp_momentum_kernel<T, Tp, PER, MODE, FINAL, 2><<<nb, 128, 0, ctx->stream>>>(a); return; }
            if (ctx->stage_ty == 4) { ssp_momentum_kernel<T, Tp, PER, MODE, FINAL, 4><<<nb, 128, 0, ctx->stream>>>(a); return; }
            if (ctx->stage_ty == 8) { ssp_momentum_kernel<T, Tp, PER, MODE, FINAL, 8><<<nb, 128, 0, ctx->stream>>>(a); return; }
            if (ctx->stage_ty == 16) { ssp_momentum_kernel<T, Tp, PER, MODE, FINAL, 16><<<nb, 128, 0, ctx->stream>>>(a); return; }
        }
        ssp_momentum_kernel<T, Tp, PER, MODE, FINAL, STAGE_TY><<<nb, 128, 0, ctx->stream>>>(a);
    }
    // the point-wise linear kernels run their ring with 256 threads per block
    template <class Args>
    static Args ring256(const Args& a) {
        Args b = a;
        b.nring_blocks = ring_blocks(a.g, 256);
        return b;
    }
    static LinearRhs<T, Tp> linear_rhs(sw_ctx* ctx, const Tp* u, const Tp* v, const Tp* e, T Fxt, T Fyt) {
        LinearRhs<T, Tp> L;
        L.g = ctx->g;
        L.u = u; L.v = v; L.e = e;
        L.fu = sf<T>(ctx->fu); L.fv = sf<T>(ctx->fv); L.Fx = sf<T>(ctx->Fx); L.Fy = sf<T>(ctx->Fy);
        L.g_ = (T)ctx->cfg.g; L.Fxt = Fxt; L.Fyt = Fyt;
        return L;
    }
    template <bool PER, bool FIRST, bool LAST>
    static void lin_rk_launch(sw_ctx* ctx, const StageArgs<T, Tp>& a) {
        const Geom& g = a.g;
        const int ncb = (int)(((long long)g.N * g.M + 255) / 256);
        const StageArgs<T, Tp> b = ring256(a);
        lin_rk_stage_kernel<T, Tp, PER, FIRST, LAST><<<ncb + b.nring_blocks, 256, 0, ctx->stream>>>(
            b, linear_rhs(ctx, a.u1, a.v1, a.e1, a.Fxt, a.Fyt), ncb);
    }
    static void lin_rk_dispatch(sw_ctx* ctx, const StageArgs<T, Tp>& a, bool per, bool first, bool last) {
        if (per) {
            if (first) lin_rk_launch<true, true, false>(ctx, a);
            else if (last) lin_rk_launch<true, false, true>(ctx, a);
            else lin_rk_launch<true, false, false>(ctx, a);
        } else {
            if (first) lin_rk_launch<false, true, false>(ctx, a);
            else if (last) lin_rk_launch<false, false, true>(ctx, a);
            else lin_rk_launch<false, false, false>(ctx, a);
        }
    }
    template <int MODE, bool FINAL>
    int ssp_stage(sw_ctx* ctx, const SspArgs<T, Tp>& a) {
        int rc = launch(ctx, 0, [&] {
            if (a.g.ep) ssp_launch<true, MODE, FINAL>(ctx, a);
            else ssp_launch<false, MODE, FINAL>(ctx, a);
        });
        if (rc) return rc;
        return launch(ctx, 0, [&] {
            dim3 grid((a.g.N + 255) / 256, a.g.M);
            ssp_continuity_kernel<T, Tp, MODE, FINAL><<<grid, 256, 0, ctx->stream>>>(a);
        });
    }
    // The stages of SSPRK2 / SSPRK3 / 4SSPRK3.  X is the state at the step
    // start; the final u0, v0 go to Acc when the tail follows (else to Y), the
    // final eta0 to Y.  Stage buffers rotate through A, B, C avoiding the
    // current input and the SSPRK3 snapshot u0 (src/time_integration.jl:148-152),
    // which starts as the state: u0 equals u at every step start.
    int ssp_stages(sw_ctx* ctx, Fields3& X, Fields3& Y, bool tail_now, T Fxt, T Fyt) {
        const sw_config& c = ctx->cfg;
        const Geom& g = ctx->g;
        Fields3 fin;
        fin.u = tail_now ? ctx->Acc.u : Y.u;
        fin.v = tail_now ? ctx->Acc.v : Y.v;
        fin.e = Y.e;
        const Fields3* pool[3] = {&ctx->A, &ctx->B, &ctx->C};
        const Fields3* cur = &X;
        const Fields3* snap = &X;

        SspArgs<T, Tp> a;
        a.g = g;
        a.nsx = (g.N + STRIP - 1) / STRIP; a.nsy = (g.M + ctx->stage_ty - 1) / ctx->stage_ty;
        a.nring_blocks = ring_blocks(g, 128);
        a.uS = (const Tp*)X.u; a.vS = (const Tp*)X.v; a.eS = (const Tp*)X.e;
        a.ufo = a.vfo = a.efo = nullptr;
        a.H = sf<T>(ctx->H); a.fq = sf<T>(ctx->fq); a.Fx = sf<T>(ctx->Fx); a.Fy = sf<T>(ctx->Fy);
        a.g_ = (T)c.g; a.Fxt = Fxt; a.Fyt = Fyt;
        set_cont(ctx, a);
        a.k.half = (Tp)0.5;
        a.k.kna = (Tp)c.ssp_kna; a.k.knb = (Tp)c.ssp_knb;
        a.gr = rule(ctx);
        a.st = ctx->dst;

        int first = 1, last = 0;
        if (c.time_scheme == SW_SSPRK2) { first = 1; last = c.RKs; }
        else if (c.time_scheme == SW_SSPRK3) { first = 2; last = c.ssp_s + 1; }
        else { first = 1; last = 4; }
        auto free_buf = [&](const Fields3* busy) {
            for (const Fields3* f : pool)
                if (f != cur && f != snap && f != busy) return f;
            return (const Fields3*)nullptr;
        };
        for (int rki = first; rki <= last; rki++) {
            const bool is_last = rki == last;
            // the other schemes' last u1 is the final state itself; SSPRK2 keeps
            // u1 and writes the final combination beside it
            const bool to_fin = is_last && c.time_scheme != SW_SSPRK2;
            const bool combo = (c.time_scheme == SW_SSPRK2 && is_last) ||
                               (c.time_scheme == SW_4SSPRK3 && rki == 3);
            const Fields3* out = to_fin ? &fin : free_buf(nullptr);
            const Fields3* cmb = nullptr;
            if (combo) cmb = is_last ? &fin : free_buf(out);
            if (!out || (combo && !cmb)) return fail(ctx, SW_ERR_ARG, "no free SSP stage buffer");
            a.u1 = (const Tp*)cur->u; a.v1 = (const Tp*)cur->v; a.e1 = (const Tp*)cur->e;
            if (is_last) ctx->rhs_in = *cur;
            a.uZ = (const Tp*)snap->u; a.vZ = (const Tp*)snap->v; a.eZ = (const Tp*)snap->e;
            a.u1o = (Tp*)out->u; a.v1o = (Tp*)out->v; a.e1o = (Tp*)out->e;
            if (combo) {
                a.ufo = (Tp*)cmb->u; a.vfo = (Tp*)cmb->v; a.efo = (Tp*)cmb->e;
                if (c.time_scheme == SW_SSPRK2) {                // (:107-109)
                    a.k.fa = (Tp)(1.0 / c.RKs); a.k.fb = (Tp)((double)(c.RKs - 1) / c.RKs);
                } else {                                         // (:186-191)
                    a.k.fa = (Tp)(2.0 / 3.0); a.k.fb = (Tp)(1.0 / 3.0);
                }
            }
            int rc;
            if (c.time_scheme == SW_SSPRK2) {
                a.k.x = (Tp)c.Dt_Ds;
                rc = combo ? ssp_stage<SSP_AXB, true>(ctx, a) : ssp_stage<SSP_AXB, false>(ctx, a);
            } else if (c.time_scheme == SW_SSPRK3) {
                if (rki == c.ssp_kn) { a.k.x = (Tp)c.ssp_Dt_Dnc; rc = ssp_stage<SSP_KN, false>(ctx, a); }
                else { a.k.x = (Tp)c.ssp_Dt_Dn; rc = ssp_stage<SSP_AXB, false>(ctx, a); }
            } else {
                a.k.x = (Tp)c.Dt_D;
                rc = combo ? ssp_stage<SSP_4, true>(ctx, a) : ssp_stage<SSP_4, false>(ctx, a);
            }
            if (rc) return rc;
            if (c.time_scheme == SW_SSPRK3 && rki == c.ssp_mn) snap = out;   // u0 = u1 (:148-152)
            cur = combo ? cmb : out;
        }
        return SW_OK;
    }

    // The arguments of RK stage k for a step from the state S[p]: stage k reads
    // S[p] (k = 1) or the stage buffer A/B and writes the other one; the
    // accumulator X0 lives in Acc; the last stage puts u, v in Acc when the tail
    // follows (else in S[1-p]) and eta in S[1-p].
    StageArgs<T, Tp> stage_args(sw_ctx* ctx, int k, int p, bool tail_now, T Fxt, T Fyt) const {
        const sw_config& c = ctx->cfg;
        const Geom& g = ctx->g;
        const Fields3& X = ctx->S[p];
        const Fields3& Y = ctx->S[1 - p];
        StageArgs<T, Tp> a;
        a.g = g;
        a.nsx = (g.N + STRIP - 1) / STRIP; a.nsy = (g.M + ctx->stage_ty - 1) / ctx->stage_ty;
        a.nring_blocks = ring_blocks(g, 128);
        const Fields3& in = (k == 1) ? X : ((k % 2 == 0) ? ctx->A : ctx->B);
        const Fields3& out1 = (k % 2 == 1) ? ctx->A : ctx->B;
        a.u1 = (const Tp*)in.u; a.v1 = (const Tp*)in.v; a.e1 = (const Tp*)in.e;
        a.uX = (const Tp*)X.u; a.vX = (const Tp*)X.v; a.eX = (const Tp*)X.e;
        a.u0i = (const Tp*)ctx->Acc.u; a.v0i = (const Tp*)ctx->Acc.v; a.e0i = (const Tp*)ctx->Acc.e;
        const bool last = (k == c.RKo);
        if (!last) { a.u1o = (Tp*)out1.u; a.v1o = (Tp*)out1.v; a.e1o = (Tp*)out1.e; }
        else { a.u1o = a.v1o = a.e1o = nullptr; }
        if (last) {
            // the final X0: u, v to Acc when the tail follows, else straight into
            // the new state; eta always into the new state (the tail keeps eta)
            a.u0o = (Tp*)(tail_now ? ctx->Acc.u : Y.u);
            a.v0o = (Tp*)(tail_now ? ctx->Acc.v : Y.v);
            a.e0o = (Tp*)Y.e;
        } else {
            a.u0o = (Tp*)ctx->Acc.u; a.v0o = (Tp*)ctx->Acc.v; a.e0o = (Tp*)ctx->Acc.e;
        }
        a.H = sf<T>(ctx->H); a.fq = sf<T>(ctx->fq); a.Fx = sf<T>(ctx->Fx); a.Fy = sf<T>(ctx->Fy);
        a.a = (Tp)c.RKaDt[k - 1];
        a.b = (k < c.RKo) ? (Tp)c.RKbDt[k - 1] : Tp(0);
        a.g_ = (T)c.g;
        a.Fxt = Fxt; a.Fyt = Fyt;
        set_cont(ctx, a);
        a.gr = rule(ctx);
        a.st = ctx->dst;
        a.spin_limit = ctx->spin_limit;
        a.skip_chunk = ctx->test_skip_chunk;
        return a;
    }
    // The tail's arguments for a step from S[p]: u0, v0 in Acc, eta0 in S[1-p]
    TailArgs<T, Tp> tail_args(sw_ctx* ctx, int p) const {
        const sw_config& c = ctx->cfg;
        const Geom& g = ctx->g;
        const Fields3& Y = ctx->S[1 - p];
        TailArgs<T, Tp> a;
        a.g = g;
        a.nsx = (g.N + STRIP - 1) / STRIP; a.nsy = (g.M + ctx->tail_ty - 1) / ctx->tail_ty;
        a.nring_blocks = ring_blocks(g, 128);
        a.u0 = (const Tp*)ctx->Acc.u; a.v0 = (const Tp*)ctx->Acc.v; a.e0 = (const Tp*)Y.e;
        a.uo = (Tp*)Y.u; a.vo = (Tp*)Y.v;
        a.H = sf<T>(ctx->H);
        a.cD = (T)c.cD; a.rD = (T)c.rD; a.cSmag = (T)c.cSmag; a.nuB = (T)c.nuB;
        a.Dt_diff = (Tp)c.Dt_diff;
        a.gr = rule(ctx);
        a.st = ctx->dst;
        return a;
    }
    // The tracer's arguments for a step from S[p], reading sst[sp] and writing sst[1-sp]
    TracerArgs<T, Tp> tracer_args(sw_ctx* ctx, int p, int sp) const {
        const sw_config& c = ctx->cfg;
        const Fields3& Y = ctx->S[1 - p];
        TracerArgs<T, Tp> a;
        a.g = ctx->g;
        a.u = (const Tp*)Y.u; a.v = (const Tp*)Y.v;
        a.um = (const T*)ctx->um; a.vm = (const T*)ctx->vm;
        a.sst = (const Tp*)ctx->sst[sp];
        a.sst_o = (Tp*)ctx->sst[1 - sp];
        a.dtadvu = (T)c.dtadvu; a.dtadvv = (T)c.dtadvv;
        a.half_dtadvu = (T)c.half_dtadvu; a.half_dtadvv = (T)c.half_dtadvv;
        a.jSST = (T)c.jSST; a.SSTmin = (T)c.SSTmin;
        a.gr = rule(ctx);
        a.st = ctx->dst;
        return a;
    }

    int step(sw_ctx* ctx, long long i) override {
        const sw_config& c = ctx->cfg;
        const Geom& g = ctx->g;
        Fields3& X = ctx->S[ctx->p];
        Fields3& Y = ctx->S[1 - ctx->p];
        const bool tail_now = (i % c.nstep_diff) == 0;
        const T one = T(1);
        T Fxt = c.seasonal_wind_x ? (T)std::sin(c.omegaFx * (double)ctx->t) : one;
        T Fyt = c.seasonal_wind_y ? (T)std::sin(c.omegaFy * (double)ctx->t) : one;

        // ------------------------------------------------ RK stages (:55-78)
        const int nsx = (g.N + STRIP - 1) / STRIP, nsy = (g.M + ctx->stage_ty - 1) / ctx->stage_ty;
        const int nring = ring_blocks(g, 128);
        const int nblk = (nsx * nsy + 3) / 4 + nring;
        if (c.time_scheme != SW_RK) {
            if (int rc = ssp_stages(ctx, X, Y, tail_now, Fxt, Fyt)) return rc;
        } else {
        for (int k = 1; k <= c.RKo; k++) {
            StageArgs<T, Tp> a = stage_args(ctx, k, ctx->p, tail_now, Fxt, Fyt);
            const Fields3& in = (k == 1) ? X : ((k % 2 == 0) ? ctx->A : ctx->B);
            const bool first = (k == 1), last = (k == c.RKo);
            if (last) ctx->rhs_in = in;
            int rc;
            if (c.dynamics == SW_LINEAR) {
                rc = launch(ctx, 0, [&] { lin_rk_dispatch(ctx, a, g.ep != 0, first, last); });
            } else if (TMA_TYPES && ctx->use_tma && a.cont == 0 && !a.sadourny && !a.qS) {
                StageMaps mp;
                mp.in_u = ctx->tmaps[in.u].in; mp.in_v = ctx->tmaps[in.v].in; mp.in_e = ctx->tmaps[in.e].in;
                mp.x_u = ctx->tmaps[X.u].x; mp.x_v = ctx->tmaps[X.v].x; mp.x_e = ctx->tmaps[X.e].x;
                mp.a_u = ctx->tmaps[ctx->Acc.u].x; mp.a_v = ctx->tmaps[ctx->Acc.v].x; mp.a_e = ctx->tmaps[ctx->Acc.e].x;
                int lr = 0;
                rc = launch(ctx, 0, [&] { lr = stage_tma_dispatch(ctx, a, mp, g.ep != 0, first, last); });
                if (!rc && lr) rc = fail(ctx, SW_ERR_CUDA, "TMA stage kernel could not be configured");
            } else {
                rc = launch(ctx, 0, [&] { stage_dispatch(a, g.ep != 0, first, last, nblk, ctx->stream, ctx->stage_ty); });
            }
            if (rc) return rc;
        }

        }

        // ---------------------- advection/Coriolis refresh (:208-211)
        if (ctx->qS && (i % c.nstep_advcor) == 0) {
            const void* u0 = tail_now ? ctx->Acc.u : Y.u;
            const void* v0 = tail_now ? ctx->Acc.v : Y.v;
            if (int rc = advcor_refresh(ctx, u0, v0, Y.e, false)) return rc;
        }

        // -------------------------------------- drag + diffusion (:216-221)
        if (tail_now) {
            TailArgs<T, Tp> a = tail_args(ctx, ctx->p);
            const int nb = (a.nsx * a.nsy + 3) / 4 + a.nring_blocks;
            const bool smag = (c.diffusion == SW_DIFF_SMAGORINSKY);
            const int rc = launch(ctx, 1, [&] {
                if (g.ep) tail_dispatch2<true>(a, c.bottom_drag, smag, nb, ctx->stream, ctx->tail_ty);
                else tail_dispatch2<false>(a, c.bottom_drag, smag, nb, ctx->stream, ctx->tail_ty);
            });
            if (rc) return rc;
            // bottom_drag_quadratic! leaves its KEu, KEv (of u0) for the next stages
            if (ctx->qS && c.bottom_drag == SW_DRAG_QUADRATIC)
                if (int rq = advcor_refresh(ctx, ctx->Acc.u, ctx->Acc.v, Y.e, true)) return rq;
        }
        ctx->t += c.dtint;

        // ------------------------------------------------ tracer (:226-228)
        if (c.tracer_advection) {
            if (c.nadvstep > 1 && ((i + c.nadvstep_half) % c.nadvstep) == 0) {
                int rc = launch(ctx, 5, [&] {
                    copy_convert_kernel<T, Tp><<<296, 256, 0, ctx->stream>>>(
                        (const Tp*)Y.u, (const Tp*)Y.v, (T*)ctx->um, (T*)ctx->vm, (long long)ctx->nelem, ctx->dst);
                });
                if (rc) return rc;
            }
            if ((i % c.nadvstep) == 0) {
                TracerArgs<T, Tp> a = tracer_args(ctx, ctx->p, ctx->sp);
                const bool um_is_u = (c.nadvstep == 1);
                const dim3 grid = tracer_grid(ctx);
                int rc = launch(ctx, 2, [&] {
                    if (g.ep) tracer_dispatch2<true>(a, um_is_u, c.tracer_consumption != 0, grid, ctx->stream);
                    else tracer_dispatch2<false>(a, um_is_u, c.tracer_consumption != 0, grid, ctx->stream);
                });
                if (rc) return rc;
                ctx->sp = 1 - ctx->sp;
            }
        }

        return SW_OK;
    }

    // advection/Coriolis refresh (nstep_advcor > 0) from u, v, eta with valid
    // ghosts; KE only after a quadratic-drag tail (sw_advcor.cuh)
    int advcor_refresh(sw_ctx* ctx, const void* u, const void* v, const void* e, bool ke_only) {
        const Geom& g = ctx->g;
        dim3 grid((g.N + 4 + 255) / 256, g.M + 2);
        return launch(ctx, 3, [&] {
            auto args = [&](auto kern) {
                kern<<<grid, 256, 0, ctx->stream>>>(g, (const Tp*)u, (const Tp*)v, (const Tp*)e, sf<T>(ctx->H),
                                                    sf<T>(ctx->fq), (T*)ctx->qS, (T*)ctx->KEuS, (T*)ctx->KEvS);
            };
            if (g.ep) {
                if (ke_only) args(advcor_refresh_kernel<T, Tp, true, true>);
                else args(advcor_refresh_kernel<T, Tp, true, false>);
            } else {
                if (ke_only) args(advcor_refresh_kernel<T, Tp, false, true>);
                else args(advcor_refresh_kernel<T, Tp, false, false>);
            }
        });
    }
    // the prologue of time_integration (src/time_integration.jl:20-31): the
    // advection/Coriolis terms of the initial state
    int prologue(sw_ctx* ctx) override {
        if (!ctx->qS) return SW_OK;
        const Fields3& X = ctx->S[ctx->p];
        return advcor_refresh(ctx, X.u, X.v, X.e, false);
    }

    int diagnostics(sw_ctx* ctx, sw_diag* out) override {
        if (!ctx->diag) {
            const size_t bytes = (DIAG_BLOCKS + 1) * sizeof(DiagPartial);
            CK(cached_malloc((void**)&ctx->diag, bytes));
            ctx->allocs.push_back({ctx->diag, bytes});
        }
        const Fields3& X = ctx->S[ctx->p];
        int rc = launch(ctx, 5, [&] {
            diag_partial_kernel<T, Tp><<<DIAG_BLOCKS, DIAG_THREADS, 0, ctx->stream>>>(
                ctx->g, (const Tp*)X.u, (const Tp*)X.v, (const Tp*)X.e, (const Tp*)ctx->sst[ctx->sp], sf<T>(ctx->H),
                ctx->cfg.g, ctx->diag);
            diag_final_kernel<<<1, 32, 0, ctx->stream>>>(ctx->diag, DIAG_BLOCKS, ctx->diag + DIAG_BLOCKS);
        });
        if (rc) return rc;
        DiagPartial r;
        CK(cudaMemcpyAsync(&r, ctx->diag + DIAG_BLOCKS, sizeof(r), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        out->mass = r.mass;
        out->energy = r.energy;
        out->max_speed = r.max_speed;
        out->nan_count = (int64_t)r.nan_count;
        return SW_OK;
    }

    // NaN check of step i (src/time_integration.jl:232-237): u, v, eta before
    // the step (still S[p]) and sst after it
    int nan_check(sw_ctx* ctx, long long i) override {
        const Geom& g = ctx->g;
        const Fields3& X = ctx->S[ctx->p];
        return launch(ctx, 4, [&] {
            nan_check_kernel<Tp><<<148, 256, 0, ctx->stream>>>(g, (const Tp*)X.u, (const Tp*)X.v, (const Tp*)X.e,
                                                              (const Tp*)ctx->sst[ctx->sp], i, ctx->dst);
        });
    }
};

// The 16-bit storage form (sw_s16.cuh): T = Tprog = Float32 arithmetic on a
// state held in 16-bit pairs.  The FP32 buffers of the context carry the
// state only across uploads, downloads and diagnostics (S[p], sst[sp]); the
// last RK stage's X0 goes to Acc (u0, v0, eta0) as in the native form.  The
// rest of a step lives in 16-bit arrays: the state pairs of both parities, the
// stage values X1 (two sets), the increments D and the tracer (two parities).
template <class S16>
struct Engine16 : Engine<float, float> {
    using Base = Engine<float, float>;
    struct F3 { S16* u = nullptr; S16* v = nullptr; S16* e = nullptr; };
    F3 hi[2], lo[2], X1[2], D[2];   // X1: stage increments δ, D: accumulated increments (each read from one and written to the other)
    S16* sst16[2] = {nullptr, nullptr};
    float s = 1024.f, inv_s = 1.f / 1024.f;

    int init(sw_ctx* ctx) {
        const sw_config& c = ctx->cfg;
        s = (float)c.storage_scale_uv;
        inv_s = (float)(1.0 / c.storage_scale_uv);
        const size_t bytes = ctx->nelem * sizeof(S16);
        auto alloc = [&](S16** p) -> int {
            void* q = nullptr;
            CK(cached_malloc(&q, bytes));
            ctx->allocs.push_back({q, bytes});
            ctx->zeroed.push_back({q, bytes});
            CK(cudaMemsetAsync(q, 0, bytes, ctx->stream));
            *p = static_cast<S16*>(q);
            return SW_OK;
        };
        for (F3* f : {&hi[0], &hi[1], &lo[0], &lo[1], &X1[0], &X1[1], &D[0], &D[1]})
            for (S16** p : {&f->u, &f->v, &f->e})
                if (int rc = alloc(p)) return rc;
        for (S16** p : {&sst16[0], &sst16[1]})
            if (int rc = alloc(p)) return rc;
        return SW_OK;
    }

    int state_uploaded(sw_ctx* ctx) override {
        const Fields3& F = ctx->S[ctx->p];
        const int p = ctx->p;
        return launch(ctx, 5, [&] {
            s16_pack_kernel<S16><<<4 * ctx->nsm, 256, 0, ctx->stream>>>(
                (const float*)F.u, (const float*)F.v, (const float*)F.e, (const float*)ctx->sst[ctx->sp],
                hi[p].u, lo[p].u, hi[p].v, lo[p].v, hi[p].e, lo[p].e, sst16[ctx->sp], (long long)ctx->nelem, s);
        });
    }
    int state_to_fp32(sw_ctx* ctx) override {
        const Fields3& F = ctx->S[ctx->p];
        const int p = ctx->p;
        return launch(ctx, 5, [&] {
            s16_unpack_kernel<S16><<<4 * ctx->nsm, 256, 0, ctx->stream>>>(
                hi[p].u, lo[p].u, hi[p].v, lo[p].v, hi[p].e, lo[p].e, sst16[ctx->sp], (float*)F.u, (float*)F.v,
                (float*)F.e, (float*)ctx->sst[ctx->sp], (long long)ctx->nelem, inv_s);
        });
    }
    int diagnostics(sw_ctx* ctx, sw_diag* out) override {
        if (int rc = state_to_fp32(ctx)) return rc;
        return Base::diagnostics(ctx, out);
    }
    int nan_check(sw_ctx* ctx, long long i) override {
        const int p = ctx->p;
        return launch(ctx, 4, [&] {
            s16_nan_check_kernel<S16><<<148, 256, 0, ctx->stream>>>(ctx->g, hi[p].u, hi[p].v, hi[p].e,
                                                                    sst16[ctx->sp], i, ctx->dst);
        });
    }

    template <bool PER, bool FIRST, bool LAST, int TY>
    static void stage16(const S16StageArgs<S16>& a, int nblk, cudaStream_t st) {
        s16_stage_kernel<S16, PER, FIRST, LAST, TY><<<nblk, 128, 0, st>>>(a);
    }
    template <bool PER, bool FIRST, bool LAST>
    static void stage16_ty(const S16StageArgs<S16>& a, int nblk, cudaStream_t st, int ty) {
        if (ty == 8) stage16<PER, FIRST, LAST, 8>(a, nblk, st);
        else if (ty == 16) stage16<PER, FIRST, LAST, 16>(a, nblk, st);
        else stage16<PER, FIRST, LAST, 32>(a, nblk, st);
    }
    template <bool PER, int DRAG, bool SMAG>
    static void tail16(const TailArgs<float, float>& a, const TailStorePair<S16>& o, int nblk, cudaStream_t st, int ty) {
        if (ty == 8) s16_tail_kernel<S16, PER, DRAG, SMAG, 8><<<nblk, 128, 0, st>>>(a, o);
        else if (ty == 16) s16_tail_kernel<S16, PER, DRAG, SMAG, 16><<<nblk, 128, 0, st>>>(a, o);
        else s16_tail_kernel<S16, PER, DRAG, SMAG, 32><<<nblk, 128, 0, st>>>(a, o);
    }
    template <bool PER>
    static void tail16_opts(const TailArgs<float, float>& a, const TailStorePair<S16>& o, int drag, bool smag,
                            int nblk, cudaStream_t st, int ty) {
        if (smag) {
            if (drag == SW_DRAG_QUADRATIC) tail16<PER, SW_DRAG_QUADRATIC, true>(a, o, nblk, st, ty);
            else if (drag == SW_DRAG_LINEAR) tail16<PER, SW_DRAG_LINEAR, true>(a, o, nblk, st, ty);
            else tail16<PER, SW_DRAG_NONE, true>(a, o, nblk, st, ty);
        } else {
            if (drag == SW_DRAG_QUADRATIC) tail16<PER, SW_DRAG_QUADRATIC, false>(a, o, nblk, st, ty);
            else if (drag == SW_DRAG_LINEAR) tail16<PER, SW_DRAG_LINEAR, false>(a, o, nblk, st, ty);
            else tail16<PER, SW_DRAG_NONE, false>(a, o, nblk, st, ty);
        }
    }
    template <bool PER>
    static void tracer16(const TracerArgs<float, float>& a, const TracerIO16<S16>& io, bool um_is_u, bool cons,
                         dim3 grid, cudaStream_t st) {
        if (um_is_u) {
            if (cons) s16_tracer_kernel<S16, PER, true, true><<<grid, 128, 0, st>>>(a, io);
            else s16_tracer_kernel<S16, PER, true, false><<<grid, 128, 0, st>>>(a, io);
        } else {
            if (cons) s16_tracer_kernel<S16, PER, false, true><<<grid, 128, 0, st>>>(a, io);
            else s16_tracer_kernel<S16, PER, false, false><<<grid, 128, 0, st>>>(a, io);
        }
    }

    // The operands of RK stage k from the pairs of parity p: stage k reads the
    // increment δ of stage k-1 (X1 = state + δ) and writes its own.
    S16StageArgs<S16> stage16_args(sw_ctx* ctx, int k, int p, float Fxt, float Fyt) const {
        const sw_config& c = ctx->cfg;
        const Geom& g = ctx->g;
        const int q = 1 - p;
        S16StageArgs<S16> a;
        a.g = g;
        a.nsx = (g.N + STRIP - 1) / STRIP; a.nsy = (g.M + ctx->stage_ty - 1) / ctx->stage_ty;
        a.nring_blocks = ring_blocks(g, 128);
        a.uh = hi[p].u; a.vh = hi[p].v; a.eh = hi[p].e;
        a.ul = lo[p].u; a.vl = lo[p].v; a.el = lo[p].e;
        const F3& din1 = X1[k % 2 == 0 ? 0 : 1];
        const F3& dout1 = X1[k % 2 == 1 ? 0 : 1];
        a.ud = din1.u; a.vd = din1.v; a.ed = din1.e;
        a.udo = dout1.u; a.vdo = dout1.v; a.edo = dout1.e;
        const F3& din = D[k % 2], &dout = D[(k + 1) % 2];
        a.uD = din.u; a.vD = din.v; a.eD = din.e;
        a.uDo = dout.u; a.vDo = dout.v; a.eDo = dout.e;
        a.u0o = (float*)ctx->Acc.u; a.v0o = (float*)ctx->Acc.v; a.e0o = (float*)ctx->Acc.e;
        a.eho = hi[q].e; a.elo = lo[q].e;
        a.H = sf<float>(ctx->H); a.fq = sf<float>(ctx->fq); a.Fx = sf<float>(ctx->Fx); a.Fy = sf<float>(ctx->Fy);
        a.a = (float)c.RKaDt[k - 1];
        a.b = (k < c.RKo) ? (float)c.RKbDt[k - 1] : 0.f;
        a.g_ = (float)c.g; a.Fxt = Fxt; a.Fyt = Fyt;
        a.s = s; a.inv_s = inv_s;
        a.gr = rule(ctx);
        a.st = ctx->dst;
        return a;
    }
    // the tail from parity p: X0 of the last stage in, the new u, v pairs of 1 - p out
    TailArgs<float, float> tail16_args(sw_ctx* ctx, int p) const {
        TailArgs<float, float> t = tail_args(ctx, p);
        t.e0 = (const float*)ctx->Acc.e;     // the last stage's FP32 eta (depth of the drag)
        return t;
    }
    TailStorePair<S16> tail16_out(int p) const {
        const int q = 1 - p;
        return TailStorePair<S16>{hi[q].u, lo[q].u, hi[q].v, lo[q].v, s};
    }
    // the tracer after a step from parity p, from sst16[sp] to sst16[1 - sp]
    TracerArgs<float, float> tracer16_args(sw_ctx* ctx, int p, int sp) const {
        const int q = 1 - p;
        TracerArgs<float, float> t = tracer_args(ctx, p, sp);
        t.u = reinterpret_cast<const float*>(hi[q].u);
        t.v = reinterpret_cast<const float*>(hi[q].v);
        t.sst = reinterpret_cast<const float*>(sst16[sp]);
        t.sst_o = reinterpret_cast<float*>(sst16[1 - sp]);
        return t;
    }

    // One time step from the pairs of parity p to those of 1 - p: RK stages
    // (src/time_integration.jl:55-78), the tail (:216-221) and the tracer
    // (:226-228), as in Engine::step, on the 16-bit arrays.
    int step(sw_ctx* ctx, long long i) override {
        const sw_config& c = ctx->cfg;
        const Geom& g = ctx->g;
        const int p = ctx->p, q = 1 - p;
        const bool tail_now = (i % c.nstep_diff) == 0;
        const float Fxt = c.seasonal_wind_x ? (float)std::sin(c.omegaFx * (double)ctx->t) : 1.f;
        const float Fyt = c.seasonal_wind_y ? (float)std::sin(c.omegaFy * (double)ctx->t) : 1.f;

        for (int k = 1; k <= c.RKo; k++) {
            const S16StageArgs<S16> a = stage16_args(ctx, k, p, Fxt, Fyt);
            const int nblk = (a.nsx * a.nsy + 3) / 4 + a.nring_blocks;
            const bool first = k == 1, last = k == c.RKo;
            const int rc = launch(ctx, 0, [&] {
                if (g.ep) {
                    if (first) stage16_ty<true, true, false>(a, nblk, ctx->stream, ctx->stage_ty);
                    else if (last) stage16_ty<true, false, true>(a, nblk, ctx->stream, ctx->stage_ty);
                    else stage16_ty<true, false, false>(a, nblk, ctx->stream, ctx->stage_ty);
                } else {
                    if (first) stage16_ty<false, true, false>(a, nblk, ctx->stream, ctx->stage_ty);
                    else if (last) stage16_ty<false, false, true>(a, nblk, ctx->stream, ctx->stage_ty);
                    else stage16_ty<false, false, false>(a, nblk, ctx->stream, ctx->stage_ty);
                }
            });
            if (rc) return rc;
        }

        if (tail_now) {
            const TailArgs<float, float> t = tail16_args(ctx, p);
            const TailStorePair<S16> o = tail16_out(p);
            const int nb = (t.nsx * t.nsy + 3) / 4 + t.nring_blocks;
            const bool smag = c.diffusion == SW_DIFF_SMAGORINSKY;
            const int rc = launch(ctx, 1, [&] {
                if (g.ep) tail16_opts<true>(t, o, c.bottom_drag, smag, nb, ctx->stream, ctx->tail_ty);
                else tail16_opts<false>(t, o, c.bottom_drag, smag, nb, ctx->stream, ctx->tail_ty);
            });
            if (rc) return rc;
        } else {
            const int rc = launch(ctx, 5, [&] {
                s16_pack_uv_kernel<S16><<<4 * ctx->nsm, 256, 0, ctx->stream>>>(
                    (const float*)ctx->Acc.u, (const float*)ctx->Acc.v, hi[q].u, lo[q].u, hi[q].v, lo[q].v,
                    (long long)ctx->nelem, s, ctx->dst);
            });
            if (rc) return rc;
        }
        ctx->t += c.dtint;

        if (c.tracer_advection) {
            if (c.nadvstep > 1 && ((i + c.nadvstep_half) % c.nadvstep) == 0) {
                const int rc = launch(ctx, 5, [&] {
                    s16_copy_uv_kernel<S16><<<296, 256, 0, ctx->stream>>>(hi[q].u, hi[q].v, (float*)ctx->um,
                                                                          (float*)ctx->vm, (long long)ctx->nelem,
                                                                          inv_s, ctx->dst);
                });
                if (rc) return rc;
            }
            if ((i % c.nadvstep) == 0) {
                const TracerArgs<float, float> t = tracer16_args(ctx, p, ctx->sp);
                const TracerIO16<S16> io{inv_s};
                const bool um_is_u = c.nadvstep == 1;
                const dim3 grid = tracer_grid(ctx);
                const int rc = launch(ctx, 2, [&] {
                    if (g.ep) tracer16<true>(t, io, um_is_u, c.tracer_consumption != 0, grid, ctx->stream);
                    else tracer16<false>(t, io, um_is_u, c.tracer_consumption != 0, grid, ctx->stream);
                });
                if (rc) return rc;
                ctx->sp = 1 - ctx->sp;
            }
        }
        return SW_OK;
    }
};

// ------------------------------------------------------------------ helpers

int check_config(const sw_config* c, std::string& why) {
    if (c->abi_version != SWB200_ABI_VERSION) { why = "abi_version mismatch"; return SW_ERR_ARG; }
    if (c->nx < 4 || c->ny < 4) { why = "nx and ny must be >= 4"; return SW_ERR_ARG; }
    if (c->halo != 2 || c->haloeta != 1 || c->halosstx != 1 || c->halossty != 0) {
        why = "halo sizes must be (2,1,1,0) as in src/grid.jl:50-53";
        return SW_ERR_ARG;
    }
    if (!fmt_size(c->T) || !fmt_size(c->Tprog) || !fmt_size(c->Tcomm)) { why = "unknown number format"; return SW_ERR_ARG; }
    if (c->nstep_diff < 1 || c->nadvstep < 1 || c->nout < 1 || c->dtint < 1) { why = "step counts must be >= 1"; return SW_ERR_ARG; }
    if (c->time_scheme < SW_RK || c->time_scheme > SW_4SSPRK3) { why = "unknown time_scheme"; return SW_ERR_ARG; }
    if (c->time_scheme == SW_SSPRK2 && c->RKs < 2) { why = "SSPRK2 needs RKs >= 2"; return SW_ERR_ARG; }
    if (c->time_scheme == SW_SSPRK3 && (c->ssp_s < 2 || c->ssp_kn < 2 || c->ssp_kn > c->ssp_s + 1)) {
        why = "inconsistent SSPRK3 coefficients";
        return SW_ERR_ARG;
    }
    if (c->time_scheme == SW_RK && (c->RKo < 2 || c->RKo > 4)) { why = "RKo must be 2, 3 or 4"; return SW_ERR_ARG; }
    if (c->dynamics != SW_NONLINEAR && c->dynamics != SW_LINEAR) { why = "unknown dynamics"; return SW_ERR_ARG; }
    if (c->adv_scheme != SW_ARAKAWA_HSU && c->adv_scheme != SW_SADOURNY) { why = "unknown adv_scheme"; return SW_ERR_ARG; }
    if (c->nstep_advcor < 0) { why = "nstep_advcor must be >= 0"; return SW_ERR_ARG; }
    if (c->surface_relax && c->surface_forcing) { why = "surface_relax and surface_forcing are exclusive"; return SW_ERR_ARG; }
    if (c->storage != SW_STORE_NATIVE && c->storage != SW_STORE_BF16 && c->storage != SW_STORE_F16) {
        why = "unknown storage";
        return SW_ERR_ARG;
    }
    if (c->storage != SW_STORE_NATIVE) {
        const double s = c->storage_scale_uv;
        int ex = 0;
        if (!(s > 0) || std::frexp(s, &ex) != 0.5 || c->T != SW_FLOAT32 || c->Tprog != SW_FLOAT32) {
            why = "16-bit storage needs T = Tprog = Float32 and a power-of-two storage_scale_uv";
            return SW_ERR_ARG;
        }
        if (c->time_scheme != SW_RK || c->dynamics != SW_NONLINEAR || c->adv_scheme != SW_ARAKAWA_HSU ||
            c->nstep_advcor != 0 || c->surface_relax || c->surface_forcing) {
            why = "the 16-bit storage form is built for RK, nonlinear dynamics with Arakawa-Hsu advection, "
                  "nstep_advcor = 0 and the plain continuity equation";
            return SW_ERR_UNSUPPORTED;
        }
    }
    bool ok = (c->T == SW_FLOAT32 && c->Tprog == SW_FLOAT32) || (c->T == SW_FLOAT64 && c->Tprog == SW_FLOAT64) ||
              (c->T == SW_FLOAT32 && c->Tprog == SW_FLOAT64) || (c->T == SW_FLOAT16 && c->Tprog == SW_FLOAT32) ||
              (c->T == SW_FLOAT16 && c->Tprog == SW_FLOAT16);
    if (!ok) { why = "(T, Tprog) pair not built"; return SW_ERR_UNSUPPORTED; }
    return SW_OK;
}

// Rows [j0, j1) of a w-wide host field with W-sized elements (bitwise):
// whether every row is constant along x (the row equals itself shifted by one
// element), and whether every row equals row 0.  memcmp compares in wide
// words; a row stays in cache between its two comparisons.
template <class W>
void scan_rows(const unsigned char* src, int w, int j0, int j1, bool& cx, bool& cy) {
    const size_t rb = (size_t)w * sizeof(W);
    for (int j = j0; j < j1 && (cx || cy); j++) {
        const unsigned char* r = src + (size_t)j * rb;
        if (cx && w > 1) cx = std::memcmp(r, r + sizeof(W), rb - sizeof(W)) == 0;
        if (cy && j > 0) cy = std::memcmp(r, src, rb) == 0;
    }
}

// Both tests over the whole field, on the OpenMP threads when it is large
// (host arrays are element-aligned, so they are read as W words).
template <class W>
void scan_field(const unsigned char* src, int w, int h, bool& const_x, bool& const_y) {
    bool cx = true, cy = true;
    const long long bytes = (long long)w * h * sizeof(W);
    static const int ncpu = std::max(1, omp_get_num_procs());
    const int nt = (int)std::min<long long>(std::min(16, ncpu), std::max<long long>(1, bytes >> 20));
#pragma omp parallel for num_threads(nt) reduction(&& : cx, cy) schedule(static) if (nt > 1)
    for (int k = 0; k < nt; k++) {
        bool x = true, y = true;
        scan_rows<W>(src, w, (int)((long long)h * k / nt), (int)((long long)h * (k + 1) / nt), x, y);
        cx = cx && x;
        cy = cy && y;
    }
    const_x = cx;
    const_y = cy;
}

// Host-side packing of a static field (T, x fastest, host column 0 at
// physical x = hx0, row 0 at y = hy0, size w x h) into its strided SField
// form: constant fields and fields that vary along one axis only become
// broadcast vectors.
struct PackedStatic { std::vector<unsigned char> buf; int sx = 0, sy = 0; };
PackedStatic pack_static(const sw_ctx* ctx, const void* host, int w, int h, int hx0, int hy0) {
    const size_t ts = ctx->tsz;
    const unsigned char* src = static_cast<const unsigned char*>(host);
    auto el = [&](int i, int j) { return src + ((size_t)j * w + i) * ts; };
    bool const_x = true, const_y = true;
    if (ts == 2) scan_field<uint16_t>(src, w, h, const_x, const_y);
    else if (ts == 4) scan_field<uint32_t>(src, w, h, const_x, const_y);
    else scan_field<uint64_t>(src, w, h, const_x, const_y);
    const Geom& g = ctx->g;
    PackedStatic out;
    std::vector<unsigned char>& buf = out.buf;
    if (const_x && const_y) {
        buf.assign(ts, 0);
        std::memcpy(buf.data(), el(0, 0), ts);
        out.sx = 0; out.sy = 0;
    } else if (const_x) {                      // varies with y only: indexed by row
        buf.assign((size_t)g.R * ts, 0);
        for (int j = 0; j < h; j++) std::memcpy(&buf[(size_t)(hy0 + j + ROW0) * ts], el(0, j), ts);
        out.sx = 0; out.sy = 1;
    } else if (const_y) {                      // varies with x only: indexed by column
        buf.assign((size_t)g.P * ts, 0);
        for (int i = 0; i < w; i++) std::memcpy(&buf[(size_t)(hx0 + i + COL0) * ts], el(i, 0), ts);
        out.sx = 1; out.sy = 0;
    } else {
        buf.assign((size_t)g.P * g.R * ts, 0);
        for (int j = 0; j < h; j++)
            std::memcpy(&buf[((size_t)(hy0 + j + ROW0) * g.P + (hx0 + COL0)) * ts], el(0, j), ts * (size_t)w);
        out.sx = 1; out.sy = g.P;
    }
    return out;
}

// Upload a static field into out.  A field already on the device with the
// same packed layout is overwritten in place (its address, and so every
// captured step graph, stays valid); SW_ERR_UNSUPPORTED tells a caller that
// refreshes a context that the layout changed.  The copy is asynchronous on
// the context's stream: the packed buffer is kept in ctx->staging until the
// caller synchronises.
int upload_static(sw_ctx* ctx, sw_ctx::SF& out, PackedStatic&& pk) {
    if (out.p) {
        if (out.bytes != pk.buf.size() || out.sx != pk.sx || out.sy != pk.sy) return SW_ERR_UNSUPPORTED;
    } else {
        CK(cached_malloc(&out.p, pk.buf.size()));
        ctx->allocs.push_back({out.p, pk.buf.size()});
        out.bytes = pk.buf.size();
        out.sx = pk.sx; out.sy = pk.sy;
    }
    CK(cudaMemcpyAsync(out.p, pk.buf.data(), pk.buf.size(), cudaMemcpyHostToDevice, ctx->stream));
    ctx->staging.push_back(std::move(pk.buf));
    return SW_OK;
}

// The static fields of a context (src/grid.jl:93-95, src/forcing.jl:1-53):
// uploaded at creation, and again when a cached context is reused.
// All fields are scanned and packed on the host first, then copied: a copy
// from pageable memory waits for the work before it on the stream, and the
// scans should overlap that work (the state's copies of a refreshed context).
int upload_statics(sw_ctx* ctx, const sw_static* st) {
    const sw_config* cfg = &ctx->cfg;
    const Geom& g = ctx->g;
    const int N = g.N, M = g.M, nux = g.ep ? N : N - 1;
    struct Job { sw_ctx::SF* out; const void* host; int w, h, hx0, hy0; };
    std::vector<Job> jobs = {{&ctx->fq, st->f_q, N + 1, M + 1, 0, 0}, {&ctx->Fx, st->Fx, nux, M, 1 - g.ep, 0},
                             {&ctx->Fy, st->Fy, N, M - 1, 0, 1}, {&ctx->H, st->H, N + 2, M + 2, -1, -1}};
    if (cfg->dynamics == SW_LINEAR) {
        if (!st->f_u || !st->f_v) return fail(ctx, SW_ERR_ARG, "linear dynamics needs f_u and f_v");
        jobs.push_back({&ctx->fu, st->f_u, nux, M, 1 - g.ep, 0});
        jobs.push_back({&ctx->fv, st->f_v, N, M - 1, 0, 1});
    }
    if (cfg->surface_relax) {
        if (!st->eta_ref) return fail(ctx, SW_ERR_ARG, "surface_relax needs eta_ref");
        jobs.push_back({&ctx->eref, st->eta_ref, N, M, 0, 0});
    }
    if (cfg->surface_forcing) {
        if (!st->Feta) return fail(ctx, SW_ERR_ARG, "surface_forcing needs Feta");
        jobs.push_back({&ctx->Feta, st->Feta, N, M, 0, 0});
    }
    std::vector<PackedStatic> packed;
    for (const Job& j : jobs) packed.push_back(pack_static(ctx, j.host, j.w, j.h, j.hx0, j.hy0));
    for (size_t k = 0; k < jobs.size(); k++)
        if (int rc = upload_static(ctx, *jobs[k].out, std::move(packed[k]))) return rc;
    return SW_OK;
}

// state transfers: host arrays with halo <-> device layout
struct HostShape { int w, h, x0, y0; };
HostShape shape_u(const Geom& g) { return {(g.ep ? g.N : g.N - 1) + 4, g.M + 4, g.ep ? -2 : -1, -2}; }
HostShape shape_v(const Geom& g) { return {g.N + 4, g.M + 3, -2, -1}; }
HostShape shape_e(const Geom& g) { return {g.N + 2, g.M + 2, -1, -1}; }
HostShape shape_s(const Geom& g) { return {g.N + 2, g.M, -1, 0}; }

int copy_in(sw_ctx* ctx, void* dev, const void* host, HostShape s) {
    const size_t es = ctx->tpsz;
    char* d = static_cast<char*>(dev) + ((size_t)(s.y0 + ROW0) * ctx->g.P + (s.x0 + COL0)) * es;
    CK(cudaMemcpy2DAsync(d, ctx->g.P * es, host, s.w * es, s.w * es, s.h, cudaMemcpyHostToDevice, ctx->stream));
    return SW_OK;
}
int copy_out(sw_ctx* ctx, void* host, const void* dev, HostShape s) {
    const size_t es = ctx->tpsz;
    const char* d = static_cast<const char*>(dev) + ((size_t)(s.y0 + ROW0) * ctx->g.P + (s.x0 + COL0)) * es;
    CK(cudaMemcpy2DAsync(host, s.w * es, d, ctx->g.P * es, s.w * es, s.h, cudaMemcpyDeviceToHost, ctx->stream));
    return SW_OK;
}

// What a step launches, beyond the fixed buffers: the state and tracer
// parities and which sub-steps are due.  Steps with equal keys launch the same
// kernels with the same arguments (the seasonal wind factors excepted, which
// is why those runs are not graphed).
unsigned step_key(const sw_ctx* ctx, long long i) {
    const sw_config& c = ctx->cfg;
    const bool tail_now = (i % c.nstep_diff) == 0;
    const bool tracer_now = c.tracer_advection && (i % c.nadvstep) == 0;
    const bool copy_now = c.tracer_advection && c.nadvstep > 1 && ((i + c.nadvstep_half) % c.nadvstep) == 0;
    const bool refresh_now = c.nstep_advcor > 0 && (i % c.nstep_advcor) == 0;
    return (unsigned)ctx->p | (unsigned)ctx->sp << 1 | (unsigned)tail_now << 2 | (unsigned)tracer_now << 3 |
           (unsigned)copy_now << 4 | (unsigned)refresh_now << 5;
}

// One time step: replayed from a CUDA graph when possible, captured on first use.
int do_step(sw_ctx* ctx, long long i) {
    const sw_config& c = ctx->cfg;
    if (!ctx->use_graphs || ctx->prof || c.seasonal_wind_x || c.seasonal_wind_y || c.surface_forcing)
        return ctx->eng->step(ctx, i);
    const unsigned key = step_key(ctx, i);
    auto it = ctx->graphs.find(key);
    if (it == ctx->graphs.end()) {
        const long long t0 = ctx->t, l0 = ctx->launches;
        const int sp0 = ctx->sp;
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        int rc = ctx->eng->step(ctx, i);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
        sw_ctx::StepGraph sg;
        sg.launches = ctx->launches - l0;
        sg.flips_sp = ctx->sp != sp0;
        sg.rhs_in = ctx->rhs_in;
        ctx->t = t0; ctx->launches = l0; ctx->sp = sp0;
        if (!rc && e == cudaSuccess) e = cudaGraphInstantiate(&sg.exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (rc) return rc;
        if (e != cudaSuccess) {
            // capture is an optimisation: run this context without graphs
            (void)cudaGetLastError();
            ctx->use_graphs = false;
            return ctx->eng->step(ctx, i);
        }
        it = ctx->graphs.emplace(key, sg).first;
    }
    CK(cudaGraphLaunch(it->second.exec, ctx->stream));
    ctx->launches += it->second.launches;
    ctx->t += c.dtint;
    if (it->second.flips_sp) ctx->sp = 1 - ctx->sp;
    ctx->rhs_in = it->second.rhs_in;
    return SW_OK;
}

int run_steps(sw_ctx* ctx, long long nsteps, sw_status* status) {
    const sw_config& c = ctx->cfg;
    long long done = 0;
    int code = SW_OK;
    for (long long s = 0; s < nsteps; s++) {
        long long i = ctx->step + 1;
        int rc = do_step(ctx, i);
        if (rc) return rc;
        done++;
        bool check = (i % c.nout) == 0;
        if (check) {
            if ((rc = ctx->eng->nan_check(ctx, i))) return rc;
            CK(cudaMemcpyAsync(ctx->hst, ctx->dst, sizeof(DevStatus), cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            if (ctx->hst->error) {
                code = ctx->hst->error;
                ctx->step = i;
                break;
            }
            if (ctx->hst->stop) {
                // state stays S[p] (before this step); the tracer already moved sst
                ctx->step = i;
                code = SW_NAN_DETECTED;
                break;
            }
        }
        ctx->p = 1 - ctx->p;
        ctx->step = i;
    }
    if (code == SW_OK) {
        CK(cudaMemcpyAsync(ctx->hst, ctx->dst, sizeof(DevStatus), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (ctx->hst->error) code = ctx->hst->error;
    }
    if (status) {
        status->steps_done = done;
        status->step = ctx->step;
        status->nan_step = (code == SW_NAN_DETECTED) ? ctx->step : -1;
        status->code = code;
    }
    if (code == SW_ERR_DEPARTURE) ctx->err = "tracer departure point outside the domain";
    if (code == SW_NAN_DETECTED) ctx->err = "NaNs detected at time step " + std::to_string(ctx->step);
    return code;
}

// The environment settings a context reads at creation (kernel choices and
// test caps); a cached context is reused only under the same settings.
std::string env_settings() {
    std::string s;
    for (const char* k : {"SWB200_TMA", "SWB200_GRAPHS", "SWB200_STAGE_BLOCKS", "SWB200_TAIL_TY", "SWB200_STAGE_TY",
                          "SWB200_TEST_WAIT_LIMIT", "SWB200_TEST_SKIP_CHUNK"}) {
        const char* v = getenv(k);
        s += k;
        s += '=';
        s += v ? v : "";
        s += ';';
    }
    return s;
}

// ----------------------------------------------------------------- drop-in cache
// sw_time_integration keeps the contexts of its finished calls (at most
// DROPIN_CACHE) and gives one to a later call whose configuration equals it in
// everything but nt, in the same CUDA context and under the same environment
// settings.  Such a call skips creation (allocation, tensor-map encoding, step
// graph capture): it zeroes the context's buffers as creation would, uploads
// the static fields again (in place; if their packed layout changed, the
// context is rebuilt) and then runs exactly as on a new context.
constexpr size_t DROPIN_CACHE = 4;
struct DropinCache {
    std::mutex mu;
    std::vector<sw_ctx*> idle;     // oldest first
};
DropinCache& dropin_cache() {
    static DropinCache* c = new DropinCache();   // never destroyed: may be used during process exit
    return *c;
}

bool same_run_config(const sw_config& a, const sw_config& b) {
    sw_config x = a, y = b;
    x.nt = y.nt = 0;
    return std::memcmp(&x, &y, sizeof(sw_config)) == 0;
}

sw_ctx* take_dropin(const sw_config* cfg) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    const unsigned long long cid = current_context_id();
    if (!cid) return nullptr;
    const std::string env = env_settings();
    DropinCache& c = dropin_cache();
    std::lock_guard<std::mutex> lock(c.mu);
    for (size_t k = c.idle.size(); k-- > 0;) {
        sw_ctx* x = c.idle[k];
        if (x->device == dev && x->context_id == cid && x->env == env && same_run_config(x->cfg, *cfg)) {
            c.idle.erase(c.idle.begin() + (long)k);
            return x;
        }
    }
    return nullptr;
}

// Zero the context's buffers (as sw_create leaves them) and upload the static
// fields of this call; anything but SW_OK means: do not use this context.
// sw_set_state in two parts: the state's copies into the device layout
// (asynchronous), then the kernels that read it (the prologue, which may read
// the static fields too, the ghost points and the storage form's copy).
int state_copy_in(sw_ctx* ctx, const void* u, const void* v, const void* eta, const void* sst) {
    ctx->p = 0; ctx->sp = 0; ctx->step = 0; ctx->t = 0;
    ctx->rhs_in = Fields3();
    int rc;
    if ((rc = copy_in(ctx, ctx->S[0].u, u, shape_u(ctx->g)))) return rc;
    if ((rc = copy_in(ctx, ctx->S[0].v, v, shape_v(ctx->g)))) return rc;
    if ((rc = copy_in(ctx, ctx->S[0].e, eta, shape_e(ctx->g)))) return rc;
    if ((rc = copy_in(ctx, ctx->sst[0], sst, shape_s(ctx->g)))) return rc;
    CK(cudaMemsetAsync(ctx->dst, 0, sizeof(DevStatus), ctx->stream));
    CK(cudaMemsetAsync(ctx->sched, 0, sizeof(TileSched), ctx->stream));
    return SW_OK;
}
int state_prepare(sw_ctx* ctx) {
    int rc;
    // the prologue reads the state as given, before any ghost point copy
    // (src/time_integration.jl:20-31)
    if ((rc = ctx->eng->prologue(ctx))) return rc;
    // ghost_points!(u,v,eta) opens every step (src/time_integration.jl:48); it is
    // idempotent after the first, so it is applied once here
    if ((rc = ctx->eng->ghost_state(ctx))) return rc;
    return ctx->eng->state_uploaded(ctx);
}

// A cached context made ready for a call: its buffers zeroed, the state's
// copies issued first so that the host's scan of the static fields overlaps
// them, the static fields uploaded in place, then the state's kernels.
int refresh_dropin(sw_ctx* ctx, const sw_config* cfg, const sw_static* st, const void* u, const void* v,
                   const void* eta, const void* sst) {
    ctx->cfg.nt = cfg->nt;
    ctx->err.clear();
    for (auto& z : ctx->zeroed) CK(cudaMemsetAsync(z.first, 0, z.second, ctx->stream));
    int rc;
    if ((rc = state_copy_in(ctx, u, v, eta, sst))) return rc;
    if ((rc = upload_statics(ctx, st))) return rc;
    if ((rc = state_prepare(ctx))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->staging.clear();
    return SW_OK;
}

}  // namespace

extern "C" void sw_destroy(sw_ctx* ctx);

namespace {

void put_dropin(sw_ctx* ctx) {
    sw_ctx* evict = nullptr;
    {
        DropinCache& c = dropin_cache();
        std::lock_guard<std::mutex> lock(c.mu);
        c.idle.push_back(ctx);
        if (c.idle.size() > DROPIN_CACHE) {
            evict = c.idle.front();
            c.idle.erase(c.idle.begin());
        }
    }
    if (evict) {
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(evict->device);
        sw_destroy(evict);
        cudaSetDevice(cur);
    }
}

// destroys every cached drop-in context (sw_trim_memory)
void release_dropin_contexts() {
    std::vector<sw_ctx*> all;
    {
        DropinCache& c = dropin_cache();
        std::lock_guard<std::mutex> lock(c.mu);
        all.swap(c.idle);
    }
    int cur = 0;
    cudaGetDevice(&cur);
    for (sw_ctx* x : all) {
        cudaSetDevice(x->device);
        if (current_context_id() == x->context_id) sw_destroy(x);
        else delete x;      // its CUDA context is gone, and its blocks and stream with it
    }
    cudaSetDevice(cur);
}

}  // namespace

// ======================================================================= batches
// An ensemble advanced with one launch per sub-step for all members that share
// the boundary type and options (sw_batch.cuh).  Each member is a full context
// (its buffers, static fields and state); the batch adds the device tables of
// every member's kernel arguments.  A global step is replayed from one of two
// CUDA graphs (by the parity of the step): each group's launches run on a
// stream of its own, forked from and joined back to the batch stream, and a
// last one-thread kernel moves the device-side step counter on.
// Rows per warp strip of the batched stage and tail kernels: the candidates
// the batch's autotuner times on the first steps of a run.  Every candidate
// computes the same values (only the assignment of rows to warps differs).
constexpr int BATCH_NTY = 4;
constexpr int BATCH_TYS[BATCH_NTY] = {4, 8, 16, 32};

struct BatchGroup {
    int per = 1, rko = 4, drag = 0, storage = SW_STORE_NATIVE;
    bool smag = false, um_is_u = true, cons = false, tracer_any = false;
    std::vector<int> idx;                      // member indices
    // argument tables: StageArgs, TailArgs, TracerArgs, BatchCopy, BatchNan for
    // native members; S16StageArgs, S16TailBatchArgs, S16TracerBatchArgs,
    // BatchCopy16, BatchNan16 of the storage type for 16-bit members
    void* stage[BATCH_NTY][2][4] = {};          // per tile height, parity of X, stage
    void* tail[BATCH_NTY][2] = {};
    void* tracer[2] = {};                       // 2n entries: k odd, then k even
    void* copy[2] = {};
    void* nan[2] = {};                          // 2n entries: even, then odd tracer count
    BatchMember* memb = nullptr;
    int *b_stage[BATCH_NTY] = {}, *b_tail[BATCH_NTY] = {}, *b_tracer = nullptr, *nbx_tracer = nullptr,
        *b_copy = nullptr, *b_nan = nullptr;
    int n_stage[BATCH_NTY] = {}, n_tail[BATCH_NTY] = {}, n_tracer = 0, n_copy = 0, n_nan = 0;
};

struct sw_batch {
    std::vector<sw_ctx*> mem;
    std::vector<BatchGroup> groups;
    std::vector<std::pair<void*, size_t>> tables;
    cudaStream_t stream = nullptr;
    std::vector<cudaStream_t> gstreams;        // one per group
    std::vector<cudaEvent_t> events;           // fork, then one join per group
    long long* d_step = nullptr;               // the global step the next replay runs
    cudaGraphExec_t graph[BATCH_NTY][2] = {};  // per tile height; global steps i with (i - 1) % 2 == 0, 1
    int ty = -1;                               // chosen tile height (index into BATCH_TYS), -1 until tuned
    std::string shape_key;                     // member shapes and options, the autotuner's cache key
    long long step = 0, max_nt = 0;
    long long launches = 0, launches_per_step[BATCH_NTY][2] = {};
    std::string err;
};

namespace {

template <class V>
int upload_table(sw_batch* b, const std::vector<V>& host, V** dev) {
    const size_t bytes = host.size() * sizeof(V);
    void* p = nullptr;
    if (cached_malloc(&p, bytes) != cudaSuccess) return SW_ERR_NOMEM;
    b->tables.push_back({p, bytes});
    if (cudaMemcpyAsync(p, host.data(), bytes, cudaMemcpyHostToDevice, b->stream) != cudaSuccess) return SW_ERR_CUDA;
    *dev = static_cast<V*>(p);
    return SW_OK;
}

std::vector<int> prefix(const std::vector<int>& counts) {
    std::vector<int> o(counts.size() + 1, 0);
    for (size_t k = 0; k < counts.size(); k++) o[k + 1] = o[k] + counts[k];
    return o;
}

int batch_check(const sw_config& c, std::string& why) {
    if (c.T != SW_FLOAT32 || c.Tprog != SW_FLOAT32) why = "batched members compute in Float32";
    else if (c.time_scheme != SW_RK) why = "batched members use the RK schemes";
    else if (c.dynamics != SW_NONLINEAR || c.nstep_advcor != 0) why = "batched members use nonlinear dynamics without nstep_advcor";
    else if (c.nstep_diff != 1) why = "batched members apply drag and diffusion every step (nstep_diff = 1)";
    else if (c.seasonal_wind_x || c.seasonal_wind_y || c.surface_forcing) why = "batched members have no time-dependent forcing";
    else return SW_OK;
    return SW_ERR_UNSUPPORTED;
}

template <class V>
int upload_table(sw_batch* b, const std::vector<V>& host, void** dev) {
    V* d = nullptr;
    const int rc = upload_table(b, host, &d);
    *dev = d;
    return rc;
}

// the argument tables of a group of native members, per state parity p
int batch_tables(sw_batch* b, BatchGroup& gr) {
    using E = Engine<float, float>;
    const int n = (int)gr.idx.size();
    int rc;
    for (int p = 0; p < 2; p++) {
        for (int ti = 0; ti < BATCH_NTY; ti++) {
            for (int k = 1; k <= gr.rko; k++) {
                std::vector<StageArgs<float, float>> v;
                for (int m : gr.idx) {
                    v.push_back(dynamic_cast<E*>(b->mem[m]->eng.get())->stage_args(b->mem[m], k, p, true, 1.f, 1.f));
                    v.back().nsy = (b->mem[m]->g.M + BATCH_TYS[ti] - 1) / BATCH_TYS[ti];
                }
                if ((rc = upload_table(b, v, &gr.stage[ti][p][k - 1]))) return rc;
            }
            std::vector<TailArgs<float, float>> vt;
            for (int m : gr.idx) {
                vt.push_back(dynamic_cast<E*>(b->mem[m]->eng.get())->tail_args(b->mem[m], p));
                vt.back().nsy = (b->mem[m]->g.M + BATCH_TYS[ti] - 1) / BATCH_TYS[ti];
            }
            if ((rc = upload_table(b, vt, &gr.tail[ti][p]))) return rc;
        }
        std::vector<TracerArgs<float, float>> vr(2 * n);
        std::vector<BatchCopy> vc;
        std::vector<BatchNan> vn(2 * n);
        for (int q = 0; q < n; q++) {
            sw_ctx* ctx = b->mem[gr.idx[q]];
            E* e = dynamic_cast<E*>(ctx->eng.get());
            vr[q] = e->tracer_args(ctx, p, 0);          // k odd: sst[0] -> sst[1]
            vr[n + q] = e->tracer_args(ctx, p, 1);      // k even: sst[1] -> sst[0]
            const Fields3& X = ctx->S[p];
            const Fields3& Y = ctx->S[1 - p];
            vc.push_back(BatchCopy{(const float*)Y.u, (const float*)Y.v, (float*)ctx->um, (float*)ctx->vm,
                                   (long long)ctx->nelem, ctx->dst});
            for (int par = 0; par < 2; par++)
                vn[par * n + q] = BatchNan{ctx->g, (const float*)X.u, (const float*)X.v, (const float*)X.e,
                                           (const float*)ctx->sst[par], ctx->dst};
        }
        if ((rc = upload_table(b, vr, &gr.tracer[p]))) return rc;
        if ((rc = upload_table(b, vc, &gr.copy[p]))) return rc;
        if ((rc = upload_table(b, vn, &gr.nan[p]))) return rc;
    }
    return SW_OK;
}

// the same for 16-bit members, from the arguments their lone steps launch with
// (Engine16::stage16_args, tail16_args, tail16_out, tracer16_args)
template <class S16>
int batch_tables16(sw_batch* b, BatchGroup& gr) {
    using E = Engine16<S16>;
    const int n = (int)gr.idx.size();
    auto eng = [&](int m) { return dynamic_cast<E*>(b->mem[m]->eng.get()); };
    int rc;
    for (int p = 0; p < 2; p++) {
        for (int ti = 0; ti < BATCH_NTY; ti++) {
            for (int k = 1; k <= gr.rko; k++) {
                std::vector<S16StageArgs<S16>> v;
                for (int m : gr.idx) {
                    v.push_back(eng(m)->stage16_args(b->mem[m], k, p, 1.f, 1.f));
                    v.back().nsy = (b->mem[m]->g.M + BATCH_TYS[ti] - 1) / BATCH_TYS[ti];
                }
                if ((rc = upload_table(b, v, &gr.stage[ti][p][k - 1]))) return rc;
            }
            std::vector<S16TailBatchArgs<S16>> vt;
            for (int m : gr.idx) {
                vt.push_back(S16TailBatchArgs<S16>{eng(m)->tail16_args(b->mem[m], p), eng(m)->tail16_out(p)});
                vt.back().t.nsy = (b->mem[m]->g.M + BATCH_TYS[ti] - 1) / BATCH_TYS[ti];
            }
            if ((rc = upload_table(b, vt, &gr.tail[ti][p]))) return rc;
        }
        std::vector<S16TracerBatchArgs<S16>> vr(2 * n);
        std::vector<BatchCopy16<S16>> vc;
        std::vector<BatchNan16<S16>> vn(2 * n);
        for (int q = 0; q < n; q++) {
            sw_ctx* ctx = b->mem[gr.idx[q]];
            E* e = eng(gr.idx[q]);
            const TracerIO16<S16> io{e->inv_s};
            vr[q] = S16TracerBatchArgs<S16>{e->tracer16_args(ctx, p, 0), io};       // k odd: sst16[0] -> sst16[1]
            vr[n + q] = S16TracerBatchArgs<S16>{e->tracer16_args(ctx, p, 1), io};   // k even: sst16[1] -> sst16[0]
            const int r = 1 - p;
            vc.push_back(BatchCopy16<S16>{e->hi[r].u, e->hi[r].v, (float*)ctx->um, (float*)ctx->vm,
                                          (long long)ctx->nelem, e->inv_s, ctx->dst});
            for (int par = 0; par < 2; par++)
                vn[par * n + q] = BatchNan16<S16>{ctx->g, e->hi[p].u, e->hi[p].v, e->hi[p].e, e->sst16[par], ctx->dst};
        }
        if ((rc = upload_table(b, vr, &gr.tracer[p]))) return rc;
        if ((rc = upload_table(b, vc, &gr.copy[p]))) return rc;
        if ((rc = upload_table(b, vn, &gr.nan[p]))) return rc;
    }
    return SW_OK;
}

int batch_build(sw_batch* b) {
    using E = Engine<float, float>;
    std::map<std::vector<int>, int> key_group;
    for (int m = 0; m < (int)b->mem.size(); m++) {
        const sw_config& c = b->mem[m]->cfg;
        const std::vector<int> key = {c.periodic != 0, c.nadvstep == 1 || !c.tracer_advection, c.RKo,
                                      c.bottom_drag, c.diffusion, c.tracer_consumption, c.storage};
        auto it = key_group.find(key);
        if (it == key_group.end()) {
            it = key_group.emplace(key, (int)b->groups.size()).first;
            BatchGroup gr;
            gr.per = c.periodic != 0;
            gr.um_is_u = key[1] != 0;
            gr.rko = c.RKo;
            gr.drag = c.bottom_drag;
            gr.smag = c.diffusion == SW_DIFF_SMAGORINSKY;
            gr.cons = c.tracer_consumption != 0;
            gr.storage = c.storage;
            b->groups.push_back(gr);
        }
        b->groups[it->second].idx.push_back(m);
    }
    for (BatchGroup& gr : b->groups) {
        const int n = (int)gr.idx.size();
        std::vector<int> cs[BATCH_NTY], ct[BATCH_NTY], ctr, nbx, cc, cn;
        std::vector<BatchMember> mems;
        for (int m : gr.idx) {
            sw_ctx* ctx = b->mem[m];
            const Geom& g = ctx->g;
            const sw_config& c = ctx->cfg;
            E* e = dynamic_cast<E*>(ctx->eng.get());
            const StageArgs<float, float> s1 = e->stage_args(ctx, 1, 0, true, 1.f, 1.f);
            const TailArgs<float, float> t0 = e->tail_args(ctx, 0);
            for (int ti = 0; ti < BATCH_NTY; ti++) {
                const int nsy = (g.M + BATCH_TYS[ti] - 1) / BATCH_TYS[ti];
                cs[ti].push_back((s1.nsx * nsy + 3) / 4 + s1.nring_blocks);
                ct[ti].push_back((t0.nsx * nsy + 3) / 4 + t0.nring_blocks);
            }
            b->shape_key += std::to_string(g.N) + "x" + std::to_string(g.M) + (c.periodic ? "p" : "n") + ",";
            const int bx = (g.N + 127) / 128, gy = std::min(g.M, 256);
            nbx.push_back(bx);
            ctr.push_back(bx * gy);
            cc.push_back(16);
            cn.push_back(8);
            BatchMember bm;
            bm.nt = c.nt; bm.tracer = c.tracer_advection; bm.nadvstep = c.nadvstep;
            bm.nadvstep_half = c.nadvstep_half; bm.nout = c.nout; bm.cells = g.N * g.M;
            mems.push_back(bm);
            gr.tracer_any = gr.tracer_any || c.tracer_advection;
            b->max_nt = std::max(b->max_nt, (long long)c.nt);
        }
        int rc;
        b->shape_key += "|" + std::to_string(gr.per) + std::to_string(gr.um_is_u) + std::to_string(gr.rko) +
                        std::to_string(gr.drag) + std::to_string(gr.smag) + std::to_string(gr.cons) +
                        std::to_string(gr.storage) + ";";
        if (gr.storage == SW_STORE_BF16) rc = batch_tables16<__nv_bfloat16>(b, gr);
        else if (gr.storage == SW_STORE_F16) rc = batch_tables16<__half>(b, gr);
        else rc = batch_tables(b, gr);
        if (rc) return rc;
        for (int ti = 0; ti < BATCH_NTY; ti++) {
            const std::vector<int> ps = prefix(cs[ti]), pt = prefix(ct[ti]);
            gr.n_stage[ti] = ps.back();
            gr.n_tail[ti] = pt.back();
            if ((rc = upload_table(b, ps, &gr.b_stage[ti])) || (rc = upload_table(b, pt, &gr.b_tail[ti]))) return rc;
        }
        const std::vector<int> ptr = prefix(ctr), pc = prefix(cc), pn = prefix(cn);
        gr.n_tracer = ptr.back(); gr.n_copy = pc.back(); gr.n_nan = pn.back();
        if ((rc = upload_table(b, ptr, &gr.b_tracer)) || (rc = upload_table(b, nbx, &gr.nbx_tracer)) ||
            (rc = upload_table(b, pc, &gr.b_copy)) || (rc = upload_table(b, pn, &gr.b_nan)) ||
            (rc = upload_table(b, mems, &gr.memb)))
            return rc;
    }
    if (const int rc = upload_table(b, std::vector<long long>{1}, &b->d_step)) return rc;
    for (size_t g = 0; g <= b->groups.size(); g++) {
        cudaEvent_t ev;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return SW_ERR_CUDA;
        b->events.push_back(ev);
        if (g == b->groups.size()) break;
        cudaStream_t st;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return SW_ERR_CUDA;
        b->gstreams.push_back(st);
    }
    return cudaStreamSynchronize(b->stream) == cudaSuccess ? SW_OK : SW_ERR_CUDA;
}

// the launches of group gr for a global step of parity p (the step read from
// b->d_step), on stream s; returns how many
template <bool PER, int TY>
int batch_group_step(sw_batch* b, const BatchGroup& gr, int p, cudaStream_t s, int ti) {
    const int n = (int)gr.idx.size();
    const long long* i = b->d_step;
    int launches = 0;
    const int nst = gr.n_stage[ti], ntl = gr.n_tail[ti];
    const int* bst = gr.b_stage[ti];
    for (int k = 1; k <= gr.rko; k++) {
        const auto* a = static_cast<const StageArgs<float, float>*>(gr.stage[ti][p][k - 1]);
        if (k == 1) rk_stage_batch<float, float, PER, true, false, TY><<<nst, 128, 0, s>>>(a, bst, n, gr.memb, i);
        else if (k == gr.rko) rk_stage_batch<float, float, PER, false, true, TY><<<nst, 128, 0, s>>>(a, bst, n, gr.memb, i);
        else rk_stage_batch<float, float, PER, false, false, TY><<<nst, 128, 0, s>>>(a, bst, n, gr.memb, i);
    }
    const auto* ta = static_cast<const TailArgs<float, float>*>(gr.tail[ti][p]);
    auto tail = [&](auto kern) { kern<<<ntl, 128, 0, s>>>(ta, gr.b_tail[ti], n, gr.memb, i); };
    if (gr.smag) {
        if (gr.drag == SW_DRAG_QUADRATIC) tail(tail_batch<float, float, PER, SW_DRAG_QUADRATIC, true, TY>);
        else if (gr.drag == SW_DRAG_LINEAR) tail(tail_batch<float, float, PER, SW_DRAG_LINEAR, true, TY>);
        else tail(tail_batch<float, float, PER, SW_DRAG_NONE, true, TY>);
    } else {
        if (gr.drag == SW_DRAG_QUADRATIC) tail(tail_batch<float, float, PER, SW_DRAG_QUADRATIC, false, TY>);
        else if (gr.drag == SW_DRAG_LINEAR) tail(tail_batch<float, float, PER, SW_DRAG_LINEAR, false, TY>);
        else tail(tail_batch<float, float, PER, SW_DRAG_NONE, false, TY>);
    }
    launches += gr.rko + 1;
    if (gr.tracer_any) {
        if (!gr.um_is_u) {
            copy_batch<<<gr.n_copy, 256, 0, s>>>(static_cast<const BatchCopy*>(gr.copy[p]), gr.b_copy, n, gr.memb, i);
            launches++;
        }
        const auto* ra = static_cast<const TracerArgs<float, float>*>(gr.tracer[p]);
        auto tr = [&](auto kern) { kern<<<gr.n_tracer, 128, 0, s>>>(ra, gr.b_tracer, gr.nbx_tracer, n, gr.memb, i); };
        if (gr.um_is_u) { if (gr.cons) tr(tracer_batch<float, float, PER, true, true>); else tr(tracer_batch<float, float, PER, true, false>); }
        else { if (gr.cons) tr(tracer_batch<float, float, PER, false, true>); else tr(tracer_batch<float, float, PER, false, false>); }
        launches++;
    }
    nan_batch<<<gr.n_nan, 256, 0, s>>>(static_cast<const BatchNan*>(gr.nan[p]), gr.b_nan, n, gr.memb, i);
    return launches + 1;
}

// the same for a group of 16-bit members (the launches of Engine16::step)
template <class S16, bool PER, int TY>
int batch16_group_step(sw_batch* b, const BatchGroup& gr, int p, cudaStream_t s, int ti) {
    const int n = (int)gr.idx.size();
    const long long* i = b->d_step;
    int launches = 0;
    const int nst = gr.n_stage[ti], ntl = gr.n_tail[ti];
    const int* bst = gr.b_stage[ti];
    for (int k = 1; k <= gr.rko; k++) {
        const auto* a = static_cast<const S16StageArgs<S16>*>(gr.stage[ti][p][k - 1]);
        if (k == 1) s16_stage_batch<S16, PER, true, false, TY><<<nst, 128, 0, s>>>(a, bst, n, gr.memb, i);
        else if (k == gr.rko) s16_stage_batch<S16, PER, false, true, TY><<<nst, 128, 0, s>>>(a, bst, n, gr.memb, i);
        else s16_stage_batch<S16, PER, false, false, TY><<<nst, 128, 0, s>>>(a, bst, n, gr.memb, i);
    }
    const auto* ta = static_cast<const S16TailBatchArgs<S16>*>(gr.tail[ti][p]);
    auto tail = [&](auto kern) { kern<<<ntl, 128, 0, s>>>(ta, gr.b_tail[ti], n, gr.memb, i); };
    if (gr.smag) {
        if (gr.drag == SW_DRAG_QUADRATIC) tail(s16_tail_batch<S16, PER, SW_DRAG_QUADRATIC, true, TY>);
        else if (gr.drag == SW_DRAG_LINEAR) tail(s16_tail_batch<S16, PER, SW_DRAG_LINEAR, true, TY>);
        else tail(s16_tail_batch<S16, PER, SW_DRAG_NONE, true, TY>);
    } else {
        if (gr.drag == SW_DRAG_QUADRATIC) tail(s16_tail_batch<S16, PER, SW_DRAG_QUADRATIC, false, TY>);
        else if (gr.drag == SW_DRAG_LINEAR) tail(s16_tail_batch<S16, PER, SW_DRAG_LINEAR, false, TY>);
        else tail(s16_tail_batch<S16, PER, SW_DRAG_NONE, false, TY>);
    }
    launches += gr.rko + 1;
    if (gr.tracer_any) {
        if (!gr.um_is_u) {
            s16_copy_batch<S16><<<gr.n_copy, 256, 0, s>>>(static_cast<const BatchCopy16<S16>*>(gr.copy[p]), gr.b_copy,
                                                          n, gr.memb, i);
            launches++;
        }
        const auto* ra = static_cast<const S16TracerBatchArgs<S16>*>(gr.tracer[p]);
        auto tr = [&](auto kern) { kern<<<gr.n_tracer, 128, 0, s>>>(ra, gr.b_tracer, gr.nbx_tracer, n, gr.memb, i); };
        if (gr.um_is_u) { if (gr.cons) tr(s16_tracer_batch<S16, PER, true, true>); else tr(s16_tracer_batch<S16, PER, true, false>); }
        else { if (gr.cons) tr(s16_tracer_batch<S16, PER, false, true>); else tr(s16_tracer_batch<S16, PER, false, false>); }
        launches++;
    }
    s16_nan_batch<S16><<<gr.n_nan, 256, 0, s>>>(static_cast<const BatchNan16<S16>*>(gr.nan[p]), gr.b_nan, n,
                                                gr.memb, i);
    return launches + 1;
}

template <bool PER, int TY>
int batch_group_step_storage(sw_batch* b, const BatchGroup& gr, int p, cudaStream_t s, int ti) {
    if (gr.storage == SW_STORE_BF16) return batch16_group_step<__nv_bfloat16, PER, TY>(b, gr, p, s, ti);
    if (gr.storage == SW_STORE_F16) return batch16_group_step<__half, PER, TY>(b, gr, p, s, ti);
    return batch_group_step<PER, TY>(b, gr, p, s, ti);
}

template <bool PER>
int batch_group_step_ty(sw_batch* b, const BatchGroup& gr, int p, cudaStream_t s, int ti) {
    switch (BATCH_TYS[ti]) {
        case 4: return batch_group_step_storage<PER, 4>(b, gr, p, s, ti);
        case 8: return batch_group_step_storage<PER, 8>(b, gr, p, s, ti);
        case 16: return batch_group_step_storage<PER, 16>(b, gr, p, s, ti);
        default: return batch_group_step_storage<PER, 32>(b, gr, p, s, ti);
    }
}

// captures the graph of a global step of parity p with tile height index ti:
// fork to the group streams, each group's launches, join, then batch_advance
int batch_graph(sw_batch* b, int p, int ti) {
    cudaStream_t s = b->stream;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return SW_ERR_CUDA;
    int launches = 0;
    cudaError_t e = cudaEventRecord(b->events[0], s);
    for (size_t g = 0; g < b->groups.size() && e == cudaSuccess; g++) {
        const BatchGroup& gr = b->groups[g];
        cudaStream_t gs = b->gstreams[g];
        if ((e = cudaStreamWaitEvent(gs, b->events[0], 0)) != cudaSuccess) break;
        launches += gr.per ? batch_group_step_ty<true>(b, gr, p, gs, ti) : batch_group_step_ty<false>(b, gr, p, gs, ti);
        if ((e = cudaEventRecord(b->events[g + 1], gs)) != cudaSuccess) break;
        e = cudaStreamWaitEvent(s, b->events[g + 1], 0);
    }
    if (e == cudaSuccess) {
        batch_advance<<<1, 32, 0, s>>>(b->d_step);
        launches++;
        e = cudaGetLastError();
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(s, &graph);
    if (e == cudaSuccess) e = ec;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph[ti][p], graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        b->err = std::string("batch graph: ") + cudaGetErrorString(e);
        return SW_ERR_CUDA;
    }
    b->launches_per_step[ti][p] = launches;
    return SW_OK;
}

int batch_graphs(sw_batch* b, int ti) {
    for (int p = 0; p < 2; p++)
        if (!b->graph[ti][p])
            if (const int rc = batch_graph(b, p, ti)) return rc;
    return SW_OK;
}

// tile heights chosen earlier in this process, by batch shape
std::mutex g_tune_mu;
std::map<std::string, int> g_tune_cache;

}  // namespace

// ======================================================================= C ABI
extern "C" {

int sw_abi_version(void) { return SWB200_ABI_VERSION; }

#ifndef SWB_FAST_BUILD
#define SWB_FAST_BUILD 0
#endif
int sw_build_kind(void) { return SWB_FAST_BUILD ? SW_BUILD_FAST : SW_BUILD_PARITY; }

const char* sw_strerror(int code) { return err_name(code); }

const char* sw_last_error(const sw_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

int64_t sw_kernel_launches(const sw_ctx* ctx) { return ctx ? ctx->launches : 0; }

int sw_batch_create(int32_t n, const sw_config* cfgs, const sw_static* statics, sw_batch** out) {
    if (n < 1 || !cfgs || !statics || !out) return SW_ERR_ARG;
    *out = nullptr;
    std::string why;
    for (int m = 0; m < n; m++) {
        const int rc = batch_check(cfgs[m], why);
        if (rc) {
            fprintf(stderr, "swb200: batch member %d: %s\n", m, why.c_str());
            return rc;
        }
    }
    std::unique_ptr<sw_batch> b(new sw_batch());
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return SW_ERR_CUDA;
    for (int m = 0; m < n; m++) {
        sw_ctx* ctx = nullptr;
        const int rc = sw_create(&cfgs[m], &statics[m], &ctx);
        if (rc) {
            sw_batch_destroy(b.release());
            return rc;
        }
        b->mem.push_back(ctx);
    }
    if (const int rc = batch_build(b.get())) {
        sw_batch_destroy(b.release());
        return rc;
    }
    *out = b.release();
    return SW_OK;
}

int sw_batch_set_state(sw_batch* b, int32_t member, const void* u, const void* v, const void* eta, const void* sst) {
    if (!b || member < 0 || member >= (int)b->mem.size()) return SW_ERR_ARG;
    const int rc = sw_set_state(b->mem[member], u, v, eta, sst);
    if (rc) return rc;
    b->step = 0;
    return SW_OK;
}

int sw_batch_run(sw_batch* b, int64_t nsteps, sw_status* statuses) {
    if (!b || nsteps < 0) return SW_ERR_ARG;
    for (sw_ctx* ctx : b->mem)          // states uploaded on the members' own streams
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return SW_ERR_CUDA;
    const long long until = std::min(b->max_nt, b->step + (long long)nsteps);
    const long long next = b->step + 1;
    cudaError_t e = cudaMemcpyAsync(b->d_step, &next, sizeof(next), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    long long i = next;
    auto launch_step = [&](int ti) {
        const int p = (int)((i - 1) % 2);
        e = cudaGraphLaunch(b->graph[ti][p], b->stream);
        b->launches += b->launches_per_step[ti][p];
        i++;
    };
    if (b->ty < 0) {   // the tile height: forced, remembered for this shape, or timed now
        const char* env = getenv("SWB200_BATCH_TY");
        const int want = env ? atoi(env) : 0;
        for (int ti = 0; ti < BATCH_NTY; ti++)
            if (BATCH_TYS[ti] == want) b->ty = ti;
        if (b->ty < 0) {
            std::lock_guard<std::mutex> lock(g_tune_mu);
            auto it = g_tune_cache.find(b->shape_key);
            if (it != g_tune_cache.end()) b->ty = it->second;
        }
    }
    // Autotuner: with no choice yet and enough steps in this call, every
    // candidate first advances two untimed global steps (both parities: the
    // graphs' first launches), then TUNE_ROUNDS interleaved rounds time
    // TUNE_STEPS steps of each candidate; the best round of each decides.
    // These are real steps of the run (every candidate computes the same
    // values).  The choice is kept for the batch and for later batches of the
    // same shape in this process.  SWB200_TUNE_LOG=1 prints the timings.
    constexpr int TUNE_STEPS = 3, TUNE_ROUNDS = 3;
    constexpr long long TUNE_TOTAL = (long long)BATCH_NTY * (2 + TUNE_ROUNDS * TUNE_STEPS);
    if (b->ty < 0 && until - next + 1 > TUNE_TOTAL) {
        cudaEvent_t ev[TUNE_ROUNDS][BATCH_NTY][2] = {};
        for (int ti = 0; ti < BATCH_NTY && e == cudaSuccess; ti++) {
            if (const int rc = batch_graphs(b, ti)) return rc;
            launch_step(ti);
            if (e == cudaSuccess) launch_step(ti);
        }
        for (int r = 0; r < TUNE_ROUNDS && e == cudaSuccess; r++)
            for (int ti = 0; ti < BATCH_NTY && e == cudaSuccess; ti++) {
                e = cudaEventCreate(&ev[r][ti][0]);
                if (e == cudaSuccess) e = cudaEventCreate(&ev[r][ti][1]);
                if (e == cudaSuccess) e = cudaEventRecord(ev[r][ti][0], b->stream);
                for (int k = 0; k < TUNE_STEPS && e == cudaSuccess; k++) launch_step(ti);
                if (e == cudaSuccess) e = cudaEventRecord(ev[r][ti][1], b->stream);
            }
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        float best_ms[BATCH_NTY];
        for (float& x : best_ms) x = 1e30f;
        for (int r = 0; r < TUNE_ROUNDS && e == cudaSuccess; r++)
            for (int ti = 0; ti < BATCH_NTY && e == cudaSuccess; ti++) {
                float ms = 0.f;
                e = cudaEventElapsedTime(&ms, ev[r][ti][0], ev[r][ti][1]);
                best_ms[ti] = std::min(best_ms[ti], ms);
            }
        for (auto& rr : ev)
            for (auto& pr : rr)
                for (cudaEvent_t x : pr)
                    if (x) cudaEventDestroy(x);
        if (e == cudaSuccess) {
            int best = BATCH_NTY - 1;
            for (int ti = 0; ti < BATCH_NTY; ti++)
                if (best_ms[ti] < best_ms[best]) best = ti;
            const char* lg = getenv("SWB200_TUNE_LOG");
            if (lg && lg[0] == '1') {
                fprintf(stderr, "swb200: batch tile rows:");
                for (int ti = 0; ti < BATCH_NTY; ti++) fprintf(stderr, " %d: %.3f ms", BATCH_TYS[ti], best_ms[ti]);
                fprintf(stderr, " -> %d\n", BATCH_TYS[best]);
            }
            b->ty = best;
            std::lock_guard<std::mutex> lock(g_tune_mu);
            g_tune_cache[b->shape_key] = best;
        }
    }
    const int ti = b->ty >= 0 ? b->ty : BATCH_NTY - 1;   // short calls before any tuning: the tallest tile
    if (e == cudaSuccess)
        if (const int rc = batch_graphs(b, ti)) return rc;
    while (i <= until && e == cudaSuccess) launch_step(ti);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) {
        b->err = std::string("batch run: ") + cudaGetErrorString(e);
        return SW_ERR_CUDA;
    }
    b->step = until;
    int code = SW_OK;
    for (int m = 0; m < (int)b->mem.size(); m++) {
        sw_ctx* ctx = b->mem[m];
        DevStatus ds;
        if (cudaMemcpy(&ds, ctx->dst, sizeof(ds), cudaMemcpyDeviceToHost) != cudaSuccess) return SW_ERR_CUDA;
        long long done = std::min(b->step, (long long)ctx->cfg.nt);
        int mc = SW_OK;
        if (ds.error) {
            mc = ds.error;
        } else if (ds.stop) {
            mc = SW_NAN_DETECTED;
            done = ds.nan_step;
        }
        // the member's state: before the failing step on a NaN stop, else after its last step
        const long long last = mc == SW_NAN_DETECTED ? done - 1 : done;
        ctx->p = (int)(last % 2);
        ctx->sp = ctx->cfg.tracer_advection ? (int)((done / ctx->cfg.nadvstep) % 2) : 0;
        ctx->step = done;
        if (statuses) {
            statuses[m].steps_done = done;
            statuses[m].step = done;
            statuses[m].nan_step = mc == SW_NAN_DETECTED ? done : -1;
            statuses[m].code = mc;
            statuses[m].reserved = 0;
        }
        if (mc && !code) code = mc;
    }
    return code;
}

int sw_batch_get_state(sw_batch* b, int32_t member, void* u, void* v, void* eta, void* sst) {
    if (!b || member < 0 || member >= (int)b->mem.size()) return SW_ERR_ARG;
    return sw_get_state(b->mem[member], u, v, eta, sst);
}

int64_t sw_batch_launches(const sw_batch* b) { return b ? b->launches : 0; }

int32_t sw_batch_tile_rows(const sw_batch* b) { return (b && b->ty >= 0) ? BATCH_TYS[b->ty] : 0; }

sw_ctx* sw_batch_member(sw_batch* b, int32_t member) {
    return (b && member >= 0 && member < (int)b->mem.size()) ? b->mem[member] : nullptr;
}

void sw_batch_destroy(sw_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (auto& gp : b->graph)
        for (cudaGraphExec_t g : gp)
            if (g) cudaGraphExecDestroy(g);
    for (cudaEvent_t ev : b->events) cudaEventDestroy(ev);
    for (cudaStream_t st : b->gstreams) cudaStreamDestroy(st);
    for (auto& t : b->tables) cached_free(t.first, t.second);
    for (sw_ctx* ctx : b->mem) sw_destroy(ctx);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int sw_trim_memory(void) {
    release_dropin_contexts();
    BlockCache& c = block_cache();
    std::lock_guard<std::mutex> lock(c.mu);
    int cur = 0;
    cudaGetDevice(&cur);
    for (auto& kv : c.dev) {
        // blocks of a context that no longer exists are dropped, not freed
        if (cudaSetDevice(kv.first.device) != cudaSuccess) continue;
        if (current_context_id() == kv.first.context) cudaFree(kv.second);
    }
    cudaSetDevice(cur);
    for (auto& kv : c.pinned) cudaFreeHost(kv.second);
    c.dev.clear();
    c.pinned.clear();
    c.cached = 0;
    return SW_OK;
}

void sw_destroy(sw_ctx* ctx) {
    if (!ctx) return;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second.exec);
    for (auto& a : ctx->allocs) cached_free(a.first, a.second);
    if (ctx->hst) cached_free_host(ctx->hst, sizeof(DevStatus));
    if (ctx->flush) cudaFree(ctx->flush);
    for (auto e : ctx->evpool) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int sw_create(const sw_config* cfg, const sw_static* st, sw_ctx** out) {
    if (!cfg || !st || !out) return SW_ERR_ARG;
    *out = nullptr;
    std::string why;
    int rc = check_config(cfg, why);
    if (rc) {
        fprintf(stderr, "swb200: %s\n", why.c_str());
        return rc;
    }
    if (!st->f_q || !st->Fx || !st->Fy || !st->H) return SW_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return SW_ERR_NODEVICE;

    std::unique_ptr<sw_ctx> holder(new sw_ctx());
    sw_ctx* ctx = holder.get();
    ctx->cfg = *cfg;
    CK(cudaGetDevice(&ctx->device));
    Geom& g = ctx->g;
    g.N = cfg->nx; g.M = cfg->ny; g.ep = cfg->periodic ? 1 : 0;
    g.P = ((g.N + 8 + PADX) + 31) / 32 * 32;
    g.R = g.M + 4 + PADY;
    ctx->nelem = (size_t)g.P * g.R;
    ctx->tsz = fmt_size(cfg->T);
    ctx->tpsz = fmt_size(cfg->Tprog);
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    ctx->context_id = current_context_id();
    ctx->env = env_settings();

    auto alloc = [&](void** p, size_t bytes) -> int {
        CK(cached_malloc(p, bytes));
        ctx->allocs.push_back({*p, bytes});
        ctx->zeroed.push_back({*p, bytes});
        CK(cudaMemsetAsync(*p, 0, bytes, ctx->stream));
        return SW_OK;
    };
    const size_t fb = ctx->nelem * ctx->tpsz;
    for (Fields3* f : {&ctx->S[0], &ctx->S[1], &ctx->A, &ctx->B, &ctx->Acc})
        for (void** p : {&f->u, &f->v, &f->e})
            if ((rc = alloc(p, fb))) return rc;
    if (cfg->time_scheme != SW_RK)
        for (void** p : {&ctx->C.u, &ctx->C.v, &ctx->C.e})
            if ((rc = alloc(p, fb))) return rc;
    if (cfg->dynamics == SW_NONLINEAR && cfg->nstep_advcor > 0)
        for (void** p : {&ctx->qS, &ctx->KEuS, &ctx->KEvS})
            if ((rc = alloc(p, ctx->nelem * ctx->tsz))) return rc;
    if ((rc = alloc(&ctx->sst[0], fb))) return rc;
    if ((rc = alloc(&ctx->sst[1], fb))) return rc;
    if (cfg->tracer_advection && cfg->nadvstep > 1) {
        if ((rc = alloc(&ctx->um, ctx->nelem * ctx->tsz))) return rc;
        if ((rc = alloc(&ctx->vm, ctx->nelem * ctx->tsz))) return rc;
    }
    {
        void* p = nullptr;
        if ((rc = alloc(&p, sizeof(DevStatus)))) return rc;
        ctx->dst = static_cast<DevStatus*>(p);
        if ((rc = alloc(&p, sizeof(TileSched)))) return rc;
        ctx->sched = static_cast<TileSched*>(p);
    }
    CK(cached_malloc_host((void**)&ctx->hst, sizeof(DevStatus)));
    std::memset(ctx->hst, 0, sizeof(DevStatus));

    if ((rc = upload_statics(ctx, st))) return rc;

    {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, dev);
        // The TMA stage kernel from four of its tiles per SM up (1536x768 and
        // larger); on smaller grids the streaming kernel with short strips
        // (measured faster: 110.8 against 115.4 us per step at 1024x512, 74
        // against 97 at 512x256; at 1536x768 the TMA kernel takes 156 against
        // 251 us).  SWB200_TMA=0|1 forces it.
        const char* env = getenv("SWB200_TMA");
        const long long tma_tiles = (long long)((g.N + BAND - 1) / BAND) * ((g.M + STAGE_TMA_TY - 1) / STAGE_TMA_TY);
        bool want = env ? env[0] != '0' : tma_tiles >= 4LL * ctx->nsm;
        bool ok = want && encode_fn() != nullptr;
        // a cap on the TMA stage kernel's persistent blocks (SWB200_STAGE_BLOCKS),
        // so that small grids also run blocks that take several tiles each
        const char* envb = getenv("SWB200_STAGE_BLOCKS");
        ctx->stage_blocks_cap = envb ? std::max(1, atoi(envb)) : 0;
        // test only: a shorter bounded wait and a chunk that is never filled,
        // to make rk_stage_tma's waits run out (SW_ERR_TIMEOUT)
        const char* envw = getenv("SWB200_TEST_WAIT_LIMIT");
        if (envw && atoi(envw) > 0) ctx->spin_limit = (uint32_t)atoi(envw);
        const char* envk = getenv("SWB200_TEST_SKIP_CHUNK");
        ctx->test_skip_chunk = envk ? atoi(envk) : -1;
        for (Fields3* f : {&ctx->S[0], &ctx->S[1], &ctx->A, &ctx->B, &ctx->Acc})
            for (void* p : {f->u, f->v, f->e}) {
                if (!ok) break;
                sw_ctx::Maps mp;
                ok = make_map(&mp.in, p, ctx->tpsz, g.P, g.R, BOXW_IN, STAGE_TMA_K) &&
                     make_map(&mp.x, p, ctx->tpsz, g.P, g.R, BOXW_X, STAGE_TMA_K);
                ctx->tmaps[p] = mp;
            }
        ctx->use_tma = ok;
        const char* envg = getenv("SWB200_GRAPHS");
        ctx->use_graphs = !(envg && envg[0] == '0');
        // strips of 1, 2 or 4 rows: the RK stage, SSP momentum and tail kernels of the native storage
        const bool native = cfg->storage == SW_STORE_NATIVE;
        ctx->tail_ty = pick_strip_ty(*cfg, g, ctx->nsm, "SWB200_TAIL_TY", native);
        ctx->stage_ty = pick_strip_ty(*cfg, g, ctx->nsm, "SWB200_STAGE_TY", native);
    }
    if (cfg->storage == SW_STORE_BF16) {
        auto* e = new Engine16<__nv_bfloat16>(); ctx->eng.reset(e); if ((rc = e->init(ctx))) return rc;
    } else if (cfg->storage == SW_STORE_F16) {
        auto* e = new Engine16<__half>(); ctx->eng.reset(e); if ((rc = e->init(ctx))) return rc;
    } else if (cfg->T == SW_FLOAT32 && cfg->Tprog == SW_FLOAT32) {
        auto* e = new Engine<float, float>(); ctx->eng.reset(e); if ((rc = e->init(ctx))) return rc;
    } else if (cfg->T == SW_FLOAT64 && cfg->Tprog == SW_FLOAT64) {
        auto* e = new Engine<double, double>(); ctx->eng.reset(e); if ((rc = e->init(ctx))) return rc;
    } else if (cfg->T == SW_FLOAT32 && cfg->Tprog == SW_FLOAT64) {
        auto* e = new Engine<float, double>(); ctx->eng.reset(e); if ((rc = e->init(ctx))) return rc;
    } else if (cfg->T == SW_FLOAT16 && cfg->Tprog == SW_FLOAT32) {
        auto* e = new Engine<jf16, float>(); ctx->eng.reset(e); if ((rc = e->init(ctx))) return rc;
    } else {
        auto* e = new Engine<jf16, jf16>(); ctx->eng.reset(e); if ((rc = e->init(ctx))) return rc;
    }
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->staging.clear();
    *out = holder.release();
    return SW_OK;
}

int sw_set_state(sw_ctx* ctx, const void* u, const void* v, const void* eta, const void* sst) {
    if (!ctx || !u || !v || !eta || !sst) return SW_ERR_ARG;
    int rc;
    if ((rc = state_copy_in(ctx, u, v, eta, sst)) || (rc = state_prepare(ctx))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return SW_OK;
}

int sw_get_state(sw_ctx* ctx, void* u, void* v, void* eta, void* sst) {
    if (!ctx || !u || !v || !eta || !sst) return SW_ERR_ARG;
    const Fields3& X = ctx->S[ctx->p];
    int rc;
    if ((rc = ctx->eng->state_to_fp32(ctx))) return rc;
    if ((rc = copy_out(ctx, u, X.u, shape_u(ctx->g)))) return rc;
    if ((rc = copy_out(ctx, v, X.v, shape_v(ctx->g)))) return rc;
    if ((rc = copy_out(ctx, eta, X.e, shape_e(ctx->g)))) return rc;
    if ((rc = copy_out(ctx, sst, ctx->sst[ctx->sp], shape_s(ctx->g)))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return SW_OK;
}

int sw_get_rhs_input(sw_ctx* ctx, void* u, void* v, void* eta) {
    if (!ctx || !u || !v || !eta) return SW_ERR_ARG;
    if (ctx->cfg.storage != SW_STORE_NATIVE)
        return fail(ctx, SW_ERR_UNSUPPORTED, "the 16-bit storage form keeps its stage values in 16 bits");
    const Fields3& X = ctx->rhs_in.u ? ctx->rhs_in : ctx->S[ctx->p];
    int rc;
    if ((rc = copy_out(ctx, u, X.u, shape_u(ctx->g)))) return rc;
    if ((rc = copy_out(ctx, v, X.v, shape_v(ctx->g)))) return rc;
    if ((rc = copy_out(ctx, eta, X.e, shape_e(ctx->g)))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return SW_OK;
}

int sw_run(sw_ctx* ctx, int64_t nsteps, sw_status* status) {
    if (!ctx || nsteps < 0) return SW_ERR_ARG;
    return run_steps(ctx, nsteps, status);
}

// Per-step CUDA-event intervals around run_steps(ctx, 1), with an optional L2
// flush between steps outside the intervals.  Shared by the two timed runs.
static int run_timed_steps(sw_ctx* ctx, int64_t nsteps, int64_t l2_flush_bytes, double* step_ms_total,
                           long long* done_out) {
    if (l2_flush_bytes > 0 && (size_t)l2_flush_bytes > ctx->flush_bytes) {
        if (ctx->flush) cudaFree(ctx->flush);
        ctx->flush = nullptr;
        ctx->flush_bytes = 0;
        CK(cudaMalloc(&ctx->flush, (size_t)l2_flush_bytes));
        ctx->flush_bytes = (size_t)l2_flush_bytes;
    }
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> steps;
    int code = SW_OK;
    long long done = 0;
    for (long long s = 0; s < nsteps; s++) {
        if (l2_flush_bytes > 0) CK(cudaMemsetAsync(ctx->flush, (int)(s & 0xff), (size_t)l2_flush_bytes, ctx->stream));
        cudaEvent_t a = ctx->evget(), b = ctx->evget();
        CK(cudaEventRecord(a, ctx->stream));
        sw_status st1;
        code = run_steps(ctx, 1, &st1);
        CK(cudaEventRecord(b, ctx->stream));
        steps.push_back({a, b});
        done += st1.steps_done;
        if (code) break;
    }
    CK(cudaStreamSynchronize(ctx->stream));
    *step_ms_total = 0;
    for (auto& pr : steps) {
        float ms = 0;
        cudaEventElapsedTime(&ms, pr.first, pr.second);
        *step_ms_total += ms;
    }
    *done_out = done;
    return code;
}

int sw_run_timed(sw_ctx* ctx, int64_t nsteps, int64_t l2_flush_bytes, double* step_ms_total, sw_status* status) {
    if (!ctx || !step_ms_total || nsteps < 0) return SW_ERR_ARG;
    ctx->evnext = 0;
    long long done = 0;
    const int code = run_timed_steps(ctx, nsteps, l2_flush_bytes, step_ms_total, &done);
    if (status) {
        status->steps_done = done;
        status->step = ctx->step;
        status->code = code;
        status->nan_step = code == SW_NAN_DETECTED ? ctx->step : -1;
    }
    return code;
}

int sw_run_profiled(sw_ctx* ctx, int64_t nsteps, int64_t l2_flush_bytes, sw_profile* prof, sw_status* status) {
    if (!ctx || !prof || nsteps < 0) return SW_ERR_ARG;
    std::memset(prof, 0, sizeof(*prof));
    ctx->prof = true;
    ctx->marks.clear();
    ctx->evnext = 0;
    long long done = 0;
    const int code = run_timed_steps(ctx, nsteps, l2_flush_bytes, &prof->step_ms_total, &done);
    ctx->prof = false;
    for (auto& m : ctx->marks) {
        float ms = 0;
        cudaEventElapsedTime(&ms, m.a, m.b);
        prof->kernel_ms[m.kind] += ms;
        prof->launches[m.kind]++;
    }
    prof->steps = done;
    if (status) {
        status->steps_done = done;
        status->step = ctx->step;
        status->code = code;
        status->nan_step = code == SW_NAN_DETECTED ? ctx->step : -1;
    }
    return code;
}

int sw_diagnostics(sw_ctx* ctx, sw_diag* out) {
    if (!ctx || !out) return SW_ERR_ARG;
    return ctx->eng->diagnostics(ctx, out);
}

int sw_time_integration(const sw_config* cfg, const sw_static* st, void* u, void* v, void* eta, void* sst,
                        sw_status* status) {
    if (!cfg || !st) return SW_ERR_ARG;
    if (!u || !v || !eta || !sst) return SW_ERR_ARG;
    sw_ctx* ctx = take_dropin(cfg);
    int rc = SW_OK;
    if (ctx && refresh_dropin(ctx, cfg, st, u, v, eta, sst) != SW_OK) {
        sw_destroy(ctx);
        ctx = nullptr;
    }
    if (!ctx) {
        if ((rc = sw_create(cfg, st, &ctx))) return rc;
        rc = sw_set_state(ctx, u, v, eta, sst);
    }
    if (!rc) {
        int rr = sw_run(ctx, cfg->nt, status);
        if (rr == SW_OK || rr == SW_NAN_DETECTED) {
            int rg = sw_get_state(ctx, u, v, eta, sst);
            rc = rg ? rg : rr;
        } else {
            rc = rr;
        }
    }
    if (rc && rc != SW_NAN_DETECTED) fprintf(stderr, "swb200: %s\n", ctx->err.c_str());
    if (rc == SW_OK || rc == SW_NAN_DETECTED) put_dropin(ctx);
    else sw_destroy(ctx);
    return rc;
}

}  // extern "C"
