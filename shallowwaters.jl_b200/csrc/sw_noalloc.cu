// sw_noalloc.cu -- sw_diagnostics_noalloc: the FP64 diagnostics reduction of
// sw_diagnostics for callers that cannot allocate device memory.
//
// Who needs it.  A host program that hands its device memory to a pool
// allocator of its own (CUDA.jl's or PyTorch's caching allocator, a fixed
// arena in an embedded application) often cannot, or must not, call
// cudaMalloc/cudaFree at the point where it wants a mass/energy/CFL check:
// the pool may already hold all free memory, and cudaFree synchronises the
// whole device, which stalls a running time loop.  Such a caller keeps the
// model state in its own device buffers and wants the diagnostics of those
// buffers without the library allocating anything.  sw_diagnostics needs a
// context (whose creation allocates) and allocates its reduction scratch on
// first use; this entry point takes the fields as plain device pointers and
// uses a fixed scratch array compiled into the library instead.
//
// Scratch.  NOALLOC_MAX_PARTIALS per-block partial sums plus one result slot
// live in a file-scope __device__ array (about 64 KiB), which every GPU that
// loads the library holds until the process exits.  One block reduces
// NOALLOC_CELLS_PER_BLOCK T-cells, so domains of up to
// NOALLOC_MAX_PARTIALS * NOALLOC_CELLS_PER_BLOCK = 16,777,216 cells (4096 x
// 4096) fit; larger ones are rejected with SW_ERR_ARG.  Every slot a call
// reads was written earlier in the same call, so nothing has to start at zero
// and the previous call's contents are never seen.  All calls on one device
// share the array: calls whose kernels overlap on the GPU (two streams, two
// host threads) race and must be serialised by the caller.
//
// The first call on a device looks up the array's device address with
// cudaGetSymbolAddress (with that device current), which also loads the
// library's device code there if nothing has yet; make that first call before
// any stream capture.  The address is remembered per device and per CUDA
// context, so after cudaDeviceReset the next call looks it up again.  A CUDA
// error that is already pending when the call starts (from the caller's own
// work) is reported as such, returned as SW_ERR_CUDA and left pending.  Nothing else is allocated: no cudaMalloc, no cudaFree,
// no pinned buffers (the 32-byte result is copied into the caller's sw_diag
// through an ordinary stream copy).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>
#include <vector>

#include "swb200.h"
#include "sw_common.cuh"

namespace {

using namespace swb;

struct NaPartial {
    double mass, energy;
    float max_speed;
    unsigned long long nan_count;
};

constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_CELLS_PER_THREAD = 32;
constexpr int NOALLOC_CELLS_PER_BLOCK = NOALLOC_THREADS * NOALLOC_CELLS_PER_THREAD;   // 8192
constexpr int NOALLOC_MAX_PARTIALS = 2048;
constexpr long long NOALLOC_MAX_CELLS = (long long)NOALLOC_MAX_PARTIALS * NOALLOC_CELLS_PER_BLOCK;
constexpr int NOALLOC_MAX_DEVICES = 64;

// the scratch: partials [0, NOALLOC_MAX_PARTIALS) and the result slot after them
static __device__ __align__(256) NaPartial g_noalloc_scratch[NOALLOC_MAX_PARTIALS + 1];

// device address of g_noalloc_scratch per device and CUDA context (host code
// may not use the array's name as an address: that is a host-side stand-in).
// A context destroyed and created again (cudaDeviceReset) may load the
// module at another address, so the lookup is keyed by the context's id.
struct ScratchAddr {
    int device;
    unsigned long long context;
    NaPartial* addr;
};
std::vector<ScratchAddr> g_scratch_addr;
std::mutex g_scratch_mu;

// Index of a point in the host-ABI arrays (x fastest, with halo; the shapes
// of include/swb200.h), from the physical indices used by the kernels:
// u at face F, row b; v at column a, face G; eta, H, sst at T-cell (a, b).
struct FlatGeom {
    int N, M, ep;
    int wu;   // u row length nux + 4
    __device__ long long u(int F, int b) const { return (long long)(b + 2) * wu + (F + 1 + ep); }
    __device__ long long v(int a, int G) const { return (long long)(G + 1) * (N + 4) + (a + 2); }
    __device__ long long e(int a, int b) const { return (long long)(b + 1) * (N + 2) + (a + 1); }
    __device__ long long s(int a, int b) const { return (long long)b * (N + 2) + (a + 1); }
};

// The quantities of diag_partial_kernel (sw_diag.cuh) over the host-ABI
// layout: mass, energy, max |u|,|v| and NaNs; one partial per block.
template <class T, class Tp>
__global__ void __launch_bounds__(NOALLOC_THREADS)
noalloc_partial_kernel(FlatGeom f, const Tp* __restrict__ u, const Tp* __restrict__ v, const Tp* __restrict__ e,
                       const Tp* __restrict__ sst, const T* __restrict__ H, double gravity, NaPartial* part) {
    double mass = 0.0, energy = 0.0;
    float vmax = 0.f;
    unsigned long long nans = 0;
    const int N = f.N, M = f.M;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < (long long)N * M; k += stride) {
        const int a = (int)(k % N), b = (int)(k / N);
        const double eta = cvt<double>(e[f.e(a, b)]);
        const double h = eta + cvt<double>(H[f.e(a, b)]);
        const double u0 = cvt<double>(u[f.u(a, b)]), u1 = cvt<double>(u[f.u(a + 1, b)]);
        const double v0 = cvt<double>(v[f.v(a, b)]), v1 = cvt<double>(v[f.v(a, b + 1)]);
        mass += eta;
        energy += 0.5 * h * (0.5 * (u0 * u0 + u1 * u1) + 0.5 * (v0 * v0 + v1 * v1)) + 0.5 * gravity * eta * eta;
        vmax = fmaxf(vmax, fmaxf(fabsf((float)u0), fabsf((float)v0)));
        const double s = cvt<double>(sst[f.s(a, b)]);
        nans += (unsigned long long)(s != s);
    }
    // NaNs over the whole arrays of u, v and eta, halos included
    const long long nu = (long long)f.wu * (M + 4), nv = (long long)(N + 4) * (M + 3), ne = (long long)(N + 2) * (M + 2);
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nu + nv + ne; k += stride) {
        const double x = k < nu ? cvt<double>(u[k]) : k < nu + nv ? cvt<double>(v[k - nu]) : cvt<double>(e[k - nu - nv]);
        nans += (unsigned long long)(x != x);
    }
    __shared__ double sm[NOALLOC_THREADS], se[NOALLOC_THREADS];
    __shared__ float sv[NOALLOC_THREADS];
    __shared__ unsigned long long sn[NOALLOC_THREADS];
    const int t = threadIdx.x;
    sm[t] = mass; se[t] = energy; sv[t] = vmax; sn[t] = nans;
    __syncthreads();
    for (int w = NOALLOC_THREADS / 2; w > 0; w >>= 1) {
        if (t < w) {
            sm[t] += sm[t + w];
            se[t] += se[t + w];
            sv[t] = fmaxf(sv[t], sv[t + w]);
            sn[t] += sn[t + w];
        }
        __syncthreads();
    }
    if (t == 0) part[blockIdx.x] = NaPartial{sm[0], se[0], sv[0], sn[0]};
}

// partials [0, n) -> part[NOALLOC_MAX_PARTIALS], in a fixed order
__global__ void __launch_bounds__(32) noalloc_final_kernel(NaPartial* part, int n) {
    if (threadIdx.x != 0) return;
    NaPartial r{0.0, 0.0, 0.f, 0ull};
    for (int i = 0; i < n; i++) {
        r.mass += part[i].mass;
        r.energy += part[i].energy;
        r.max_speed = fmaxf(r.max_speed, part[i].max_speed);
        r.nan_count += part[i].nan_count;
    }
    part[NOALLOC_MAX_PARTIALS] = r;
}

int reject(const char* why) {
    fprintf(stderr, "swb200: sw_diagnostics_noalloc: %s\n", why);
    return SW_ERR_ARG;
}

// p must be device (or managed) memory of the current device, aligned to its element size
bool device_ptr_ok(const void* p, size_t elem, int dev) {
    if (!p || (reinterpret_cast<uintptr_t>(p) % elem) != 0) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    if (at.type == cudaMemoryTypeManaged) return true;
    return at.type == cudaMemoryTypeDevice && at.device == dev;
}

template <class T, class Tp>
int run(const sw_config* cfg, const void* u, const void* v, const void* eta, const void* sst, const void* H,
        cudaStream_t stream, NaPartial* scratch, sw_diag* out) {
    FlatGeom f;
    f.N = cfg->nx; f.M = cfg->ny; f.ep = cfg->periodic ? 1 : 0;
    f.wu = (f.ep ? f.N : f.N - 1) + 4;
    const long long cells = (long long)f.N * f.M;
    const int nblocks = (int)((cells + NOALLOC_CELLS_PER_BLOCK - 1) / NOALLOC_CELLS_PER_BLOCK);
    noalloc_partial_kernel<T, Tp><<<nblocks, NOALLOC_THREADS, 0, stream>>>(
        f, (const Tp*)u, (const Tp*)v, (const Tp*)eta, (const Tp*)sst, (const T*)H, cfg->g, scratch);
    noalloc_final_kernel<<<1, 32, 0, stream>>>(scratch, nblocks);
    cudaError_t e = cudaGetLastError();
    NaPartial r;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&r, scratch + NOALLOC_MAX_PARTIALS, sizeof(r), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        fprintf(stderr, "swb200: sw_diagnostics_noalloc: %s\n", cudaGetErrorString(e));
        return SW_ERR_CUDA;
    }
    out->mass = r.mass;
    out->energy = r.energy;
    out->max_speed = r.max_speed;
    out->nan_count = (int64_t)r.nan_count;
    return SW_OK;
}

}  // namespace

extern "C" int sw_diagnostics_noalloc(const sw_config* cfg, const void* u, const void* v, const void* eta,
                                      const void* sst, const void* H, void* stream, sw_diag* out) {
    if (!cfg || !out) return reject("cfg and out must not be NULL");
    if (cfg->abi_version != SWB200_ABI_VERSION) return reject("abi_version mismatch");
    if (cfg->nx < 4 || cfg->ny < 4) return reject("nx and ny must be >= 4");
    if ((long long)cfg->nx * cfg->ny > NOALLOC_MAX_CELLS) {
        char msg[160];
        snprintf(msg, sizeof msg, "nx*ny = %lld cells exceeds the fixed scratch limit of %lld cells",
                 (long long)cfg->nx * cfg->ny, NOALLOC_MAX_CELLS);
        return reject(msg);
    }
    const bool f32 = cfg->T == SW_FLOAT32 && cfg->Tprog == SW_FLOAT32;
    const bool f64 = cfg->T == SW_FLOAT64 && cfg->Tprog == SW_FLOAT64;
    const bool mix = cfg->T == SW_FLOAT32 && cfg->Tprog == SW_FLOAT64;
    if (!f32 && !f64 && !mix) return reject("(T, Tprog) must be (Float32, Float32), (Float64, Float64) or (Float32, Float64)");

    int ndev = 0, dev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        (void)cudaGetLastError();
        return SW_ERR_NODEVICE;
    }
    // an error left by the caller's own earlier work is reported as such and
    // left pending for the caller, not taken for one of this call's launches
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
        fprintf(stderr, "swb200: sw_diagnostics_noalloc: a CUDA error was pending before the call: %s\n",
                cudaGetErrorString(pending));
        return SW_ERR_CUDA;
    }
    if (cudaGetDevice(&dev) != cudaSuccess) return SW_ERR_CUDA;
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return reject("device index beyond the supported range");

    const size_t tp = f64 || mix ? 8 : 4, ts = f64 ? 8 : 4;
    if (!device_ptr_ok(u, tp, dev) || !device_ptr_ok(v, tp, dev) || !device_ptr_ok(eta, tp, dev) ||
        !device_ptr_ok(sst, tp, dev) || !device_ptr_ok(H, ts, dev))
        return reject("u, v, eta, sst and H must be aligned device memory of the current device");

    NaPartial* scratch = nullptr;
    {
        const unsigned long long cid = current_context_id();
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        for (const ScratchAddr& a : g_scratch_addr)
            if (cid && a.device == dev && a.context == cid) scratch = a.addr;
        if (!scratch) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                fprintf(stderr, "swb200: sw_diagnostics_noalloc: cudaGetSymbolAddress: %s\n", cudaGetErrorString(e));
                return SW_ERR_CUDA;
            }
            scratch = static_cast<NaPartial*>(p);
            if (cid) g_scratch_addr.push_back({dev, cid, scratch});
        }
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (f32) return run<float, float>(cfg, u, v, eta, sst, H, s, scratch, out);
    if (f64) return run<double, double>(cfg, u, v, eta, sst, H, s, scratch, out);
    return run<float, double>(cfg, u, v, eta, sst, H, s, scratch, out);
}
