// sw_diag.cuh -- global diagnostics of the current state, reduced in FP64.
//
// mass    = sum over T-cells of eta
// energy  = sum over T-cells of  1/2 h (KEu + KEv)  +  1/2 g eta^2, with
//           h = eta + H, KEu = (u(a)^2 + u(a+1)^2)/2, KEv = (v(b)^2 + v(b+1)^2)/2
//           (the T-point kinetic energy of src/rhs.jl:142-159 and
//           src/bottom_drag.jl:38-48, here accumulated in double)
// max_speed = max |u|, |v| over the interior faces
// nan_count = NaNs in u, v, eta (with halo) and sst (interior)
// Two passes with a fixed reduction order, so results are reproducible.
#pragma once
#include "sw_common.cuh"

namespace swb {

struct DiagPartial {
    double mass, energy;
    float max_speed;
    unsigned long long nan_count;
};

constexpr int DIAG_THREADS = 256;
constexpr int DIAG_BLOCKS = 592;   // 4 per SM on 148 SMs

template <class T, class Tp>
__global__ void __launch_bounds__(DIAG_THREADS)
diag_partial_kernel(Geom g, const Tp* u, const Tp* v, const Tp* e, const Tp* sst, SField<T> H, double gravity,
                    DiagPartial* part) {
    double mass = 0.0, energy = 0.0;
    float vmax = 0.f;
    unsigned long long nans = 0;
    const int N = g.N, M = g.M;
    // T-cells: mass, energy; u at the cell's left face, v at its bottom face
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < (long long)N * M;
         k += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(k % N), b = (int)(k / N);
        const double eta = cvt<double>(e[g.idx(a, b)]);
        const double h = eta + cvt<double>(H.at(a, b));
        const double u0 = cvt<double>(u[g.idx(a, b)]), u1 = cvt<double>(u[g.idx(a + 1, b)]);
        const double v0 = cvt<double>(v[g.idx(a, b)]), v1 = cvt<double>(v[g.idx(a, b + 1)]);
        mass += eta;
        energy += 0.5 * h * (0.5 * (u0 * u0 + u1 * u1) + 0.5 * (v0 * v0 + v1 * v1)) + 0.5 * gravity * eta * eta;
        vmax = fmaxf(vmax, fmaxf(fabsf((float)u0), fabsf((float)v0)));
        const double s = cvt<double>(sst[g.idx(a, b)]);
        nans += (unsigned long long)(s != s);
    }
    // NaNs over the full padded-halo footprint of u, v, eta
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < (long long)(N + 4) * (M + 4);
         k += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(k % (N + 4)) - 2, y = (int)(k / (N + 4)) - 2;
        const double fu = cvt<double>(u[g.idx(x, y)]), fv = cvt<double>(v[g.idx(x, y)]);
        nans += (unsigned long long)(fu != fu) + (unsigned long long)(fv != fv);
        if (x >= -1 && x <= N && y >= -1 && y <= M) {
            const double fe = cvt<double>(e[g.idx(x, y)]);
            nans += (unsigned long long)(fe != fe);
        }
    }
    // block reduction in a fixed order
    __shared__ double sm[DIAG_THREADS], se[DIAG_THREADS];
    __shared__ float sv[DIAG_THREADS];
    __shared__ unsigned long long sn[DIAG_THREADS];
    const int t = threadIdx.x;
    sm[t] = mass; se[t] = energy; sv[t] = vmax; sn[t] = nans;
    __syncthreads();
    for (int w = DIAG_THREADS / 2; w > 0; w >>= 1) {
        if (t < w) {
            sm[t] += sm[t + w];
            se[t] += se[t + w];
            sv[t] = fmaxf(sv[t], sv[t + w]);
            sn[t] += sn[t + w];
        }
        __syncthreads();
    }
    if (t == 0) part[blockIdx.x] = DiagPartial{sm[0], se[0], sv[0], sn[0]};
}

__global__ void __launch_bounds__(32) diag_final_kernel(const DiagPartial* part, int n, DiagPartial* out) {
    if (threadIdx.x != 0) return;
    DiagPartial r{0.0, 0.0, 0.f, 0ull};
    for (int i = 0; i < n; i++) {
        r.mass += part[i].mass;
        r.energy += part[i].energy;
        r.max_speed = fmaxf(r.max_speed, part[i].max_speed);
        r.nan_count += part[i].nan_count;
    }
    *out = r;
}

}  // namespace swb
