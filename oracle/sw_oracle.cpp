// sw_oracle.cpp -- C entry points of the CPU oracle (test infrastructure only).
//
// Built as oracle/liboracle.so by oracle/Makefile.  Only tests/, the smoke
// check and the benchmark's CPU-baseline leg load it; the shipped library
// never does.  The functions mirror the library's C ABI (include/swb200.h)
// so the two can be driven with identical inputs.
#include <cstdio>
#include <exception>
#include <map>
#include <memory>
#include <string>

#include "sw_oracle.hpp"
#if defined(_OPENMP)
#include <omp.h>
#endif

using namespace swo;

namespace {

struct Base {
    std::string err;
    virtual ~Base() = default;
    virtual void set_state(const void*, const void*, const void*, const void*) = 0;
    virtual void get_state(void*, void*, void*, void*) const = 0;
    virtual int64_t run(int64_t n, int64_t* nan_step) = 0;
    virtual int64_t step() const = 0;
    virtual bool field(const std::string& name, void* out, int64_t* m, int64_t* n, int* elsize) = 0;
};

template <class T, class Tp>
struct Impl : Base {
    Model<T, Tp> M;
    Impl(const sw_config& c, const sw_static& s) : M(c, s) {}
    void set_state(const void* u, const void* v, const void* e, const void* s) override {
        M.set_state(u, v, e, s);
    }
    void get_state(void* u, void* v, void* e, void* s) const override { M.get_state(u, v, e, s); }
    int64_t run(int64_t n, int64_t* nan_step) override { return M.run(n, nan_step); }
    int64_t step() const override { return M.step; }

    template <class X>
    bool put(const Arr<X>& a, void* out, int64_t* m, int64_t* n, int* elsize) {
        *m = a.m; *n = a.n; *elsize = (int)sizeof(X);
        if (out) std::memcpy(out, a.d.data(), a.size() * sizeof(X));
        return true;
    }
    bool field(const std::string& nm, void* out, int64_t* m, int64_t* n, int* es) override {
        auto& A = M;
#define F(x) if (nm == #x) return put(A.x, out, m, n, es);
        F(u) F(v) F(eta) F(sst) F(u0) F(v0) F(eta0) F(u1) F(v1) F(eta1) F(du) F(dv) F(deta)
        F(h) F(h_u) F(U) F(h_v) F(V) F(dUdx) F(dVdy) F(h_q) F(q) F(qhu) F(qhv)
        F(dudx) F(dudy) F(dvdx) F(dvdy) F(u2) F(v2) F(KEu) F(KEv) F(p) F(dpdx) F(dpdy)
        F(sqrtKE) F(sqrtKE_u) F(sqrtKE_v) F(Bu) F(Bv) F(qa) F(qb) F(qc) F(qd)
        F(Lu) F(Lv) F(dLudx) F(dLudy) F(dLvdx) F(dLvdy) F(DT) F(DS) F(nuSmag) F(DS_q)
        F(nuSmag_q) F(S12) F(S21) F(S11) F(S22) F(LLu1) F(LLu2) F(LLv1) F(LLv2)
        F(xd) F(yd) F(um) F(vm) F(u_T) F(um_T) F(v_T) F(vm_T) F(uinterp) F(vinterp) F(ssti)
#undef F
        return false;
    }
};

template <class T>
Base* make_tp(const sw_config& c, const sw_static& s) {
    switch (c.Tprog) {
        case SW_FLOAT16: return new Impl<T, f16>(c, s);
        case SW_FLOAT32: return new Impl<T, float>(c, s);
        case SW_FLOAT64: return new Impl<T, double>(c, s);
    }
    throw std::invalid_argument("Tprog");
}

Base* make(const sw_config& c, const sw_static& s) {
    switch (c.T) {
        case SW_FLOAT16: return make_tp<f16>(c, s);
        case SW_FLOAT32: return make_tp<float>(c, s);
        case SW_FLOAT64: return make_tp<double>(c, s);
    }
    throw std::invalid_argument("T");
}

thread_local std::string g_err;

}  // namespace

extern "C" {

int oracle_create(const sw_config* cfg, const sw_static* st, void** out) {
    try {
        if (!cfg || !st || !out) return SW_ERR_ARG;
        if (cfg->abi_version != SWB200_ABI_VERSION) return SW_ERR_ARG;
        *out = make(*cfg, *st);
        return SW_OK;
    } catch (std::exception& e) {
        g_err = e.what();
        return SW_ERR_ARG;
    }
}

int oracle_set_state(void* h, const void* u, const void* v, const void* eta, const void* sst) {
    auto* b = static_cast<Base*>(h);
    try {
        b->set_state(u, v, eta, sst);
        return SW_OK;
    } catch (std::exception& e) {
        b->err = e.what();
        return SW_ERR_ARG;
    }
}

int oracle_get_state(void* h, void* u, void* v, void* eta, void* sst) {
    static_cast<Base*>(h)->get_state(u, v, eta, sst);
    return SW_OK;
}

int oracle_run(void* h, int64_t nsteps, sw_status* st) {
    auto* b = static_cast<Base*>(h);
    int64_t nan_step = -1, done = 0;
    int code = SW_OK;
    try {
        done = b->run(nsteps, &nan_step);
        if (nan_step >= 0) code = SW_NAN_DETECTED;
    } catch (BoundsError& e) {
        b->err = e.what();
        code = std::string(e.what()) == "departure" ? SW_ERR_DEPARTURE : SW_ERR_ARG;
    } catch (std::exception& e) {
        b->err = e.what();
        code = SW_ERR_ARG;
    }
    if (st) {
        st->steps_done = done;
        st->step = b->step();
        st->nan_step = nan_step;
        st->code = code;
    }
    return code;
}

// Copies a named diagnostic array (reference names, ASCII) into out; with
// out == NULL only reports its shape.  Returns 0 if the name is unknown.
int oracle_field(void* h, const char* name, void* out, int64_t* m, int64_t* n, int* elsize) {
    return static_cast<Base*>(h)->field(name, out, m, n, elsize) ? 1 : 0;
}

const char* oracle_last_error(void* h) {
    return h ? static_cast<Base*>(h)->err.c_str() : g_err.c_str();
}

void oracle_destroy(void* h) { delete static_cast<Base*>(h); }

// Threads used by the OpenMP loops (the reference itself is single-threaded).
int oracle_set_threads(int n) {
#if defined(_OPENMP)
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int oracle_time_integration(const sw_config* cfg, const sw_static* st, void* u, void* v, void* eta,
                            void* sst, sw_status* status) {
    void* h = nullptr;
    int rc = oracle_create(cfg, st, &h);
    if (rc) return rc;
    rc = oracle_set_state(h, u, v, eta, sst);
    if (!rc) {
        rc = oracle_run(h, cfg->nt, status);
        oracle_get_state(h, u, v, eta, sst);
    }
    oracle_destroy(h);
    return rc;
}


// Directional derivative of J = sum over the interior of (eta after nsteps -
// eta_obs)^2 along (du, dv, deta, dFx), by running the restated time loop
// with the forward-mode Dual number type (value and derivative carried
// together; sqrt'(0) = 0).  This is the check of the library's adjoint
// (sw_adjoint_run): <gradient, direction> must equal *dJ.  cfg must be
// Float64 (T = Tprog); static fields and the state are double arrays in the
// swb200.h shapes, eta_obs is nx x ny.  du, dv, deta, dFx may be NULL (zero).
int oracle_jvp(const sw_config* cfg, const sw_static* st, const double* u, const double* v, const double* eta,
               const double* du, const double* dv, const double* deta, const double* dFx,
               const double* eta_obs, int64_t nsteps, double* J, double* dJ) {
    try {
        if (!cfg || !st || !u || !v || !eta || !eta_obs || !J || !dJ) return SW_ERR_ARG;
        if (cfg->T != SW_FLOAT64 || cfg->Tprog != SW_FLOAT64) return SW_ERR_ARG;
        sw_static none{};
        Model<Dual, Dual> M(*cfg, none);
        auto fill = [](Arr<Dual>& a, const void* p, const double* d) {
            if (!p) return;
            const double* x = static_cast<const double*>(p);
            for (size_t k = 0; k < a.size(); k++) a[k] = Dual(x[k], d ? d[k] : 0.0);
        };
        fill(M.f_q, st->f_q, nullptr); fill(M.f_u, st->f_u, nullptr); fill(M.f_v, st->f_v, nullptr);
        fill(M.Fx, st->Fx, dFx); fill(M.Fy, st->Fy, nullptr); fill(M.H, st->H, nullptr);
        fill(M.eta_ref, st->eta_ref, nullptr); fill(M.Feta, st->Feta, nullptr);
        fill(M.u, u, du); fill(M.v, v, dv); fill(M.eta, eta, deta);
        M.step = 0;
        M.t = 0;
        M.prologue();
        int64_t nan_step = -1;
        M.run(nsteps, &nan_step);
        if (nan_step >= 0) return SW_NAN_DETECTED;
        Dual s(0.0, 0.0);
        for (int j = 1; j <= M.ny; j++)
            for (int i = 1; i <= M.nx; i++) {
                const Dual d = M.eta(i + 1, j + 1) - Dual(eta_obs[(size_t)(i - 1) + (size_t)(j - 1) * M.nx], 0.0);
                s = s + d * d;
            }
        *J = s.v;
        *dJ = s.d;
        return SW_OK;
    } catch (std::exception& e) {
        g_err = e.what();
        return SW_ERR_ARG;
    }
}

}  // extern "C"
