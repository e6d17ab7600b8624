"""Second, independent restatement of the reference time loop in numpy.

TEST INFRASTRUCTURE ONLY.  Written directly from the Julia source with array
slicing (one numpy expression per Julia loop), so that the loop-based C++
oracle (oracle/sw_oracle.hpp) can be checked against it bit for bit.  Arrays
are stored [j][i] (x fastest); a Julia array A of size (m, n) is a numpy array
of shape (n, m) and A[i,j] is a[j-1, i-1].  numpy evaluates float32/float64
element-wise in IEEE arithmetic without FMA contraction, like Julia.

Covers T == Tprog (Float32 or Float64), all time schemes, both boundary
conditions, ArakawaHsu/Sadourny, linear/nonlinear dynamics, all drag and
diffusion options, surface relaxation/forcing and the tracer.  Cited lines are
the reference's.
"""
from __future__ import annotations

import math

import numpy as np


# ---------------------------------------------------------------- operators
def dx(u):                       # ∂x! src/gradients.jl:3-13
    return u[:, 1:] - u[:, :-1]


def dy(u):                       # ∂y! src/gradients.jl:16-26
    return u[1:, :] - u[:-1, :]


def lap(u):                      # ∇²! src/gradients.jl:29-42
    c = u[1:-1, 1:-1]
    return ((u[1:-1, :-2] - c) + (u[1:-1, 2:] - c)) + ((u[:-2, 1:-1] - c) + (u[2:, 1:-1] - c))


def Ix(u):                       # Ix! src/interpolations.jl:3-15
    h = u.dtype.type(0.5)
    return h * (u[:, 1:] + u[:, :-1])


def Iy(u):                       # Iy! src/interpolations.jl:18-30
    h = u.dtype.type(0.5)
    return h * (u[1:, :] + u[:-1, :])


def Ixy(u):                      # Ixy! src/interpolations.jl:33-45
    q = u.dtype.type(0.25)
    return q * (u[:-1, :-1] + u[:-1, 1:]) + q * (u[1:, :-1] + u[1:, 1:])


class NumpyModel:
    def __init__(self, S):
        P, G, K, F = S.parameters, S.grid, S.constants, S.forcing
        assert P.T == P.Tprog, "numpy port covers T == Tprog"
        self.P, self.G, self.K = P, G, K
        T = self.T = P.T
        self.ep = G.ep
        self.f_q, self.f_u, self.f_v = G.f_q.astype(T), G.f_u.astype(T), G.f_v.astype(T)
        self.Fx, self.Fy, self.H = F.Fx.astype(T), F.Fy.astype(T), F.H.astype(T)
        self.eta_ref, self.Feta = F.η_ref.astype(T), F.Fη.astype(T)
        N, M, nux = G.nx, G.ny, G.nux
        z = lambda m, n: np.zeros((n, m), T)
        # persistent diagnostic arrays that may be read stale (src/preallocate.jl)
        self.U, self.V = z(N + 1, M + 2), z(N + 2, M + 1)
        self.qa, self.qb, self.qc, self.qd = z(N, M), z(N + 1, M), z(N + 1, M), z(N, M)
        self.q_u, self.q_v = z(N + 1, M), z(N, M + 1)
        self.KEu, self.KEv = z(nux + 3, M + 4), z(N + 4, M + 2)
        self.um, self.vm = z(nux + 4, M + 4), z(N + 4, M + 3)
        self.du, self.dv, self.deta = z(nux + 4, M + 4), z(N + 4, M + 3), z(N + 2, M + 2)
        self.h = None
        self.t = 0
        self.step = 0

    # ------------------------------------------------------------ ghost points
    def gp_uv(self, u, v):       # src/ghost_points.jl:202-216
        T = self.T
        if self.ep:
            for a in (u, v):
                a[:, 0], a[:, 1] = self._c(a[:, -4]), self._c(a[:, -3])
                a[:, -2], a[:, -1] = self._c(a[:, 2]), self._c(a[:, 3])
        else:
            oma = T(self.K.one_minus_α)
            u[0, :], u[1, :] = oma * u[3, :], oma * u[2, :]
            u[-2, :], u[-1, :] = oma * u[-3, :], oma * u[-4, :]
            v[:, 0], v[:, 1] = oma * v[:, 3], oma * v[:, 2]
            v[:, -2], v[:, -1] = oma * v[:, -3], oma * v[:, -4]

    def gp_eta(self, e):         # src/ghost_points.jl:102-133
        if self.ep:
            e[:, 0], e[:, -1] = self._c(e[:, -2]), self._c(e[:, 1])
        else:
            e[:, 0], e[:, -1] = e[:, 1], e[:, -2]
        e[0, :], e[-1, :] = e[1, :], e[-2, :]

    def gp(self, u, v, e):       # src/ghost_points.jl:182-199
        self.gp_uv(u, v)
        self.gp_eta(e)

    def gp_sst(self, s):         # src/ghost_points.jl:136-179
        if self.ep:
            s[:, 0], s[:, -1] = self._c(s[:, -2]), self._c(s[:, 1])
        else:
            s[:, 0], s[:, -1] = s[:, 1], s[:, -2]

    def _c(self, x):             # T(Tcomm(x))
        Tc = self.P.Tcomm
        return x if Tc is self.T else x.astype(Tc).astype(self.T)

    # ------------------------------------------------------------------- rhs
    def uvfluxes(self, u, v, e):  # src/rhs.jl:307-324
        ep = self.ep
        self.h = e + self.H
        self.h_u, self.h_v = Ix(self.h), Iy(self.h)
        m, n = self.h_u.shape[1], self.h_u.shape[0]
        self.U = u[1:1 + n, 1 + ep:1 + ep + m] * self.h_u             # Uflux! :277-291
        m, n = self.h_v.shape[1], self.h_v.shape[0]
        self.V = v[1:1 + n, 1:1 + m] * self.h_v                       # Vflux! :294-304

    def advection_coriolis(self, u, v):  # src/rhs.jl:89-128
        T, ep = self.T, self.ep
        h_q = Ixy(self.h)
        dvdx, dudy = dx(v), dy(u)
        self.KEu, self.KEv = Ix(u * u), Iy(v * v)
        n, m = h_q.shape                                              # PV! src/PV_advection.jl:2-18
        q = (self.f_q + dvdx[1:1 + n, 1:1 + m] - dudy[1:1 + n, 1 + ep:1 + ep + m]) / h_q
        self.q = q
        if self.P.adv_scheme == "Sadourny":
            self.q_u, self.q_v = Iy(q), Ix(q)
        else:
            o12 = T(1 / 12)
            self.qa = o12 * (q[:-1, :-1] + q[1:, :-1] + q[1:, 1:])                 # AHα! :88-99
            qm1 = np.concatenate([q[:, -1:], q[:, :-1]], axis=1)                     # q[i-1] with q[end] at i=1
            self.qb = o12 * (q[:-1, :] + q[1:, :] + qm1[1:, :])                      # AHβ! :103-115
            qc = o12 * (q[:-1, :] + qm1[:-1, :] + q[1:, :])                          # AHγ! :119-131
            qc[:, 0] = o12 * (q[:-1, 0] + q[1:, 0] + q[:-1, -1])                    # i=1 sums in another order
            self.qc = qc
            self.qd = o12 * (q[:-1, :-1] + q[1:, :-1] + q[:-1, 1:])                 # AHδ! :135-146

    def pvadvection(self):       # src/PV_advection.jl:21-84
        ep, G = self.ep, self.G
        U, V = self.U, self.V
        nux, nuy, nvx, nvy = G.nux, G.nuy, G.nvx, G.nvy
        if self.P.adv_scheme == "Sadourny":
            V_u, U_v = Ixy(V), Ixy(U)
            self.qhv = self.q_u[:, 1 - ep:1 - ep + nux] * V_u[:, 1 - ep:1 - ep + nux]
            self.qhu = self.q_v[1:1 + nvy, :] * U_v[1:1 + nvy, :]
        else:
            a, b, c, d = self.qa, self.qb, self.qc, self.qd
            s = slice(1 - ep, 1 - ep + nux)
            self.qhv = (a[:, s] * V[1:, 2 - ep:2 - ep + nux] + b[:, s] * V[1:, 1 - ep:1 - ep + nux]
                        + c[:, s] * V[:-1, 1 - ep:1 - ep + nux] + d[:, s] * V[:-1, 2 - ep:2 - ep + nux])
            self.qhu = (a[:nvy, :] * U[1:1 + nvy, :nvx] + b[:nvy, 1:] * U[1:1 + nvy, 1:1 + nvx]
                        + c[1:1 + nvy, 1:] * U[2:2 + nvy, 1:1 + nvx] + d[1:1 + nvy, :nvx] * U[2:2 + nvy, :nvx])

    def momentum(self, e, t, linear=False):  # src/rhs.jl:162-180, 218-274
        T, ep, G, P = self.T, self.ep, self.G, self.P
        if not linear:
            n, m = G.ny + 2, G.nx + 2
            p = T(0.5) * (self.KEu[1:1 + n, ep:ep + m] + self.KEv[:n, 1:1 + m]) + T(self.K.g) * e
            dpdx, dpdy = dx(p), dy(p)
        else:
            ge = T(self.K.g) * e
            dpdx, dpdy = dx(ge), dy(ge)
        Fxt = T(math.sin(self.K.ωFx * t)) if P.seasonal_wind_x else T(1)
        Fyt = T(math.sin(self.K.ωFy * t)) if P.seasonal_wind_y else T(1)
        nux, nuy, nvx, nvy = G.nux, G.nuy, G.nvx, G.nvy
        self.du[2:2 + nuy, 2:2 + nux] = (self.qhv - dpdx[1:1 + nuy, 1 - ep:1 - ep + nux]) + Fxt * self.Fx
        self.dv[2:2 + nvy, 2:2 + nvx] = -(self.qhu + dpdy[1:1 + nvy, 1:1 + nvx]) + Fyt * self.Fy

    def rhs(self, u, v, e, t):   # src/rhs.jl:2-86
        ep = self.ep
        if self.P.dynamics == "linear":
            v_u, u_v = Ixy(v), Ixy(u)
            self.qhv = self.f_u * v_u[1:1 + self.G.nuy, 2 - ep:2 - ep + self.G.nux]   # fv! :183-198
            self.qhu = self.f_v * u_v[2:2 + self.G.nvy, 1 + ep:1 + ep + self.G.nvx]   # fu! :201-215
            self.momentum(e, t, linear=True)
            return
        self.uvfluxes(u, v, e)
        if self.P.nstep_advcor == 0:
            self.advection_coriolis(u, v)
        self.pvadvection()
        self.momentum(e, t)

    def continuity(self, u, v, e, t):  # src/continuity.jl:72-97
        if self.P.time_scheme != "RK":
            self.uvfluxes(u, v, e)
        dUdx, dVdy = dx(self.U), dy(self.V)
        N, M = self.G.nx, self.G.ny
        d = -(dUdx[1:1 + M, :] + dVdy[:, 1:1 + N])
        T = self.T
        if self.P.surface_relax:                                       # :3-24
            d = d + T(self.K.γ) * (self.eta_ref - e[1:-1, 1:-1])
        elif self.P.surface_forcing:                                   # :27-49
            d = d + T(math.sin(self.K.ωFη * t)) * self.Feta
        self.deta[1:-1, 1:-1] = d

    # ------------------------------------------------------------------ tail
    def drag(self, u, v, e):     # src/bottom_drag.jl:2-119
        T, ep, G = self.T, self.ep, self.G
        N, M = G.nx, G.ny
        kind = self.P.bottom_drag
        if kind == "quadratic":
            h = e + self.H
            h_u, h_v = Ix(h), Iy(h)
            KEu, KEv = Ix(u * u), Iy(v * v)
            # bottom_drag_quadratic! writes Diag.Bernoulli's KEu/KEv, which
            # bernoulli! reads stale when nstep_advcor > 0
            self.KEu, self.KEv = KEu, KEv
            sq = np.sqrt(KEu[1:1 + M + 2, ep:ep + N + 2] + KEv[:M + 2, 1:1 + N + 2])
            cD = T(self.K.cD)
            Bu = cD * Ix(sq) * u[1:1 + M + 2, 1 + ep:1 + ep + N + 1] / h_u
            Bv = cD * Iy(sq) * v[1:1 + M + 1, 1:1 + N + 2] / h_v
        elif kind == "linear":
            rD = T(self.K.rD)
            Bu = rD * u[1:1 + M + 2, 1 + ep:1 + ep + N + 1]
            Bv = rD * v[1:1 + M + 1, 1:1 + N + 2]
        else:
            Bu, Bv = np.zeros((M + 2, N + 1), T), np.zeros((M + 1, N + 2), T)
        return Bu, Bv

    def diffusion(self, u, v):   # src/diffusion.jl:2-218
        T, ep, G = self.T, self.ep, self.G
        N, M, nux = G.nx, G.ny, G.nux
        Lu, Lv = lap(u), lap(v)                                        # stress_tensor! :114-122
        dLudx, dLudy, dLvdx, dLvdy = dx(Lu), dy(Lu), dx(Lv), dy(Lv)
        if self.P.diffusion == "Smagorinsky":
            dudx, dvdy, dvdx, dudy = dx(u), dy(v), dx(v), dy(u)
            s = dudy[:, ep:ep + N + 3] + dvdx                             # smagorinsky_coeff! :68-111
            DS = Ixy(s * s)
            s = dudx[1:1 + M + 2, ep:ep + N + 2] + dvdy[:M + 2, 1:1 + N + 2]
            DT = s * s
            nu = T(self.K.cSmag) * np.sqrt(DS + DT)
            nu_q = Ixy(nu)
            S11 = nu[:, 1 - ep:1 - ep + nux + 1] * dLudx             # viscous_tensor_smagorinsky! :126-171
            S12 = nu_q * dLudy[:, ep:ep + N + 1]
            S21 = nu_q * dLvdx
            S22 = nu[1:1 + M, :] * dLvdy
        else:
            nuB = T(self.K.νB)                                         # viscous_tensor_constant! :175-218
            S11 = nuB * dLudx
            S12 = nuB * dLudy[:, ep:ep + N + 1]
            S21 = nuB * dLvdx
            S22 = nuB * dLvdy
        return dx(S11), dy(S12), dx(S21), dy(S22)

    def add_drag_diff(self, u, v, Bu, Bv, LLu1, LLu2, LLv1, LLv2):  # src/diffusion.jl:221-251
        T, ep, G = self.T, self.ep, self.G
        nux, nuy, nvx, nvy = G.nux, G.nuy, G.nvx, G.nvy
        dt = T(G.Δt_diff)
        u[2:2 + nuy, 2:2 + nux] += dt * (Bu[1:1 + nuy, 1 - ep:1 - ep + nux] + LLu1[1:1 + nuy, :]
                                         + LLu2[:, 1 - ep:1 - ep + nux])
        v[2:2 + nvy, 2:2 + nvx] += dt * (Bv[1:1 + nvy, 1:1 + nvx] + LLv1[1:1 + nvy, :]
                                         + LLv2[:, 1:1 + nvx])

    # ---------------------------------------------------------------- tracer
    def tracer(self, i, u, v, sst):  # src/tracer_advection.jl:1-275
        P, G, T, ep = self.P, self.G, self.T, self.ep
        if not P.tracer_advection:
            return
        if (i + G.nadvstep_half) % G.nadvstep == 0:
            self.um, self.vm = u.copy(), v.copy()
        if i % G.nadvstep != 0:
            return
        N, M = G.nx, G.ny
        u_T, um_T, v_T, vm_T = Ix(u), Ix(self.um), Iy(v), Iy(self.vm)
        xd = -T(G.half_dtadvu) * u_T[2:2 + M, 1 + ep:1 + ep + N]                  # backtraj! :96-124
        yd = -T(G.half_dtadvv) * v_T[1:1 + M, 2:2 + N]
        ui = self._interp(um_T, xd, yd, 1 + ep, 1, 2, 2)
        vi = self._interp(vm_T, xd, yd, 2, 2, 1, 1)
        xd = -T(G.dtadvu) * ui
        yd = -T(G.dtadvv) * vi
        ssti = np.zeros_like(sst)
        ssti[:, 1:1 + N] = self._interp(sst, xd, yd, 1, 1, 0, 0)                  # adv_sst! :179-206
        if P.tracer_consumption:                                                    # :262-275
            ssti[:, 1:-1] += T(self.K.jSST) * (T(self.K.SSTmin) - ssti[:, 1:-1])
        self.gp_sst(ssti)
        sst[:] = ssti

    def _interp(self, f, xx, yy, xh1, xh2, yh1, yh2):  # interp_uv!/adv_sst! with clip/wrap/bilin
        T = self.T
        nf, mf = f.shape
        n, m = xx.shape
        if not (np.all(np.isfinite(xx)) and np.all(np.isfinite(yy))):
            raise FloatingPointError("departure")
        xi = np.floor(xx).astype(np.int64)
        yi = np.floor(yy).astype(np.int64)
        I = np.arange(1, m + 1)[None, :]
        J = np.arange(1, n + 1)[:, None]
        xs = xi + I + xh1
        x0 = xx - xi.astype(T)
        if self.ep:                                                   # wrap :227-240
            k = np.where(xs < 1 + xh1, xs + mf - xh1 - xh2, np.where(xs > mf - 1, xs - mf + xh1 + xh2, xs))
        else:                                                         # clip :211-223
            k = np.where(xs < 1 + xh1, 1 + xh1, np.where(xs > mf - 1, mf - 1, xs))
            x0 = np.where(xs < 1 + xh1, T(0), np.where(xs > mf - 1, T(1), x0)).astype(T)
        ys = yi + J + yh1
        l = np.where(ys < 1 + yh1, 1 + yh1, np.where(ys > nf - 1, nf - 1, ys))
        y0 = np.where(ys < 1 + yh1, T(0), np.where(ys > nf - 1, T(1), yy - yi.astype(T))).astype(T)
        if k.min() < 1 or k.max() + 1 > mf:
            raise IndexError("departure")
        k0, l0 = k - 1, l - 1
        f00, f10 = f[l0, k0], f[l0, k0 + 1]
        f01, f11 = f[l0 + 1, k0], f[l0 + 1, k0 + 1]
        one = T(1)
        return (f00 * (one - x0) * (one - y0) + f10 * x0 * (one - y0)       # bilin :243-246
                + f01 * (one - x0) * y0 + f11 * x0 * y0)

    # ------------------------------------------------------------ time loop
    def prologue(self, u, v, e):  # src/time_integration.jl:20-31
        self.h = e + self.H
        self.advection_coriolis(u, v)
        if self.P.dynamics == "nonlinear":
            self.pvadvection()

    def time_step(self, u, v, e, sst):  # src/time_integration.jl:45-243
        P, G, K, T = self.P, self.G, self.K, self.T
        i = self.step + 1
        t = self.t
        self.gp(u, v, e)
        u0, v0, e0 = u.copy(), v.copy(), e.copy()
        u1, v1, e1 = u.copy(), v.copy(), e.copy()
        if P.time_scheme == "RK":
            a = [T(x) for x in K.RKaΔt]
            b = [T(x) for x in K.RKbΔt]
            for rki in range(1, P.RKo + 1):
                if rki > 1:
                    self.gp(u1, v1, e1)
                self.rhs(u1, v1, e1, t)
                self.continuity(u1, v1, e1, t)
                if rki < P.RKo:
                    u1 = u + b[rki - 1] * self.du
                    v1 = v + b[rki - 1] * self.dv
                    e1 = e + b[rki - 1] * self.deta
                u0 = u0 + a[rki - 1] * self.du
                v0 = v0 + a[rki - 1] * self.dv
                e0 = e0 + a[rki - 1] * self.deta
        elif P.time_scheme == "SSPRK2":
            c = T(K.Δt_Δs)
            for rki in range(1, P.RKs + 1):
                if rki > 1:
                    self.gp_eta(e1)
                self.rhs(u1, v1, e1, t)
                u1 = u1 + c * self.du
                v1 = v1 + c * self.dv
                self.gp_uv(u1, v1)
                self.continuity(u1, v1, e1, t)
                e1 = e1 + c * self.deta
            x, y = T(1 / P.RKs), T((P.RKs - 1) / P.RKs)
            u0, v0, e0 = x * u + y * u1, x * v + y * v1, x * e + y * e1
        elif P.time_scheme == "SSPRK3":
            s3 = K.SSPRK3c
            s, kn, mn = s3["s"], s3["kn"], s3["mn"]
            cn, kna, knb, cnc = (T(s3[k]) for k in ("Δt_Δn", "kna", "knb", "Δt_Δnc"))
            for rki in range(2, s + 2):
                if rki > 2:
                    self.gp_eta(e1)
                self.rhs(u1, v1, e1, t)
                if rki == kn:
                    u1 = kna * u1 + knb * u0 + cnc * self.du
                    v1 = kna * v1 + knb * v0 + cnc * self.dv
                else:
                    u1 = u1 + cn * self.du
                    v1 = v1 + cn * self.dv
                self.gp_uv(u1, v1)
                self.continuity(u1, v1, e1, t)
                if rki == kn:
                    e1 = kna * e1 + knb * e0 + cnc * self.deta
                else:
                    e1 = e1 + cn * self.deta
                if rki == mn or rki == s + 1:
                    u0, v0 = u1.copy(), v1.copy()
                    self.gp_eta(e1)
                    e0 = e1.copy()
        else:  # 4SSPRK3
            c, half = T(K.Δt_Δ), T(0.5)
            for rki in range(1, 5):
                if rki > 1:
                    self.gp(u1, v1, e1)
                self.rhs(u1, v1, e1, t)
                u0 = u1 + c * self.du
                v0 = v1 + c * self.dv
                u1 = half * (u1 + u0)
                v1 = half * (v1 + v0)
                self.gp_uv(u1, v1)
                self.continuity(u1, v1, e1, t)
                e0 = e1 + c * self.deta
                e1 = half * (e1 + e0)
                if rki == 3:
                    x, y = T(2 / 3), T(1 / 3)
                    u1, v1, e1 = x * u + y * u1, x * v + y * v1, x * e + y * e1
                elif rki == 4:
                    u0, v0, e0 = u1.copy(), v1.copy(), e1.copy()
        self.gp(u0, v0, e0)
        if P.dynamics == "nonlinear" and P.nstep_advcor > 0 and i % P.nstep_advcor == 0:
            self.uvfluxes(u0, v0, e0)
            self.advection_coriolis(u0, v0)
        if i % P.nstep_diff == 0:
            Bu, Bv = self.drag(u0, v0, e0)
            LL = self.diffusion(u0, v0)
            self.add_drag_diff(u0, v0, Bu, Bv, *LL)
            self.gp_uv(u0, v0)
        self.t = t + G.dtint
        self.tracer(i, u0, v0, sst)
        self.step = i
        nan = (i % G.nout == 0) and any(np.isnan(a).any() for a in (u, v, e, sst))
        if nan:
            return True
        u[:], v[:], e[:] = u0, v0, e0
        return False

    def run(self, Prog, nsteps):
        u, v, e, sst = (np.array(a, copy=True) for a in Prog)
        if self.step == 0:
            self.prologue(u, v, e)
        for _ in range(nsteps):
            if self.time_step(u, v, e, sst):
                break
        return u, v, e, sst
