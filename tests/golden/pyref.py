"""Pure-Python restatement of one SFINCS time step on a small regular grid.

A second, independent restatement (plain loops, FP64) of the reference's step
for the plain configuration, used only to pin the C++ oracle on tiny grids:
  * time step control       sfincs_lib.f90:390-415
  * boundary levels         sfincs_boundaries.f90:682-758, 800-876 (one bnd point)
  * boundary fluxes         sfincs_boundaries.f90:941-1113 (regular bathymetry)
  * momentum                sfincs_momentum.f90:157-752 (no advection/viscosity/
                            Coriolis/wind; friction2d on)
  * continuity              sfincs_continuity.f90:112-255 (regular)
Cells are addressed by (n, m) on the full grid; missing neighbours follow the
reference's rules (u neighbours of absent cells -> the face itself, absent
faces -> the zero dummy).
"""
from __future__ import annotations

import math

import numpy as np


# the exponents are real*4 literals in the reference (sfincs_momentum.f90:92, 616)
E53 = float(np.float32(5.0) / np.float32(3.0))
E13 = float(np.float32(1.0) / np.float32(3.0))


class PyRef:
    def __init__(self, msk, zb, dx, dy, zini, huthresh, alpha, gn2_sea, gn2_land, rgh_lev, t_bnd, zs_bnd,
                 dtmax=60.0, hmin_cfl=0.1, btfilter=60.0, btrelax=3600.0, uvlim=10.0, huvmin=0.0, g=9.81):
        # constants and inputs carry real*4 values in the reference (even where arithmetic is promoted)
        f = np.float32
        g = float(f(g))
        huthresh, alpha = float(f(huthresh)), float(f(alpha))
        gn2_sea, gn2_land = float(f(gn2_sea)), float(f(gn2_land))
        self.dxinv, self.dyinv = float(f(1.0) / f(dx)), float(f(1.0) / f(dy))
        self.nmax = len(msk)
        self.mmax = len(msk[0])
        self.msk = [list(r) for r in msk]
        self.zb = [list(map(float, r)) for r in zb]
        self.dx, self.dy, self.g = float(dx), float(dy), g
        self.huthresh, self.alpha, self.uvlim, self.huvmin = huthresh, alpha, uvlim, huvmin
        self.t_bnd, self.zs_bnd = list(t_bnd), list(zs_bnd)
        self.btfilter, self.btrelax = btfilter, btrelax
        dxymin = min(dx, dy)
        f = np.float32
        self.dtmax = float(min(f(dtmax), f(alpha) * f(dxymin) / np.sqrt(f(9.81) * f(hmin_cfl))))
        self.zs = [[max(self.zb[n][m], zini) for m in range(self.mmax)] for n in range(self.nmax)]
        # faces: u[(n,m)] joins (n,m)-(n,m+1); v[(n,m)] joins (n,m)-(n+1,m)
        self.kcu, self.kcv = {}, {}
        for n in range(self.nmax):
            for m in range(self.mmax):
                if self.act(n, m) and self.act(n, m + 1):
                    self.kcu[(n, m)] = self.kcuv(self.msk[n][m], self.msk[n][m + 1])
                if self.act(n, m) and self.act(n + 1, m):
                    self.kcv[(n, m)] = self.kcuv(self.msk[n][m], self.msk[n + 1][m])
        self.qu = {k: 0.0 for k in self.kcu}
        self.qv = {k: 0.0 for k in self.kcv}
        self.uu = {k: 0.0 for k in self.kcu}
        self.vv = {k: 0.0 for k in self.kcv}
        self.kfu = {k: 0 for k in self.kcu}
        self.kfv = {k: 0 for k in self.kcv}
        self.gn2u, self.gn2v = {}, {}
        for d, store, kc in ((0, self.gn2u, self.kcu), (1, self.gn2v, self.kcv)):
            for (n, m) in kc:
                n2, m2 = (n, m + 1) if d == 0 else (n + 1, m)
                zbuv = 0.5 * (self.zb[n][m] + self.zb[n2][m2])
                store[(n, m)] = gn2_land if zbuv > rgh_lev else gn2_sea
        self.uvmean = {}
        self.t = 0.0
        self.min_dt = 1.0e-6
        self.dt = 0.0

    def act(self, n, m):
        return 0 <= n < self.nmax and 0 <= m < self.mmax and self.msk[n][m] > 0

    @staticmethod
    def kcuv(a, b):
        if a > 1 and b > 1:
            return 0
        if a * b == 0:
            return 0
        if {a, b} == {1, 2} or {a, b} == {1, 3} or {a, b} == {1, 5}:
            return 2
        if {a, b} == {1, 6}:
            return 6
        return 1

    def _q(self, d, n, m):
        return (self.qu if d == 0 else self.qv).get((n, m), 0.0)

    def _uv(self, d, n, m):
        return (self.uu if d == 0 else self.vv).get((n, m), 0.0)

    def zst(self):
        """update_boundary_points for one point: real*4 interpolation with tb = real(t)
        (sfincs_boundaries.f90:700-732)."""
        f = np.float32
        t, tb, zb = self.t, self.t_bnd, self.zs_bnd
        if tb[0] > t - 1e-3:
            return float(f(zb[0]))
        if tb[-1] < t + 1e-3:
            return float(f(zb[-1]))
        for i in range(1, len(tb)):
            if tb[i] > t + 1e-6:
                fac = (f(t) - f(tb[i - 1])) / max(f(tb[i]) - f(tb[i - 1]), f(1e-6))
                return float(f(zb[i - 1]) + (f(zb[i]) - f(zb[i - 1])) * fac)

    def step(self):
        g, ht = self.g, self.huthresh
        # dt and min_dt are real*4 in the reference (sfincs_lib.f90:59, sfincs_data.f90:9)
        self.dt = dt = float(np.float32(np.float32(self.alpha) * np.float32(self.min_dt)))
        self.t += dt
        # ---- boundary fluxes at kcuv == 2 faces
        zsb = float(np.float32(self.zst()))
        factime = float(min(np.float32(dt) / np.float32(self.btfilter), np.float32(1.0)))
        facrel = float(np.float32(1.0) - min(np.float32(dt) / np.float32(self.btrelax), np.float32(1.0)))
        for d, kc in ((0, self.kcu), (1, self.kcv)):
            for (n, m), k in kc.items():
                if k != 2:
                    continue
                n2, m2 = (n, m + 1) if d == 0 else (n + 1, m)
                if self.msk[n][m] == 1:
                    (nb, mb), (ni, mi), sgn = (n2, m2), (n, m), -1.0
                else:
                    (nb, mb), (ni, mi), sgn = (n, m), (n2, m2), 1.0
                # real*4 locals in the reference's boundary routine (sfincs_boundaries.f90:933-937)
                f = np.float32
                zsnmb = max(f(zsb), f(self.zb[nb][mb]))
                zs0nmb = zsnmb
                zsnmi = f(self.zs[ni][mi])
                zbuv = f(0.5) * (f(self.zb[n][m]) + f(self.zb[n2][m2]))
                h = max(f(0.5) * (zsnmb + zsnmi) - zbuv, f(ht))
                um = f(self.uvmean.get((d, n, m), 0.0))
                if h < f(ht) + f(1e-6):
                    q = uv = f(0.0)
                    um = f(0.0)
                else:
                    sq = np.sqrt(f(g) / h)
                    ui = sq * (zsnmb - zs0nmb)
                    ub = f(sgn) * (f(2.0) * ui - sq * (zsnmi - zs0nmb))
                    q = ub * h + um
                    if zsnmi - f(self.zb[ni][mi]) <= f(ht):
                        q = max(q, f(0.0)) if sgn > 0 else min(q, f(0.0))
                    if zsnmb - f(self.zb[nb][mb]) < f(ht):
                        q = min(q, f(0.0)) if sgn > 0 else max(q, f(0.0))
                    uv = max(min(q / h, f(4.0)), f(-4.0))
                q, uv = float(q), float(uv)
                (self.qu if d == 0 else self.qv)[(n, m)] = q
                (self.uu if d == 0 else self.vv)[(n, m)] = uv
                fq, fr = np.float32(factime), np.float32(facrel)
                self.uvmean[(d, n, m)] = float(fq * np.float32(q) + fr * (np.float32(1.0) - fq) * um)
                self.zs[nb][mb] = max(zsb, self.zb[nb][mb])  # zs(nmb) = zsb (sfincs_boundaries.f90:1097)
        # ---- momentum (old q/uv from before this loop)
        q0u, q0v, u0u, u0v = dict(self.qu), dict(self.qv), dict(self.uu), dict(self.vv)

        def Q(d, n, m):
            return (q0u if d == 0 else q0v).get((n, m), 0.0)

        def U(d, n, m):
            return (u0u if d == 0 else u0v).get((n, m), 0.0)

        min_dt = self.dtmax
        newq = {}
        for d, kc in ((0, self.kcu), (1, self.kcv)):
            for (n, m), k in kc.items():
                if k not in (1, 6):
                    continue
                n2, m2 = (n, m + 1) if d == 0 else (n + 1, m)
                zsu = max(self.zs[n][m], self.zs[n2][m2])
                # zbuvmx is a real*4 array (sfincs_domain.f90:1708)
                zbmx = float(np.float32(np.float32(max(self.zb[n][m], self.zb[n2][m2])) + np.float32(ht)))
                kf = (self.kfu if d == 0 else self.kfv)
                if not zsu > zbmx:
                    newq[(d, n, m)] = (0.0, 0.0)
                    kf[(n, m)] = 0
                    continue
                if d == 0:
                    dxi = self.dxinv
                    qx = Q(0, n, m)
                    vu = (U(1, n - 1, m) + U(1, n - 1, m + 1) + U(1, n, m) + U(1, n, m + 1)) / 4
                else:
                    dxi = self.dyinv
                    qx = Q(1, n, m)
                    vu = (U(0, n, m - 1) + U(0, n + 1, m - 1) + U(0, n, m) + U(0, n + 1, m)) / 4
                hu = max(zsu - zbmx, ht)
                gn2 = (self.gn2u if d == 0 else self.gn2v)[(n, m)]
                dzdx = (self.zs[n2][m2] - self.zs[n][m]) * dxi
                frc = -g * hu * dzdx
                if kf[(n, m)] == 0:
                    qfr = math.sqrt(abs(dzdx) / (max(gn2, 1e-5) / 10)) * hu ** E53
                else:
                    qfr = math.sqrt(qx ** 2 + (hu * vu) ** 2)
                hu73 = hu ** 2 * hu ** E13
                q = (qx + frc * dt) / (1.0 + gn2 * dt * qfr / hu73)
                if self.zs[n][m] < self.zb[n][m]:
                    q = min(q, 0.0)
                if self.zs[n2][m2] < self.zb[n2][m2]:
                    q = max(q, 0.0)
                q = min(max(q, -hu * self.uvlim), hu * self.uvlim)
                uv = q / max(hu, self.huvmin)
                newq[(d, n, m)] = (q, uv)
                kf[(n, m)] = 1
                min_dt = min(min_dt, 1.0 / (max(math.sqrt(g * hu), abs(uv)) * dxi))
        for (d, n, m), (q, uv) in newq.items():
            (self.qu if d == 0 else self.qv)[(n, m)] = q
            (self.uu if d == 0 else self.vv)[(n, m)] = uv
        self.min_dt = float(np.float32(min_dt))
        # ---- continuity (regular)
        for n in range(self.nmax):
            for m in range(self.mmax):
                if self.msk[n][m] != 1:
                    continue
                div = (self._q(0, n, m - 1) - self._q(0, n, m)) * self.dxinv + \
                      (self._q(1, n - 1, m) - self._q(1, n, m)) * self.dyinv
                self.zs[n][m] += div * dt
