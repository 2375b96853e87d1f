"""The oracle's infiltration models with state (curve number with and without
recovery, Green-Ampt, Horton; sfincs_infiltration.f90:609-1039) against a
second, independent restatement in numpy float32 written from the same
Fortran.  Each step the restatement takes the oracle's start-of-step water
levels, the step's dt and the uniform rain rate, and must give the oracle's
net rain (prcp - qinfmap) of every cell."""
import numpy as np
import pytest

from sfincs_b200 import synth

F = np.float32


def _model(tmp_path, kind, rain_until=900.0):
    m = synth.plain_regular(nmax=10, mmax=12, dx=300.0, tstop=3600.0, seed=4, nbumps=3)
    m.msk[:, 0] = 1  # closed basin
    m.bnd = m.bzs = None
    m.params["zsini"] = -4.0
    m.prcp = np.array([[0.0, 40.0], [rain_until, 40.0], [rain_until + 1.0, 0.0], [7200.0, 0.0]])
    rng = np.random.default_rng(17)
    shp = m.msk.shape
    if kind == "cna":
        m.cell_fields["scsfile"] = rng.uniform(0.05, 2.0, shp)  # S in inches
    elif kind == "cnb":
        m.cell_fields["smaxfile"] = rng.uniform(0.005, 0.05, shp)
        m.cell_fields["sefffile"] = rng.uniform(0.002, 0.03, shp)
        m.cell_fields["ksfile"] = rng.uniform(10.0, 20000.0, shp)
    elif kind == "gai":
        m.cell_fields["psifile"] = rng.uniform(50.0, 300.0, shp)
        m.cell_fields["sigmafile"] = rng.uniform(0.1, 0.4, shp)
        m.cell_fields["ksfile"] = rng.uniform(5.0, 20000.0, shp)
    else:
        m.cell_fields["fcfile"] = rng.uniform(5.0, 20.0, shp)
        m.cell_fields["f0file"] = rng.uniform(50.0, 150.0, shp)
        m.cell_fields["kdfile"] = rng.uniform(1.0, 5.0, shp)
    return m.write(str(tmp_path)), m


class Restated:
    """update_infiltration_map for one model, every cell, float32 throughout."""

    def __init__(self, kind, m):
        self.kind = kind
        c = {k: m.compact(v).astype(F) for k, v in m.cell_fields.items()}
        n = next(iter(c.values())).size
        self.zb = m.compact(m.zb).astype(F)
        z = lambda: np.zeros(n, F)  # noqa: E731
        self.q = z()
        self.cumprcp, self.cuminf = z(), z()
        if kind == "cna":
            self.S = c["scsfile"] * F(0.0254)
        elif kind == "cnb":
            self.smax, self.se = c["smaxfile"], c["sefffile"].copy()
            self.kr = np.sqrt(c["ksfile"] / F(25.4)) / F(75.0)
            self.p1, self.f1, self.s1, self.t1 = z(), z(), z(), z()
            self.rain = np.zeros(n, bool)
        elif kind == "gai":
            ks = c["ksfile"]
            self.kr = np.sqrt(ks / F(25.4)) / F(75.0)
            self.lu = F(4.0) * np.sqrt(F(25.4)) * np.sqrt(ks) / F(1000.0)
            self.head = c["psifile"] / F(1000.0)
            self.ks = ks / F(1000.0) / F(3600.0)
            self.smax, self.sig = c["sigmafile"], c["sigmafile"].copy()
            self.F, self.t1 = z(), z()
        else:
            self.fc, self.f0, self.kd = c["fcfile"], c["f0file"], c["kdfile"]
            self.t1 = z()

    def step(self, p, dt, zs):
        p, dt = F(p), F(dt)
        sf = F(0.2)
        if self.kind == "cna":
            self.cumprcp = self.cumprcp + p * dt
            cp = self.cumprcp
            a = cp - sf * self.S
            run = a * a / (cp + (F(1.0) - sf) * self.S)
            q = np.where(cp > sf * self.S, ((cp - run) - self.cuminf) / dt, p).astype(F)
            self.cuminf = self.cuminf + q * dt
        elif self.kind == "cnb":
            self.cumprcp = self.cumprcp + p * dt
            if p > 0:
                new = ~self.rain
                self.p1[new], self.f1[new], self.s1[new] = 0, 0, self.se[new]
                self.rain[:] = True
                self.p1 = self.p1 + p * dt
                a = self.p1 - sf * self.s1
                i = self.p1 - a * a / (self.p1 + (F(1.0) - sf) * self.s1)
                runoff = self.p1 > sf * self.s1
                q = np.where(runoff, (i - self.f1) / dt, p).astype(F)
                self.f1 = np.where(runoff, i, self.p1).astype(F)
                self.se = np.maximum(self.se - q * dt, F(0.0))
                q = np.maximum(q, F(0.0))
            else:
                self.t1[self.rain] = 0
                self.rain[:] = False
                q = np.zeros_like(self.se)
                self.t1 = self.t1 + dt / F(3600.0)
                rec = self.t1 > F(0.06) / self.kr
                se2 = np.minimum(self.se + self.kr * self.smax * dt / F(3600.0), self.smax)
                self.se = np.where(rec, se2, self.se).astype(F)
            self.cuminf = self.cuminf + q * dt
        elif self.kind == "gai":
            hs = self.head[-1] * self.sig[-1]
            if p > 0:
                with np.errstate(divide="ignore", invalid="ignore"):
                    g = self.ks * (F(1.0) + hs / self.F)
                g = np.maximum(np.fmin(g, p), F(0.0))
                q = np.where(p < self.ks, p, g).astype(F)
                self.sig = np.maximum(self.sig - q * dt / self.lu, F(0.0))
                self.F = self.F + q * dt
                self.t1[:] = 0
                self.q = q
            else:
                q = self.q
                self.t1 = self.t1 + dt / F(3600.0)
                rec = self.t1 > F(0.06) / self.kr
                sig2 = np.minimum(self.sig + self.kr * self.smax * dt / F(3600.0), self.smax)
                f2 = np.maximum(self.F - self.kr * self.smax * dt / F(3600.0) * self.lu, F(0.0))
                self.sig = np.where(rec, sig2, self.sig).astype(F)
                self.F = np.where(rec, f2, self.F).astype(F)
        else:
            hh = (zs - self.zb.astype(np.float64)).astype(F)
            on = (hh > 0) | (p > 0)
            t1 = np.where(self.t1 > 0, F(0.0), self.t1 - dt).astype(F)
            e = np.exp((self.kd * t1 / F(3600.0)).astype(np.float64)).astype(F)
            low = e < F(0.01)
            q = np.where(low, self.fc / F(3600.0) / F(1000.0),
                         (self.fc + (self.f0 - self.fc) * e) / F(3600.0) / F(1000.0)).astype(F)
            t1 = np.where(low, t1 + dt, t1).astype(F)
            avail = np.where(hh > 0, p * dt + hh, p * dt).astype(F)
            want = q * dt
            q = np.where(want > avail, q * avail / want, q).astype(F)
            self.t1 = np.where(on, t1, self.t1 + dt / F(10.0)).astype(F)
            q = np.where(on, q, F(0.0)).astype(F)
        return q


@pytest.mark.parametrize("kind", ["cna", "cnb", "gai", "hor"])
def test_infiltration_models_match_restatement(tmp_path, kind):
    from oracle.oracle import Oracle

    d, m = _model(tmp_path, kind, rain_until=600.0 if kind in ("cnb", "gai") else 1800.0)
    o = Oracle(d, "ref")
    r = Restated(kind, m)
    active = 0
    for k in range(120):
        zs = o.get("zs")
        o.update(-1000.0, 1)
        s = o.scalars()
        p = F(o.get("prcp")[0])  # the step's uniform rain rate (m/s)
        q = r.step(p, s["dt"], zs)
        net = o.get("netprcp")
        expect = (p - q).astype(np.float64)
        assert np.allclose(net, expect, rtol=1e-6, atol=1e-12), (kind, k, np.abs(net - expect).max())
        active += int(np.any(q != 0))
    assert active > 10
