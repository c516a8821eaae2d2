"""Independent pure-Python transliteration of MaterialPointSolver.jl's OS/MUSL
uGIMP step, written directly from the Julia source (not from oracle/), used to
cross-check the C++ oracle on tiny cases.  Loops are plain Python: keep the
inputs small.  Arrays follow the reference's column-major `n x k` shapes as
numpy (n, k) arrays; ids stored in arrays are 1-based like the reference's.
"""
import math

import numpy as np


def sign(x):
    x = float(x)
    return float((x > 0) - (x < 0))


def jl_mod(x, y):                      # Julia mod for floats
    r = math.fmod(x, y)
    if r == 0.0:
        return math.copysign(r, y)
    if (r > 0) != (y > 0):
        return r + y
    return r


def fld(a, b):                          # Julia fld = div(a, b, RoundDown)
    return float(round((a - jl_mod(a, b)) / b))   # Python round: ties to even, like Julia


def cld(a, b):                          # Julia cld = div(a, b, RoundUp)
    return float(round((a - jl_mod(a, -b)) / b))


def ugimp(d, h, lp):                   # mpbasisfunc.jl:40-53
    N = dN = 0.0
    a = abs(d)
    if a < 0.5 * lp:
        N = 1.0 - ((4.0 * d * d + lp * lp) / (4.0 * h * lp))
        dN = -((8.0 * d) / (4.0 * h * lp))
    elif 0.5 * lp <= a < h - 0.5 * lp:
        N = 1.0 - (a / h)
        dN = sign(d) * (-1.0 / h)
    elif h - 0.5 * lp <= a < h + 0.5 * lp:
        N = ((h + 0.5 * lp - a) * (h + 0.5 * lp - a)) / (2.0 * h * lp)
        dN = -sign(d) * ((h + 0.5 * lp - a) / (h * lp))
    return N, dN


def icld(a, b):
    return -((-a) // b)


P2ND_3D = [
    (-1, -1, -1, 0), (-1, 0, -1, 0), (0, 0, -1, 0), (0, -1, -1, 0), (0, -2, -1, 0), (-1, -2, -1, 0),
    (-2, -2, -1, 0), (-2, -1, -1, 0), (-2, 0, -1, 0), (-2, 1, -1, 0), (-1, 1, -1, 0), (0, 1, -1, 0),
    (1, 1, -1, 0), (1, 0, -1, 0), (1, -1, -1, 0), (1, -2, -1, 0), (-1, -1, -1, 1), (-1, 0, -1, 1),
    (0, 0, -1, 1), (0, -1, -1, 1), (0, -2, -1, 1), (-1, -2, -1, 1), (-2, -2, -1, 1), (-2, -1, -1, 1),
    (-2, 0, -1, 1), (-2, 1, -1, 1), (-1, 1, -1, 1), (0, 1, -1, 1), (1, 1, -1, 1), (1, 0, -1, 1),
    (1, -1, -1, 1), (1, -2, -1, 1), (-1, -1, 0, 1), (-1, 0, 0, 1), (0, 0, 0, 1), (0, -1, 0, 1),
    (0, -2, 0, 1), (-1, -2, 0, 1), (-2, -2, 0, 1), (-2, -1, 0, 1), (-2, 0, 0, 1), (-2, 1, 0, 1),
    (-1, 1, 0, 1), (0, 1, 0, 1), (1, 1, 0, 1), (1, 0, 0, 1), (1, -1, 0, 1), (1, -2, 0, 1),
    (-1, -1, 0, 2), (-1, 0, 0, 2), (0, 0, 0, 2), (0, -1, 0, 2), (0, -2, 0, 2), (-1, -2, 0, 2),
    (-2, -2, 0, 2), (-2, -1, 0, 2), (-2, 0, 0, 2), (-2, 1, 0, 2), (-1, 1, 0, 2), (0, 1, 0, 2),
    (1, 1, 0, 2), (1, 0, 0, 2), (1, -1, 0, 2), (1, -2, 0, 2)]     # grid.jl:289-301


class PyModel:
    """FP64 state for the transliteration, copied from the host structs."""

    def __init__(self, args, grid, mp, attr, bc):
        self.D = grid.dim
        D = self.D
        self.g = grid
        self.args = args
        self.gxi = np.array(grid.xi, np.float64)
        ni, npart, NIC = grid.ni, mp.np, mp.NIC
        self.ni, self.np, self.NIC = ni, npart, NIC
        self.lp = (mp.dx, mp.dy, mp.dz if D == 3 else 1.0)
        self.h = (grid.dx, grid.dy, grid.dz if D == 3 else 1.0)
        f = lambda a: np.array(a, np.float64)
        self.xi, self.vs, self.sig, self.eps, self.F = f(mp.xi), f(mp.vs), f(mp.sig), f(mp.eps), f(mp.F)
        self.Omega, self.Omega0, self.rho, self.rho0 = f(mp.Omega), f(mp.Omega0), f(mp.rho), f(mp.rho0)
        self.epsq, self.epsk, self.epsv, self.sigm = f(mp.epsq), f(mp.epsk), f(mp.epsv), f(mp.sigm)
        nv = 4 if D == 2 else 6
        self.deps = np.zeros((npart, nv))
        self.sij = np.zeros((npart, nv))
        self.dF = np.zeros((npart, D * D))
        self.ps = np.zeros((npart, D))
        self.ms = np.zeros(npart)
        self.p2c = np.zeros(npart, np.int64)
        self.p2n = np.zeros((npart, NIC), np.int64)
        self.Nij = np.zeros((npart, NIC))
        self.dN = np.zeros((D, npart, NIC))
        self.nid = np.array(attr.nid, np.int64)
        self.attr = attr
        self.bcidx = [np.array(getattr(bc, f"v{c}_s_idx"), np.int64) for c in "xyz"[:D]]
        self.bcval = [np.array(getattr(bc, f"v{c}_s_val"), np.float64) for c in "xyz"[:D]]
        self.gms = np.zeros(ni)
        self.gps, self.gfs, self.gvs, self.gvsT, self.gas, self.gdus = (np.zeros((ni, D)) for _ in range(6))

    # resetmpstatus_OS_CPU!, utils_OS.jl:235-277 / 363-415
    def resetmp(self):
        g, D = self.g, self.D
        for ix in range(self.np):
            self.ms[ix] = self.Omega[ix] * self.rho[ix]
            self.ps[ix] = self.ms[ix] * self.vs[ix]
            x = self.xi[ix]
            if D == 2:
                p2c = int(math.trunc(cld(x[1] - g.y1, g.dy) + fld(x[0] - g.x1, g.dx) * g.ncy))
            else:
                p2c = int(math.trunc(cld(x[1] - g.y1, g.dy) + fld(x[2] - g.z1, g.dz) * g.ncy * g.ncx +
                                     fld(x[0] - g.x1, g.dx) * g.ncy))
            self.p2c[ix] = p2c
            self.Nij[ix] = 0.0
            self.dN[:, ix] = 0.0
            viy = 1
            for iy in range(16 if D == 2 else 64):
                if D == 2:
                    nny = g.nny
                    tab = [(a, b) for a in (-nny, 0, nny, 2 * nny) for b in (2, 1, 0, -1)]
                    col = icld(p2c, g.ncy)
                    row = p2c - (col - 1) * g.ncy
                    ltn = col * nny - row
                    p2n = ltn + tab[iy][0] + tab[iy][1]
                else:
                    layer = icld(p2c, g.ncx * g.ncy)
                    l_idx = icld(p2c - (layer - 1) * g.ncx * g.ncy, g.ncy)
                    l_idy = (p2c - (layer - 1) * g.ncx * g.ncy) - (l_idx - 1) * g.ncy
                    t = P2ND_3D[iy]
                    p2n = (layer + t[0]) * g.nnx * g.nny + (l_idx + t[1]) * g.nny + (l_idy + t[2]) + t[3]
                d = [x[k] - self.gxi[p2n - 1, k] for k in range(D)]
                if all(abs(d[k]) < self.h[k] + 0.5 * self.lp[k] for k in range(D)):
                    w = [ugimp(d[k], self.h[k], self.lp[k]) for k in range(D)]
                    s = viy - 1
                    if D == 2:
                        self.Nij[ix, s] = w[0][0] * w[1][0]
                        self.dN[0, ix, s] = w[0][1] * w[1][0]
                        self.dN[1, ix, s] = w[1][1] * w[0][0]
                    else:
                        self.Nij[ix, s] = w[0][0] * w[1][0] * w[2][0]
                        self.dN[0, ix, s] = w[0][1] * w[1][0] * w[2][0]
                        self.dN[1, ix, s] = w[1][1] * w[0][0] * w[2][0]
                        self.dN[2, ix, s] = w[2][1] * w[0][0] * w[1][0]
                    self.p2n[ix, s] = p2n
                    viy += 1
                if viy > self.NIC:
                    break

    def step(self, dt, Ti):
        a, D = self.args, self.D
        G = a.gravity / a.Te * Ti if Ti < a.Te else a.gravity
        self.gms[:] = 0; self.gps[:] = 0; self.gfs[:] = 0
        self.resetmp()
        sg = self.sig
        # P2G_OS!, utils_OS.jl:424-496
        for ix in range(self.np):
            for s in range(self.NIC):
                Ni = self.Nij[ix, s]
                if Ni == 0.0:
                    continue
                n = self.p2n[ix, s] - 1
                vol = self.Omega[ix]
                NiM = self.ms[ix] * Ni
                self.gms[n] += NiM
                self.gps[n] += Ni * self.ps[ix]
                dx, dy = self.dN[0, ix, s], self.dN[1, ix, s]
                if D == 2:
                    self.gfs[n, 0] += -vol * (dx * sg[ix, 0] + dy * sg[ix, 3])
                    self.gfs[n, 1] += -vol * (dy * sg[ix, 1] + dx * sg[ix, 3]) + NiM * G
                else:
                    dz = self.dN[2, ix, s]
                    self.gfs[n, 0] += -vol * (dx * sg[ix, 0] + dy * sg[ix, 3] + dz * sg[ix, 5])
                    self.gfs[n, 1] += -vol * (dy * sg[ix, 1] + dx * sg[ix, 3] + dz * sg[ix, 4])
                    self.gfs[n, 2] += -vol * (dz * sg[ix, 2] + dx * sg[ix, 5] + dy * sg[ix, 4]) + NiM * G
        # eps(T2), T2 the reference's float type (utils_OS.jl:515, 555)
        eps = float(np.finfo(np.float32 if getattr(a, "precision", "FP64") == "FP32" else np.float64).eps)
        if getattr(a, "scheme", "MUSL") == "USL":
            self._usl_a(dt, eps)
        else:
            self._musl_a(dt, eps)
        # G2P_OS!, utils_OS.jl:1025-1153
        self._g2p(dt, Ti)

    def _usl_a(self, dt, eps):
        """solvegrid_a_USL_OS! + doublemapping1_a_USL_OS!, OS_USL.jl:147-320."""
        a, D = self.args, self.D
        for i in range(self.ni):
            md = 0.0 if self.gms[i] < eps else 1.0 / self.gms[i]
            for d in range(D):
                if self.bcidx[d][i] != 0:
                    self.gps[i, d] = self.bcval[d][i]
            self.gvs[i] = self.gps[i] * md
            damp = -a.zeta_s * math.sqrt(float(np.sum(self.gfs[i] ** 2)))
            Fs = [self.gfs[i, d] + damp * sign(self.gvs[i, d]) for d in range(D)]
            for d in range(D):
                self.gvs[i, d] += Fs[d] * dt * md
                self.gas[i, d] = Fs[d] * md
            for d in range(D):
                if self.bcidx[d][i] != 0:
                    self.gvs[i, d] = self.bcval[d][i]
                    self.gas[i, d] = self.bcval[d][i]
            self.gdus[i] = self.gvs[i] * dt
        for ix in range(self.np):
            tp = np.zeros(D); tv = np.zeros(D)
            for s in range(self.NIC):
                Ni = self.Nij[ix, s]
                if Ni == 0.0:
                    continue
                n = self.p2n[ix, s] - 1
                tp += Ni * self.gvs[n]
                tv += Ni * self.gas[n]
            self.xi[ix] += tp * dt
            self.vs[ix] = a.FLIP * self.vs[ix] + a.PIC * tp + tv * dt
            self.ps[ix] = self.ms[ix] * self.vs[ix]

    def _musl_a(self, dt, eps):
        a, D = self.args, self.D
        # solvegrid_a_OS!, utils_OS.jl:547-640
        for i in range(self.ni):
            md = 0.0 if self.gms[i] < eps else 1.0 / self.gms[i]
            for d in range(D):
                if self.bcidx[d][i] != 0:
                    self.gps[i, d] = self.bcval[d][i]
            self.gvs[i] = self.gps[i] * md
            damp = -a.zeta_s * math.sqrt(float(np.sum(self.gfs[i] ** 2)))
            Fs = [self.gfs[i, d] + damp * sign(self.gvs[i, d]) for d in range(D)]
            for d in range(D):
                self.gvsT[i, d] = self.gvs[i, d] + Fs[d] * dt * md
                self.gas[i, d] = Fs[d] * md
            for d in range(D):
                if self.bcidx[d][i] != 0:
                    self.gvsT[i, d] = self.bcval[d][i]
                    self.gas[i, d] = self.bcval[d][i]
            self.gps[i] = 0.0
        # doublemapping1_a_OS!, utils_OS.jl:745-788 / 856-908
        for ix in range(self.np):
            tv = np.zeros(D); tp = np.zeros(D); tT = np.zeros(D)
            for s in range(self.NIC):
                Ni = self.Nij[ix, s]
                if Ni == 0.0:
                    continue
                n = self.p2n[ix, s] - 1
                tp += Ni * self.gvsT[n]
                tv += Ni * self.gas[n]
                tT += Ni * self.gvs[n]
            self.xi[ix] += tp * dt
            self.vs[ix] = a.FLIP * self.vs[ix] + a.PIC * tT + tv * dt
            self.ps[ix] = self.ms[ix] * self.vs[ix]
        # doublemapping2_OS!
        for ix in range(self.np):
            for s in range(self.NIC):
                Ni = self.Nij[ix, s]
                if Ni != 0.0:
                    self.gps[self.p2n[ix, s] - 1] += self.ps[ix] * Ni
        # doublemapping3_OS!
        for i in range(self.ni):
            md = 0.0 if self.gms[i] < eps else 1.0 / self.gms[i]
            self.gvs[i] = self.gps[i] * md
            for d in range(D):
                if self.bcidx[d][i] != 0:
                    self.gvs[i, d] = self.bcval[d][i]
            self.gdus[i] = self.gvs[i] * dt

    def _g2p(self, dt, Ti):
        a, D = self.args, self.D
        for ix in range(self.np):
            dF = np.zeros((D, D))
            for s in range(self.NIC):
                if self.Nij[ix, s] == 0.0:
                    continue
                n = self.p2n[ix, s] - 1
                for r in range(D):
                    for c in range(D):
                        dF[r, c] += self.gdus[n, r] * self.dN[c, ix, s]
            self.dF[ix] = dF.ravel()
            e = dF / dt
            if D == 2:
                exy = 0.5 * (dF[0, 1] + dF[1, 0]) / dt
                self.epsv[ix] = math.sqrt(e[0, 0] ** 2 + e[1, 1] ** 2 + 2.0 * exy * exy)
                de = [dF[0, 0], dF[1, 1], self.deps[ix, 2], dF[0, 1] + dF[1, 0]]
                self.deps[ix, 0], self.deps[ix, 1], self.deps[ix, 3] = de[0], de[1], de[3]
                self.eps[ix, 0] += de[0]; self.eps[ix, 1] += de[1]; self.eps[ix, 3] += de[3]
                f = self.F[ix].copy()
                self.F[ix] = [(dF[0, 0] + 1) * f[0] + dF[0, 1] * f[2], (dF[0, 0] + 1) * f[1] + dF[0, 1] * f[3],
                              (dF[1, 1] + 1) * f[2] + dF[1, 0] * f[0], (dF[1, 1] + 1) * f[3] + dF[1, 0] * f[1]]
                Fn = self.F[ix]
                J = Fn[0] * Fn[3] - Fn[1] * Fn[2]
            else:
                exy = 0.5 * (dF[0, 1] + dF[1, 0]) / dt
                eyz = 0.5 * (dF[1, 2] + dF[2, 1]) / dt
                exz = 0.5 * (dF[0, 2] + dF[2, 0]) / dt
                self.epsv[ix] = math.sqrt(e[0, 0] ** 2 + e[1, 1] ** 2 + e[2, 2] ** 2 +
                                          2.0 * (exy * exy + eyz * eyz + exz * exz))
                de = [dF[0, 0], dF[1, 1], dF[2, 2], dF[0, 1] + dF[1, 0], dF[1, 2] + dF[2, 1], dF[0, 2] + dF[2, 0]]
                self.deps[ix] = de
                self.eps[ix] += de
                f = self.F[ix].reshape(3, 3).copy()
                self.F[ix] = ((np.eye(3) + dF) @ f).ravel()
                g9 = self.F[ix]
                J = (g9[0] * g9[4] * g9[8] + g9[1] * g9[5] * g9[6] + g9[2] * g9[3] * g9[7] -
                     g9[6] * g9[4] * g9[2] - g9[7] * g9[5] * g9[0] - g9[8] * g9[3] * g9[1])
            self.Omega[ix] = J * self.Omega0[ix]
            self.rho[ix] = self.rho0[ix] / J
        # liE! then dpP! / mcP! (OS_MUSL.jl:82-96)
        for ix in range(self.np):
            mat = self.nid[ix] - 1
            K, Gm = float(self.attr.Ks[mat]), float(self.attr.Gs[mat])
            s = self.sig[ix]
            dFv = self.dF[ix]
            if D == 2:
                w = 0.5 * (dFv[1] - dFv[2])
                s1, s2, s4 = s[0], s[1], s[3]
                s[0] += w * s4 * 2.0
                s[1] += -w * s4 * 2.0
                s[3] += w * (s2 - s1)
            else:
                wxy, wyz, wxz = 0.5 * (dFv[3] - dFv[1]), 0.5 * (dFv[7] - dFv[5]), 0.5 * (dFv[6] - dFv[2])
                s1, s2, s3, s4, s5, s6 = s
                s[0] += 2.0 * (s4 * wxy + s6 * wxz)
                s[1] += -2.0 * (s4 * wxy - s5 * wyz)
                s[2] += -2.0 * (s6 * wxz + s5 * wyz)
                s[3] += wxy * (s2 - s1) + wxz * s5 + wyz * s6
                s[4] += wyz * (s3 - s2) - wxz * s4 - wxy * s6
                s[5] += wxz * (s3 - s1) + wxy * s5 - wyz * s4
            de = self.deps[ix]
            Dt, Dd = K + 1.333333 * Gm, K - 0.666667 * Gm
            s[0] += Dt * de[0] + Dd * de[1] + Dd * de[2]
            s[1] += Dd * de[0] + Dt * de[1] + Dd * de[2]
            s[2] += Dd * de[0] + Dd * de[1] + Dt * de[2]
            for k in range(3, len(s)):
                s[k] += Gm * de[k]
            sm = (s[0] + s[1] + s[2]) * 0.333333
            sij = s.copy(); sij[:3] -= sm
            if Ti >= a.Te and a.constitutive == "druckerprager":
                sm, sij = self._dp(ix, s, sm, sij, mat, K, Gm)
            elif Ti >= a.Te and a.constitutive == "mohrcoulomb" and D == 2:
                sm, sij = self._mc2d(ix, s, mat, K, Gm)
            self.sigm[ix] = sm
            self.sij[ix] = sij

    # dpP!, druckerprager.jl:22-155
    def _dp(self, ix, s, sm, sij, mat, K, Gm):
        at = self.attr
        c, phi, psi, st = float(at.c[mat]), float(at.phi[mat]), float(at.psi[mat]), float(at.sigt[mat])
        tt = 0.5 * (sij[0] ** 2 + sij[1] ** 2 + sij[2] ** 2) + sum(sij[k] ** 2 for k in range(3, len(sij)))
        tau = math.sqrt(tt)
        kphi = (6.0 * c * math.cos(phi)) / (1.732051 * (3.0 + math.sin(phi)))
        qphi = (6.0 * math.sin(phi)) / (1.732051 * (3.0 + math.sin(phi)))
        qpsi = (6.0 * math.sin(psi)) / (1.732051 * (3.0 + math.sin(psi)))
        st = min(st, kphi / qphi)
        ab = math.sqrt(1.0 + qphi * qphi) - qphi
        tb = kphi - qphi * st
        fs = tau + qphi * sm - kphi
        ft = sm - st
        BF = (tau - tb) - (ab * (sm - st))
        if (sm < st and fs > 0.0) or (sm >= st and BF > 0.0):
            dl = fs / (Gm + K * qphi * qpsi)
            t1 = sm - K * qpsi * dl
            t2 = (kphi - qphi * t1) / tau
            s[:3] = sij[:3] * t2 + t1
            s[3:] = sij[3:] * t2
            self.epsq[ix] += dl * math.sqrt(0.333333 + 0.222222 * qpsi * qpsi)
            self.epsk[ix] += dl * qpsi
        if sm >= st and BF <= 0.0:
            dl = ft / K
            s[:3] = sij[:3] + st
            self.epsq[ix] += dl * 0.333333 * 1.414214
            self.epsk[ix] += dl
        sm = (s[0] + s[1] + s[2]) * 0.333333
        sij = s.copy(); sij[:3] -= sm
        return sm, sij

    # mcP! 2D, mohrcoulomb.jl:22-86
    def _mc2d(self, ix, s, mat, K, Gm):
        at = self.attr
        c = max(float(at.c[mat]) + float(at.Hp[mat]) * self.epsq[ix], float(at.cr[mat]))
        phi = float(at.phi[mat])
        ds = s[0] - s[1]
        tau = math.sqrt(0.25 * ds ** 2 + s[3] ** 2)
        sg = 0.5 * (s[0] + s[1])
        f = tau + sg * math.sin(phi) - c * math.cos(phi)
        sn = s.copy()
        dsigB = c / math.tan(phi)
        if sg <= dsigB and f > 0.0:
            beta = abs(c * math.cos(phi) - sg * math.sin(phi)) / tau
            dsigA = 0.5 * beta * ds
            sn[0], sn[1], sn[3] = sg + dsigA, sg - dsigA, beta * s[3]
        if sg > dsigB and f > 0.0:
            sn[0], sn[1], sn[3] = dsigB, dsigB, 0.0
        d = sn - s
        s[:] = sn
        Dt, Dd = K + 1.333333 * Gm, K - 0.666667 * Gm
        base = 1.0 / ((Dd - Dt) * (2.0 * Dd + Dt))
        exx = -(Dd * d[0] + Dt * d[0] - Dd * d[1] - Dd * d[2]) * base
        eyy = -(-Dd * d[0] + Dd * d[1] + Dt * d[1] - Dd * d[2]) * base
        ezz = -(-Dd * d[0] - Dd * d[1] + Dd * d[2] + Dt * d[2]) * base
        exy = d[3] / Gm
        self.epsk[ix] = exx + eyy + ezz
        self.epsq[ix] += math.sqrt(0.666667 * (exx * exx + eyy * eyy + ezz * ezz + exy * exy * 2.0))
        sm = (s[0] + s[1] + s[2]) * 0.333333
        sij = s.copy(); sij[:3] -= sm
        return sm, sij

    def run(self, dt, Ti0, nsteps):
        Ti = Ti0
        for _ in range(nsteps):
            self.step(dt, Ti)
            Ti += dt
        return Ti


class PyModelTS(PyModel):
    """Two-phase MUSL step (procedure!(…, Val(:TS), Val(:MUSL)), TS_MUSL.jl:24-53,
    utils_TS.jl), transliterated with the same repairs as the C++ oracle:
    ρs0 / ρw0 for the missing ρs_init / ρw_init (utils_TS.jl:849-850, 953-954),
    ΔFs for Δfs (:893-895), and the one-phase support-filtered uGIMP stencil
    instead of the first NIC candidates (:216-227, 266-283)."""

    def __init__(self, args, grid, mp, attr, bc):
        super().__init__(args, grid, mp, attr, bc)
        D, ni, npart = self.D, self.ni, self.np
        f = lambda a: np.array(a, np.float64)
        self.n, self.rhow, self.rhow0, self.sigw = f(mp.n), f(mp.rho_w), f(mp.rho_w0), f(mp.sigw)
        self.vw, self.epsw = f(mp.vw), f(mp.epsw)
        self.pw = np.zeros((npart, D))
        self.mw = np.zeros(npart)
        self.mi = np.zeros(npart)
        self.depsw = np.zeros_like(self.epsw)
        nm = len(attr.Es)
        self.Kw = np.broadcast_to(np.array(attr.Kw, np.float64), (nm,))
        self.kp = np.broadcast_to(np.array(attr.k, np.float64), (nm,))
        self.wbcidx, self.wbcval = [], []
        for c in "xyz"[:D]:
            idx = np.array(getattr(bc, f"v{c}_w_idx"), np.int64)
            ok = len(idx) == ni
            self.wbcidx.append(idx if ok else np.zeros(ni, np.int64))
            self.wbcval.append(np.array(getattr(bc, f"v{c}_w_val"), np.float64) if ok else np.zeros(ni))
        self.gmi, self.gmw = np.zeros(ni), np.zeros(ni)
        self.gpw, self.gfw, self.gfd, self.gvw, self.gvwT, self.gaw, self.gduw = (
            np.zeros((ni, D)) for _ in range(7))

    def step(self, dt, Ti):
        a, D = self.args, self.D
        G = a.gravity / a.Te * Ti if Ti < a.Te else a.gravity
        for arr in (self.gms, self.gps, self.gfs, self.gmi, self.gmw, self.gpw, self.gfw, self.gfd):
            arr[:] = 0.0
        # resetmpstatus_TS! (weights: the one-phase stencil)
        self.resetmp()
        for ix in range(self.np):
            n, vol = self.n[ix], self.Omega[ix]
            self.ms[ix] = vol * self.rho[ix]
            self.mw[ix] = vol * self.rhow[ix]
            self.mi[ix] = vol * ((1.0 - n) * self.rho[ix] + n * self.rhow[ix])
            self.ps[ix] = self.ms[ix] * self.vs[ix] * (1.0 - n)
            self.pw[ix] = self.mw[ix] * self.vw[ix] * n
        # P2G_TS!, utils_TS.jl:295-393
        for ix in range(self.np):
            n, vol, sw, s = self.n[ix], self.Omega[ix], self.sigw[ix], self.sig[ix]
            tdg = (n * self.mw[ix] * G) / self.kp[self.nid[ix] - 1]
            for q in range(self.NIC):
                Ni = self.Nij[ix, q]
                if Ni == 0.0:
                    continue
                nd = self.p2n[ix, q] - 1
                dN = [self.dN[k, ix, q] for k in range(D)]
                self.gms[nd] += Ni * self.ms[ix] * (1.0 - n)
                self.gmi[nd] += Ni * self.mw[ix] * n
                self.gmw[nd] += Ni * self.mw[ix]
                self.gps[nd] += Ni * self.ps[ix]
                self.gpw[nd] += Ni * self.pw[ix]
                for d in range(D):
                    self.gfw[nd, d] += -vol * (dN[d] * sw) + (Ni * self.mw[ix] * G if d == D - 1 else 0.0)
                if D == 2:
                    self.gfs[nd, 0] += -vol * (dN[0] * (s[0] + sw) + dN[1] * s[3])
                    self.gfs[nd, 1] += -vol * (dN[1] * (s[1] + sw) + dN[0] * s[3]) + Ni * self.mi[ix] * G
                else:
                    self.gfs[nd, 0] += -vol * (dN[0] * (s[0] + sw) + dN[1] * s[3] + dN[2] * s[5])
                    self.gfs[nd, 1] += -vol * (dN[1] * (s[1] + sw) + dN[0] * s[3] + dN[2] * s[4])
                    self.gfs[nd, 2] += (-vol * (dN[2] * (s[2] + sw) + dN[0] * s[5] + dN[1] * s[4]) +
                                        Ni * self.mi[ix] * G)
                self.gfd[nd] += Ni * tdg * (self.vw[ix] - self.vs[ix])
        # solvegrid_TS!, utils_TS.jl:404-532
        for i in range(self.ni):
            msd = 0.0 if self.gms[i] == 0.0 else 1.0 / self.gms[i]
            mwd = 0.0 if self.gmw[i] == 0.0 else 1.0 / self.gmw[i]
            self.gvs[i] = self.gps[i] * msd
            self.gvw[i] = self.gpw[i] * mwd
            tw = -a.zeta_w * math.sqrt(float(np.sum(self.gfw[i] ** 2)))
            tsd = -a.zeta_s * math.sqrt(float(np.sum((self.gfs[i] - self.gfw[i]) ** 2)))
            for d in range(D):
                dw, ds = tw * sign(self.gvw[i, d]), tsd * sign(self.gvs[i, d])
                self.gaw[i, d] = mwd * (self.gfw[i, d] + dw + self.gfd[i, d])
                self.gas[i, d] = msd * (-self.gmi[i] * self.gaw[i, d] + self.gfs[i, d] + dw + ds)
                self.gvsT[i, d] = self.gvs[i, d] + self.gas[i, d] * dt
                self.gvwT[i, d] = self.gvw[i, d] + self.gaw[i, d] * dt
            for d in range(D):
                if self.bcidx[d][i] != 0:
                    self.gvsT[i, d] = self.bcval[d][i]
                if self.wbcidx[d][i] != 0:
                    self.gvwT[i, d] = self.wbcval[d][i]
            self.gps[i] = 0.0
            self.gpw[i] = 0.0
        # doublemapping1_TS!, utils_TS.jl:543-648
        for ix in range(self.np):
            pos, s1, s2, w1, w2 = (np.zeros(D) for _ in range(5))
            for q in range(self.NIC):
                Ni = self.Nij[ix, q]
                if Ni == 0.0:
                    continue
                nd = self.p2n[ix, q] - 1
                pos += Ni * self.gvsT[nd]
                s1 += Ni * (self.gvsT[nd] - self.gvs[nd])
                s2 += Ni * self.gvsT[nd]
                w1 += Ni * (self.gvwT[nd] - self.gvw[nd])
                w2 += Ni * self.gvwT[nd]
            n = self.n[ix]
            self.xi[ix] += dt * pos
            self.vs[ix] = a.FLIP * (self.vs[ix] + s1) + a.PIC * s2
            self.vw[ix] = a.FLIP * (self.vw[ix] + w1) + a.PIC * w2
            self.ps[ix] = self.ms[ix] * self.vs[ix] * (1.0 - n)
            self.pw[ix] = self.mw[ix] * self.vw[ix] * n
        # doublemapping2_TS!
        for ix in range(self.np):
            for q in range(self.NIC):
                Ni = self.Nij[ix, q]
                if Ni != 0.0:
                    nd = self.p2n[ix, q] - 1
                    self.gps[nd] += self.ps[ix] * Ni
                    self.gpw[nd] += self.pw[ix] * Ni
        # doublemapping3_TS!
        for i in range(self.ni):
            msd = 0.0 if self.gms[i] == 0.0 else 1.0 / self.gms[i]
            mwd = 0.0 if self.gmw[i] == 0.0 else 1.0 / self.gmw[i]
            self.gvs[i] = self.gps[i] * msd
            self.gvw[i] = self.gpw[i] * mwd
            for d in range(D):
                if self.bcidx[d][i] != 0:
                    self.gvs[i, d] = self.bcval[d][i]
                if self.wbcidx[d][i] != 0:
                    self.gvw[i, d] = self.wbcval[d][i]
            self.gdus[i] = self.gvs[i] * dt
            self.gduw[i] = self.gvw[i] * dt
        # G2P_TS!: the solid part and the constitutive update are G2P_OS! + liE!/dpP!;
        # the water part needs the pre-step volume
        vol_old = self.Omega.copy()
        self._g2p(dt, Ti)
        for ix in range(self.np):
            dw = np.zeros((D, D))
            for q in range(self.NIC):
                if self.Nij[ix, q] == 0.0:
                    continue
                nd = self.p2n[ix, q] - 1
                for r in range(D):
                    for c in range(D):
                        dw[r, c] += self.gduw[nd, r] * self.dN[c, ix, q]
            dF = self.dF[ix].reshape(D, D)
            if D == 2:
                dew = [dw[0, 0], dw[1, 1], 0.0, dw[0, 1] + dw[1, 0]]
                self.depsw[ix, [0, 1, 3]] = [dew[0], dew[1], dew[3]]
                self.epsw[ix, [0, 1, 3]] += [dew[0], dew[1], dew[3]]
            else:
                self.depsw[ix] = [dw[0, 0], dw[1, 1], dw[2, 2], dw[0, 1] + dw[1, 0], dw[1, 2] + dw[2, 1],
                                  dw[0, 2] + dw[2, 0]]
                # the solid increments, as utils_TS.jl:929-934 writes them
                self.epsw[ix] += [dF[0, 0], dF[1, 1], dF[2, 2], dF[0, 1] + dF[1, 0], dF[1, 2] + dF[2, 1],
                                  dF[0, 2] + dF[2, 0]]
            Fv = self.F[ix]
            if D == 2:
                J = Fv[0] * Fv[3] - Fv[1] * Fv[2]
            else:
                J = (Fv[0] * Fv[4] * Fv[8] + Fv[1] * Fv[5] * Fv[6] + Fv[2] * Fv[3] * Fv[7] -
                     Fv[6] * Fv[4] * Fv[2] - Fv[7] * Fv[5] * Fv[0] - Fv[8] * Fv[3] * Fv[1])
            dJ = J * self.Omega0[ix] / vol_old[ix]
            self.rhow[ix] = self.rhow0[ix] / J
            n = self.n[ix]
            trs, trw = float(np.trace(dF)), float(np.trace(dw))
            self.sigw[ix] += (self.Kw[self.nid[ix] - 1] / n) * ((1.0 - n) * trs + n * trw)
            self.n[ix] = 1.0 - (1.0 - n) / dJ
