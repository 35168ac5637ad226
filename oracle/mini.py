"""Independent numpy restatement of one RK3 stage (TEST INFRASTRUCTURE ONLY).

Where oracle/les_oracle.cpp follows the reference's sliding z-window and
ring buffers (comp1.f90:67-186), this file states the same stage level by
level: every padded plane quantity is a function of the level index with the
boundary rules made explicit.  Agreement of the two (tests/test_oracle.py)
pins the restatement of the ring-buffer control flow, and this level form is
the one the CUDA path implements.  FFTs come from numpy (pocketfft), not from
the oracle's own DFT, so the transforms are independent too.

Boundary rules read off the reference (U = expand(u), E = max(expand(e), emin)):
  ghosts       u(0)=v(0)=0, w(-1)=w(0)=0, e(0)=e(1)        lowerbc.f90:9-18
               u,v(nnz+1..nnz+2)=0, w(nnz..nnz+2)=0,
               e(nnz..nnz+1)=e(nnz-1), rw(nnz)=0            upperbc.f90:12-28
  UX,UY,VX,VY  0 at L=0 and L=nnz+1, spectral otherwise     derivs1.f90:29-33, derivs2.f90:23-26
  WZ           0 at L=0 and L=nnz+1, (W[L]-W[L-1])/dz       derivs1.f90:21-22, derivs2.f90:14, 29
  UZ,VZ        (U[L+1]-U[L])/dz, L=1..nnz-1; copies at 0, nnz derivs1.f90:24, 37, derivs2.f90:15, 27
  WX,WY        0 at L=0 and L=nnz, spectral otherwise       derivs1.f90:26-27, 35-36, derivs2.f90:17-18, 30-31
  EX,EY        at level iz use E[min(iz, nnz-2)]            derivs2.f90:20-21 (not set for iz>=nnz-1)
  XKK[L]       L=0..nnz from E[L] (imodel 3) or SHEAR[L]     complen.f90:13-24, compsgs1.f90:22-38
"""
import numpy as np

GAMA = (8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0)
ZETAS = (0.0, 17.0 / 60.0, 5.0 / 12.0)


def wavenumbers(n, length):
    k = np.arange(n, dtype=np.float64)
    k[k > n // 2] -= n
    return k * 2.0 * np.pi / length


def xderiv(a, length):
    n = a.shape[-1]
    f = np.fft.fft(a, axis=-1)
    k = wavenumbers(n, length)
    k[0] = 0.0
    k[n // 2] = 0.0
    return np.fft.ifft(f * (1j * k), axis=-1).real


def yderiv(a, length):
    n = a.shape[-2]
    f = np.fft.fft(a, axis=-2)
    k = wavenumbers(n, length)
    k[0] = 0.0
    k[n // 2] = 0.0
    return np.fft.ifft(f * (1j * k)[:, None], axis=-2).real


def r2c(a):
    n2, n1 = a.shape[-2:]
    return np.fft.rfft2(a) / (n1 * n2)


def c2r(z, n1):
    n2 = z.shape[-2]
    return np.fft.irfft2(z, s=(n2, n1)) * (n1 * n2)


def expand(a):
    ny, nx = a.shape[-2:]
    nyb, nxb = 3 * ny // 2, 3 * nx // 2
    z = r2c(a)
    zl = np.zeros(a.shape[:-2] + (nyb, nxb // 2 + 1), dtype=np.complex128)
    zl[..., : ny // 2, : nx // 2] = z[..., : ny // 2, : nx // 2]
    zl[..., ny // 2 + 1 + (nyb - ny):, : nx // 2] = z[..., ny // 2 + 1:, : nx // 2]
    return c2r(zl, nxb)


def compress(a):
    nyb, nxb = a.shape[-2:]
    ny, nx = 2 * nyb // 3, 2 * nxb // 3
    z = r2c(a)
    zs = np.zeros(a.shape[:-2] + (ny, nx // 2 + 1), dtype=np.complex128)
    zs[..., : ny // 2, : nx // 2] = z[..., : ny // 2, : nx // 2]
    zs[..., ny // 2 + 1:, : nx // 2] = z[..., ny // 2 + 1 + (nyb - ny):, : nx // 2]
    return c2r(zs, nx)


def deal(a):
    ny, nx = a.shape[-2:]
    z = r2c(a)
    z[..., nx // 2] = 0.0
    z[..., ny // 2, : nx // 2] = 0.0
    return c2r(z, nx)


class MiniLes:
    """State arrays are (nnz, ny, nx) float64 for levels 1..nnz."""

    def __init__(self, cfg):
        self.nx, self.ny, self.nz = cfg.nnx, cfg.nny, cfg.nnz
        self.xl, self.yl, self.zl, self.z0 = cfg.xl, cfg.yl, cfg.zl, cfg.z0
        self.imodel, self.isurface = cfg.imodel, cfg.isurface
        self.tke_production, self.nu = cfg.tke_production, cfg.nu
        self.dt, self.emin, self.forcing = cfg.dt, cfg.emin, cfg.forcing
        self.dx, self.dy, self.dz = self.xl / self.nx, self.yl / self.ny, self.zl / self.nz
        self.dsl = (self.dx * self.dy * self.dz) ** (1.0 / 3.0)
        self.ceps = 0.93 / self.dsl
        self.zody = np.log(self.dz / 2.0 / self.z0)
        sh = (self.nz, self.ny, self.nx)
        self.u, self.v, self.w, self.e = (np.zeros(sh) for _ in range(4))
        self.p = np.zeros(sh)
        self.ru, self.rv, self.rw, self.re = (np.zeros(sh) for _ in range(4))
        self.meanbuf = np.zeros((19, self.nz))
        self.utau = self.utau_s = self.dudt = self.dvdt = 0.0
        # ghost e levels persist between stages exactly as in the reference
        self.e_ghost_bot = np.zeros((self.ny, self.nx))
        self.e_ghost_top = np.zeros((self.ny, self.nx))

    # ---- the level form of comp1 -------------------------------------
    def comp1(self, mnout, istage, dtab2, xkmax):
        nz, dz = self.nz, self.dz
        dzm, dzm2, todzm = 1.0 / dz, 1.0 / dz ** 2, 0.5 / dz
        xl, yl, emin = self.xl, self.yl, self.emin
        # lower/upper ghosts (lowerbc.f90:9-18, upperbc.f90:12-28)
        self.e_ghost_bot = self.e[0].copy()
        self.e_ghost_top = self.e[nz - 2].copy()
        self.e[nz - 1] = self.e_ghost_top
        self.w[nz - 1] = 0.0
        zero = np.zeros((1, self.ny, self.nx))
        # padded planes; index L maps to array row L+off
        U = expand(np.concatenate([zero, self.u, zero, zero]))          # L = 0..nz+2
        V = expand(np.concatenate([zero, self.v, zero, zero]))
        wl = self.w.copy()
        wl[nz - 1] = 0.0
        W = expand(np.concatenate([zero, zero, wl, zero, zero]))        # L = -1..nz+2
        el = np.concatenate([self.e_ghost_bot[None], self.e[: nz - 1], self.e_ghost_top[None], self.e_ghost_top[None]])
        E = np.maximum(expand(el), emin)                                # L = 0..nz+1
        u_ = lambda L: U[L]
        v_ = lambda L: V[L]
        w_ = lambda L: W[L + 1]
        e_ = lambda L: E[L]
        nb = U.shape[1:]
        zb = np.zeros(nb)

        def dx_(f, L, lo, hi):
            return zb if (L < lo or L > hi) else xderiv(f(L), xl)

        def dy_(f, L, lo, hi):
            return zb if (L < lo or L > hi) else yderiv(f(L), yl)

        UX = {L: dx_(u_, L, 1, nz) for L in range(0, nz + 2)}
        UY = {L: dy_(u_, L, 1, nz) for L in range(0, nz + 2)}
        VX = {L: dx_(v_, L, 1, nz) for L in range(0, nz + 2)}
        VY = {L: dy_(v_, L, 1, nz) for L in range(0, nz + 2)}
        WZ = {L: (zb if L in (0, nz + 1) else (w_(L) - w_(L - 1)) * dzm) for L in range(0, nz + 2)}
        UZ = {L: (u_(L + 1) - u_(L)) * dzm for L in range(1, nz)}
        UZ[0], UZ[nz] = UZ[1], UZ[nz - 1]
        VZ = {L: (v_(L + 1) - v_(L)) * dzm for L in range(1, nz)}
        VZ[0], VZ[nz] = VZ[1], VZ[nz - 1]
        WX = {L: dx_(w_, L, 1, nz - 1) for L in range(0, nz + 1)}
        WY = {L: dy_(w_, L, 1, nz - 1) for L in range(0, nz + 1)}

        def shear(L):
            return (UX[L] ** 2 + UX[L + 1] ** 2 + VY[L] ** 2 + VY[L + 1] ** 2 + WZ[L] ** 2 + WZ[L + 1] ** 2
                    + 0.5 * (UY[L] + VX[L]) ** 2 + 0.5 * (UY[L + 1] + VX[L + 1]) ** 2
                    + (UZ[L] + WX[L]) ** 2 + (VZ[L] + WY[L]) ** 2)

        SH = {L: shear(L) for L in range(0, nz + 1)}
        if self.imodel == 4:
            XKK = {L: np.minimum((0.1 * self.dsl) ** 2 * np.sqrt(SH[L]), xkmax) + self.nu for L in range(0, nz + 1)}
        else:
            XKK = {L: np.minimum(0.1 * self.dsl * np.sqrt(e_(L)), xkmax) + self.nu for L in range(0, nz + 1)}

        # wall stresses (lowerbc.f90:25-165, upperbc.f90:33-160), isurface 1..6
        self.dudt = self.ru.sum() / self.ru.size
        self.dvdt = self.rv.sum() / self.rv.size
        self.utau_s = np.sqrt(self.zl / 2 * np.sqrt(self.dvdt ** 2 + (self.forcing - self.dudt) ** 2))

        def wall(L, sg):
            """sg = -1 lower wall (sufsim), +1 upper wall (sufsim_upper)."""
            U0, V0 = U[L], V[L]
            u1, v1 = U0.mean(), V0.mean()
            wind = np.sqrt(U0 * U0 + V0 * V0)
            windm = max(wind.mean(), 0.0, 0.01)   # max(windm, ufree), max(windm, 0.01); ufree = 0
            vsfc = max(np.sqrt(u1 * u1 + v1 * v1), 0.01)
            ut = vsfc * 0.4 / self.zody
            ut2 = ut * ut
            uf, vf = U0 - u1, V0 - v1             # ufluc, vfluc (ugal = 0)
            th = np.arccos(min(max(u1 / vsfc, -1.0), 1.0))
            au = sg * ut2 * np.cos(th)             # auuwm, auvwm (lowerbc.f90:88-89, upperbc.f90:87-88)
            av = sg * ut2 * np.sin(th) * np.copysign(1.0, v1)
            if self.isurface == 1:
                return sg * ut2 / vsfc * U0, sg * ut2 / vsfc * V0, ut
            if self.isurface == 2:
                c = sg * ut2 / (windm * vsfc)
                return c * (windm * uf + wind * u1), c * (windm * vf + wind * v1), ut
            if self.isurface == 3:
                return (au - sg * 0.35 * uf * ut2 / np.sqrt((uf * uf).mean()),
                        av - sg * 0.35 * vf * ut2 / np.sqrt((vf * vf).mean()), ut)
            sf = wind - windm
            if self.isurface == 4:
                den = np.sqrt((windm * u1 + (uf * sf).mean()) ** 2 + (windm * v1 + (vf * sf).mean()) ** 2)
                return sg * ut2 * wind * U0 / den, sg * ut2 * wind * V0 / den, ut
            if self.isurface == 5:
                mu, mv = sf * u1 + windm * uf, sf * v1 + windm * vf
                root = np.sqrt((mu * mu).mean())  # moengv2m is built from moengu2 (lowerbc.f90:121)
                return au - sg * 0.35 * ut2 * mu / root, av - sg * 0.35 * ut2 * mv / root, ut
            a6u = -self.zl / 2 * (self.forcing - self.dudt)
            a6v = -self.zl / 2 * (-self.dvdt)
            if sg < 0:
                return a6u - ut * self.utau_s * uf / vsfc, a6v - ut * self.utau_s * vf / vsfc, ut
            return -a6u + ut * self.utau_s * uf / vsfc, -a6v + ut * self.utau_s * vf / vsfc, ut

        TUW, TVW = {}, {}
        TUW[0], TVW[0], self.utau_lower = wall(1, -1.0)
        for L in range(1, nz):
            TUW[L] = -XKK[L] * (UZ[L] + WX[L])
            TVW[L] = -XKK[L] * (VZ[L] + WY[L])
        TUW[nz], TVW[nz], self.utau = wall(nz, +1.0)
        TWW = {L: -(XKK[L - 1] + XKK[L]) * WZ[L] for L in range(1, nz + 1)}
        TWW[nz + 1] = zb

        ru_new = np.zeros_like(self.ru)
        rv_new = np.zeros_like(self.rv)
        rw_new = np.zeros_like(self.rw)
        re_new = np.zeros_like(self.re)
        for iz in range(1, nz + 1):
            U0, U1, Um = u_(iz), u_(iz + 1), u_(iz - 1)
            V0, V1, Vm = v_(iz), v_(iz + 1), v_(iz - 1)
            W0, W1, Wm = w_(iz), w_(iz + 1), w_(iz - 1)
            s = XKK[iz - 1] + XKK[iz]
            tuu, tvv, tuv = -s * UX[iz], -s * VY[iz], -s * (UY[iz] + VX[iz]) * 0.5
            self.meanbuf[2, iz - 1] = np.sum((UX[iz] + VY[iz] + WZ[iz]) ** 2) / U0.size
            rub = (-xderiv(U0 * U0, xl) - yderiv(U0 * V0, yl) - ((U1 + U0) * W0 - (Um + U0) * Wm) * todzm
                   + self.forcing - xderiv(tuu, xl) - yderiv(tuv, yl) - (TUW[iz] - TUW[iz - 1]) * dzm)
            rvb = (-xderiv(U0 * V0, xl) - yderiv(V0 * V0, yl) - ((V1 + V0) * W0 - (Vm + V0) * Wm) * todzm
                   - xderiv(tuv, xl) - yderiv(tvv, yl) - (TVW[iz] - TVW[iz - 1]) * dzm)
            ru_new[iz - 1] = compress(rub)
            rv_new[iz - 1] = compress(rvb)
            if iz != nz:
                rwb = (-0.5 * xderiv((U0 + U1) * W0, xl) - 0.5 * yderiv((V0 + V1) * W0, yl)
                       - ((0.5 * (W1 + W0)) ** 2 - (0.5 * (W0 + Wm)) ** 2) * dzm
                       - xderiv(TUW[iz], xl) - yderiv(TVW[iz], yl) - (TWW[iz + 1] - TWW[iz]) * dzm)
                le = min(iz, nz - 2)
                EX, EY = xderiv(e_(le), xl), yderiv(e_(le), yl)
                E0, E1, Em = e_(iz), e_(iz + 1), e_(iz - 1)
                reb = (-0.5 * (xderiv(E0 * (U0 + U1), xl) + yderiv(E0 * (V0 + V1), yl))
                       - (W1 * E1 - Wm * Em) * todzm
                       + xderiv(2 * XKK[iz] * EX, xl) + yderiv(2 * XKK[iz] * EY, yl)
                       + ((XKK[iz + 1] + XKK[iz]) * (E1 - E0) - (XKK[iz] + XKK[iz - 1]) * (E0 - Em)) * dzm2
                       - self.ceps * E0 * np.sqrt(E0))
                if self.tke_production:
                    reb = reb + XKK[iz] * SH[iz]
                r = compress(rwb)
                rw_new[iz - 1] = r - r.mean()
                re_new[iz - 1] = compress(reb)
            if mnout and istage == 1:
                self.meanbuf[13, iz - 1] = tuu.mean()
                self.meanbuf[14, iz - 1] = tvv.mean()
                self.meanbuf[15, iz - 1] = tuv.mean()
                self.meanbuf[16, iz - 1] = TWW[iz].mean()
                self.meanbuf[17, iz - 1] = TUW[iz].mean()
                self.meanbuf[18, iz - 1] = TVW[iz].mean()
        # zeta part of the stage, applied to the stored fields (comp1.f90:126-133)
        if istage != 1:
            self.u -= dtab2 * self.ru
            self.v -= dtab2 * self.rv
            self.w[: nz - 1] -= dtab2 * self.rw[: nz - 1]
            self.e[: nz - 1] -= dtab2 * self.re[: nz - 1]
        self.ru, self.rv, self.rw, self.re = ru_new, rv_new, rw_new, re_new

    # ---- comprhs + press + comp2 (comprhs.f90, press.F90, comp2.f90) ----
    def project(self, dtab1):
        nz, dz, nx, ny = self.nz, self.dz, self.nx, self.ny
        dtabm = 1.0 / dtab1
        f1 = xderiv(self.ru + self.u * dtabm, self.xl)
        f2 = yderiv(self.rv + self.v * dtabm, self.yl)
        q = self.w * dtabm + self.rw
        q[nz - 1] = 0.0  # w(nnz) = rw(nnz) = 0
        qm = np.concatenate([np.zeros((1, ny, nx)), q[:-1]])
        rhs = f1 + f2 + (q - qm) / dz
        ph = r2c(rhs)  # (nz, ny, nx/2+1)
        xk = wavenumbers(nx, self.xl)[: nx // 2 + 1]
        yk = wavenumbers(ny, self.yl)
        k2 = yk[:, None] ** 2 + xk[None, :] ** 2
        b = np.empty((nz,) + k2.shape)
        b[:] = -dz * dz * k2 - 2.0
        b[0] = -dz * dz * k2 - 1.0
        b[-1] = -dz * dz * k2 - 1.0
        r = dz * dz * ph
        b[:, 0, 0] = 1.0
        r[:, 0, 0] = 0.0
        # Thomas with unit off-diagonals (tridv.f90:1-55)
        dinv = np.empty_like(b)
        dinv[0] = 1.0 / b[0]
        zero_mode = np.zeros(k2.shape, dtype=bool)
        zero_mode[0, 0] = True
        off = np.where(zero_mode, 0.0, 1.0)
        rr = r.copy()
        for i in range(1, nz):
            fac = off * dinv[i - 1]
            dinv[i] = 1.0 / (b[i] - fac * off)
            rr[i] = rr[i] - fac * rr[i - 1]
        rr[nz - 1] = rr[nz - 1] * dinv[nz - 1]
        for i in range(nz - 2, -1, -1):
            rr[i] = dinv[i] * (rr[i] - off * rr[i + 1])
        rr[:, 0, 0] = 0.0
        rr[:, :, nx // 2] = 0.0
        rr[:, ny // 2, :] = 0.0
        p = c2r(rr, nx)
        self.p = p
        self.ru = self.ru - xderiv(p, self.xl)
        self.rv = self.rv - yderiv(p, self.yl)
        rw = self.rw.copy()
        rw[: nz - 1] = rw[: nz - 1] - (p[1:] - p[:-1]) / dz
        rw[: nz - 1] -= rw[: nz - 1].mean(axis=(1, 2), keepdims=True)
        self.rw = rw
        self.u = self.u + dtab1 * self.ru
        self.v = self.v + dtab1 * self.rv
        self.w[: nz - 1] = self.w[: nz - 1] + dtab1 * self.rw[: nz - 1]
        self.e[: nz - 1] = np.maximum(self.e[: nz - 1] + dtab1 * self.re[: nz - 1], self.emin)
        self.w[: nz - 1] -= self.w[: nz - 1].mean(axis=(1, 2), keepdims=True)

    def stage(self, mnout, istage):
        dtab1 = self.dt * GAMA[istage - 1]
        dtab2 = self.dt * ZETAS[istage - 1]
        xkmax = self.dz * self.dz / self.dt / 5.0
        self.comp1(mnout, istage, dtab2, xkmax)
        self.project(dtab1)
