"""ORACLE (test infrastructure only): numpy restatement of the learned
closure's grid operations, independent of the C++ oracle's Stockham DFT.

- features(): the network inputs at the cell centres of a state (the
  gradient stencils of the learned stage: spectral x/y derivatives, w
  averaged to the centres, centred z differences of u, v that are
  one-sided at the walls as derivs1.f90 / derivs2.f90 set the wall rows),
  made dimensionless: g / |G|, min(z_w / Delta, 16), z_w / h, with the
  output scale Delta |G| (tau = (Delta |G|)^2 c);
- divergence(): the dealiased stress divergence added to ru, rv, rw;
- filter_fields(): the explicit filter that makes training data from a
  fine run (z box average, x-y box-filter transfer with truncation to the
  coarse modes as in redim.f90:277-318, tau_ij = filt(u_i u_j) -
  filt(u_i) filt(u_j));
- mlp(): the network in numpy with bfloat16 rounding of inputs, weights and
  hidden activations.
Fields are (nz, ny, nx) arrays (x fastest); w holds w-levels 1..nz with
w(nz) = 0, and w(0) = 0 below.
"""
import numpy as np

from oracle import oracle as O


def bf16(a):
    f = np.asarray(a, dtype=np.float64).astype(np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32).view(np.float32).astype(np.float64)


def mlp(P, x, round_bf16=True):
    q = bf16 if round_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    W = [P[o:o + int(np.prod(sh))].reshape(sh) for (o, sh) in O.mlp_slices()]
    c, a = np.sqrt(2 / np.pi), 0.044715
    gelu = lambda z: 0.5 * z * (1 + np.tanh(c * (z + a * z ** 3)))
    h = q(x)
    for k in range(3):
        h = q(gelu(h @ q(W[2 * k]).T + W[2 * k + 1]))
    return h @ q(W[6]).T + W[7]


class Spec:
    """Spectral x/y derivatives and Nyquist removal on (..., ny, nx) planes."""

    def __init__(self, nx, ny, xl, yl):
        self.nx, self.ny = nx, ny
        self.kx = 2 * np.pi / xl * np.arange(nx // 2 + 1)
        self.ky = 2 * np.pi / yl * np.fft.fftfreq(ny, 1.0 / ny)
        self.mask = np.ones((ny, nx // 2 + 1))
        self.mask[:, nx // 2] = 0
        self.mask[ny // 2, :] = 0

    def dx(self, f):
        return np.fft.irfft2(np.fft.rfft2(f) * 1j * self.kx * self.mask, s=f.shape[-2:])

    def dy(self, f):
        return np.fft.irfft2(np.fft.rfft2(f) * 1j * self.ky[:, None] * self.mask, s=f.shape[-2:])

    def deal(self, f):
        return np.fft.irfft2(np.fft.rfft2(f) * self.mask, s=f.shape[-2:])


def _wl(w, k, nz):
    return w[k - 1] if 1 <= k <= nz - 1 else np.zeros(w.shape[1:])


def gradients(u, v, w, xl, yl, zl):
    """Nine gradient planes per level: (9, nz, ny, nx) in feature order
    (ux, vx, wx, uy, vy, wy, uz, vz, wz)."""
    nz, ny, nx = u.shape
    sp = Spec(nx, ny, xl, yl)
    dz = zl / nz
    g = np.zeros((9, nz, ny, nx))
    for k in range(1, nz + 1):
        wc = 0.5 * (_wl(w, k, nz) + _wl(w, k - 1, nz))
        g[0, k - 1], g[1, k - 1], g[2, k - 1] = sp.dx(u[k - 1]), sp.dx(v[k - 1]), sp.dx(wc)
        g[3, k - 1], g[4, k - 1], g[5, k - 1] = sp.dy(u[k - 1]), sp.dy(v[k - 1]), sp.dy(wc)
        for c, a in enumerate((u, v)):
            if k == 1:
                d = (a[1] - a[0]) / dz
            elif k == nz:
                d = (a[nz - 1] - a[nz - 2]) / dz
            else:
                d = (a[k] - a[k - 2]) / (2 * dz)
            g[6 + c, k - 1] = d
        g[8, k - 1] = (_wl(w, k, nz) - _wl(w, k - 1, nz)) / dz
    return g


ZW_CAP = 16.0


def features(u, v, w, xl, yl, zl):
    """Raw network inputs (nz*ny*nx, 11) and the output scale Delta |G|
    (nz*ny*nx,): inputs g_j / |G| (the nine gradients over their Frobenius
    norm), min(z_w / Delta, 16), z_w / h (z_w the distance to the nearest
    wall, h = zl / 2)."""
    nz, ny, nx = u.shape
    dz = zl / nz
    dsl = (xl / nx * yl / ny * dz) ** (1.0 / 3.0)
    g = gradients(u, v, w, xl, yl, zl)
    gm = np.sqrt((g ** 2).sum(axis=0))
    rg = np.where(gm > 0, 1.0 / np.where(gm > 0, gm, 1.0), 0.0)
    zc = (np.arange(nz) + 0.5) * dz
    zw = np.minimum(zc, zl - zc)
    f = np.zeros((nz, ny, nx, 11))
    for j in range(9):
        f[..., j] = g[j] * rg
    f[..., 9] = np.minimum(zw / dsl, ZW_CAP)[:, None, None]
    f[..., 10] = (zw / (zl / 2))[:, None, None]
    return f.reshape(-1, 11), (gm * dsl).reshape(-1)


def dissipation(g, tau):
    """Mean of -tau_ij S_ij over all points; g from gradients(), tau (6, ...)
    in the order tau11, tau22, tau33, tau12, tau13, tau23."""
    s11, s22, s33 = g[0], g[4], g[8]
    s12, s13, s23 = 0.5 * (g[3] + g[1]), 0.5 * (g[6] + g[2]), 0.5 * (g[7] + g[5])
    d = -(tau[0] * s11 + tau[1] * s22 + tau[2] * s33 + 2 * (tau[3] * s12 + tau[4] * s13 + tau[5] * s23))
    return float(d.mean())


def project_backscatter(g, tau):
    """Remove local backscatter: where tau:S > 0 the stress's component
    along S is subtracted, tau' = tau - (tau:S / S:S) S, so -tau':S =
    max(-tau:S, 0) at every point.  g from gradients(), tau (6, ...)."""
    S = [g[0], g[4], g[8], 0.5 * (g[3] + g[1]), 0.5 * (g[6] + g[2]), 0.5 * (g[7] + g[5])]
    w = [1.0, 1.0, 1.0, 2.0, 2.0, 2.0]
    ts = sum(w[i] * tau[i] * S[i] for i in range(6))
    ss = sum(w[i] * S[i] * S[i] for i in range(6))
    a = np.where((ts > 0) & (ss > 0), -ts / np.where(ss > 0, ss, 1.0), 0.0)
    return np.stack([tau[i] + a * S[i] for i in range(6)])


def reference_dissipation(g, dsl, cs=0.17):
    """Mean of (cs dsl)^2 |S|^3 over all cell centres, |S|^2 = 2 S_ij S_ij:
    the Smagorinsky estimate with Lilly's constant."""
    s11, s22, s33 = g[0], g[4], g[8]
    s12, s13, s23 = 0.5 * (g[3] + g[1]), 0.5 * (g[6] + g[2]), 0.5 * (g[7] + g[5])
    ss = 2 * (s11 ** 2 + s22 ** 2 + s33 ** 2 + 2 * (s12 ** 2 + s13 ** 2 + s23 ** 2))
    return float((cs * cs * dsl * dsl * ss * np.sqrt(ss)).mean())


def network_used(dis_raw, dis_applied, dis_r, guard):
    """The stage's fallback rule: the raw network's mean dissipation must be
    >= 0 and, with guard > 0, the applied one within a factor guard of the
    reference's."""
    if not dis_raw >= 0:
        return 0
    if guard > 0 and not (dis_r > 0 and dis_applied <= guard * dis_r and guard * dis_applied >= dis_r):
        return 0
    return 1


def network_viscosity(g, tau, xkmax):
    """Face values (index j = w-level j) of the network's effective
    viscosity: per level -sum(tau13 uz + tau23 vz) / sum(uz^2 + vz^2)
    clipped to [0, xkmax], averaged over the cells j and j+1."""
    nz = g.shape[1]
    a = (tau[4] * g[6] + tau[5] * g[7]).reshape(nz, -1).sum(axis=1)
    b = (g[6] ** 2 + g[7] ** 2).reshape(nz, -1).sum(axis=1)
    nuc = np.clip(np.where(b > 0, -a / np.where(b > 0, b, 1.0), 0.0), 0.0, xkmax)
    out = np.zeros(nz + 1)
    for j in range(1, nz):
        out[j] = 0.5 * (nuc[j - 1] + nuc[j])
    return out


def divergence(tau, xl, yl, zl, u=None, v=None, nut=None):
    """Dealiased stress divergence (lru, lrv, lrw), each (nz, ny, nx).  With
    u, v and the face viscosity nut (network_viscosity()), the compact-stencil
    correction -nut(j) (3 (u(j+1) - u(j)) - (u(j+2) - u(j-1))) / (4 dz) is
    added to tau13, tau23 on the faces 2..nz-2 (it damps odd-even modes)."""
    _, nz, ny, nx = tau.shape
    sp = Spec(nx, ny, xl, yl)
    dz = zl / nz
    # tau13, tau23 averaged to the interior w-levels; 0 on the walls (the
    # wall model's stresses stay in the padded kernels)
    tw = lambda f, k: 0.5 * (tau[f, k - 1] + tau[f, k]) if 1 <= k <= nz - 1 else np.zeros((ny, nx))
    lru = np.zeros((nz, ny, nx)); lrv = np.zeros_like(lru); lrw = np.zeros_like(lru)
    for k in range(1, nz + 1):
        t = lambda f: tau[f, k - 1]
        lru[k - 1] = sp.deal(-sp.dx(t(0)) - sp.dy(t(3)) - (tw(4, k) - tw(4, k - 1)) / dz)
        lrv[k - 1] = sp.deal(-sp.dx(t(3)) - sp.dy(t(1)) - (tw(5, k) - tw(5, k - 1)) / dz)
        if k <= nz - 1:
            lrw[k - 1] = sp.deal(-sp.dx(tw(4, k)) - sp.dy(tw(5, k)) - (tau[2, k] - tau[2, k - 1]) / dz)
    if nut is not None:
        def tc(a, j):
            if j < 2 or j > nz - 2:
                return np.zeros((ny, nx))
            return -nut[j] * (3 * (a[j] - a[j - 1]) - (a[j + 1] - a[j - 2])) / (4 * dz)
        for k in range(1, nz + 1):
            lru[k - 1] -= (tc(u, k) - tc(u, k - 1)) / dz
            lrv[k - 1] -= (tc(v, k) - tc(v, k - 1)) / dz
    return lru, lrv, lrw


def box_transfer(k, width):
    a = 0.5 * np.asarray(k, dtype=np.float64) * width
    out = np.ones_like(a)
    nz = a != 0
    out[nz] = np.sin(a[nz]) / a[nz]
    return out


def _filter_xy(q, nxc, nyc, xl, yl):
    ny, nx = q.shape
    F = np.fft.rfft2(q) / (nx * ny)
    kxc = np.arange(nxc // 2)
    kyc = np.fft.fftfreq(nyc, 1.0 / nyc).astype(int)
    G = box_transfer(2 * np.pi / xl * kxc, xl / nxc)[None, :] * box_transfer(2 * np.pi / yl * kyc, yl / nyc)[:, None]
    C = np.zeros((nyc, nxc // 2 + 1), dtype=np.complex128)
    for i, sk in enumerate(kyc):
        if i == nyc // 2:
            continue
        C[i, :nxc // 2] = F[sk % ny, :nxc // 2] * G[i]
    return np.fft.irfft2(C * (nxc * nyc), s=(nyc, nxc))


def model_stress(u, v, w, e, xl, yl, zl, emin=1e-6):
    """The fine run's Deardorff stress -2 nu_t S_ij at the cell centres,
    nu_t = 0.1 dsl sqrt(max(e_c, emin)), e_c the mean of the cell's two
    faces (e holds faces 1..nz at levels 1..nz; faces 0 and nz take the
    values of faces 1 and nz-1).  Order tau11, tau22, tau33, tau12, tau13,
    tau23."""
    nz, ny, nx = u.shape
    dz = zl / nz
    dsl = (xl / nx * yl / ny * dz) ** (1.0 / 3.0)
    g = gradients(u, v, w, xl, yl, zl)
    face = lambda k: e[min(max(k, 1), nz - 1) - 1]
    ec = np.stack([0.5 * (face(k) + face(k - 1)) for k in range(1, nz + 1)])
    nu2 = 0.2 * dsl * np.sqrt(np.maximum(ec, emin))
    return np.stack([-nu2 * g[0], -nu2 * g[4], -nu2 * g[8], -nu2 * 0.5 * (g[3] + g[1]),
                     -nu2 * 0.5 * (g[6] + g[2]), -nu2 * 0.5 * (g[7] + g[5])])


def filter_fields(u, v, w, xl, yl, fxy, fz, tau_model=None):
    """(9, nz/fz, ny/fxy, nx/fxy): u, v, w (coarse w-levels), tau11, tau22,
    tau33, tau12, tau13, tau23; with tau_model (the fine run's own stress at
    the cell centres, model_stress()) the stresses are the filtered total
    sub-filter stress."""
    nz, ny, nx = u.shape
    nzc, nyc, nxc = nz // fz, ny // fxy, nx // fxy
    wc = np.stack([0.5 * (_wl(w, k, nz) + _wl(w, k - 1, nz)) for k in range(1, nz + 1)])
    q = [u, v, wc, u * u, v * v, wc * wc, u * v, u * wc, v * wc]
    if tau_model is not None:
        for i in range(6):
            q[3 + i] = q[3 + i] + tau_model[i]
    qz = [a.reshape(nzc, fz, ny, nx).mean(axis=1) for a in q]
    if fz == 1:
        wst = np.stack([_wl(w, K, nz) for K in range(1, nzc + 1)])
    else:
        # the box of fz fine cells centred on coarse face K by the trapezoid
        # rule: weights 1/(2 fz) on faces fz K -/+ fz/2, 1/fz between
        h = fz // 2
        wst = np.stack([(0.5 * (_wl(w, fz * K - h, nz) + _wl(w, fz * K + h, nz)) +
                         sum(_wl(w, j, nz) for j in range(fz * K - h + 1, fz * K + h))) / fz
                        for K in range(1, nzc + 1)])
    qz.append(wst)
    Q = np.array([[_filter_xy(a[K], nxc, nyc, xl, yl) for K in range(nzc)] for a in qz])
    out = np.zeros((9, nzc, nyc, nxc))
    out[0], out[1], out[2] = Q[0], Q[1], Q[9]
    out[3] = Q[3] - Q[0] ** 2
    out[4] = Q[4] - Q[1] ** 2
    out[5] = Q[5] - Q[2] ** 2
    out[6] = Q[6] - Q[0] * Q[1]
    out[7] = Q[7] - Q[0] * Q[2]
    out[8] = Q[8] - Q[1] * Q[2]
    return out
