"""Restatement of the reference's spectral regridding program redim.f90 in
numpy.  Test infrastructure only: the GPU regrid (les_gpu_regrid) is checked
against it.

What the reference does (redim.f90):
  * interpol (redim.f90:202-269) walks the old levels with a window of three
    (m, a, b) and linearly inter/extrapolates every new level from them:
    cell-centre fields (u, v, p) at zh = (izn - 1/2) dz_new from levels a, b
    (redim.f90:237-243); face fields (w, e) at zf = izn dz_new from (m, a) or
    (a, b) (redim.f90:245-251).  The window starts with a = level 1, b =
    level 2, w(m) = 0 and e(m) = e(1) (redim.f90:207-217).
  * subroutine redim (redim.f90:277-318) moves each x-y plane to the new grid
    through the scaled forward transform, zeroes the old x and y Nyquist
    modes, copies kx <= min(nx)/2 and ky in [0, min(ny)/2] plus the negative
    ky band (-(min(ny)/2 - 1) .. -1), and transforms back unscaled.
  * e is clamped to [1e-10, max over the plane of the interpolated e]
    (redim.f90:262-263).
A run that restarts from the output deals u, v, w, e (les.F90:185-190,
filter_fftw.f90:316-329: zero the x and y Nyquist modes); `restart_state`
applies that step too, plus the solver's w(nnz) = 0.

With nyquist=False the output grid's Nyquist modes are dropped before e's
clamp instead of after it (the form the GPU regrid computes).  The two agree
exactly when the grid is refined in x and y (the old Nyquist modes are zero,
so the new Nyquist modes are too); when it is coarsened they differ only in e
where the clamp is active.
"""
import numpy as np


def z_table(nzold, nznew, zl):
    """Per new level izn = 1..nznew: (a, b, c, f0, f1, d) with
    centre value = B + (B - A) * c from old levels a, b (1-based) and
    face value = F1 + (F1 - F0) * d from old levels f0, f1 (0 = the wall:
    w(0) = 0, e(0) = e(1)).  Follows interpol (redim.f90:202-269)."""
    if nzold < 2:
        raise ValueError("redim needs at least two old levels")
    dzold, dznew = zl / nzold, zl / nznew
    izo = 2
    zhold = izo * dzold - 0.5 * dzold
    zfold = (izo - 1) * dzold
    out = []
    for izn in range(1, nznew + 1):
        zh = izn * dznew - 0.5 * dznew
        zf = izn * dznew
        while zhold < zh and izo < nzold:
            izo += 1
            zhold = izo * dzold - 0.5 * dzold
            zfold = (izo - 1) * dzold
        c = (zh - zhold) / dzold
        if zf <= zfold:
            f0, f1, d = izo - 2, izo - 1, (zf - zfold) / dzold
        else:
            f0, f1, d = izo - 1, izo, (zf - (zfold + dzold)) / dzold
        out.append((izo - 1, izo, c, f0, f1, d))
    return out


def regrid_plane(x, nxo, nyo, nyquist=True):
    """subroutine redim (redim.f90:277-318) on one plane x[ny][nx]."""
    nyi, nxi = x.shape
    if (nxi, nyi) == (nxo, nyo):
        return np.array(x, dtype=np.float64)
    W = np.fft.rfft2(x) / (nxi * nyi)      # forward, sign -1, scaled
    W[:, nxi // 2] = 0.0                    # wavein(nxin+1:nxin+2,:) = 0
    W[nyi // 2, :] = 0.0                    # wavein(1:nxin,nyin/2+1) = 0
    nxm, nym = min(nxi, nxo), min(nyi, nyo)
    O = np.zeros((nyo, nxo // 2 + 1), dtype=np.complex128)
    O[:nym // 2 + 1, :nxm // 2 + 1] = W[:nym // 2 + 1, :nxm // 2 + 1]
    if nym // 2 > 1:
        O[nyo - nym // 2 + 1:, :nxm // 2 + 1] = W[nyi - nym // 2 + 1:, :nxm // 2 + 1]
    if not nyquist:
        O[:, nxo // 2] = 0.0
        O[nyo // 2, :] = 0.0
    return np.fft.irfft2(O * (nxo * nyo), s=(nyo, nxo))


def deal(x):
    """deal (filter_fftw.f90:316-329) on every plane of x[..., ny, nx]."""
    ny, nx = x.shape[-2:]
    W = np.fft.rfft2(x)
    W[..., :, nx // 2] = 0.0
    W[..., ny // 2, :] = 0.0
    return np.fft.irfft2(W, s=(ny, nx))


def redim_fields(u, v, w, e, p, zl, nxo, nyo, nzo, nyquist=True):
    """The output planes of redim.f90 for fields [nz][ny][nx] (levels 1..nz
    of the restart file).  Returns dict u, v, w, e, p of [nzo][nyo][nxo]."""
    nzi = u.shape[0]
    tab = z_table(nzi, nzo, zl)
    res = {k: np.zeros((nzo, nyo, nxo)) for k in "uvwep"}
    for n, (a, b, c, f0, f1, d) in enumerate(tab):
        for k, f in (("u", u), ("v", v), ("p", p)):
            A, B = f[a - 1], f[b - 1]
            res[k][n] = regrid_plane(B + (B - A) * c, nxo, nyo, nyquist)
        w0 = np.zeros_like(w[0]) if f0 == 0 else w[f0 - 1]
        res["w"][n] = regrid_plane(w[f1 - 1] + (w[f1 - 1] - w0) * d, nxo, nyo, nyquist)
        e0 = e[0] if f0 == 0 else e[f0 - 1]
        eh = e[f1 - 1] + (e[f1 - 1] - e0) * d
        en = regrid_plane(eh, nxo, nyo, nyquist)
        res["e"][n] = np.minimum(eh.max(), np.maximum(en, 1e-10))
    return res


def restart_state(fields):
    """The state a run holds after restarting from redim's output: u, v, w,
    e dealt (les.F90:185-190), w(nnz) = 0, and p without its Nyquist modes
    (the spectral pressure state carries none)."""
    out = {k: deal(fields[k]) for k in "uvwep"}
    out["w"][-1] = 0.0
    return out
