"""Fingerprints of a channel state, shared by the fixture generator
(make_channel_golden.py) and the GPU parity tests that read the fixtures.

A C2 state (128 x 128 x 96, five fields) is 63 MB in float64, too large to
commit, so a fixture keeps what the parity checks need:
  * four x-y planes (levels 1, nnz/4+1, nnz/2+1, nnz-1 in the reference's
    1-based numbering) of u, v, w, e sampled every second point in x and y;
  * per level and field, the RMS over the plane and the projection onto a
    fixed seeded N(0,1) weight plane (a pointwise change of size d moves it
    by about d*sqrt(nx*ny), so it fingerprints every point of every level);
  * compmn's meanbuf(19, nnz) and the wall-model scalars;
  * the 1D x-spectra (spectra2.f90:24-32) of u at the sampled levels;
  * the discrete divergence after every projection (below).
"""
import numpy as np

WEIGHT_SEED = 20241204


def sample_levels(nz):
    return [0, nz // 4, nz // 2, nz - 2]


def weight_plane(ny, nx):
    return np.random.default_rng(WEIGHT_SEED).standard_normal((ny, nx))


def divergence(u, v, w, xl, yl, zl):
    """Discrete divergence of a (nz, ny, nx) state as comprhs.f90:17-35
    forms it: spectral d/dx u + d/dy v with the DC and Nyquist modes zeroed
    (filter_fftw.f90:138-248) plus (w(iz) - w(iz-1))/dz with w(0) = 0."""
    nz, ny, nx = u.shape
    dz = zl / nz
    kx = np.fft.rfftfreq(nx, 1.0 / nx) * 2 * np.pi / xl
    ky = np.fft.fftfreq(ny, 1.0 / ny) * 2 * np.pi / yl
    kx[nx // 2] = 0.0
    ky[ny // 2] = 0.0
    uh = np.fft.rfft2(u, axes=(1, 2))
    vh = np.fft.rfft2(v, axes=(1, 2))
    dh = 1j * kx[None, None, :] * uh + 1j * ky[None, :, None] * vh
    d = np.fft.irfft2(dh, s=(ny, nx), axes=(1, 2))
    wm = np.concatenate([np.zeros((1, ny, nx)), w[:-1]], axis=0)
    return d + (w - wm) / dz


def divergence_ratio(f, xl, yl, zl):
    """max |div| relative to the velocity-gradient scale max|u| nz / zl."""
    d = divergence(f["u"], f["v"], f["w"], xl, yl, zl)
    scale = max(np.abs(f["u"]).max(), 1e-300) * f["u"].shape[0] / zl
    return float(np.abs(d).max() / scale)


def fingerprint(f):
    """Dictionary of arrays (see module docstring) of a state f with keys
    u, v, w, e shaped (nz, ny, nx)."""
    nz, ny, nx = f["u"].shape
    lv = sample_levels(nz)
    r = weight_plane(ny, nx)
    out = {}
    for k in "uvwe":
        a = f[k]
        out["plane_" + k] = a[lv][:, ::2, ::2].copy()
        out["rms_" + k] = np.sqrt((a * a).mean(axis=(1, 2)))
        out["proj_" + k] = np.einsum("zyx,yx->z", a, r)
    return out


def xspectrum(plane):
    """1D x-spectrum of one (ny, nx) plane as spectra2.f90:18-32 forms it:
    sum over ky of |a_hat(kx, ky)|^2 with a_hat = FFT2/(nx ny), doubled for
    0 < kx < nx/2."""
    ny, nx = plane.shape
    a = np.fft.rfft2(plane) / (nx * ny)
    s = (np.abs(a) ** 2).sum(axis=0)
    s[1:nx // 2] *= 2.0
    return s
