"""ctypes bindings of the CPU oracle (oracle/les_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg as the checker, never by the product path.

The oracle restates the reference routines of paes-channelflow (les.F90,
comp1.f90, derivs1/2.f90, compadv1.f90, complen.f90, compsgs1/3.f90,
lowerbc.f90, upperbc.f90, filter_fftw.f90, comprhs.f90, press.F90,
tridv.f90, comp2.f90, compmn.F90, spectra2.f90).  Parity unpinned: the
reference ships no golden vectors and cannot be built here; the restatement
is pinned by analytic known answers and by the independent numpy
restatement in oracle/mini.py.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


class LesConfig(ctypes.Structure):
    """Mirror of `les_config` in include/les_gpu.h."""

    _fields_ = [
        ("nnx", ctypes.c_int), ("nny", ctypes.c_int), ("nnz", ctypes.c_int),
        ("imodel", ctypes.c_int), ("isurface", ctypes.c_int),
        ("tke_production", ctypes.c_int), ("precision", ctypes.c_int),
        ("device", ctypes.c_int),
        ("xl", ctypes.c_double), ("yl", ctypes.c_double), ("zl", ctypes.c_double),
        ("z0", ctypes.c_double), ("dt", ctypes.c_double),
        ("cb", ctypes.c_double), ("skc", ctypes.c_double), ("nu", ctypes.c_double),
        ("ugal", ctypes.c_double), ("vgal", ctypes.c_double), ("ufree", ctypes.c_double),
        ("emin", ctypes.c_double), ("forcing", ctypes.c_double),
    ]


def make_config(nnx, nny, nnz, dt=1e-3, re_tau=180.0, imodel=3, isurface=6,
                tke_production=0, precision=8, xl=2 * np.pi, yl=np.pi, zl=2.0,
                nu=0.0):
    """Channel configuration: Lx=2pi, Ly=pi, walls at z=0 and z=2, roughness
    z0 = exp(-kappa*B)*h/Re_tau (kappa=0.4, B=5, h=zl/2)."""
    c = LesConfig()
    c.nnx, c.nny, c.nnz = nnx, nny, nnz
    c.imodel, c.isurface, c.tke_production, c.precision = imodel, isurface, tke_production, precision
    c.device = 0
    c.xl, c.yl, c.zl = xl, yl, zl
    c.z0 = float(np.exp(-0.4 * 5.0) * (zl / 2.0) / re_tau)
    c.dt = dt
    c.cb, c.skc, c.nu = 0.0, 1.0, nu
    c.ugal = c.vgal = c.ufree = 0.0
    c.emin, c.forcing = 1e-6, 0.016
    return c


def bulk_velocity(re_tau, utau=np.sqrt(0.016), kappa=0.4, b=5.0):
    """Bulk mean of the log law over the half channel: ub/utau = (ln Re_tau - 1)/kappa + B."""
    return utau * ((np.log(re_tau) - 1.0) / kappa + b)


_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        D = ctypes.POINTER(ctypes.c_double)
        L.orc_create.restype = P
        L.orc_create.argtypes = [ctypes.POINTER(LesConfig), ctypes.c_int]
        L.orc_free.argtypes = [P]
        L.orc_error.restype = ctypes.c_char_p
        L.orc_error.argtypes = [P]
        for name in ("orc_set_fields", "orc_get_fields"):
            getattr(L, name).argtypes = [P, D, D, D, D, D]
        for name in ("orc_set_tendencies", "orc_get_tendencies"):
            getattr(L, name).argtypes = [P, D, D, D, D]
        L.orc_deal_fields.argtypes = [P]
        L.orc_stage.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_step.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_stats.argtypes = [P, D, D]
        L.orc_compmn.argtypes = [P]
        L.orc_spectra.argtypes = [P, ctypes.c_int, ctypes.c_int, D, D]
        L.orc_make_ic.argtypes = [P, ctypes.c_ulonglong, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double]
        L.orc_cfl_dt.restype = ctypes.c_double
        L.orc_cfl_dt.argtypes = [P, ctypes.c_double]
        L.orc_set_dt.argtypes = [P, ctypes.c_double]
        for name in ("orc_xderiv", "orc_yderiv"):
            getattr(L, name).argtypes = [D, D, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        for name in ("orc_expand", "orc_compress", "orc_r2c", "orc_c2r"):
            getattr(L, name).argtypes = [D, D, ctypes.c_int, ctypes.c_int]
        L.orc_deal.argtypes = [D, ctypes.c_int, ctypes.c_int]
        L.orc_dft.argtypes = [D, ctypes.c_int, ctypes.c_int]
        L.orc_tridv.argtypes = [D, ctypes.c_int, ctypes.c_int]
        L.orc_threads.restype = ctypes.c_int
        LL = ctypes.c_longlong
        L.orc_mlp_nparam.restype = ctypes.c_int
        L.orc_mlp_forward.argtypes = [D, D, LL, D, ctypes.c_int]
        L.orc_mlp_loss_grad.restype = ctypes.c_double
        L.orc_mlp_loss_grad.argtypes = [D, D, D, LL, D]
        L.orc_mlp_loss.restype = ctypes.c_double
        L.orc_mlp_loss.argtypes = [D, D, D, LL]
        L.orc_mlp_adam.argtypes = [D, D, D, D, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.orc_set_mlp.argtypes = [P, D, D, ctypes.c_double, ctypes.c_int]
        L.orc_learned_status.argtypes = [P, ctypes.POINTER(ctypes.c_int), D]
        L.orc_learned_reference.argtypes = [P]
        L.orc_learned_reference.restype = ctypes.c_double
        L.orc_learned_raw.argtypes = [P]
        L.orc_learned_raw.restype = ctypes.c_double
        L.orc_set_learned_guard.argtypes = [P, ctypes.c_double]
        L.orc_get_learned.argtypes = [P, D, D, D]
        L.orc_bf16_round.restype = ctypes.c_double
        L.orc_bf16_round.argtypes = [ctypes.c_double]
        _lib = L
    return _lib


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Oracle:
    """One oracle model instance.  Fields are numpy float64 arrays of shape
    (nnz, nny, nnx) (C order == the reference's column-major (x,y,z))."""

    def __init__(self, cfg, real_bytes=8):
        self.cfg = cfg
        self.shape = (cfg.nnz, cfg.nny, cfg.nnx)
        self.h = lib().orc_create(ctypes.byref(cfg), real_bytes)
        if not self.h:
            raise ValueError("oracle rejected the configuration")

    def close(self):
        if self.h:
            lib().orc_free(self.h)
            self.h = None

    __del__ = close

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError("oracle: " + lib().orc_error(self.h).decode())

    def set_fields(self, u=None, v=None, w=None, e=None, p=None):
        c = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w, e, p)]
        self._check(lib().orc_set_fields(self.h, *[_ptr(a) for a in c]))

    def get_fields(self):
        out = [np.zeros(self.shape) for _ in range(5)]
        self._check(lib().orc_get_fields(self.h, *[_ptr(a) for a in out]))
        return dict(zip("uvwep", out))

    def set_tendencies(self, ru=None, rv=None, rw=None, re=None):
        c = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (ru, rv, rw, re)]
        self._check(lib().orc_set_tendencies(self.h, *[_ptr(a) for a in c]))

    def get_tendencies(self):
        out = [np.zeros(self.shape) for _ in range(4)]
        self._check(lib().orc_get_tendencies(self.h, *[_ptr(a) for a in out]))
        return dict(zip(("ru", "rv", "rw", "re"), out))

    def deal_fields(self):
        self._check(lib().orc_deal_fields(self.h))

    def stage(self, it, mnout, istage):
        self._check(lib().orc_stage(self.h, it, int(mnout), istage))

    def step(self, it0=0, nsteps=1, mnout_every=0):
        self._check(lib().orc_step(self.h, it0, nsteps, mnout_every))

    def stats(self):
        mb = np.zeros(19 * self.cfg.nnz)
        sc = np.zeros(5)
        self._check(lib().orc_stats(self.h, _ptr(mb), _ptr(sc)))
        return mb.reshape(self.cfg.nnz, 19).T.copy(), sc

    def compmn(self):
        self._check(lib().orc_compmn(self.h))

    def spectra(self, field, iz):
        n = self.cfg.nnx // 2 + 1
        a, b = np.zeros(n), np.zeros(n)
        self._check(lib().orc_spectra(self.h, field, iz, _ptr(a), _ptr(b)))
        return a, b

    def make_ic(self, seed=12345, ub=None, amp=0.1, utau=np.sqrt(0.016), e0=1e-4, re_tau=180.0):
        if ub is None:
            ub = bulk_velocity(re_tau, utau)
        self._check(lib().orc_make_ic(self.h, seed, ub, amp, utau, e0))

    def cfl_dt(self, cfl=0.5):
        return lib().orc_cfl_dt(self.h, cfl)

    def set_mlp(self, params, norm, re_tau, bf16=True):
        """Attach the learned closure's network (imodel = 5)."""
        self._mlp_keep = (np.ascontiguousarray(params, dtype=np.float64), np.ascontiguousarray(norm, dtype=np.float64))
        self._check(lib().orc_set_mlp(self.h, _ptr(self._mlp_keep[0]), _ptr(self._mlp_keep[1]), re_tau, int(bf16)))

    def learned_divergence(self):
        n = (self.cfg.nnz, self.cfg.nny, self.cfg.nnx)
        a, b, c = np.zeros(n), np.zeros(n), np.zeros(n)
        self._check(lib().orc_get_learned(self.h, _ptr(a), _ptr(b), _ptr(c)))
        return a, b, c

    def learned_status(self):
        used = ctypes.c_int()
        d = np.zeros(1)
        lib().orc_learned_status(self.h, ctypes.byref(used), _ptr(d))
        return used.value, float(d[0])

    def learned_raw(self):
        """Raw network mean dissipation (before the backscatter projection)
        of the last learned stage."""
        return float(lib().orc_learned_raw(self.h))

    def learned_reference(self):
        """Reference (Smagorinsky) mean dissipation of the last learned stage."""
        return float(lib().orc_learned_reference(self.h))

    def set_learned_guard(self, ratio):
        """Factor of the dissipation test against Deardorff (<= 0: off)."""
        lib().orc_set_learned_guard(self.h, float(ratio))

    def set_dt(self, dt):
        lib().orc_set_dt(self.h, dt)


# --- operator-level helpers (FP64) ---
def xderiv(a, length):
    a = np.ascontiguousarray(a, dtype=np.float64)
    n2, n1 = a.shape
    o = np.zeros_like(a)
    lib().orc_xderiv(_ptr(a), _ptr(o), n1, n2, length)
    return o


def yderiv(a, length):
    a = np.ascontiguousarray(a, dtype=np.float64)
    n2, n1 = a.shape
    o = np.zeros_like(a)
    lib().orc_yderiv(_ptr(a), _ptr(o), n1, n2, length)
    return o


def expand(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    ny, nx = a.shape
    o = np.zeros((3 * ny // 2, 3 * nx // 2))
    lib().orc_expand(_ptr(a), _ptr(o), nx, ny)
    return o


def compress(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    nyb, nxb = a.shape
    o = np.zeros((2 * nyb // 3, 2 * nxb // 3))
    lib().orc_compress(_ptr(a), _ptr(o), 2 * nxb // 3, 2 * nyb // 3)
    return o


def deal(a):
    a = np.array(a, dtype=np.float64, order="C")
    ny, nx = a.shape
    lib().orc_deal(_ptr(a), nx, ny)
    return a


def r2c(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    n2, n1 = a.shape
    o = np.zeros((n2, n1 // 2 + 1), dtype=np.complex128)
    lib().orc_r2c(_ptr(a), o.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n1, n2)
    return o


def c2r(z, n1):
    z = np.ascontiguousarray(z, dtype=np.complex128)
    n2 = z.shape[0]
    o = np.zeros((n2, n1))
    lib().orc_c2r(z.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _ptr(o), n1, n2)
    return o


def dft(x, sign=-1):
    x = np.array(x, dtype=np.complex128)
    lib().orc_dft(x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), x.size, sign)
    return x


def tridv(bdar):
    """bdar: float64 array shaped (4, n, ny) in C order == Fortran (ny, n, 4)."""
    b = np.array(bdar, dtype=np.float64, order="C")
    _, n, ny = b.shape
    lib().orc_tridv(_ptr(b), ny, n)
    return b


# ---- learned SGS closure: the FP64 multilayer perceptron (mlp_oracle.h) ----
MLP_NIN, MLP_NHID, MLP_NOUT, MLP_NPARAM = 11, 64, 6, 9478
MLP_NNORM = 2 * MLP_NIN + 2 * MLP_NOUT


def mlp_slices():
    """Offsets of W1, b1, W2, b2, W3, b3, W4, b4 in the flat parameter vector."""
    shapes = [(64, 11), (64,), (64, 64), (64,), (64, 64), (64,), (6, 64), (6,)]
    out, o = [], 0
    for sh in shapes:
        n = int(np.prod(sh))
        out.append((o, sh))
        o += n
    assert o == MLP_NPARAM
    return out


def mlp_init(seed=0, scale=1.0):
    """Seeded parameters with the variance-preserving scale 1/sqrt(fan_in)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(MLP_NPARAM)
    for (o, sh) in mlp_slices():
        if len(sh) == 2:
            p[o:o + sh[0] * sh[1]] = rng.standard_normal(sh[0] * sh[1]) * scale / np.sqrt(sh[1])
        else:
            p[o:o + sh[0]] = rng.standard_normal(sh[0]) * 0.1 * scale
    return p


def mlp_forward(params, x, bf16=False):
    params = np.ascontiguousarray(params, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[0]
    y = np.zeros((n, MLP_NOUT))
    lib().orc_mlp_forward(_ptr(params), _ptr(x), n, _ptr(y), int(bf16))
    return y


def mlp_loss_grad(params, x, t):
    params = np.ascontiguousarray(params, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    t = np.ascontiguousarray(t, dtype=np.float64)
    g = np.zeros(MLP_NPARAM)
    loss = lib().orc_mlp_loss_grad(_ptr(params), _ptr(x), _ptr(t), x.shape[0], _ptr(g))
    return loss, g


def mlp_loss(params, x, t):
    params = np.ascontiguousarray(params, dtype=np.float64)
    return lib().orc_mlp_loss(_ptr(params), _ptr(np.ascontiguousarray(x, dtype=np.float64)),
                              _ptr(np.ascontiguousarray(t, dtype=np.float64)), x.shape[0])


def mlp_adam(params, m, v, g, lr, step, b1=0.9, b2=0.999, eps=1e-8):
    for a in (params, m, v):
        assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    g = np.ascontiguousarray(g, dtype=np.float64)
    lib().orc_mlp_adam(_ptr(params), _ptr(m), _ptr(v), _ptr(g), params.size, lr, b1, b2, eps, step)


def bf16_round(a):
    f = lib().orc_bf16_round
    return np.vectorize(f, otypes=[np.float64])(np.asarray(a, dtype=np.float64))
