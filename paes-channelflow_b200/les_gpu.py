"""Host layer of the B200 LES hot path: ctypes bindings of libles_gpu.so
(include/les_gpu.h) with the reference's per-stage interface.

The reference drives one RK3 stage as (les.F90:254-285)::

    lower; upper; comp1(it, mnout, istart, iend, nm, np, istage)
    comprhs(istart, iend); press(...); comp2(istart, iend)

`LesGpu` exposes the same calls on a device-resident domain (`lower`,
`upper`, `comp1`, `comprhs`, `press`, `comp2`), the fused `stage` and
graph-replayed `step`, and the lifecycle around them (init / upload /
download / stats / spectra / finalize).  Every call goes through the C ABI;
there is no CPU fallback: if the CUDA library or a device is missing, the
constructor raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libles_gpu.so")

LES_OK, LES_EINVAL, LES_ECUDA, LES_ENAN, LES_ETIMEOUT, LES_EUTAU, LES_ENOMEM, LES_ESTATE, LES_ENOTBUILT = range(9)
SGS_DEARDORFF, SGS_SMAG, SGS_LEARNED = 3, 4, 5
PREC_FP64, PREC_MIXED = 8, 4

# RK3 coefficients of les.F90:26-27 (Wray's low-storage scheme)
GAMA = (8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0)
ZETAS = (0.0, 17.0 / 60.0, 5.0 / 12.0)


class LesError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("les_gpu error %d: %s" % (code, msg))
        self.code = code


class LesConfig(ctypes.Structure):
    """Mirror of `les_config` (include/les_gpu.h)."""

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


def channel_config(nnx, nny, nnz, dt=1e-3, re_tau=180.0, imodel=SGS_DEARDORFF, isurface=6,
                   tke_production=0, precision=PREC_FP64, device=0, nu=0.0):
    """Channel of the benchmark configurations: Lx=2pi, Ly=pi, walls at z=0
    and z=2 (half height 1), forcing 0.016 (u_tau = sqrt(0.016)), and Re_tau
    mapped onto the wall-model roughness z0 = exp(-kappa*B) h / Re_tau with
    kappa=0.4, B=5 (the reference has no molecular viscosity)."""
    c = LesConfig()
    c.nnx, c.nny, c.nnz = nnx, nny, nnz
    c.imodel, c.isurface, c.tke_production, c.precision, c.device = imodel, isurface, tke_production, precision, device
    c.xl, c.yl, c.zl = 2 * np.pi, np.pi, 2.0
    c.z0 = float(np.exp(-0.4 * 5.0) * 1.0 / re_tau)
    c.dt = dt
    c.cb, c.skc, c.nu = 0.0, 1.0, nu
    c.ugal = c.vgal = c.ufree = 0.0
    c.emin, c.forcing = 1e-6, 0.016
    return c


def bulk_velocity(re_tau, utau=float(np.sqrt(0.016)), kappa=0.4, b=5.0):
    """Bulk mean of the log law over the half channel: ub/utau = (ln Re_tau - 1)/kappa + B."""
    return utau * ((np.log(re_tau) - 1.0) / kappa + b)


_lib = None


def lib():
    """Load libles_gpu.so (built in this directory); raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise LesError(LES_ENOTBUILT, "libles_gpu.so not built: run `make -C %s`" % HERE)
    L = ctypes.CDLL(LIB_PATH)
    P, I, D, VP = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    H = ctypes.c_void_p
    sig = {
        "les_gpu_default_config": (None, [ctypes.POINTER(LesConfig)]),
        "les_gpu_config_size": (ctypes.c_size_t, []),
        "les_gpu_init": (I, [ctypes.POINTER(LesConfig), ctypes.POINTER(H)]),
        "les_gpu_finalize": (None, [H]),
        "les_gpu_last_error": (ctypes.c_char_p, [H]),
        "les_gpu_upload": (I, [H, VP, VP, VP, VP, VP, I]),
        "les_gpu_download": (I, [H, VP, VP, VP, VP, VP, I]),
        "les_gpu_upload_tendencies": (I, [H, VP, VP, VP, VP, I]),
        "les_gpu_download_tendencies": (I, [H, VP, VP, VP, VP, I]),
        "les_gpu_lower": (I, [H]),
        "les_gpu_upper": (I, [H]),
        "les_gpu_comp1": (I, [H, I, I, I, D, D, D]),
        "les_gpu_comprhs": (I, [H, D]),
        "les_gpu_press": (I, [H]),
        "les_gpu_comp2": (I, [H, D]),
        "les_gpu_stage": (I, [H, I, I, I, D, D, D]),
        "les_gpu_step": (I, [H, I, I, D]),
        "les_gpu_stats": (I, [H, VP, VP]),
        "les_gpu_spectra": (I, [H, I, I, VP, VP]),
        "les_gpu_sync": (I, [H, D]),
        "les_gpu_make_ic": (I, [H, ctypes.c_ulonglong, D, D, D, D]),
        "les_gpu_cfl_dt": (I, [H, D, ctypes.POINTER(D)]),
        "les_gpu_kernel_launches": (ctypes.c_longlong, [H]),
        "les_gpu_profile_stage": (I, [H, I, D, VP, VP, I, ctypes.POINTER(I)]),
        "les_gpu_kernel_name": (I, [VP, ctypes.c_char_p, I]),
        "les_gpu_stream": (VP, [H]),
        "les_op_xderiv": (I, [VP, VP, I, I, I, D, I, VP]),
        "les_op_yderiv": (I, [VP, VP, I, I, I, D, I, VP]),
        "les_op_expand": (I, [VP, VP, I, I, I, I, VP]),
        "les_op_compress": (I, [VP, VP, I, I, I, I, VP]),
        "les_op_deal": (I, [VP, I, I, I, I, VP]),
        "les_op_tridv": (I, [VP, I, I, I, VP]),
        "les_op_last_error": (ctypes.c_char_p, []),
        "les_probe_fma_rate": (I, [I, I, ctypes.POINTER(D)]),
        # learned closure (les_mlp.h)
        "les_mlp_create": (I, [I, ctypes.POINTER(VP)]),
        "les_mlp_destroy": (None, [VP]),
        "les_mlp_last_error": (ctypes.c_char_p, [VP]),
        "les_mlp_set_params": (I, [VP, VP, VP]),
        "les_mlp_get_params": (I, [VP, VP, VP]),
        "les_mlp_set_wait_limit": (I, [VP, ctypes.c_double]),
        "les_mlp_forward": (I, [VP, VP, ctypes.c_longlong, VP, VP]),
        "les_mlp_loss_grad": (I, [VP, VP, VP, ctypes.c_longlong, VP, ctypes.POINTER(D), VP]),
        "les_mlp_adam_step": (I, [VP, VP, VP, ctypes.c_longlong, ctypes.c_float, ctypes.POINTER(D), VP]),
        "les_gpu_set_mlp": (I, [H, VP, D]),
        "les_gpu_learned_status": (I, [H, ctypes.POINTER(I), ctypes.POINTER(D)]),
        "les_gpu_set_learned_guard": (I, [H, D]),
        "les_gpu_learned_reference": (I, [H, ctypes.POINTER(D)]),
        "les_gpu_learned_counts": (I, [H, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
        "les_gpu_learn_filter": (I, [H, I, I, I, VP]),
        "les_gpu_write_field": (I, [H, ctypes.c_char_p, D, I, I]),
        "les_gpu_field_wait": (I, [H]),
        "les_gpu_read_field": (I, [H, ctypes.c_char_p, I, ctypes.POINTER(D)]),
        "les_gpu_regrid": (I, [H, H]),
        "les_gpu_field_header": (I, [ctypes.c_char_p, I, ctypes.POINTER(I), ctypes.POINTER(D)]),
        "les_gpu_learned_features": (I, [H, VP]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    if L.les_gpu_config_size() != ctypes.sizeof(LesConfig):
        raise LesError(LES_EINVAL, "les_config layout mismatch between header and bindings")
    _lib = L
    return L


def exported_symbols():
    """Entry points declared in include/les_gpu.h and include/les_mlp.h."""
    import re
    names = set()
    for h in ("les_gpu.h", "les_mlp.h"):
        text = open(os.path.join(os.path.dirname(HERE), "include", h)).read()
        names.update(re.findall(r"\b(les_(?:gpu|op|mlp)_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return int(a)


class LesGpu:
    """One device-resident channel domain (one handle, one CUDA stream).

    Field arrays are (nnz, nny, nnx) C-ordered numpy arrays (== the
    reference's column-major (nnx, nny, nnz) levels 1..nnz), float64 or
    float32, or pinned torch tensors for asynchronous host transfers."""

    def __init__(self, cfg):
        self.cfg = cfg
        self.shape = (cfg.nnz, cfg.nny, cfg.nnx)
        h = ctypes.c_void_p()
        rc = lib().les_gpu_init(ctypes.byref(cfg), ctypes.byref(h))
        if rc != LES_OK:
            raise LesError(rc, lib().les_gpu_last_error(None).decode())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().les_gpu_finalize(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != LES_OK:
            raise LesError(rc, lib().les_gpu_last_error(self.h).decode())

    @staticmethod
    def _rb(arrs):
        for a in arrs:
            if a is None:
                continue
            if isinstance(a, np.ndarray):
                return a.dtype.itemsize
            return a.element_size()
        return 8

    # lifecycle / transfer
    def upload(self, u=None, v=None, w=None, e=None, p=None):
        arrs = [None if a is None else (np.ascontiguousarray(a) if isinstance(a, np.ndarray) else a)
                for a in (u, v, w, e, p)]
        self._check(lib().les_gpu_upload(self.h, *[_ptr(a) for a in arrs], self._rb(arrs)))

    def download(self, dtype=np.float64, fields="uvwep"):
        out = {k: np.zeros(self.shape, dtype=dtype) for k in fields}
        self._check(lib().les_gpu_download(self.h, *[_ptr(out.get(k)) for k in "uvwep"], np.dtype(dtype).itemsize))
        return out

    def download_into(self, u=None, v=None, w=None, e=None, p=None):
        arrs = (u, v, w, e, p)
        self._check(lib().les_gpu_download(self.h, *[_ptr(a) for a in arrs], self._rb(arrs)))

    def upload_tendencies(self, ru=None, rv=None, rw=None, re=None):
        arrs = [None if a is None else np.ascontiguousarray(a) for a in (ru, rv, rw, re)]
        self._check(lib().les_gpu_upload_tendencies(self.h, *[_ptr(a) for a in arrs], self._rb(arrs)))

    def download_tendencies(self, dtype=np.float64):
        out = {k: np.zeros(self.shape, dtype=dtype) for k in ("ru", "rv", "rw", "re")}
        self._check(lib().les_gpu_download_tendencies(self.h, *[_ptr(out[k]) for k in ("ru", "rv", "rw", "re")],
                                                      np.dtype(dtype).itemsize))
        return out

    # the reference's per-stage routines
    def lower(self):
        self._check(lib().les_gpu_lower(self.h))

    def upper(self):
        self._check(lib().les_gpu_upper(self.h))

    def comp1(self, it, mnout, istage, dtab1, dtab2, xkmax):
        self._check(lib().les_gpu_comp1(self.h, it, int(mnout), istage, dtab1, dtab2, xkmax))

    def comprhs(self, dtabm):
        self._check(lib().les_gpu_comprhs(self.h, dtabm))

    def press(self):
        self._check(lib().les_gpu_press(self.h))

    def comp2(self, dtab1):
        self._check(lib().les_gpu_comp2(self.h, dtab1))

    def stage(self, it, mnout, istage, dt=None):
        dt = self.cfg.dt if dt is None else dt
        dz = self.cfg.zl / self.cfg.nnz
        self._check(lib().les_gpu_stage(self.h, it, int(mnout), istage, dt * GAMA[istage - 1],
                                        dt * ZETAS[istage - 1], dz * dz / dt / 5.0))

    def stage_split(self, it, mnout, istage, dt=None):
        """One stage through the six reference-named entry points."""
        dt = self.cfg.dt if dt is None else dt
        dz = self.cfg.zl / self.cfg.nnz
        dtab1, dtab2 = dt * GAMA[istage - 1], dt * ZETAS[istage - 1]
        self.lower()
        self.upper()
        self.comp1(it, mnout, istage, dtab1, dtab2, dz * dz / dt / 5.0)
        self.comprhs(1.0 / dtab1)
        self.press()
        self.comp2(dtab1)

    def step(self, it=1, mnout=False, dt=None):
        dt = self.cfg.dt if dt is None else dt
        self._check(lib().les_gpu_step(self.h, it, int(mnout), dt))

    def set_mlp(self, mlp, re_tau):
        """Attach the learned closure's network (configuration imodel = 5);
        mlp=None detaches."""
        self._mlp = mlp
        self._check(lib().les_gpu_set_mlp(self.h, mlp.h if mlp is not None else None, re_tau))

    def learned_status(self):
        """(used, dissipation) of the last stage (synchronising)."""
        used = ctypes.c_int()
        d = ctypes.c_double()
        self._check(lib().les_gpu_learned_status(self.h, ctypes.byref(used), ctypes.byref(d)))
        return used.value, d.value

    def set_learned_guard(self, ratio):
        """Factor of the fallback test against the reference (Smagorinsky-Lilly,
        C_s = 0.17) dissipation (default 4; <= 0 keeps only the sign test)."""
        self._check(lib().les_gpu_set_learned_guard(self.h, float(ratio)))

    def learned_reference(self):
        """Reference (Smagorinsky) mean dissipation of the last learned
        stage (synchronising)."""
        d = ctypes.c_double()
        self._check(lib().les_gpu_learned_reference(self.h, ctypes.byref(d)))
        return d.value

    def learned_counts(self):
        """(stages evaluated, stages that used the network) since set_mlp."""
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(lib().les_gpu_learned_counts(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def learn_filter(self, fxy, fz, with_model=True):
        """Filtered coarse fields of the current state: float64 CUDA tensor
        (9, nnz/fz, nny/fxy, nnx/fxy) = u, v, w, tau11, tau22, tau33, tau12,
        tau13, tau23 (with_model: tau includes the filtered Deardorff stress
        of this run)."""
        import torch
        c = self.cfg
        out = torch.empty((9, c.nnz // fz, c.nny // fxy, c.nnx // fxy), dtype=torch.float64,
                          device="cuda:%d" % c.device)
        self._check(lib().les_gpu_learn_filter(self.h, fxy, fz, int(with_model), out.data_ptr()))
        return out

    def learned_features(self):
        """Raw network inputs at every cell centre: float32 CUDA tensor
        (N, 16), columns 0..10 the inputs, column 11 Delta |G|."""
        import torch
        c = self.cfg
        out = torch.empty((c.nnx * c.nny * c.nnz, 16), dtype=torch.float32, device="cuda:%d" % c.device)
        self._check(lib().les_gpu_learned_features(self.h, out.data_ptr()))
        return out

    def write_field(self, path, time=0.0, real_bytes=8, background=False):
        """Restart file in the reference's .field layout (read_write.f90)."""
        self._check(lib().les_gpu_write_field(self.h, os.fsencode(path), time, real_bytes, int(background)))

    def field_wait(self):
        self._check(lib().les_gpu_field_wait(self.h))

    def read_field(self, path, real_bytes=8):
        """Load a restart file of this grid; returns its start time."""
        t = ctypes.c_double()
        self._check(lib().les_gpu_read_field(self.h, os.fsencode(path), real_bytes, ctypes.byref(t)))
        return t.value

    def regrid_from(self, src):
        """This handle's state := src's state moved onto this grid (redim.f90
        followed by the restart's deal); see les_gpu_regrid."""
        self._check(lib().les_gpu_regrid(self.h, src.h))

    def sync(self, timeout_s=60.0):
        self._check(lib().les_gpu_sync(self.h, timeout_s))

    # diagnostics
    def stats(self):
        mb = np.zeros(19 * self.cfg.nnz)
        sc = np.zeros(5)
        self._check(lib().les_gpu_stats(self.h, _ptr(mb), _ptr(sc)))
        return mb.reshape(self.cfg.nnz, 19).T.copy(), sc

    def spectra(self, field, iz):
        n = self.cfg.nnx // 2 + 1
        a, b = np.zeros(n), np.zeros(n)
        self._check(lib().les_gpu_spectra(self.h, field, iz, _ptr(a), _ptr(b)))
        return a, b

    def make_ic(self, seed=12345, ub=None, amp=0.1, utau=float(np.sqrt(0.016)), e0=1e-4, re_tau=180.0):
        if ub is None:
            ub = bulk_velocity(re_tau, utau)
        self._check(lib().les_gpu_make_ic(self.h, seed, ub, amp, utau, e0))

    def cfl_dt(self, cfl=0.5):
        d = ctypes.c_double()
        self._check(lib().les_gpu_cfl_dt(self.h, cfl, ctypes.byref(d)))
        return d.value

    def kernel_launches(self):
        return lib().les_gpu_kernel_launches(self.h)

    def stream_handle(self):
        """The handle's cudaStream_t as an integer (torch.cuda.ExternalStream)."""
        return lib().les_gpu_stream(self.h) or 0

    def profile_stage(self, istage=2, dt=None):
        """Run one stage eagerly with CUDA events between the kernels; returns
        [(kernel name, ms)] in launch order (advances the state)."""
        dt = self.cfg.dt if dt is None else dt
        cap = 64
        ms = (ctypes.c_double * cap)()
        fn = (ctypes.c_void_p * cap)()
        n = ctypes.c_int()
        self._check(lib().les_gpu_profile_stage(self.h, istage, dt, ms, fn, cap, ctypes.byref(n)))
        return [(kernel_name(fn[i]), ms[i]) for i in range(min(n.value, cap))]


def kernel_name(addr):
    """Short name of a kernel from its host stub address: the device name
    (les_gpu_kernel_name) lightly demangled from les::k_<name><T, N>."""
    import re
    buf = ctypes.create_string_buffer(1024)
    if not addr or lib().les_gpu_kernel_name(ctypes.c_void_p(addr), buf, len(buf)) != LES_OK:
        return hex(addr or 0)
    raw = buf.value.decode()
    m = re.match(r"_ZN3les(?:12_GLOBAL__N_1)?L?(\d+)(k_\w+)", raw)
    if not m:
        return raw
    n = int(m.group(1))
    name = m.group(2)[:n]
    tail = raw[m.end(1) + n:]
    tp = "f64" if tail.startswith("Id") else ("f32" if tail.startswith("If") else "")
    num = re.match(r"I[df]Li(\d+)", tail)
    return name + ("<%s%s>" % (tp, "," + num.group(1) if num else "") if tp else "")


# --- operator-level entry points on torch CUDA tensors (float64 or float32) ---
def _op_check(rc):
    if rc != LES_OK:
        raise LesError(rc, lib().les_op_last_error().decode())


def _stream(t):
    import torch
    return torch.cuda.current_stream(t.device).cuda_stream


def xderiv(a, length, out=None):
    """xderiv (filter_fftw.f90:138-187) of (howmany, n2, n1) planes."""
    out = a.new_empty(a.shape) if out is None else out
    n2, n1 = a.shape[-2], a.shape[-1]
    howmany = a.numel() // (n1 * n2)
    _op_check(lib().les_op_xderiv(a.data_ptr(), out.data_ptr(), n1, n2, howmany, length, a.element_size(), _stream(a)))
    return out


def yderiv(a, length, out=None):
    """yderiv (filter_fftw.f90:194-248) of (howmany, n2, n1) planes."""
    out = a.new_empty(a.shape) if out is None else out
    n2, n1 = a.shape[-2], a.shape[-1]
    howmany = a.numel() // (n1 * n2)
    _op_check(lib().les_op_yderiv(a.data_ptr(), out.data_ptr(), n1, n2, howmany, length, a.element_size(), _stream(a)))
    return out


def expand(a):
    """expand (filter_fftw.f90:254-278): (.., ny, nx) -> (.., 3ny/2, 3nx/2)."""
    ny, nx = a.shape[-2], a.shape[-1]
    howmany = a.numel() // (nx * ny)
    out = a.new_empty(a.shape[:-2] + (3 * ny // 2, 3 * nx // 2))
    _op_check(lib().les_op_expand(a.data_ptr(), out.data_ptr(), nx, ny, howmany, a.element_size(), _stream(a)))
    return out


def compress(a):
    """compress (filter_fftw.f90:285-308): (.., 3ny/2, 3nx/2) -> (.., ny, nx)."""
    nyb, nxb = a.shape[-2], a.shape[-1]
    nx, ny = 2 * nxb // 3, 2 * nyb // 3
    howmany = a.numel() // (nxb * nyb)
    out = a.new_empty(a.shape[:-2] + (ny, nx))
    _op_check(lib().les_op_compress(a.data_ptr(), out.data_ptr(), nx, ny, howmany, a.element_size(), _stream(a)))
    return out


def deal(a):
    """deal (filter_fftw.f90:316-329), in place on a copy."""
    out = a.clone()
    ny, nx = a.shape[-2], a.shape[-1]
    _op_check(lib().les_op_deal(out.data_ptr(), nx, ny, a.numel() // (nx * ny), a.element_size(), _stream(a)))
    return out


def tridv(bdar):
    """tridv (tridv.f90:1-55) on a float64 CUDA tensor shaped (4, n, ny)."""
    out = bdar.clone()
    _, n, ny = out.shape
    _op_check(lib().les_op_tridv(out.data_ptr(), ny, n, 8, _stream(out)))
    return out


# --- learned closure: the perceptron (les_mlp.h) ---
MLP_NIN, MLP_NOUT, MLP_NPARAM, MLP_NNORM = 11, 6, 9478, 34


class Mlp:
    """The learned closure's network on one device.  Samples are torch CUDA
    tensors: features bfloat16 (n, 16) normalised (columns 11..15 zero),
    outputs / targets float32 (n, 8) (columns 6, 7 unused)."""

    def __init__(self, params=None, norm=None, device=0):
        h = ctypes.c_void_p()
        rc = lib().les_mlp_create(device, ctypes.byref(h))
        if rc != LES_OK:
            raise LesError(rc, "les_mlp_create failed")
        self.h = h
        self.device = device
        if params is not None:
            self.set_params(params, norm)

    def close(self):
        if getattr(self, "h", None):
            lib().les_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != LES_OK:
            raise LesError(rc, lib().les_mlp_last_error(self.h).decode())

    def set_params(self, params, norm=None):
        p = np.ascontiguousarray(params, dtype=np.float32)
        if norm is None:
            norm = np.concatenate([np.zeros(MLP_NIN), np.ones(MLP_NIN), np.ones(MLP_NOUT), np.zeros(MLP_NOUT)])
        nm = np.ascontiguousarray(norm, dtype=np.float32)
        assert p.size == MLP_NPARAM and nm.size == MLP_NNORM
        self._check(lib().les_mlp_set_params(self.h, p.ctypes.data, nm.ctypes.data))

    def get_params(self):
        p = np.zeros(MLP_NPARAM, dtype=np.float32)
        nm = np.zeros(MLP_NNORM, dtype=np.float32)
        self._check(lib().les_mlp_get_params(self.h, p.ctypes.data, nm.ctypes.data))
        return p, nm

    def set_wait_limit(self, seconds):
        """Limit of each tensor-core MMA wait of this network's kernels
        (les_mlp_set_wait_limit); default 1 s."""
        self._check(lib().les_mlp_set_wait_limit(self.h, ctypes.c_double(seconds)))

    def forward(self, feat):
        import torch
        n = feat.shape[0]
        y = torch.empty((n, 8), dtype=torch.float32, device=feat.device)
        self._check(lib().les_mlp_forward(self.h, feat.data_ptr(), n, y.data_ptr(), _stream(feat)))
        return y

    def loss_grad(self, feat, target):
        import torch
        g = torch.empty(MLP_NPARAM, dtype=torch.float32, device=feat.device)
        loss = ctypes.c_double()
        self._check(lib().les_mlp_loss_grad(self.h, feat.data_ptr(), target.data_ptr(), feat.shape[0],
                                            g.data_ptr(), ctypes.byref(loss), _stream(feat)))
        return loss.value, g

    def adam_step(self, feat, target, lr=1e-3, want_loss=False):
        loss = ctypes.c_double()
        self._check(lib().les_mlp_adam_step(self.h, feat.data_ptr(), target.data_ptr(), feat.shape[0], lr,
                                            ctypes.byref(loss) if want_loss else None, _stream(feat)))
        return loss.value if want_loss else None


def to_feat(x):
    """(n, 11) array of normalised features -> bfloat16 (n, 16) CUDA tensor."""
    import torch
    x = torch.as_tensor(np.asarray(x), dtype=torch.float32)
    f = torch.zeros((x.shape[0], 16), dtype=torch.float32)
    f[:, :MLP_NIN] = x
    return f.to(torch.bfloat16).cuda()


def to_target(t):
    """(n, 6) array -> float32 (n, 8) CUDA tensor."""
    import torch
    t = torch.as_tensor(np.asarray(t), dtype=torch.float32)
    o = torch.zeros((t.shape[0], 8), dtype=torch.float32)
    o[:, :MLP_NOUT] = t
    return o.cuda()


def regrid_field(path_in, path_out, nnx, nny, nnz, real_bytes=8, precision=PREC_FP64, device=0):
    """The reference's redim program on restart files: read path_in (any
    grid), regrid its state onto nnx x nny x nnz on the GPU and write
    path_out with the input's time, lengths, dt and z0."""
    dims, hdr = field_header(path_in, real_bytes)
    cfgs = []
    for n in (dims, (nnx, nny, nnz)):
        c = channel_config(*n, dt=hdr["dt"], precision=precision, device=device)
        c.xl, c.yl, c.zl, c.z0 = hdr["xl"], hdr["yl"], hdr["zl"], hdr["z0"]
        cfgs.append(c)
    src, dst = LesGpu(cfgs[0]), LesGpu(cfgs[1])
    try:
        t = src.read_field(path_in, real_bytes)
        dst.regrid_from(src)
        dst.write_field(path_out, time=t, real_bytes=real_bytes)
    finally:
        dst.close()
        src.close()


def field_header(path, real_bytes=8):
    """(nnx, nny, nnz), dict of the 13 header values of a restart file."""
    dims = (ctypes.c_int * 3)()
    hdr = (ctypes.c_double * 13)()
    rc = lib().les_gpu_field_header(os.fsencode(path), real_bytes, dims, hdr)
    if rc != LES_OK:
        raise LesError(rc, lib().les_gpu_last_error(None).decode())
    keys = ("time", "xl", "yl", "zl", "dt", "z0", "utau", "divgls", "fcor", "ugtop", "ugbot", "vgtop", "vgbot")
    return tuple(dims), dict(zip(keys, list(hdr)))


def fma_rate(real_bytes, device=0):
    """Vector FMA throughput of the device in flop/s (les_probe_fma_rate)."""
    r = ctypes.c_double()
    rc = lib().les_probe_fma_rate(real_bytes, device, ctypes.byref(r))
    if rc != LES_OK:
        raise LesError(rc, "les_probe_fma_rate failed")
    return r.value
