"""Python front end of the test oracle (TEST INFRASTRUCTURE ONLY).

Two CPU backends with one interface:

* ``ref``   — the reference's own C functions compiled in place from the
              reference tree (``oracle/_ref/libdenise_ref.so``, built by
              ``oracle/Makefile``; ``libdenise_ref_fast.so`` is the -O3 timing
              build used only as the CPU baseline),
* ``port``  — this repository's C restatement (``oracle/_ref/libdsh_oracle.so``),
              in FP32 (``fp64=False``, bit-identical to ``ref``) or FP64.

Array conventions: grid fields are numpy float32 ``[NY, NX]``; traces
``[ntr, NT]``; source tables ``[8, nsrc]`` (grid x, grid y, 0, tshift, fc, amp,
angle, type); receiver tables ``[2, ntr]`` int32 grid indices (1-based, as the
reference's ``recpos``).  Only tests, the smoke check and the CPU-baseline leg
of bench.py import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
# the reference source tree: $DSH_REFERENCE, by default a directory named
# "reference" next to this repository's root
DEFAULT_REFERENCE = os.path.abspath(os.path.join(HERE, "..", "..", "reference"))

FIELD = {"vy": 0, "sxy": 1, "syz": 2, "vyp1": 3, "uy": 4, "uyx": 5, "uip": 6, "ujp": 7, "rho": 8, "vs": 9,
         "fipjp": 10, "f": 11, "Ws": 12, "Wr": 13, "We": 14, "g_u": 15, "g_rho": 16, "hess_u": 17,
         "hess_rho": 18, "taus": 19, "tausipjp": 20}
PML = ["K_x", "a_x", "b_x", "K_x_half", "a_x_half", "b_x_half", "K_y", "a_y", "b_y", "K_y_half", "a_y_half",
       "b_y_half", "d_x", "d_x_half", "d_y", "d_y_half"]


class Params(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("nx", "ny", "nt", "fdorder", "maxrelerror", "fw", "free_surf", "l",
                                      "quellart", "eprecond")] + \
               [(n, C.c_float) for n in ("dh", "dt", "damping", "fpml", "npower", "k_max_pml")] + \
               [("fl", C.c_float * 8)]


@dataclass
class Model:
    """One SH model and its time-stepping settings (mirrors the reference's .inp keys)."""
    nx: int
    ny: int
    nt: int
    dh: float
    dt: float
    vs: np.ndarray
    rho: np.ndarray
    qs: np.ndarray | None = None
    fdorder: int = 4
    maxrelerror: int = 1
    fw: int = 20
    free_surf: int = 1
    l: int = 0
    fl: tuple = ()
    quellart: int = 1
    eprecond: int = 1
    damping: float | None = None
    fpml: float = 30.0
    npower: float = 4.0
    k_max_pml: float = 1.0
    extra: dict = field(default_factory=dict)

    def params(self) -> Params:
        p = Params()
        p.nx, p.ny, p.nt = self.nx, self.ny, self.nt
        p.fdorder, p.maxrelerror, p.fw, p.free_surf = self.fdorder, self.maxrelerror, self.fw, self.free_surf
        p.l, p.quellart, p.eprecond = self.l, self.quellart, self.eprecond
        p.dh, p.dt = self.dh, self.dt
        p.damping = float(self.damping if self.damping is not None else float(np.max(self.vs)))
        p.fpml, p.npower, p.k_max_pml = self.fpml, self.npower, self.k_max_pml
        for i, v in enumerate(self.fl[:8]):
            p.fl[i] = v
        return p


def build(reference: str | None = None, quiet: bool = True) -> None:
    """Build the oracle libraries (the reference part only if its tree exists)."""
    targets = ["port"]
    ref = reference or os.environ.get("DSH_REFERENCE", DEFAULT_REFERENCE)
    if os.path.isdir(os.path.join(ref, "src")):
        targets.insert(0, "ref")
    out = subprocess.run(["make", "-C", HERE, f"REF={ref}", *targets], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


def available(kind: str) -> bool:
    name = {"ref": "libdenise_ref.so", "ref_fast": "libdenise_ref_fast.so", "port": "libdsh_oracle.so"}[kind]
    return os.path.exists(os.path.join(REF_DIR, name))


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a, t=C.c_float):
    return a.ctypes.data_as(C.POINTER(t))


class Oracle:
    """A CPU oracle session for one model (one process-wide session per backend)."""

    def __init__(self, model: Model, kind: str = "ref", fp64: bool = False, fd12_compat: bool = True,
                 grad_q: bool = False):
        self.kind, self.fp64, self.m = kind, fp64, model
        lib = {"ref": "libdenise_ref.so", "ref_fast": "libdenise_ref_fast.so", "port": "libdsh_oracle.so"}[kind]
        path = os.path.join(REF_DIR, lib)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        self.pre = "refh_" if kind.startswith("ref") else "dsho_"
        if fp64 and not kind == "port":
            raise ValueError("FP64 runs exist only for the restatement")
        self._fn("init").restype = C.c_int
        self._fn("residual").argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]
        vs, rho = _f32(model.vs), _f32(model.rho)
        qs = _f32(model.qs) if model.qs is not None else np.ones_like(vs)
        self._keep = (vs, rho, qs)
        self.params = model.params()
        if grad_q and self.pre != "dsho_":
            raise ValueError("the Qs gradient exists only in the restatement (the reference has none)")
        if self.pre == "dsho_":
            self.lib.dsho_set_fd12_compat(int(fd12_compat))
            self.lib.dsho_set_grad_q(int(grad_q))
            rc = self.lib.dsho_init(C.byref(self.params), _ptr(vs), _ptr(rho), _ptr(qs), int(fp64))
        else:
            rc = self.lib.refh_init(C.byref(self.params), _ptr(vs), _ptr(rho), _ptr(qs))
        if rc != 0:
            raise ValueError(f"oracle init failed ({rc})")
        self.ntr = 0

    def _fn(self, name):
        return getattr(self.lib, self.pre + name)

    # --- coefficients -------------------------------------------------
    def hc(self):
        out = np.zeros(7, np.float32)
        self._fn("get_hc")(_ptr(out))
        return out

    def cnorm(self):
        out = np.zeros(2, np.float32)
        self._fn("get_cnorm")(_ptr(out))
        return out

    def pml(self, name):
        out = np.zeros(2 * self.m.fw, np.float32)
        rc = self._fn("get_pml")(PML.index(name), _ptr(out))
        if rc != 0:
            raise ValueError(name)
        return out

    def sls(self):
        outs = [np.zeros(max(self.m.l, 1), np.float32) for _ in range(4)]
        self._fn("get_sls")(*[_ptr(o) for o in outs])
        return [o[: self.m.l] for o in outs]

    def field(self, name, l: int | None = None, f64: bool = False):
        code = FIELD[name] if l is None else {"r": 100, "q": 200, "dip": 300, "d": 400}[name] + l
        if f64:
            out = np.zeros((self.m.ny, self.m.nx), np.float64)
            rc = self.lib.dsho_get_field_f64(code, _ptr(out, C.c_double))
        else:
            out = np.zeros((self.m.ny, self.m.nx), np.float32)
            rc = self._fn("get_field")(code, _ptr(out))
        if rc != 0:
            raise ValueError(name)
        return out

    def psi(self, which):
        idx = ["psi_sxy_x", "psi_vyx", "psi_syz_y", "psi_vyy"].index(which)
        shape = (self.m.ny, 2 * self.m.fw) if idx < 2 else (2 * self.m.fw, self.m.nx)
        out = np.zeros(shape, np.float32)
        rc = self._fn("get_psi")(idx, _ptr(out))
        if rc != 0:
            raise ValueError(which)
        return out

    def wavelet(self, srcpos8):
        sp = _f32(srcpos8)
        nsrc = sp.shape[1]
        out = np.zeros((nsrc, self.m.nt), np.float32)
        self._fn("wavelet")(nsrc, _ptr(sp), _ptr(out))
        return out

    # --- time loops ---------------------------------------------------
    def forward(self, srcpos8, recpos, signals=None, nsteps=None, store=False, hessian=False):
        sp = _f32(srcpos8)
        rp = np.ascontiguousarray(recpos, dtype=np.int32)
        nsrc, ntr = sp.shape[1], rp.shape[1]
        nsteps = self.m.nt if nsteps is None else nsteps
        seis = np.zeros((max(ntr, 1), self.m.nt), np.float32)
        sig = _f32(signals) if signals is not None else None
        self._keep_fwd = (sp, rp, sig)
        if self.fp64:
            s64 = np.zeros((max(ntr, 1), self.m.nt), np.float64)
            rc = self.lib.dsho_forward_f64(nsrc, _ptr(sp), _ptr(sig) if sig is not None else None, ntr,
                                           _ptr(rp, C.c_int), nsteps, int(store), int(hessian), _ptr(s64, C.c_double))
            seis = s64
        else:
            rc = self._fn("forward")(nsrc, _ptr(sp), _ptr(sig) if sig is not None else None, ntr,
                                     _ptr(rp, C.c_int), nsteps, int(store), int(hessian), _ptr(seis))
        if rc != 0:
            raise RuntimeError("oracle forward failed")
        self.ntr = ntr
        return seis[:ntr]

    def set_lnorm(self, lnorm):
        """Misfit norm of residual() (calc_res.c LNORM 1..5; default 2)."""
        if self._fn("set_lnorm")(int(lnorm)) != 0:
            raise ValueError("LNORM must be 1..5")

    def residual(self, obs):
        ob = _f32(obs)
        res = np.zeros((self.ntr, self.m.nt), np.float32)
        l2 = C.c_double(0.0)
        rc = self._fn("residual")(ob.ctypes.data, res.ctypes.data, C.byref(l2))
        if rc != 0:
            raise RuntimeError("oracle residual failed")
        return res, l2.value

    def adjoint(self, adj=None, nsteps=None):
        nsteps = self.m.nt if nsteps is None else nsteps
        a = _f32(adj) if adj is not None else None
        rc = self._fn("adjoint")(_ptr(a) if a is not None else None, nsteps)
        if rc != 0:
            raise RuntimeError("oracle adjoint failed")

    def eprecond_scale(self):
        self._fn("eprecond_scale")()

    def convert(self, wu, wrho):
        a, b = _f32(wu), _f32(wrho)
        gv, gr = np.zeros_like(a), np.zeros_like(b)
        self._fn("convert")(_ptr(a), _ptr(b), _ptr(gv), _ptr(gr))
        return gv, gr

    def grad_q(self):
        """dJ/dQs (J = sum res^2) of the last shot's adjoint, float64 [NY, NX]
        (restatement only; the reference computes no Q gradient)."""
        out = np.zeros((self.m.ny, self.m.nx), np.float64)
        if self.lib.dsho_get_grad_q(_ptr(out, C.c_double)) != 0:
            raise RuntimeError("no Qs gradient (needs L > 0 and grad_q=True)")
        return out

    def hessian_out(self):
        hv = np.zeros((self.m.ny, self.m.nx), np.float32)
        hr = np.zeros_like(hv)
        self._fn("hessian_out")(_ptr(hv), _ptr(hr))
        return hv, hr

    def psource(self, nt, sxx, syy, srcpos8, signals):
        a, b, sp, sig = _f32(sxx).copy(), _f32(syy).copy(), _f32(srcpos8), _f32(signals)
        self._fn("psource")(nt, _ptr(a), _ptr(b), sp.shape[1], _ptr(sp), _ptr(sig))
        return a, b

    def shot_gradient(self, srcpos8, recpos, obs, signals=None, nsteps=None, lnorm=None):
        """Forward + residual + adjoint + eprecond scaling for one shot (denise.c:875-1694).

        Returns dict(seis, res, l2, g_u, g_rho, Ws, Wr, We)."""
        if lnorm is not None:
            self.set_lnorm(lnorm)
        seis = self.forward(srcpos8, recpos, signals=signals, nsteps=nsteps, store=True)
        res, l2 = self.residual(obs)
        self.adjoint(nsteps=nsteps)
        out = {"seis": seis, "res": res, "l2": l2, "Ws": self.field("Ws"), "Wr": self.field("Wr")}
        self.eprecond_scale()
        out.update(g_u=self.field("g_u"), g_rho=self.field("g_rho"), We=self.field("We"))
        return out

    def close(self):
        self._fn("free")()


def gauss_filter_size(wd_damp, c_vs, fc_end, dh):
    """SPATFILTER=3 filter length (src/gauss_filt.c:58-69), from the restatement."""
    lib = C.CDLL(os.path.join(REF_DIR, "libdsh_oracle.so"))
    lib.dsho_gauss_filter_size.argtypes = [C.c_float] * 4
    return int(lib.dsho_gauss_filter_size(wd_damp, c_vs, fc_end, dh))


def gauss_filt(grad, filt):
    """SPATFILTER=3 Gaussian smoothing of a [ny, nx] gradient (src/gauss_filt.c), restatement."""
    lib = C.CDLL(os.path.join(REF_DIR, "libdsh_oracle.so"))
    g = _f32(grad)
    out = np.empty_like(g)
    ny, nx = g.shape
    if lib.dsho_gauss_filt(nx, ny, int(filt), _ptr(g), _ptr(out)) != 0:
        raise ValueError("gauss_filt failed")
    return out


def timedomain_filt(data, dt, fc, order, method):
    """The reference's Butterworth trace filter (src/timedomain_filt.c + libcseife), data [ntr, ns]."""
    lib = C.CDLL(os.path.join(REF_DIR, "libdenise_ref.so"))
    lib.refh_timedomain_filt.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int]
    d = _f32(data).copy()
    ntr, ns = d.shape
    lib.refh_timedomain_filt(d.ctypes.data, ntr, ns, dt, fc, order, method)
    return d


def pcg(g_new, g_old, dir, nx, ny):
    """The reference's PCG direction update (src/PCG.c, Polak-Ribiere with
    reset): vectors of nclass*nx*ny floats, each class x-major as
    src/store_PCG_SH.c stores it.  Returns the new direction."""
    lib = C.CDLL(os.path.join(REF_DIR, "libdenise_ref.so"))
    lib.refh_pcg.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    a, b = _f32(g_new).ravel(), _f32(g_old).ravel()
    d = _f32(dir).ravel().copy()
    nclass = a.size // (nx * ny)
    lib.refh_pcg(nx, ny, nclass, a.ctypes.data, b.ctypes.data, d.ctypes.data)
    return d


def pcg_port(g_new, g_old, dir, nclass, beta_kind):
    """Restatement of src/PCG.c:25-102 for every beta choice (the reference
    compiles only Polak-Ribiere): float32 sums in vector order, one Python
    step per element, so only for small vectors."""
    f = np.float32
    a = _f32(g_new).ravel().reshape(nclass, -1)
    b = _f32(g_old).ravel().reshape(nclass, -1)
    d = _f32(dir).ravel().reshape(nclass, -1).copy()
    betas = []
    for k in range(nclass):
        num, den = f(0), f(0)
        for x, y, z in zip(a[k], b[k], d[k]):
            if beta_kind == 1:
                num, den = f(num + x * x), f(den + y * y)
            elif beta_kind == 2:
                num, den = f(num + x * f(x - y)), f(den + y * y)
            elif beta_kind == 3:
                num, den = f(num + f(-x) * f(x - y)), f(den + z * f(x - y))
            else:
                num, den = f(num + f(-x) * x), f(den + z * f(x - y))
        beta = f(num / den) if den != 0 else f(0)
        if beta_kind == 2 and beta < 0:
            beta = f(0)
        betas.append(beta)
        d[k] = a[k] + beta * d[k]
    return d.ravel(), np.array(betas, np.float32)


def taper(g, sws, dh, gradt=(0, 0, 0, 0), srtshape=1, srtradius=5.0, filtsize=1, src_xy=None, recpos=None,
          shot=0, file_vals=None):
    """The reference's gradient taper (src/taper_grad.c; shot = k >= 1:
    src/taper_grad_shot.c for source k) applied to g [ny, nx].  Returns
    (tapered g, coefficient field).  Files the reference writes or reads
    (its coefficient files, taper.bin for sws 5/6) go to a temporary
    directory."""
    import tempfile

    lib = C.CDLL(os.path.join(REF_DIR, "libdenise_ref.so"))
    lib.refh_taper.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_void_p, C.c_int,
                               C.c_float, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    out = _f32(g).copy()
    ny, nx = out.shape
    tc = np.zeros_like(out)
    sxy = _f32(src_xy if src_xy is not None else np.zeros((2, 0)))
    rp = np.ascontiguousarray(recpos if recpos is not None else np.zeros((2, 0)), np.int32)
    gt = np.ascontiguousarray(gradt, np.int32)
    with tempfile.TemporaryDirectory() as d:
        if file_vals is not None:
            _f32(file_vals).tofile(os.path.join(d, "taper.bin"))
        rc = lib.refh_taper(d.encode(), sws, shot, nx, ny, dh, gt.ctypes.data, srtshape, srtradius, filtsize,
                            sxy.shape[1], sxy.ctypes.data, rp.shape[1], rp.ctypes.data, out.ctypes.data,
                            tc.ctypes.data)
    if rc != 0:
        raise RuntimeError("refh_taper failed")
    return out, tc


def gauss_filt_var(grad, vel, dh, wd_damp, wd_damp1, fc_end):
    """The reference's spatially variable Gaussian smoothing (src/gauss_filt_var.c,
    SPATFILTER=4) of grad [ny, nx] for the velocity vel [ny, nx]; its
    temporary files go to a temporary directory."""
    import tempfile

    lib = C.CDLL(os.path.join(REF_DIR, "libdenise_ref.so"))
    lib.refh_gauss_filt_var.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                        C.c_void_p, C.c_void_p]
    g = _f32(grad).copy()
    v = _f32(vel)
    ny, nx = g.shape
    with tempfile.TemporaryDirectory(dir="/tmp") as d:      # a short path: the reference's names are char[74]
        rc = lib.refh_gauss_filt_var(d.encode(), nx, ny, dh, wd_damp, wd_damp1, fc_end, v.ctypes.data,
                                     g.ctypes.data)
    if rc != 0:
        raise RuntimeError("refh_gauss_filt_var failed")
    return g


def builtin_model(l, nx, ny, dh, dt, fl=()):
    """The reference's built-in start model for READMOD=0: model() of
    src/model_grad_visc.c (l > 0) or model_elastic() of src/check_start.c
    (l == 0).  Returns vs, rho, taus (None for l == 0), eta (None for l == 0)
    and the bytes of the vs file the reference writes (merged, x outer)."""
    import tempfile

    lib = C.CDLL(os.path.join(REF_DIR, "libdenise_ref.so"))
    lib.refh_builtin_model.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    vs = np.zeros((ny, nx), np.float32)
    rho = np.zeros((ny, nx), np.float32)
    taus = np.zeros((ny, nx), np.float32)
    eta = np.zeros(max(l, 1), np.float32)
    flv = np.asarray(list(fl) + [0.0] * (8 - len(fl)), np.float32)
    with tempfile.TemporaryDirectory(dir="/tmp") as d:      # a short path: the reference's names are char[74]
        rc = lib.refh_builtin_model(d.encode(), l, nx, ny, dh, dt, flv.ctypes.data, vs.ctypes.data,
                                    rho.ctypes.data, taus.ctypes.data, eta.ctypes.data)
        name = os.path.join(d, "inv_vs_it_0.bin" if l > 0 else "mod.mu")
        vs_file = open(name, "rb").read() if rc == 0 else b""
    if rc != 0:
        raise RuntimeError("refh_builtin_model failed")
    return vs, rho, (taus if l > 0 else None), (eta[:l] if l > 0 else None), vs_file


def checkfd(vs, rho, qs, fl, dh, dt, ts, fdorder, maxrelerror, fw):
    """The reference's FD grid check (checkfd_ssg_visc for fl non-empty, else
    checkfd_ssg_elastic) on arguments that pass it; returns its report."""
    import tempfile

    lib = C.CDLL(os.path.join(REF_DIR, "libdenise_ref.so"))
    lib.refh_checkfd.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_float, C.c_float, C.c_float,
                                 C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    vs, rho = _f32(vs), _f32(rho)
    ny, nx = vs.shape
    l = len(fl)
    q = _f32(qs) if l > 0 else np.ones_like(vs)
    flv = np.asarray(list(fl) + [0.0] * (8 - l), np.float32)
    with tempfile.TemporaryDirectory() as d:
        log = os.path.join(d, "checkfd.log")
        if lib.refh_checkfd(log.encode(), l, nx, ny, flv.ctypes.data, dh, dt, ts, fdorder, maxrelerror, fw,
                            vs.ctypes.data, rho.ctypes.data, q.ctypes.data) != 0:
            raise RuntimeError("refh_checkfd failed")
        return open(log).read()


def calc_misfit(obs, syn, lnorm, dt, l2_in=0.0):
    """The reference's calc_misfit (src/calc_misfit.c) of traces [ntr, ns]."""
    lib = C.CDLL(os.path.join(REF_DIR, "libdenise_ref.so"))
    lib.refh_calc_misfit.restype = C.c_double
    lib.refh_calc_misfit.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float]
    o, s = _f32(obs), _f32(syn)
    return lib.refh_calc_misfit(o.ctypes.data, s.ctypes.data, o.shape[0], o.shape[1], lnorm, dt, l2_in)


def calc_energy(obs, dt, energy_in=0.0):
    """The reference's calc_energy (src/calc_energy.c) of traces [ntr, ns]."""
    lib = C.CDLL(os.path.join(REF_DIR, "libdenise_ref.so"))
    lib.refh_calc_energy.restype = C.c_double
    lib.refh_calc_energy.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float]
    o = _f32(obs)
    return lib.refh_calc_energy(o.ctypes.data, o.shape[0], o.shape[1], dt, energy_in)


def model_update(vs, rho, d_vs, d_rho, eps_scale, scalerho, it, inv_vs_iter, inv_rho_iter, limits):
    """The reference's model update (src/calc_mat_change_test.c, itest = 1):
    returns vs_new, rho_new, eps_u, eps_rho."""
    lib = C.CDLL(os.path.join(REF_DIR, "libdenise_ref.so"))
    lib.refh_model_update.restype = C.c_float
    lib.refh_model_update.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 4 + [C.c_float, C.c_float, C.c_int, C.c_int,
                                                                              C.c_int] + [C.c_void_p] * 4
    a = [_f32(x) for x in (vs, rho, d_vs, d_rho)]
    ny, nx = a[0].shape
    lim = _f32(limits)
    vn, rn = np.zeros_like(a[0]), np.zeros_like(a[0])
    er = C.c_float()
    eu = lib.refh_model_update(nx, ny, *[x.ctypes.data for x in a], eps_scale, scalerho, it, inv_vs_iter,
                               inv_rho_iter, lim.ctypes.data, vn.ctypes.data, rn.ctypes.data, C.addressof(er))
    return vn, rn, np.float32(eu), np.float32(er.value)


def lbfgs_ring(it, y, s, q, pointer, nlbfgs):
    """The reference's L-BFGS step (src/LBFGS.c) on ring buffers y, s
    [nlbfgs, nvec]; returns (q after the first loop, r)."""
    lib = C.CDLL(os.path.join(REF_DIR, "libdenise_ref.so"))
    lib.refh_lbfgs.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
    y, s = _f32(y), _f32(s)
    q = _f32(q).copy()
    r = np.zeros_like(q)
    lib.refh_lbfgs(it, y.ctypes.data, s.ctypes.data, q.ctypes.data, r.ctypes.data, pointer, nlbfgs, q.size)
    return q, r


def opt_step(l2t, epst):
    """The reference's parabolic step (src/calc_opt_step.c, src/solvelin.c)."""
    lib = C.CDLL(os.path.join(REF_DIR, "libdenise_ref.so"))
    lib.refh_opt_step.restype = C.c_float
    lib.refh_opt_step.argtypes = [C.c_void_p, C.c_void_p]
    a, e = _f32(l2t), _f32(epst)
    return np.float32(lib.refh_opt_step(a.ctypes.data, e.ctypes.data))


def smooth_model(vs, rho, filt_size):
    """The reference's median model smoothing (src/smooth_model.c with
    src/median.c, MODEL_FILTER=1): returns vs, rho and FILT_SIZE after it."""
    import tempfile

    lib = C.CDLL(os.path.join(REF_DIR, "libdenise_ref.so"))
    lib.refh_smooth_model.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    v, r = _f32(vs).copy(), _f32(rho).copy()
    ny, nx = v.shape
    with tempfile.TemporaryDirectory(dir="/tmp") as d:      # a short path: the reference's names are char[74]
        fs = lib.refh_smooth_model(d.encode(), nx, ny, filt_size, v.ctypes.data, r.ctypes.data)
    if fs == -999:
        raise RuntimeError("refh_smooth_model failed")
    return v, r, fs


def calc_mres(u, u0):
    """The reference's relative model change (src/calc_mres.c)."""
    lib = C.CDLL(os.path.join(REF_DIR, "libdenise_ref.so"))
    lib.refh_calc_mres.restype = C.c_float
    lib.refh_calc_mres.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    a, b = _f32(u), _f32(u0)
    return np.float32(lib.refh_calc_mres(a.shape[1], a.shape[0], a.ctypes.data, b.ctypes.data))
