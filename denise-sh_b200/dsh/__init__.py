"""dsh — Python host interface of the B200 SH time-stepping / FWI-gradient engine.

A thin ctypes layer over the in-tree C-ABI library ``libdsh.so`` (declared in
``include/dsh.h``).  It mirrors the reference's per-shot workflow
(src/denise.c): set a model, model shots forward, or compute the energy-
preconditioned vs/rho gradient of the L2 waveform misfit and the
pseudo-Hessian diagonal.  There is no CPU fallback: if the CUDA library is
missing or no GPU is visible, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libdsh.so")

DSH_OK = 0
EPRECOND_ENERGY_ONLY = 10      # dsh_params.eprecond: raw gradient plus the energies Ws, Wr
ERRORS = {-1: "invalid parameter", -2: "CUDA error", -3: "out of device memory or budget",
          -4: "simulation is unstable (non-finite wavefield)", -5: "call out of order", -6: "device wait timed out"}
ERR_PARAM, ERR_CUDA, ERR_OOM, ERR_UNSTABLE, ERR_STATE, ERR_TIMEOUT = -1, -2, -3, -4, -5, -6

FIELD = {"vy": 0, "sxy": 1, "syz": 2, "Ws": 12, "Wr": 13, "We": 14, "g_u": 15, "g_rho": 16, "hess_u": 17,
         "hess_rho": 18, "brho": 300, "uip": 301, "ujp": 302, "muip": 303, "mujp": 304, "tausipjp": 305,
         "taus": 306}


class DshError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        super().__init__(f"{what}: {ERRORS.get(code, code)} ({code})")
        self.code = code


class Params(C.Structure):
    """Mirror of ``dsh_params`` (include/dsh.h)."""
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nt", C.c_int), ("dh", C.c_float), ("dt", C.c_float),
                ("fdorder", C.c_int), ("maxrelerror", C.c_int), ("fw", C.c_int), ("free_surf", C.c_int),
                ("damping", C.c_float), ("fpml", C.c_float), ("npower", C.c_float), ("k_max_pml", C.c_float),
                ("l", C.c_int), ("fl", C.c_float * 8), ("quellart", C.c_int), ("eprecond", C.c_int),
                ("max_shots", C.c_int), ("compat_fd12", C.c_int), ("mem_budget", C.c_longlong),
                ("ckpt_every", C.c_int), ("grad_q", C.c_int)]


class ShotC(C.Structure):
    _fields_ = [("nsrc", C.c_int), ("srcpos", C.POINTER(C.c_float)), ("signals", C.POINTER(C.c_float)),
                ("ntr", C.c_int), ("recpos", C.POINTER(C.c_int))]


class Stats(C.Structure):
    _fields_ = [("ms_forward", C.c_double), ("ms_adjoint", C.c_double), ("ms_total", C.c_double),
                ("kernel_launches", C.c_longlong), ("point_updates", C.c_longlong),
                ("storage_bytes", C.c_longlong), ("checkpoint_interval", C.c_int)]


class BatchStats(C.Structure):
    _fields_ = [("ms_total", C.c_double), ("kernel_launches", C.c_longlong), ("point_updates", C.c_longlong),
                ("v_variant", C.c_int), ("s_variant", C.c_int), ("phases", C.c_int), ("v_ms", C.c_float * 4),
                ("s_ms", C.c_float * 4)]


_lib = None


def lib() -> C.CDLL:
    """Load the CUDA engine; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} not built (run __graft_entry__.build() or make -C denise-sh_b200/csrc)")
        L = C.CDLL(LIB_PATH)
        L.dsh_create.restype = C.c_void_p
        L.dsh_create.argtypes = [C.POINTER(Params), C.c_int, C.POINTER(C.c_int)]
        L.dsh_destroy.argtypes = [C.c_void_p]
        L.dsh_error_string.restype = C.c_char_p
        L.dsh_set_model.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.dsh_forward.argtypes = [C.c_void_p, C.POINTER(ShotC), C.c_int, C.c_void_p]
        L.dsh_forward_device.argtypes = [C.c_void_p, C.POINTER(ShotC), C.c_int, C.c_void_p]
        L.dsh_gradient.argtypes = [C.c_void_p, C.POINTER(ShotC), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.POINTER(C.c_double), C.c_void_p, C.c_void_p, C.c_void_p]
        L.dsh_gradient_device.argtypes = [C.c_void_p, C.POINTER(ShotC), C.c_int, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.POINTER(C.c_double)]
        L.dsh_hessian_diag.argtypes = [C.c_void_p, C.POINTER(ShotC), C.c_int, C.c_void_p, C.c_void_p]
        L.dsh_get_field.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.dsh_get_stats.argtypes = [C.c_void_p, C.POINTER(Stats)]
        L.dsh_params_default.argtypes = [C.POINTER(Params)]
        L.dsh_set_stream.argtypes = [C.c_void_p, C.c_void_p]
        L.dsh_profile_step.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.dsh_residual_noalloc.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p]
        L.dsh_timedomain_filt.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int,
                                          C.c_int, C.c_void_p]
        L.dsh_smooth_gauss.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.dsh_gauss_filter_size.argtypes = [C.c_float] * 4
        L.dsh_smooth_gauss_var.argtypes = [C.c_int, C.c_int] + [C.c_float] * 4 + [C.c_void_p] * 4
        L.dsh_setup_gauss_var.argtypes = [C.c_int, C.c_int] + [C.c_float] * 4 + [C.c_void_p, C.c_void_p, C.c_int,
                                                                                    C.c_void_p, C.c_int, C.c_void_p]
        L.dsh_taper_coeff.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_void_p, C.c_int, C.c_float, C.c_int,
                                      C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.dsh_taper_apply.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.dsh_set_shot_taper.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_int]
        L.dsh_set_misfit.argtypes = [C.c_void_p, C.c_int]
        L.dsh_set_wait_limits.argtypes = [C.c_void_p, C.c_longlong, C.c_double]
        L.dsh_get_gradient_q.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.dsh_set_step_variant.argtypes = [C.c_void_p, C.c_int]
        L.dsh_batch_set_host_timeout.argtypes = [C.c_void_p, C.c_double]
        L.dsh_autotune.argtypes = [C.c_void_p, C.POINTER(ShotC), C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_int)]
        L.dsh_profile_fused.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.dsh_get_shot_misfits.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.dsh_get_energy_sums.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.dsh_batch_create.restype = C.c_void_p
        L.dsh_batch_create.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int)]
        L.dsh_batch_destroy.argtypes = [C.c_void_p]
        L.dsh_batch_set_model.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.dsh_batch_forward.argtypes = [C.c_void_p, C.POINTER(ShotC), C.c_void_p, C.c_void_p]
        L.dsh_batch_forward_device.argtypes = [C.c_void_p, C.POINTER(ShotC), C.c_void_p, C.c_void_p]
        L.dsh_batch_set_stream.argtypes = [C.c_void_p, C.c_void_p]
        L.dsh_batch_set_variant.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.dsh_batch_get_stats.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(BatchStats)]
        L.dsh_setup_holberg.argtypes = [C.c_int, C.c_int, C.c_void_p]
        L.dsh_setup_pml.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                    C.c_float, C.c_float, C.c_void_p]
        L.dsh_setup_model.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_float] + [C.c_void_p] * 15
        L.dsh_setup_visc_base.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_float] + [C.c_void_p] * 8
        L.dsh_setup_wavelet.argtypes = [C.c_int, C.c_int, C.c_float, C.c_int, C.c_void_p, C.c_void_p]
        L.dsh_setup_dt_limit.restype = C.c_double
        L.dsh_setup_dt_limit.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float]
        _lib = L
    return _lib


def _check(code, what):
    if code != DSH_OK:
        raise DshError(code, what)


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None


@dataclass
class Shot:
    """One shot: source table [8, nsrc] (grid x, grid y, 0, tshift, fc, amp, angle, type),
    receivers [2, ntr] (grid x, grid y), optional signals [nsrc, nt]."""
    srcpos: np.ndarray
    recpos: np.ndarray
    signals: np.ndarray | None = None

    def __post_init__(self):
        self.srcpos = np.ascontiguousarray(self.srcpos, np.float32)
        self.recpos = np.ascontiguousarray(self.recpos, np.int32)
        if self.signals is not None:
            self.signals = np.ascontiguousarray(self.signals, np.float32)

    @property
    def ntr(self):
        return self.recpos.shape[1]


def point_source(ix: int, iy: int, fc: float, amp: float = 1.0, tshift: float = 0.0) -> np.ndarray:
    """Source table of one vertical point force (type 3) at grid (ix, iy)."""
    sp = np.zeros((8, 1), np.float32)
    sp[:, 0] = [ix, iy, 0.0, tshift, fc, amp, 0.0, 3.0]
    return sp


def _shots_c(shots):
    arr = (ShotC * len(shots))()
    for k, s in enumerate(shots):
        arr[k].nsrc = s.srcpos.shape[1]
        arr[k].srcpos = _fptr(s.srcpos)
        arr[k].signals = _fptr(s.signals)
        arr[k].ntr = s.ntr
        arr[k].recpos = s.recpos.ctypes.data_as(C.POINTER(C.c_int))
    return arr


def make_params(nx, ny, nt, dh, dt, **kw) -> Params:
    p = Params()
    lib().dsh_params_default(C.byref(p))
    p.nx, p.ny, p.nt, p.dh, p.dt = nx, ny, nt, dh, dt
    fl = kw.pop("fl", ())
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    for i, v in enumerate(fl):
        p.fl[i] = v
    return p


class Engine:
    """A device context for one model (``dsh_ctx``)."""

    def __init__(self, params: Params, device: int = 0):
        self.p = params
        st = C.c_int(0)
        self.h = lib().dsh_create(C.byref(params), device, C.byref(st))
        if not self.h:
            raise DshError(st.value, "dsh_create")

    def close(self):
        if getattr(self, "h", None):
            lib().dsh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def shape(self):
        return (self.p.ny, self.p.nx)

    def set_model(self, vs, rho, qs=None):
        self._vs = np.ascontiguousarray(vs, np.float32)
        self._rho = np.ascontiguousarray(rho, np.float32)
        self._qs = np.ascontiguousarray(qs, np.float32) if qs is not None else None
        _check(lib().dsh_set_model(self.h, self._vs.ctypes.data, self._rho.ctypes.data,
                                   self._qs.ctypes.data if self._qs is not None else None), "dsh_set_model")

    def forward(self, shots):
        shots = list(shots)
        total = sum(s.ntr for s in shots) * self.p.nt
        out = np.zeros(max(total, 1), np.float32)
        arr = _shots_c(shots)
        _check(lib().dsh_forward(self.h, arr, len(shots), out.ctypes.data), "dsh_forward")
        return _split(out, shots, self.p.nt)

    def gradient(self, shots, obs, want_seis=False, want_energy=False):
        """obs: list of [ntr, nt] arrays (one per shot).  Returns a dict with
        g_vs, g_rho, l2 (and seis, Ws, Wr if asked)."""
        shots = list(shots)
        flat = np.ascontiguousarray(np.concatenate([np.asarray(o, np.float32).ravel() for o in obs]))
        ny, nx = self.shape
        gv = np.zeros((ny, nx), np.float32)
        gr = np.zeros((ny, nx), np.float32)
        l2 = C.c_double(0)
        seis = np.zeros(max(flat.size, 1), np.float32) if want_seis else None
        ws = np.zeros((len(shots), ny, nx), np.float32) if want_energy else None
        wr = np.zeros((len(shots), ny, nx), np.float32) if want_energy else None
        arr = _shots_c(shots)
        _check(lib().dsh_gradient(self.h, arr, len(shots), flat.ctypes.data, gv.ctypes.data, gr.ctypes.data,
                                  C.byref(l2), seis.ctypes.data if want_seis else None,
                                  ws.ctypes.data if want_energy else None, wr.ctypes.data if want_energy else None),
               "dsh_gradient")
        out = {"g_vs": gv, "g_rho": gr, "l2": l2.value}
        if want_seis:
            out["seis"] = _split(seis, shots, self.p.nt)
        if want_energy:
            out["Ws"], out["Wr"] = ws, wr
        return out

    def gradient_q(self):
        """dJ/dQs [ny, nx] of the last gradient (params.grad_q = 1; J = the returned L2 misfit)."""
        out = np.zeros(self.shape, np.float32)
        _check(lib().dsh_get_gradient_q(self.h, out.ctypes.data, None), "dsh_get_gradient_q")
        return out

    def gradient_device(self, shots, obs_dev_ptr: int, g_vs_ptr: int, g_rho_ptr: int) -> float:
        """Device-resident gradient (pointers from e.g. torch tensors)."""
        arr = _shots_c(list(shots))
        l2 = C.c_double(0)
        _check(lib().dsh_gradient_device(self.h, arr, len(arr), obs_dev_ptr, g_vs_ptr, g_rho_ptr, C.byref(l2)),
               "dsh_gradient_device")
        return l2.value

    def forward_device(self, shots, seis_dev_ptr: int):
        arr = _shots_c(list(shots))
        _check(lib().dsh_forward_device(self.h, arr, len(arr), seis_dev_ptr), "dsh_forward_device")

    def hessian_diag(self, shots):
        shots = list(shots)
        ny, nx = self.shape
        hv = np.zeros((ny, nx), np.float32)
        hr = np.zeros((ny, nx), np.float32)
        _check(lib().dsh_hessian_diag(self.h, _shots_c(shots), len(shots), hv.ctypes.data, hr.ctypes.data),
               "dsh_hessian_diag")
        return hv, hr

    def field(self, name, shot=0, l=None):
        code = FIELD[name] if l is None else {"r": 100, "q": 200}[name] + l
        out = np.zeros(self.shape, np.float32)
        _check(lib().dsh_get_field(self.h, shot, code, out.ctypes.data), "dsh_get_field")
        return out

    def set_stream(self, stream_handle: int | None):
        """Run on a caller's CUDA stream (e.g. torch.cuda.Stream().cuda_stream)."""
        _check(lib().dsh_set_stream(self.h, stream_handle), "dsh_set_stream")

    PASSES = {"forward": 0, "forward_store": 1, "forward_hessian": 2, "adjoint": 3}

    def profile_step(self, pass_name: str, nsteps: int) -> dict:
        """Mean device ms per launch of the velocity, injection and stress kernels."""
        out = np.zeros(3, np.float32)
        _check(lib().dsh_profile_step(self.h, self.PASSES[pass_name], nsteps, out.ctypes.data), "dsh_profile_step")
        return {"v_step": float(out[0]), "inject_sample": float(out[1]), "s_step": float(out[2])}

    VARIANTS = ("kernel pair", "kernel pair, staged velocity taps", "fused step", "persistent launch",
                "cluster-resident launch", "temporally blocked launch")

    def autotune(self, shots, nsteps=64):
        """Times each step-kernel variant on these shots, keeps the fastest; returns (name, ms per step each)."""
        ms = np.zeros(len(self.VARIANTS), np.float32)
        ch = C.c_int(0)
        _check(lib().dsh_autotune(self.h, _shots_c(list(shots)), len(shots), nsteps, ms.ctypes.data, C.byref(ch)),
               "dsh_autotune")
        return self.VARIANTS[ch.value], {n: float(t) for n, t in zip(self.VARIANTS, ms)}

    def profile_fused(self, pass_name: str, nsteps: int):
        """Mean device ms per launch of the fused step kernel, or None when it does not serve this pass."""
        out = np.zeros(1, np.float32)
        rc = lib().dsh_profile_fused(self.h, self.PASSES[pass_name], nsteps, out.ctypes.data)
        if rc == -5:
            return None
        _check(rc, "dsh_profile_fused")
        return float(out[0])

    def set_wait_limits(self, device_polls: int = 0, host_seconds: float = 0.0):
        """Poll limit of the device's bounded waits and wall-clock limit of the
        host's waits (0 = defaults); expiry returns DSH_ERR_TIMEOUT."""
        _check(lib().dsh_set_wait_limits(self.h, C.c_longlong(int(device_polls)), C.c_double(float(host_seconds))),
               "dsh_set_wait_limits")

    def set_step_variant(self, variant: int):
        """Pin a step-kernel variant (index into VARIANTS; -1 = defaults)."""
        _check(lib().dsh_set_step_variant(self.h, int(variant)), "dsh_set_step_variant")

    LNORM = {"l1": 1, "l2": 2, "cauchy": 3, "sech": 4, "global_correlation": 5}

    def set_misfit(self, lnorm):
        """Misfit norm of the residual (calc_res.c LNORM 1..5, or a key of LNORM)."""
        _check(lib().dsh_set_misfit(self.h, self.LNORM.get(lnorm, lnorm)), "dsh_set_misfit")

    def set_shot_taper(self, srtshape=1, srtradius=5.0, filtsize=1, enable=True):
        """SWS_TAPER_CIRCULAR_PER_SHOT: taper every shot's gradient around its
        first source before the shot sum (src/taper_grad_shot.c)."""
        _check(lib().dsh_set_shot_taper(self.h, int(bool(enable)), int(srtshape), float(srtradius), int(filtsize)),
               "dsh_set_shot_taper")

    def shot_misfits(self, nshots):
        out = np.zeros(nshots, np.float64)
        _check(lib().dsh_get_shot_misfits(self.h, nshots, out.ctypes.data), "dsh_get_shot_misfits")
        return out

    def energy_sums(self):
        ny, nx = self.shape
        ws, wr = np.zeros((ny, nx), np.float32), np.zeros((ny, nx), np.float32)
        _check(lib().dsh_get_energy_sums(self.h, ws.ctypes.data, wr.ctypes.data), "dsh_get_energy_sums")
        return ws, wr

    def stats(self) -> dict:
        s = Stats()
        _check(lib().dsh_get_stats(self.h, C.byref(s)), "dsh_get_stats")
        return {k: getattr(s, k) for k, _ in Stats._fields_}


class Batch:
    """An uneven batch of models advanced together (``dsh_batch``): one
    velocity and one stress launch per time step for every shot of every
    model; the block shape is chosen by the batch's autotuner."""

    VARIANTS = ("128x8 points x 1 shot", "128x4 points x 2 shots", "128x2 points x 4 shots",
                "128x4 points x 1 shot")

    def __init__(self, params_list, device: int = 0):
        self.params = list(params_list)
        arr = (Params * len(self.params))(*self.params)
        st = C.c_int(0)
        self.h = lib().dsh_batch_create(arr, len(self.params), device, C.byref(st))
        if not self.h:
            raise DshError(st.value, "dsh_batch_create")
        self._keep = {}

    def close(self):
        if getattr(self, "h", None):
            lib().dsh_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_model(self, k, vs, rho, qs=None):
        arrs = [np.ascontiguousarray(x, np.float32) if x is not None else None for x in (vs, rho, qs)]
        self._keep[k] = arrs
        _check(lib().dsh_batch_set_model(self.h, k, *[a.ctypes.data if a is not None else None for a in arrs]),
               "dsh_batch_set_model")

    def set_variant(self, v=-1, s=-1):
        _check(lib().dsh_batch_set_variant(self.h, v, s), "dsh_batch_set_variant")

    def set_stream(self, stream_handle):
        _check(lib().dsh_batch_set_stream(self.h, stream_handle), "dsh_batch_set_stream")

    def set_host_timeout(self, host_seconds: float):
        """Wall-clock limit of the batch's host waits (0 = default); expiry returns DSH_ERR_TIMEOUT."""
        _check(lib().dsh_batch_set_host_timeout(self.h, C.c_double(float(host_seconds))), "dsh_batch_set_host_timeout")

    def _flat(self, shots_per_model):
        flat = [s for group in shots_per_model for s in group]
        n = np.array([len(g) for g in shots_per_model], np.int32)
        return flat, n

    def forward(self, shots_per_model):
        """shots_per_model[k]: list of Shot for model k -> [[seis [ntr, nt_k] per shot] per model]."""
        flat, n = self._flat(shots_per_model)
        total = sum(s.ntr * p.nt for g, p in zip(shots_per_model, self.params) for s in g)
        out = np.zeros(max(total, 1), np.float32)
        _check(lib().dsh_batch_forward(self.h, _shots_c(flat), n.ctypes.data, out.ctypes.data), "dsh_batch_forward")
        res, o = [], 0
        for g, p in zip(shots_per_model, self.params):
            m = sum(s.ntr for s in g) * p.nt
            res.append(_split(out[o:o + m], g, p.nt))
            o += m
        return res

    def forward_device(self, shots_per_model, seis_dev_ptr: int):
        flat, n = self._flat(shots_per_model)
        _check(lib().dsh_batch_forward_device(self.h, _shots_c(flat), n.ctypes.data, seis_dev_ptr),
               "dsh_batch_forward_device")

    def stats(self) -> dict:
        ms = np.zeros(len(self.params), np.float64)
        s = BatchStats()
        _check(lib().dsh_batch_get_stats(self.h, ms.ctypes.data, C.byref(s)), "dsh_batch_get_stats")
        return {"ms_total": s.ms_total, "kernel_launches": s.kernel_launches, "point_updates": s.point_updates,
                "v_variant": s.v_variant, "s_variant": s.s_variant, "phases": s.phases,
                "v_ms": list(s.v_ms)[:len(self.VARIANTS)], "s_ms": list(s.s_ms)[:len(self.VARIANTS)],
                "model_ms": ms}


def smooth_gauss(grad, filt, stream=None):
    """SPATFILTER=3 Gaussian smoothing of a [ny, nx] gradient on the GPU (dsh_smooth_gauss)."""
    import torch

    g = torch.from_numpy(np.ascontiguousarray(grad, np.float32)).cuda()
    out = torch.empty_like(g)
    ny, nx = g.shape
    _check(lib().dsh_smooth_gauss(nx, ny, int(filt), g.data_ptr(), out.data_ptr(), stream), "dsh_smooth_gauss")
    torch.cuda.synchronize()
    return out.cpu().numpy()


def smooth_gauss_var(grad, vel, dh, wd_damp, wd_damp1, fc_end, stream=None):
    """SPATFILTER=4 Gaussian smoothing whose size follows the velocity vel
    [ny, nx], on the GPU (dsh_smooth_gauss_var)."""
    import torch

    g = torch.from_numpy(np.ascontiguousarray(grad, np.float32)).cuda()
    out = torch.empty_like(g)
    v = np.ascontiguousarray(vel, np.float32)
    ny, nx = g.shape
    _check(lib().dsh_smooth_gauss_var(nx, ny, dh, wd_damp, wd_damp1, fc_end, v.ctypes.data, g.data_ptr(),
                                      out.data_ptr(), stream), "dsh_smooth_gauss_var")
    return out.cpu().numpy()


def gauss_var_tables(vel, dh, wd_damp, wd_damp1, fc_end, max_pairs=4096, max_weights=1 << 22):
    """Host tables of SPATFILTER=4 (dsh_setup_gauss_var): per-point kernel
    index (-1: none) [ny, nx], per kernel (hx, hz, weight offset, weight
    sum), and the weights."""
    v = np.ascontiguousarray(vel, np.float32)
    ny, nx = v.shape
    mp = np.zeros((ny, nx), np.int32)
    pairs = np.zeros(4 * max_pairs, np.int32)
    w = np.zeros(max_weights, np.float32)
    n = lib().dsh_setup_gauss_var(nx, ny, dh, wd_damp, wd_damp1, fc_end, v.ctypes.data, mp.ctypes.data, max_pairs,
                                  pairs.ctypes.data, max_weights, w.ctypes.data)
    if n < 0:
        raise DshError(ERR_PARAM, "dsh_setup_gauss_var")
    pr = pairs[:4 * n].reshape(n, 4)
    return mp, [(int(a), int(b), int(c), float(np.int32(d).view(np.float32))) for a, b, c, d in pr], w


def gauss_filter_size(wd_damp, c_vs, fc_end, dh):
    return int(lib().dsh_gauss_filter_size(wd_damp, c_vs, fc_end, dh))


TAPER_VERTICAL, TAPER_HORIZONTAL, TAPER_SOURCES, TAPER_FILE_VS, TAPER_FILE_RHO = 1, 2, 3, 5, 6


def taper_coeff(sws, nx, ny, dh, gradt=(0, 0, 0, 0), srtshape=1, srtradius=5.0, filtsize=1, src_xy=None,
                recpos=None, file_vals=None):
    """Host coefficients of the gradient taper sws (src/taper_grad.c):
    returns (coeff [ny, nx] float32, zero [ny, nx] bool).  src_xy [2, nsrc]
    source x, y in metres; recpos [2, ntr] 1-based grid points; file_vals
    nx*ny floats, x outer (sws 5, 6)."""
    coeff = np.zeros((ny, nx), np.float32)
    zero = np.zeros((ny, nx), np.uint8)
    sxy = np.ascontiguousarray(src_xy if src_xy is not None else np.zeros((2, 0)), np.float32)
    rp = np.ascontiguousarray(recpos if recpos is not None else np.zeros((2, 0)), np.int32)
    gt = np.ascontiguousarray(gradt, np.int32)
    fv = np.ascontiguousarray(file_vals, np.float32) if file_vals is not None else None
    _check(lib().dsh_taper_coeff(sws, nx, ny, dh, gt.ctypes.data, srtshape, srtradius, filtsize, sxy.shape[1],
                                 sxy.ctypes.data, rp.shape[1], rp.ctypes.data,
                                 fv.ctypes.data if fv is not None else None, coeff.ctypes.data, zero.ctypes.data),
           "dsh_taper_coeff")
    return coeff, zero.astype(bool)


def taper_apply(g_dev, coeff, zero, stream=None):
    """g = zero ? 0 : g*coeff in place on a CUDA tensor g_dev [ny, nx]
    (dsh_taper_apply); coeff, zero: host arrays from taper_coeff."""
    import torch

    ny, nx = g_dev.shape
    if g_dev.dtype != torch.float32 or not g_dev.is_cuda or not g_dev.is_contiguous():
        raise ValueError("g_dev must be a contiguous float32 CUDA tensor")
    c = torch.from_numpy(np.ascontiguousarray(coeff, np.float32)).to(g_dev.device)
    z = torch.from_numpy(np.ascontiguousarray(zero, np.uint8)).to(g_dev.device)
    _check(lib().dsh_taper_apply(g_dev.data_ptr(), nx, ny, c.data_ptr(), z.data_ptr(), stream), "dsh_taper_apply")
    torch.cuda.synchronize(g_dev.device)
    return g_dev


NOALLOC_MAX_SHOTS = 64


def residual_noalloc(nshots: int, ntr: int, nt: int, syn_ptr: int, obs_ptr: int, res_ptr: int, l2_ptr: int,
                     stream: int | None = None) -> None:
    """Allocation-free residual + L2 on device pointers (see dsh_residual_noalloc in include/dsh.h)."""
    _check(lib().dsh_residual_noalloc(nshots, ntr, nt, syn_ptr, obs_ptr, res_ptr, l2_ptr, stream),
           "dsh_residual_noalloc")


def _split(flat, shots, nt):
    out, o = [], 0
    for s in shots:
        n = s.ntr * nt
        out.append(flat[o:o + n].reshape(s.ntr, nt))
        o += n
    return out


# ---------------- host-side coefficient helpers (for parity checks) ----------------

def holberg(fdorder: int, maxrelerror: int) -> np.ndarray:
    hc = np.zeros(7, np.float32)
    _check(lib().dsh_setup_holberg(fdorder, maxrelerror, hc.ctypes.data), "dsh_setup_holberg")
    return hc


PML_NAMES = ["K_x", "a_x", "b_x", "K_x_half", "a_x_half", "b_x_half", "K_y", "a_y", "b_y", "K_y_half",
             "a_y_half", "b_y_half", "d_x", "d_x_half", "d_y", "d_y_half"]
MAX_FW = 256


def pml_profiles(nx, ny, fw, dh, dt, damping, fpml, npower=4.0, k_max_pml=1.0) -> dict:
    buf = np.zeros(16 * (2 * MAX_FW + 1), np.float32)
    lib().dsh_setup_pml(nx, ny, fw, dh, dt, damping, fpml, npower, k_max_pml, buf.ctypes.data)
    v = buf.reshape(16, 2 * MAX_FW + 1)
    return {n: v[k, 1:2 * fw + 1].copy() for k, n in enumerate(PML_NAMES)}


def model_coefficients(vs, rho, qs=None, l=0, fl=(), dt=1e-4) -> dict:
    vs = np.ascontiguousarray(vs, np.float32)
    rho = np.ascontiguousarray(rho, np.float32)
    ny, nx = vs.shape
    n = nx * ny
    qs = np.ascontiguousarray(qs if qs is not None else np.ones_like(vs), np.float32)
    flv = np.zeros(8, np.float32)
    flv[:len(fl)] = fl
    out = {k: np.zeros((ny, nx), np.float32) for k in ("brho", "uip", "ujp", "fipjp", "f")}
    dip = np.zeros((max(l, 1), ny, nx), np.float32)
    d = np.zeros((max(l, 1), ny, nx), np.float32)
    sls = [np.zeros(4, np.float32) for _ in range(4)]
    cn = np.zeros(2, np.float32)
    rc = lib().dsh_setup_model(nx, ny, l, flv.ctypes.data, dt, vs.ctypes.data, rho.ctypes.data, qs.ctypes.data,
                               out["brho"].ctypes.data, out["uip"].ctypes.data, out["ujp"].ctypes.data,
                               out["fipjp"].ctypes.data, out["f"].ctypes.data, dip.ctypes.data, d.ctypes.data,
                               *[x.ctypes.data for x in sls], cn.ctypes.data)
    _check(rc, "dsh_setup_model")
    out.update(dip=dip[:l], d=d[:l], bip=sls[0][:l], bjm=sls[1][:l], cip=sls[2][:l], cjm=sls[3][:l], cnorm=cn)
    return out


def visc_base(vs, rho, qs, l, fl, dt) -> dict:
    """dsh_setup_visc_base on the host: relaxed moduli muip, mujp, tausipjp, taus and eta."""
    vs = np.ascontiguousarray(vs, np.float32)
    rho = np.ascontiguousarray(rho, np.float32)
    qs = np.ascontiguousarray(qs, np.float32)
    ny, nx = vs.shape
    flv = np.zeros(8, np.float32)
    flv[:len(fl)] = fl
    out = {k: np.zeros((ny, nx), np.float32) for k in ("muip", "mujp", "tausipjp", "taus")}
    eta = np.zeros(8, np.float32)
    _check(lib().dsh_setup_visc_base(nx, ny, l, flv.ctypes.data, dt, vs.ctypes.data, rho.ctypes.data,
                                     qs.ctypes.data, out["muip"].ctypes.data, out["mujp"].ctypes.data,
                                     out["tausipjp"].ctypes.data, out["taus"].ctypes.data, eta.ctypes.data),
           "dsh_setup_visc_base")
    out["eta"] = eta[:l]
    return out


def wavelet(quellart: int, nt: int, dt: float, srcpos8) -> np.ndarray:
    sp = np.ascontiguousarray(srcpos8, np.float32)
    out = np.zeros((sp.shape[1], nt), np.float32)
    _check(lib().dsh_setup_wavelet(quellart, nt, dt, sp.shape[1], sp.ctypes.data, out.ctypes.data),
           "dsh_setup_wavelet")
    return out


def dt_limit(fdorder: int, maxrelerror: int, dh: float, vmax: float) -> float:
    return lib().dsh_setup_dt_limit(fdorder, maxrelerror, dh, vmax)


def check_fd(vs, rho, qs=None, fl=(), *, dh: float, dt: float, ts: float, fdorder: int, maxrelerror: int = 1,
             fw: int = 20):
    """The reference's FD grid check of a starting model (checkfd_ssg_visc /
    checkfd_ssg_elastic): returns (status, dict(cmin, cmax, dtstab, dhstab),
    warn bits); status is DSH_OK, ERR_UNSTABLE (DT above the stability
    limit) or ERR_PARAM (FW wider than the grid), as the reference's stops."""
    vs = np.ascontiguousarray(vs, np.float32)
    rho = np.ascontiguousarray(rho, np.float32)
    ny, nx = vs.shape
    l = len(fl)
    q = np.ascontiguousarray(qs, np.float32) if l > 0 else None
    flv = (C.c_float * 8)(*fl)
    out = (C.c_float * 4)()
    warn = C.c_int(0)
    L = lib()
    L.dsh_check_fd.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_int,
                               C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]
    rc = L.dsh_check_fd(nx, ny, l, C.cast(flv, C.c_void_p), dh, dt, ts, fdorder, maxrelerror, fw, vs.ctypes.data,
                        rho.ctypes.data, q.ctypes.data if q is not None else None, C.cast(out, C.c_void_p),
                        C.byref(warn))
    vals = dict(zip(("cmin", "cmax", "dtstab", "dhstab"), (np.float32(v) for v in out)))
    return rc, vals, warn.value
