"""The reference's file formats through libdsh.so (include/dsh_io.h):
.inp / .json parameter files, FWI workflow table, source and receiver files,
float32 model files and SU seismograms."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import Params, _check, lib

PATH = 256


class Inp(C.Structure):
    """Mirror of ``dsh_inp``."""
    _fields_ = [(n, C.c_int) for n in ("nprocx", "nprocy", "fdorder", "maxrelerror", "nx", "ny")] + \
               [(n, C.c_float) for n in ("dh", "time", "dt")] + \
               [("quellart", C.c_int), ("quelltyp", C.c_int)] + \
               [(n, C.c_float) for n in ("angle", "plane_wave_depth", "phi")] + \
               [("signal_file", C.c_char * PATH), ("ts", C.c_float), ("srcrec", C.c_int),
                ("source_file", C.c_char * PATH), ("run_multiple_shots", C.c_int), ("readmod", C.c_int),
                ("mfile", C.c_char * PATH), ("l", C.c_int), ("fl", C.c_float * 8), ("tau", C.c_float),
                ("free_surf", C.c_int), ("fw", C.c_int), ("damping", C.c_float), ("fpml", C.c_float),
                ("boundary", C.c_int), ("seismo", C.c_int), ("readrec", C.c_int), ("rec_file", C.c_char * PATH),
                ("refrec", C.c_float * 2), ("ndt", C.c_int), ("seis_format", C.c_int),
                ("seis_file_vy", C.c_char * PATH), ("data_dir", C.c_char * PATH), ("invmat1", C.c_int),
                ("invmat", C.c_int), ("quelltypb", C.c_int), ("npower", C.c_float), ("k_max_pml", C.c_float),
                ("hessian", C.c_int), ("fc_hessian", C.c_float), ("grad_method", C.c_int), ("lnorm", C.c_int),
                ("dtinv", C.c_int), ("lines", C.c_int)]


class Stage(C.Structure):
    """Mirror of ``dsh_stage`` (one workflow row)."""
    _fields_ = [("pro", C.c_float), ("time_filt", C.c_int), ("fc_start", C.c_float), ("fc_end", C.c_float),
                ("order", C.c_int), ("timewin", C.c_int), ("gamma", C.c_float), ("twlength_minus", C.c_float),
                ("twlength_plus", C.c_float), ("inv_vp_iter", C.c_int), ("inv_vs_iter", C.c_int),
                ("inv_rho_iter", C.c_int), ("spatfilter", C.c_int), ("wd_damp1", C.c_float), ("wd_damp", C.c_float),
                ("eprecond", C.c_int), ("lnorm", C.c_int), ("inv_stf", C.c_int), ("offsetc_stf", C.c_float),
                ("eps_stf", C.c_float), ("normalize", C.c_int), ("offset_mute", C.c_int), ("offsetc", C.c_float),
                ("scalerho", C.c_float)]


def _b(s):
    return s.encode() if isinstance(s, str) else s


_configured = False


def _lib():
    global _configured
    L = lib()
    if not _configured:
        vp, cp, ci, cf = C.c_void_p, C.c_char_p, C.c_int, C.c_float
        L.dsh_read_inp.argtypes = [cp, vp]
        L.dsh_read_json.argtypes = [cp, vp]
        L.dsh_inp_params.argtypes = [vp, vp]
        L.dsh_read_workflow.argtypes = [cp, ci, vp]
        L.dsh_read_sources.argtypes = [cp, cf, ci, ci, ci, vp, vp, vp]
        L.dsh_read_receivers.argtypes = [cp, cf, vp, ci, vp, vp]
        L.dsh_read_model.argtypes = [cp, ci, ci, ci, vp, vp, vp]
        L.dsh_write_model.argtypes = [cp, ci, ci, vp]
        L.dsh_builtin_model.argtypes = [ci, ci, ci, cf, vp, vp, vp]
        L.dsh_write_su.argtypes = [cp, ci, ci, vp, vp, vp, cf, cf, cf, cf, ci, vp]
        L.dsh_read_su.argtypes = [cp, ci, ci, vp]
        L.dsh_stager_create.restype = vp
        L.dsh_stager_create.argtypes = [ci, C.c_longlong, ci, C.POINTER(ci)]
        L.dsh_stager_submit.argtypes = [vp, ci, C.POINTER(cp), vp, ci]
        L.dsh_stager_acquire.argtypes = [vp, vp, C.POINTER(vp), C.POINTER(C.c_longlong)]
        L.dsh_stager_acquire_host.argtypes = [vp, C.POINTER(vp), C.POINTER(C.c_longlong)]
        L.dsh_stager_release.argtypes = [vp, vp]
        L.dsh_stager_destroy.argtypes = [vp]
        _configured = True
    return L


def read_inp(path: str) -> Inp:
    out = Inp()
    _check(_lib().dsh_read_inp(_b(path), C.byref(out)), "dsh_read_inp")
    return out


def read_json(path: str) -> Inp:
    out = Inp()
    _check(_lib().dsh_read_json(_b(path), C.byref(out)), "dsh_read_json")
    return out


def params_from(inp: Inp, **overrides) -> Params:
    p = Params()
    _check(_lib().dsh_inp_params(C.byref(inp), C.byref(p)), "dsh_inp_params")
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def read_workflow(path: str, stage: int) -> Stage:
    out = Stage()
    _check(_lib().dsh_read_workflow(_b(path), stage, C.byref(out)), "dsh_read_workflow")
    return out


def read_sources(path: str, dh: float, nx: int, ny: int, max_sources: int = 4096):
    sp = np.zeros((8, max_sources), np.float32)
    sm = np.zeros((2, max_sources), np.float32)
    n = C.c_int(0)
    _check(_lib().dsh_read_sources(_b(path), C.c_float(dh), nx, ny, max_sources, C.byref(n), sp.ctypes.data,
                                  sm.ctypes.data), "dsh_read_sources")
    return np.ascontiguousarray(sp[:, :n.value]), np.ascontiguousarray(sm[:, :n.value])


def read_receivers(path: str, dh: float, refrec=(0.0, 0.0), max_receivers: int = 65536):
    rp = np.zeros((2, max_receivers), np.int32)
    ref = (C.c_float * 2)(*refrec)
    n = C.c_int(0)
    _check(_lib().dsh_read_receivers(_b(path), C.c_float(dh), ref, max_receivers, C.byref(n), rp.ctypes.data),
           "dsh_read_receivers")
    return np.ascontiguousarray(rp[:, :n.value])


def read_model(mfile: str, nx: int, ny: int, l: int = 0):
    vs = np.zeros((ny, nx), np.float32)
    rho = np.zeros((ny, nx), np.float32)
    qs = np.zeros((ny, nx), np.float32) if l > 0 else None
    _check(_lib().dsh_read_model(_b(mfile), nx, ny, l, vs.ctypes.data, rho.ctypes.data,
                                qs.ctypes.data if qs is not None else None), "dsh_read_model")
    return vs, rho, qs


def builtin_model(l: int, nx: int, ny: int, dh: float):
    """The reference's start model for READMOD=0 (src/model_grad_visc.c for
    l > 0, src/check_start.c for l == 0): (vs, rho, qs) as [ny, nx] float32,
    qs None when l == 0."""
    vs = np.empty((ny, nx), np.float32)
    rho = np.empty((ny, nx), np.float32)
    qs = np.empty((ny, nx), np.float32) if l > 0 else None
    _check(_lib().dsh_builtin_model(l, nx, ny, dh, vs.ctypes.data, rho.ctypes.data,
                                    qs.ctypes.data if qs is not None else None), "dsh_builtin_model")
    return vs, rho, qs


def write_model(path: str, field) -> None:
    f = np.ascontiguousarray(field, np.float32)
    _check(_lib().dsh_write_model(_b(path), f.shape[1], f.shape[0], f.ctypes.data), "dsh_write_model")


def write_su(path: str, section, recpos, xs: float, ys: float, dh: float, dt: float, ndt: int = 1,
             refrec=(0.0, 0.0), tracl=None) -> None:
    sec = np.ascontiguousarray(section, np.float32)
    rp = np.ascontiguousarray(recpos, np.int32)
    tr = np.ascontiguousarray(tracl, np.int32) if tracl is not None else None
    ref = (C.c_float * 2)(*refrec)
    _check(_lib().dsh_write_su(_b(path), sec.shape[0], sec.shape[1], sec.ctypes.data, rp.ctypes.data,
                              tr.ctypes.data if tr is not None else None, C.c_float(xs), C.c_float(ys),
                              C.c_float(dh), C.c_float(dt), ndt, ref), "dsh_write_su")


def read_su(path: str, ntr: int, ns: int):
    sec = np.zeros((ntr, ns), np.float32)
    _check(_lib().dsh_read_su(_b(path), ntr, ns, sec.ctypes.data), "dsh_read_su")
    return sec


class Stager:
    """Asynchronous reader of observed SU data (dsh_stager): submit batches of
    files, then acquire them in order - on the device (use_device=True: a
    device pointer the given CUDA stream may use once the upload completes)
    or as host arrays - and release each before the next acquire."""

    def __init__(self, nbuf: int, max_floats: int, use_device: bool = True):
        st = C.c_int(0)
        self.h = _lib().dsh_stager_create(nbuf, max_floats, int(use_device), C.byref(st))
        if not self.h:
            _check(st.value or -1, "dsh_stager_create")
        self.device = use_device

    def submit(self, paths, ntr, ns: int) -> None:
        arr = (C.c_char_p * len(paths))(*[_b(p) for p in paths])
        n = np.ascontiguousarray(ntr, np.int32)
        _check(_lib().dsh_stager_submit(self.h, len(paths), arr, n.ctypes.data, ns), "dsh_stager_submit")

    def acquire(self, stream: int | None = None):
        """(device pointer, number of floats) of the oldest batch."""
        ptr, n = C.c_void_p(), C.c_longlong()
        _check(_lib().dsh_stager_acquire(self.h, stream, C.byref(ptr), C.byref(n)), "dsh_stager_acquire")
        return ptr.value, n.value

    def acquire_host(self):
        """A copy of the oldest batch as a float32 array."""
        ptr, n = C.c_void_p(), C.c_longlong()
        _check(_lib().dsh_stager_acquire_host(self.h, C.byref(ptr), C.byref(n)), "dsh_stager_acquire_host")
        return np.ctypeslib.as_array((C.c_float * n.value).from_address(ptr.value)).copy()

    def release(self, stream: int | None = None) -> None:
        _check(_lib().dsh_stager_release(self.h, stream), "dsh_stager_release")

    def close(self) -> None:
        if self.h:
            _lib().dsh_stager_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
