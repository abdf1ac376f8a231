"""The host-side functions of the reference-signature layer (libdsh_compat.so:
seismo_ssg, hess_save, hessian, zero_fdveps, zero_fdveps_visc, psource) are a
drop-in for the reference's own: the reference's per-shot loops run once with
the reference's functions and once with the library's swapped in through the
C ABI, on the same Numerical-Recipes arrays and globals, and every output must
be bit-identical.  These functions never touch a GPU (the velocity and stress
updates stay the reference's here; tests/test_gpu_compat.py swaps those)."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O
from conftest import golden, oracle_model

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
AUX = ("seismo_ssg", "hess_save", "hessian", "zero_fdveps", "zero_fdveps_visc", "psource")

pytestmark = pytest.mark.skipif(not O.available("ref"), reason="reference not compiled here")


def _libs():
    ref = C.CDLL(os.path.join(O.REF_DIR, "libdenise_ref.so"), mode=C.RTLD_GLOBAL)   # defines the globals
    comp = C.CDLL(os.path.join(ROOT, "denise-sh_b200", "libdsh_compat.so"))
    return ref, comp


def _swap(ref, comp, on):
    if on:
        ptr = lambda f: C.c_void_p(C.cast(getattr(comp, f), C.c_void_p).value)
        ref.refh_set_impl_aux(*[ptr(f) for f in AUX])
    else:
        ref.refh_set_impl_aux(*([None] * len(AUX)))


def _shot_loops(d):
    """Forward with the Hessian (hess_save every step, hessian at the end),
    then forward with storage, residual, adjoint and eprecond scaling."""
    m = oracle_model(d)
    o = O.Oracle(m, "ref")
    out = {"seis_h": o.forward(d["srcpos"], d["recpos"], hessian=True)}
    out["hess_vs"], out["hess_rho"] = o.hessian_out()
    for k in ("vy", "sxy", "syz", "uy", "uyx", "vyp1"):
        out["fwd_" + k] = o.field(k)
    g = o.shot_gradient(d["srcpos"], d["recpos"], d["obs"])
    out.update({k: g[k] for k in ("seis", "res", "Ws", "Wr", "We", "g_u", "g_rho")})
    for k in ("vy", "sxy", "syz", "uy", "uyx", "vyp1"):
        out["adj_" + k] = o.field(k)
    for l in range(m.l):
        out[f"adj_r{l}"], out[f"adj_q{l}"] = o.field("r", l), o.field("q", l)
    o.close()
    return out


@pytest.mark.parametrize("name", ["elastic_fd4_fs", "elastic_fd2_pml", "visc_fd8_L2", "visc_fd6_L3_pml",
                                  "visc_fd10_L1", "elastic_fd12_fs"])
def test_host_functions_are_drop_in(name):
    ref, comp = _libs()
    d = golden(name)
    _swap(ref, comp, False)
    base = _shot_loops(d)
    _swap(ref, comp, True)
    try:
        lib = _shot_loops(d)
    finally:
        _swap(ref, comp, False)
    for k in base:
        assert np.array_equal(lib[k], base[k]), k
    # and both equal the fixtures the reference wrote
    assert np.array_equal(lib["seis"], d["seis"])
    assert np.array_equal(lib["hess_vs"], d["hess_vs"]) and np.array_equal(lib["hess_rho"], d["hess_rho"])


def test_zeroing_clears_dirty_state():
    """zero_fdveps(_visc) must clear a state left non-zero by a previous
    shot: run a gradient, then a second one with the library's zeroing; the
    second must equal a fresh reference run."""
    ref, comp = _libs()
    d = golden("visc_fd6_L3_pml")
    _swap(ref, comp, False)
    fresh = _shot_loops(d)
    m = oracle_model(d)
    _swap(ref, comp, True)
    try:
        o = O.Oracle(m, "ref")
        o.shot_gradient(d["srcpos"], d["recpos"], d["obs"] * np.float32(0.5))     # leaves every field dirty
        g = o.shot_gradient(d["srcpos"], d["recpos"], d["obs"])
        o.close()
    finally:
        _swap(ref, comp, False)
    for k in ("seis", "Ws", "Wr", "g_u", "g_rho"):
        assert np.array_equal(g[k], fresh[k]), k


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_psource_matches_reference(seed):
    """psource (src/psource.c:9-38, P-SV, not linked into the SH program) on
    random fields and signals, at the first, an inner and the last step, with
    two sources on one point."""
    ref, comp = _libs()
    d = golden("elastic_fd4_fs")
    m = oracle_model(d)
    rng = np.random.default_rng(seed)
    nsrc = 3
    sp = np.zeros((8, nsrc), np.float32)
    sp[0] = rng.integers(1, m.nx + 1, nsrc)
    sp[1] = rng.integers(1, m.ny + 1, nsrc)
    sp[:, 2] = sp[:, 1]                                  # sources 2 and 3 share a point
    sig = rng.standard_normal((nsrc, m.nt)).astype(np.float32)
    sxx = rng.standard_normal((m.ny, m.nx)).astype(np.float32)
    syy = rng.standard_normal((m.ny, m.nx)).astype(np.float32)
    o = O.Oracle(m, "ref")
    try:
        for nt in (1, m.nt // 2, m.nt):
            _swap(ref, comp, False)
            a = o.psource(nt, sxx, syy, sp, sig)
            _swap(ref, comp, True)
            b = o.psource(nt, sxx, syy, sp, sig)
            _swap(ref, comp, False)
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), nt
            assert not np.array_equal(a[0], sxx)
    finally:
        _swap(ref, comp, False)
        o.close()
