"""The reference-signature layer (libdsh_compat.so) is a drop-in for the
reference's own functions: the reference's per-shot loops (forward with
storage, residual, adjoint with correlation, eprecond) run once with the
reference's update_v_PML / update_s_*_PML / eprecond / eprecond1 and once
with the library's, on the same Numerical-Recipes arrays and globals; every
output must be bit-identical (and equal to the golden fixtures)."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O
from conftest import golden, oracle_model

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _libs():
    ref = C.CDLL(os.path.join(O.REF_DIR, "libdenise_ref.so"), mode=C.RTLD_GLOBAL)   # defines the globals
    comp = C.CDLL(os.path.join(ROOT, "denise-sh_b200", "libdsh_compat.so"))
    return ref, comp


def _run(d):
    m = oracle_model(d)
    o = O.Oracle(m, "ref")
    g = o.shot_gradient(d["srcpos"], d["recpos"], d["obs"])
    out = {k: g[k] for k in ("seis", "res", "Ws", "Wr", "We", "g_u", "g_rho")}
    out["l2"] = g["l2"]
    for k in ("vy", "sxy", "syz", "uy", "uyx", "vyp1"):
        out["end_" + k] = o.field(k)
    o.close()
    return out


@pytest.mark.skipif(not O.available("ref"), reason="reference not compiled here")
@pytest.mark.parametrize("name", ["elastic_fd4_fs", "elastic_fd2_pml", "visc_fd8_L2", "visc_fd6_L3_pml",
                                  "elastic_fd12_fs"])
def test_compat_layer_is_drop_in(name):
    ref, comp = _libs()
    d = golden(name)
    ref.refh_set_impl(None, None, None, None, None)
    base = _run(d)
    ptr = lambda f: C.cast(getattr(comp, f), C.c_void_p).value
    ref.refh_set_impl(C.c_void_p(ptr("update_v_PML")), C.c_void_p(ptr("update_s_elastic_PML")),
                      C.c_void_p(ptr("update_s_visc_PML")), C.c_void_p(ptr("eprecond")), C.c_void_p(ptr("eprecond1")))
    try:
        gpu = _run(d)
    finally:
        ref.refh_set_impl(None, None, None, None, None)
    for k in base:
        assert np.array_equal(np.asarray(gpu[k]), np.asarray(base[k])), k
    assert np.array_equal(gpu["seis"], d["seis"])
    assert np.array_equal(gpu["g_u"], d["g_u"])


def _use_compat(ref, comp):
    ptr = lambda f: C.c_void_p(C.cast(getattr(comp, f), C.c_void_p).value)
    ref.refh_set_impl(ptr("update_v_PML"), ptr("update_s_elastic_PML"), ptr("update_s_visc_PML"), ptr("eprecond"),
                      ptr("eprecond1"))


def _unstable_forward(d):
    """The reference's forward loop with DT 20x beyond the stability limit."""
    d = dict(d, dt=np.float32(d["dt"] * 20))
    o = O.Oracle(oracle_model(d), "ref")
    o.forward(d["srcpos"], d["recpos"])
    o.close()


@pytest.mark.skipif(not O.available("ref"), reason="reference not compiled here")
def test_compat_status_reports_instability():
    """The layer keeps the reference's void signatures; dsh_compat_status
    reports (and clears) the first error: none after a stable run,
    DSH_ERR_UNSTABLE after a run whose wavefield became non-finite."""
    ref, comp = _libs()
    comp.dsh_compat_status.restype = C.c_int
    d = golden("elastic_fd4_fs")
    _use_compat(ref, comp)
    try:
        comp.dsh_compat_status()
        _run(d)
        assert comp.dsh_compat_status() == 0
        _unstable_forward(d)
        assert comp.dsh_compat_status() == -4            # DSH_ERR_UNSTABLE
        assert comp.dsh_compat_status() == 0             # cleared by the read
    finally:
        ref.refh_set_impl(None, None, None, None, None)


@pytest.mark.skipif(os.environ.get("DSH_COMPAT_ABORT") != "1", reason="run by the abort-mode test in a child")
def test_compat_abort_mode_child():
    ref, comp = _libs()
    _use_compat(ref, comp)
    _unstable_forward(golden("elastic_fd4_fs"))


@pytest.mark.skipif(not O.available("ref"), reason="reference not compiled here")
def test_compat_abort_mode_exits_like_the_reference():
    """With DSH_COMPAT_ABORT=1 an error ends the process as the reference's
    err() does: the run-time error banner with the message on stdout and
    exit status 1 (in a child process)."""
    import subprocess
    import sys

    env = dict(os.environ, DSH_COMPAT_ABORT="1")
    code = ("import sys; sys.argv=['x']; import pytest; "
            "sys.exit(pytest.main(['-q', '-s', '-p', 'no:cacheprovider', '-m', 'gpu', "
            "'tests/test_gpu_compat.py::test_compat_abort_mode_child']))")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 1, out.stdout[-2000:] + out.stderr[-2000:]
    assert "R U N - T I M E  E R R O R" in out.stdout and "Simulation is unstable" in out.stdout


@pytest.mark.skipif(not O.available("ref"), reason="reference not compiled here")
@pytest.mark.parametrize("name", ["elastic_fd4_fs", "visc_fd8_L2", "visc_fd6_L3_pml", "visc_fd10_L1"])
def test_every_layer1_function_swapped_at_once(name):
    """All of the layer's functions in the reference's loops at the same time
    (velocity, stress, eprecond, eprecond1 on the GPU; seismo_ssg, hess_save,
    hessian, zero_fdveps(_visc) on the host), including a forward pass with the
    Hessian: bit-identical to the reference's own functions."""
    from test_compat_host import _shot_loops, _swap

    ref, comp = _libs()
    d = golden(name)
    ref.refh_set_impl(None, None, None, None, None)
    _swap(ref, comp, False)
    base = _shot_loops(d)
    _use_compat(ref, comp)
    _swap(ref, comp, True)
    try:
        gpu = _shot_loops(d)
        assert comp.dsh_compat_status() == 0
    finally:
        ref.refh_set_impl(None, None, None, None, None)
        _swap(ref, comp, False)
    for k in base:
        assert np.array_equal(gpu[k], base[k]), k
    assert np.array_equal(gpu["hess_vs"], d["hess_vs"]) and np.array_equal(gpu["hess_rho"], d["hess_rho"])
