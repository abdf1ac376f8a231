"""The C-ABI library loads without a GPU, exports every entry point that
include/dsh.h declares, and rejects invalid parameters with DSH_ERR_PARAM
before touching a device."""
import ctypes as C
import os
import re

import pytest

import dsh

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    """Function names declared in an include/ header."""
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"#define[^\n]*", "", src)
    return sorted(set(re.findall(r"\b(?:void|int|float|double|dsh_ctx \*|dsh_batch \*|const char \*)\s*\**\s*([A-Za-z_][A-Za-z0-9_]*)\s*\(", src)))


def _library_for(header):
    if header == "dsh_compat.h":
        import oracle as O

        if not O.available("ref"):
            pytest.skip("the compat layer resolves the reference's globals from the program that loads it")
        C.CDLL(os.path.join(O.REF_DIR, "libdenise_ref.so"), mode=C.RTLD_GLOBAL)
        return C.CDLL(os.path.join(ROOT, "denise-sh_b200", "libdsh_compat.so"))
    if header == "dsh_nn.h":
        return C.CDLL(os.path.join(ROOT, "denise-sh_b200", "libdsh_nn.so"))
    return dsh.lib()


@pytest.mark.parametrize("header", sorted(f for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")))
def test_every_declared_symbol_is_exported(header):
    lib = _library_for(header)
    names = declared(header)
    assert len(names) >= 4, (header, names)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layout():
    # dsh_params / dsh_shot / dsh_stats as the header lays them out on x86-64
    assert C.sizeof(dsh.Params) == 120
    assert dsh.Params.mem_budget.offset == 104
    assert dsh.Params.ckpt_every.offset == 112
    assert C.sizeof(dsh.ShotC) == 40
    assert C.sizeof(dsh.Stats) == 56


@pytest.mark.parametrize("bad", [dict(fdorder=5), dict(fdorder=14), dict(maxrelerror=5), dict(l=5), dict(nx=0),
                                 dict(fw=-1), dict(fw=400), dict(dt=0.0), dict(eprecond=2), dict(max_shots=0),
                                 dict(quellart=7), dict(l=2, fl=(10.0,)), dict(ckpt_every=-1)])
def test_invalid_params_rejected_before_device_use(bad):
    kw = dict(nx=64, ny=32, nt=10, dh=0.5, dt=1e-4, l=0)
    kw.update(bad)
    fl = kw.pop("fl", None)
    p = dsh.make_params(**kw, **({"fl": fl} if fl else {}))
    if kw.get("l", 0) == 2 and fl:
        p.fl[1] = 0.0
    st = C.c_int(0)
    h = dsh.lib().dsh_create(C.byref(p), 0, C.byref(st))
    assert not h
    assert st.value == -1


def test_error_strings():
    lib = dsh.lib()
    for code in (0, -1, -2, -3, -4, -5, -6):
        assert lib.dsh_error_string(code)


def test_batch_rejects_unsupported_models_without_gpu():
    """Parameter checks of dsh_batch_create run before any CUDA call."""
    import ctypes as C

    import dsh

    ok = dsh.make_params(64, 48, 100, 0.5, 1e-4, fdorder=4)
    for bad in (dict(fdorder=10), dict(fdorder=8, l=3), dict(fdorder=2)):
        p = dsh.make_params(64, 48, 100, 0.5, 1e-4, **bad)
        arr = (dsh.Params * 2)(ok, p)
        st = C.c_int(0)
        assert not dsh.lib().dsh_batch_create(arr, 2, 0, C.byref(st))
        assert st.value == -1
    st = C.c_int(0)
    assert not dsh.lib().dsh_batch_create(None, 0, 0, C.byref(st))
    assert st.value == -1
