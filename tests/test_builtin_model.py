"""The reference's built-in start models (READMOD=0, src/denise.c:609-615)
from dsh_builtin_model against the reference's own model() of
src/model_grad_visc.c and model_elastic() of src/check_start.c compiled into
the oracle: identical vs and rho, Qs whose taus = 2/Qs equals the
reference's, and the model file written with dsh_write_model byte-identical
to the one the reference writes."""
import numpy as np
import pytest

import oracle as O
from dsh import io

ref_only = pytest.mark.skipif(not O.available("ref"), reason="reference build not present")


@ref_only
@pytest.mark.parametrize("l,nx,ny,dh", [(3, 37, 29, 0.25), (1, 12, 200, 0.5), (2, 5, 64, 1.3), (0, 23, 17, 0.5)])
def test_builtin_model_matches_reference(tmp_path, l, nx, ny, dh):
    fl = [5.0, 20.0, 80.0][:l]
    vs_r, rho_r, taus_r, eta_r, vs_file = O.builtin_model(l, nx, ny, dh, 2e-4, fl)
    vs, rho, qs = io.builtin_model(l, nx, ny, dh)
    assert np.array_equal(vs, vs_r) and np.array_equal(rho, rho_r)
    if l > 0:
        assert np.array_equal((2.0 / qs.astype(np.float64)).astype(np.float32), taus_r)    # readmod.c:99
        assert np.all(np.diff(vs[:, 0]) > 0)                                                # velocity grows with depth
    else:
        assert qs is None and np.all(vs == np.float32(164.0))
    path = str(tmp_path / "vs.bin")
    io.write_model(path, vs)
    assert open(path, "rb").read() == vs_file


def test_builtin_model_rejects_bad_arguments():
    import dsh

    with pytest.raises(dsh.DshError):
        io.builtin_model(2, 0, 10, 0.5)
