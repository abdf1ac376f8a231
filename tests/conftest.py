import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "denise-sh_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the CUDA path")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Make sure the in-tree libraries exist (they are prebuilt when the tree is
    shipped to a GPU host; here they are built on first use)."""
    import __graft_entry__ as ge

    need = [os.path.join(ROOT, "denise-sh_b200", "libdsh.so"), os.path.join(ROOT, "oracle", "_ref", "libdsh_oracle.so")]
    if not all(os.path.exists(p) for p in need):
        ge.build()
    yield


def golden(name):
    import numpy as np

    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def oracle_model(d):
    """oracle.Model from a golden fixture dict."""
    from oracle import Model

    return Model(nx=int(d["nx"]), ny=int(d["ny"]), nt=int(d["nt"]), dh=float(d["dh"]), dt=float(d["dt"]),
                 vs=d["vs"], rho=d["rho"], qs=d["qs"], fdorder=int(d["fdorder"]), fw=int(d["fw"]),
                 free_surf=int(d["free_surf"]), l=int(d["l"]), fl=tuple(float(x) for x in d["fl"]),
                 fpml=float(d["fpml"]), damping=float(d["damping"]))
