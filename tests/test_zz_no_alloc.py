"""The allocation-free residual entry point (dsh_residual_noalloc) gives the
same L2 misfit as the regular gradient path and the same time-reversed
residual as the oracle, on two calls in a row.

It serves callers that cannot allocate device memory (their device memory is
owned by their own pool, or the misfit runs in a loop that must not touch the
allocator): its reduction scratch is a fixed array inside the library, so this
test also checks that back-to-back calls, which reuse that array, agree.
Kept in a file that pytest collects last."""
import numpy as np
import pytest

import dsh
import oracle as O
from conftest import golden, oracle_model

pytestmark = pytest.mark.gpu


def _l2_tol(n):
    return max(n - 1, 1) * 2.0 ** -24


def test_noalloc_residual_matches_existing_paths():
    import torch

    d = golden("visc_fd8_L2")
    shot = dsh.Shot(d["srcpos"], d["recpos"])
    p = dsh.make_params(nx=int(d["nx"]), ny=int(d["ny"]), nt=int(d["nt"]), dh=float(d["dh"]), dt=float(d["dt"]),
                        fdorder=int(d["fdorder"]), fw=int(d["fw"]), free_surf=int(d["free_surf"]), l=int(d["l"]),
                        fl=tuple(float(x) for x in d["fl"]), damping=float(d["damping"]), fpml=float(d["fpml"]))
    with dsh.Engine(p) as e:
        e.set_model(d["vs"], d["rho"], d["qs"])
        syn = e.forward([shot])[0]
        obs_list = [d["obs"], (d["obs"] * np.float32(0.5)).astype(np.float32)]
        l2_existing = [e.gradient([shot], [ob])["l2"] for ob in obs_list]

    m = oracle_model(d)
    ntr, nt = syn.shape
    syn_d = torch.from_numpy(np.ascontiguousarray(syn)).cuda()
    for ob, l2_ref in zip(obs_list, l2_existing):          # two calls in a row, reusing the static scratch
        obs_d = torch.from_numpy(np.ascontiguousarray(ob)).cuda()
        res_d = torch.full((ntr, nt), np.nan, dtype=torch.float32, device="cuda")
        l2_d = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
        dsh.residual_noalloc(1, ntr, nt, syn_d.data_ptr(), obs_d.data_ptr(), res_d.data_ptr(), l2_d.data_ptr())
        torch.cuda.synchronize()
        l2 = float(l2_d.item())
        assert abs(l2 - l2_ref) <= _l2_tol(syn.size) * abs(l2_ref), (l2, l2_ref)
        o = O.Oracle(m, "port")
        o.forward(shot.srcpos, shot.recpos)
        res_ref, _ = o.residual(ob)
        o.close()
        assert np.array_equal(res_d.cpu().numpy(), res_ref)


def test_noalloc_rejects_too_many_shots():
    import torch

    n = dsh.NOALLOC_MAX_SHOTS + 1
    x = torch.zeros((n, 2, 3), dtype=torch.float32, device="cuda")
    l2 = torch.zeros(n, dtype=torch.float64, device="cuda")
    with pytest.raises(dsh.DshError) as ei:
        dsh.residual_noalloc(n, 2, 3, x.data_ptr(), x.data_ptr(), x.data_ptr(), l2.data_ptr())
    assert ei.value.code == -1
