"""The allocation-free residual entry point (dsh_residual_noalloc) gives the
same per-shot L2 misfit as the regular gradient path and the same
time-reversed residual as the oracle, on calls in a row.

It serves callers that cannot allocate device memory (their device memory is
owned by their own pool, or the misfit runs in a loop that must not touch the
allocator): its reduction scratch is a fixed array inside the library, so this
test also checks that back-to-back calls, which reuse that array, agree.  The
entry point partitions every shot's samples over the same 296 blocks and sums
them in the same order as dsh_gradient's residual step, so the misfits must be
equal, not merely close.  Kept in a file that pytest collects last."""
import numpy as np
import pytest

import dsh
import oracle as O
from conftest import golden, oracle_model

pytestmark = pytest.mark.gpu


def _params(d, max_shots=1):
    return dsh.make_params(nx=int(d["nx"]), ny=int(d["ny"]), nt=int(d["nt"]), dh=float(d["dh"]), dt=float(d["dt"]),
                           fdorder=int(d["fdorder"]), fw=int(d["fw"]), free_surf=int(d["free_surf"]), l=int(d["l"]),
                           fl=tuple(float(x) for x in d["fl"]), damping=float(d["damping"]), fpml=float(d["fpml"]),
                           max_shots=max_shots)


def _shots(d, n):
    """n shots of the fixture's model with the source moved along the surface."""
    nx = int(d["nx"])
    out = []
    for k in range(n):
        sp = np.array(d["srcpos"], np.float32, copy=True)
        sp[0, :] = 2 + (3 * k) % (nx - 3)
        out.append(dsh.Shot(sp, d["recpos"]))
    return out


def _noalloc(syn, obs):
    """dsh_residual_noalloc on stacked [nshots][ntr][nt] device arrays."""
    import torch

    ns, ntr, nt = syn.shape
    syn_d = torch.from_numpy(np.ascontiguousarray(syn)).cuda()
    obs_d = torch.from_numpy(np.ascontiguousarray(obs)).cuda()
    res_d = torch.full((ns, ntr, nt), np.nan, dtype=torch.float32, device="cuda")
    l2_d = torch.full((ns,), np.nan, dtype=torch.float64, device="cuda")
    dsh.residual_noalloc(ns, ntr, nt, syn_d.data_ptr(), obs_d.data_ptr(), res_d.data_ptr(), l2_d.data_ptr())
    torch.cuda.synchronize()
    return res_d.cpu().numpy(), l2_d.cpu().numpy()


def _oracle_residual(m, shot, ob):
    o = O.Oracle(m, "port")
    o.forward(shot.srcpos, shot.recpos)
    res, _ = o.residual(ob)
    o.close()
    return res


def test_noalloc_residual_matches_existing_paths():
    d = golden("visc_fd8_L2")
    shot = dsh.Shot(d["srcpos"], d["recpos"])
    obs_list = [d["obs"], (d["obs"] * np.float32(0.5)).astype(np.float32)]
    with dsh.Engine(_params(d)) as e:
        e.set_model(d["vs"], d["rho"], d["qs"])
        syn = e.forward([shot])[0]
        l2_existing = [e.gradient([shot], [ob])["l2"] for ob in obs_list]
    m = oracle_model(d)
    for ob, l2_ref in zip(obs_list, l2_existing):          # two calls in a row, reusing the static scratch
        res, l2 = _noalloc(syn[None], ob[None])
        assert float(l2[0]) == l2_ref, (float(l2[0]), l2_ref)
        assert np.array_equal(res[0], _oracle_residual(m, shot, ob))


@pytest.mark.parametrize("nshots", [3, 64])
def test_noalloc_multi_shot(nshots):
    """Several shots per call, each with its own observed data: every shot's
    misfit equals the gradient path's per-shot misfit and every residual the
    oracle's; the call is made twice in a row."""
    d = golden("elastic_fd4_fs")
    shots = _shots(d, nshots)
    rng = np.random.default_rng(nshots)
    with dsh.Engine(_params(d, max_shots=nshots)) as e:
        e.set_model(d["vs"], d["rho"], None)
        syn = np.stack(e.forward(shots))
        obs = np.stack([(s * np.float32(rng.uniform(0.3, 0.9)) + np.float32(1e-4) * rng.standard_normal(s.shape))
                        .astype(np.float32) for s in syn])
        e.gradient(shots, list(obs))
        l2_existing = e.shot_misfits(nshots)
    m = oracle_model(d)
    check = sorted({0, nshots // 2, nshots - 1})
    for _ in range(2):
        res, l2 = _noalloc(syn, obs)
        assert np.array_equal(l2, l2_existing), (l2, l2_existing)
        for s in check:
            assert np.array_equal(res[s], _oracle_residual(m, shots[s], obs[s])), s


def test_noalloc_rejects_too_many_shots():
    import torch

    n = dsh.NOALLOC_MAX_SHOTS + 1
    x = torch.zeros((n, 2, 3), dtype=torch.float32, device="cuda")
    y = torch.zeros((n, 2, 3), dtype=torch.float32, device="cuda")
    l2 = torch.zeros(n, dtype=torch.float64, device="cuda")
    with pytest.raises(dsh.DshError) as ei:
        dsh.residual_noalloc(n, 2, 3, x.data_ptr(), x.data_ptr(), y.data_ptr(), l2.data_ptr())
    assert ei.value.code == -1


def test_noalloc_rejects_in_place_residual():
    """The residual is time-reversed, so it cannot overwrite syn or obs: such
    a call is rejected before any launch."""
    import torch

    x = torch.ones((1, 4, 10), dtype=torch.float32, device="cuda")
    y = torch.zeros((1, 4, 10), dtype=torch.float32, device="cuda")
    l2 = torch.zeros(1, dtype=torch.float64, device="cuda")
    for res, syn, obs in ((x, x, y), (y, x, y), (x[:, 1:], x[:, :-1], y[:, :-1])):
        with pytest.raises(dsh.DshError) as ei:
            dsh.residual_noalloc(1, res.shape[1], 10, syn.data_ptr(), obs.data_ptr(), res.data_ptr(), l2.data_ptr())
        assert ei.value.code == -1
    assert float(x.sum()) == 40.0 and float(y.sum()) == 0.0
