"""Checkpoint-and-recompute: with a device-memory budget below full storage
the forward pass keeps only state checkpoints every C steps and the adjoint
recomputes each segment; the gradient must be bit-identical to full storage
(and therefore to the reference), including a partial last segment and
multi-slot batches."""
import numpy as np
import pytest

import dsh
import oracle as O
from conftest import oracle_model
from test_gpu_parity import _case, _oracle_gradient, engine_from, l2_tol

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nt,L,fdo,max_shots", [(161, 2, 8, 2), (150, 0, 4, 1), (97, 3, 6, 3)])
def test_checkpointed_gradient_equals_full_storage(nt, L, fdo, max_shots):
    d, shots = _case(300 + nt, nx=61, ny=45, nt=nt, fdo=fdo, L=L, fs=1, fw=8, nshots=3)
    m = oracle_model(d)
    obs = []
    for sh in shots:
        o = O.Oracle(m, "port")
        obs.append((o.forward(sh.srcpos, sh.recpos) * np.float32(0.8)).astype(np.float32))
        o.close()
    with engine_from(d, max_shots=max_shots) as e:
        full = e.gradient(shots, obs, want_seis=True, want_energy=True)
        st_full = e.stats()
    budget = st_full["storage_bytes"] // 2           # below full storage: forces checkpoints
    with engine_from(d, max_shots=max_shots, mem_budget=budget) as e:
        ck = e.gradient(shots, obs, want_seis=True, want_energy=True)
        st_ck = e.stats()
    assert st_full["checkpoint_interval"] == 0
    assert st_ck["checkpoint_interval"] > 0 and nt % st_ck["checkpoint_interval"] != 0
    assert st_ck["storage_bytes"] <= budget
    for k in ("g_vs", "g_rho", "Ws", "Wr"):
        assert np.array_equal(ck[k], full[k]), k
    for a, b in zip(ck["seis"], full["seis"]):
        assert np.array_equal(a, b)
    assert ck["l2"] == full["l2"]
    gv, gr, l2, _ = _oracle_gradient(d, shots, obs)
    assert np.array_equal(ck["g_vs"], gv)
    assert np.array_equal(ck["g_rho"], gr)


def test_budget_too_small_is_reported():
    d, shots = _case(400, nx=40, ny=30, nt=60, fdo=4, L=0, fs=1, fw=6)
    with engine_from(d, mem_budget=1024) as e:
        with pytest.raises(dsh.DshError) as ei:
            e.gradient(shots, [np.zeros((shots[0].ntr, 60), np.float32)])
        assert ei.value.code == -3


def test_64_shots_one_launch_checkpointed():
    """The batched-gradient layout: 64 shots advance in one launch per
    half-step (grid z = shot) with checkpoints; the shot sum is bit-identical
    to the reference's shot loop."""
    nt = 130
    d, _ = _case(964, nx=72, ny=40, nt=nt, fdo=8, L=2, fs=1, fw=8, nshots=1)
    shots = []
    for k in range(64):           # 64 sources along the surface, receivers within a few points of each
        sp = np.array([[4 + k], [2], [0], [-0.01], [60.0], [1.0], [0], [3]], np.float32)
        xi = np.clip(4 + k + np.array([-3, -1, 1, 2, 4]), 1, 72)
        shots.append(dsh.Shot(sp, np.array([xi, [1, 1, 2, 3, 1]], np.int32)))
    m = oracle_model(d)
    obs = []
    for sh in shots:
        o = O.Oracle(m, "port")
        obs.append((o.forward(sh.srcpos, sh.recpos) * np.float32(0.9)).astype(np.float32))
        o.close()
    with engine_from(d, max_shots=64) as e:
        full = e.gradient(shots, obs)
        st_full = e.stats()
    with engine_from(d, max_shots=64, mem_budget=st_full["storage_bytes"] // 2) as e:
        ck = e.gradient(shots, obs)
        st = e.stats()
    assert st["checkpoint_interval"] > 0
    gv, gr, l2, _ = _oracle_gradient(d, shots, obs)
    for out in (full, ck):
        assert np.array_equal(out["g_vs"], gv)
        assert np.array_equal(out["g_rho"], gr)
        assert abs(out["l2"] - l2) <= l2_tol(sum(o.size for o in obs)) * abs(l2)
