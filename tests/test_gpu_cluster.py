"""The cluster-resident forward-modelling launch (step variant 4): plain
elastic forward modelling of a small grid in one launch, one thread-block
cluster per shot holding the wavefield and the model in its CTAs' shared
memory, halo rows exchanged through distributed shared memory between
hardware cluster barriers.

Bit-exact against the CPU oracle (pinned to the reference's
update_v_PML.c / update_s_elastic_PML.c / seismo_ssg.c) over FDORDER 2-8,
free surface on and off, DH a power of two or not, grid widths that are not
a multiple of 4, strips of 3 to 13 rows (16-CTA clusters) and the 8-CTA
fallback (FDORDER 8 on a 40-row grid), several shots in one launch, and the
500 x 200 x 2000 benchmark case; the end state written back to the slots
equals the kernel pair's; an unstable model reports DSH_ERR_UNSTABLE."""
import numpy as np
import pytest

import dsh
import oracle as O
from conftest import oracle_model
from dsh import configs
from test_gpu_parity import _case, engine_from

pytestmark = pytest.mark.gpu

CLUSTER = dsh.Engine.VARIANTS.index("cluster-resident launch")


def _inside(d, shots):
    """receivers clipped into the grid (the fused sampling lists need every position inside)"""
    out = []
    for sh in shots:
        rec = sh.recpos.copy()
        rec[1] = np.clip(rec[1], 1, int(d["ny"]))
        out.append(dsh.Shot(sh.srcpos, rec))
    return out


def _oracle_forward(d, shot):
    o = O.Oracle(oracle_model(d), "port")
    ref = o.forward(shot.srcpos, shot.recpos)
    o.close()
    return ref


def _run(d, shots, variant, max_shots=1):
    with engine_from(d, max_shots=max_shots) as e:
        e.set_step_variant(variant)
        seis = e.forward(shots)
        st = e.stats()
        end = [{k: e.field(k, shot=s) for k in ("vy", "sxy", "syz")} for s in range(len(shots))]
    return seis, st, end


@pytest.mark.parametrize("fdo", [2, 4, 6, 8])
@pytest.mark.parametrize("nx,ny,fs,dh", [(70, 40, 1, 0.5), (203, 97, 0, 0.6), (500, 200, 1, 0.5)])
def test_cluster_forward_matches_oracle(fdo, nx, ny, fs, dh):
    d, shots = _case(3000 + 10 * fdo + nx, nx=nx, ny=ny, nt=130, fdo=fdo, L=0, fs=fs, fw=10)
    d["dh"] = dh
    shots = _inside(d, shots)
    ref = _oracle_forward(d, shots[0])
    seis, st, end = _run(d, shots, CLUSTER)
    assert np.array_equal(seis[0], ref)
    assert st["kernel_launches"] <= 8          # one cluster launch for all steps (+ counter, transposes)
    _, st_pair, end_pair = _run(d, shots, 0)
    assert st_pair["kernel_launches"] >= 2 * 130
    for k in ("vy", "sxy", "syz"):
        assert np.array_equal(end[0][k], end_pair[0][k]), k


def test_cluster_several_shots_in_one_launch():
    d, shots = _case(3100, nx=150, ny=64, nt=150, fdo=4, L=0, fs=1, fw=10, nshots=3)
    shots = _inside(d, shots)
    seis, st, end = _run(d, shots, CLUSTER, max_shots=3)
    assert st["kernel_launches"] <= 8
    _, _, end_pair = _run(d, shots, 0, max_shots=3)
    for s, sh in enumerate(shots):
        assert np.array_equal(seis[s], _oracle_forward(d, sh)), s
        for k in ("vy", "sxy", "syz"):
            assert np.array_equal(end[s][k], end_pair[s][k]), (s, k)


def test_cluster_benchmark_case_matches_oracle():
    """The 500 x 200, FDORDER 4, NT 2000 elastic forward case in one launch."""
    cfg = configs.config1()
    p = cfg["params"]
    sh = cfg["shots"][0]
    with dsh.Engine(dsh.make_params(**p)) as e:
        e.set_model(cfg["vs"], cfg["rho"], None)
        e.set_step_variant(CLUSTER)
        seis = e.forward([sh])[0]
        assert e.stats()["kernel_launches"] <= 8
    m = O.Model(nx=p["nx"], ny=p["ny"], nt=p["nt"], dh=p["dh"], dt=p["dt"], vs=cfg["vs"], rho=cfg["rho"], qs=None,
                fdorder=p["fdorder"], fw=p["fw"], free_surf=p["free_surf"], l=0, fl=(), fpml=p["fpml"],
                damping=p["damping"])
    o = O.Oracle(m, "port")
    ref = o.forward(sh.srcpos, sh.recpos)
    o.close()
    assert np.array_equal(seis, ref)


def test_cluster_unstable_model_reports_error():
    d, shots = _case(80, nx=40, ny=32, nt=400, fdo=4, L=0, fs=1, fw=6)
    shots = _inside(d, shots)
    d["dt"] = np.float32(5e-3)
    with engine_from(d) as e:
        e.set_step_variant(CLUSTER)
        with pytest.raises(dsh.DshError) as ei:
            e.forward(shots)
        assert ei.value.code == -4
    d["dt"] = np.float32(2e-4)
    with engine_from(d) as e:
        e.set_step_variant(CLUSTER)
        assert np.array_equal(e.forward(shots)[0], _oracle_forward(d, shots[0]))


def test_cluster_variant_falls_back_where_it_does_not_apply():
    """Viscoelastic models keep the kernel pair under variant 4 (bit-identical)."""
    d, shots = _case(3200, nx=60, ny=40, nt=100, fdo=4, L=2, fs=1, fw=8)
    shots = _inside(d, shots)
    seis, st, _ = _run(d, shots, CLUSTER)
    assert st["kernel_launches"] >= 2 * 100
    assert np.array_equal(seis[0], _oracle_forward(d, shots[0]))
