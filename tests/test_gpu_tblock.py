"""The temporally blocked forward-modelling launches (step variant 5): plain
elastic forward modelling of a small grid with k time steps per launch, each
thread block advancing its tile (32 points wide, 8-64 rows high so that all
tiles run in one wave) and a recomputed halo of k*(FDORDER-1) points in
shared memory.

Bit-exact against the CPU oracle (pinned to the reference's
update_v_PML.c / update_s_elastic_PML.c / seismo_ssg.c) over FDORDER 2-8,
free surface on and off (CPML on all four sides), DH a power of two or not,
grid widths that are not a multiple of the tile, steps per launch from 1 to
7 (a pass whose NT is not a multiple of k ends with a shorter launch), tile
heights of 5, 8, 16 and 24 rows,
several shots in one launch and the 500 x 200 x 2000 benchmark case; the end
state written back to the slots equals the kernel pair's; an unstable model
reports DSH_ERR_UNSTABLE."""
import math

import numpy as np
import pytest

import dsh
import oracle as O
from dsh import configs
from test_gpu_cluster import _inside, _oracle_forward
from test_gpu_parity import _case, engine_from

pytestmark = pytest.mark.gpu

TBLOCK = dsh.Engine.VARIANTS.index("temporally blocked launch")
K_DEFAULT = {2: 8, 4: 4, 6: 3, 8: 2}


def _run(d, shots, variant, max_shots=1):
    with engine_from(d, max_shots=max_shots) as e:
        e.set_step_variant(variant)
        seis = e.forward(shots)
        st = e.stats()
        end = [{k: e.field(k, shot=s) for k in ("vy", "sxy", "syz")} for s in range(len(shots))]
    return seis, st, end


@pytest.mark.parametrize("fdo", [2, 4, 6, 8])
@pytest.mark.parametrize("nx,ny,fs,dh", [(70, 40, 1, 0.5), (203, 97, 0, 0.6), (500, 200, 1, 0.5)])
def test_tblock_forward_matches_oracle(fdo, nx, ny, fs, dh):
    nt = 130
    d, shots = _case(4000 + 10 * fdo + nx, nx=nx, ny=ny, nt=nt, fdo=fdo, L=0, fs=fs, fw=10)
    d["dh"] = dh
    shots = _inside(d, shots)
    ref = _oracle_forward(d, shots[0])
    seis, st, end = _run(d, shots, TBLOCK)
    assert np.array_equal(seis[0], ref)
    assert st["kernel_launches"] <= math.ceil(nt / K_DEFAULT[fdo]) + 8
    _, _, end_pair = _run(d, shots, 0)
    for k in ("vy", "sxy", "syz"):
        assert np.array_equal(end[0][k], end_pair[0][k]), k


@pytest.mark.parametrize("k", [1, 3, 7])
def test_tblock_steps_per_launch(k, monkeypatch):
    """Other k (DSH_TB_STEPS): NT 101 is a multiple of none of them."""
    monkeypatch.setenv("DSH_TB_STEPS", str(k))
    d, shots = _case(4100 + k, nx=90, ny=50, nt=101, fdo=4, L=0, fs=0, fw=8)
    shots = _inside(d, shots)
    seis, st, _ = _run(d, shots, TBLOCK)
    assert st["kernel_launches"] <= math.ceil(101 / k) + 8
    assert np.array_equal(seis[0], _oracle_forward(d, shots[0]))


@pytest.mark.parametrize("rows", [16, 5])
def test_tblock_pinned_tile_heights(rows, monkeypatch):
    """Tile heights the single-wave choice does not pick here (DSH_TB_ROWS):
    16 rows (two CTAs per SM on this grid) and an odd 5."""
    monkeypatch.setenv("DSH_TB_ROWS", str(rows))
    d, shots = _case(4150 + rows, nx=203, ny=97, nt=90, fdo=6, L=0, fs=0, fw=10)
    shots = _inside(d, shots)
    seis, _, end = _run(d, shots, TBLOCK)
    assert np.array_equal(seis[0], _oracle_forward(d, shots[0]))
    _, _, end_pair = _run(d, shots, 0)
    for k in ("vy", "sxy", "syz"):
        assert np.array_equal(end[0][k], end_pair[0][k]), k


def test_tblock_several_shots_in_one_launch():
    d, shots = _case(4200, nx=150, ny=64, nt=150, fdo=4, L=0, fs=1, fw=10, nshots=3)
    shots = _inside(d, shots)
    seis, _, end = _run(d, shots, TBLOCK, max_shots=3)
    _, _, end_pair = _run(d, shots, 0, max_shots=3)
    for s, sh in enumerate(shots):
        assert np.array_equal(seis[s], _oracle_forward(d, sh)), s
        for k in ("vy", "sxy", "syz"):
            assert np.array_equal(end[s][k], end_pair[s][k]), (s, k)


def test_tblock_benchmark_case_matches_oracle():
    """The 500 x 200, FDORDER 4, NT 2000 elastic forward case, 4 steps per launch."""
    cfg = configs.config1()
    p = cfg["params"]
    sh = cfg["shots"][0]
    with dsh.Engine(dsh.make_params(**p)) as e:
        e.set_model(cfg["vs"], cfg["rho"], None)
        e.set_step_variant(TBLOCK)
        seis = e.forward([sh])[0]
        assert e.stats()["kernel_launches"] <= p["nt"] // 4 + 8
    m = O.Model(nx=p["nx"], ny=p["ny"], nt=p["nt"], dh=p["dh"], dt=p["dt"], vs=cfg["vs"], rho=cfg["rho"], qs=None,
                fdorder=p["fdorder"], fw=p["fw"], free_surf=p["free_surf"], l=0, fl=(), fpml=p["fpml"],
                damping=p["damping"])
    o = O.Oracle(m, "port")
    ref = o.forward(sh.srcpos, sh.recpos)
    o.close()
    assert np.array_equal(seis, ref)


def test_tblock_unstable_model_reports_error():
    d, shots = _case(80, nx=40, ny=32, nt=400, fdo=4, L=0, fs=1, fw=6)
    shots = _inside(d, shots)
    d["dt"] = np.float32(5e-3)
    with engine_from(d) as e:
        e.set_step_variant(TBLOCK)
        with pytest.raises(dsh.DshError) as ei:
            e.forward(shots)
        assert ei.value.code == -4
    d["dt"] = np.float32(2e-4)
    with engine_from(d) as e:
        e.set_step_variant(TBLOCK)
        assert np.array_equal(e.forward(shots)[0], _oracle_forward(d, shots[0]))


def test_tblock_variant_falls_back_where_it_does_not_apply():
    """Viscoelastic models keep the kernel pair under variant 5 (bit-identical)."""
    d, shots = _case(4300, nx=60, ny=40, nt=100, fdo=4, L=2, fs=1, fw=8)
    shots = _inside(d, shots)
    seis, st, _ = _run(d, shots, TBLOCK)
    assert st["kernel_launches"] >= 2 * 100
    assert np.array_equal(seis[0], _oracle_forward(d, shots[0]))


def test_autotuner_times_the_tblock_variant():
    cfg = configs.config1()
    p = dict(cfg["params"], nt=200)
    with dsh.Engine(dsh.make_params(**p)) as e:
        e.set_model(cfg["vs"], cfg["rho"], None)
        _, ms = e.autotune(cfg["shots"], nsteps=64)
    assert ms["temporally blocked launch"] > 0
    print("ms per step", ms)
