"""The reference's file formats: this library's readers and SU writer
(include/dsh_io.h) against the reference's own read_par, sources+splitsrc,
receiver and outseis_glob, compiled in place into the oracle."""
import ctypes as C
import os

import numpy as np
import pytest

import dsh
import oracle as O
from dsh import io

HAVE_REF = O.available("ref")
needs_ref = pytest.mark.skipif(not HAVE_REF, reason="reference not compiled here")

# value kinds of the reference's 138 positional .inp lines, in order
KINDS = ("iiiiii" "fff" "ii" "fff" "s" "f" "i" "s" "ii" "s" "i" "L" "f" "ii" "ff" "ii" "fff" "iii" "s" "ii" "s"
         "FFF" "ii" "ff" "iii" "ssssss" "iii" "s" "i" "ss" "iii" "A" "iii" "B" "iiiii" "f" "iii" "f" "iiii" "s"
         "iiii" "ffffffff" "i" "ff" "i" "f" "iiiii" "s" "iii" "fff" "iii" "f" "i" "ff" "i" "s" "i" "s" "fff"
         "i" "s" "iiiiii" "s")


def _ref():
    return C.CDLL(os.path.join(O.REF_DIR, "libdenise_ref.so"))


def _write_inp(path, rng, L=3):
    lines = ["#-----------------------------", "# parameter file written by the test", "#"]
    vals = {}
    for n, k in enumerate(KINDS, start=1):
        key = f"parameter_{n}_(P{n})"
        if n == 1 or n == 2:
            v = "1"
        elif n == 22:
            v = str(L)
        elif n in (5, 6):                     # NX, NY must be positive for a usable file
            v = str(int(rng.integers(8, 900)))
        elif k == "i":
            v = str(int(rng.integers(0, 9)))
        elif k == "f":
            v = f"{rng.uniform(0.001, 900):.6g}"
        elif k == "s":
            v = f"./dir{n}/file_{n}.dat"
        elif k == "L":
            v = " ".join(f"{x:.4f}" for x in rng.uniform(1, 50, L))
        elif k == "F":
            v = f"{rng.uniform(0, 10):.3f} , {rng.uniform(0, 10):.3f}"
        elif k == "A":
            v = "1, 6, 4900, 5000"
        else:
            v = "4, 84, 10"
        vals[n] = v
        lines.append(f"{key} = {v}")
        if n % 7 == 0:
            lines.append("# a comment between parameters")
    open(path, "w").write("\n".join(lines) + "\n")
    return vals


@needs_ref
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_inp_reader_matches_reference(tmp_path, seed):
    rng = np.random.default_rng(seed)
    p = str(tmp_path / "par.inp")
    _write_inp(p, rng)
    v = np.zeros(64, np.float64)
    strs = C.create_string_buffer(4096)
    n = _ref().refh_read_par(p.encode(), v.ctypes.data_as(C.POINTER(C.c_double)), strs, 4096)
    assert n > 40
    mine = io.read_inp(p)
    f32 = lambda x: float(np.float32(x))
    expect = [mine.nprocx, mine.nprocy, mine.fdorder, mine.maxrelerror, mine.nx, mine.ny, f32(mine.dh),
              f32(mine.time), f32(mine.dt), mine.quellart, mine.quelltyp, mine.srcrec, mine.run_multiple_shots,
              mine.readmod, mine.l] + [f32(mine.fl[k]) if k < mine.l else 0.0 for k in range(8)] + \
             [f32(mine.tau), mine.free_surf, mine.fw, f32(mine.damping), f32(mine.fpml), mine.boundary, mine.seismo,
              mine.readrec, f32(mine.refrec[0]), f32(mine.refrec[1]), mine.ndt, mine.seis_format, mine.invmat1,
              mine.invmat, mine.quelltypb, f32(mine.npower), f32(mine.k_max_pml), mine.hessian, f32(mine.fc_hessian),
              mine.grad_method, mine.lnorm, mine.dtinv]
    assert np.array_equal(np.array(expect, np.float64), v[:n])
    ref_strs = strs.value.decode().split("\n")
    assert ref_strs == [mine.signal_file.decode(), mine.source_file.decode(), mine.mfile.decode(),
                        mine.rec_file.decode(), mine.seis_file_vy.decode(), mine.data_dir.decode()]
    assert mine.lines >= len(KINDS)       # a final newline before EOF counts as a line, as in read_par


def test_json_reader_and_params(tmp_path):
    p = tmp_path / "par.json"
    p.write_text('{\n "NPROCX" : "1", "NPROCY" : "1",\n "FDORDER" : "8", "MAXRELERROR" : "1",\n'
                 ' "NX" : "2000", "NY" : "800", "DH" : "0.25", "TIME" : "0.6", "DT" : "1e-4",\n'
                 ' "L" : "3", "FL1" : "10.0", "FL2" : "40.0", "FL3" : "160.0", "FW" : "20",\n'
                 ' "FREE_SURF" : "1", "DAMPING" : "500.0", "FPML" : "40.0", "QUELLART" : "1",\n'
                 ' "MFILE" : "start/model", "REFRECX" : "1.5", "REFRECY" : "0.5", "npower" : "4.0"\n}\n')
    inp = io.read_json(str(p))
    assert (inp.nx, inp.ny, inp.fdorder, inp.l, inp.fw) == (2000, 800, 8, 3, 20)
    assert inp.mfile == b"start/model" and abs(inp.refrec[0] - 1.5) < 1e-7
    par = io.params_from(inp, max_shots=2)
    assert par.nt == 6000 and abs(par.dh - 0.25) < 1e-9 and list(par.fl[:3]) == [10.0, 40.0, 160.0]
    assert par.max_shots == 2


def test_workflow_reader(tmp_path):
    p = tmp_path / "workflow.txt"
    head = " ".join(f"COL{k}" for k in range(24))
    rows = ["0.01 0 10 20 6 0 20 0.01 0.4 0 0 0 0 5.0 5.0 1 2 0 0 0 0 0 0 1",
            "0.01 1 10 40 6 0 20 0.01 0.4 0 0 0 0 5.0 5.0 3 5 0 0 0 0 0 0 1"]
    p.write_text(head + "\n" + "\n".join(rows) + "\n")
    s1, s2 = io.read_workflow(str(p), 1), io.read_workflow(str(p), 2)
    assert (s1.eprecond, s1.lnorm, s1.fc_end) == (1, 2, 20.0)
    assert (s2.eprecond, s2.lnorm, s2.time_filt, s2.fc_end) == (3, 5, 1, 40.0)


@needs_ref
def test_sources_match_reference(tmp_path):
    p = tmp_path / "source.dat"
    p.write_text("5\n125.0 0.0 1.0 0.0 30.0 1.0 0.0 3\n10.2 0.0 2.4 0.01 20.0 2.0\n"
                 "999.0 0.0 1.0 0.0 30.0 1.0 0.0 3\n0.1 0.0 0.2 0.0 30.0 1.0 45.0 1\n40.26 0 3.74 0 25 -1 0 3\n")
    dh, nx, ny = 0.5, 400, 100
    sp, sm = io.read_sources(str(p), dh, nx, ny)
    ref_m = np.zeros((8, 16), np.float32)
    ref_l = np.zeros((8, 16), np.float32)
    nloc = C.c_int(0)
    n = _ref().refh_sources(str(p).encode(), C.c_float(dh), nx, ny, 16, ref_m.ctypes.data_as(C.c_void_p),
                            ref_l.ctypes.data_as(C.c_void_p), C.byref(nloc))
    assert n == 5 and nloc.value == sp.shape[1] == 4      # x = 999 m lies outside the grid
    assert np.array_equal(sp, ref_l[:, :nloc.value])


@needs_ref
def test_receivers_match_reference(tmp_path):
    p = tmp_path / "rec.dat"
    xs = [77.5, 78.0, 78.2, 80.0, 80.1, 172.5, 3.0]
    p.write_text("".join(f"{x} {0.5 if k % 3 else 0.8}\n" for k, x in enumerate(xs)))
    dh = 0.5
    rp = io.read_receivers(str(p), dh, refrec=(0.25, 0.0))
    ref = np.zeros((3, 16), np.int32)
    n = _ref().refh_receivers(str(p).encode(), C.c_float(dh), C.c_float(0.25), C.c_float(0.0), 16,
                              ref.ctypes.data_as(C.c_void_p))
    assert n == rp.shape[1] and n < len(xs)            # grid duplicates removed
    assert np.array_equal(rp, ref[:2, :n])


def test_model_files_are_x_major(tmp_path):
    rng = np.random.default_rng(3)
    vs = rng.uniform(100, 500, (7, 11)).astype(np.float32)
    rho = rng.uniform(1500, 2000, (7, 11)).astype(np.float32)
    qs = rng.uniform(20, 60, (7, 11)).astype(np.float32)
    base = str(tmp_path / "m")
    for ext, a in (("vs", vs), ("rho", rho), ("qs", qs)):
        io.write_model(f"{base}.{ext}", a)
    raw = np.fromfile(f"{base}.vs", np.float32)
    assert np.array_equal(raw[:7], vs[:, 0])            # first the whole depth column at x index 1
    v2, r2, q2 = io.read_model(base, 11, 7, l=3)
    assert np.array_equal(v2, vs) and np.array_equal(r2, rho) and np.array_equal(q2, qs)


@needs_ref
def test_su_output_matches_reference(tmp_path):
    rng = np.random.default_rng(4)
    ntr, ns, dh, dt = 5, 300, 0.5, 2e-4
    sec = rng.standard_normal((ntr, ns)).astype(np.float32)
    rec = np.array([[155, 157, 159, 200, 345], [1, 1, 1, 2, 1]], np.int32)
    tracl = np.array([1, 2, 3, 5, 8], np.int32)
    mine, theirs = str(tmp_path / "a.su"), str(tmp_path / "b.su")
    io.write_su(mine, sec, rec, xs=125.0, ys=1.0, dh=dh, dt=dt, tracl=tracl, refrec=(0.5, 0.25))
    rp3 = np.ascontiguousarray(np.vstack([rec, tracl[None]]), np.int32)
    assert _ref().refh_write_su(theirs.encode(), ntr, ns, sec.ctypes.data_as(C.c_void_p),
                                rp3.ctypes.data_as(C.c_void_p), C.c_float(125.0), C.c_float(1.0), C.c_float(dh),
                                C.c_float(dt), C.c_float(0.5), C.c_float(0.25)) == 0
    a, b = open(mine, "rb").read(), open(theirs, "rb").read()
    assert len(a) == len(b) == ntr * (240 + 4 * ns)
    for k in range(ntr):
        o = k * (240 + 4 * ns)
        # header bytes 210..239 are never assigned by the reference's writer
        assert a[o:o + 210] == b[o:o + 210], k
        assert a[o + 240:o + 240 + 4 * ns] == b[o + 240:o + 240 + 4 * ns], k
    back = io.read_su(mine, ntr, ns)
    assert back[:, 0].tolist() == [0.0] * ntr and np.array_equal(back[:, 1:], sec[:, 1:])
