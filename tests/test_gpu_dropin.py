"""The drop-in elastic_wave() (time_evolution/elastic_wave.c:1-3 signature),
called as seisfem/seisfem.c:277-278 calls it, in a working directory with
./mesh and ./outputfile: its text outputs against the FP64 oracle."""
import ctypes as C
import os

import numpy as np
import pytest

from seisfem_b200 import api
from seisfem_b200.problem import small_problem

pytestmark = pytest.mark.gpu


def _call_dropin(p, workdir, solver=b"masslump", use_exterior=1):
    L = api.lib()
    f = L.elastic_wave
    f.restype = None
    f.argtypes = ([C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.POINTER(C.c_double)),
                   C.c_int, C.c_int, C.c_int] + [C.c_double] * 8 + [C.c_int] * 3 +
                  [C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int), C.c_char_p, C.c_int, C.c_int])
    m = p.mesh
    en = np.ascontiguousarray(m.element_node, np.int32)
    x, y = np.ascontiguousarray(m.x), np.ascontiguousarray(m.y)
    xy = (C.POINTER(C.c_double) * 2)(x.ctypes.data_as(C.POINTER(C.c_double)), y.ctypes.data_as(C.POINTER(C.c_double)))
    src = np.ascontiguousarray(p.src_node, np.int32)
    rec = np.ascontiguousarray(p.rec_node, np.int32)
    cwd = os.getcwd()
    os.chdir(workdir)
    try:
        f(m.type_name.encode(), m.node_num, m.element_num, m.order, en.ctypes.data_as(C.POINTER(C.c_int)),
          C.cast(xy, C.POINTER(C.POINTER(C.c_double))), m.element_num * m.order ** 2, m.node_num + 1, p.step, p.dt,
          p.f0, p.t0, p.edge_size, m.xmin, m.xmax, m.ymin, m.ymax, p.pml_nx, p.pml_ny, len(src),
          src.ctypes.data_as(C.POINTER(C.c_int)), len(rec), rec.ctypes.data_as(C.POINTER(C.c_int)), solver,
          use_exterior, p.free_surface)
    finally:
        os.chdir(cwd)


def _read(path):
    return np.array([np.array(l.split(), dtype=np.float64) for l in open(path) if l.strip()])


def test_dropin_files_match_oracle(oracle, tmp_path):
    p = small_problem("Q4", n=24, step=402, pml=4, seed=5, shots=2)
    os.makedirs(tmp_path / "mesh")
    os.makedirs(tmp_path / "outputfile")
    md = p.model
    cols = np.stack([md.rho, md.vp, md.vs, md.c[0], md.c[1], md.c[2], md.c[3]], axis=1)
    with open(tmp_path / "mesh" / "velocity_and_density.txt", "w") as fh:
        fh.write("".join(" ".join("%.17g" % v for v in row) + "\n" for row in cols))
    _call_dropin(p, str(tmp_path))
    ref = oracle.run(p)
    for s in range(2):
        su = _read(tmp_path / "outputfile" / f"seismogram_u_shot_{s + 1}.txt")
        sw = _read(tmp_path / "outputfile" / f"seismogram_w_shot_{s + 1}.txt")
        wu = _read(tmp_path / "outputfile" / f"wavefield_u_shot_{s + 1}.txt")
        assert su.shape == ref["seis_u"][s].shape and wu.shape == ref["snap_u"][s].shape
        scale = np.abs(ref["seis_u"][s]).max()
        # %f text (5e-7) plus the FP32 path's error
        assert np.abs(su - ref["seis_u"][s]).max() <= 1e-6 + 1e-4 * scale
        assert np.abs(sw - ref["seis_w"][s]).max() <= 1e-6 + 1e-4 * scale
        assert np.abs(wu - ref["snap_u"][s]).max() <= 1e-6 + 1e-4 * np.abs(ref["snap_u"][s]).max()
    # the same seismogram row layout as the reference: "%f   " per receiver
    line = open(tmp_path / "outputfile" / "seismogram_u_shot_1.txt").readline()
    assert line.endswith("   \n") and len(line.split()) == len(p.rec_node)


def test_dropin_builtin_model_writes_velocity_file(tmp_path):
    p = small_problem("T3", n=10, step=20, pml=2)
    os.makedirs(tmp_path / "mesh")
    os.makedirs(tmp_path / "outputfile")
    _call_dropin(p, str(tmp_path), use_exterior=0)
    rows = _read(tmp_path / "mesh" / "velocity_and_density.txt")
    # model_elastic_parameter.c:34-45 (rho 2200, vp 2000, vs 1154.7)
    assert rows.shape == (p.mesh.node_num, 7)
    assert np.allclose(rows[:, :3], [2200.0, 2000.0, 1154.7])
