"""Generate the golden fixtures in tests/golden/ (run here, where the
reference sources are available; the fixtures travel, the reference does not).

  csr_small.npz   small meshes of each element type with a seeded density:
                  the reference's own M, K1..K6 canonical CSRs, lumped mass and
                  M-PML profiles (oracle/_ref, compiled from the reference's C)
  runs_small.npz  small complete elastic_wave() runs of the reference (FP64
                  seismograms and snapshots captured from its output calls)
  examples.npz    subsets of the reference's committed EXAMPLE outputs
                  (example 2: Q4 internal mesh, snapshots; example 6: T3
                  exterior mesh with a free surface, seismograms) and the mesh
                  of example 6 (its input files)

Usage: make -C oracle && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

REF = os.environ.get("SEISFEM_REFERENCE", "/root/reference")

from oracle import Reference  # noqa: E402
from seisfem_b200.problem import small_problem, structured_mesh  # noqa: E402


def csr_small(R):
    out = {}
    for t in ("T3", "T6", "Q4", "Q9"):
        m = structured_mesh(t, 5, 4, 0.0, 50.0, 0.0, 40.0)
        rho = 2000.0 + 100.0 * np.sin(np.arange(m.node_num) * 0.37)
        out[f"{t}_element_node"] = m.element_node
        out[f"{t}_x"], out[f"{t}_y"], out[f"{t}_rho"] = m.x, m.y, rho
        mats = [R.mass(m, rho, 0)] + [R.stif(m, k) for k in range(1, 7)]
        for k, coo in enumerate(mats):
            Bp, Bj, Bx = R.coo2csr(m.node_num, *coo)
            out[f"{t}_m{k}_p"], out[f"{t}_m{k}_j"], out[f"{t}_m{k}_x"] = Bp, Bj, Bx
        out[f"{t}_lump"] = R.mass(m, rho, 1)
        out[f"{t}_mpml"] = R.abc_mpml(m, 1, 1, 10.0, (m.xmin, m.xmax, m.ymin, m.ymax), 3100.0)
    np.savez_compressed(os.path.join(HERE, "csr_small.npz"), **out)


RUNS = [("Q4", 16, 262, 1e-3, 4, 7), ("T3", 16, 262, 1e-3, 4, 8), ("Q9", 8, 262, 5e-4, 2, 9)]


def runs_small(R):
    out = {}
    for t, n, step, dt, pml, seed in RUNS:
        p = small_problem(t, n=n, step=step, pml=pml, seed=seed, dt=dt)
        r = R.run(p, nthreads=4)
        assert r["status"] == 0
        key = f"{t}_{n}"
        out[key + "_seis_u"], out[key + "_seis_w"] = r["seis_u"], r["seis_w"]
        out[key + "_snap_u"], out[key + "_snap_w"] = r["snap_u"], r["snap_w"]
    np.savez_compressed(os.path.join(HERE, "runs_small.npz"), **out)


def read_rows(path, stride=1, max_rows=None):
    rows = []
    with open(path) as f:
        for i, line in enumerate(f):
            if max_rows is not None and i >= max_rows:
                break
            if i % stride == 0:
                rows.append(np.array(line.split(), dtype=np.float64))
    return np.array(rows)


def examples():
    out = {}
    ex2 = os.path.join(REF, "EXAMPLE", "example2_first_order_quadrilateral_mesh", "outputfile")
    snap = read_rows(os.path.join(ex2, "wavefield_u_shot_1.txt"))
    idx = np.arange(0, snap.shape[1], 37)
    out["ex2_nodes"] = idx.astype(np.int32)
    out["ex2_snap_u"] = snap[:, idx]
    out["ex2_snap_w"] = read_rows(os.path.join(ex2, "wavefield_w_shot_1.txt"))[:, idx]
    ex6 = os.path.join(REF, "EXAMPLE", "example6_surface_wave")
    en = np.loadtxt(os.path.join(ex6, "mesh", "element_node.txt"), dtype=np.int64)
    xy = np.loadtxt(os.path.join(ex6, "mesh", "node_xy.txt"))
    out["ex6_element_node"] = en.astype(np.int32).ravel()
    out["ex6_x"], out["ex6_y"] = xy[:, 0].copy(), xy[:, 1].copy()
    out["ex6_seis_u"] = read_rows(os.path.join(ex6, "outputfile", "seismogram_u_shot_1.txt"), stride=10)
    out["ex6_seis_w"] = read_rows(os.path.join(ex6, "outputfile", "seismogram_w_shot_1.txt"), stride=10)
    np.savez_compressed(os.path.join(HERE, "examples.npz"), **out)


if __name__ == "__main__":
    R = Reference()
    csr_small(R)
    runs_small(R)
    examples()
    for f in ("csr_small.npz", "runs_small.npz", "examples.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")
