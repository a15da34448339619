"""Generate the golden fixtures in tests/golden/ (run here, where the
reference sources are available; the fixtures travel, the reference does not).

  csr_small.npz   small meshes of each element type with a seeded density:
                  the reference's own M, K1..K6 canonical CSRs, lumped mass and
                  M-PML profiles (oracle/_ref, compiled from the reference's C)
  runs_small.npz  small complete elastic_wave() runs of the reference (FP64
                  seismograms and snapshots captured from its output calls)
  acoustic_small.npz  small runs of the reference's scalar acoustic solvers
                  (time_evolution/acoustic.c and acoustic_pml.c, compiled in
                  place by oracle/ref_acoustic_harness.c): u snapshots and
                  energy per step, with the seeded vp, the lumped mass of
                  density 1 and the canonical CSR of stiffness type 0
  consistent_small.npz  small elastic_wave() runs of the reference's
                  consistent-mass branch (solver "mgmres": restarted GMRES + ILU
                  on M, solver/mgmres/mgmres.c), dt inside that scheme's
                  stability limit
  config1_reference.npz, config2_reference.npz  the reference's FP64 runs of
                  the two benchmark configurations at full size and length
                  (Q4 200x200, 1000 steps; Q9 400x400 layered, 3000 steps):
                  every 4th / 10th receiver over all time steps, and the
                  200-step snapshots on a coarse grid of nodes (every 8th /
                  16th grid line), with checksums of the inputs they belong to
  examples.npz    subsets of the reference's committed EXAMPLE outputs
                  (example 2: Q4 internal mesh, snapshots; example 6: T3
                  exterior mesh with a free surface, seismograms) and the mesh
                  of example 6 (its input files)

Usage: SEISFEM_REFERENCE=<reference tree> make -C oracle &&
       SEISFEM_REFERENCE=<reference tree> python tests/golden/make_golden.py [acoustic|consistent|config1|config2]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

REF = os.environ.get("SEISFEM_REFERENCE")
if not REF or not os.path.isdir(os.path.join(REF, "time_evolution")):
    raise SystemExit("set SEISFEM_REFERENCE to the reference source tree (the directory holding "
                     "time_evolution/, assemble/, EXAMPLE/, ...) and build oracle/_ref with "
                     "`make -C oracle REF=$SEISFEM_REFERENCE` first")

from oracle import Reference, ReferenceAcoustic  # noqa: E402
from fixture_keys import FULL_CONFIG_STRIDES, full_config_subset, input_checksum  # noqa: E402
from seisfem_b200 import problem as P  # noqa: E402
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


# (type, nx, ny, step, dt, pml, seed): Q9 and T6 with PML, and T6 without,
# exceed the reference's own energy bound / grow without bound -- kept, the
# outputs before that point are the fixture.  Without PML every mesh has at
# least `step` nodes: acoustic.c sizes its energy array by the node count.
ACOUSTIC_RUNS = [("Q4", 16, 12, 202, 1e-3, 0, 21), ("Q4", 16, 12, 202, 1e-3, 1, 22),
                 ("T3", 16, 14, 202, 1e-3, 0, 23), ("T3", 14, 12, 202, 1e-3, 1, 24),
                 ("Q9", 8, 6, 202, 5e-4, 0, 25), ("Q9", 8, 6, 202, 5e-4, 1, 26),
                 ("T6", 8, 6, 62, 5e-4, 0, 27), ("T6", 8, 6, 202, 5e-4, 1, 28)]


def acoustic_case(t, nx, ny, seed):
    """Mesh, vp and source node of one acoustic fixture case (also used by the tests)."""
    m = structured_mesh(t, nx, ny, 0.0, 10.0 * nx, 0.0, 10.0 * ny)
    rng = np.random.default_rng(seed)
    vp = 1800.0 + 400.0 * rng.random(m.node_num)
    src = int(np.argmin((m.x - 5.0 * nx) ** 2 + (m.y - 5.0 * ny) ** 2))
    return m, vp, src


def acoustic_small(R, RA):
    out = {}
    for t, nx, ny, step, dt, pml, seed in ACOUSTIC_RUNS:
        m, vp, src = acoustic_case(t, nx, ny, seed)
        r = RA.run(m, vp, step, dt, 25.0, 0.0, src, bool(pml), 10.0, 3, 3, nthreads=4)
        key = f"{t}_{'pml' if pml else 'plain'}"
        out[key + "_snap"], out[key + "_energy"] = r["snap"], r["energy"]
        out[key + "_status"] = np.int32(r["status"])
        out[key + "_lump"] = R.mass(m, np.ones(m.node_num), 1)
        if not pml:
            Bp, Bj, Bx = R.coo2csr(m.node_num, *R.stif(m, 0))
            out[key + "_k0_p"], out[key + "_k0_j"], out[key + "_k0_x"] = Bp, Bj, Bx
    np.savez_compressed(os.path.join(HERE, "acoustic_small.npz"), **out)


CONSISTENT_RUNS = [("Q4", 16, 402, 5e-4, 3, 5), ("T3", 14, 402, 5e-4, 3, 6)]


def consistent_small(R):
    out = {}
    for t, n, step, dt, pml, seed in CONSISTENT_RUNS:
        p = small_problem(t, n=n, step=step, pml=pml, seed=seed, dt=dt)
        r = R.run(p, nthreads=4, solver="mgmres")
        assert r["status"] == 0
        key = f"{t}_{n}"
        out[key + "_seis_u"], out[key + "_seis_w"] = r["seis_u"], r["seis_w"]
        out[key + "_snap_u"], out[key + "_snap_w"] = r["snap_u"], r["snap_w"]
    np.savez_compressed(os.path.join(HERE, "consistent_small.npz"), **out)


FULL_CONFIGS = {"config1": P.config_1, "config2": P.config_2}


def full_config(R, name):
    build = FULL_CONFIGS[name]
    rec_stride, grid_stride = FULL_CONFIG_STRIDES[name]
    P.use_scan_locator()
    prob = build()
    rec, nodes = full_config_subset(prob, rec_stride, grid_stride)
    r = R.run(prob, nthreads=os.cpu_count() or 1)
    assert r["status"] == 0, r["status"]
    out = {"checksum": input_checksum(prob), "rec": rec, "nodes": nodes, "seconds": np.float64(r["seconds"]),
           "seis_u": r["seis_u"][0][:, rec], "seis_w": r["seis_w"][0][:, rec],
           "snap_u": r["snap_u"][0][:, nodes], "snap_w": r["snap_w"][0][:, nodes],
           # norms of the full outputs, so that a subset's error can be scaled
           "norm_seis_u": np.linalg.norm(r["seis_u"]), "norm_seis_w": np.linalg.norm(r["seis_w"]),
           "norm_snap_u": np.linalg.norm(r["snap_u"]), "norm_snap_w": np.linalg.norm(r["snap_w"])}
    np.savez_compressed(os.path.join(HERE, f"{name}_reference.npz"), **out)


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
    part = sys.argv[1] if len(sys.argv) > 1 else "all"
    if part == "all":
        csr_small(R)
        runs_small(R)
        examples()
    if part in ("all", "acoustic"):
        acoustic_small(R, ReferenceAcoustic())
    if part in ("all", "consistent"):
        consistent_small(R)
    for name in FULL_CONFIGS:
        if part in ("all", name):
            full_config(R, name)
    for f in ("csr_small.npz", "runs_small.npz", "examples.npz", "acoustic_small.npz", "consistent_small.npz",
              "config1_reference.npz", "config2_reference.npz"):
        if not os.path.exists(os.path.join(HERE, f)):
            continue
        print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")
