"""The consistent-mass branch of elastic_wave() (solver "pardiso" / "mgmres",
time_evolution/elastic_wave.c:664-680, 730-746): every step's 14 right-hand
sides are solved with the consistent mass matrix M instead of divided by the
lumped mass.

The reference solves with PARDISO (absent: a proprietary library) or with its
own restarted GMRES + ILU (solver/mgmres/mgmres.c, relative tolerance 1e-8).
The scheme is stable only below a smaller time step than the lumped one (Q4
at dt = 1 ms passes the energy bound; at 0.5 ms it runs), which is why the
fixtures use dt = 0.5 ms.

CPU: the oracle's restatement (conjugate gradients with the Jacobi
preconditioner to a 1e-12 relative residual) against the reference's GMRES
runs -- committed fixtures tests/golden/consistent_small.npz and, where
oracle/_ref is built, live -- to 1e-8 relative L2 (measured 1e-11 .. 6e-10:
the reference's own solver tolerance).  GPU (SFG_FP64_CONSISTENT through the
C ABI): against the restatement to 1e-9 and against the reference fixtures
to 1e-8; the drop-in elastic_wave() with solver "mgmres".
"""
import os

import numpy as np
import pytest

from conftest import rel_l2
from seisfem_b200.problem import small_problem

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "consistent_small.npz")
# (type, n, step, dt, pml, seed): the cases of tests/golden/make_golden.py
CASES = [("Q4", 16, 402, 5e-4, 3, 5), ("T3", 14, 402, 5e-4, 3, 6)]
KEYS = ("seis_u", "seis_w", "snap_u", "snap_w")
REF_TOL = 1e-8


def _problem(c):
    t, n, step, dt, pml, seed = c
    return small_problem(t, n=n, step=step, pml=pml, seed=seed, dt=dt)


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("c", CASES, ids=[c[0] for c in CASES])
def test_restatement_matches_reference_gmres_fixture(oracle, golden, c):
    r = oracle.run(_problem(c), solver="mgmres")
    assert r["status"] == 0
    for k in KEYS:
        ref = golden[f"{c[0]}_{c[1]}_{k}"]
        assert rel_l2(r[k], ref) < REF_TOL, (k, rel_l2(r[k], ref))


def test_restatement_matches_reference_gmres_live(oracle, reference):
    p = small_problem("Q4", n=13, step=302, pml=3, seed=8, dt=5e-4)
    a = oracle.run(p, solver="mgmres")
    b = reference.run(p, nthreads=4, solver="mgmres")
    assert a["status"] == b["status"] == 0
    for k in KEYS:
        assert rel_l2(a[k], b[k]) < REF_TOL, k
    # the consistent scheme differs from the lumped one by far more than that
    lumped = oracle.run(p)
    assert rel_l2(lumped["seis_u"], a["seis_u"]) > 1e-2


def test_restatement_reports_the_energy_bound(oracle, reference):
    # dt = 1 ms is above the consistent scheme's stability limit for this mesh
    p = small_problem("Q4", n=12, step=300, pml=3, seed=5)
    assert oracle.run(p)["status"] == 0                 # lumped: stable
    assert oracle.run(p, solver="mgmres")["status"] == 1
    assert reference.run(p, nthreads=4, solver="mgmres")["status"] == 1


# ------------------------------------------------------------------ GPU

@pytest.mark.gpu
@pytest.mark.parametrize("c", CASES, ids=[c[0] for c in CASES])
def test_gpu_consistent_matches_restatement_and_reference(ctx, oracle, golden, c):
    p = _problem(c)
    ctx.setup(p)
    out = ctx.run(p, precision="fp64cm", want_snapshots=True)
    assert out["status"] == 0
    ref = oracle.run(p, solver="mgmres")
    for k in KEYS:
        assert rel_l2(out[k], ref[k]) < 1e-9, (k, rel_l2(out[k], ref[k]))
        g = golden[f"{c[0]}_{c[1]}_{k}"]
        assert rel_l2(out[k], g) < REF_TOL, (k, rel_l2(out[k], g))


@pytest.mark.gpu
def test_gpu_consistent_energy_bound(ctx, oracle):
    from seisfem_b200.api import SFG_ERR_BLOWUP
    p = small_problem("Q4", n=12, step=300, pml=3, seed=5)
    ctx.setup(p)
    out = ctx.run(p, precision="fp64cm", raise_on_blowup=False)
    assert out["status"] == SFG_ERR_BLOWUP
    assert oracle.run(p, solver="mgmres")["status"] == 1


@pytest.mark.gpu
def test_gpu_dropin_mgmres(oracle, tmp_path):
    """elastic_wave() with solver "mgmres" takes the GPU consistent-mass path
    and writes the reference's files."""
    from test_gpu_dropin import _call_dropin, _read
    p = small_problem("Q4", n=14, step=302, pml=3, seed=9, dt=5e-4)
    os.makedirs(tmp_path / "mesh")
    os.makedirs(tmp_path / "outputfile")
    md = p.model
    cols = np.stack([md.rho, md.vp, md.vs, md.c[0], md.c[1], md.c[2], md.c[3]], axis=1)
    with open(tmp_path / "mesh" / "velocity_and_density.txt", "w") as fh:
        fh.write("".join(" ".join("%.17g" % v for v in row) + "\n" for row in cols))
    _call_dropin(p, str(tmp_path), solver=b"mgmres")
    ref = oracle.run(p, solver="mgmres")
    su = _read(tmp_path / "outputfile" / "seismogram_u_shot_1.txt")
    assert su.shape == ref["seis_u"][0].shape
    assert np.abs(su - ref["seis_u"][0]).max() <= 1e-6 + 1e-9 * np.abs(ref["seis_u"][0]).max()
