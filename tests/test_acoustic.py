"""The scalar acoustic solvers (time_evolution/acoustic.c, acoustic_pml.c).

CPU: the oracle's restatement (oracle/sfo.c: sfo_acoustic_run) against the
reference's own code -- the committed fixtures tests/golden/acoustic_small.npz
(made by tests/golden/make_golden.py from the reference compiled in place)
and, where oracle/_ref is built, live runs of other cases -- bit for bit.

GPU (sfg_acoustic_run through the C ABI): given the reference's lumped mass
the snapshots are bit-identical to the reference's (FP64, the reference's
operation order); with the lumped mass assembled on the GPU (its
normalisation sum is parallel, ~1e-14 relative, which the schemes' undamped
zero-frequency mode amplifies over a run) they agree to 1e-6 relative L2.
Runs that the reference ends on its energy bound end at the same step.  The
drop-in acoustic() / acoustic_pml() write the reference's files.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import rel_l2
from seisfem_b200.problem import structured_mesh

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "acoustic_small.npz")

# (type, nx, ny, step, dt, pml, seed): the cases of tests/golden/make_golden.py
CASES = [("Q4", 16, 12, 202, 1e-3, 0, 21), ("Q4", 16, 12, 202, 1e-3, 1, 22),
         ("T3", 16, 14, 202, 1e-3, 0, 23), ("T3", 14, 12, 202, 1e-3, 1, 24),
         ("Q9", 8, 6, 202, 5e-4, 0, 25), ("Q9", 8, 6, 202, 5e-4, 1, 26),
         ("T6", 8, 6, 62, 5e-4, 0, 27), ("T6", 8, 6, 202, 5e-4, 1, 28)]
IDS = [f"{c[0]}_{'pml' if c[5] else 'plain'}" for c in CASES]
F0, T0, EDGE, PML_N = 25.0, 0.0, 10.0, 3


def case(t, nx, ny, seed):
    m = structured_mesh(t, nx, ny, 0.0, 10.0 * nx, 0.0, 10.0 * ny)
    rng = np.random.default_rng(seed)
    vp = 1800.0 + 400.0 * rng.random(m.node_num)
    src = int(np.argmin((m.x - 5.0 * nx) ** 2 + (m.y - 5.0 * ny) ** 2))
    return m, vp, src


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def _oracle_run(oracle, m, vp, src, step, dt, pml):
    return oracle.acoustic_run(m, vp, step, dt, F0, T0, src, bool(pml), EDGE, PML_N, PML_N)


@pytest.mark.parametrize("c", CASES, ids=IDS)
def test_restatement_matches_reference_fixture(oracle, golden, c):
    t, nx, ny, step, dt, pml, seed = c
    m, vp, src = case(t, nx, ny, seed)
    key = f"{t}_{'pml' if pml else 'plain'}"
    r = _oracle_run(oracle, m, vp, src, step, dt, pml)
    ref_snap, ref_e = golden[key + "_snap"], golden[key + "_energy"]
    assert r["status"] == int(golden[key + "_status"])
    assert np.array_equal(r["snap"][:ref_snap.shape[0]], ref_snap)
    assert np.array_equal(r["energy"][:ref_e.shape[0]], ref_e)
    if r["status"] == 0:
        assert ref_snap.shape[0] == r["snap"].shape[0] and ref_e.shape[0] == step


@pytest.mark.parametrize("t", ["Q4", "Q9", "T3", "T6"])
def test_laplacian_csr_matches_reference_fixture(oracle, golden, t):
    c = next(c for c in CASES if c[0] == t and not c[5])
    m, _, _ = case(c[0], c[1], c[2], c[6])
    ci, cj, cx = oracle.stif_coo(m, 0)
    Bp, Bj, Bx = oracle.coo2csr(m.node_num, ci, cj, cx)
    key = f"{t}_plain"
    assert np.array_equal(Bp, golden[key + "_k0_p"])
    assert np.array_equal(Bj, golden[key + "_k0_j"])
    assert np.array_equal(Bx, golden[key + "_k0_x"])


def test_restatement_matches_reference_live(oracle):
    from oracle import LIBACOUSTIC, ReferenceAcoustic
    if not os.path.exists(LIBACOUSTIC):
        pytest.skip("reference build (oracle/_ref) not present")
    R = ReferenceAcoustic()
    for t, nx, ny, step, pml, seed in (("Q4", 22, 19, 181, 1, 31), ("Q9", 9, 8, 151, 0, 32),
                                       ("T3", 20, 15, 141, 1, 33)):
        m, vp, src = case(t, nx, ny, seed)
        dt = 5e-4 if t == "Q9" else 1e-3
        a = _oracle_run(oracle, m, vp, src, step, dt, pml)
        b = R.run(m, vp, step, dt, F0, T0, src, bool(pml), EDGE, PML_N, PML_N, nthreads=2)
        assert a["status"] == b["status"] == 0
        assert np.array_equal(a["snap"], b["snap"]) and np.array_equal(a["energy"], b["energy"])


# ------------------------------------------------------------------ GPU

def _gpu_run(ctx, m, vp, src, step, dt, pml, mass_lump=None):
    return ctx.acoustic_run(m, vp, step, dt, F0, T0, src, bool(pml), EDGE, PML_N, PML_N, mass_lump=mass_lump)


@pytest.mark.gpu
@pytest.mark.parametrize("c", CASES, ids=IDS)
def test_gpu_bit_identical_with_reference_lumped_mass(ctx, golden, c):
    from seisfem_b200.api import SFG_ERR_BLOWUP
    t, nx, ny, step, dt, pml, seed = c
    m, vp, src = case(t, nx, ny, seed)
    key = f"{t}_{'pml' if pml else 'plain'}"
    r = _gpu_run(ctx, m, vp, src, step, dt, pml, mass_lump=golden[key + "_lump"])
    ref_snap, ref_e = golden[key + "_snap"], golden[key + "_energy"]
    assert r["status"] == (SFG_ERR_BLOWUP if int(golden[key + "_status"]) else 0)
    assert np.array_equal(r["snap"][:ref_snap.shape[0]], ref_snap)
    assert not r["snap"][ref_snap.shape[0]:].any()
    # energy: a parallel sum (block partials, atomically combined)
    n = ref_e.shape[0]
    fin = np.isfinite(ref_e)
    assert np.allclose(r["energy"][:n][fin], ref_e[fin], rtol=1e-12, atol=0.0)
    if r["status"]:
        assert r["stats"]["blowup_step"] == n and not r["energy"][n:].any()


@pytest.mark.gpu
@pytest.mark.parametrize("t,pml", [("Q4", 0), ("Q4", 1), ("T3", 1), ("Q9", 0)])
def test_gpu_assembled_mass_matches_oracle(ctx, oracle, t, pml):
    # a larger mesh than the fixtures: 90 x 70 elements (Q9: 45 x 35)
    nx, ny = (45, 35) if t == "Q9" else (90, 70)
    m, vp, src = case(t, nx, ny, 41 + pml)
    dt = 5e-4 if t == "Q9" else 1e-3
    step = 402
    a = _gpu_run(ctx, m, vp, src, step, dt, pml)
    b = _oracle_run(oracle, m, vp, src, step, dt, pml)
    assert a["status"] == 0 and b["status"] == 0
    # The only difference is the lumped mass's normalisation sum (parallel on
    # the GPU, ~1e-14 relative).  The schemes carry an undamped zero-frequency
    # mode (u_new = 2 u - u_old where M u / m = u) whose growth over the run
    # amplifies it: 2.5e-8 measured on the Q4 case without PML.
    assert rel_l2(a["snap"], b["snap"]) < 1e-6, rel_l2(a["snap"], b["snap"])
    assert rel_l2(a["energy"], b["energy"]) < 1e-6
    st = a["stats"]
    assert st["kernel_launches"] == step - 2 and st["loop_ms"] > 0.0
    assert st["union_nnz"] >= max(st["csr_nnz"])


@pytest.mark.gpu
def test_gpu_no_source_stays_zero(ctx):
    m, vp, _ = case("Q4", 20, 20, 3)
    r = _gpu_run(ctx, m, vp, -1, 102, 1e-3, 1)
    assert r["status"] == 0 and not r["snap"].any() and not r["energy"].any()


@pytest.mark.gpu
def test_gpu_bad_arguments(ctx):
    from seisfem_b200.api import SfgError
    m, vp, _ = case("Q4", 8, 8, 3)
    with pytest.raises(SfgError) as e:
        _gpu_run(ctx, m, vp, m.node_num, 52, 1e-3, 0)
    assert e.value.status == 5          # SFG_ERR_BADINDEX
    with pytest.raises(SfgError) as e:
        ctx.acoustic_run(m, vp, 52, 1e-3, F0, T0, 0, True, 0.0, 0, 0)
    assert e.value.status == 1          # SFG_ERR_ARG: PML without thickness


def _read(path):
    return np.array([np.array(l.split(), dtype=np.float64) for l in open(path) if l.strip()])


@pytest.mark.gpu
@pytest.mark.parametrize("pml", [0, 1])
def test_gpu_dropin_files(oracle, tmp_path, pml):
    """acoustic() / acoustic_pml() called as a C caller would: the model of
    acoustic_model.c (vp 2000 where x >= 0 and y >= 0, else 3000), u.dat and
    energy.dat in the working directory, and stif_{p,j,x}.dat with PML."""
    from seisfem_b200 import api
    L = api.lib()
    m = structured_mesh("Q4", 24, 20, -60.0, 180.0, -40.0, 160.0)
    src = int(np.argmin((m.x - 60.0) ** 2 + (m.y - 60.0) ** 2))
    step, dt = 242, 1e-3
    en = np.ascontiguousarray(m.element_node, np.int32)
    x, y = np.ascontiguousarray(m.x), np.ascontiguousarray(m.y)
    xy = (C.POINTER(C.c_double) * 2)(x.ctypes.data_as(C.POINTER(C.c_double)), y.ctypes.data_as(C.POINTER(C.c_double)))
    xyp = C.cast(xy, C.POINTER(C.POINTER(C.c_double)))
    head = (m.type_name.encode(), m.node_num, m.element_num, m.order, en.ctypes.data_as(C.POINTER(C.c_int)), xyp,
            m.element_num * m.order ** 2, m.node_num + 1, step, dt, F0, T0)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        if pml:
            f = L.acoustic_pml
            f.restype = None
            f.argtypes = ([C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.POINTER(C.c_double)),
                           C.c_int, C.c_int, C.c_int] + [C.c_double] * 8 + [C.c_int] * 3 + [C.c_char_p])
            f(*head, EDGE, m.xmin, m.xmax, m.ymin, m.ymax, PML_N, PML_N, src, b"masslump")
        else:
            f = L.acoustic
            f.restype = None
            f.argtypes = ([C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.POINTER(C.c_double)),
                           C.c_int, C.c_int, C.c_int] + [C.c_double] * 3 + [C.c_int, C.c_char_p])
            f(*head, src, b"masslump")
    finally:
        os.chdir(cwd)
    vp = np.where((m.x >= 0) & (m.y >= 0), 2000.0, 3000.0)
    ref = oracle.acoustic_run(m, vp, step, dt, F0, T0, src, bool(pml), EDGE, PML_N, PML_N)
    u = _read(tmp_path / "u.dat")
    e = np.array([float(l) for l in open(tmp_path / "energy.dat")])
    assert u.shape == ref["snap"].shape and e.shape == (step,)
    # "%f" text: six decimals
    assert np.abs(u - ref["snap"]).max() <= 1e-6 + 1e-9 * np.abs(ref["snap"]).max()
    assert np.abs(e - ref["energy"]).max() <= 1e-6 + 1e-9 * np.abs(ref["energy"]).max()
    if pml:
        ci, cj, cx = oracle.stif_coo(m, 6)
        Bp, Bj, Bx = oracle.coo2csr(m.node_num, ci, cj, cx)
        assert np.array_equal(np.loadtxt(tmp_path / "stif_p.dat", dtype=np.int64), Bp)
        assert np.array_equal(np.loadtxt(tmp_path / "stif_j.dat", dtype=np.int64), Bj)
        assert np.abs(np.loadtxt(tmp_path / "stif_x.dat") - Bx).max() <= 5e-7
