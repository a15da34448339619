"""The value dictionary of the one-shot step kernels (sfg_dict.cu): on meshes
of congruent elements the union entries reduce to a few dozen tuples
(M / rho_row, K1..K6) and the kernels read (column, tuple id) slots.  Checked
against the FP64 oracle, against the full-value slots of the same problem
(SFG_NO_VALUE_DICT=1), and on a mesh whose elements all differ (sinusoidal
topography), where set-up keeps the full-value slots."""
import numpy as np
import pytest

from conftest import rel_l2
from seisfem_b200.problem import config_2, config_4, small_problem

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-4


def _run(p, monkeypatch, no_dict):
    from seisfem_b200.api import Context
    if no_dict:
        monkeypatch.setenv("SFG_NO_VALUE_DICT", "1")
    else:
        monkeypatch.delenv("SFG_NO_VALUE_DICT", raising=False)
    ctx = Context(0)
    try:
        ctx.setup(p)
        tuples = ctx.stats()["value_tuples"]
        out = ctx.run(p, precision="fp32k")
    finally:
        ctx.close()
    return tuples, out


@pytest.mark.parametrize("make", [lambda: config_2(n=40, step=402, pml=6),
                                  lambda: small_problem("Q4", n=48, step=302, pml=6, seed=11),
                                  lambda: config_4(nx=30, ny=60, pml=5, step=202, amp=0.0)],
                         ids=["q9_layered", "q4_smooth_model", "t6_flat_vti"])
def test_dictionary_matches_full_values_and_oracle(oracle, monkeypatch, make):
    p = make()
    t_dict, a = _run(p, monkeypatch, no_dict=False)
    t_full, b = _run(p, monkeypatch, no_dict=True)
    assert 0 < t_dict <= 512 and t_full == 0, (t_dict, t_full)
    ref = oracle.run(p)
    for k in ("seis_u", "seis_w", "snap_u", "snap_w"):
        # the two slot layouts round the same FP32 products in another order
        assert rel_l2(a[k], b[k]) < 1e-5, (k, rel_l2(a[k], b[k]))
        assert rel_l2(a[k], ref[k]) < FP32_TOL, (k, rel_l2(a[k], ref[k]))


def test_distinct_elements_keep_full_value_slots(oracle, monkeypatch):
    # every element of the topography mesh has its own shape
    p = config_4(nx=30, ny=60, pml=5, step=202)
    t, out = _run(p, monkeypatch, no_dict=False)
    assert t == 0
    ref = oracle.run(p)
    for k in ("seis_u", "seis_w"):
        assert rel_l2(out[k], ref[k]) < FP32_TOL, k


def _run_shape(p, monkeypatch, shape_a, shape_z, no_tiles=False, morton=False):
    from seisfem_b200.api import Context
    monkeypatch.delenv("SFG_NO_VALUE_DICT", raising=False)
    monkeypatch.setenv("SFG_MORTON", "1" if morton else "0")
    if no_tiles:
        monkeypatch.setenv("SFG_NO_TILES", "1")
    else:
        monkeypatch.delenv("SFG_NO_TILES", raising=False)
    monkeypatch.setenv("SFG_SHAPE_A", str(shape_a))
    monkeypatch.setenv("SFG_SHAPE_Z", str(shape_z))
    ctx = Context(0)
    try:
        ctx.setup(p)
        out = ctx.run(p, precision="fp32k")
        out["rows_per_block"] = ctx.stats()["rows_per_block"]
    finally:
        ctx.close()
    return out


TILE = 6           # the staged-gather tile kernels' launch shape
STAGED_SLOTS = 7   # one-shot kernels with their slot streams staged in shared memory


@pytest.mark.parametrize("make", [lambda: config_2(n=40, step=402, pml=6),
                                  lambda: small_problem("Q4", n=48, step=302, pml=6, seed=11),
                                  lambda: small_problem("T6", n=24, step=102, pml=4, seed=5, dt=2.5e-4)],
                         ids=["q9_layered", "q4_smooth_model", "t6"])
def test_staged_tiles_match_unstaged_kernels_and_oracle(oracle, monkeypatch, make):
    """The staged-gather tile kernels (halo in shared memory, 4-byte slots;
    Morton order inside the classes, SFG_MORTON=1) against the unstaged
    dictionary kernels on the same numbering, and both against the FP64
    oracle; also with one class staged and the other not, and with staged
    slot streams."""
    p = make()
    morton = True
    tiles = _run_shape(p, monkeypatch, TILE, TILE, morton=morton)
    assert tiles["rows_per_block"] == TILE * 16 + TILE
    plain = _run_shape(p, monkeypatch, 0, 0, morton=morton)
    mixed = _run_shape(p, monkeypatch, TILE, 0, morton=morton)
    staged = _run_shape(p, monkeypatch, STAGED_SLOTS, STAGED_SLOTS, morton=morton)
    ref = oracle.run(p)
    for k in ("seis_u", "seis_w", "snap_u", "snap_w"):
        assert rel_l2(tiles[k], plain[k]) < 1e-6, (k, rel_l2(tiles[k], plain[k]))
        assert rel_l2(mixed[k], plain[k]) < 1e-6, (k, rel_l2(mixed[k], plain[k]))
        # the staged slot streams change nothing in the arithmetic
        assert np.array_equal(staged[k], plain[k]), (k, rel_l2(staged[k], plain[k]))
        assert rel_l2(tiles[k], ref[k]) < FP32_TOL, (k, rel_l2(tiles[k], ref[k]))


def test_mesh_order_without_tiles_matches(oracle, monkeypatch):
    """Without SFG_MORTON=1 (here also SFG_NO_TILES=1) the classes keep the
    mesh order and no tiles are built: the staged slot streams still work,
    bit for bit, and a pinned tile shape is refused."""
    from seisfem_b200.api import SfgError
    p = config_2(n=30, step=302, pml=5)
    a = _run_shape(p, monkeypatch, 0, 0, no_tiles=True)
    ref = oracle.run(p)
    b = _run_shape(p, monkeypatch, STAGED_SLOTS, STAGED_SLOTS, no_tiles=True)
    for k in ("seis_u", "seis_w"):
        assert rel_l2(a[k], ref[k]) < FP32_TOL, k
        assert np.array_equal(a[k], b[k]), k
    with pytest.raises(SfgError):
        _run_shape(p, monkeypatch, TILE, TILE, no_tiles=True)


def test_class_a_rows_are_a_multiple_of_32(oracle):
    """The set-up moves the last few class-A rows into class Z so that the
    class-A row count is a multiple of 32 (the one-shot state blocks of the
    two classes line up); the moved rows run the split-field step and the
    results stay within the FP32 tolerance of the oracle."""
    from seisfem_b200.api import Context
    for p in (config_2(n=30, step=202, pml=5), small_problem("Q4", n=37, step=202, pml=3, seed=4)):
        ctx = Context(0)
        try:
            ctx.setup(p)
            out = ctx.run(p, precision="fp32k", want_snapshots=True)
            st = ctx.stats()
        finally:
            ctx.close()
        assert st["interior_rows"] % 32 == 0 and st["interior_rows"] > 0
        ref = oracle.run(p)
        for k in ("seis_u", "seis_w", "snap_u", "snap_w"):
            assert rel_l2(out[k], ref[k]) < FP32_TOL, k


def test_tuple_table_in_parameters_matches_shared_memory(monkeypatch):
    """The one-shot kernels read the tuple table from their parameters (at
    most 128 tuples) or from shared memory (more tuples, the multi-mesh
    kernels, SFG_TABLE_SMEM=1): the same values, so the same results bit for
    bit."""
    p = config_2(n=40, step=302, pml=6)
    monkeypatch.delenv("SFG_TABLE_SMEM", raising=False)
    a = _run_shape(p, monkeypatch, 0, 0, no_tiles=True)
    monkeypatch.setenv("SFG_TABLE_SMEM", "1")
    b = _run_shape(p, monkeypatch, 0, 0, no_tiles=True)
    for k in ("seis_u", "seis_w", "snap_u", "snap_w"):
        assert np.array_equal(a[k], b[k]), (k, rel_l2(a[k], b[k]))
