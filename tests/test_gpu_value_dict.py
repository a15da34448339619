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
