"""GPU seams (reference-shaped entry points) against the oracle, bit-exact."""
import numpy as np
import pytest

from seisfem_b200 import api
from seisfem_b200.problem import small_problem

pytestmark = pytest.mark.gpu

KAT_AI = [0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 3, 2, 2, 2, 1, 1, 1]
KAT_AJ = [0, 1, 2, 0, 1, 2, 0, 1, 2, 3, 2, 1, 3, 2, 1, 3, 2, 1]
KAT_AX = [1.0, -0.5, -0.5, -0.5, 0.5, 0.0, -0.5, 0.0, 0.5, 1.0, -0.5, -0.5, -0.5, 0.5, 0.0, -0.5, 0.0, 0.5]


def test_coo2csr_known_answer():
    # sparse_matrix/test_coo2csr_lib.c:10-12, expected result derived from the F90
    Bp, Bj, Bx = api.coo2csr_canonical(4, KAT_AI, KAT_AJ, KAT_AX)
    assert Bp.tolist() == [0, 3, 6, 9, 12]
    assert Bj.tolist() == [0, 1, 2, 0, 1, 3, 0, 2, 3, 1, 2, 3]
    assert Bx.tolist() == [1, -.5, -.5, -.5, 1, -.5, -.5, 1, -.5, -.5, -.5, 1]


def test_coo2csr_random_matches_oracle(oracle):
    rng = np.random.default_rng(4)
    n = 50
    ci = rng.integers(0, n, 4000).astype(np.int32)
    cj = rng.integers(0, n, 4000).astype(np.int32)
    cx = rng.choice([-1.0, 0.0, 0.5, 1e-300, 3.0], 4000)
    a = api.coo2csr_canonical(n, ci, cj, cx)
    b = oracle.coo2csr(n, ci, cj, cx)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


@pytest.mark.parametrize("etype", ["Q4", "Q9", "T3", "T6"])
def test_assembly_seams_bit_exact(oracle, etype):
    p = small_problem(etype, n=7, step=10, pml=2, seed=9)
    m = p.mesh
    a = api.mass_sparse_all(m, p.model.rho, 0)
    b = oracle.mass_coo(m, p.model.rho)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
    assert np.max(np.abs(api.mass_sparse_all(m, p.model.rho, 1) / oracle.mass_lumped(m, p.model.rho) - 1)) < 1e-13
    for k in range(7):
        a = api.stif_sparse_all(m, k)
        b = oracle.stif_coo(m, k)
        for u, v in zip(a, b):
            assert np.array_equal(u, v), (etype, k)


def test_mpml_and_matvec_seams(oracle):
    p = small_problem("Q9", n=10, step=10, pml=3, seed=2)
    m = p.mesh
    for use in [(1, 1, 1, 1), (1, 0, 1, 1)]:
        a = api.abc_mpml(m, 3, 3, p.edge_size, (m.xmin, m.xmax, m.ymin, m.ymax), 3500.0, use)
        b = oracle.abc_mpml(m, 3, 3, p.edge_size, (m.xmin, m.xmax, m.ymin, m.ymax), 3500.0, use)
        assert np.array_equal(a, b)
    Bp, Bj, Bx = oracle.coo2csr(m.node_num, *oracle.stif_coo(m, 3))
    x = np.random.default_rng(1).standard_normal(m.node_num)
    assert np.array_equal(api.csr_matvec(Bp, Bj, Bx, x), oracle.csr_matvec(Bp, Bj, Bx, x))
