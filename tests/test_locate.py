"""sfg_node_location (grid buckets) against the oracle's restatement of
source_receiver/node_location.c:13-27 (a scan keeping the last match):
identical answers on structured and scattered nodes, with points on the
edge_size / 2 boundaries, duplicated coordinates, misses and degenerate
edge sizes."""
import numpy as np

from seisfem_b200.api import node_location
from seisfem_b200.problem import structured_mesh


def _check(oracle, x, y, edge, px, py):
    class M:
        pass
    m = M()
    m.node_num, m.x, m.y = len(x), np.ascontiguousarray(x, np.float64), np.ascontiguousarray(y, np.float64)
    got = node_location(x, y, edge, px, py)
    want = np.array([oracle.node_location(m, edge, a, b) for a, b in zip(px, py)], np.int32)
    assert np.array_equal(got, want), np.nonzero(got != want)
    return got


def test_structured_meshes_and_boundaries(oracle):
    for typ, n in (("Q4", 20), ("Q9", 10), ("T6", 8)):
        mesh = structured_mesh(typ, n, n, 0.0, n * 10.0, 0.0, n * 10.0)
        rng = np.random.default_rng(n)
        h = 10.0
        # every node, points half an edge away (on the boundary), between nodes, outside
        px = np.concatenate([mesh.x, mesh.x + h / 2, mesh.x - h / 2, rng.uniform(-20, n * 10 + 20, 300)])
        py = np.concatenate([mesh.y, mesh.y, mesh.y + h / 2, rng.uniform(-20, n * 10 + 20, 300)])
        got = _check(oracle, mesh.x, mesh.y, h, px, py)
        assert (got[:mesh.node_num] >= 0).all()
        _check(oracle, mesh.x, mesh.y, h / 2, px, py)   # the Q9/T6 node spacing


def test_scattered_nodes_duplicates_and_degenerate_edges(oracle):
    rng = np.random.default_rng(7)
    x = rng.uniform(0, 1000, 2000)
    y = rng.uniform(-300, 300, 2000)
    x[1500:1600] = x[:100]           # duplicated coordinates: the later index wins
    y[1500:1600] = y[:100]
    px = np.concatenate([x[:200], rng.uniform(-50, 1050, 500), [np.inf, -1e300, 1e300]])
    py = np.concatenate([y[:200], rng.uniform(-350, 350, 500), [0.0, 0.0, 5.0]])
    for edge in (25.0, 3.0, 0.0, -1.0, 5000.0, 1e-9):
        got = _check(oracle, x, y, edge, px, py)
        if edge == 0.0:
            assert (got[:200] >= 0).all()
    assert (node_location(x, y, 25.0, x[:100], y[:100]) >= 1500).all()
