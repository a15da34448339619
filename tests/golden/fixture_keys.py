"""What identifies and what is kept in the full-size reference fixtures
(config1_reference.npz, config2_reference.npz).  Shared by the script that
writes them (make_golden.py) and the tests that read them."""
import numpy as np

# config -> (receiver stride, grid-line stride of the snapshot nodes)
FULL_CONFIG_STRIDES = {"config1": (4, 8), "config2": (10, 16)}


def input_checksum(prob) -> np.ndarray:
    """Sums that identify a problem's inputs (mesh, model, nodes, loop)."""
    m = prob.mesh
    return np.array([m.node_num, m.element_num, float(m.element_node.sum()), m.x.sum(), m.y.sum(),
                     prob.model.rho.sum(), prob.model.c.sum(), float(prob.src_node.sum()),
                     float(prob.rec_node.sum()), prob.step, prob.dt, prob.f0], np.float64)


def full_config_subset(prob, rec_stride, grid_stride):
    """Receiver columns and snapshot nodes kept in a full-size fixture: every
    rec_stride-th receiver, and the nodes on every grid_stride-th grid line of
    the structured node grid in both directions."""
    side = int(round(prob.mesh.node_num ** 0.5))
    assert side * side == prob.mesh.node_num
    rec = np.arange(0, len(prob.rec_node), rec_stride)
    g = np.arange(0, side, grid_stride)
    nodes = (g[None, :] + side * g[:, None]).ravel()
    return rec.astype(np.int32), nodes.astype(np.int32)
