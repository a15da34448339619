"""sfg_abc_mpml_device_noalloc: the M-PML profiles of device-resident node
arrays, computed with the library's fixed device scratch instead of
allocations.  Compared bit for bit with the allocating seam sfg_abc_mpml on
two calls in a row (the second on a smaller mesh with a node that no element
references, so flags left over from the first call would show).  The first
call runs on a non-blocking stream (the kind the header recommends), the
second on the legacy default stream."""
import ctypes as C

import numpy as np
import pytest

from seisfem_b200 import api
from seisfem_b200.problem import Mesh, structured_mesh

pytestmark = pytest.mark.gpu

SFG_ERR_ARG, SFG_ERR_BADINDEX, SFG_ERR_LIMIT = 1, 5, 11
MAX_NODES = 1 << 22


def _fn():
    f = api.lib().sfg_abc_mpml_device_noalloc
    f.restype = C.c_int
    f.argtypes = ([C.c_int] * 3 + [C.c_void_p] * 3 + [C.c_int] * 2 + [C.c_double] * 6 + [C.c_int] * 4 +
                  [C.c_void_p, C.c_void_p])
    return f


def _with_orphan(m):
    """The mesh plus one node, inside the left M-PML strip, that no element uses."""
    x = np.append(m.x, m.xmin + 1.0)
    y = np.append(m.y, 0.5 * (m.ymin + m.ymax))
    return Mesh(m.type_name, m.element_node, x, y, m.xmin, m.xmax, m.ymin, m.ymax)


def _device_arrays(m, fill):
    import torch
    dev = torch.device("cuda:0")
    en = torch.from_numpy(np.ascontiguousarray(m.element_node, np.int32)).to(dev)
    x = torch.from_numpy(np.ascontiguousarray(m.x)).to(dev)
    y = torch.from_numpy(np.ascontiguousarray(m.y)).to(dev)
    out = torch.full((6, m.node_num), fill, dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    return en, x, y, out


def _noalloc(m, pml, h, vp_max, use, fill, stream=None):
    en, x, y, out = _device_arrays(m, fill)
    rc = _fn()(m.node_num, m.element_num, m.order, en.data_ptr(), x.data_ptr(), y.data_ptr(), pml, pml, h,
               m.xmin, m.xmax, m.ymin, m.ymax, vp_max, *use, out.data_ptr(), stream)
    return rc, out.cpu().numpy()


def _seam(m, pml, h, vp_max, use, fill):
    L = api.lib()
    outs = [np.full(m.node_num, fill) for _ in range(6)]
    rc = L.sfg_abc_mpml(m.node_num, m.element_num, m.order, m.element_node,
                        C.cast(api._xy(m.x, m.y), C.c_void_p), pml, pml, h, m.xmin, m.xmax, m.ymin, m.ymax,
                        vp_max, *use, *outs)
    assert rc == 0
    return np.stack(outs)


def test_noalloc_matches_allocating_seam_two_calls_in_a_row():
    import torch
    big = structured_mesh("Q9", 60, 50, 0.0, 600.0, 0.0, 500.0)
    small = _with_orphan(structured_mesh("Q4", 30, 20, 0.0, 300.0, 0.0, 200.0))
    # torch's pool streams are created with cudaStreamNonBlocking
    s = torch.cuda.Stream(torch.device("cuda:0"))
    calls = [(big, 8, 10.0, 4200.0, (1, 1, 1, 1), 0.0, s.cuda_stream),
             (small, 5, 10.0, 3100.0, (1, 0, 1, 1), 7.0, None)]
    for m, pml, h, vp, use, fill, stream in calls:
        rc, got = _noalloc(m, pml, h, vp, use, fill, stream)
        assert rc == 0
        want = _seam(m, pml, h, vp, use, fill)
        assert np.array_equal(got, want)
    assert np.all(got[:, -1] == 7.0)          # the orphan node keeps its value
    assert np.any(got[0] != 0.0)


def test_noalloc_limits_and_bad_index():
    import torch
    m = structured_mesh("Q4", 8, 8, 0.0, 80.0, 0.0, 80.0)
    dev = torch.device("cuda:0")
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    p = buf.data_ptr()
    f = _fn()
    assert f(MAX_NODES + 1, 1, 4, p, p, p, 2, 2, 10.0, 0.0, 80.0, 0.0, 80.0, 3000.0, 1, 1, 1, 1, p, None) == SFG_ERR_LIMIT
    assert api.lib().sfg_error_string(SFG_ERR_LIMIT) == b"size above the fixed limit of a no-allocation entry point"
    en = np.array(m.element_node, np.int32)
    en[5] = m.node_num + 3                      # out of range: reported, nothing written
    bad = Mesh("Q4", en, m.x, m.y, m.xmin, m.xmax, m.ymin, m.ymax)
    rc, got = _noalloc(bad, 2, 10.0, 3000.0, (1, 1, 1, 1), -3.0)
    assert rc == SFG_ERR_BADINDEX
    assert np.all(got == -3.0)
    rc, got = _noalloc(m, 2, 10.0, 3000.0, (1, 1, 1, 1), 0.0)   # the error word is cleared per call
    assert rc == 0 and np.array_equal(got, _seam(m, 2, 10.0, 3000.0, (1, 1, 1, 1), 0.0))


def test_noalloc_refuses_a_capturing_stream():
    """The call reads its error word back and waits for its stream, which a
    capturing stream does not allow: it returns SFG_ERR_ARG and the caller's
    capture stays valid."""
    import torch
    m = structured_mesh("Q4", 8, 8, 0.0, 80.0, 0.0, 80.0)
    en, x, y, out = _device_arrays(m, 0.0)
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream(torch.device("cuda:0"))
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            rc = _fn()(m.node_num, m.element_num, m.order, en.data_ptr(), x.data_ptr(), y.data_ptr(), 2, 2, 10.0,
                       m.xmin, m.xmax, m.ymin, m.ymax, 3000.0, 1, 1, 1, 1, out.data_ptr(), s.cuda_stream)
            out.add_(1.0)                       # the capture goes on after the refusal
    assert rc == SFG_ERR_ARG
    g.replay()
    torch.cuda.synchronize()
    assert torch.all(out == 1.0)
