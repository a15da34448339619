"""Python host mirror of the libseisfem_b200.so C ABI (include/seisfem_b200.h).

``Context`` wraps the sfg_ctx API (assemble once, run many shots);
``elastic_wave`` mirrors the reference entry point
(time_evolution/elastic_wave.c:1-3) with arrays in and results returned
instead of text files.  Every call goes through the shared library; there is
no CPU or PyTorch fallback: a missing library or device raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .problem import Problem

LIBPATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libseisfem_b200.so")

SFG_OK, SFG_ERR_BLOWUP, SFG_ERR_NOCONV = 0, 6, 12
# "fp64cm": FP64 with the consistent mass matrix (solver "pardiso" / "mgmres")
PRECISIONS = {"fp32k": 0, "fp32": 1, "fp64": 2, "plain": 3, "fp64cm": 4}

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


class SfgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"sfg status {status}: {msg}")
        self.status = status


class Mesh_(C.Structure):
    _fields_ = [("type", C.c_char_p), ("node_num", C.c_int), ("element_num", C.c_int),
                ("element_order", C.c_int), ("element_node", C.c_void_p), ("x", C.c_void_p),
                ("y", C.c_void_p), ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double),
                ("ymax", C.c_double), ("edge_size", C.c_double), ("pml_nx", C.c_int), ("pml_ny", C.c_int),
                ("free_surface", C.c_int)]


class Model_(C.Structure):
    _fields_ = [("rho", C.c_void_p), ("vp", C.c_void_p), ("vs", C.c_void_p), ("c", C.c_void_p)]


class RunDesc_(C.Structure):
    _fields_ = [("step", C.c_int), ("dt", C.c_double), ("f0", C.c_double), ("t0", C.c_double),
                ("src_num", C.c_int), ("src_node", C.c_void_p), ("rec_num", C.c_int), ("rec_node", C.c_void_p),
                ("precision", C.c_int), ("snap_every", C.c_int), ("shots_per_batch", C.c_int)]


class Stats_(C.Structure):
    _fields_ = [("setup_ms", C.c_double), ("loop_ms", C.c_double), ("total_ms", C.c_double),
                ("dof_steps", C.c_longlong), ("union_nnz", C.c_longlong), ("csr_nnz", C.c_longlong * 7),
                ("kernel_launches", C.c_int), ("rows_per_block", C.c_int), ("blowup_step", C.c_int),
                ("interior_rows", C.c_int), ("pml_rows", C.c_int), ("value_tuples", C.c_int),
                ("cm_iterations", C.c_int)]


class AcousticDesc_(C.Structure):
    _fields_ = [("pml", C.c_int), ("step", C.c_int), ("dt", C.c_double), ("f0", C.c_double), ("t0", C.c_double),
                ("source_node", C.c_int), ("mass_lump", C.c_void_p)]


class AcousticStats_(C.Structure):
    _fields_ = [("setup_ms", C.c_double), ("loop_ms", C.c_double), ("union_nnz", C.c_longlong),
                ("csr_nnz", C.c_longlong * 5), ("kernel_launches", C.c_int), ("blowup_step", C.c_int)]


_LIB = None

# every symbol the header declares (checked by the CPU test suite)
EXPORTS = ["sfg_create", "sfg_destroy", "sfg_error_string", "sfg_last_error", "sfg_setup", "sfg_csr_nnz",
           "sfg_csr_copy", "sfg_lumped_mass_copy", "sfg_lumped_mass_set", "sfg_union_copy", "sfg_mpml_copy", "sfg_run", "sfg_snapshot_rows",
           "sfg_get_stats", "sfg_run_device", "sfg_sync", "sfg_plan_create", "sfg_plan_batches",
           "sfg_plan_launches", "sfg_plan_launch", "sfg_plan_finish", "sfg_plan_destroy", "elastic_wave", "sfg_mass_sparse_all",
           "sfg_stif_sparse_all", "sfg_coo2csr_canonical", "sfg_abc_mpml", "sfg_csr_matvec", "sfg_node_location",
           "sfg_abc_mpml_device_noalloc", "sfg_plan_create_models", "sfg_run_models", "sfg_group_create", "sfg_group_launch", "sfg_group_launches",
           "sfg_group_fused", "sfg_group_destroy",
           # scalar acoustic solvers (include/seisfem_acoustic.h)
           "sfg_acoustic_snapshot_rows", "sfg_acoustic_run", "acoustic", "acoustic_pml",
           # learned surrogate (include/seisfem_fno.h)
           "sfg_fno_gemm", "sfg_fno_dft_combine", "sfg_fno_dft_combine_bwd", "sfg_fno_expand_weights",
           "sfg_fno_fold_weights", "sfg_fno_gelu_bwd", "sfg_fno_cast_bf16", "sfg_fno_bias_grad", "sfg_fno_swap01",
           "sfg_fno_zero", "sfg_fno_scale", "sfg_fno_rel_loss", "sfg_fno_adam", "sfg_fno_tc_timeouts",
           "sfg_fno_head_infer"]


def lib(path: str = LIBPATH):
    """Load the C-ABI library (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m seisfem_b200.build`")
    L = C.CDLL(path)
    L.sfg_create.restype = C.c_void_p
    L.sfg_create.argtypes = [C.c_int]
    L.sfg_destroy.argtypes = [C.c_void_p]
    L.sfg_error_string.restype = C.c_char_p
    L.sfg_error_string.argtypes = [C.c_int]
    L.sfg_last_error.restype = C.c_char_p
    L.sfg_last_error.argtypes = [C.c_void_p]
    L.sfg_setup.argtypes = [C.c_void_p, C.POINTER(Mesh_), C.POINTER(Model_)]
    L.sfg_csr_nnz.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    L.sfg_csr_copy.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    L.sfg_lumped_mass_copy.argtypes = [C.c_void_p, C.c_void_p]
    L.sfg_mpml_copy.argtypes = [C.c_void_p, C.c_void_p]
    L.sfg_lumped_mass_set.argtypes = [C.c_void_p, C.c_void_p]
    L.sfg_union_copy.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_longlong)]
    L.sfg_run.argtypes = [C.c_void_p, C.POINTER(RunDesc_)] + [C.c_void_p] * 4
    L.sfg_run_device.argtypes = [C.c_void_p, C.POINTER(RunDesc_), C.c_void_p, C.c_void_p, C.c_void_p]
    L.sfg_sync.argtypes = [C.c_void_p]
    L.sfg_plan_create.argtypes = [C.c_void_p, C.POINTER(RunDesc_), C.POINTER(C.c_void_p)]
    L.sfg_plan_batches.argtypes = [C.c_void_p]
    L.sfg_run_models.argtypes = [C.c_void_p, C.POINTER(RunDesc_), C.c_void_p] + [C.c_void_p] * 4
    L.sfg_plan_create_models.argtypes = [C.c_void_p, C.POINTER(RunDesc_), C.c_void_p, C.POINTER(C.c_void_p)]
    L.sfg_group_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]
    L.sfg_group_launch.argtypes = [C.c_void_p, C.c_void_p]
    L.sfg_group_launches.argtypes = [C.c_void_p]
    L.sfg_group_fused.argtypes = [C.c_void_p]
    L.sfg_group_destroy.argtypes = [C.c_void_p]
    L.sfg_plan_launches.argtypes = [C.c_void_p]
    L.sfg_plan_launch.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    L.sfg_plan_finish.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 5
    L.sfg_plan_destroy.argtypes = [C.c_void_p]
    L.sfg_snapshot_rows.argtypes = [C.c_int, C.c_int]
    L.sfg_get_stats.argtypes = [C.c_void_p, C.POINTER(Stats_)]
    L.sfg_mass_sparse_all.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, _i32p, C.c_void_p, _f64p,
                                      _i32p, _i32p, _f64p, C.c_int]
    L.sfg_stif_sparse_all.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, _i32p, C.c_void_p,
                                      _i32p, _i32p, _f64p, C.c_int]
    L.sfg_coo2csr_canonical.argtypes = [C.POINTER(C.c_int)] * 3 + [_i32p, _i32p, _f64p, _i32p, _i32p, _f64p]
    L.sfg_abc_mpml.argtypes = ([C.c_int, C.c_int, C.c_int, _i32p, C.c_void_p, C.c_int, C.c_int] +
                               [C.c_double] * 6 + [C.c_int] * 4 + [_f64p] * 6)
    L.sfg_csr_matvec.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
    L.sfg_acoustic_snapshot_rows.argtypes = [C.c_int, C.c_int]
    L.sfg_acoustic_run.argtypes = [C.c_void_p, C.POINTER(Mesh_), C.c_void_p, C.POINTER(AcousticDesc_),
                                   C.c_void_p, C.c_void_p, C.POINTER(AcousticStats_)]
    _LIB = L
    return L


def node_location(x, y, edge_size: float, px, py):
    """Node index per point (sfg_node_location: the last node within
    edge_size / 2 in both axes, -1 when none)."""
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    px = np.ascontiguousarray(np.atleast_1d(px), np.float64)
    py = np.ascontiguousarray(np.atleast_1d(py), np.float64)
    out = np.empty(len(px), np.int32)
    f = lib().sfg_node_location
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    rc = f(len(x), float(edge_size), x.ctypes.data, y.ctypes.data, len(px), px.ctypes.data, py.ctypes.data,
           out.ctypes.data)
    if rc:
        raise SfgError(rc, "sfg_node_location")
    return out


def _xy(x, y):
    arr = (C.POINTER(C.c_double) * 2)(x.ctypes.data_as(C.POINTER(C.c_double)),
                                      y.ctypes.data_as(C.POINTER(C.c_double)))
    return arr


class Context:
    """One device context: ``setup(problem)`` assembles on the GPU,
    ``run(...)`` advances shots and returns seismograms/snapshots."""

    def __init__(self, device: int = 0):
        self.L = lib()
        self.ptr = self.L.sfg_create(device)
        if not self.ptr:
            raise RuntimeError(f"sfg_create({device}) failed: no sm_100 CUDA device")
        self._keep = []

    def close(self):
        if self.ptr:
            self.L.sfg_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, allow=()):
        if rc != SFG_OK and rc not in allow:
            raise SfgError(rc, self.L.sfg_last_error(self.ptr).decode())
        return rc

    def setup(self, prob: Problem):
        m, md = prob.mesh, prob.model
        self._keep = [np.ascontiguousarray(a) for a in (m.element_node, m.x, m.y, md.rho, md.vp, md.vs, md.c)]
        en, x, y, rho, vp, vs, c = self._keep
        self._type = m.type_name.encode()
        mesh = Mesh_(self._type, m.node_num, m.element_num, m.order, en.ctypes.data, x.ctypes.data, y.ctypes.data,
                     m.xmin, m.xmax, m.ymin, m.ymax, prob.edge_size, prob.pml_nx, prob.pml_ny, prob.free_surface)
        model = Model_(rho.ctypes.data, vp.ctypes.data, vs.ctypes.data, c.ctypes.data)
        self._check(self.L.sfg_setup(self.ptr, C.byref(mesh), C.byref(model)))
        self.node_num = m.node_num
        return self

    def acoustic_run(self, mesh, vp, step: int, dt: float, f0: float, t0: float, source_node: int,
                     pml: bool = False, edge_size: float = 0.0, pml_nx: int = 0, pml_ny: int = 0,
                     mass_lump=None, snapshots: bool = True) -> dict:
        """The scalar acoustic solvers (time_evolution/acoustic.c, acoustic_pml.c)
        on the GPU: {"snap": [rows][N] or None, "energy": [step], "status",
        "stats"}.  ``mesh`` is a problem.Mesh; ``mass_lump`` (optional) replaces
        the lumped mass assembled on the GPU.  A run that the PML solver's
        energy bound ends returns status SFG_ERR_BLOWUP with the outputs
        written before it."""
        en, x, y = (np.ascontiguousarray(a) for a in (mesh.element_node, mesh.x, mesh.y))
        vp = np.ascontiguousarray(vp, np.float64)
        tname = mesh.type_name.encode()
        md = Mesh_(tname, mesh.node_num, mesh.element_num, mesh.order, en.ctypes.data, x.ctypes.data,
                   y.ctypes.data, mesh.xmin, mesh.xmax, mesh.ymin, mesh.ymax, edge_size, pml_nx, pml_ny, 0)
        ml = None if mass_lump is None else np.ascontiguousarray(mass_lump, np.float64)
        desc = AcousticDesc_(int(bool(pml)), step, dt, f0, t0, source_node, None if ml is None else ml.ctypes.data)
        rows = self.L.sfg_acoustic_snapshot_rows(step, int(bool(pml)))
        snap = np.zeros((rows, mesh.node_num)) if snapshots else None
        energy = np.zeros(step)
        st = AcousticStats_()
        rc = self._check(self.L.sfg_acoustic_run(self.ptr, C.byref(md), vp.ctypes.data, C.byref(desc),
                                                 None if snap is None else snap.ctypes.data, energy.ctypes.data,
                                                 C.byref(st)), allow=(SFG_ERR_BLOWUP,))
        stats = {k: getattr(st, k) for k, _ in AcousticStats_._fields_}
        stats["csr_nnz"] = list(st.csr_nnz)
        return {"snap": snap, "energy": energy, "status": rc, "stats": stats}

    def csr(self, matrix: int):
        n = C.c_int()
        self._check(self.L.sfg_csr_nnz(self.ptr, matrix, C.byref(n)))
        p = np.zeros(self.node_num + 1, np.int32)
        j = np.zeros(max(n.value, 1), np.int32)
        x = np.zeros(max(n.value, 1))
        self._check(self.L.sfg_csr_copy(self.ptr, matrix, p.ctypes.data, j.ctypes.data, x.ctypes.data))
        return p, j[:n.value], x[:n.value]

    def lumped_mass(self):
        m = np.zeros(self.node_num)
        self._check(self.L.sfg_lumped_mass_copy(self.ptr, m.ctypes.data))
        return m

    def union_pattern(self):
        n = C.c_longlong()
        self._check(self.L.sfg_union_copy(self.ptr, None, None, C.byref(n)))
        p = np.zeros(self.node_num + 1, np.int32)
        j = np.zeros(max(n.value, 1), np.int32)
        self._check(self.L.sfg_union_copy(self.ptr, p.ctypes.data, j.ctypes.data, C.byref(n)))
        return p, j[:n.value]

    def set_lumped_mass(self, m):
        m = np.ascontiguousarray(m, np.float64)
        self._check(self.L.sfg_lumped_mass_set(self.ptr, m.ctypes.data))

    def mpml(self):
        m = np.zeros(6 * self.node_num)
        self._check(self.L.sfg_mpml_copy(self.ptr, m.ctypes.data))
        return m.reshape(6, self.node_num)

    def stats(self) -> dict:
        s = Stats_()
        self.L.sfg_get_stats(self.ptr, C.byref(s))
        d = {k: getattr(s, k) for k, _ in Stats_._fields_}
        d["csr_nnz"] = list(s.csr_nnz)
        return d

    def run(self, prob: Problem, precision: str = "fp32k", snap_every: int = 200, shots_per_batch: int = 0,
            src_node=None, want_snapshots: bool = True, raise_on_blowup: bool = True):
        src = np.ascontiguousarray(prob.src_node if src_node is None else src_node, np.int32)
        rec = np.ascontiguousarray(prob.rec_node, np.int32)
        S, R, step, N = len(src), len(rec), prob.step, prob.mesh.node_num
        ns = self.L.sfg_snapshot_rows(step, snap_every) if (snap_every and want_snapshots) else 0
        out = {"seis_u": np.zeros((S, step - 2, R)), "seis_w": np.zeros((S, step - 2, R))}
        if ns:
            out["snap_u"] = np.zeros((S, ns, N))
            out["snap_w"] = np.zeros((S, ns, N))
        desc = RunDesc_(step, prob.dt, prob.f0, prob.t0, S, src.ctypes.data, R, rec.ctypes.data,
                        PRECISIONS[precision], snap_every if ns else 0, shots_per_batch)
        rc = self.L.sfg_run(self.ptr, C.byref(desc), out["seis_u"].ctypes.data, out["seis_w"].ctypes.data,
                            out["snap_u"].ctypes.data if ns else None, out["snap_w"].ctypes.data if ns else None)
        self._check(rc, allow=() if raise_on_blowup else (SFG_ERR_BLOWUP,))
        out["status"] = rc
        out["stats"] = self.stats()
        return out

    def run_models(self, prob: Problem, models, shots_per_batch: int = 0, snap_every: int = 0,
                   raise_on_blowup: bool = True):
        """Shot s of prob.src_node runs in models[s] (a Model on this mesh):
        sfg_run_models, compensated FP32, batches of 32 or 64 shots."""
        src = np.ascontiguousarray(prob.src_node, np.int32)
        rec = np.ascontiguousarray(prob.rec_node, np.int32)
        S, R, step, N = len(src), len(rec), prob.step, prob.mesh.node_num
        if len(models) != S:
            raise ValueError("one model per shot")
        keep = [[np.ascontiguousarray(a, np.float64) for a in (md.rho, md.vp, md.vs, md.c)] for md in models]
        arr = (Model_ * S)(*[Model_(*(a.ctypes.data for a in k)) for k in keep])
        ns = self.L.sfg_snapshot_rows(step, snap_every) if snap_every else 0
        out = {"seis_u": np.zeros((S, step - 2, R)), "seis_w": np.zeros((S, step - 2, R))}
        if ns:
            out["snap_u"] = np.zeros((S, ns, N))
            out["snap_w"] = np.zeros((S, ns, N))
        desc = RunDesc_(step, prob.dt, prob.f0, prob.t0, S, src.ctypes.data, R, rec.ctypes.data,
                        PRECISIONS["fp32k"], snap_every if ns else 0, shots_per_batch)
        rc = self.L.sfg_run_models(self.ptr, C.byref(desc), arr, out["seis_u"].ctypes.data,
                                   out["seis_w"].ctypes.data, out["snap_u"].ctypes.data if ns else None,
                                   out["snap_w"].ctypes.data if ns else None)
        self._check(rc, allow=() if raise_on_blowup else (SFG_ERR_BLOWUP,))
        out["status"] = rc
        out["stats"] = self.stats()
        return out

    def run_device(self, prob: Problem, d_seis_u: int, d_seis_w: int, stream: int = 0, precision: str = "fp32k",
                   shots_per_batch: int = 0, src_node=None):
        """Device-resident run: seismograms [S][step-2][R] FP64 written to the
        given device pointers; no host copies of outputs."""
        src = np.ascontiguousarray(prob.src_node if src_node is None else src_node, np.int32)
        rec = np.ascontiguousarray(prob.rec_node, np.int32)
        desc = RunDesc_(prob.step, prob.dt, prob.f0, prob.t0, len(src), src.ctypes.data, len(rec), rec.ctypes.data,
                        PRECISIONS[precision], 0, shots_per_batch)
        self._check(self.L.sfg_run_device(self.ptr, C.byref(desc), d_seis_u, d_seis_w, stream or None))
        return self.stats()


class Plan:
    """A prepared run (sfg_plan_*): one CUDA-graph launch per batch of shots."""

    def __init__(self, ctx: Context, prob: Problem, precision: str = "fp32k", snap_every: int = 0,
                 shots_per_batch: int = 0, src_node=None):
        self.ctx, self.L = ctx, ctx.L
        self.src = np.ascontiguousarray(prob.src_node if src_node is None else src_node, np.int32)
        self.rec = np.ascontiguousarray(prob.rec_node, np.int32)
        self.step, self.N = prob.step, prob.mesh.node_num
        self.desc = RunDesc_(prob.step, prob.dt, prob.f0, prob.t0, len(self.src), self.src.ctypes.data,
                             len(self.rec), self.rec.ctypes.data, PRECISIONS[precision], snap_every, shots_per_batch)
        h = C.c_void_p()
        ctx._check(self.L.sfg_plan_create(ctx.ptr, C.byref(self.desc), C.byref(h)))
        self.ptr = h
        self.batches = self.L.sfg_plan_batches(h)
        self.launches = self.L.sfg_plan_launches(h)
        self.snap_rows = self.L.sfg_snapshot_rows(prob.step, snap_every) if snap_every else 0

    def launch(self, batch: int = 0, stream: int = 0):
        self.ctx._check(self.L.sfg_plan_launch(self.ptr, batch, stream or None))
        # plans queued directly (consistent mass) count their kernels as they queue them
        self.launches = self.L.sfg_plan_launches(self.ptr)

    def finish(self, batch: int = 0, out=None, stream: int = 0, raise_on_blowup: bool = True):
        """Wait for `batch`, copy its outputs into `out` (dict of host arrays;
        created when None) and apply the energy bound."""
        S, R = len(self.src), len(self.rec)
        if out is None:
            out = {"seis_u": np.zeros((S, self.step - 2, R)), "seis_w": np.zeros((S, self.step - 2, R))}
            if self.snap_rows:
                out["snap_u"] = np.zeros((S, self.snap_rows, self.N))
                out["snap_w"] = np.zeros((S, self.snap_rows, self.N))
        ptr = lambda k: out[k].ctypes.data if k in out else None
        rc = self.L.sfg_plan_finish(self.ptr, batch, ptr("seis_u"), ptr("seis_w"), ptr("snap_u"), ptr("snap_w"),
                                    stream or None)
        self.ctx._check(rc, allow=() if raise_on_blowup else (SFG_ERR_BLOWUP,))
        out["status"] = rc
        return out

    def finish_device(self, batch: int, d_seis_u: int, d_seis_w: int, stream: int = 0,
                      raise_on_blowup: bool = True) -> int:
        """Wait for `batch` and copy its seismograms into device buffers
        (the full [src_num][step-2][rec] layout, this batch's shots at their
        offset); no host copies of outputs."""
        rc = self.L.sfg_plan_finish(self.ptr, batch, d_seis_u, d_seis_w, None, None, stream or None)
        self.ctx._check(rc, allow=() if raise_on_blowup else (SFG_ERR_BLOWUP,))
        return rc

    def close(self):
        if self.ptr:
            self.L.sfg_plan_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_runner(ctx: "Context", precision: str = "fp32k", stream=None):
    """A runner for shots.run_sharded: advances a (sub-)problem's shots on
    the context's device with a Plan and returns its seismograms as CUDA
    tensors [shots][step-2][rec] (torch owns the output memory)."""
    import torch

    def run(sub):
        S, R, rows = len(sub.src_node), len(sub.rec_node), sub.step - 2
        dev = torch.device("cuda", torch.cuda.current_device())
        su = torch.empty((S, rows, R), dtype=torch.float64, device=dev)
        sw = torch.empty((S, rows, R), dtype=torch.float64, device=dev)
        if S == 0:                 # a rank with no shots still joins the gather
            return su, sw
        sh = stream.cuda_stream if stream is not None else 0
        plan = Plan(ctx, sub, precision=precision, snap_every=0)
        try:
            for b in range(plan.batches):
                plan.launch(b, sh)
                plan.finish_device(b, su.data_ptr(), sw.data_ptr(), sh)
        finally:
            plan.close()
        return su, sw
    return run


class Group:
    """Several single-batch plans (independent meshes) as one CUDA-graph
    launch (sfg_group_*); results are read per plan with Plan.finish().
    ``fused``: the graph runs one class-A and one class-Z kernel per time
    step for all meshes (otherwise the plans' own graphs side by side)."""

    def __init__(self, plans):
        self.plans = list(plans)
        self.L = self.plans[0].L
        arr = (C.c_void_p * len(self.plans))(*[p.ptr.value for p in self.plans])
        h = C.c_void_p()
        rc = self.L.sfg_group_create(arr, len(self.plans), C.byref(h))
        if rc:
            raise SfgError(rc, "sfg_group_create")
        self.ptr = h
        self.launches = self.L.sfg_group_launches(h)
        f = self.L.sfg_group_fused(h)
        self.fused = f > 0
        self.shapes = {"variant_A": (f - 1) // 16, "variant_Z": (f - 1) % 16} if f > 0 else None

    def launch(self, stream: int = 0):
        rc = self.L.sfg_group_launch(self.ptr, stream or None)
        if rc:
            raise SfgError(rc, "sfg_group_launch")

    def close(self):
        if self.ptr:
            self.L.sfg_group_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def elastic_wave(prob: Problem, precision: str = "fp32k", device: int = 0, snap_every: int = 200):
    """Mirror of the reference's elastic_wave(): one call, assembled and run on
    the GPU; returns seismograms [src][step-2][rec] and snapshots."""
    ctx = Context(device)
    try:
        ctx.setup(prob)
        return ctx.run(prob, precision=precision, snap_every=snap_every)
    finally:
        ctx.close()


# ------------------------------------------------------------- the seams

def mass_sparse_all(mesh, rho, lumpflag: int):
    """assemble/mass_sparse_all.c:13-68 on the GPU (COO, or the lumped mass)."""
    L = lib()
    p, E = mesh.order, mesh.element_num
    n = E * p * p
    mi, mj = np.zeros(n, np.int32), np.zeros(n, np.int32)
    mx = np.zeros(max(n, mesh.node_num))
    rc = L.sfg_mass_sparse_all(mesh.type_name.encode(), mesh.node_num, E, p, mesh.element_node,
                               C.cast(_xy(mesh.x, mesh.y), C.c_void_p), np.ascontiguousarray(rho, np.float64),
                               mi, mj, mx, lumpflag)
    if rc:
        raise SfgError(rc, "sfg_mass_sparse_all")
    return mx[:mesh.node_num].copy() if lumpflag == 1 else (mi, mj, mx[:n].copy())


def stif_sparse_all(mesh, stif_type: int):
    L = lib()
    p, E = mesh.order, mesh.element_num
    n = E * p * p
    si, sj, sx = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n)
    rc = L.sfg_stif_sparse_all(mesh.type_name.encode(), mesh.node_num, E, p, mesh.element_node,
                               C.cast(_xy(mesh.x, mesh.y), C.c_void_p), si, sj, sx, stif_type)
    if rc:
        raise SfgError(rc, "sfg_stif_sparse_all")
    return si, sj, sx


def coo2csr_canonical(n_rows, ci, cj, cx):
    """coo2csr_lib.f90:6-41 on the GPU (ci/cj are copied, not mutated)."""
    L = lib()
    ci = np.array(ci, np.int32)
    cj = np.array(cj, np.int32)
    nnz, ps, z = C.c_int(len(ci)), C.c_int(n_rows + 1), C.c_int()
    Bp = np.zeros(n_rows + 1, np.int32)
    Bj = np.zeros(max(len(ci), 1), np.int32)
    Bx = np.zeros(max(len(ci), 1))
    rc = L.sfg_coo2csr_canonical(C.byref(nnz), C.byref(ps), C.byref(z), ci, cj,
                                 np.ascontiguousarray(cx, np.float64), Bp, Bj, Bx)
    if rc:
        raise SfgError(rc, "sfg_coo2csr_canonical")
    return Bp, Bj[:z.value].copy(), Bx[:z.value].copy()


def abc_mpml(mesh, pml_nx, pml_ny, h, bounds, vp_max, use=(1, 1, 1, 1)):
    L = lib()
    outs = [np.zeros(mesh.node_num) for _ in range(6)]
    rc = L.sfg_abc_mpml(mesh.node_num, mesh.element_num, mesh.order, mesh.element_node,
                        C.cast(_xy(mesh.x, mesh.y), C.c_void_p), pml_nx, pml_ny, h, *bounds, vp_max, *use, *outs)
    if rc:
        raise SfgError(rc, "sfg_abc_mpml")
    return np.stack(outs)


def csr_matvec(Bp, Bj, Bx, x):
    L = lib()
    y = np.zeros(len(Bp) - 1)
    rc = L.sfg_csr_matvec(len(Bp), np.ascontiguousarray(Bp, np.int32), np.ascontiguousarray(Bj, np.int32),
                          np.ascontiguousarray(Bx, np.float64), np.ascontiguousarray(x, np.float64), y)
    if rc:
        raise SfgError(rc, "sfg_csr_matvec")
    return y
