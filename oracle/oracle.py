"""ctypes bindings for the CPU oracle (test infrastructure only).

``Oracle`` wraps ``oracle/_build/libsfo.so`` (the C restatement, always
present after ``make -C oracle``); ``Reference`` wraps ``oracle/_ref/libsfref.so``
(the reference's own sources compiled in place, present only where the
reference tree was available at build time).  Only tests/, bench.py's CPU
baseline leg and ``__graft_entry__.smoke()`` import this module; the product
package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBSFO = os.path.join(HERE, "_build", "libsfo.so")
LIBREF = os.path.join(HERE, "_ref", "libsfref.so")
LIBACOUSTIC = os.path.join(HERE, "_ref", "libsfacoustic.so")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
TYPE_CODES = {"T3": 1, "T6": 2, "T10": 3, "Q4": 4, "Q9": 5, "Q16": 6}
ORDERS = {"T3": 3, "T6": 6, "T10": 10, "Q4": 4, "Q9": 9, "Q16": 16}


def _ptr(a, ct):
    return None if a is None else a.ctypes.data_as(C.POINTER(ct))


class _Problem(C.Structure):
    _fields_ = [
        ("type_code", C.c_int), ("node_num", C.c_int), ("element_num", C.c_int), ("order", C.c_int),
        ("element_node", C.POINTER(C.c_int)),
        ("x", C.POINTER(C.c_double)), ("y", C.POINTER(C.c_double)),
        ("rho", C.POINTER(C.c_double)), ("vp", C.POINTER(C.c_double)),
        ("vs", C.POINTER(C.c_double)), ("c", C.POINTER(C.c_double)),
        ("step", C.c_int), ("dt", C.c_double), ("f0", C.c_double), ("t0", C.c_double),
        ("edge_size", C.c_double),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double), ("ymax", C.c_double),
        ("pml_nx", C.c_int), ("pml_ny", C.c_int),
        ("src_num", C.c_int), ("src_node", C.POINTER(C.c_int)),
        ("rec_num", C.c_int), ("rec_node", C.POINTER(C.c_int)),
        ("free_surface", C.c_int), ("snap_every", C.c_int), ("nthreads", C.c_int),
        ("timing", C.POINTER(C.c_double)), ("consistent", C.c_int),
    ]


class _AcousticProblem(C.Structure):
    _fields_ = [
        ("type_code", C.c_int), ("node_num", C.c_int), ("element_num", C.c_int), ("order", C.c_int),
        ("element_node", C.POINTER(C.c_int)),
        ("x", C.POINTER(C.c_double)), ("y", C.POINTER(C.c_double)), ("vp", C.POINTER(C.c_double)),
        ("step", C.c_int), ("dt", C.c_double), ("f0", C.c_double), ("t0", C.c_double),
        ("source_node", C.c_int), ("pml", C.c_int),
        ("edge_size", C.c_double), ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double),
        ("ymax", C.c_double), ("pml_nx", C.c_int), ("pml_ny", C.c_int), ("nthreads", C.c_int),
    ]


def acoustic_snapshot_rows(step: int, pml: bool) -> int:
    """Rows of u the reference's acoustic solvers print: the zero row, then
    every 10 steps (acoustic.c:197) or 20 (acoustic_pml.c:448)."""
    return snapshot_rows(step, 20 if pml else 10)


def snapshot_rows(step: int, snap_every: int = 200) -> int:
    return 1 + sum(1 for it in range(2, step) if (it + 1) % snap_every == 0)


class Oracle:
    """The C restatement (FP64)."""

    def __init__(self, path: str = LIBSFO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = self.lib = C.CDLL(path)
        L.sfo_mass_coo.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _f64p, _f64p, _f64p, _i32p, _i32p, _f64p]
        L.sfo_mass_lumped.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _f64p, _f64p, _f64p, _f64p]
        L.sfo_stif_coo.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _f64p, _f64p, _i32p, _i32p, _f64p]
        L.sfo_coo2csr_canonical.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p]
        L.sfo_iargsort.argtypes = [_i32p, C.c_int, _i32p]
        L.sfo_abc_mpml.argtypes = ([C.c_int, C.c_int, C.c_int, _i32p, _f64p, _f64p, C.c_int, C.c_int] +
                                   [C.c_double] * 6 + [C.c_int] * 4 + [_f64p] * 6)
        L.sfo_ricker.restype = C.c_double
        L.sfo_ricker.argtypes = [C.c_double] * 4
        L.sfo_node_location.argtypes = [C.c_int, C.c_double, _f64p, _f64p, C.c_double, C.c_double]
        L.sfo_elastic_run.argtypes = [C.POINTER(_Problem)] + [C.c_void_p] * 6
        L.sfo_csr_matvec.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
        L.sfo_acoustic_run.argtypes = [C.POINTER(_AcousticProblem), C.c_void_p, C.c_void_p]
        L.sfo_abc_pml.argtypes = ([C.c_int, C.c_int, C.c_int, _i32p, _f64p, _f64p, C.c_int, C.c_int] +
                                  [C.c_double] * 6 + [C.c_int] * 4 + [_f64p] * 4)

    # assembly -----------------------------------------------------------
    def mass_coo(self, mesh, rho):
        p, E = mesh.order, mesh.element_num
        n = E * p * p
        mi, mj, mx = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n)
        rc = self.lib.sfo_mass_coo(mesh.type_code, mesh.node_num, E, mesh.element_node, mesh.x, mesh.y,
                                   np.ascontiguousarray(rho, np.float64), mi, mj, mx)
        assert rc == 0, rc
        return mi, mj, mx

    def mass_lumped(self, mesh, rho):
        m = np.zeros(mesh.node_num)
        rc = self.lib.sfo_mass_lumped(mesh.type_code, mesh.node_num, mesh.element_num, mesh.element_node,
                                      mesh.x, mesh.y, np.ascontiguousarray(rho, np.float64), m)
        assert rc == 0, rc
        return m

    def stif_coo(self, mesh, stif_type):
        p, E = mesh.order, mesh.element_num
        n = E * p * p
        si, sj, sx = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n)
        rc = self.lib.sfo_stif_coo(mesh.type_code, stif_type, mesh.node_num, E, mesh.element_node,
                                   mesh.x, mesh.y, si, sj, sx)
        assert rc == 0, rc
        return si, sj, sx

    def coo2csr(self, n_rows, ci, cj, cx):
        nnz = len(ci)
        Bp = np.zeros(n_rows + 1, np.int32)
        Bj = np.zeros(max(nnz, 1), np.int32)
        Bx = np.zeros(max(nnz, 1))
        z = self.lib.sfo_coo2csr_canonical(nnz, n_rows + 1, np.ascontiguousarray(ci, np.int32),
                                           np.ascontiguousarray(cj, np.int32),
                                           np.ascontiguousarray(cx, np.float64), Bp, Bj, Bx)
        return Bp, Bj[:z].copy(), Bx[:z].copy()

    def iargsort(self, vec):
        vec = np.ascontiguousarray(vec, np.int32)
        m = np.zeros(max(len(vec), 1), np.int32)
        self.lib.sfo_iargsort(vec, len(vec), m)
        return m[:len(vec)]

    def abc_mpml(self, mesh, pml_nx, pml_ny, h, bounds, vp_max, use=(1, 1, 1, 1)):
        N = mesh.node_num
        outs = [np.zeros(N) for _ in range(6)]
        self.lib.sfo_abc_mpml(N, mesh.element_num, mesh.order, mesh.element_node, mesh.x, mesh.y,
                              pml_nx, pml_ny, h, *bounds, vp_max, *use, *outs)
        return np.stack(outs)

    def ricker(self, f0, t0, mag, t):
        return self.lib.sfo_ricker(f0, t0, mag, t)

    def node_location(self, mesh, edge_size, px, py):
        return self.lib.sfo_node_location(mesh.node_num, edge_size, mesh.x, mesh.y, px, py)

    def csr_matvec(self, Bp, Bj, Bx, x):
        y = np.zeros(len(Bp) - 1)
        self.lib.sfo_csr_matvec(len(Bp), Bp, Bj, Bx, np.ascontiguousarray(x, np.float64), y)
        return y

    # time loop ------------------------------------------------------------
    def run(self, prob, snap_every: int = 200, nthreads: int = 0, energy: bool = False,
            solver: str = "masslump"):
        """FP64 elastic_wave() run; returns dict of seismograms/snapshots.
        solver "masslump", or "mgmres" / "pardiso": the consistent-mass branch
        (the systems solved with M by Jacobi-preconditioned CG)."""
        m = prob.mesh
        S, R, N, step = len(prob.src_node), len(prob.rec_node), m.node_num, prob.step
        ns = snapshot_rows(step, snap_every)
        out = {
            "seis_u": np.zeros((S, step - 2, R)), "seis_w": np.zeros((S, step - 2, R)),
            "snap_u": np.zeros((S, ns, N)), "snap_w": np.zeros((S, ns, N)),
        }
        if energy:
            out["energy_u"] = np.zeros((S, step))
            out["energy_w"] = np.zeros((S, step))
        keep = [prob.model.c, prob.src_node, prob.rec_node]
        timing = np.zeros(2)
        pb = _Problem(
            m.type_code, N, m.element_num, m.order, _ptr(m.element_node, C.c_int),
            _ptr(m.x, C.c_double), _ptr(m.y, C.c_double),
            _ptr(prob.model.rho, C.c_double), _ptr(prob.model.vp, C.c_double),
            _ptr(prob.model.vs, C.c_double), _ptr(prob.model.c, C.c_double),
            step, prob.dt, prob.f0, prob.t0, prob.edge_size,
            m.xmin, m.xmax, m.ymin, m.ymax, prob.pml_nx, prob.pml_ny,
            S, _ptr(prob.src_node, C.c_int), R, _ptr(prob.rec_node, C.c_int),
            prob.free_surface, snap_every, nthreads, _ptr(timing, C.c_double), int(solver != "masslump"))
        ptrs = [out[k].ctypes.data for k in ("seis_u", "seis_w", "snap_u", "snap_w")]
        ptrs += [out["energy_u"].ctypes.data, out["energy_w"].ctypes.data] if energy else [None, None]
        rc = self.lib.sfo_elastic_run(C.byref(pb), *ptrs)
        del keep
        out["status"] = rc
        out["setup_seconds"], out["loop_seconds"] = float(timing[0]), float(timing[1])
        return out


    def abc_pml(self, mesh, pml_nx, pml_ny, h, bounds, vp_max, use=(1, 1, 1, 1)):
        out = np.zeros((4, mesh.node_num))
        self.lib.sfo_abc_pml(mesh.node_num, mesh.element_num, mesh.order, mesh.element_node, mesh.x, mesh.y,
                             pml_nx, pml_ny, h, *bounds, vp_max, *use, out[0], out[1], out[2], out[3])
        return out

    def acoustic_run(self, mesh, vp, step, dt, f0, t0, source_node, pml=False, edge_size=0.0,
                     pml_nx=0, pml_ny=0, nthreads: int = 0):
        """The acoustic solvers (acoustic.c / acoustic_pml.c) restated:
        {"snap": [rows][N], "energy": [step], "status"}."""
        N = mesh.node_num
        vp = np.ascontiguousarray(vp, np.float64)
        rows = acoustic_snapshot_rows(step, pml)
        snap, energy = np.zeros((rows, N)), np.zeros(step)
        pb = _AcousticProblem(TYPE_CODES[mesh.type_name], N, mesh.element_num, mesh.order,
                              _ptr(mesh.element_node, C.c_int), _ptr(mesh.x, C.c_double),
                              _ptr(mesh.y, C.c_double), _ptr(vp, C.c_double), step, dt, f0, t0,
                              source_node, int(bool(pml)), edge_size, mesh.xmin, mesh.xmax, mesh.ymin,
                              mesh.ymax, pml_nx, pml_ny, nthreads)
        rc = self.lib.sfo_acoustic_run(C.byref(pb), snap.ctypes.data, energy.ctypes.data)
        return {"snap": snap, "energy": energy, "status": rc}


class ReferenceAcoustic:
    """The reference's acoustic solvers compiled in place (oracle/_ref)."""

    def __init__(self, path: str = LIBACOUSTIC):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing (reference not built here)")
        L = self.lib = C.CDLL(path)
        tail = [_f64p, _f64p, C.c_long, _f64p, C.c_long, C.POINTER(C.c_long), C.POINTER(C.c_long),
                C.POINTER(C.c_double)]
        head = [C.c_char_p, C.c_int, C.c_char_p, C.c_int, C.c_int, C.c_int, _i32p, _f64p, _f64p, C.c_int,
                C.c_double, C.c_double, C.c_double]
        L.sfa_acoustic.argtypes = head + [C.c_int, C.c_char_p] + tail
        L.sfa_acoustic_pml.argtypes = head + [C.c_double] * 5 + [C.c_int] * 3 + [C.c_char_p] + tail
        L.sfa_set_step_times.argtypes = [C.c_void_p, C.c_long]

    def run(self, mesh, vp, step, dt, f0, t0, source_node, pml=False, edge_size=0.0, pml_nx=0, pml_ny=0,
            nthreads: int = 0, solver: str = "masslump", workdir: str | None = None):
        """{"snap": [rows][N] (rows printed so far), "energy": [step],
        "energy_values", "status", "seconds"}; status 0, 1 (exit on the energy
        bound), 3 (unknown solver)."""
        N = mesh.node_num
        rows = acoustic_snapshot_rows(step, pml)
        snap, energy = np.zeros(rows * N), np.zeros(step)
        ns, ne, secs = C.c_long(), C.c_long(), C.c_double()
        tmp = workdir or tempfile.mkdtemp(prefix="sfacoustic_")
        vp = np.ascontiguousarray(vp, np.float64)
        common = (tmp.encode(), nthreads, mesh.type_name.encode(), N, mesh.element_num, mesh.order,
                  mesh.element_node, mesh.x, mesh.y, step, dt, f0, t0)
        outs = (vp, snap, snap.size, energy, energy.size, C.byref(ns), C.byref(ne), C.byref(secs))
        stamps = np.zeros(step)
        self.lib.sfa_set_step_times(stamps.ctypes.data, step)
        try:
            if pml:
                rc = self.lib.sfa_acoustic_pml(*common, edge_size, mesh.xmin, mesh.xmax, mesh.ymin, mesh.ymax,
                                               pml_nx, pml_ny, source_node, solver.encode(), *outs)
            else:
                rc = self.lib.sfa_acoustic(*common, source_node, solver.encode(), *outs)
        finally:
            self.lib.sfa_set_step_times(None, 0)
        # seconds of each completed time step (from its energy.dat write)
        step_seconds = np.diff(stamps[1:ne.value]) if ne.value > 2 else np.zeros(0)
        if workdir is None:
            shutil.rmtree(tmp, ignore_errors=True)
        return {"snap": snap.reshape(rows, N)[:ns.value // N], "energy": energy[:ne.value],
                "energy_values": ne.value, "status": rc, "seconds": secs.value, "step_seconds": step_seconds,
                "workdir": workdir}


class Reference:
    """The reference's own C sources, compiled in place (oracle/_ref)."""

    def __init__(self, path: str = LIBREF):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing (reference not built here)")
        L = self.lib = C.CDLL(path)
        L.sfr_mass_sparse_all.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, _i32p, _f64p, _f64p, _f64p,
                                          _i32p, _i32p, _f64p, C.c_int]
        L.sfr_stif_sparse_all.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, _i32p, _f64p, _f64p,
                                          _i32p, _i32p, _f64p, C.c_int]
        L.sfr_abc_mpml.argtypes = ([C.c_int, C.c_int, C.c_int, _i32p, _f64p, _f64p, C.c_int, C.c_int] +
                                   [C.c_double] * 6 + [C.c_int] * 4 + [_f64p])
        L.sfr_seismic_source.restype = C.c_double
        L.sfr_seismic_source.argtypes = [C.c_double] * 4
        L.sfr_node_location.argtypes = [C.c_int, C.c_double, _f64p, _f64p, C.c_double, C.c_double]
        L.sfr_mesh.argtypes = [C.c_char_p, C.c_int, C.c_int] + [C.c_double] * 4 + [_i32p, _f64p, _f64p]
        L.sfr_mesh_sizes.argtypes = [C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        # getattr: a double-underscore name would be mangled inside the class body
        self._coo2csr = getattr(L, "__coo2csr_lib_MOD_coo2csr_canonical")
        self._coo2csr.argtypes = [C.POINTER(C.c_int)] * 3 + [_i32p, _i32p, _f64p, _i32p, _i32p, _f64p]
        L.sfr_elastic_wave.argtypes = ([C.c_char_p, C.c_int, C.c_char_p, C.c_int, C.c_int, C.c_int, _i32p,
                                        _f64p, _f64p, C.c_int] + [C.c_double] * 8 + [C.c_int, C.c_int,
                                        C.c_int, _i32p, C.c_int, _i32p, C.c_char_p, C.c_int, C.c_int] +
                                       [C.c_void_p] * 4 + [C.c_int, C.POINTER(C.c_double), C.c_void_p, C.c_int])
        L.sfr_now.restype = C.c_double

    def mesh(self, type_name, nx, ny, xmin, xmax, ymin, ymax):
        N, E = C.c_int(), C.c_int()
        p = self.lib.sfr_mesh_sizes(type_name.encode(), nx, ny, C.byref(N), C.byref(E))
        en = np.zeros(E.value * p, np.int32)
        x, y = np.zeros(N.value), np.zeros(N.value)
        self.lib.sfr_mesh(type_name.encode(), nx, ny, xmin, xmax, ymin, ymax, en, x, y)
        return en, x, y

    def mass(self, mesh, rho, lump):
        p, E = mesh.order, mesh.element_num
        n = E * p * p
        mi, mj, mx = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(max(n, mesh.node_num))
        self.lib.sfr_mass_sparse_all(mesh.type_name.encode(), mesh.node_num, E, p, mesh.element_node,
                                     mesh.x, mesh.y, np.ascontiguousarray(rho, np.float64), mi, mj, mx, lump)
        return (mx[:mesh.node_num].copy() if lump else (mi, mj, mx[:n].copy()))

    def stif(self, mesh, stif_type):
        p, E = mesh.order, mesh.element_num
        n = E * p * p
        si, sj, sx = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n)
        self.lib.sfr_stif_sparse_all(mesh.type_name.encode(), mesh.node_num, E, p, mesh.element_node,
                                     mesh.x, mesh.y, si, sj, sx, stif_type)
        return si, sj, sx

    def coo2csr(self, n_rows, ci, cj, cx):
        nnz = C.c_int(len(ci))
        ps = C.c_int(n_rows + 1)
        z = C.c_int()
        Bp = np.zeros(n_rows + 1, np.int32)
        Bj = np.zeros(len(ci), np.int32)
        Bx = np.zeros(len(ci))
        ci, cj = np.array(ci, np.int32), np.array(cj, np.int32)
        self._coo2csr(C.byref(nnz), C.byref(ps), C.byref(z), ci, cj,
                                                     np.ascontiguousarray(cx, np.float64), Bp, Bj, Bx)
        return Bp, Bj[:z.value].copy(), Bx[:z.value].copy()

    def abc_mpml(self, mesh, pml_nx, pml_ny, h, bounds, vp_max, use=(1, 1, 1, 1)):
        out = np.zeros(6 * mesh.node_num)
        self.lib.sfr_abc_mpml(mesh.node_num, mesh.element_num, mesh.order, mesh.element_node, mesh.x, mesh.y,
                              pml_nx, pml_ny, h, *bounds, vp_max, *use, out)
        return out.reshape(6, mesh.node_num)

    def run(self, prob, nthreads: int = 0, workdir: str | None = None, want_snapshots: bool = True,
            solver: str = "masslump"):
        """Run the reference elastic_wave() (solver "masslump", or "mgmres":
        its consistent-mass branch with the reference's own GMRES,
        solver/mgmres/mgmres.c) through its exterior-model path: the model is
        written to mesh/velocity_and_density.txt with %.17g so it reads back
        exactly."""
        m = prob.mesh
        S, R, N, step = len(prob.src_node), len(prob.rec_node), m.node_num, prob.step
        ns = snapshot_rows(step, 200)
        out = {"seis_u": np.zeros((S, step - 2, R)), "seis_w": np.zeros((S, step - 2, R))}
        if want_snapshots:
            out["snap_u"] = np.zeros((S, ns, N))
            out["snap_w"] = np.zeros((S, ns, N))
        step_t = np.zeros(step)
        tmp = workdir or tempfile.mkdtemp(prefix="sfref_")
        os.makedirs(os.path.join(tmp, "mesh"), exist_ok=True)
        os.makedirs(os.path.join(tmp, "outputfile"), exist_ok=True)
        md = prob.model
        with open(os.path.join(tmp, "mesh", "velocity_and_density.txt"), "w") as f:
            cols = np.stack([md.rho, md.vp, md.vs, md.c[0], md.c[1], md.c[2], md.c[3]], axis=1)
            f.write("".join(" ".join("%.17g" % v for v in row) + "\n" for row in cols))
        secs = C.c_double()
        t_call = self.lib.sfr_now()
        rc = self.lib.sfr_elastic_wave(
            tmp.encode(), nthreads, m.type_name.encode(), N, m.element_num, m.order, m.element_node,
            m.x, m.y, step, prob.dt, prob.f0, prob.t0, prob.edge_size, m.xmin, m.xmax, m.ymin, m.ymax,
            prob.pml_nx, prob.pml_ny, S, np.ascontiguousarray(prob.src_node, np.int32), R,
            np.ascontiguousarray(prob.rec_node, np.int32), solver.encode(), 1, prob.free_surface,
            out["seis_u"].ctypes.data, out["seis_w"].ctypes.data,
            out["snap_u"].ctypes.data if want_snapshots else None,
            out["snap_w"].ctypes.data if want_snapshots else None, ns, C.byref(secs), step_t.ctypes.data, step)
        out["status"] = rc
        nst = int(np.count_nonzero(step_t))
        out["step_end_times"] = step_t[:nst] - t_call     # seconds since the call began
        out["seconds"] = secs.value
        if workdir is None:
            # the text files were read back through the harness; a temporary
            # directory made here goes (a caller's own directory stays)
            shutil.rmtree(tmp, ignore_errors=True)
        out["workdir"] = workdir
        return out
