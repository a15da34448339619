"""Meshes, models and run descriptions for the SeisFEM elastic M-PML path.

Host-side data structures keep the reference's conventions so the same
arrays can be handed to the reference's ``elastic_wave()`` or to this
library's C-ABI unchanged:

* ``element_node``: int32, 1-based, element-major ``[element_num * order]``
  (seisfem/seisfem.c:169-182);
* ``x``, ``y``: float64 node coordinates (the reference's ``node_xy[0]`` and
  ``node_xy[1]``, seisfem.c:170-189);
* model: per-node ``rho, vp, vs`` and ``c[4] = (c11, c13, c33, c44)``
  (time_evolution/elastic_wave.c:186-220).

Axes follow the reference's free-surface convention: ``x`` is the vertical
axis (increasing upward, free surface at ``x = xmax``) and ``y`` the
horizontal one (EXAMPLE/example6_surface_wave/README:3-5).  The hard-coded
force direction (``Angle_force = 90``, elastic_wave.c:66) therefore drives
the vertical component ``u``; ``w`` is horizontal.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

TYPE_CODES = {"T3": 1, "T6": 2, "T10": 3, "Q4": 4, "Q9": 5, "Q16": 6}
ORDERS = {"T3": 3, "T6": 6, "T10": 10, "Q4": 4, "Q9": 9, "Q16": 16}


@dataclasses.dataclass
class Mesh:
    type_name: str
    element_node: np.ndarray      # int32, 1-based, [element_num * order]
    x: np.ndarray                 # float64 [node_num]
    y: np.ndarray                 # float64 [node_num]
    xmin: float = 0.0
    xmax: float = 0.0
    ymin: float = 0.0
    ymax: float = 0.0

    @property
    def type_code(self) -> int:
        return TYPE_CODES[self.type_name]

    @property
    def order(self) -> int:
        return ORDERS[self.type_name]

    @property
    def node_num(self) -> int:
        return int(self.x.shape[0])

    @property
    def element_num(self) -> int:
        return int(self.element_node.shape[0] // self.order)


@dataclasses.dataclass
class Model:
    rho: np.ndarray
    vp: np.ndarray
    vs: np.ndarray
    c: np.ndarray                 # [4, node_num]: c11, c13, c33, c44


@dataclasses.dataclass
class Problem:
    mesh: Mesh
    model: Model
    step: int
    dt: float
    f0: float
    t0: float
    edge_size: float
    pml_nx: int
    pml_ny: int
    src_node: np.ndarray          # int32 [src_num]
    rec_node: np.ndarray          # int32 [rec_num]
    free_surface: int = 0
    name: str = ""

    @property
    def dof(self) -> int:
        return 2 * self.mesh.node_num


# --------------------------------------------------------------- meshes

def structured_mesh(type_name: str, nelemx: int, nelemy: int, xmin: float, xmax: float,
                    ymin: float, ymax: float) -> Mesh:
    """Structured mesh with the reference's node numbering and coordinates.

    Q4/T3 nodes: mesh/mesh_xy_q4.c:40-47 (``((n-i)*min + i*max)/(1.0*n)``);
    Q9/T6 nodes: mesh/mesh_xy_q9.c:44-51 (``i*(max-min)/(2.0*n)``, no offset);
    Q16/T10 nodes: mesh/mesh_xy_q16.c (``i*(max-min)/(3.0*n)``, no offset);
    connectivity: mesh/mesh_element_{q4,t3,q9,t6,q16,t10}.c.
    """
    nx, ny = nelemx, nelemy
    if type_name in ("Q4", "T3"):
        i = np.arange(nx + 1)
        j = np.arange(ny + 1)
        xs = ((nx - i) * xmin + i * xmax) / (1.0 * nx)
        ys = ((ny - j) * ymin + j * ymax) / (1.0 * ny)
        X = np.tile(xs, ny + 1)
        Y = np.repeat(ys, nx + 1)
        jj, ii = np.meshgrid(np.arange(1, ny + 1), np.arange(1, nx + 1), indexing="ij")
        sw = (ii + (jj - 1) * (nx + 1)).ravel()
        se = sw + 1
        nw = (ii + jj * (nx + 1)).ravel()
        ne = nw + 1
        if type_name == "Q4":
            en = np.stack([sw, se, ne, nw], axis=1)
        else:
            en = np.stack([np.stack([sw, se, nw], 1), np.stack([ne, nw, se], 1)], axis=1).reshape(-1, 3)
    elif type_name in ("Q9", "T6"):
        i = np.arange(2 * nx + 1)
        j = np.arange(2 * ny + 1)
        xs = i * (xmax - xmin) / (2.0 * nx)
        ys = j * (ymax - ymin) / (2.0 * ny)
        X = np.tile(xs, 2 * ny + 1)
        Y = np.repeat(ys, 2 * nx + 1)
        jj, ii = np.meshgrid(np.arange(1, ny + 1), np.arange(1, nx + 1), indexing="ij")
        sw = (2 * (jj - 1) * (2 * nx + 1) + 2 * (ii - 1) + 1).ravel()
        w = sw + 2 * nx + 1
        nw = sw + 2 * (2 * nx + 1)
        s = sw + 1
        c = sw + 1 + 2 * nx + 1
        n = sw + 1 + 2 * (2 * nx + 1)
        se = sw + 2
        e = sw + 2 + 2 * nx + 1
        ne = sw + 2 + 2 * (2 * nx + 1)
        if type_name == "Q9":
            en = np.stack([sw, se, ne, nw, s, e, n, w, c], axis=1)
        else:
            en = np.stack([np.stack([sw, se, nw, s, c, w], 1), np.stack([ne, nw, se, n, c, e], 1)],
                          axis=1).reshape(-1, 6)
    elif type_name in ("Q16", "T10"):
        # cubic elements on the (3nx+1) x (3ny+1) node grid:
        # mesh/mesh_xy_{q16,t10}.c (``i*(max-min)/(3.0*n)``, no offset),
        # mesh/mesh_element_{q16,t10}.c (element base node, then rows of 4)
        row = 3 * nx + 1
        i = np.arange(row)
        j = np.arange(3 * ny + 1)
        xs = i * (xmax - xmin) / (3.0 * nx)
        ys = j * (ymax - ymin) / (3.0 * ny)
        X = np.tile(xs, 3 * ny + 1)
        Y = np.repeat(ys, row)
        jj, ii = np.meshgrid(np.arange(1, ny + 1), np.arange(1, nx + 1), indexing="ij")
        b = ((jj - 1) * 3 * row + 3 * ii - 2).ravel()
        g = lambda r, c: b + r * row + c          # node in grid row r, column c of the element
        if type_name == "Q16":
            en = np.stack([g(r, c) for r in range(4) for c in range(4)], axis=1)
        else:
            lower = [g(0, 0), g(0, 1), g(0, 2), g(0, 3), g(1, 2), g(2, 1), g(3, 0), g(2, 0), g(1, 0), g(1, 1)]
            upper = [g(3, 3), g(3, 2), g(3, 1), g(3, 0), g(2, 1), g(1, 2), g(0, 3), g(1, 3), g(2, 3), g(2, 2)]
            en = np.stack([np.stack(lower, 1), np.stack(upper, 1)], axis=1).reshape(-1, 10)
    else:
        raise NotImplementedError(f"structured {type_name} meshes are not generated here")
    return Mesh(type_name, np.ascontiguousarray(en.ravel(), np.int32),
                np.ascontiguousarray(X, np.float64), np.ascontiguousarray(Y, np.float64),
                float(xmin), float(xmax), float(ymin), float(ymax))


def mesh_bounds_from_nodes(mesh: Mesh) -> Mesh:
    """Exterior-mesh bounds: running min/max starting from 0 (seisfem.c:192-214)."""
    mesh.xmin = min(0.0, float(mesh.x.min()))
    mesh.ymin = min(0.0, float(mesh.y.min()))
    mesh.xmax = max(0.0, float(mesh.x.max()))
    mesh.ymax = max(0.0, float(mesh.y.max()))
    return mesh


# --------------------------------------------------------------- models

def isotropic_model(vp, vs, rho) -> Model:
    """c11 = c33 = rho vp^2, c44 = rho vs^2, c13 = c11 - 2 c44
    (model_elastic_parameter/model_elastic_parameter.c:34-45)."""
    vp, vs, rho = (np.ascontiguousarray(a, np.float64) for a in (vp, vs, rho))
    mu = vs * vs * rho
    lam = vp * vp * rho - 2 * mu
    c = np.stack([lam + 2 * mu, lam, lam + 2 * mu, mu])
    return Model(rho.copy(), vp.copy(), vs.copy(), np.ascontiguousarray(c))


def vti_model(n, vp0, vs0, rho0, eps, delta) -> Model:
    """VTI constants from Thomsen parameters; the symmetry axis is the
    vertical x axis, so c[0] (xx) holds c33 and c[2] (yy) holds c11."""
    c33 = rho0 * vp0 ** 2
    c44 = rho0 * vs0 ** 2
    c11 = c33 * (1 + 2 * eps)
    c13 = math.sqrt(2 * delta * c33 * (c33 - c44) + (c33 - c44) ** 2) - c44
    one = np.ones(n)
    c = np.stack([c33 * one, c13 * one, c11 * one, c44 * one])
    return Model(rho0 * one, vp0 * one, vs0 * one, np.ascontiguousarray(c))


def gaussian_random_field(shape, spacing, corr_len, mean, std, lo, hi, seed) -> np.ndarray:
    """FFT-filtered white noise with a Gaussian covariance of correlation
    length corr_len, rescaled to (mean, std) and clipped to [lo, hi]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    noise = rng.standard_normal(shape)
    kx = np.fft.fftfreq(shape[0], d=spacing) * 2 * np.pi
    ky = np.fft.fftfreq(shape[1], d=spacing) * 2 * np.pi
    k2 = kx[:, None] ** 2 + ky[None, :] ** 2
    filt = np.exp(-k2 * corr_len ** 2 / 8.0)       # sqrt of the Gaussian spectrum
    field = np.real(np.fft.ifft2(np.fft.fft2(noise) * filt))
    field = (field - field.mean()) / (field.std() + 1e-30)
    return np.clip(mean + std * field, lo, hi)


def gardner_rho(vp):
    return 310.0 * np.asarray(vp) ** 0.25


# ------------------------------------------------------ sources, receivers

def node_location(mesh: Mesh, edge_size: float, px: float, py: float) -> int:
    """Last node within edge_size/2 in both axes, -1 on a miss
    (source_receiver/node_location.c:13-27)."""
    hit = np.nonzero((np.abs(mesh.x - px) <= edge_size / 2.0) & (np.abs(mesh.y - py) <= edge_size / 2.0))[0]
    return int(hit[-1]) if hit.size else -1


def line_points(n, first, last):
    """Evenly spaced points (source_receiver/set_rec_and_src.c:5-31)."""
    if n == 1:
        return [first]
    return [(first[0] + i * (last[0] - first[0]) / (1.0 * (n - 1)),
             first[1] + i * (last[1] - first[1]) / (1.0 * (n - 1))) for i in range(n)]


_SCAN_LOCATOR = False


def use_scan_locator(on: bool = True) -> None:
    """Make ``locate`` use the numpy scan (``node_location``) instead of the
    library's grid locator.  A process that times the reference's own code
    builds its problems this way, so it never loads libseisfem_b200.so; both
    locators return the same nodes (the last-match rule)."""
    global _SCAN_LOCATOR
    _SCAN_LOCATOR = bool(on)


def locate(mesh, edge_size, pts):
    """Node indices of points (sfg_node_location: the reference's rule with a
    grid instead of a scan per point)."""
    pts = np.asarray(pts, np.float64).reshape(-1, 2)
    if _SCAN_LOCATOR:
        out = np.array([node_location(mesh, edge_size, px, py) for px, py in pts], np.int32)
    else:
        from .api import node_location as locate_all
        out = locate_all(mesh.x, mesh.y, edge_size, pts[:, 0], pts[:, 1])
    if (out < 0).any():
        raise ValueError("a source or receiver lies outside the mesh")
    return out


# ------------------------------------------------------------ the configs

def config_1(n: int = 200, h: float = 10.0, step: int = 1000) -> Problem:
    """Q4 200x200, dx=10 m, homogeneous vp=3000 vs=1732 rho=2000, M-PML 20,
    Ricker 25 Hz at the centre, dt=1 ms, 181 receivers on the top interior row."""
    L = n * h
    mesh = structured_mesh("Q4", n, n, 0.0, L, 0.0, L)
    N = mesh.node_num
    model = isotropic_model(np.full(N, 3000.0), np.full(N, 1732.0), np.full(N, 2000.0))
    pml = 20
    src = locate(mesh, h, [(L / 2, L / 2)])
    xr = L - pml * h
    rec = locate(mesh, h, line_points(181, (xr, pml * h / 2), (xr, L - pml * h / 2)))
    return Problem(mesh, model, step, 1e-3, 25.0, 0.0, h, pml, pml, src, rec, 0, "config1_q4_200")


def layered_model(mesh: Mesh, nlayer: int, L: float, seed: int) -> Model:
    rng = np.random.Generator(np.random.PCG64(seed))
    cuts = np.sort(rng.uniform(0.0, L, nlayer - 1))
    vps = rng.uniform(1500.0, 4500.0, nlayer)
    layer = np.searchsorted(cuts, mesh.x, side="right")
    vp = vps[layer]
    return isotropic_model(vp, vp / math.sqrt(3.0), gardner_rho(vp))


def config_2(n: int = 400, h: float = 10.0, step: int = 3000, pml: int = 30) -> Problem:
    """Q9 400x400 over 4000 m (node spacing 5 m), 6 seeded horizontal layers,
    Ricker 15 Hz at the centre, dt=0.5 ms, M-PML 30."""
    L = n * h
    mesh = structured_mesh("Q9", n, n, 0.0, L, 0.0, L)
    model = layered_model(mesh, 6, L, seed=2)
    src = locate(mesh, h, [(L / 2, L / 2)])
    xr = L - pml * h
    nrec = int(round((L - 2 * pml * h) / h)) + 1
    rec = locate(mesh, h, line_points(nrec, (xr, pml * h), (xr, L - pml * h)))
    return Problem(mesh, model, step, 5e-4, 15.0, 0.0, h, pml, pml, src, rec, 0, f"config2_q9_{n}")


def grf_model(mesh: Mesh, n: int, h: float, corr_len: float, seed: int) -> Model:
    """GRF vp on the Q4 node grid, vs = vp/sqrt(3), Gardner density."""
    vp_grid = gaussian_random_field((n + 1, n + 1), h, corr_len, 3000.0, 400.0, 1800.0, 4500.0, seed)
    vp = vp_grid.ravel()                       # node k = i + j*(n+1): row j, column i
    return isotropic_model(vp, vp / math.sqrt(3.0), gardner_rho(vp))


def config_3a(n: int = 400, h: float = 10.0, step: int = 2000, shots: int = 64, pml: int = 20) -> Problem:
    """Q4 400x400 GRF model, 64 Ricker sources at 20 Hz along the surface
    (one element below the top M-PML), dt = 1 ms."""
    L = n * h
    mesh = structured_mesh("Q4", n, n, 0.0, L, 0.0, L)
    model = grf_model(mesh, n, h, 200.0, seed=3)
    xs = L - (pml + 1) * h
    src = locate(mesh, h, line_points(shots, (xs, (pml + 1) * h), (xs, L - (pml + 1) * h)))
    xr = L - pml * h
    nrec = int(round((L - 2 * pml * h) / h)) + 1
    rec = locate(mesh, h, line_points(nrec, (xr, pml * h), (xr, L - pml * h)))
    return Problem(mesh, model, step, 1e-3, 20.0, 0.0, h, pml, pml, src, rec, 0, f"config3a_q4_{n}_s{shots}")


def small_problem(type_name: str = "Q4", n: int = 40, h: float = 10.0, step: int = 300, pml: int = 8,
                  f0: float = 25.0, dt: float = 1e-3, shots: int = 1, free_surface: int = 0,
                  seed: int | None = None) -> Problem:
    """A small case for parity tests (homogeneous or, with seed, GRF-like)."""
    L = n * h
    mesh = structured_mesh(type_name, n, n, 0.0, L, 0.0, L)
    N = mesh.node_num
    if seed is None:
        model = isotropic_model(np.full(N, 3000.0), np.full(N, 1732.0), np.full(N, 2000.0))
    else:
        rng = np.random.Generator(np.random.PCG64(seed))
        vp = 3000.0 + 300.0 * np.sin(mesh.x / 97.0 + rng.uniform()) * np.cos(mesh.y / 71.0)
        model = isotropic_model(vp, vp / math.sqrt(3.0), gardner_rho(vp))
    if shots == 1:
        src = locate(mesh, h, [(L / 2, L / 2)])
    else:
        xs = L - (pml + 1) * h
        src = locate(mesh, h, line_points(shots, (xs, (pml + 1) * h), (xs, L - (pml + 1) * h)))
    xr = L - pml * h
    nrec = int(round((L - 2 * pml * h) / h)) + 1
    rec = locate(mesh, h, line_points(nrec, (xr, pml * h), (xr, L - pml * h)))
    return Problem(mesh, model, step, dt, f0, 0.0, h, pml, pml, src, rec, free_surface,
                   f"small_{type_name}_{n}")


def config_5(seed: int, n: int = 128, h: float = 10.0, samples: int = 1000, nrec: int = 64, pml: int = 16,
             f0: float = 15.0, corr_len: float = 150.0) -> Problem:
    """One surrogate training shot: Q4 n x n (1280 m for n = 128), GRF vp
    (mean 3000, std 400, correlation length 150 m, clipped 1800-4500, seeded),
    vs = vp/sqrt(3), Gardner density; free surface at x = xmax with the M-PML
    (16 elements) on the other three sides; the source one element below the
    surface at a horizontal position drawn uniformly over the receiver span;
    nrec receivers evenly along the surface row; dt = 1 ms, samples + 2 steps
    (the loop records step - 2 samples)."""
    L = n * h
    mesh = structured_mesh("Q4", n, n, 0.0, L, 0.0, L)
    model = grf_model(mesh, n, h, corr_len, seed)
    rng = np.random.Generator(np.random.PCG64(seed + 1_000_003))
    y0, y1 = pml * h, L - pml * h
    ys = round(rng.uniform(y0, y1) / h) * h
    src = locate(mesh, h, [(L - h, ys)])
    rec = locate(mesh, h, line_points(nrec, (L, y0), (L, y1)))
    return Problem(mesh, model, samples + 2, 1e-3, f0, 0.0, h, pml, pml, src, rec, 1, f"config5_q4_{n}_seed{seed}")


def config_4(nx: int = 150, ny: int = 300, h: float = 10.0, step: int = 4000, dt: float = 4e-4, pml: int = 20,
             amp: float = 40.0, wavelength: float = 600.0, f0: float = 20.0, rec_every: int = 1) -> Problem:
    """T6 mesh of a 3000 m x 1500 m domain (for nx = 150, ny = 300) with a
    sinusoidal free-surface topography: the structured T6 grid (x vertical,
    nx elements; y horizontal, ny elements) is mapped by
    x' = x + (x / xmax) * amp * sin(2 pi y / wavelength), so the top follows
    the sinusoid and the bottom stays flat.  VTI medium from Thomsen
    parameters (vp0 3000, vs0 1500, rho 2200, epsilon 0.2, delta 0.1, axis
    vertical).  Free surface at the top (x = xmax), M-PML on the bottom and
    both sides; a vertical force one element below the surface at the centre;
    receivers on the surface nodes every `rec_every` element edges inside the
    M-PML span."""
    xmax, ymax = nx * h, ny * h
    mesh = structured_mesh("T6", nx, ny, 0.0, xmax, 0.0, ymax)
    topo = amp * np.sin(2.0 * np.pi * mesh.y / wavelength)
    mesh.x = mesh.x + (mesh.x / xmax) * topo
    mesh.xmin, mesh.xmax, mesh.ymin, mesh.ymax = 0.0, xmax, 0.0, ymax
    model = vti_model(mesh.node_num, 3000.0, 1500.0, 2200.0, 0.2, 0.1)
    yc = ymax / 2.0
    xs = xmax + amp * math.sin(2.0 * np.pi * yc / wavelength) - h
    src = locate(mesh, h / 2.0, [(xs, yc)])
    ys = np.arange(pml * h, ymax - pml * h + 1e-9, rec_every * h)
    rec = locate(mesh, h / 2.0, [(xmax + amp * math.sin(2.0 * np.pi * y / wavelength), y) for y in ys])
    return Problem(mesh, model, step, dt, f0, 0.0, h, pml, pml, src, rec, 1, f"config4_t6_{nx}x{ny}_topo")


def config_3b(count: int = 16, lo: int = 100, hi: int = 600, seed: int = 4, h: float = 10.0, step: int = 2000,
              pml: int = 20, f0: float = 20.0):
    """Independent Q4 problems with edge lengths drawn from [lo, hi]
    elements (seeded): each a square of n h with a GRF model (the config-3a
    recipe, its own seed), one 20 Hz source at the centre, receivers on the
    top interior row, dt = 1 ms."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = rng.integers(lo, hi + 1, count)
    probs = []
    for k, n in enumerate(sizes):
        n = int(n)
        L = n * h
        mesh = structured_mesh("Q4", n, n, 0.0, L, 0.0, L)
        model = grf_model(mesh, n, h, 200.0, seed=seed * 1000 + k)
        src = locate(mesh, h, [(round(n / 2) * h, round(n / 2) * h)])
        xr = L - pml * h
        nrec = n - 2 * pml + 1
        rec = locate(mesh, h, line_points(nrec, (xr, pml * h), (xr, L - pml * h)))
        probs.append(Problem(mesh, model, step, 1e-3, f0, 0.0, h, pml, pml, src, rec, 0, f"config3b_q4_{n}"))
    return probs


class AcousticCase:
    """A scalar acoustic run (time_evolution/acoustic.c / acoustic_pml.c):
    mesh, vp per node, source node and loop parameters."""

    def __init__(self, mesh, vp, src, step, dt, f0, pml, edge_size, pml_n, name):
        self.mesh, self.vp, self.src, self.step, self.dt, self.f0 = mesh, vp, src, step, dt, f0
        self.pml, self.edge_size, self.pml_n, self.name = pml, edge_size, pml_n, name


def acoustic_grf(n: int = 800, h: float = 10.0, step: int = 1002, dt: float = 5e-4, pml: bool = True,
                 pml_n: int = 20, seed: int = 6) -> AcousticCase:
    """Q4 n x n elements, GRF vp (mean 3000 m/s, std 400, correlation length
    200 m, clipped to 1800-4500, seeded), 20 Hz Ricker source at the centre,
    classical PML pml_n elements thick on four sides; dt keeps vp dt / h at
    or below 0.225."""
    L = n * h
    mesh = structured_mesh("Q4", n, n, 0.0, L, 0.0, L)
    vp = gaussian_random_field((n + 1, n + 1), h, 200.0, 3000.0, 400.0, 1800.0, 4500.0, seed).ravel()
    src = locate(mesh, h, [(L / 2, L / 2)])[0]
    kind = "pml" if pml else "plain"
    return AcousticCase(mesh, vp, int(src), step, dt, 20.0, pml, h, pml_n, f"acoustic_{kind}_q4_{n}")
