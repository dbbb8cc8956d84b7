"""Case generation and the reference's case-file formats.

A case is a single structured block of hexahedral elements with a high-order
grid, a flow state at the nodal solution DOFs, and the run parameters. This
module writes the three files the reference solver reads for such a case:

* ``param.cfg``  -- "keyword: value" parameter file plus the subface table
  (parser: src/InputParamClass.cpp:155-444, 1441-1580);
* the PLOT3D grid -- Fortran unformatted records, single block, i fastest,
  x block then y block then z block (reader: src/SolverClass.cpp:2893-3032);
* the SU2 restart -- header {535532, nVar, nDOFs, 1, 8}, 33-byte variable
  names, then per element (i fastest) and per nodal DOF (i fastest) the values
  x, y, z, rho, rho u, rho v, rho w, rho E in dimensional form, then one int
  and 8 doubles of metadata (reader: src/SolverClass.cpp:3040-3376 and
  include/SolverClass.hpp:679-740; writer: src/SolverClass.cpp:4375-4808).

The same arrays are handed to the GPU path directly, so both solvers start
from identical grids and states. The analytic initial states (isentropic
vortex, Taylor-Green vortex, Gaussian pressure pulse) are evaluated here in
dimensional variables with the reference conditions of
InputParamClass::ComputeReferenceConditions (src/InputParamClass.cpp:605-761).
"""
from __future__ import annotations

import dataclasses
import math
import os
import struct
from typing import Optional, Sequence, Tuple

import numpy as np

GAMMA = 1.4
R_GAS = 287.058
# Boundary-condition names of the subface table (src/InputParamClass.cpp:1441-1580).
BC_NAMES = {"periodic": "Periodic1to1Trans", "outflow_nscbc": "BCOutflowNSCBC",
            "inflow_static_nscbc": "BCInflowStaticNSCBC",
            "inflow_total_nscbc": "BCInflowTotalNSCBC",
            "wall_heat_flux": "BCWallHeatFlux", "wall_isothermal": "BCWallIsothermal",
            "wall_inviscid": "BCWallInviscid", "farfield": "BCFarfield",
            "inflow_subsonic": "BCInflowSubsonic", "inflow_supersonic": "BCInflowSupersonic",
            "outflow_subsonic": "BCOutflowSubsonic", "outflow_supersonic": "BCOutflowSupersonic"}
MU_DIM = 1.716e-5
SU2_MAGIC = 535532
NAME_LEN = 33


def lgl_points(n: int) -> np.ndarray:
    """Gauss-Lobatto-Legendre points on [-1, 1] (n points).

    Closed forms for n <= 7 as used by LocationDOFs1D
    (src/StandAloneFunctions.cpp:182-327); Newton iteration on
    (1 - x^2) P'_{n-1}(x) otherwise.
    """
    if n == 1:
        return np.zeros(1)
    if n == 2:
        return np.array([-1.0, 1.0])
    if n == 3:
        return np.array([-1.0, 0.0, 1.0])
    if n == 4:
        a = math.sqrt(1.0 / 5.0)
        return np.array([-1.0, -a, a, 1.0])
    if n == 5:
        a = math.sqrt(3.0 / 7.0)
        return np.array([-1.0, -a, 0.0, a, 1.0])
    if n == 6:
        t1 = 2.0 * math.sqrt(7.0) / 21.0
        t2 = math.sqrt(1.0 / 3.0 + t1)
        t3 = math.sqrt(1.0 / 3.0 - t1)
        return np.array([-1.0, -t2, -t3, t3, t2, 1.0])
    if n == 7:
        t1 = 2.0 * math.sqrt(5.0 / 3.0) / 11.0
        t2 = math.sqrt(5.0 / 11.0 + t1)
        t3 = math.sqrt(5.0 / 11.0 - t1)
        return np.array([-1.0, -t2, -t3, 0.0, t3, t2, 1.0])
    N = n - 1
    x = -np.cos(np.pi * np.arange(n) / N)
    for _ in range(100):
        P0, P1 = np.ones_like(x), x.copy()
        for k in range(2, N + 1):
            P0, P1 = P1, ((2 * k - 1) * x * P1 - (k - 1) * P0) / k
        dx = (x * P1 - P0) / (n * P1)
        x = x - dx
        if np.max(np.abs(dx)) < 1e-16:
            break
    x[0], x[-1] = -1.0, 1.0
    return x


def equidistant_points(n: int) -> np.ndarray:
    return np.array([-1.0 + i * 2.0 / (n - 1) for i in range(n)]) if n > 1 else np.zeros(1)


@dataclasses.dataclass
class CaseSpec:
    """Everything that defines one case (grid, physics, discretisation)."""

    name: str = "case"
    kind: str = "vortex"                 # vortex | tgv | pulse | uniform
    n_elem: Tuple[int, int, int] = (8, 8, 8)
    p: int = 3                           # polynomial degree of the solution
    p_grid: Optional[int] = None         # polynomial degree of the grid (default p)
    n_poly_int: Optional[int] = None     # integration rule degree (default 3p)
    lo: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    hi: Tuple[float, float, float] = (10.0, 10.0, 10.0)
    mach: float = 0.5
    reynolds: float = 1.0e4
    reynolds_length: float = 1.0
    t_inf: float = 288.15
    vel_dir: Tuple[float, float, float] = (1.0, 0.0, 0.0)
    riemann: str = "IsmailRoe"           # IsmailRoe | Roe
    theta_sym: float = 1.0
    penalty: float = 1.0
    cfl: float = 0.5
    # Grid deformation: "sine" = x_i + amp sin(pi x_j/h) sin(pi x_k/h) with h = L/2,
    # "random" = seeded uniform node perturbation of amp * element size,
    # applied to nodes not on the block boundary; "none" = uniform grid.
    grid_map: str = "sine"
    grid_amp: float = 0.05
    seed: int = 1
    # Isentropic vortex strength and centre.
    beta: float = 5.0
    center: Tuple[float, float, float] = (5.0, 5.0, 5.0)
    # Pressure pulse amplitude (relative) and width.
    pulse_amp: float = 1.0e-3
    pulse_width: float = 0.5
    # Block-face boundary conditions (iMin, iMax, jMin, jMax, kMin, kMax): "periodic",
    # "outflow_nscbc" (BCOutflowNSCBC, prescribed static pressure) or
    # "inflow_static_nscbc" (BCInflowStaticNSCBC, prescribed density and velocity) or
    # "inflow_total_nscbc" (BCInflowTotalNSCBC, prescribed total pressure, total
    # temperature and velocity direction), or a condition through a boundary
    # state: "wall_heat_flux", "wall_isothermal", "wall_inviscid", "farfield",
    # "inflow_subsonic" (total conditions), "inflow_supersonic",
    # "outflow_subsonic" (static pressure), "outflow_supersonic".
    bc: Tuple[str, ...] = ("periodic",) * 6
    p_inf: float = 101325.0          # free-stream static pressure of open cases (Pa)
    # NSCBC tuning parameters (src/InputParamClass.cpp:406-424).
    outlet_len: float = 1.0
    outlet_sigma: float = 0.25
    outlet_beta_l: float = 0.5
    outlet_beta_t: float = 0.5
    outlet_one_minus_beta: bool = True
    inlet_len: float = 1.0
    inlet_sigma: float = 1.0
    inlet_incoming: bool = False
    # Sponge layers: elements per block face, damping constant and exponent; the
    # characteristic matching layer acts in every sponge element.
    sponge: Tuple[int, ...] = (0,) * 6
    sponge_sigma: float = 20.0           # one value, or one per block face
    sponge_alpha: float = 2.0            # one value, or one per block face
    cml: bool = False
    # Prescribed data of the characteristic boundaries (dimensional), per block
    # face: outflow pressure and inflow (rho, u, v, w); None: the free stream.
    prescribed_p: Optional[Tuple[float, ...]] = None
    prescribed_inflow: Optional[Tuple[Tuple[float, float, float, float], ...]] = None
    # Total inflow per block face: (p_t, T_t, direction x, y, z); None: from the
    # free stream (total_inflow_values).
    prescribed_total: Optional[Tuple[Tuple[float, float, float, float, float], ...]] = None
    # Sponge-layer target state (rho, u, v, w, p, dimensional); None: the free stream.
    sponge_state: Optional[Tuple[float, ...]] = None
    # Per block face: heat flux (W/m^2) of heat-flux walls or temperature (K) of
    # isothermal walls; None: adiabatic walls and walls at t_inf.
    wall_data: Optional[Tuple[float, ...]] = None
    # Supersonic inflow state per face (rho, u, v, w, p) and the far-field state,
    # dimensional; None: the free stream.
    prescribed_super: Optional[Tuple[Tuple[float, ...], ...]] = None
    free_stream: Optional[Tuple[float, ...]] = None
    # Subgrid-scale model: "none", "wale" or "vreman" (src/SGSModel.cpp).
    sgs: str = "none"
    # Wall force coefficients in the monitoring data ("Monitor forces") and their
    # reference area.
    monitor_forces: bool = False
    ref_area: float = 1.0
    # Body force per unit volume (N/m^3, x, y, z); None: none.
    body_force: Optional[Tuple[float, float, float]] = None
    # "Location of the DOFs" of the solution ("lgl" or "equidistant") and whether
    # the grid nodes sit at LGL positions (generated grids do).
    dof_location: str = "lgl"
    grid_lgl: bool = True
    # Several subfaces per block face: entries (face, (b0, e0, b1, e1), bc) or
    # (face, (b0, e0, b1, e1), bc, data), the element rectangle [b0, e0) x [b1, e1)
    # of block face `face` along its two in-plane directions in i, j, k order. A
    # block face named here takes its conditions from its subfaces, which must
    # cover it (its bc entry then only marks it as non-periodic). data, when
    # given, is the subface's prescribed data (dimensional): (p,) for outflows,
    # (rho, u, v, w) for the static inflow, (p_t, T_t, dir x, y, z) for total
    # inflows, (value,) for walls, (rho, u, v, w, p) for the supersonic inflow;
    # otherwise the face's data apply.
    subfaces: Optional[Tuple[tuple, ...]] = None
    # "Outlet use local (element) averaged Mach number".
    outlet_local_mach: bool = False

    def __post_init__(self):
        if self.p_grid is None:
            self.p_grid = self.p
        if self.n_poly_int is None:
            self.n_poly_int = 3 * self.p
        self.n_elem = tuple(int(v) for v in self.n_elem)
        self.bc = tuple(str(b) for b in self.bc)
        self.sponge = tuple(int(v) for v in self.sponge)
        for d in range(3):
            a, b = self.bc[2 * d], self.bc[2 * d + 1]
            if (a == "periodic") != (b == "periodic"):
                raise ValueError("a direction is periodic on both faces or on neither")
        for b in self.bc:
            if b not in BC_NAMES:
                raise ValueError(f"unknown boundary condition {b!r}")
        if self.cml and not any(self.sponge):
            raise ValueError("the matching layer needs sponge layers")
        if self.subfaces is not None:
            self.subfaces = tuple(
                (int(e[0]), tuple(int(v) for v in e[1]), str(e[2]),
                 tuple(float(v) for v in e[3]) if len(e) > 3 and e[3] is not None else None)
                for e in self.subfaces)
            for f, r, b, _ in self.subfaces:
                if b not in BC_NAMES or b == "periodic" or self.bc[f] == "periodic":
                    raise ValueError(f"subface on face {f}: {b!r} on a non-periodic face only")

    def face_subfaces(self, f: int):
        """The subfaces of block face f as (range, bc, data); one covering the whole
        face with bc[f] and the face's data when none are given."""
        if self.subfaces and any(sf[0] == f for sf in self.subfaces):
            return [(r, b, dat) for g, r, b, dat in self.subfaces if g == f]
        d = f // 2
        a0, a1 = (1, 2) if d == 0 else ((0, 2) if d == 1 else (0, 1))
        return [((0, self.n_elem[a0], 0, self.n_elem[a1]), self.bc[f], None)]

    @property
    def is_open(self) -> bool:
        return any(b != "periodic" for b in self.bc) or any(self.sponge)

    @property
    def periodic(self) -> Tuple[int, int, int]:
        return tuple(int(self.bc[2 * d] == "periodic") for d in range(3))

    @property
    def n_dofs_1d(self) -> int:
        return self.p + 1

    @property
    def n_elements(self) -> int:
        return self.n_elem[0] * self.n_elem[1] * self.n_elem[2]

    @property
    def n_dofs(self) -> int:
        return self.n_elements * self.n_dofs_1d ** 3


@dataclasses.dataclass
class RefConditions:
    """Reference state for a case with only periodic faces.

    Follows the far-field branch of ComputeReferenceConditions
    (src/InputParamClass.cpp:605-761): v_inf = M sqrt(gamma R T),
    rho_ref = Re mu / (L v_inf), p_ref = rho_ref R T, u_ref = sqrt(p_ref/rho_ref),
    and the non-dimensional viscosity mu u_ref / p_ref.
    """

    p_ref: float
    rho_ref: float
    u_ref: float
    mu_nondim: float
    v_inf: float
    vel_dir: Tuple[float, float, float]


def reference_conditions(spec: CaseSpec) -> RefConditions:
    """With a prescribed outflow pressure and inflow density (open cases) those are
    the reference pressure and density and the Reynolds number is not used, as in
    the reference; otherwise the far-field branch."""
    v_inf = spec.mach * math.sqrt(GAMMA * R_GAS * spec.t_inf)
    d = np.asarray(spec.vel_dir, dtype=float)
    d = d / math.sqrt(float(d @ d))
    outflow_p = any(b in ("outflow_nscbc", "outflow_subsonic") for b in spec.bc)
    total_in = any(b in ("inflow_total_nscbc", "inflow_subsonic") for b in spec.bc)
    if outflow_p and "inflow_static_nscbc" in spec.bc:
        p_ref = spec.p_inf
        rho_ref = spec.p_inf / (R_GAS * spec.t_inf)
    elif outflow_p and total_in:
        # Static outflow pressure and total temperature: rho_ref = p / (R T_t).
        p_ref = spec.p_inf
        rho_ref = spec.p_inf / (R_GAS * total_inflow_values(spec)[1])
    elif outflow_p or total_in:
        raise NotImplementedError("generated cases pair a pressure outflow with a static "
                                  "or total-condition inflow")
    else:
        rho_ref = spec.reynolds * MU_DIM / (spec.reynolds_length * v_inf)
        p_ref = rho_ref * R_GAS * spec.t_inf
    u_ref = math.sqrt(p_ref / rho_ref)
    return RefConditions(p_ref, rho_ref, u_ref, MU_DIM * u_ref / p_ref, v_inf,
                         tuple(float(c) for c in d))


# ---------------------------------------------------------------------------
# Grid
# ---------------------------------------------------------------------------

def _nodes_1d(n_elem: int, p: int, lo: float, hi: float) -> np.ndarray:
    """Block node coordinates along one index direction: LGL nodes per element."""
    r = lgl_points(p + 1)
    h = (hi - lo) / n_elem
    out = np.empty(n_elem * p + 1)
    for e in range(n_elem):
        out[e * p:(e + 1) * p + 1] = lo + h * (e + 0.5 * (r + 1.0))
    out[-1] = hi
    return out


def make_grid(spec: CaseSpec) -> np.ndarray:
    """Block grid nodes, shape (3, kl, jl, il): x, y, z with i fastest."""
    pg = spec.p_grid
    xs = [_nodes_1d(spec.n_elem[d], pg, spec.lo[d], spec.hi[d]) for d in range(3)]
    Z, Y, X = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
    if spec.grid_map == "sine":
        h = [0.5 * (spec.hi[d] - spec.lo[d]) for d in range(3)]
        a = spec.grid_amp
        sx = np.sin(np.pi * (X - spec.lo[0]) / h[0])
        sy = np.sin(np.pi * (Y - spec.lo[1]) / h[1])
        sz = np.sin(np.pi * (Z - spec.lo[2]) / h[2])
        Xn, Yn, Zn = X + a * sy * sz, Y + a * sx * sz, Z + a * sx * sy
        X, Y, Z = Xn, Yn, Zn
    elif spec.grid_map == "random":
        rng = np.random.default_rng(spec.seed)
        dh = [(spec.hi[d] - spec.lo[d]) / spec.n_elem[d] for d in range(3)]
        pert = rng.uniform(-1.0, 1.0, size=(3,) + X.shape)
        interior = np.zeros(X.shape, dtype=bool)
        interior[1:-1, 1:-1, 1:-1] = True
        X = X + np.where(interior, spec.grid_amp * dh[0] * pert[0], 0.0)
        Y = Y + np.where(interior, spec.grid_amp * dh[1] * pert[1], 0.0)
        Z = Z + np.where(interior, spec.grid_amp * dh[2] * pert[2], 0.0)
    elif spec.grid_map != "none":
        raise ValueError(f"unknown grid_map {spec.grid_map!r}")
    return np.stack([X, Y, Z])


def element_nodes(grid: np.ndarray, n_elem: Sequence[int], p: int) -> np.ndarray:
    """Per-element grid nodes, shape (nElem, 3, (p+1)^3); elements and nodes i fastest.

    Same gathering as SolverClass::ReadGrid (src/SolverClass.cpp:2993-3032).
    """
    nI, nJ, nK = n_elem
    n1 = p + 1
    g = np.ascontiguousarray(grid)
    s3, sk, sj, si = g.strides
    # View [k, j, i, x, c, b, a] of the overlapping element blocks (stride p nodes).
    view = np.lib.stride_tricks.as_strided(
        g, shape=(nK, nJ, nI, 3, n1, n1, n1),
        strides=(p * sk, p * sj, p * si, s3, sk, sj, si), writeable=False)
    return np.ascontiguousarray(view).reshape(nI * nJ * nK, 3, n1 ** 3)


# ---------------------------------------------------------------------------
# Initial states (dimensional primitive -> conservative at the nodal DOFs)
# ---------------------------------------------------------------------------

def primitive_state(spec: CaseSpec, xyz: np.ndarray, ref: RefConditions):
    """Dimensional (rho, u, v, w, p) at points xyz (shape (3, ...))."""
    x, y, z = xyz[0], xyz[1], xyz[2]
    rho_inf, p_inf, c_u = ref.rho_ref, ref.p_ref, ref.u_ref
    u_inf = [ref.v_inf * d for d in ref.vel_dir]
    if spec.kind == "uniform":
        ones = np.ones_like(x)
        return rho_inf * ones, u_inf[0] * ones, u_inf[1] * ones, u_inf[2] * ones, p_inf * ones
    if spec.kind == "vortex":
        # Shu's isentropic vortex about the z axis: velocity perturbation scaled by
        # sqrt(p_inf/rho_inf), temperature T/T_inf = 1 - (g-1) b^2/(8 g pi^2) e^(1-r^2).
        dx, dy = x - spec.center[0], y - spec.center[1]
        r2 = dx * dx + dy * dy
        b = spec.beta
        f = b / (2.0 * np.pi) * np.exp(0.5 * (1.0 - r2))
        T = 1.0 - (GAMMA - 1.0) * b * b / (8.0 * GAMMA * np.pi ** 2) * np.exp(1.0 - r2)
        rho = rho_inf * T ** (1.0 / (GAMMA - 1.0))
        p = p_inf * T ** (GAMMA / (GAMMA - 1.0))
        u = u_inf[0] - c_u * f * dy
        v = u_inf[1] + c_u * f * dx
        w = u_inf[2] + 0.0 * x
        return rho, u, v, w, p
    if spec.kind == "tgv":
        # Taylor-Green vortex with V0 = v_inf, rho0 = rho_ref, p0 = p_ref, unit length.
        V0 = ref.v_inf
        u = V0 * np.sin(x) * np.cos(y) * np.cos(z)
        v = -V0 * np.cos(x) * np.sin(y) * np.cos(z)
        w = 0.0 * x
        p = p_inf + rho_inf * V0 * V0 / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
        rho = p / (R_GAS * spec.t_inf)
        return rho, u, v, w, p
    if spec.kind == "pulse":
        # Gaussian pressure pulse p = p_inf (1 + a exp(-r^2/(2 w^2))) on the free
        # stream, density unchanged (the reference's "Pressure pulse" fluctuation,
        # src/ElementClass.cpp:600-663).
        r2 = sum((c - spec.center[d]) ** 2 for d, c in enumerate((x, y, z)))
        p = p_inf * (1.0 + spec.pulse_amp * np.exp(-r2 * (0.5 / (spec.pulse_width ** 2))))
        ones = np.ones_like(x)
        return rho_inf * ones, u_inf[0] * ones, u_inf[1] * ones, u_inf[2] * ones, p
    raise ValueError(f"unknown case kind {spec.kind!r}")


def conservative_state(spec: CaseSpec, xyz: np.ndarray, ref: RefConditions) -> np.ndarray:
    """Dimensional conservative variables, shape (5,) + xyz.shape[1:]."""
    rho, u, v, w, p = primitive_state(spec, xyz, ref)
    rE = p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return np.stack([rho, rho * u, rho * v, rho * w, rE])


def _lagrange_1d(nodes: np.ndarray, points: np.ndarray) -> np.ndarray:
    """L[j, i]: the Lagrange polynomial of node j at point i."""
    L = np.ones((len(nodes), len(points)))
    for j in range(len(nodes)):
        for m in range(len(nodes)):
            if m != j:
                L[j] *= (points - nodes[m]) / (nodes[j] - nodes[m])
    return L


def dof_location_code(spec: CaseSpec) -> int:
    """enum vcpg_dof_location of a case: solution DOF and grid node positions."""
    sol_lgl = spec.dof_location.lower() == "lgl"
    return {(True, True): 1, (False, False): 0, (False, True): 2, (True, False): 3}[
        (sol_lgl, bool(spec.grid_lgl))]


def solution_dof_coordinates(spec: CaseSpec, elem_nodes: np.ndarray) -> np.ndarray:
    """Coordinates of the nodal solution DOFs per element, shape (nElem, 3, K^3):
    the grid interpolated with its Lagrange polynomials to the DOF positions
    (ElementClass::ComputeCoorNodalSolDOFs, src/ElementClass.cpp:816-918). With
    DOFs at the grid's own positions they are the grid nodes."""
    Kg, K = spec.p_grid + 1, spec.p + 1
    sol_lgl = spec.dof_location.lower() == "lgl"
    if Kg == K and sol_lgl == bool(spec.grid_lgl):
        return elem_nodes
    rg = lgl_points(Kg) if spec.grid_lgl else equidistant_points(Kg)
    rs = lgl_points(K) if sol_lgl else equidistant_points(K)
    L = _lagrange_1d(rg, rs)                                  # [Kg, K]
    x = elem_nodes.reshape(elem_nodes.shape[0], 3, Kg, Kg, Kg)   # (k, j, i)
    for ax in (4, 3, 2):
        x = np.moveaxis(np.tensordot(x, L, axes=([ax], [0])), -1, ax)
    return np.ascontiguousarray(x.reshape(elem_nodes.shape[0], 3, K ** 3))


# ---------------------------------------------------------------------------
# File formats
# ---------------------------------------------------------------------------

def write_plot3d(path: str, grid: np.ndarray) -> None:
    """Single-block PLOT3D file with Fortran record markers (double precision)."""
    _, kl, jl, il = grid.shape
    n = il * jl * kl
    with open(path, "wb") as f:
        f.write(struct.pack("<iii", 4, 1, 4))
        f.write(struct.pack("<iiiii", 12, il, jl, kl, 12))
        f.write(struct.pack("<i", 24 * n))
        f.write(np.ascontiguousarray(grid, dtype="<f8").tobytes())
        f.write(struct.pack("<i", 24 * n))


def read_plot3d(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        data = f.read()
    if struct.unpack_from("<i", data, 0)[0] == 4:
        off = 12
    else:
        off = 0
    _, il, jl, kl, _ = struct.unpack_from("<iiiii", data, off)
    off += 20 + 4
    n = il * jl * kl
    arr = np.frombuffer(data, dtype="<f8", count=3 * n, offset=off)
    return arr.reshape(3, kl, jl, il).copy()


def write_su2_restart(path: str, dof_xyz: np.ndarray, cons: np.ndarray,
                      extra: Optional[np.ndarray] = None, extra_names=()) -> None:
    """SU2 restart: per element, per DOF: x y z rho rhou rhov rhow rhoE (doubles),
    followed by the `extra` variables (shape (nElem, nExtra, nDOFs)) if given.

    dof_xyz has shape (nElem, 3, nDOFs); cons has shape (nElem, 5, nDOFs).
    """
    n_elem, _, n_dofs = dof_xyz.shape
    names = ["x", "y", "z", "Density", "Momentum_x", "Momentum_y", "Momentum_z", "Energy"]
    cols = [dof_xyz, cons]
    if extra is not None:
        names += list(extra_names)
        cols.append(extra)
    body = np.concatenate(cols, axis=1).transpose(0, 2, 1)  # elem, dof, var
    with open(path, "wb") as f:
        f.write(struct.pack("<5i", SU2_MAGIC, len(names), n_elem * n_dofs, 1, 8))
        for nm in names:
            f.write(nm.encode().ljust(NAME_LEN, b"\0")[:NAME_LEN])
        f.write(np.ascontiguousarray(body, dtype="<f8").tobytes())
        f.write(struct.pack("<i", 0))
        f.write(np.zeros(8, dtype="<f8").tobytes())


def read_su2_restart(path: str, n_elem: int, n_dofs: int):
    with open(path, "rb") as f:
        data = f.read()
    hdr = struct.unpack_from("<5i", data, 0)
    if hdr[0] != SU2_MAGIC:
        raise ValueError("not an SU2 restart file")
    nvar = hdr[1]
    off = 20 + nvar * NAME_LEN
    body = np.frombuffer(data, dtype="<f8", count=n_elem * n_dofs * nvar, offset=off)
    body = body.reshape(n_elem, n_dofs, nvar).transpose(0, 2, 1)
    return body[:, :3].copy(), body[:, 3:8].copy()


def _subfaces(spec: CaseSpec) -> str:
    """Subface table: periodic faces (1-to-1 with a translation) over the whole
    face; physical faces as one subface or as the spec's subfaces, with node
    index ranges (the elements [b, e) of an in-plane direction span the nodes
    b + 1 .. e + 1)."""
    nI, nJ, nK = spec.n_elem
    L = [spec.hi[d] - spec.lo[d] for d in range(3)]
    I, J, K = nI + 1, nJ + 1, nK + 1
    rows = [
        (f"1 1 1 {J} 1 {K}", f"{I} {I} 1 {J} 1 {K}", (L[0], 0.0, 0.0)),
        (f"{I} {I} 1 {J} 1 {K}", f"1 1 1 {J} 1 {K}", (-L[0], 0.0, 0.0)),
        (f"1 {I} 1 1 1 {K}", f"1 {I} {J} {J} 1 {K}", (0.0, L[1], 0.0)),
        (f"1 {I} {J} {J} 1 {K}", f"1 {I} 1 1 1 {K}", (0.0, -L[1], 0.0)),
        (f"1 {I} 1 {J} 1 1", f"1 {I} 1 {J} {K} {K}", (0.0, 0.0, L[2])),
        (f"1 {I} 1 {J} {K} {K}", f"1 {I} 1 {J} 1 1", (0.0, 0.0, -L[2])),
    ]
    nodes = (I, J, K)
    out = []
    for face, (own, donor, t) in enumerate(rows, start=1):
        bc = spec.bc[face - 1]
        if bc == "periodic":
            out.append(f"    {face}    1")
            out.append(f"        Periodic1to1Trans  {own}   {donor}   1 2 3   "
                       f"{t[0]!r} {t[1]!r} {t[2]!r}")
            continue
        subs = spec.face_subfaces(face - 1)
        out.append(f"    {face}    {len(subs)}")
        d = (face - 1) // 2
        plane = 1 if (face - 1) % 2 == 0 else nodes[d]
        a0, a1 = (1, 2) if d == 0 else ((0, 2) if d == 1 else (0, 1))
        for (b0, e0, b1, e1), sbc, _ in subs:
            rng = [None] * 3
            rng[d] = (plane, plane)
            rng[a0] = (b0 + 1, e0 + 1)
            rng[a1] = (b1 + 1, e1 + 1)
            out.append(f"        {BC_NAMES[sbc]}  " + " ".join(f"{x} {y}" for x, y in rng))
    return "\n".join(out)


def _open_blocks(spec: CaseSpec, ref: "RefConditions") -> Tuple[str, str, str]:
    """(parameter lines, sponge block, prescribed-data block) of an open case."""
    if not spec.is_open:
        return "", "", ""
    yn = lambda v: "yes" if v else "no"
    params = f"""Outlet characteristic length: {spec.outlet_len!r}
Outlet normal relaxation (sigma): {spec.outlet_sigma!r}
Outlet use one minus beta transverse relaxation: {yn(spec.outlet_one_minus_beta)}
Outlet use local (element) averaged Mach number: {yn(spec.outlet_local_mach)}
Outlet coupled   transverse relaxation (beta_l): {spec.outlet_beta_l!r}
Outlet uncoupled transverse relaxation (beta_t): {spec.outlet_beta_t!r}
Inlet characteristic length: {spec.inlet_len!r}
Inlet normal relaxation (sigma): {spec.inlet_sigma!r}
Inlet use outgoing wave amplitude: {yn(spec.inlet_incoming)}
"""
    sponge = ""
    if any(spec.sponge):
        params += f"""Sponge layer: yes
Characteristic matching layer: {yn(spec.cml)}
Averaged solution file name: averaged.dat
"""
        rows = "\n".join(f"    {f + 1}    {spec.sponge[f]}    {spec.sponge_sigma!r}    "
                         f"{spec.sponge_alpha!r}" for f in range(6))
        sponge = f"""
Sponge layer information
#Face nBufferElem DampingConstant DampingExponent
{rows}
"""
    p_out, rho_in, vel_in = prescribed_values(spec, ref)
    lines = []
    for f, fbc in enumerate(spec.bc):
        if fbc == "periodic":
            continue
        for si, (_, bc, dat) in enumerate(spec.face_subfaces(f), start=1):
            head = f"    {f + 1}    {si}    1    "
            names = _DATA_NAMES.get(bc)
            if dat is not None and names:
                lines.append(head + " ".join(names))
                lines.append("        " + " ".join(repr(float(v)) for v in dat))
            elif bc == "outflow_nscbc":
                lines.append(head + "Pressure")
                lines.append(f"        {p_out!r}")
            elif bc == "inflow_static_nscbc":
                lines.append(head + "Density VelocityX VelocityY VelocityZ")
                lines.append(f"        {rho_in!r} {vel_in[0]!r} {vel_in[1]!r} {vel_in[2]!r}")
            elif bc == "outflow_subsonic":
                lines.append(head + "Pressure")
                lines.append(f"        {p_out!r}")
            elif bc in ("wall_heat_flux", "wall_isothermal"):
                val = spec.wall_data[f] if spec.wall_data else (
                    0.0 if bc == "wall_heat_flux" else spec.t_inf)
                name = "HeatFlux" if bc == "wall_heat_flux" else "Temperature"
                lines.append(head + name)
                lines.append(f"        {float(val)!r}")
            elif bc == "inflow_supersonic":
                q = spec.prescribed_super[f] if spec.prescribed_super else (rho_in, *vel_in, p_out)
                lines.append(head + "Density VelocityX VelocityY VelocityZ Pressure")
                lines.append("        " + " ".join(repr(float(v)) for v in q))
            elif bc in ("inflow_total_nscbc", "inflow_subsonic"):
                t = total_inflow_values(spec)
                lines.append(head + "TotalPressure TotalTemperature VelocityDirX "
                             "VelocityDirY VelocityDirZ")
                lines.append("        " + " ".join(repr(float(v)) for v in t))
    presc = ""
    if lines:
        presc = "\nPrescribed boundary data\n" + "\n".join(lines) + "\n"
    return params, sponge, presc


# Prescribed-data variable names of a subface's data tuple, per condition.
_DATA_NAMES = {
    "outflow_nscbc": ("Pressure",), "outflow_subsonic": ("Pressure",),
    "inflow_static_nscbc": ("Density", "VelocityX", "VelocityY", "VelocityZ"),
    "inflow_total_nscbc": ("TotalPressure", "TotalTemperature", "VelocityDirX", "VelocityDirY",
                           "VelocityDirZ"),
    "inflow_subsonic": ("TotalPressure", "TotalTemperature", "VelocityDirX", "VelocityDirY",
                        "VelocityDirZ"),
    "wall_heat_flux": ("HeatFlux",), "wall_isothermal": ("Temperature",),
    "inflow_supersonic": ("Density", "VelocityX", "VelocityY", "VelocityZ", "Pressure"),
}


def total_inflow_values(spec: CaseSpec):
    """Total pressure and temperature of the free stream (p_inf, t_inf, Mach) and
    the flow direction: the prescribed data of a generated total inflow."""
    ff = 1.0 + 0.5 * (GAMMA - 1.0) * spec.mach ** 2
    d = np.asarray(spec.vel_dir, dtype=float)
    d = d / math.sqrt(float(d @ d))
    return (spec.p_inf * ff ** (GAMMA / (GAMMA - 1.0)), spec.t_inf * ff,
            float(d[0]), float(d[1]), float(d[2]))


def prescribed_values(spec: CaseSpec, ref: "RefConditions"):
    """Outflow pressure, inflow density and velocity (dimensional): the free stream."""
    vel = tuple(float(ref.v_inf * c) for c in ref.vel_dir)
    return float(ref.p_ref), float(ref.rho_ref), vel


_SGS_NAMES = {"none": "None", "wale": "WALE", "vreman": "Vreman"}


def _body_force_line(spec: CaseSpec) -> str:
    if spec.body_force is None:
        return ""
    f = spec.body_force
    return f"Body force per unit volume (x,y,z): {f[0]!r} {f[1]!r} {f[2]!r}\n"


def free_stream_values(spec: CaseSpec) -> Tuple[float, float, float, float, float]:
    """Dimensional free stream (rho, u, v, w, p) of a generated case as the
    reference derives it from the prescribed boundary data of its parameter file
    (DetermineNonDimPrimVarFreeStream, src/InputParamClass.cpp:991-1192): the
    far-field state and the default of CaseSpec.free_stream."""
    from . import param_file
    pf = param_file.parse(param_cfg_text(spec))
    return param_file.reference_conditions(pf).free_stream


def param_cfg_text(spec: CaseSpec, grid_file="grid.xyz", restart_file="restart.dat",
                   restart=True) -> str:
    d = spec.vel_dir
    open_params, sponge, presc = _open_blocks(spec, reference_conditions(spec))
    return f"""# Generated case {spec.name} ({spec.kind})
Polynomial degree grid: {spec.p_grid}
Polynomial degree solution: {spec.p}
Polynomial degree integration rule: {spec.n_poly_int}
Location of the DOFs: {"LGL" if spec.dof_location.lower() == "lgl" else "Equidistant"}
Grid file name: {grid_file}
Solution file name: data/Solution
Restart file name: {restart_file}
Restart: {"yes" if restart else "no"}
Paraview visualization file name: anim/Solution.vtk
Space average data file name: proc/SpaceAverage.vtk
SU2 grid file name: proc/GridSU2.su2
Write SU2 grid file: no
Save solution every: 100000000
Write time history info every: 1
FEM working variables: Entropy
Riemann solver: {spec.riemann}
Subgrid scale model: {_SGS_NAMES[spec.sgs.lower()]}
Wall modeling: No wall model
Theta parameter symmetrizing terms: {spec.theta_sym!r}
Relative penalty parameter: {spec.penalty!r}
Mach number: {spec.mach!r}
Reynolds number: {spec.reynolds!r}
Reynolds length: {spec.reynolds_length!r}
Free stream temperature: {spec.t_inf!r}
Free stream velocity direction: {d[0]!r} {d[1]!r} {d[2]!r}
Fluctuations to add to initial solution: No fluctuations
Monitor forces: {"yes" if spec.monitor_forces else "no"}
Reference area force coefficients: {spec.ref_area!r}
{_body_force_line(spec)}Number of synchronization time steps: 1
Synchronization time step: 1.0
CFL number: {spec.cfl!r}
Compute average solution: no
{open_params}{sponge}
Subface information
{_subfaces(spec)}
{presc}"""


@dataclasses.dataclass
class CaseData:
    spec: CaseSpec
    ref: RefConditions
    grid: np.ndarray           # (3, kl, jl, il)
    elem_nodes: np.ndarray     # (nElem, 3, K^3)
    dof_xyz: np.ndarray        # (nElem, 3, K^3)
    cons: np.ndarray           # (nElem, 5, K^3) dimensional conservative


def build_case(spec: CaseSpec) -> CaseData:
    ref = reference_conditions(spec)
    grid = make_grid(spec)
    nodes = element_nodes(grid, spec.n_elem, spec.p_grid)
    xyz = solution_dof_coordinates(spec, nodes)
    cons = conservative_state(spec, xyz.transpose(1, 0, 2), ref).transpose(1, 0, 2)
    return CaseData(spec, ref, grid, nodes, xyz, np.ascontiguousarray(cons))


def write_case(case: CaseData, directory: str) -> str:
    """Write param.cfg, grid.xyz and restart.dat into directory; returns the cfg path."""
    os.makedirs(directory, exist_ok=True)
    for sub in ("data", "anim", "proc"):
        os.makedirs(os.path.join(directory, sub), exist_ok=True)
    write_plot3d(os.path.join(directory, "grid.xyz"), case.grid)
    write_su2_restart(os.path.join(directory, "restart.dat"), case.dof_xyz, case.cons)
    if any(case.spec.sponge):
        write_averaged_solution(os.path.join(directory, "averaged.dat"), case)
    cfg = os.path.join(directory, "param.cfg")
    with open(cfg, "w") as f:
        f.write(param_cfg_text(case.spec))
    return cfg


def write_averaged_solution(path: str, case: CaseData) -> None:
    """The averaged-solution file that supplies the sponge-layer damping state
    (SolverClass::ReadAveragedSolutionSpongeLayer, src/SpongeLayer.cpp:667-843):
    an SU2 restart with the solution, the averaged primitive variables
    (density, velocity, pressure), six averaged velocity products and the
    averaged eddy viscosity. The averaged state written here is the free stream."""
    ref = case.ref
    n_elem, _, n_dofs = case.dof_xyz.shape
    vel = [ref.v_inf * c for c in ref.vel_dir]
    avg = np.zeros((n_elem, 12, n_dofs))
    avg[:, 0] = ref.rho_ref
    avg[:, 1], avg[:, 2], avg[:, 3] = vel
    avg[:, 4] = ref.p_ref
    names = ["Density_avg", "VelocityX_avg", "VelocityY_avg", "VelocityZ_avg", "Pressure_avg",
             "R_uu", "R_vv", "R_ww", "R_uv", "R_uw", "R_vw", "EddyVisc_avg"]
    write_su2_restart(path, case.dof_xyz, case.cons, avg, names)
