"""The reference solver's parameter file, read for the path this library runs.

A restatement of InputParamClass (src/InputParamClass.cpp) for the options the
GPU path supports:

* ``keyword: value`` lines (AnalyzeString, src/InputParamClass.cpp:155-441):
  tabs and returns become blanks, ``#`` starts a comment, the keyword is
  matched in lower case after stripping leading and trailing blanks; an
  unknown keyword is an error, as in the reference.
* the "Subface information" block (ReadSubfaceInformation, :1441-1576),
* the "Prescribed boundary data" block (ReadBoundaryData, :1340-1404),
* the "Sponge layer information" block (ReadSpongeLayerData, :1196-1336),
* the reference conditions and the free-stream state that follow from the
  prescribed data (ComputeReferenceConditions :605-761,
  DetermineNonDimPrimVarFreeStream :991-1192).

Options outside the path (conservative working variables, subgrid-scale and
wall models, the symmetry plane, random or
synthetic fluctuations, several subfaces per block face, spatially varying
prescribed data) raise UnsupportedOption with the option named.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, List, Optional, Sequence, Tuple

GAMMA = 1.4
R_GAS = 287.058
MU_DIM = 1.716e-5


class ParamFileError(ValueError):
    """The file is malformed (the reference terminates on it too)."""


class UnsupportedOption(NotImplementedError):
    """A valid option of the reference that this library does not run."""


# keyword (lower case) -> (field, type). Types: int, float, vec3, str, yesno,
# or a tuple of the accepted lower-case values of an enumeration.
_KEYS: Dict[str, Tuple[str, object]] = {
    "location of the dofs": ("dof_location", ("equidistant", "lgl")),
    "fem working variables": ("fem_variables", ("conservative", "entropy")),
    "riemann solver": ("riemann", ("roe", "ismailroe")),
    "wall modeling": ("wall_model", ("no wall model", "equilibrium wall model",
                                     "logarithmic wall model")),
    "subgrid scale model": ("sgs_model", ("none", "wale", "vreman")),
    "fluctuations to add to initial solution": (
        "fluctuations", ("no fluctuations", "random fluctuations", "sine_and_cosine",
                         "synthetic fluctuations", "pressure pulse")),
    "pressure pulse center": ("pulse_center", "vec3"),
    "pressure pulse strength": ("pulse_strength", "float"),
    "pressure pulse width": ("pulse_width", "float"),
    "one-dimensional pulse": ("pulse_1d", "yesno"),
    "pulse (x-)direction": ("pulse_direction", ("upstream", "downstream")),
    "lower coordinates box for fluctuations": ("box_lower", "vec3"),
    "upper coordinates box for fluctuations": ("box_upper", "vec3"),
    "polynomial degree grid": ("p_grid", "int"),
    "polynomial degree solution": ("p", "int"),
    "polynomial degree integration rule": ("n_poly_int", "int"),
    "mach number": ("mach", "float"),
    "reynolds number": ("reynolds", "float"),
    "reynolds length": ("reynolds_length", "float"),
    "free stream temperature": ("t_inf", "float"),
    "free stream velocity direction": ("vel_dir", "vec3"),
    "lift direction": ("lift_dir", "vec3"),
    "body force per unit volume (x,y,z)": ("body_force", "vec3"),
    "exchange location wall model": ("wm_exchange", "float"),
    "number of grid points equilibrium wall model": ("wm_points", "int"),
    "expansion ratio grid equilibrium wall model": ("wm_ratio", "float"),
    "grid file name": ("grid_file", "str"),
    "solution file name": ("solution_file", "str"),
    "restart file name": ("restart_file", "str"),
    "paraview visualization file name": ("paraview_file", "str"),
    "space average data file name": ("space_average_file", "str"),
    "su2 grid file name": ("su2_grid_file", "str"),
    "restart": ("restart", "yesno"),
    "write su2 grid file": ("write_su2_grid", "yesno"),
    "compute average solution": ("compute_average", "yesno"),
    "continue averaging from restart": ("continue_averaging", "yesno"),
    "allow block splitting in i-direction": ("split_i", "yesno"),
    "allow block splitting in j-direction": ("split_j", "yesno"),
    "allow block splitting in k-direction": ("split_k", "yesno"),
    "monitor forces": ("monitor_forces", "yesno"),
    "reference area force coefficients": ("reference_area", "float"),
    "number of synchronization time steps": ("n_sync", "int"),
    "save solution every": ("n_save", "int"),
    "write time history info every": ("n_history", "int"),
    "synchronization time step": ("dt_sync", "float"),
    "cfl number": ("cfl", "float"),
    "theta parameter symmetrizing terms": ("theta_sym", "float"),
    "relative penalty parameter": ("penalty", "float"),
    "outlet use local (element) averaged mach number": ("outlet_local_mach", "yesno"),
    "outlet use one minus beta transverse relaxation": ("outlet_one_minus_beta", "yesno"),
    "outlet characteristic length": ("outlet_len", "float"),
    "outlet normal relaxation (sigma)": ("outlet_sigma", "float"),
    "outlet coupled   transverse relaxation (beta_l)": ("outlet_beta_l", "float"),
    "outlet uncoupled transverse relaxation (beta_t)": ("outlet_beta_t", "float"),
    "inlet characteristic length": ("inlet_len", "float"),
    "inlet normal relaxation (sigma)": ("inlet_sigma", "float"),
    "inlet use outgoing wave amplitude": ("inlet_incoming", "yesno"),
    "averaged solution file name": ("averaged_file", "str"),
    "sponge layer": ("sponge_layer", "yesno"),
    "characteristic matching layer": ("cml", "yesno"),
}

# Boundary conditions the reference accepts (ReadSubfaceInformation) and the
# ones this library runs, by their lower-case names.
_ALL_BCS = ("internal1to1", "periodic1to1trans", "bcfarfield", "bcwallisothermal",
            "bcwallisothermalwm", "bcwallheatflux", "bcwallheatfluxwm", "bcwallinviscid",
            "bcsymmetryplane", "bcinflowsubsonic", "bcinflowsupersonic", "bcoutflowsubsonic",
            "bcoutflowsupersonic", "bcinflowstaticnscbc", "bcinflowtotalnscbc",
            "bcoutflownscbc")
_BC_TO_CASE = {"periodic1to1trans": "periodic", "bcoutflownscbc": "outflow_nscbc",
               "bcinflowstaticnscbc": "inflow_static_nscbc",
               "bcinflowtotalnscbc": "inflow_total_nscbc",
               "bcwallheatflux": "wall_heat_flux", "bcwallisothermal": "wall_isothermal",
               "bcwallinviscid": "wall_inviscid", "bcfarfield": "farfield",
               "bcinflowsubsonic": "inflow_subsonic", "bcinflowsupersonic": "inflow_supersonic",
               "bcoutflowsubsonic": "outflow_subsonic",
               "bcoutflowsupersonic": "outflow_supersonic"}
_WHY_NOT = {"bcsymmetryplane": "BCSymmetryPlane (the reference terminates on it: not "
                               "implemented there either)",
            "bcwallisothermalwm": "BCWallIsothermalWM (wall model)",
            "bcwallheatfluxwm": "BCWallHeatFluxWM (wall model)",
            "internal1to1": "Internal1to1 (multi-block grids)"}
_NSCBC = ("bcinflowstaticnscbc", "bcinflowtotalnscbc", "bcoutflownscbc")


@dataclasses.dataclass
class Subface:
    bc: str                                # name as written
    own: Tuple[int, int, int, int, int, int]   # 1-based element-node index range
    rest: Tuple[str, ...]                  # remaining tokens (periodic donor data)

    @property
    def kind(self) -> str:
        return self.bc.lower()


@dataclasses.dataclass
class ParamFile:
    """The parsed file. Fields not given keep the reference's defaults
    (InputParamClass::InputParamClass, src/InputParamClass.cpp:20-101)."""

    path: str = ""
    dof_location: str = ""              # required
    fem_variables: str = ""             # required
    riemann: str = ""                   # required
    wall_model: str = "no wall model"
    sgs_model: str = "none"
    fluctuations: str = "no fluctuations"
    pulse_center: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    pulse_strength: float = 0.5
    pulse_width: float = 0.5
    pulse_1d: bool = False
    pulse_direction: str = "downstream"
    box_lower: Optional[Tuple[float, float, float]] = None
    box_upper: Optional[Tuple[float, float, float]] = None
    p_grid: int = -1
    p: int = -1
    n_poly_int: int = -1
    mach: float = -1.0
    reynolds: float = -1.0
    reynolds_length: float = -1.0
    t_inf: float = -1.0
    vel_dir: Optional[Tuple[float, float, float]] = None
    lift_dir: Optional[Tuple[float, float, float]] = None
    body_force: Optional[Tuple[float, float, float]] = None
    wm_exchange: float = -1.0
    wm_points: int = -1
    wm_ratio: float = -1.0
    grid_file: str = ""
    solution_file: str = "Solution.dat"
    restart_file: str = ""
    paraview_file: str = "Solution.vtk"
    space_average_file: str = "SpaceAverage.vtk"
    su2_grid_file: str = "Grid.su2"
    restart: bool = False
    write_su2_grid: bool = False
    compute_average: bool = False
    continue_averaging: bool = False
    split_i: bool = True
    split_j: bool = True
    split_k: bool = True
    monitor_forces: bool = True
    reference_area: float = 1.0
    n_sync: int = -1
    n_save: int = 0
    n_history: int = 1
    dt_sync: float = -1.0
    cfl: float = -1.0
    theta_sym: float = 1.0
    penalty: float = 1.0
    outlet_local_mach: bool = False
    outlet_one_minus_beta: bool = True
    outlet_len: float = 1.0
    outlet_sigma: float = 0.0
    outlet_beta_l: float = 1.0
    outlet_beta_t: float = 1.0
    inlet_len: float = 1.0
    inlet_sigma: float = 1.0
    inlet_incoming: bool = True
    averaged_file: str = ""
    sponge_layer: bool = False
    cml: bool = False
    subfaces: List[List[Subface]] = dataclasses.field(default_factory=list)
    # (face, subface) -> {variable name: value}; one point per subface.
    prescribed: Dict[Tuple[int, int], Dict[str, float]] = dataclasses.field(default_factory=dict)
    # per face (elements, damping constant, damping exponent)
    sponge: Optional[List[Tuple[int, float, float]]] = None

    def file(self, name: str) -> str:
        """A file name of the parameter file, relative to its directory."""
        if not name or os.path.isabs(name):
            return name
        return os.path.join(os.path.dirname(self.path), name)


def _lines(text: str) -> List[str]:
    return [ln.replace("\t", " ").replace("\r", " ") for ln in text.split("\n")]


def _value(field: str, kind, key: str, value: str):
    if kind == "int":
        try:
            return int(value.split()[0])
        except (ValueError, IndexError):
            raise ParamFileError(f'"{key}" wrongly specified: {value!r}') from None
    if kind == "float":
        try:
            return float(value.split()[0])
        except (ValueError, IndexError):
            raise ParamFileError(f'"{key}" wrongly specified: {value!r}') from None
    if kind == "vec3":
        parts = value.split()
        try:
            if len(parts) < 3:
                raise ValueError
            return tuple(float(v) for v in parts[:3])
        except ValueError:
            raise ParamFileError(f'"{key}" needs three numbers: {value!r}') from None
    if kind == "str":
        return value
    if kind == "yesno":
        v = value.lower()
        if v not in ("yes", "no"):
            raise ParamFileError(f'"{key}" wrongly specified. It should be yes or no.')
        return v == "yes"
    v = value.lower()
    if v not in kind:
        raise ParamFileError(f'"{key}": unknown value {value!r}')
    return v


def _find_block(lines: Sequence[str], title: str) -> Optional[int]:
    for n, ln in enumerate(lines):
        if ln.strip().lower() == title:
            return n + 1
    return None


def _leading_ints(line: str, count: int) -> Optional[List[int]]:
    parts = line.split()
    if len(parts) < count:
        return None
    try:
        return [int(p) for p in parts[:count]]
    except ValueError:
        return None


def parse(text: str, path: str = "") -> ParamFile:
    pf = ParamFile(path=path)
    lines = _lines(text)
    for ln in lines:
        body = ln.split("#", 1)[0]
        if ":" not in body:
            continue
        key, value = body.split(":", 1)
        key, value = key.strip().lower(), value.strip()
        if not key or not value:
            continue
        if key not in _KEYS:
            raise ParamFileError(f'Unknown keyword "{key}" encountered')
        field, kind = _KEYS[key]
        setattr(pf, field, _value(field, kind, key, value))

    # Subface information: for each face a "face nSubfaces" line, then one line
    # per subface (src/InputParamClass.cpp:1481-1570).
    start = _find_block(lines, "subface information")
    if start is None:
        raise ParamFileError('Keyword "Subface information" not found')
    n = start
    for face in range(6):
        found = None
        while n < len(lines):
            ints = _leading_ints(lines[n], 1)
            n += 1
            if ints and ints[0] == face + 1:
                found = _leading_ints(lines[n - 1], 2)
                break
        if not found:
            raise ParamFileError(f"Subface information for face {face + 1} not found")
        subs = []
        for _ in range(found[1]):
            if n >= len(lines):
                raise ParamFileError("unexpected end of the subface information")
            parts = lines[n].split()
            n += 1
            if not parts or parts[0].lower() not in _ALL_BCS:
                raise ParamFileError(f'Unknown boundary condition "{parts[0] if parts else ""}"')
            try:
                own = tuple(int(v) for v in parts[1:7])
            except ValueError:
                raise ParamFileError(f"bad subface index range: {lines[n - 1]!r}") from None
            if len(own) != 6:
                raise ParamFileError(f"bad subface index range: {lines[n - 1]!r}")
            subs.append(Subface(parts[0], own, tuple(parts[7:])))
        pf.subfaces.append(subs)

    # Prescribed boundary data: "face subface nPoints names..." then nPoints lines.
    start = _find_block(lines, "prescribed boundary data")
    if start is not None:
        n = start
        while n < len(lines):
            ln = lines[n]
            n += 1
            ints = _leading_ints(ln.split("#", 1)[0], 3)
            if not ints:
                continue
            face, sub, npts = ints[0] - 1, ints[1] - 1, ints[2]
            names = ln.split("#", 1)[0].split()[3:]
            if not (0 <= face < 6 and 0 <= sub < len(pf.subfaces[face])):
                raise ParamFileError(f"prescribed data for a missing subface: {ln!r}")
            if npts != 1:
                raise UnsupportedOption("spatially varying prescribed boundary data")
            if n >= len(lines):
                raise ParamFileError("Unexpected end of the file while reading prescribed data")
            vals = lines[n].split()
            n += 1
            if len(vals) < len(names):
                raise ParamFileError("Something wrong while reading prescribed data")
            pf.prescribed[(face, sub)] = {nm: float(v) for nm, v in zip(names, vals)}

    # Sponge layer information: "face nElem dampingConstant dampingExponent".
    if pf.sponge_layer or pf.cml:
        start = _find_block(lines, "sponge layer information")
        if start is None:
            raise ParamFileError('Keyword "Sponge layer information" not found')
        rows, n = [], start
        for face in range(6):
            row = None
            while n < len(lines):
                ln = lines[n]
                n += 1
                ints = _leading_ints(ln, 1)
                if ints is None:
                    continue
                if ints[0] != face + 1:
                    raise ParamFileError(f"Sponge layer is not specified for face: {face + 1}")
                parts = ln.split()
                row = (int(parts[1]), float(parts[2]), float(parts[3]))
                if row[0] < 0:
                    raise ParamFileError("Sponge layer cannot have negative number of elements")
                break
            if row is None:
                raise ParamFileError(f"Sponge layer is not specified for face: {face + 1}")
            rows.append(row)
        pf.sponge = rows
    return pf


def read(path: str) -> ParamFile:
    with open(path) as f:
        pf = parse(f.read(), path)
    check_parameters(pf)
    return pf


def check_parameters(pf: ParamFile) -> None:
    """The consistency checks of InputParamClass::CheckParameters
    (src/InputParamClass.cpp:468-600) that concern the path."""
    def need(ok: bool, msg: str):
        if not ok:
            raise ParamFileError(msg)
    need(bool(pf.dof_location), '"Location of the DOFs" not specified in parameter file')
    need(bool(pf.fem_variables), '"FEM working variables" not specified in parameter file')
    need(bool(pf.riemann), '"Riemann solver" not specified in parameter file')
    need(0 < pf.p_grid <= 9, '"Polynomial degree grid" not or wrongly specified')
    need(0 < pf.p <= 9, '"Polynomial degree solution" not or wrongly specified')
    need(pf.n_poly_int > 0, '"Polynomial degree integration rule" not or wrongly specified')
    need(pf.n_poly_int >= 2 * pf.p, '"Polynomial degree integration rule" is too low')
    need(bool(pf.grid_file), '"Grid file name" not specified in parameter file')
    need(bool(pf.restart_file) or not pf.restart,
         '"Restart file name" not specified in parameter file')
    need(pf.n_sync > 0, '"Number of synchronization time steps" not or wrongly specified')
    need(pf.dt_sync > 0, '"Synchronization time step" not or wrongly specified')
    need(pf.cfl > 0, '"CFL number" not or wrongly specified')
    need(pf.penalty > 0, '"Relative penalty parameter" wrongly specified')
    need(pf.reference_area > 0, '"Reference area force coefficients" wrongly specified')
    if pf.box_lower is not None and pf.box_upper is not None:
        for d in range(3):
            need(pf.box_lower[d] < pf.box_upper[d],
                 f"Wrong {'xyz'[d]}-coordinates of the box for fluctuations")
    need(not pf.sponge_layer or bool(pf.averaged_file),
         '"Averaged solution file name" not specified in parameter file')
    pf.n_save = max(pf.n_save, 0)
    if pf.n_history <= 0:
        pf.n_history = 1


# ---------------------------------------------------------------------------
# Reference conditions and the free stream
# ---------------------------------------------------------------------------

@dataclasses.dataclass
class Reference:
    p_ref: float
    rho_ref: float
    u_ref: float
    mu_nondim: float
    free_stream: Tuple[float, float, float, float, float]   # dimensional rho, u, v, w, p


def _prescribed_values(pf: ParamFile) -> Dict[str, float]:
    """The last value of every prescribed variable over all subfaces, as the
    reference's loops leave them."""
    out: Dict[str, float] = {}
    for face in range(6):
        for sub in range(len(pf.subfaces[face])):
            out.update(pf.prescribed.get((face, sub), {}))
    return out


def reference_conditions(pf: ParamFile) -> Reference:
    """ComputeReferenceConditions and DetermineNonDimPrimVarFreeStream
    (src/InputParamClass.cpp:605-761, 991-1192), dimensional free stream."""
    pv = _prescribed_values(pf)
    get = lambda nm: pv.get(nm, -1.0)
    p, p_tot, rho, rho_tot = get("Pressure"), get("TotalPressure"), get("Density"), get("TotalDensity")
    T, T_tot = get("Temperature"), get("TotalTemperature")
    if abs(pf.mach) < 1.0e-10:
        raise UnsupportedOption("quiescent flow (Mach number 0)")
    p_ref = p if p > 0 else (p_tot if p_tot > 0 else -1.0)
    rho_ref = rho if rho > 0 else (rho_tot if rho_tot > 0 else -1.0)
    if rho_ref < 0 and p_ref > 0:
        t_ref = T if T > 0 else (T_tot if T_tot > 0 else -1.0)
        if t_ref > 0:
            rho_ref = p_ref / (R_GAS * t_ref)
    if pf.vel_dir is None:
        vel_dir = None
    else:
        n = math.sqrt(sum(c * c for c in pf.vel_dir))
        vel_dir = tuple(c / n for c in pf.vel_dir)
    if p_ref < 0 or rho_ref < 0:
        if pf.mach <= 0:
            raise ParamFileError('"Mach number" not or wrongly specified in parameter file')
        if pf.reynolds <= 0:
            raise ParamFileError('"Reynolds number" not or wrongly specified in parameter file')
        if pf.reynolds_length <= 0:
            raise ParamFileError('"Reynolds length" not or wrongly specified in parameter file')
        if pf.t_inf < 0:
            raise ParamFileError('"Free stream temperature" not or wrongly specified')
        if vel_dir is None:
            raise ParamFileError('"Free stream velocity direction" not or wrongly specified')
        v_inf = pf.mach * math.sqrt(GAMMA * R_GAS * pf.t_inf)
        rho_ref = pf.reynolds * MU_DIM / (pf.reynolds_length * v_inf)
        p_ref = rho_ref * R_GAS * pf.t_inf
    u_ref = math.sqrt(p_ref / rho_ref)
    mu_nondim = MU_DIM * u_ref / p_ref
    return Reference(p_ref, rho_ref, u_ref, mu_nondim,
                     _free_stream(pf, pv, p_ref, rho_ref, u_ref, mu_nondim, vel_dir))


def _free_stream(pf, pv, p_ref, rho_ref, u_ref, mu_nondim, vel_dir):
    big = 1.0e10
    get = lambda nm, d=-1.0: pv.get(nm, d)
    p, p_tot, rho, rho_tot = get("Pressure"), get("TotalPressure"), get("Density"), get("TotalDensity")
    T, T_tot = get("Temperature"), get("TotalTemperature")
    u, v, w = get("VelocityX", big), get("VelocityY", big), get("VelocityZ", big)
    ud, vd, wd = get("VelocityDirX", big), get("VelocityDirY", big), get("VelocityDirZ", big)
    if u < big and v < big and w < big:
        n_spec = (p > 0) + (rho > 0) + (T > 0)
        if n_spec >= 2:
            if p <= 0:
                p = rho * R_GAS * T
            if rho <= 0:
                rho = p / (R_GAS * T)
            return (rho, u, v, w, p)
        if n_spec == 1 and T <= 0:
            vel2 = u * u + v * v + w * w
            if p <= 0:
                p = 0.95 * rho * vel2 / GAMMA
            else:
                rho = GAMMA * p / (0.95 * vel2)
            return (rho, u, v, w, p)
    elif ud < big and vd < big and wd < big:
        n = math.sqrt(ud * ud + vd * vd + wd * wd)
        ud, vd, wd = ud / n, vd / n, wd / n
        gm1 = GAMMA - 1.0
        m2 = 0.95 * 0.95
        if p_tot > 0 and p > 0:
            m2 = ((p_tot / p) ** (gm1 / GAMMA) - 1.0) * 2.0 / gm1
        elif rho_tot > 0 and rho > 0:
            m2 = ((rho_tot / rho) ** (1.0 / GAMMA) - 1.0) * 2.0 / gm1
        elif T_tot > 0 and T > 0:
            m2 = (T_tot / T - 1.0) * 2.0 / gm1
        n_tot = (p_tot > 0) + (rho_tot > 0) + (T_tot > 0)
        if n_tot >= 2:
            if p_tot <= 0:
                p_tot = rho_tot * R_GAS * T_tot
            if rho_tot <= 0:
                rho_tot = p_tot / (R_GAS * T_tot)
            tmp = 1.0 + 0.5 * gm1 * m2
            p = p_tot / tmp ** (GAMMA / gm1)
            rho = rho_tot / tmp ** (1.0 / gm1)
            vel = math.sqrt(m2 * GAMMA * p / rho)
            return (rho, ud * vel, vd * vel, wd * vel, p)
    # From the free-stream parameters.
    if vel_dir is None:
        raise ParamFileError('"Free stream velocity direction" not or wrongly specified')
    v_inf = pf.mach * math.sqrt(GAMMA * R_GAS * pf.t_inf)
    mu_dim = mu_nondim * p_ref / u_ref
    rho_inf = pf.reynolds * mu_dim / (pf.reynolds_length * v_inf)
    p_inf = rho_inf * R_GAS * pf.t_inf
    return (rho_inf, v_inf * vel_dir[0], v_inf * vel_dir[1], v_inf * vel_dir[2], p_inf)


# ---------------------------------------------------------------------------
# What the GPU path runs
# ---------------------------------------------------------------------------

def check_supported(pf: ParamFile) -> None:
    """Raise UnsupportedOption for an option outside the path."""
    if pf.fem_variables != "entropy":
        raise UnsupportedOption("FEM working variables: Conservative")
    if pf.wall_model != "no wall model":
        raise UnsupportedOption(f"Wall modeling: {pf.wall_model}")
    if pf.fluctuations not in ("no fluctuations", "pressure pulse"):
        raise UnsupportedOption(f"Fluctuations to add to initial solution: {pf.fluctuations}")
    if pf.compute_average:
        raise UnsupportedOption("Compute average solution")
    for face, subs in enumerate(pf.subfaces):
        for sub in subs:
            if sub.kind not in _BC_TO_CASE:
                why = _WHY_NOT.get(sub.kind, sub.bc)
                raise UnsupportedOption(f"face {face + 1}: boundary condition {why}")
        if len(subs) > 1 and any(sub.kind == "periodic1to1trans" for sub in subs):
            raise UnsupportedOption(f"face {face + 1}: a periodic subface beside others "
                                    "(periodic connections cover whole faces here)")
    for d in range(3):
        a, b = pf.subfaces[2 * d][0].kind, pf.subfaces[2 * d + 1][0].kind
        if (a == "periodic1to1trans") != (b == "periodic1to1trans"):
            raise UnsupportedOption(f"direction {'ijk'[d]}: periodic on one face only")


def n_elements(pf: ParamFile) -> Tuple[int, int, int]:
    """Elements per direction from the subface ranges of the Max faces
    (the reference takes them from mSubfaces[1,3,5][0], SolverClass.cpp:4379-4381)."""
    return (pf.subfaces[1][0].own[0] - 1, pf.subfaces[3][0].own[2] - 1,
            pf.subfaces[5][0].own[4] - 1)


def case_bcs(pf: ParamFile) -> Tuple[str, ...]:
    """The condition of each block face (its first subface's)."""
    return tuple(_BC_TO_CASE[pf.subfaces[f][0].kind] for f in range(6))


def subface_data(pf: ParamFile, face: int, sub: int, bc: str) -> Tuple[float, ...]:
    """Prescribed data of one subface as the data tuple of a case subface."""
    if bc in ("outflow_nscbc", "outflow_subsonic"):
        return (outflow_pressure(pf, face, sub),)
    if bc == "inflow_static_nscbc":
        return inflow_static(pf, face, sub)
    if bc in ("inflow_total_nscbc", "inflow_subsonic"):
        return inflow_total(pf, face, sub)
    if bc in ("wall_heat_flux", "wall_isothermal"):
        return (wall_value(pf, face, sub),)
    if bc == "inflow_supersonic":
        return inflow_supersonic(pf, face, sub)
    return ()


def case_subfaces(pf: ParamFile):
    """Subfaces of the block faces that have more than one, as case subfaces
    (face, element range, condition, data): the node-index ranges of the file
    (1-based) give the elements [min - 1, max - 1) of each in-plane direction
    (SolverClass, src/SolverClass.cpp:1640-1660). None when every face has one."""
    out = []
    for face, subs in enumerate(pf.subfaces):
        if len(subs) < 2:
            continue
        d = face // 2
        a0, a1 = (1, 2) if d == 0 else ((0, 2) if d == 1 else (0, 1))
        for si, sub in enumerate(subs):
            lo = [min(sub.own[2 * a], sub.own[2 * a + 1]) - 1 for a in (a0, a1)]
            hi = [max(sub.own[2 * a], sub.own[2 * a + 1]) - 1 for a in (a0, a1)]
            bc = _BC_TO_CASE[sub.kind]
            out.append((face, (lo[0], hi[0], lo[1], hi[1]), bc, subface_data(pf, face, si, bc)))
    return tuple(out) if out else None


def outflow_pressure(pf: ParamFile, face: int, sub: int = 0) -> float:
    return _need(pf, face, ("Pressure",), pf.subfaces[face][sub].bc, sub)[0]


def _need(pf: ParamFile, face: int, names: Sequence[str], what: str,
          sub: int = 0) -> Tuple[float, ...]:
    data = pf.prescribed.get((face, sub), {})
    if not all(nm in data for nm in names):
        raise ParamFileError(f"face {face + 1} subface {sub + 1}: {what} needs the prescribed "
                             "data " + ", ".join(names))
    return tuple(data[nm] for nm in names)


def inflow_total(pf: ParamFile, face: int, sub: int = 0) -> Tuple[float, float, float, float, float]:
    """Total conditions of BCInflowTotalNSCBC or BCInflowSubsonic (the latter's
    density/velocity data set is not run: its boundary state uses the totals)."""
    return _need(pf, face, ("TotalPressure", "TotalTemperature", "VelocityDirX",
                            "VelocityDirY", "VelocityDirZ"), pf.subfaces[face][sub].bc, sub)


def wall_value(pf: ParamFile, face: int, sub: int = 0) -> float:
    kind = pf.subfaces[face][sub].kind
    name = "HeatFlux" if kind == "bcwallheatflux" else "Temperature"
    return _need(pf, face, (name,), pf.subfaces[face][sub].bc, sub)[0]


def inflow_supersonic(pf: ParamFile, face: int, sub: int = 0) -> Tuple[float, ...]:
    return _need(pf, face, ("Density", "VelocityX", "VelocityY", "VelocityZ", "Pressure"),
                 "BCInflowSupersonic", sub)


def inflow_static(pf: ParamFile, face: int, sub: int = 0) -> Tuple[float, float, float, float]:
    data = pf.prescribed.get((face, sub), {})
    names = ("Density", "VelocityX", "VelocityY", "VelocityZ")
    if not all(nm in data for nm in names):
        raise ParamFileError(f"face {face + 1}: BCInflowStaticNSCBC needs Density and "
                             "VelocityX/Y/Z")
    return tuple(data[nm] for nm in names)
