"""Host-side mirror of the reference solver's residual / time-step interface.

The reference drives its hot path through SolverClass
(include/SolverClass.hpp:40-124):

    solver.Residual(monitoringData, computeMonitoring)      -> Solver.residual
    solver.ExecuteTimeSynchronizationStep(monitoringData)   -> Solver.step
    ElementClass::ComputeTimeStep (min over elements)       -> Solver.time_step

Solver wraps one C-ABI handle (include/vcp3d_b200.h); every call goes through
the CUDA library. Discretization holds the host-side inputs (operators and
geometry) produced by vcpg_setup_geometry.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Optional

import numpy as np

from . import capi
from .cases import CaseData


@dataclasses.dataclass
class Discretization:
    n_elem: tuple
    n_poly: int
    n_int_1d: int
    leg_int: np.ndarray
    dleg_int: np.ndarray
    leg_face: np.ndarray
    dleg_face: np.ndarray
    w_int: np.ndarray
    leg_dofs: np.ndarray
    basis_center: np.ndarray
    vol_metric: np.ndarray      # [nE][10][M^3]
    face_metric: np.ndarray     # [nE][6][13][M^2]
    elem_scalars: np.ndarray    # [nE][15]
    neighbors: np.ndarray       # [nE][6] int32
    # With a subgrid-scale model: basis derivative at the nodal DOFs [K][K] and
    # the metric terms at the nodal DOFs [nE][10][K^3] (vcpg_setup_nodal_metrics).
    dleg_dofs: Optional[np.ndarray] = None
    vol_metric_dofs: Optional[np.ndarray] = None
    dof_location: int = 1          # enum vcpg_dof_location

    @property
    def n_elements(self) -> int:
        return int(np.prod(self.n_elem))


def make_params(case: CaseData, metric_compat: bool = True,
                precision: int = capi.FP64) -> capi.Params:
    s, r = case.spec, case.ref
    p = capi.Params()
    p.n_elem[:] = list(s.n_elem)
    p.n_poly = s.p
    p.n_int_1d = s.n_poly_int // 2 + 1
    p.riemann = capi.ISMAIL_ROE if s.riemann.lower() == "ismailroe" else capi.ROE
    p.metric_index_compat = 1 if metric_compat else 0
    p.precision = precision
    p.theta_sym = s.theta_sym
    p.rel_penalty = s.penalty
    p.cfl = s.cfl
    p.mu = r.mu_nondim
    p.p_ref, p.u_ref, p.rho_ref = r.p_ref, r.u_ref, r.rho_ref
    p.sgs_model = SGS_CODES[s.sgs.lower()]
    # The reference monitors forces only where wall faces exist
    # (src/InputParamClass.cpp:1574-1575).
    walls = any(b.startswith("wall_") for b in s.bc) or any(
        e[2].startswith("wall_") for e in (s.subfaces or ()))
    p.monitor_forces = 1 if (s.monitor_forces and walls) else 0
    p.mach, p.ref_area = s.mach, s.ref_area
    if s.body_force is not None:
        p.body_force[:] = [float(v) for v in s.body_force]
    return p


SGS_CODES = {"none": capi.SGS_NONE, "wale": capi.SGS_WALE, "vreman": capi.SGS_VREMAN}


def setup_discretization(case: CaseData, params: capi.Params,
                         periodic=None, device: bool = False) -> Discretization:
    """Operators and metric terms from the case grid: host C++ in the library
    (vcpg_setup_geometry) or, with device=True, the same arithmetic on the GPU
    (vcpg_setup_geometry_device). periodic defaults to the case's periodic
    directions."""
    if periodic is None:
        periodic = case.spec.periodic
    lib = capi.load()
    s = case.spec
    K, M, nE = s.p + 1, params.n_int_1d, s.n_elements
    d = Discretization(
        n_elem=tuple(s.n_elem), n_poly=s.p, n_int_1d=M,
        leg_int=np.zeros((K, M)), dleg_int=np.zeros((K, M)), leg_face=np.zeros((2, K)),
        dleg_face=np.zeros((2, K)), w_int=np.zeros(M), leg_dofs=np.zeros((K, K)),
        basis_center=np.zeros(K ** 3), vol_metric=np.zeros((nE, 10, M ** 3)),
        face_metric=np.zeros((nE, 6, 13, M * M)), elem_scalars=np.zeros((nE, 15)),
        neighbors=np.zeros((nE, 6), dtype=np.int32))
    per = np.asarray(periodic, dtype=np.int32)
    nodes = np.ascontiguousarray(case.elem_nodes, dtype=np.float64)
    from .cases import dof_location_code
    d.dof_location = dof_location_code(s)
    setup = lib.vcpg_setup_geometry_device if device else lib.vcpg_setup_geometry
    rc = setup(
        C.byref(params), s.p_grid, d.dof_location, capi.ptr(per), capi.ptr(nodes), capi.ptr(d.leg_int),
        capi.ptr(d.dleg_int), capi.ptr(d.leg_face), capi.ptr(d.dleg_face), capi.ptr(d.w_int),
        capi.ptr(d.leg_dofs), capi.ptr(d.basis_center), capi.ptr(d.vol_metric),
        capi.ptr(d.face_metric), capi.ptr(d.elem_scalars), capi.ptr(d.neighbors))
    if rc != capi.VCPG_OK:
        raise capi.VcpgError(rc, ("vcpg_setup_geometry_device" if device else
                                  "vcpg_setup_geometry") + " failed")
    if params.sgs_model != capi.SGS_NONE:
        d.dleg_dofs = np.zeros((K, K))
        d.vol_metric_dofs = np.zeros((nE, 10, K ** 3))
        rc = lib.vcpg_setup_nodal_metrics(C.byref(params), s.p_grid, d.dof_location, capi.ptr(nodes),
                                          capi.ptr(d.dleg_dofs), capi.ptr(d.vol_metric_dofs))
        if rc != capi.VCPG_OK:
            raise capi.VcpgError(rc, "vcpg_setup_nodal_metrics failed")
    return d


def nodal_to_modal(case: CaseData, params: capi.Params) -> np.ndarray:
    """Initial modal entropy-variable state from the case's nodal conservative state."""
    lib = capi.load()
    cons = np.ascontiguousarray(case.cons, dtype=np.float64)
    out = np.zeros_like(cons)
    from .cases import dof_location_code
    vinv = None
    if dof_location_code(case.spec) not in (1, 3):   # equidistant solution DOFs
        K = params.n_poly + 1
        vinv = np.zeros((K, K))
        rc = lib.vcpg_vandermonde_inverse(params.n_poly, dof_location_code(case.spec),
                                          capi.ptr(vinv))
        if rc != capi.VCPG_OK:
            raise capi.VcpgError(rc, "vcpg_vandermonde_inverse failed")
    rc = lib.vcpg_nodal_conservative_to_modal(C.byref(params), capi.ptr(vinv), capi.ptr(cons),
                                              capi.ptr(out), cons.shape[0])
    if rc != capi.VCPG_OK:
        raise capi.VcpgError(rc, "vcpg_nodal_conservative_to_modal failed")
    return out


BC_CODES = {"periodic": capi.BC_NONE, "outflow_nscbc": capi.BC_OUTFLOW_NSCBC,
            "inflow_static_nscbc": capi.BC_INFLOW_STATIC_NSCBC,
            "inflow_total_nscbc": capi.BC_INFLOW_TOTAL_NSCBC,
            "wall_heat_flux": capi.BC_WALL_HEAT_FLUX, "wall_isothermal": capi.BC_WALL_ISOTHERMAL,
            "wall_inviscid": capi.BC_WALL_INVISCID, "farfield": capi.BC_FARFIELD,
            "inflow_subsonic": capi.BC_INFLOW_SUBSONIC,
            "inflow_supersonic": capi.BC_INFLOW_SUPERSONIC,
            "outflow_subsonic": capi.BC_OUTFLOW_SUBSONIC,
            "outflow_supersonic": capi.BC_OUTFLOW_SUPERSONIC}


def _face_data(s, f: int, bc: str, p_out, rho_in, vel_in):
    """Prescribed data of condition bc on block face f (dimensional): outflow
    pressure, static inflow (rho, u, v, w), total inflow, wall value, supersonic
    inflow state."""
    from .cases import total_inflow_values
    po = s.prescribed_p[f] if s.prescribed_p else p_out
    inflow = tuple(s.prescribed_inflow[f]) if s.prescribed_inflow else (rho_in, *vel_in)
    total = ((s.prescribed_total[f] if s.prescribed_total else total_inflow_values(s))
             if bc in ("inflow_total_nscbc", "inflow_subsonic") else (0.0,) * 5)
    wall = ((s.wall_data[f] if s.wall_data else (0.0 if bc == "wall_heat_flux" else s.t_inf))
            if bc in ("wall_heat_flux", "wall_isothermal") else 0.0)
    sup = ((s.prescribed_super[f] if s.prescribed_super else (rho_in, *vel_in, p_out))
           if bc == "inflow_supersonic" else (0.0,) * 5)
    return po, inflow, total, wall, sup


def open_boundary(case: CaseData) -> capi.OpenBoundary:
    """vcpg_open_boundary of a case: its boundary conditions with the free stream
    as prescribed data, NSCBC tuning parameters, sponge layers and matching layer."""
    from .cases import free_stream_values, prescribed_values
    s, ref = case.spec, case.ref
    ob = capi.OpenBoundary()
    p_out, rho_in, vel_in = prescribed_values(s, ref)
    per_face = lambda v, f: v[f] if isinstance(v, (tuple, list)) else v
    for f, bc in enumerate(s.bc):
        ob.bc[f] = BC_CODES[bc]
        po, inflow, total, wall, sup = _face_data(s, f, bc, p_out, rho_in, vel_in)
        ob.p_out[f] = po
        ob.inflow[f][0], ob.inflow[f][1], ob.inflow[f][2], ob.inflow[f][3] = inflow
        for q in range(5):
            ob.inflow_total[f][q] = total[q]
            ob.inflow_super[f][q] = sup[q]
        ob.wall_data[f] = wall
        ob.sponge_elems[f] = s.sponge[f]
        ob.sponge_sigma[f] = per_face(s.sponge_sigma, f)
        ob.sponge_alpha[f] = per_face(s.sponge_alpha, f)
    ob.outlet_len, ob.outlet_sigma = s.outlet_len, s.outlet_sigma
    ob.outlet_beta_l, ob.outlet_beta_t = s.outlet_beta_l, s.outlet_beta_t
    ob.outlet_one_minus_beta = 1 if s.outlet_one_minus_beta else 0
    ob.inlet_len, ob.inlet_sigma = s.inlet_len, s.inlet_sigma
    ob.inlet_incoming = 1 if s.inlet_incoming else 0
    ob.cml = 1 if s.cml else 0
    ob.outlet_local_mach = 1 if s.outlet_local_mach else 0
    ob.sponge_state[:] = (list(s.sponge_state) if s.sponge_state else
                          [rho_in, vel_in[0], vel_in[1], vel_in[2], p_out])
    ob.free_stream[:] = list(s.free_stream if s.free_stream else free_stream_values(s))
    return ob


def subfaces(case: CaseData):
    """vcpg_subface array of a case with several subfaces per block face (None
    without): each subface with its condition and its block face's data."""
    from .cases import prescribed_values
    s = case.spec
    if not s.subfaces:
        return None
    p_out, rho_in, vel_in = prescribed_values(s, case.ref)
    arr = (capi.Subface * len(s.subfaces))()
    for i, (f, (b0, e0, b1, e1), bc, dat) in enumerate(s.subfaces):
        sf = arr[i]
        sf.face, sf.bc = f, BC_CODES[bc]
        sf.elem_begin[0], sf.elem_end[0], sf.elem_begin[1], sf.elem_end[1] = b0, e0, b1, e1
        po, inflow, total, wall, sup = _face_data(s, f, bc, p_out, rho_in, vel_in)
        if dat is not None:       # the subface's own prescribed data
            if bc in ("outflow_nscbc", "outflow_subsonic"):
                po = dat[0]
            elif bc == "inflow_static_nscbc":
                inflow = tuple(dat)
            elif bc in ("inflow_total_nscbc", "inflow_subsonic"):
                total = tuple(dat)
            elif bc in ("wall_heat_flux", "wall_isothermal"):
                wall = dat[0]
            elif bc == "inflow_supersonic":
                sup = tuple(dat)
        sf.p_out, sf.wall_data = po, wall
        sf.inflow[:] = list(inflow)
        sf.inflow_total[:] = list(total)
        sf.inflow_super[:] = list(sup)
    return arr


class Solver:
    """One GPU-resident case. All work runs in the CUDA library."""

    def __init__(self, params: capi.Params, disc: Discretization):
        self.lib = capi.load()
        self.params = params
        self.disc = disc
        self._keep = [np.ascontiguousarray(a) for a in (
            disc.leg_int, disc.dleg_int, disc.leg_face, disc.dleg_face, disc.w_int,
            disc.leg_dofs, disc.basis_center, disc.vol_metric, disc.face_metric,
            disc.elem_scalars)]
        nbr = np.ascontiguousarray(disc.neighbors, dtype=np.int32)
        self._keep.append(nbr)
        nodal = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                 for a in (disc.dleg_dofs, disc.vol_metric_dofs)]
        self._keep_nodal = nodal
        ops = capi.Operators(*[capi.ptr(a) for a in self._keep[:7]], capi.ptr(nodal[0]))
        geom = capi.Geometry(capi.ptr(self._keep[7]), capi.ptr(self._keep[8]),
                             capi.ptr(self._keep[9]), capi.ptr(nbr), capi.ptr(nodal[1]))
        h = C.c_void_p()
        rc = self.lib.vcpg_create(C.byref(params), C.byref(ops), C.byref(geom), C.byref(h))
        self.h = h
        if rc != capi.VCPG_OK:
            msg = self.lib.vcpg_last_error(h).decode() if h.value else "create failed"
            self.close()
            raise capi.VcpgError(rc, msg)
        K = params.n_poly + 1
        self.shape = (disc.n_elements, 5, K ** 3)

    def set_open_boundary(self, case: CaseData):
        """Characteristic boundaries, sponge and matching layers of an open case."""
        ob = open_boundary(case)
        self._keep_ob = (ob, np.ascontiguousarray(case.elem_nodes, dtype=np.float64))
        geom = capi.Geometry(capi.ptr(self._keep[7]), capi.ptr(self._keep[8]),
                             capi.ptr(self._keep[9]), capi.ptr(self._keep[10]))
        sfs = subfaces(case)
        self._keep_sf = sfs
        self._check(self.lib.vcpg_set_open_boundary_subfaces(
            self.h, C.byref(ob), sfs, len(sfs) if sfs is not None else 0, C.byref(geom),
            case.spec.p_grid, self.disc.dof_location, capi.ptr(self._keep_ob[1])),
            "set_open_boundary")

    def _check(self, rc: int, what: str):
        if rc != capi.VCPG_OK:
            raise capi.VcpgError(rc, f"{what}: {self.lib.vcpg_last_error(self.h).decode()}")

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.vcpg_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, modal: np.ndarray):
        a = np.ascontiguousarray(modal, dtype=np.float64).reshape(self.shape)
        self._check(self.lib.vcpg_set_state(self.h, capi.ptr(a)), "set_state")

    def get_state(self) -> np.ndarray:
        out = np.empty(self.shape)
        self._check(self.lib.vcpg_get_state(self.h, capi.ptr(out)), "get_state")
        return out

    def residual(self, monitoring: bool = False, keep_raw: bool = False):
        mon = np.zeros(8) if monitoring else None
        self._check(self.lib.vcpg_residual(self.h, capi.ptr(mon), 1 if keep_raw else 0),
                    "residual")
        return mon

    def get_state_into(self, out: np.ndarray):
        """Copies the device state into a caller-provided (e.g. pinned) array."""
        assert out.dtype == np.float64 and out.flags["C_CONTIGUOUS"] and out.size == np.prod(self.shape)
        self._check(self.lib.vcpg_get_state(self.h, capi.ptr(out)), "get_state")

    def get_residual(self) -> np.ndarray:
        out = np.empty(self.shape)
        self._check(self.lib.vcpg_get_residual(self.h, capi.ptr(out)), "get_residual")
        return out

    def get_raw_residual(self) -> np.ndarray:
        out = np.empty(self.shape)
        self._check(self.lib.vcpg_get_raw_residual(self.h, capi.ptr(out)), "get_raw_residual")
        return out

    def time_step(self) -> float:
        dt = C.c_double()
        self._check(self.lib.vcpg_time_step(self.h, C.byref(dt)), "time_step")
        return dt.value

    def step(self, n_steps: int, scheme: int = capi.SSPRK3,
             fixed_dt: float = -1.0) -> np.ndarray:
        hist = np.zeros(max(n_steps, 1))
        self._check(self.lib.vcpg_step(self.h, scheme, n_steps, fixed_dt, capi.ptr(hist)), "step")
        return hist[:n_steps]

    def synchronization_step(self, dt_sync: float, max_steps: int = 1000000,
                             monitoring: bool = False):
        """SolverClass::ExecuteTimeSynchronizationStep: SSP-RK3 CFL steps that end
        exactly on the non-dimensional synchronisation time dt_sync. Returns the
        number of RK steps and, with monitoring, the 8 monitoring values."""
        n = C.c_int32(0)
        mon = np.zeros(8)
        self._check(self.lib.vcpg_synchronization_step(
            self.h, float(dt_sync), int(max_steps), C.byref(n),
            capi.ptr(mon) if monitoring else None), "synchronization step")
        return (int(n.value), mon) if monitoring else int(n.value)

    def sync(self):
        self._check(self.lib.vcpg_sync(self.h), "sync")

    # A block split across GPUs (vcp3d_open_b200.partition).
    def set_partition(self, n_owned: int, n_face_ghost: int):
        self._check(self.lib.vcpg_set_partition(self.h, int(n_owned), int(n_face_ghost)),
                    "set_partition")

    def pack_states(self, first: int, count: int, d_buf: int):
        """States of elements [first, first + count) into the device buffer d_buf."""
        self._check(self.lib.vcpg_pack_states(self.h, int(first), int(count), C.c_void_p(d_buf)),
                    "pack_states")

    def unpack_states(self, first: int, count: int, d_buf: int):
        self._check(self.lib.vcpg_unpack_states(self.h, int(first), int(count),
                                                C.c_void_p(d_buf)), "unpack_states")

    def set_partition_parts(self, flux_ready: int, res_ready: int):
        self._check(self.lib.vcpg_set_partition_parts(self.h, int(flux_ready), int(res_ready)),
                    "set_partition_parts")

    def set_send_list(self, lst: int, elems):
        a = np.ascontiguousarray(elems, dtype=np.int32)
        self._check(self.lib.vcpg_set_send_list(self.h, int(lst),
                                                a.ctypes.data_as(C.POINTER(C.c_int32)), len(a)),
                    "set_send_list")

    def pack_send_list(self, lst: int, d_buf: int):
        """States of send list lst's elements, in list order, into the device buffer d_buf."""
        self._check(self.lib.vcpg_pack_send_list(self.h, int(lst), C.c_void_p(d_buf)),
                    "pack_send_list")

    def rk_stage(self, scheme: int, stage: int, dt: float):
        self._check(self.lib.vcpg_rk_stage(self.h, int(scheme), int(stage), float(dt)),
                    "rk_stage")

    @property
    def stream(self) -> int:
        return self.lib.vcpg_stream(self.h)

    def cg_stats(self):
        """(total CG iterations, element solves) since creation."""
        it, n = C.c_int64(), C.c_int64()
        self._check(self.lib.vcpg_stats(self.h, C.byref(it), C.byref(n)), "stats")
        return it.value, n.value

    def time_residual_kernels(self, reps: int = 10):
        """Average ms per launch of the residual's kernels, each between CUDA events
        on the library stream: (boundary kernels, FaceFluxKernel, ResidualKernel)."""
        ms = np.zeros(3)
        self._check(self.lib.vcpg_time_residual_kernels(self.h, reps, capi.ptr(ms)),
                    "time_residual_kernels")
        return tuple(float(x) for x in ms)

    @property
    def launch_count(self) -> int:
        return int(self.lib.vcpg_launch_count(self.h))


def create(case: CaseData, metric_compat: bool = True, precision: int = capi.FP64,
           disc: Optional[Discretization] = None, device_setup: bool = False) -> Solver:
    """Set-up + handle + initial state for a generated case (device_setup: the
    metric terms computed on the GPU).

    precision: capi.FP64 (the reference's arithmetic) or capi.MIXED (residual in
    FP32, state and time integration in FP64). A Discretization of the same case
    may be passed to share the host-side set-up between handles."""
    params = make_params(case, metric_compat=metric_compat, precision=precision)
    if disc is None:
        disc = setup_discretization(case, params, device=device_setup)
    s = Solver(params, disc)
    if case.spec.is_open:
        s.set_open_boundary(case)
    s.set_state(nodal_to_modal(case, params))
    return s
