"""Served ensemble: a request loop with continuous batching over the library's
GPU-resident ensemble (include/vcp3d_b200.h, vcpg_ensemble_*).

Requests (cases of differing element counts and degrees) arrive over time.
Each is prepared on the host (grid, metrics, initial state: client-side work,
run on a thread pool as requests arrive), then admitted by its HBM footprint
when its degree bucket has room, stepped together with every other resident
case of that degree (one fused launch per kernel and step, a CUDA graph per
bucket, buckets overlapping on their own streams), and retired when it has
taken its steps, which frees room for waiting requests. Reported: p50/p99
time-to-completion (arrival -> result on the host) beside the aggregate
DOF-updates/s.

    python -m vcp3d_open_b200.serving [--cases 256] [--steps 300] [--precision mixed]
    python -m vcp3d_open_b200.serving --cases 128 --offered-load 0.5,0.8,0.95

Several GPUs (one process each, torchrun): every rank serves every world-th
request of the stream on its own GPU, the cases being independent, and rank 0
prints one report for the job (summed DOF-updates over the longest rank's wall
time, percentiles over all requests):

    torchrun --nproc-per-node N --master-addr 127.0.0.1 -m vcp3d_open_b200.serving
"""
from __future__ import annotations

import argparse
import collections
import concurrent.futures as cf
import ctypes as C
import dataclasses
import json
import os
import sys
import time
from typing import Dict, List, Optional

import numpy as np

from . import capi, cases, solver

# ---------------------------------------------------------------------------
# Requests
# ---------------------------------------------------------------------------


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float            # seconds after the start of the stream
    spec: cases.CaseSpec
    steps: int


def vortex_spec(n: int, p: int, mach: float, beta: float, name: str) -> cases.CaseSpec:
    """Isentropic vortex on the periodic curvilinear cube [0, 10]^3, n^3 elements."""
    return cases.CaseSpec(name=name, kind="vortex", n_elem=(n, n, n), p=p, mach=mach, beta=beta)


def pulse_spec(n: int, p: int, mach: float, name: str) -> cases.CaseSpec:
    """The open-boundary pulse configuration scaled to n^3 elements of size 0.5:
    static-inflow and outflow PC-NSCBC, sponge layers with the matching layer on
    i-max and both j faces (n // 10 elements, at least one), k periodic."""
    L = 0.5 * n
    ns = max(1, n // 10)
    return cases.CaseSpec(name=name, kind="pulse", n_elem=(n, n, n), p=p, hi=(L, L, L),
                          mach=mach, grid_map="none", center=(0.5 * L,) * 3, pulse_amp=1.0e-3,
                          pulse_width=0.5,
                          bc=("inflow_static_nscbc", "outflow_nscbc", "outflow_nscbc",
                              "outflow_nscbc", "periodic", "periodic"),
                          sponge=(0, ns, ns, ns, 0, 0), cml=True)


def request_stream(n_cases: int = 256, seed: int = 7, mean_interarrival: float = 0.020,
                   steps: int = 300, n_range=(8, 24), degrees=(2, 3, 4, 5),
                   mach_range=(0.2, 0.6), beta_range=(2.0, 6.0)) -> List[Request]:
    """Seeded Poisson arrivals of isentropic-vortex and acoustic-pulse cases:
    elements n^3 with n ~ U{8..24}, degree ~ U{2,3,4,5}, Mach ~ U[0.2, 0.6],
    vortex strength ~ U[2, 6]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_cases):
        t += rng.exponential(mean_interarrival)
        kind = "vortex" if rng.integers(0, 2) == 0 else "pulse"
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        p = int(rng.choice(degrees))
        mach = float(rng.uniform(*mach_range))
        beta = float(rng.uniform(*beta_range))
        name = f"{kind}{i}_n{n}_p{p}"
        spec = vortex_spec(n, p, mach, beta, name) if kind == "vortex" else pulse_spec(n, p, mach, name)
        out.append(Request(i, t, spec, steps))
    return out


# ---------------------------------------------------------------------------
# Host preparation of one case
# ---------------------------------------------------------------------------


@dataclasses.dataclass
class PreparedCase:
    spec: cases.CaseSpec
    params: capi.Params
    disc: solver.Discretization
    modal: np.ndarray
    ob: Optional[capi.OpenBoundary]
    grid_nodes: Optional[np.ndarray]
    n_bfaces: int
    n_sponge: int
    subfaces: Optional[object] = None   # vcpg_subface array (several per block face)

    @property
    def n_dofs(self) -> int:
        return self.spec.n_dofs


def prepare(spec: cases.CaseSpec, precision: int) -> PreparedCase:
    case = cases.build_case(spec)
    params = solver.make_params(case, metric_compat=True, precision=precision)
    disc = solver.setup_discretization(case, params)
    modal = np.ascontiguousarray(solver.nodal_to_modal(case, params))
    ob, nodes, nb, ns, sfs = None, None, 0, 0, None
    if spec.is_open:
        ob = solver.open_boundary(case)
        sfs = solver.subfaces(case)
        nodes = np.ascontiguousarray(case.elem_nodes, dtype=np.float64)
        nbr = disc.neighbors
        nb = int(sum(np.count_nonzero(nbr[:, f] < 0) for f in range(6) if spec.bc[f] != "periodic"))
        ns = _sponge_elements(spec)
    return PreparedCase(spec, params, disc, modal, ob, nodes, nb, ns, sfs)


def _sponge_elements(spec: cases.CaseSpec) -> int:
    n = spec.n_elem
    idx = np.indices((n[2], n[1], n[0]))  # k, j, i
    ijk = (idx[2], idx[1], idx[0])
    mask = np.zeros(idx.shape[1:], dtype=bool)
    for d in range(3):
        if spec.sponge[2 * d]:
            mask |= ijk[d] < spec.sponge[2 * d]
        if spec.sponge[2 * d + 1]:
            mask |= ijk[d] >= n[d] - spec.sponge[2 * d + 1]
    return int(mask.sum())


# ---------------------------------------------------------------------------
# The ensemble (C ABI wrapper)
# ---------------------------------------------------------------------------


class Ensemble:
    def __init__(self, capacities: Dict[int, tuple], precision: int = capi.MIXED,
                 scheme: int = capi.LSRK4, max_cases: int = 256, riemann: int = capi.ISMAIL_ROE,
                 theta_sym: float = 1.0, rel_penalty: float = 1.0):
        """capacities: degree -> (elements, boundary faces, sponge elements)."""
        self.lib = capi.load()
        cfg = capi.EnsembleConfig()
        cfg.precision, cfg.scheme, cfg.riemann = precision, scheme, riemann
        cfg.metric_index_compat = 1
        cfg.theta_sym, cfg.rel_penalty = theta_sym, rel_penalty
        for p, (ne, nb, ns) in capacities.items():
            cfg.bucket_elems[p], cfg.bucket_bfaces[p], cfg.bucket_sponge[p] = ne, nb, ns
        cfg.max_cases = max_cases
        self.cfg = cfg
        self.max_cases = max_cases
        self.precision, self.scheme = precision, scheme
        h = C.c_void_p()
        rc = self.lib.vcpg_ensemble_create(C.byref(cfg), C.byref(h))
        self.h = h
        if rc != capi.VCPG_OK:
            msg = self.lib.vcpg_ensemble_last_error(h).decode() if h.value else "create failed"
            self.close()
            raise capi.VcpgError(rc, msg)
        self._keep: Dict[int, tuple] = {}

    def _err(self) -> str:
        return self.lib.vcpg_ensemble_last_error(self.h).decode()

    def submit(self, pc: PreparedCase, n_steps: int) -> Optional[int]:
        """Admits a case; None when its bucket has no room now (VCPG_E_ADMISSION)."""
        d = pc.disc
        arrs = [np.ascontiguousarray(a) for a in (d.leg_int, d.dleg_int, d.leg_face, d.dleg_face,
                                                  d.w_int, d.leg_dofs, d.basis_center,
                                                  d.vol_metric, d.face_metric, d.elem_scalars)]
        nbr = np.ascontiguousarray(d.neighbors, dtype=np.int32)
        ops = capi.Operators(*[capi.ptr(a) for a in arrs[:7]])
        geom = capi.Geometry(capi.ptr(arrs[7]), capi.ptr(arrs[8]), capi.ptr(arrs[9]), capi.ptr(nbr))
        cid = C.c_int64()
        ob = C.byref(pc.ob) if pc.ob is not None else None
        if pc.subfaces is not None:
            rc = self.lib.vcpg_ensemble_submit_subfaces(
                self.h, C.byref(pc.params), C.byref(ops), C.byref(geom), capi.ptr(pc.modal),
                n_steps, ob, pc.subfaces, len(pc.subfaces), pc.spec.p_grid,
                cases.dof_location_code(pc.spec), capi.ptr(pc.grid_nodes), C.byref(cid))
        else:
            rc = self.lib.vcpg_ensemble_submit(self.h, C.byref(pc.params), C.byref(ops),
                                               C.byref(geom), capi.ptr(pc.modal), n_steps, ob,
                                               pc.spec.p_grid, cases.dof_location_code(pc.spec),
                                               capi.ptr(pc.grid_nodes), C.byref(cid))
        if rc == 7:   # VCPG_E_ADMISSION
            return None
        if rc != capi.VCPG_OK:
            raise capi.VcpgError(rc, self._err())
        self._keep[cid.value] = (pc.modal.shape,)
        return cid.value

    def step(self):
        rc = self.lib.vcpg_ensemble_step(self.h)
        if rc != capi.VCPG_OK:
            raise capi.VcpgError(rc, self._err())

    def poll(self, max_ids: int = 1024) -> List[int]:
        ids = (C.c_int64 * max_ids)()
        n = C.c_int32()
        rc = self.lib.vcpg_ensemble_poll(self.h, ids, max_ids, C.byref(n))
        if rc != capi.VCPG_OK:
            raise capi.VcpgError(rc, self._err())
        return [ids[i] for i in range(n.value)]

    def retire(self, cid: int):
        shape = self._keep.pop(cid)[0]
        out = np.empty(shape)
        t = C.c_double()
        rc = self.lib.vcpg_ensemble_retire(self.h, cid, capi.ptr(out), C.byref(t))
        if rc != capi.VCPG_OK:
            raise capi.VcpgError(rc, self._err())
        return out, t.value

    def sync(self):
        rc = self.lib.vcpg_ensemble_sync(self.h)
        if rc != capi.VCPG_OK:
            raise capi.VcpgError(rc, self._err())

    def stats(self):
        r, n = C.c_int32(), C.c_int64()
        self.lib.vcpg_ensemble_stats(self.h, C.byref(r), C.byref(n))
        return r.value, n.value

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.vcpg_ensemble_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def footprint(spec: cases.CaseSpec, n_bfaces: int = 0, n_sponge: int = 0) -> int:
    lib = capi.load()
    M = spec.n_poly_int // 2 + 1
    return int(lib.vcpg_ensemble_footprint(spec.p, M, spec.n_elements, n_bfaces, n_sponge))


def case_sizes(spec: cases.CaseSpec):
    """(elements, characteristic boundary faces, sponge elements) of a case."""
    n = spec.n_elem
    face_elems = (n[1] * n[2], n[1] * n[2], n[0] * n[2], n[0] * n[2], n[0] * n[1], n[0] * n[1])
    nb = sum(face_elems[f] for f in range(6) if spec.bc[f] != "periodic")
    ns = _sponge_elements(spec) if any(spec.sponge) else 0
    return spec.n_elements, nb, ns


def plan_capacities(requests: List[Request], budget_bytes: int) -> Dict[int, tuple]:
    """Per-degree bucket capacities (elements, boundary faces, sponge elements):
    every degree gets the same fraction of its requests' total demand -- the
    budget over the total footprint, at most one (all resident at once) -- and
    at least its largest case."""
    demand: Dict[int, list] = collections.defaultdict(list)
    for r in requests:
        demand[r.spec.p].append(case_sizes(r.spec) + (footprint(r.spec, *case_sizes(r.spec)[1:]),))
    total = sum(c[3] for v in demand.values() for c in v)
    frac = min(1.0, budget_bytes / max(total, 1))
    caps = {}
    for p, v in demand.items():
        arr = np.array(v, dtype=np.int64)
        caps[p] = tuple(int(max(arr[:, k].max(), np.ceil(frac * arr[:, k].sum()))) for k in range(3))
    return caps


# ---------------------------------------------------------------------------
# The request loop
# ---------------------------------------------------------------------------


def serve(requests: List[Request], ens: Ensemble, prepare_workers: int = 8,
          keep_results: bool = False, progress_every: float = 0.0,
          keep_latencies: bool = False) -> dict:
    """Continuous batching: admit arrived requests whenever their bucket has room,
    step every bucket with resident cases, retire finished cases."""
    t0 = time.perf_counter()
    pool = cf.ThreadPoolExecutor(max_workers=prepare_workers)
    future_of = {}
    upcoming = collections.deque(sorted(requests, key=lambda r: r.arrival))
    waiting: List[Request] = []         # arrived (preparing or prepared), not admitted
    running: Dict[int, Request] = {}    # case id -> request
    admitted_at, finished_at, results = {}, {}, {}
    dof_updates = 0
    steps = 0
    next_report = progress_every
    slots = collections.Counter()       # resident cases per degree bucket
    max_slots = getattr(ens, "max_cases", None)
    while upcoming or waiting or running:
        now = time.perf_counter() - t0
        if progress_every and now >= next_report:
            next_report += progress_every
            print(f"[serve] t={now:.1f}s finished={len(finished_at)} running={len(running)} "
                  f"waiting={len(waiting)} upcoming={len(upcoming)} steps={steps}",
                  file=sys.stderr, flush=True)
        while upcoming and upcoming[0].arrival <= now:
            r = upcoming.popleft()
            future_of[r.rid] = pool.submit(prepare, r.spec, ens.precision)
            waiting.append(r)
        # Admission in arrival order; a request that does not fit does not block
        # smaller later ones of other degrees.
        still = []
        for r in waiting:
            fut = future_of[r.rid]
            if not fut.done() or (max_slots and slots[r.spec.p] >= max_slots):
                still.append(r)
                continue
            cid = ens.submit(fut.result(), r.steps)
            if cid is None:
                still.append(r)
                continue
            slots[r.spec.p] += 1
            running[cid] = r
            admitted_at[r.rid] = time.perf_counter() - t0
            del future_of[r.rid]
        waiting = still
        if running:
            ens.step()
            steps += 1
        elif upcoming and not waiting:
            time.sleep(max(0.0, min(0.01, upcoming[0].arrival - (time.perf_counter() - t0))))
        elif waiting:
            time.sleep(0.001)
        for cid in ens.poll():
            r = running.pop(cid)
            slots[r.spec.p] -= 1
            state, sim_time = ens.retire(cid)
            finished_at[r.rid] = time.perf_counter() - t0
            dof_updates += r.spec.n_dofs * r.steps
            if keep_results:
                results[r.rid] = (state, sim_time)
    ens.sync()
    pool.shutdown()
    wall = time.perf_counter() - t0
    lat = np.array([finished_at[r.rid] - r.arrival for r in requests])
    qwait = np.array([admitted_at[r.rid] - r.arrival for r in requests])
    out = {
        "cases": len(requests), "wall_seconds": wall, "dof_updates": float(dof_updates),
        "dof_updates_per_s": dof_updates / wall,
        "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
        "latency_max_s": float(lat.max()),
        "admission_wait_p50_s": float(np.percentile(qwait, 50)),
        "admission_wait_p99_s": float(np.percentile(qwait, 99)),
        "loop_iterations_with_steps": steps,
    }
    if keep_results:
        out["results"] = results
    if keep_latencies:
        out["latency_s"] = lat.tolist()
        out["admission_wait_s"] = qwait.tolist()
    return out


def shard_requests(requests: List[Request], rank: int, world: int) -> List[Request]:
    """The requests rank serves when world GPUs share the stream: every world-th
    request in arrival order, starting at rank (the cases are independent, so the
    ranks exchange nothing while they serve)."""
    ordered = sorted(requests, key=lambda r: (r.arrival, r.rid))
    return ordered[rank::world]


def merge_reports(reports: List[dict]) -> dict:
    """One report for the whole job from the ranks' reports (each with its raw
    latencies): DOF-updates summed over ranks per the longest rank's wall time,
    percentiles over all requests."""
    wall = max(r["wall_seconds"] for r in reports)
    dof = sum(r["dof_updates"] for r in reports)
    lat = np.concatenate([np.asarray(r["latency_s"], dtype=float) for r in reports])
    qwait = np.concatenate([np.asarray(r["admission_wait_s"], dtype=float) for r in reports])
    return {
        "cases": int(sum(r["cases"] for r in reports)), "wall_seconds": wall,
        "dof_updates": float(dof), "dof_updates_per_s": dof / wall,
        "latency_p50_s": float(np.percentile(lat, 50)),
        "latency_p99_s": float(np.percentile(lat, 99)), "latency_max_s": float(lat.max()),
        "admission_wait_p50_s": float(np.percentile(qwait, 50)),
        "admission_wait_p99_s": float(np.percentile(qwait, 99)),
        "loop_iterations_with_steps": [r["loop_iterations_with_steps"] for r in reports],
        "ranks": len(reports),
    }


def offered_load_sweep(requests: List[Request], loads: List[float], caps: Dict[int, tuple],
                       precision: int, max_cases: int, workers: int) -> dict:
    """Latency against offered load. The capacity C (DOF-updates/s) is measured
    first with every request arriving at t = 0 (the GPU never idles); then for
    each offered load rho the same requests arrive in the same order with their
    inter-arrival times scaled so that the stream offers rho C on average
    (mean inter-arrival = total work / (cases rho C)). Below capacity the
    latency reflects admission and co-scheduling rather than a backlog."""
    work = float(sum(r.spec.n_dofs * r.steps for r in requests))
    t_last = max(r.arrival for r in requests)
    rows = []

    def one(reqs):
        ens = Ensemble(caps, precision=precision, max_cases=max_cases)
        try:
            return serve(reqs, ens, prepare_workers=workers)
        finally:
            ens.close()

    rep = one([dataclasses.replace(r, arrival=0.0) for r in requests])
    cap = rep["dof_updates_per_s"]
    rows.append(dict(rep, offered_load=None, mean_interarrival_s=0.0))
    for rho in loads:
        mean_ia = work / (len(requests) * rho * cap)
        scale = mean_ia * len(requests) / t_last   # t_last ~ n * mean of the unscaled stream
        reqs = [dataclasses.replace(r, arrival=r.arrival * scale) for r in requests]
        rep = one(reqs)
        rows.append(dict(rep, offered_load=rho, mean_interarrival_s=mean_ia,
                         last_arrival_s=max(r.arrival for r in reqs)))
    return {"capacity_dof_updates_per_s": cap, "total_dof_updates": work, "rows": rows}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", type=int, default=256)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--budget-gb", type=float, default=100.0)
    ap.add_argument("--workers", type=int, default=16)
    ap.add_argument("--max-cases", type=int, default=8,
                    help="case slots per degree bucket: the cases stepped together")
    ap.add_argument("--progress", type=float, default=0.0, help="seconds between progress lines")
    ap.add_argument("--offered-load", default=None,
                    help="comma-separated fractions of the measured capacity: sweep the "
                         "arrival rate (offered_load_sweep) instead of one run")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    reqs = request_stream(a.cases, a.seed, steps=a.steps)
    prec = capi.MIXED if a.precision == "mixed" else capi.FP64
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        return _serve_ranks(a, reqs, prec, world)
    caps = plan_capacities(reqs, int(a.budget_gb * 1e9))
    if a.offered_load:
        loads = [float(x) for x in a.offered_load.split(",")]
        rep = offered_load_sweep(reqs, loads, caps, prec, a.max_cases, a.workers)
        rep.update({"precision": a.precision, "steps_per_case": a.steps, "seed": a.seed,
                    "cases": a.cases, "max_cases_per_bucket": a.max_cases,
                    "capacities": {str(k): list(v) for k, v in caps.items()}})
        line = json.dumps(rep)
        print(line)
        if a.out:
            with open(a.out, "w") as f:
                f.write(line + "\n")
        return 0
    ens = Ensemble(caps, precision=prec, max_cases=a.max_cases)
    rep = serve(reqs, ens, prepare_workers=a.workers, progress_every=a.progress)
    rep.update({"precision": a.precision, "steps_per_case": a.steps, "seed": a.seed,
                "max_cases_per_bucket": a.max_cases,
                "capacities": {str(k): list(v) for k, v in caps.items()}})
    ens.close()
    line = json.dumps(rep)
    print(line)
    if a.out:
        with open(a.out, "w") as f:
            f.write(line + "\n")
    return 0


def _serve_ranks(a, reqs, prec, world) -> int:
    """Under torchrun, one process per GPU: each rank serves its share of the
    stream (shard_requests) on its own GPU; rank 0 prints the job's report."""
    import datetime
    import torch
    import torch.distributed as dist
    if a.offered_load:
        raise SystemExit("the offered-load sweep runs on one GPU")
    rank, local = int(os.environ["RANK"]), int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=1800))
    try:
        mine = shard_requests(reqs, rank, world)
        caps = plan_capacities(mine, int(a.budget_gb * 1e9))
        ens = Ensemble(caps, precision=prec, max_cases=a.max_cases)
        try:
            rep = serve(mine, ens, prepare_workers=a.workers, progress_every=a.progress,
                        keep_latencies=True)
        finally:
            ens.close()
        reports = [None] * world
        dist.all_gather_object(reports, rep)
    finally:
        dist.destroy_process_group()
    if rank == 0:
        out = merge_reports(reports)
        out.update({"precision": a.precision, "steps_per_case": a.steps, "seed": a.seed,
                    "max_cases_per_bucket": a.max_cases, "gpus": world})
        line = json.dumps(out)
        print(line)
        if a.out:
            with open(a.out, "w") as f:
                f.write(line + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
