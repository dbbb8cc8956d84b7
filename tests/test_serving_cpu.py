"""Host logic of the served ensemble (no GPU): the request stream, capacity
planning and the continuous-batching loop against a stand-in ensemble that
admits by element capacity and completes a case one step after its last step,
as the device finalize does."""
from __future__ import annotations

import numpy as np

from vcp3d_open_b200 import capi, serving


def test_request_stream_is_seeded_and_in_range():
    a = serving.request_stream(64, seed=7)
    b = serving.request_stream(64, seed=7)
    assert [(r.arrival, r.spec.name) for r in a] == [(r.arrival, r.spec.name) for r in b]
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) > 0)
    assert 0.005 < np.mean(np.diff(arr)) < 0.05          # mean inter-arrival 20 ms
    for r in a:
        n = r.spec.n_elem[0]
        assert r.spec.n_elem == (n, n, n) and 8 <= n <= 24
        assert r.spec.p in (2, 3, 4, 5) and 0.2 <= r.spec.mach <= 0.6
        if r.spec.kind == "vortex":
            assert 2.0 <= r.spec.beta <= 6.0 and not r.spec.is_open
        else:
            assert r.spec.kind == "pulse" and r.spec.is_open and r.spec.cml
    assert {r.spec.kind for r in a} == {"vortex", "pulse"}


def test_capacities_hold_the_largest_case_and_scale_with_budget():
    reqs = serving.request_stream(40, seed=1)
    big = serving.plan_capacities(reqs, int(1e15))
    small = serving.plan_capacities(reqs, int(1e6))
    for p in big:
        sizes = [serving.case_sizes(r.spec) for r in reqs if r.spec.p == p]
        tot = np.sum(sizes, axis=0)
        mx = np.max(sizes, axis=0)
        assert tuple(big[p]) == tuple(int(v) for v in tot)          # everything resident
        assert all(s >= m for s, m in zip(small[p], mx))           # the largest case fits


class FakeEnsemble:
    def __init__(self, cap_elems):
        self.precision = capi.MIXED
        self.cap = cap_elems
        self.used = 0
        self.next = 1
        self.cases = {}   # id -> [n_elems, steps_done, target]
        self.max_resident = 0

    def submit(self, pc, n_steps):
        n = pc.spec.n_elements
        if self.used + n > self.cap:
            return None
        cid, self.next = self.next, self.next + 1
        self.cases[cid] = [n, 0, n_steps]
        self.used += n
        self.max_resident = max(self.max_resident, len(self.cases))
        return cid

    def step(self):
        for c in self.cases.values():
            c[1] += 1

    def poll(self):
        return [cid for cid, c in self.cases.items() if c[1] > c[2]]

    def retire(self, cid):
        n = self.cases.pop(cid)[0]
        self.used -= n
        return np.zeros(1), 1.0

    def sync(self):
        pass


class _Prepared:
    def __init__(self, spec):
        self.spec = spec


def test_request_loop_admits_within_capacity_and_completes(monkeypatch):
    reqs = serving.request_stream(30, seed=5, mean_interarrival=0.001, steps=4, n_range=(3, 6))
    monkeypatch.setattr(serving, "prepare", lambda spec, precision: _Prepared(spec))
    cap = 3 * max(r.spec.n_elements for r in reqs)
    ens = FakeEnsemble(cap)
    rep = serving.serve(reqs, ens, prepare_workers=2, keep_results=True)
    assert rep["cases"] == 30 and len(rep["results"]) == 30
    assert ens.used == 0 and not ens.cases
    assert 1 <= ens.max_resident < 30                      # capacity limited the batch
    assert rep["latency_p99_s"] >= rep["latency_p50_s"] >= 0.0
    assert rep["dof_updates"] == sum(r.spec.n_dofs * r.steps for r in reqs)


def test_stream_shards_across_ranks_and_reports_merge(monkeypatch):
    """Several GPUs: every rank serves every world-th request; the merged report
    sums the DOF-updates over the longest rank's wall time and takes the
    percentiles over all requests."""
    reqs = serving.request_stream(23, seed=9, mean_interarrival=0.001, steps=3, n_range=(3, 5))
    world = 3
    parts = [serving.shard_requests(reqs, r, world) for r in range(world)]
    assert sorted(r.rid for p in parts for r in p) == sorted(r.rid for r in reqs)
    assert [len(p) for p in parts] == [8, 8, 7]
    monkeypatch.setattr(serving, "prepare", lambda spec, precision: _Prepared(spec))
    reports = []
    for p in parts:
        ens = FakeEnsemble(3 * max(r.spec.n_elements for r in p))
        reports.append(serving.serve(p, ens, prepare_workers=2, keep_latencies=True))
    out = serving.merge_reports(reports)
    assert out["cases"] == 23 and out["ranks"] == world
    assert out["dof_updates"] == sum(r.spec.n_dofs * r.steps for r in reqs)
    wall = max(r["wall_seconds"] for r in reports)
    assert out["wall_seconds"] == wall and out["dof_updates_per_s"] == out["dof_updates"] / wall
    lat = np.concatenate([r["latency_s"] for r in reports])
    assert out["latency_p50_s"] == float(np.percentile(lat, 50))
    assert out["latency_max_s"] == float(lat.max())
