"""Served ensemble on the GPU: a case's result is the same alone and in the mix
(bit-identical), matches the single-case path, admission by footprint refuses
and later admits, and the request loop completes a small stream."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2
from vcp3d_open_b200 import capi, cases, serving, solver

pytestmark = pytest.mark.gpu

STEPS = 6


def _specs():
    return [
        serving.vortex_spec(4, 2, 0.3, 3.0, "v_n4_p2"),
        serving.vortex_spec(5, 3, 0.5, 5.0, "v_n5_p3"),
        serving.pulse_spec(6, 3, 0.4, "pulse_n6_p3"),
        serving.vortex_spec(3, 3, 0.25, 2.5, "v_n3_p3"),
        serving.pulse_spec(4, 2, 0.3, "pulse_n4_p2"),
        serving.pulse_spec(5, 4, 0.5, "pulse_n5_p4"),
    ]


def _caps(specs, slack=2):
    caps = {}
    for s in specs:
        ne, nb, ns = serving.case_sizes(s)
        c = caps.setdefault(s.p, [0, 0, 0])
        c[0] += slack * ne
        c[1] += slack * nb
        c[2] += slack * ns
    return {p: tuple(v) for p, v in caps.items()}


def _run_to_completion(ens, ids):
    out = {}
    for _ in range(10000):
        ens.step()
        for cid in ens.poll():
            out[cid] = ens.retire(cid)
        if all(i in out for i in ids):
            return out
    raise AssertionError("cases did not complete")


@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED])
def test_result_is_the_same_alone_and_in_the_mix(gpu_available, precision):
    specs = _specs()
    prepared = [serving.prepare(s, precision) for s in specs]
    caps = _caps(specs)
    alone = []
    for pc in prepared:
        ens = serving.Ensemble(caps, precision=precision, max_cases=8)
        cid = ens.submit(pc, STEPS)
        res = _run_to_completion(ens, [cid])
        ens.sync()
        ens.close()
        alone.append(res[cid])
    # The mix: cases join at different steps while others are running.
    ens = serving.Ensemble(caps, precision=precision, max_cases=8)
    ids = [ens.submit(prepared[0], STEPS), ens.submit(prepared[2], STEPS)]
    ens.step()
    ens.step()
    ids.append(ens.submit(prepared[1], STEPS))
    ens.step()
    ids += [ens.submit(prepared[i], STEPS) for i in (3, 4, 5)]
    res = _run_to_completion(ens, ids)
    ens.sync()
    ens.close()
    for k, cid in enumerate([ids[0], ids[2], ids[1], ids[3], ids[4], ids[5]]):
        state, t = res[cid]
        np.testing.assert_array_equal(state, alone[k][0], err_msg=specs[k].name)
        assert t == alone[k][1]
        assert t > 0.0 and np.all(np.isfinite(state))


def test_ensemble_matches_single_case_path(gpu_available):
    """An ensemble case takes the same steps as the single-case handle."""
    specs = [serving.vortex_spec(4, 3, 0.4, 4.0, "v"), serving.pulse_spec(6, 3, 0.4, "p")]
    ens = serving.Ensemble(_caps(specs), precision=capi.FP64, max_cases=4)
    ids = [ens.submit(serving.prepare(s, capi.FP64), STEPS) for s in specs]
    res = _run_to_completion(ens, ids)
    ens.close()
    for s, cid in zip(specs, ids):
        case = cases.build_case(s)
        h = solver.create(case)
        try:
            hist = h.step(STEPS, capi.LSRK4)
            state, t = res[cid]
            assert rel_l2(state, h.get_state()) < 1e-13, s.name
            assert t == pytest.approx(float(np.sum(hist)), rel=1e-13)
        finally:
            h.close()


def test_subface_case_matches_single_case_path(gpu_available):
    """A served case with several subfaces on a block face (an inflow and an
    isothermal wall on i-min, an outflow and a heat-flux wall on i-max) takes
    the same steps as the single-case handle, alone and beside a pulse case."""
    from make_golden import OPEN_SPECS
    spec = OPEN_SPECS["subfaces_p3_4x4x2"]
    other = serving.pulse_spec(5, 3, 0.4, "p")
    ens = serving.Ensemble(_caps([spec, other]), precision=capi.FP64, max_cases=4)
    ids = [ens.submit(serving.prepare(s, capi.FP64), STEPS) for s in (spec, other)]
    res = _run_to_completion(ens, ids)
    ens.close()
    h = solver.create(cases.build_case(spec))
    try:
        hist = h.step(STEPS, capi.LSRK4)
        state, t = res[ids[0]]
        assert rel_l2(state, h.get_state()) < 1e-13
        assert t == pytest.approx(float(np.sum(hist)), rel=1e-13)
    finally:
        h.close()


def test_admission_by_footprint(gpu_available):
    specs = [serving.vortex_spec(4, 3, 0.4, 4.0, "a"), serving.vortex_spec(4, 3, 0.3, 3.0, "b")]
    ne = serving.case_sizes(specs[0])[0]
    ens = serving.Ensemble({3: (ne + ne // 2, 0, 0)}, precision=capi.FP64, max_cases=4)
    pa, pb = (serving.prepare(s, capi.FP64) for s in specs)
    ida = ens.submit(pa, 3)
    assert ida is not None
    assert ens.submit(pb, 3) is None          # no contiguous room for a second case
    _run_to_completion(ens, [ida])
    idb = ens.submit(pb, 3)                   # room again after the first retired
    assert idb is not None
    _run_to_completion(ens, [idb])
    assert ens.stats()[0] == 0
    ens.close()


def test_request_loop_small_stream(gpu_available):
    reqs = serving.request_stream(10, seed=3, mean_interarrival=0.005, steps=5, n_range=(3, 6),
                                  degrees=(2, 3, 4))
    caps = serving.plan_capacities(reqs, int(2e9))
    ens = serving.Ensemble(caps, precision=capi.MIXED, max_cases=16)
    rep = serving.serve(reqs, ens, prepare_workers=4, keep_results=True)
    ens.close()
    assert rep["cases"] == 10 and len(rep["results"]) == 10
    assert rep["latency_p99_s"] >= rep["latency_p50_s"] > 0.0
    for state, t in rep["results"].values():
        assert np.all(np.isfinite(state)) and t > 0.0


def test_slot_reuse_keeps_results(gpu_available):
    """Fewer case slots than cases: slots are reused while other cases keep
    stepping; every result stays bit-identical to the case run alone."""
    specs = _specs()
    prepared = [serving.prepare(s, capi.FP64) for s in specs]
    caps = _caps(specs)
    alone = []
    for pc in prepared:
        ens = serving.Ensemble(caps, precision=capi.FP64, max_cases=2)
        cid = ens.submit(pc, STEPS)
        alone.append(_run_to_completion(ens, [cid])[cid])
        ens.close()
    ens = serving.Ensemble(caps, precision=capi.FP64, max_cases=2)
    queue = list(range(len(prepared)))
    owner, results = {}, {}
    for _ in range(10000):
        rest = []
        for k in queue:
            cid = ens.submit(prepared[k], STEPS)
            if cid is None:
                rest.append(k)
            else:
                owner[cid] = k
        queue = rest
        ens.step()
        for cid in ens.poll():
            results[owner[cid]] = ens.retire(cid)
        if len(results) == len(prepared):
            break
    ens.sync()
    ens.close()
    assert len(results) == len(prepared)
    for k in range(len(prepared)):
        np.testing.assert_array_equal(results[k][0], alone[k][0], err_msg=specs[k].name)


def test_bucket_rejects_other_solution_dof_positions(gpu_available):
    """The bucket's operator table (basis at the nodal DOFs of the time step) is
    fixed by its first case: a later case of the same degree with equidistant
    solution DOFs is refused, one with LGL DOFs is admitted."""
    import dataclasses
    lgl = serving.vortex_spec(3, 3, 0.4, 4.0, "lgl")
    equi = dataclasses.replace(serving.vortex_spec(3, 3, 0.3, 3.0, "equi"),
                               dof_location="equidistant", grid_lgl=False)
    ens = serving.Ensemble(_caps([lgl, lgl, equi], slack=3), precision=capi.FP64, max_cases=4)
    try:
        ida = ens.submit(serving.prepare(lgl, capi.FP64), 2)
        with pytest.raises(capi.VcpgError) as err:
            ens.submit(serving.prepare(equi, capi.FP64), 2)
        assert err.value.code == capi.VCPG_E_INVALID
        assert "solution-DOF positions" in str(err.value)
        idb = ens.submit(serving.prepare(dataclasses.replace(lgl, name="lgl2"), capi.FP64), 2)
        res = _run_to_completion(ens, [ida, idb])
        assert np.all(np.isfinite(res[idb][0]))
    finally:
        ens.close()
