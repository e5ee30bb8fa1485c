"""Serving loop: continuous batching with admission by an HBM budget, results alone and in the mix.

- In the mix vs alone: each request served among others (joining and leaving the batch at different steps, with
  other requests' vessels in the same launches) ends bit for bit where the same request ends when it is the only
  one served: the batched kernels apply each instance's own arithmetic to its own buffers.
- Against the dedicated single-lattice path: within relative L2 1e-5 of velocity and density (the batched and
  single-lattice kernels are compiled separately and may round differently in the last bit).
- Admission: the reserved memory never exceeds the budget; requests wait in the queue until memory frees up.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from cerebrosim_b200 import serve, workloads  # noqa: E402

SPB = 200           # steps per beat of the test workload


def specs():
    sizes = [30e3, 60e3, 20e3, 45e3, 25e3]
    beats = [2, 1, 3, 1, 2]
    sten = [0.3, 0.7, 0.0, 1.0, 0.5]
    return [{"id": k, "arrival": 0.01 * k, "seed": 200 + k, "stenosis": sten[k], "pressure": 80.0 + 10 * k,
             "beats": beats[k], "nodes": sizes[k]} for k in range(5)]


def server(storage="bf16", **kw):
    args = dict(storage=storage, steps_per_beat=SPB, chunk=50, graph_chunk=50, ahead=2)
    args.update(kw)
    return serve.Server(**args)


def l2(a, b):
    return float(np.sqrt(((a.astype(np.float64) - b) ** 2).sum() / max((b.astype(np.float64) ** 2).sum(), 1e-300)))


@pytest.mark.parametrize("schedule", ["fused", "by-instance", "concurrent:2", "concurrent:4"])
@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_served_results_same_alone_and_in_the_mix(storage, schedule):
    sv = server(storage, max_active=3, schedule=schedule)
    mix = sv.serve(specs(), realtime=False)
    assert all(r.ok for r in mix)
    # the mix really overlapped: up to three requests shared the launches, later ones joined mid-run
    assert max(n for _, n, _ in sv.trace) == 3
    assert max(r.queue_wait for r in mix) > 0
    for r in mix:
        assert len(r.beat_end) == r.beats and len(r.beat_latencies()) == r.beats
        alone = server(storage, schedule=schedule).serve([r.spec], realtime=False)[0]
        p0, u0 = alone.fields
        p1, u1 = r.fields
        assert np.array_equal(p0, p1) and np.array_equal(u0, u1), r.id


@pytest.mark.parametrize("schedule", ["fused", "by-instance"])
def test_served_matches_dedicated_solver(schedule):
    sp = specs()[0]
    r = server("f32", max_active=3, schedule=schedule).serve(specs(), realtime=False)[0]
    s = serve.default_builder(sp, "f32", 256, None, SPB)
    s.run(sp["beats"] * SPB, chunk=50)
    p, u = s.fields()
    assert l2(r.fields[1], u) <= 1e-5 and l2(3 * r.fields[0] + 1, 3 * p + 1) <= 1e-5


def test_admission_by_budget():
    records = []
    sv = server("bf16", budget_bytes=2.5 * serve.BYTES_PER_NODE["bf16"] * 60e3, log=records.append)
    reqs = sv.serve(specs(), realtime=False)
    # the per-beat metrics stream: one record per beat of every request, JSON-ready
    import json
    assert len(records) == sum(r.beats for r in reqs) and json.loads(json.dumps(records)) == records
    assert all(x["latency_s"] > 0 and x["mlups"] > 0 for x in records)
    assert all(r.ok for r in reqs)
    assert all(used <= sv.budget for _, _, used in sv.trace)
    # not everything fitted at once: some request waited for memory to free up
    assert max(n for _, n, _ in sv.trace) < len(reqs)
    assert max(r.queue_wait for r in reqs) > 0
    st = serve.summary(reqs, SPB)
    assert st["beats"] == sum(r.beats for r in reqs) and st["all_ok"]
    assert st["beat_latency_p99_s"] >= st["beat_latency_p50_s"] > 0


def test_request_over_budget_is_refused():
    sv = server("bf16", budget_bytes=1e6)
    with pytest.raises(RuntimeError, match="budget"):
        sv.serve(specs()[:1], realtime=False)


def test_on_beat_changes_apply_from_the_next_beat():
    """A per-beat hook (where the lumped circuit is recalibrated, simulate.py:330-337) rescales each request's drive
    after its first beat: served in a mix, the result equals the same schedule run on a dedicated solver."""
    def rescale(r, beat):
        s = r.solver
        s.set_drive([1.2 * c for c in s.coef.cpu().numpy()[:1 + 2 * s.nh]], period=s.period, ramp=s.ramp)

    sp = [dict(x, beats=2) for x in specs()[:3]]
    mix = server("f32", max_active=3, on_beat=rescale).serve(sp, realtime=False)
    for r in mix:
        s = serve.default_builder(r.spec, "f32", 128, None, SPB)
        s.run(SPB, chunk=50)
        s.set_drive([1.2 * c for c in s.coef.cpu().numpy()[:1 + 2 * s.nh]], period=s.period, ramp=s.ramp)
        s.run(SPB, chunk=50)
        p, u = s.fields()
        assert l2(r.fields[1], u) <= 1e-5, r.id


def test_diverged_request_is_evicted_and_the_others_are_unchanged():
    """One request's populations are poisoned with NaN from the host after its first beat (a density that has gone
    non-finite, as a diverging run's does). At its next beat end the server evicts it — slot and budget released —
    while every other request ends bit for bit where it ends when served alone."""
    import torch
    poisoned = 2                                     # three beats

    def poison(r, beat):
        if r.id == poisoned and beat == 1:
            s = r.solver
            with torch.cuda.stream(s.stream):
                s.f[s.cur][0, 10] = float("nan")
            s.synchronize()

    sv = server("f32", max_active=3, on_beat=poison)
    mix = sv.serve(specs(), realtime=False)
    bad = next(r for r in mix if r.id == poisoned)
    assert bad.evicted == 2 and bad.ok is False and bad.fields is None and bad.solver is None
    assert len(bad.beat_end) == 2
    st = serve.summary(mix, SPB)
    assert st["evicted"] == [poisoned] and not st["all_ok"]
    assert sv._used == pytest.approx(0.0, abs=1.0)   # every reservation released, the evicted one included
    for r in mix:
        if r.id == poisoned:
            continue
        assert r.ok and r.evicted is None
        alone = server("f32").serve([r.spec], realtime=False)[0]
        assert np.array_equal(alone.fields[0], r.fields[0]) and np.array_equal(alone.fields[1], r.fields[1]), r.id


SPB_CAL = 2000      # steps per beat of the calibrated requests: long enough for the inflow to cross the vessel


def calibrated_specs():
    return [{"id": k, "arrival": 0.0, "seed": 300 + k, "stenosis": s, "pressure": p, "beats": 2, "nodes": n}
            for k, (s, p, n) in enumerate([(0.5, 90.0, 30e3), (0.0, 120.0, 45e3), (0.7, 75.0, 25e3)])]


def test_served_recalibration_matches_dedicated_artery_solver():
    """Requests run as the reference runs its arteries (pressure inlet from the lumped circuit, resistance outlets,
    slab flows) with the circuit recalibrated after every beat from the beat's mean inlet pressure and inflow
    (simulate.py:330-337), served three at a time: each ends as the same schedule on a dedicated ArterySolver, with
    the same segment resistance found at every beat."""
    seen = {}

    def hook(r, beat):
        serve.recalibrate_on_beat(r, beat)
        seen[(r.id, beat)] = dict(r.solver.calibration.history[-1])

    sv = server("f32", max_active=3, builder=workloads.calibrated_builder, on_beat=hook, steps_per_beat=SPB_CAL,
                chunk=500, graph_chunk=100)
    mix = sv.serve(calibrated_specs(), realtime=False)
    assert all(r.ok for r in mix), [(r.id, r.evicted) for r in mix]
    for r in mix:
        s = workloads.calibrated_solver(r.spec, storage="f32", block=128, steps_per_beat=SPB_CAL)
        for b in range(1, r.beats + 1):
            s.run(SPB_CAL, chunk=100)
            if b < r.beats:
                s.calibration.on_beat(b)
                h, hs = s.calibration.history[-1], seen[(r.id, b)]
                assert h["steps"] == hs["steps"] == SPB_CAL
                assert h["R_seg"] == pytest.approx(hs["R_seg"], rel=1e-6, abs=1.0)
                assert h["q_in_ml_min"] == pytest.approx(hs["q_in_ml_min"], rel=1e-6)
        p, u = s.fields()
        assert l2(r.fields[1], u) <= 1e-5 and l2(3 * r.fields[0] + 1, 3 * p + 1) <= 1e-5, r.id
        # the calibration acted: a segment resistance was found from the measured beat means
        assert any(seen[(r.id, b)]["R_seg"] > 0 for b in range(1, r.beats))
