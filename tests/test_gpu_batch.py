"""Batches and the serving loop (qvti_run_batch, qvti_server_*): many shots of
uneven size in flight on one GPU.

Shots are independent and every kernel is deterministic (no atomics, fixed
reduction order), so each shot's seismograms must be bit-identical whether
it runs alone (one simulation, run_case) or among others; the tests compare
with exact equality.
"""
import time

import numpy as np
import pytest

import qvti_cases as qc

pytestmark = pytest.mark.gpu


def _cases():
    """Five small shots: different grids (runtime and compile-time transform
    lengths), isotropic and VTI, force and explosive sources, different nt."""
    specs = [((32, 32, 32), 6, 70, False, 0), ((48, 32, 40), 6, 90, True, 0), ((32, 48, 32), 6, 60, False, 1),
             ((64, 64, 64), 8, 80, True, 0), ((40, 40, 40), 6, 100, False, 0)]
    out = []
    for i, (n, pml, nt, vti, src) in enumerate(specs):
        c = qc.heterogeneous_case(n=n, pml=pml, d=(10.0, 10.0, 10.0), dt=0.8e-3, nt=nt, f0=30.0, seed=40 + i,
                                  src=(n[0] // 2, n[1] // 2, n[2] // 2), r_iz=n[2] // 2 - 6, name="b%d" % i)
        if vti:
            rng = np.random.default_rng(90 + i)
            c["eps"] = (0.05 + 0.2 * rng.random(n)).astype(np.float32)
            c["delta"] = (0.12 * rng.random(n)).astype(np.float32)
        out.append((c, vti, src))
    return out


@pytest.fixture(scope="module")
def alone(qvti):
    return [qvti.run_case(c, vti=vti, src_type=src)["rec"] for c, vti, src in _cases()]


def _requests(qvti):
    return [qvti.ShotRequest(c, vti=vti, src_type=src) for c, vti, src in _cases()]


@pytest.mark.parametrize("max_active", [1, 3])
def test_batch_matches_shots_run_alone(qvti, alone, max_active):
    reqs = _requests(qvti)
    results, wall = qvti.run_batch(reqs, max_active=max_active)
    assert wall > 0
    for r, req, ref in zip(results, reqs, alone):
        assert r["status"] == 0
        assert r["device_ms"] > 0 and r["latency_s"] >= r["queue_s"] >= 0
        assert np.array_equal(req.rec, ref)


def test_batch_with_autotuned_concurrency(qvti, alone):
    reqs = _requests(qvti)[:2]
    results, _ = qvti.run_batch(reqs, max_active=0)
    for r, req, ref in zip(results, reqs, alone[:2]):
        assert r["status"] == 0
        assert np.array_equal(req.rec, ref)


def test_autotune_reports_a_setting(qvti):
    active, kzb, form, rate, tiles = qvti.autotune(64, 64, 64, 8, 10.0, 10.0, 10.0, 0.8e-3, 30.0, vti=True,
                                                   max_active=3, probe_steps=4)
    assert 1 <= active <= 3
    assert len(tiles) == qvti.NUM_TILES and all(t == 0 or t in (2, 4, 8, 16, 32) for t in tiles)
    assert kzb in (33, 17)
    assert form == qvti.FORM_PLAIN  # no tensor-core plan without a 256-point y axis
    assert rate > 0


def test_autotune_probes_the_tensor_core_form(qvti):
    """A 256-point y axis has both forms; the tuner times each and keeps the
    faster (the plain form unless the tensor-core plan is 2 % faster)."""
    active, kzb, form, rate, _ = qvti.autotune(32, 256, 32, 6, 10.0, 10.0, 10.0, 0.8e-3, 30.0, vti=False,
                                               max_active=2, probe_steps=4)
    assert form in (qvti.FORM_PLAIN, qvti.FORM_TC) and 1 <= active <= 2 and kzb in (17, 9) and rate > 0


def test_server_admits_while_others_run(qvti, alone):
    """Continuous batching: the later requests arrive while the first runs;
    results are the same as alone, and a zero-timeout wait on an unfinished
    shot reports a timeout without consuming the ticket."""
    reqs = _requests(qvti)
    with qvti.Server(max_active=2) as srv:
        t0 = srv.submit(reqs[3])              # 64^3 VTI, the longest
        assert srv.wait(t0, timeout=0.0) is None
        tickets = [t0]
        for r in (reqs[0], reqs[1], reqs[2], reqs[4]):
            time.sleep(0.01)
            tickets.append(srv.submit(r))
        seen = []
        deadline = time.time() + 60.0
        while time.time() < deadline:   # the first admission creates a simulation (tens of ms)
            q, a, pool = srv.load()
            seen.append((a, pool))
            if q == 0 and a == 0:
                break
            time.sleep(0.002)
        assert all(a <= 2 for a, _ in seen)
        assert max(pool for _, pool in seen) > 0
        res = {t: srv.wait(t, timeout=120.0) for t in tickets}
    order = [3, 0, 1, 2, 4]
    for t, i in zip(tickets, order):
        assert res[t] is not None and res[t]["status"] == 0
        assert np.array_equal(reqs[i].rec, alone[i])


@pytest.mark.parametrize("policy", ["fifo", "smallest_first"])
def test_server_admission_policy(qvti, alone, policy):
    """One shot in flight: while the 64^3 VTI shot (21 M cell-steps) runs, a
    40^3 shot (6.4 M) and then a 32^3 shot (2.3 M) are queued.  First in,
    first out finishes them in that order; smallest first admits the 32^3
    shot ahead of the 40^3 one.  Results stay exact either way."""
    reqs = _requests(qvti)
    pol = qvti.SCHED_FIFO if policy == "fifo" else qvti.SCHED_SMALLEST_FIRST
    with qvti.Server(max_active=1, policy=pol) as srv:
        t3 = srv.submit(reqs[3])
        deadline = time.time() + 60.0
        active = 0
        while active == 0 and time.time() < deadline:  # until the 64^3 shot is admitted (its set-up and
            active = srv.load()[1]                     # 80 steps then take milliseconds)
        assert active == 1
        t4 = srv.submit(reqs[4])
        t0 = srv.submit(reqs[0])
        res = {t: srv.wait(t, timeout=120.0) for t in (t3, t4, t0)}
    for t, i in ((t3, 3), (t4, 4), (t0, 0)):
        assert res[t] is not None and res[t]["status"] == 0
        assert np.array_equal(reqs[i].rec, alone[i])
    # submitted back to back: the one admitted first finishes first
    if policy == "fifo":
        assert res[t4]["latency_s"] < res[t0]["latency_s"], res
    else:
        assert res[t0]["latency_s"] < res[t4]["latency_s"], res


def test_server_rejects_an_unknown_policy(qvti):
    with pytest.raises(qvti.QvtiError):
        qvti.Server(policy=7)


def test_server_budget_admits_one_at_a_time(qvti, alone):
    """A budget that holds one 64^3 simulation: shots queue for memory, the
    pool frees idle simulations of other grids, results stay exact."""
    reqs = _requests(qvti)
    budget = int(qvti.footprint_bytes(64, 64, 64, 8, True) * 1.2)
    with qvti.Server(max_active=4, mem_budget=budget) as srv:
        tickets = [srv.submit(r) for r in reqs]
        seen_active = 0
        while True:
            q, a, pool = srv.load()
            seen_active = max(seen_active, a)
            assert pool <= budget
            if q == 0 and a == 0:
                break
            time.sleep(0.002)
        res = [srv.wait(t, timeout=60.0) for t in tickets]
    assert seen_active >= 1
    for r, req, ref in zip(res, reqs, alone):
        assert r["status"] == 0
        assert np.array_equal(req.rec, ref)


def test_server_rejects_a_shot_beyond_the_budget(qvti):
    c, vti, src = _cases()[3]
    req = qvti.ShotRequest(c, vti=vti, src_type=src)
    with qvti.Server(max_active=1, mem_budget=1 << 20) as srv:
        with pytest.raises(qvti.QvtiError, match="allocation"):
            srv.submit(req)


def test_nonfinite_shot_fails_alone_in_the_mix(qvti, alone):
    """Shot-level failure detection, the fault made on the host: one shot's
    model holds a NaN (an interior cell of its P velocity).  The scheduler's
    sentinel (a non-finite check of the velocities after every chunk of
    steps) ends that shot early with QVTI_ERR_NONFINITE; the shots beside it
    finish with seismograms bit-identical to running alone.  The NaN shot
    runs long (2000 steps) so an early stop is visible in its device time."""
    reqs = _requests(qvti)[:3]
    bad_case = dict(_cases()[0][0])
    bad_case["velp"] = bad_case["velp"].copy()
    bad_case["velp"][16, 16, 12] = np.nan
    bad_case["nt"] = 2000
    bad_case["rik"] = qc.ricker(2000, bad_case["dt"], bad_case["f0"])
    bad = qvti.ShotRequest(bad_case)
    with qvti.Server(max_active=4) as srv:
        tickets = [srv.submit(r) for r in (reqs[0], bad, reqs[1], reqs[2])]
        res = [srv.wait(t) for t in tickets]
    assert res[1]["status"] == 6, res[1]  # QVTI_ERR_NONFINITE
    for r, req, ref in zip((res[0], res[2], res[3]), reqs, alone[:3]):
        assert r["status"] == 0
        assert np.array_equal(req.rec, ref)
    # stopped after at most a few 32-step chunks of 2000
    assert res[1]["latency_s"] < 20.0
