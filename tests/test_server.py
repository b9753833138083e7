"""Scheduler of the reconstruction server on CPU (host-only jobs that hold a
slot and an HBM reservation for a while): budget and slot limits, oversized
jobs, skip-ahead past a head that does not fit, and the starvation guard."""
from __future__ import annotations

import pytest


def _server(fbp, budget, slots):
    return fbp.Server(device=-1, hbm_budget_bytes=budget, slots=slots)


def _job(fbp, reserve, us):
    r = fbp.Request()
    r.kind = fbp.JobKind.HOST_WAIT
    r.reserve_bytes = reserve
    r.views = us
    return r


def _overlaps(res):
    ev = sorted([(r.started_ms, 1) for r in res] + [(r.finished_ms, -1) for r in res], key=lambda e: (e[0], e[1]))
    cur = best = 0
    for _, d in ev:
        cur += d
        best = max(best, cur)
    return best


def test_budget_limits_concurrency(fbp):
    s = _server(fbp, 100, 3)
    res = [s.wait(t) for t in [s.submit(_job(fbp, 60, 15000)) for _ in range(4)]]
    s.close()
    assert all(r.status == 0 for r in res)
    assert _overlaps(res) == 1  # two 60-byte jobs never fit a 100-byte budget together


def test_slots_limit_concurrency(fbp):
    s = _server(fbp, 1000, 2)
    res = [s.wait(t) for t in [s.submit(_job(fbp, 10, 15000)) for _ in range(6)]]
    s.close()
    assert _overlaps(res) == 2


def test_oversized_job_runs_alone(fbp):
    s = _server(fbp, 100, 3)
    a = s.submit(_job(fbp, 500, 10000))
    b = s.submit(_job(fbp, 10, 10000))
    ra, rb = s.wait(a), s.wait(b)
    s.close()
    assert ra.status == 0 and rb.status == 0
    assert rb.started_ms >= ra.finished_ms  # nothing runs beside a job larger than the budget


def test_small_job_passes_a_head_that_does_not_fit(fbp):
    s = _server(fbp, 100, 3)
    a = s.submit(_job(fbp, 60, 40000))  # running
    b = s.submit(_job(fbp, 80, 10000))  # head: waits for memory
    c = s.submit(_job(fbp, 30, 10000))  # fits beside a: starts first
    ra, rb, rc = s.wait(a), s.wait(b), s.wait(c)
    s.close()
    assert rc.started_ms < rb.started_ms
    assert rb.started_ms >= max(ra.finished_ms, rc.finished_ms)


def test_starvation_guard(fbp):
    """A head that keeps being passed over eventually blocks the queue and runs."""
    s = _server(fbp, 100, 3)
    first = s.submit(_job(fbp, 20, 20000))
    big = s.submit(_job(fbp, 90, 1000))
    small = [s.submit(_job(fbp, 20, 3000)) for _ in range(60)]
    rs = [s.wait(t) for t in [first] + small]
    rb = s.wait(big)
    s.close()
    before = sum(r.started_ms < rb.started_ms for r in rs)
    assert before <= 1 + 16 + 3
    assert any(r.started_ms > rb.started_ms for r in rs)


def test_close_runs_queued_jobs(fbp):
    s = _server(fbp, 100, 2)
    for _ in range(5):
        s.submit(_job(fbp, 10, 2000))
    s.close()  # returns after the queued jobs ran


def test_batching_settings_on_a_host_only_server(fbp):
    """The batching switches are accepted on a server without a device (they
    only steer cone jobs) and host-only jobs still run."""
    s = _server(fbp, 1000, 2)
    s.set_batching(True, 3e10)
    s.set_batch_limit(1e10)
    s.set_batch_limit(0.0)  # back to the default limit
    r = s.wait(s.submit(_job(fbp, 10, 1000)))
    s.close()
    assert r.status == 0


def test_a_ticket_has_one_waiter(fbp):
    """A ticket is consumed by its wait: a second caller waiting on a ticket
    that another caller already waits on gets a state error (the job keeps
    running for the first), and a consumed ticket is unknown afterwards."""
    import threading
    import time

    s = _server(fbp, 1000, 1)
    t = s.submit(_job(fbp, 10, 3000000))  # holds the slot for 3 s
    got = {}
    first = threading.Thread(target=lambda: got.setdefault("r", s.wait(t)))
    first.start()
    time.sleep(0.5)  # the first caller is waiting well before the job ends
    with pytest.raises(fbp.FBPError) as e:
        s.wait(t)
    assert e.value.status == -2
    first.join()
    assert got["r"].status == 0
    with pytest.raises(fbp.FBPError) as e:
        s.wait(t)
    assert e.value.status == -1
    s.close()
