"""The bound server's scheduling on the host (no GPU): requests start in arrival order, never more than `slots` at a
time nor more estimated device memory than the budget, late arrivals join while others run, an oversized request is
refused and a failing request is reported.  The device work of a request is replaced by a short sleep."""
import threading
import time

import numpy as np
import pytest

from lagbound_b200.serving import BoundRequest, BoundServer, latency_stats


def _request(rid, n, arrival):
    indptr = np.arange(n + 1, dtype=np.int64)
    return BoundRequest(rid, n, indptr, np.zeros(n, np.int64), np.ones(n), float(n), 0.0, np.zeros(n, np.int64),
                        arrival=arrival)


class SleepServer(BoundServer):
    """Each request sleeps for `busy` seconds; the peak concurrency and memory in use are recorded."""

    def __init__(self, busy=0.05, fail=(), **kw):
        super().__init__(**kw)
        self.busy, self.fail = busy, set(fail)
        self.active, self.peak, self.peak_bytes, self.starts = 0, 0, 0.0, []
        self.mon = threading.Lock()

    def _solve(self, req):
        with self.mon:
            self.active += 1
            self.peak = max(self.peak, self.active)
            self.peak_bytes = max(self.peak_bytes, self.used)
            self.starts.append(req.rid)
        time.sleep(self.busy)
        with self.mon:
            self.active -= 1
        if req.rid in self.fail:
            raise ValueError("device work failed")
        return float(req.rid), 0.0


def test_slots_bound_the_requests_in_flight():
    reqs = [_request(k, 1000 + 10 * k, 0.002 * k) for k in range(12)]
    srv = SleepServer(slots=3)
    res = srv.run(reqs)
    assert sorted(r.rid for r in res) == list(range(12))
    assert srv.peak == 3
    assert srv.starts == sorted(srv.starts)                 # arrival order
    assert all(r.ub == r.rid and r.admitted >= r.arrival and r.done > r.admitted for r in res)
    st = latency_stats(res)
    assert st["requests"] == 12 and st["p99_s"] >= st["p50_s"] > 0


def test_memory_budget_bounds_the_requests_in_flight():
    reqs = [_request(k, 2000, 0.0) for k in range(6)]
    need = reqs[0].device_bytes()
    srv = SleepServer(slots=6, hbm_budget=2.5 * need)
    srv.run(reqs)
    assert srv.peak == 2 and srv.peak_bytes <= 2.5 * need


def test_late_arrivals_join_while_others_run():
    reqs = [_request(0, 1000, 0.0), _request(1, 1000, 0.05)]
    srv = SleepServer(busy=0.3, slots=4)
    res = {r.rid: r for r in srv.run(reqs)}
    assert res[1].admitted < res[0].done                     # admitted before the first finished
    assert srv.peak == 2


def test_oversized_and_failing_requests_are_reported():
    small = _request(0, 1000, 0.0)
    with pytest.raises(RuntimeError, match="needs"):
        SleepServer(slots=2, hbm_budget=0.5 * small.device_bytes()).run([small])
    with pytest.raises(RuntimeError, match="request 1 failed"):
        SleepServer(slots=2, fail={1}).run([_request(0, 1000, 0.0), _request(1, 1000, 0.0)])


class PhaseServer(SleepServer):
    """Each request records two phases, as solve_bound does, and sleeps."""

    def _solve(self, req):
        req.phases["outers"] = 0.01 * (req.rid + 1)
        req.phases["estimate"] = 0.02
        return super()._solve(req)


def test_latency_stats_report_queueing_and_mean_phases():
    reqs = [_request(k, 1000, 0.0) for k in range(4)]
    srv = PhaseServer(busy=0.05, slots=2)
    res = srv.run(reqs)
    st = latency_stats(res)
    # two slots, four simultaneous arrivals: the second pair waits for the first
    assert st["mean_queue_s"] > 0.01
    assert st["mean_phase_s"]["outers"] == pytest.approx(np.mean([0.01 * (k + 1) for k in range(4)]), abs=1e-4)
    assert st["mean_phase_s"]["estimate"] == pytest.approx(0.02, abs=1e-4)
    assert all(r.log and r.log[0]["estimate"] == 0.02 for r in res)


def test_switch_interval_is_restored_after_serving():
    import sys
    before = sys.getswitchinterval()
    srv = SleepServer(busy=0.01, slots=2, switch_interval=1e-4)
    srv.run([_request(k, 1000, 0.0) for k in range(3)])
    assert sys.getswitchinterval() == before
