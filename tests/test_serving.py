"""Admission and continuous batching of the serving loop (baemm_b200/serving.py),
on the CPU with a stand-in executor: the budget and the slot count are never
exceeded, requests start in arrival order, every request completes."""
import threading
import time

import numpy as np
import pytest

from baemm_b200.serving import Scheduler, SolveServer, padded_rhs, solve_footprint_bytes, summarize


class FakeReq:
    def __init__(self, rid, fp, arrival=0.0, service=0.01):
        self.rid, self._fp, self.arrival, self.service = rid, fp, arrival, service
        self.nrhs = 1

    def footprint(self):
        return self._fp


def fake_executor(log, lock):
    def run(slot, req):
        with lock:
            log.append(("start", req.rid, time.perf_counter()))
        time.sleep(req.service)
        return np.zeros((2, 1), complex), {"gmres_iterations": 1, "gmres_relative_residual": 0.0,
                                            "gmres_converged": 1}
    return run


def test_padded_rhs_and_footprint():
    assert [padded_rhs(n) for n in (1, 16, 17, 32, 33, 64)] == [16, 16, 32, 32, 64, 64]
    with pytest.raises(ValueError):
        padded_rhs(65)
    a = solve_footprint_bytes(2562, 5120, 16)
    assert a < solve_footprint_bytes(2562, 5120, 32) < solve_footprint_bytes(40962, 81920, 32)


@pytest.mark.parametrize("slots,budget", [(1, 10), (3, 10), (4, 7), (8, 100)])
def test_budget_and_slots_respected(slots, budget):
    rng = np.random.default_rng(slots)
    reqs = [FakeReq(i, int(rng.integers(1, 5)), service=float(rng.uniform(0.001, 0.01))) for i in range(40)]
    log, lock = [], threading.Lock()
    srv = SolveServer(np.eye(3), slots=slots, budget_bytes=budget, executor=fake_executor(log, lock))
    res = srv.run(reqs, realtime=False)
    assert sorted(res) == list(range(40))
    assert srv.scheduler.peak_running <= slots
    assert srv.scheduler.peak_bytes <= budget
    starts = [rid for kind, rid, _ in sorted(log, key=lambda e: e[2]) if kind == "start"]
    assert starts == sorted(starts)          # FIFO admission
    s = summarize(res)
    assert s["requests"] == 40 and s["converged"] == 40


def test_oversized_request_runs_alone():
    log, lock = [], threading.Lock()
    reqs = [FakeReq(0, 2), FakeReq(1, 50), FakeReq(2, 2)]
    srv = SolveServer(np.eye(3), slots=3, budget_bytes=10, executor=fake_executor(log, lock))
    res = srv.run(reqs, realtime=False)
    assert sorted(res) == [0, 1, 2]
    assert srv.scheduler.peak_bytes == 50   # admitted when nothing else ran


def test_continuous_admission_overlaps_requests():
    """Requests arriving while others run are admitted as slots free up."""
    log, lock = [], threading.Lock()
    reqs = [FakeReq(i, 1, arrival=0.002 * i, service=0.03) for i in range(8)]
    srv = SolveServer(np.eye(3), slots=4, budget_bytes=100, executor=fake_executor(log, lock))
    t0 = time.perf_counter()
    res = srv.run(reqs, realtime=True)
    wall = time.perf_counter() - t0
    assert srv.scheduler.peak_running == 4
    assert wall < 8 * 0.03 * 0.75           # overlapped, not one at a time
    assert all(r.start >= r.arrival - 1e-6 for r in res.values())


def test_scheduler_close_releases_waiters():
    sch = Scheduler(2, 10)
    out = []
    t = threading.Thread(target=lambda: out.append(sch.take(0)))
    t.start()
    sch.close()
    t.join(timeout=5)
    assert out == [None]
