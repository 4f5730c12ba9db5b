"""Scheduler of the solve server on the host, with a fake executor (no GPU): admission by memory
budget and slots, arrival order, failure isolation."""

import threading
import time

import pytest

from teal_b200 import serving


def make(n, arrival=0.0, cells=(40, 20, 2)):
    return [serving.Request(id=i, cells=cells, arrival=arrival + 0.001 * i) for i in range(n)]


class FakeExec:
    def __init__(self, seconds=0.02, fail_ids=()):
        self.seconds = seconds
        self.fail_ids = set(fail_ids)
        self.lock = threading.Lock()
        self.running = 0
        self.peak = 0
        self.order = []

    def __call__(self, req):
        with self.lock:
            self.running += 1
            self.peak = max(self.peak, self.running)
            self.order.append(req.id)
        try:
            t_end = time.perf_counter() + self.seconds
            while time.perf_counter() < t_end and not req.cancelled:
                time.sleep(0.002)
            if req.id in self.fail_ids:
                raise RuntimeError("device fault injected on the host")
            req.iterations = req.steps
        finally:
            with self.lock:
                self.running -= 1


def test_admission_respects_memory_budget():
    reqs = make(6)
    per = serving.memory_estimate(reqs[0])
    ex = FakeExec()
    s = serving.Scheduler(budget_bytes=int(2.5 * per), max_active=8, execute=ex)
    done = s.run(reqs, timeout=30)
    assert len(done) == 6 and all(not r.error for r in done)
    assert ex.peak <= 2 and s.peak_active <= 2
    assert s.peak_used <= s.budget
    assert s.used == 0


def test_slot_limit_and_arrival_order():
    reqs = make(5)
    ex = FakeExec()
    s = serving.Scheduler(budget_bytes=1 << 40, max_active=1, execute=ex)
    done = s.run(reqs, timeout=30)
    assert ex.order == [0, 1, 2, 3, 4]
    assert all(r.admitted >= r.arrival for r in done)
    assert all(r.latency > 0 for r in done)


def test_failing_request_is_isolated():
    reqs = make(4)
    ex = FakeExec(fail_ids={1})
    s = serving.Scheduler(budget_bytes=1 << 40, max_active=2, execute=ex)
    done = s.run(reqs, timeout=30)
    assert "injected" in done[1].error
    assert all(not r.error for i, r in enumerate(done) if i != 1)
    assert s.used == 0 and not s.active


def test_oversized_request_is_rejected():
    big = serving.Request(id=0, cells=(2000, 2000, 100))
    small = serving.Request(id=1, cells=(10, 10, 2), arrival=0.001)
    s = serving.Scheduler(budget_bytes=1 << 30, max_active=2, execute=FakeExec())
    done = s.run([big, small], timeout=30)
    assert "budget" in done[0].error
    assert not done[1].error


def test_late_arrivals_are_admitted_while_others_run():
    reqs = make(2) + [serving.Request(id=2, cells=(40, 20, 2), arrival=0.03)]
    ex = FakeExec(seconds=0.1)
    s = serving.Scheduler(budget_bytes=1 << 40, max_active=4, execute=ex)
    done = s.run(reqs, timeout=30)
    assert ex.peak == 3  # the late request joined the two running ones


def test_poisson_requests_are_seeded():
    a = serving.poisson_requests(8, rate=10.0, seed=3)
    b = serving.poisson_requests(8, rate=10.0, seed=3)
    assert [(r.cells, r.mach, r.flux, r.arrival) for r in a] == [(r.cells, r.mach, r.flux, r.arrival) for r in b]
    assert all(20_000 * 0.8 <= r.num_cells <= 2_000_000 * 1.2 for r in a)
    assert serving.percentile([1, 2, 3, 4], 50) == pytest.approx(2.5)


def test_cancel_waiting_and_running_requests():
    reqs = make(4)
    ex = FakeExec(seconds=0.3)
    s = serving.Scheduler(budget_bytes=1 << 40, max_active=1, execute=ex)
    s.cancel(3)  # not yet arrived: never runs
    timer = threading.Timer(0.05, lambda: (s.cancel(0), s.cancel(2)))  # 0 running, 2 waiting
    timer.start()
    done = s.run(reqs, timeout=30)
    timer.join()
    assert [r.error for r in done] == ["cancelled", "", "cancelled", "cancelled"]
    assert ex.order == [0, 1]
    assert done[0].finished < 0.3  # the running request stopped early
    assert s.used == 0 and not s.active
