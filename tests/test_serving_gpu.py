"""Solve server on the GPU: requests that arrive while others run are admitted as memory frees up,
run concurrently on their own streams, and every result is the same bits as the request solved
alone."""

import numpy as np
import pytest

from teal_b200 import serving

pytestmark = pytest.mark.gpu


def test_served_results_equal_solo_results():
    reqs = serving.poisson_requests(6, rate=40.0, seed=11, min_cells=2_000, max_cells=40_000, steps=(10, 30))
    budget = 3 * max(serving.memory_estimate(r) for r in reqs)
    server = serving.Server(budget_bytes=budget, max_active=3)
    done = server.serve(reqs, timeout=300)
    assert all(not r.error for r in done), [r.error for r in done]
    assert server.scheduler.peak_active <= 3
    lat = [r.latency for r in done]
    assert serving.percentile(lat, 99) >= serving.percentile(lat, 50) > 0
    for r in done:
        solo = serving.Request(**{k: getattr(r, k) for k in ("id", "cells", "mach", "angle", "physics", "flux",
                                                              "limiter", "viscosity", "steps", "tolerance",
                                                              "courant", "precision")})
        serving.solve(solo)
        assert solo.iterations == r.iterations
        assert np.array_equal(solo.state, r.state)
        assert np.array_equal(solo.residual, r.residual)


def test_tolerance_stops_a_request_early():
    r = serving.Request(id=0, cells=(24, 12, 2), mach=0.5, steps=400, tolerance=1e-1)
    serving.solve(r)
    assert 1 < r.iterations < 400


def test_cancelled_request_stops_early():
    import threading

    server = serving.Server(max_active=2)
    reqs = [serving.Request(id=0, cells=(200, 100, 2), steps=200000, arrival=0.0),
            serving.Request(id=1, cells=(40, 20, 2), steps=20, arrival=0.0)]

    def cancel_once_running():
        import math
        import time

        for _ in range(3000):
            if not math.isnan(reqs[0].admitted) and server.scheduler.cancel(0):
                return
            time.sleep(0.01)

    timer = threading.Thread(target=cancel_once_running)
    timer.start()
    done = server.serve(reqs, timeout=300)
    timer.join()
    assert done[0].error == "cancelled" and done[0].iterations < 200000
    assert not done[1].error and done[1].iterations == 20
    assert server.scheduler.used == 0
