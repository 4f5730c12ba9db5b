"""Solve server on the GPU.

`Server` batches continuously: requests of one scheme share a lane whose arena advances all of them
in shared launches; requests that arrive while others run join the arena between rounds (it is
re-packed with every running request's exact state and clock), finished ones leave. Every result
must be the same bits as the request solved alone, whether it ran alone, joined a running batch or
saw others join and leave around it. `StreamServer` (a context and stream per request) is checked
the same way.
"""

import dataclasses
import math
import threading
import time

import numpy as np
import pytest

from teal_b200 import _lib, serving

pytestmark = pytest.mark.gpu

FIELDS = ("id", "cells", "mach", "angle", "physics", "flux", "limiter", "viscosity", "steps", "tolerance", "courant",
          "precision", "method", "mesh", "seed")


def alone(r):
    solo = serving.Request(**{k: getattr(r, k) for k in FIELDS})
    serving.solve(solo)
    return solo


def check_against_solo(done):
    for r in done:
        assert not r.error, (r.id, r.error)
        solo = alone(r)
        assert solo.iterations == r.iterations, r.id
        assert np.array_equal(solo.state, r.state), r.id
        assert np.array_equal(solo.residual, r.residual), r.id


def test_requests_joining_a_running_batch_keep_their_solo_bits():
    # one lane (same scheme): a long request first, then shorter ones arriving while it runs, one of
    # them stopping on its tolerance; a second lane (another flux) and an implicit lane alongside
    reqs = [
        serving.Request(id=0, cells=(48, 24, 2), steps=600, arrival=0.0),
        serving.Request(id=1, cells=(30, 16, 2), steps=40, arrival=0.05, mach=0.8),
        serving.Request(id=2, cells=(24, 12, 2), steps=400, tolerance=1e-1, arrival=0.1),
        serving.Request(id=3, cells=(36, 12, 2), steps=30, arrival=0.15, angle=5.0),
        serving.Request(id=4, cells=(20, 20, 2), steps=50, arrival=0.05, flux="roe"),
        serving.Request(id=5, cells=(16, 10, 2), steps=6, arrival=0.02, method="implicit euler", courant=20.0,
                        limiter="venkatakrishnan"),
        serving.Request(id=6, cells=(14, 12, 2), steps=4, arrival=0.08, method="implicit euler", courant=20.0,
                        limiter="venkatakrishnan", mach=1.5),
    ]
    server = serving.Server(max_active=16, chunk=10)
    done = server.serve([dataclasses.replace(r) for r in reqs], timeout=600)
    assert len(server.lanes) == 3
    assert server.repacks > len(server.lanes)  # requests joined or left running arenas
    assert 1 < done[2].iterations < 400  # stopped by its tolerance
    lat = [r.latency for r in done]
    assert serving.percentile(lat, 99) >= serving.percentile(lat, 50) > 0
    check_against_solo(done)
    assert server.used == 0


def test_ramp_meshes_and_navier_stokes_requests():
    reqs = serving.poisson_requests(4, rate=50.0, seed=3, min_cells=3_000, max_cells=12_000, steps=(3, 6),
                                    mesh="ramp", physics=(_lib.TG_EULER, _lib.TG_NAVIERSTOKES),
                                    method="implicit euler", courant=10.0)
    server = serving.Server(max_active=8, chunk=2)
    done = server.serve(reqs, timeout=600)
    assert {r.physics for r in done} == {_lib.TG_EULER, _lib.TG_NAVIERSTOKES} or len(done) == 4
    check_against_solo(done)


def test_memory_budget_serialises_admission():
    reqs = [serving.Request(id=i, cells=(40, 20, 2), steps=30, arrival=0.0) for i in range(4)]
    budget = serving.memory_estimate(reqs[0]) + 1  # one request at a time
    server = serving.Server(budget_bytes=budget, max_active=8, chunk=10)
    done = server.serve(reqs, timeout=300)
    assert server.peak_active == 1
    assert all(not r.error for r in done)
    admitted = sorted(r.admitted for r in done)
    finished = sorted(r.finished for r in done)
    assert all(a >= f for a, f in zip(admitted[1:], finished[:-1]))


def test_stream_server_results_equal_solo_results():
    reqs = serving.poisson_requests(4, rate=40.0, seed=11, min_cells=2_000, max_cells=40_000, steps=(10, 30))
    budget = 3 * max(serving.memory_estimate(r) for r in reqs)
    server = serving.StreamServer(budget_bytes=budget, max_active=3)
    done = server.serve(reqs, timeout=300)
    assert server.scheduler.peak_active <= 3
    check_against_solo(done)


def test_tolerance_stops_a_request_early():
    r = serving.Request(id=0, cells=(24, 12, 2), mach=0.5, steps=400, tolerance=1e-1)
    serving.solve(r)
    assert 1 < r.iterations < 400


def test_cancelled_request_leaves_its_lane():
    server = serving.Server(max_active=4, chunk=10)
    reqs = [serving.Request(id=0, cells=(200, 100, 2), steps=200000, arrival=0.0),
            serving.Request(id=1, cells=(40, 20, 2), steps=20, arrival=0.0)]

    def cancel_once_running():
        for _ in range(3000):
            if not math.isnan(reqs[0].admitted) and server.cancel(0):
                return
            time.sleep(0.01)

    timer = threading.Thread(target=cancel_once_running)
    timer.start()
    done = server.serve(reqs, timeout=300)
    timer.join()
    assert done[0].error == "cancelled" and done[0].iterations < 200000
    assert not done[1].error and done[1].iterations == 20
    assert server.used == 0
