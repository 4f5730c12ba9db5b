"""Raw state files of the run loop on the host (no GPU): round trip and rejection of a file written
for another mesh."""

import os

import numpy as np
import pytest

import teal_b200 as tb


def test_state_file_round_trip(tmp_path):
    m = tb.Mesh.create((0, 0, 0), (1, 1, 1), (6, 5, 4), (1, 1, 1))
    e = tb.Equations.euler(m)
    e.primitive[:] = np.random.default_rng(3).random(e.primitive.shape)
    saved = e.primitive.copy()
    sim = tb.Simulation(e)
    path = os.path.join(tmp_path, "s.tgstate")
    sim.save_state(path, 0.125, 7)
    e.primitive[:] = 0.0
    sim.load_state(path)
    assert np.array_equal(e.primitive, saved)
    assert sim.start_time == 0.125 and sim.start_index == 7


def test_state_file_of_another_mesh_is_rejected(tmp_path):
    a = tb.Equations.euler(tb.Mesh.create((0, 0, 0), (1, 1, 1), (6, 5, 4), (1, 1, 1)))
    path = os.path.join(tmp_path, "s.tgstate")
    tb.Simulation(a).save_state(path, 0.0, 0)
    b = tb.Equations.euler(tb.Mesh.create((0, 0, 0), (1, 1, 1), (4, 4, 4), (1, 1, 1)))
    with pytest.raises(tb.TealError):
        tb.Simulation(b).load_state(path)
    with open(path, "r+b") as f:
        f.write(b"X")
    with pytest.raises(tb.TealError):
        tb.Simulation(a).load_state(path)
