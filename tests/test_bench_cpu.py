"""bench.py helpers that run without a GPU: the batched workload's instance draw and the all-core
reference sample (two host processes on a tiny mesh)."""

import math

import pytest

import bench
from oracle import ref


def test_batch_specs_are_seeded_and_in_range():
    a = bench.batch_specs(32)
    assert a == bench.batch_specs(32)
    for n, mach, angle, seed in a:
        assert 8 <= n <= 50
        assert 0.3 <= mach <= 3.0 and 0.0 <= angle <= 10.0
    cells = [4.64 * n ** 3 for n, *_ in a]
    assert min(cells) >= 8_000 * 0.5 and max(cells) <= 512_000 * 1.5
    assert len({s for *_, s in a}) == len(a)


@pytest.mark.skipif(not ref.available(), reason="reference oracle not built")
def test_all_core_reference_sample_runs():
    value, wall, steps, procs = bench.reference_cpu_all(6, 2, "tgv", procs=2)
    assert procs == 2 and steps == 2
    assert value > 0 and math.isfinite(value) and wall > 0
