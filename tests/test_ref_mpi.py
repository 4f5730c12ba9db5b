"""The all-core CPU baseline: teal's own domain-decomposed Taylor-Green run (oracle/_ref/teal_ref_mpi)
over the fork / shared-memory MPI subset (oracle/shim/shim_mpi_fork.c).

Its split into ranks is teal's mesh_create Cartesian decomposition with halo exchanges, so every
rank count must reproduce the one-rank run: the same global cell count and time, and residuals that
differ only by the order of the global sums (and the last-ulp differences of node coordinates that
the split computes per rank).
"""

import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MPI_RUN = os.path.join(ROOT, "oracle", "_ref", "teal_ref_mpi")

pytestmark = pytest.mark.skipif(not os.path.exists(MPI_RUN), reason="oracle/_ref/teal_ref_mpi not built")


def run(ranks, n=12, steps=3, warmup=1, **env):
    e = dict(os.environ, TEAL_SHIM_RANKS=str(ranks), TEAL_SHIM_TIMEOUT="60", **env)
    r = subprocess.run([MPI_RUN, "--n", str(n), "--steps", str(steps), "--warmup", str(warmup)],
                       capture_output=True, text=True, env=e, timeout=120)
    return r


def result(ranks, **kw):
    r = run(ranks, **kw)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout  # rank 0 alone prints
    return json.loads(lines[0])


@pytest.mark.parametrize("ranks", [2, 3, 4, 8])
def test_ranks_reproduce_one_rank(ranks):
    one = result(1)
    many = result(ranks)
    assert many["ranks"] == ranks
    assert many["cells"] == one["cells"] == 12**3
    assert many["steps"] == one["steps"] == 3
    assert many["seconds"] > 0
    assert many["time"] == pytest.approx(one["time"], rel=1e-12)
    np.testing.assert_allclose(many["residual"], one["residual"], rtol=1e-10)


def test_uneven_split():
    # 10 cells per axis over 5 ranks: teal's split gives the ranks unequal slabs
    one = result(1, n=10)
    five = result(5, n=10)
    assert five["cells"] == one["cells"] == 1000
    np.testing.assert_allclose(five["residual"], one["residual"], rtol=1e-10)


def test_invalid_rank_count_fails_fast():
    r = run(0)
    assert r.returncode != 0
    assert "TEAL_SHIM_RANKS" in r.stderr


def test_small_ring_rejects_large_message():
    # a 1 MiB inbox cannot take an 80^3 gradient halo message (80 x 80 cells x 15 values, 768 KB,
    # over half the ring): the run stops with a message, all ranks end (no rank is left waiting)
    r = run(2, n=80, steps=1, warmup=0, TEAL_SHIM_RING_MB="1")
    assert r.returncode != 0
    assert "inbox ring" in r.stderr
