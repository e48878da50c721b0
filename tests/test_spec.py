"""Speculative negotiation rounds (csrc/spec.cu): route_waves' fixed-order commit with speculation, on the device.

The contract (src/router.cpp:2096-2118): whatever nets are searched together and however many searches are thrown
away, the committed paths are those of routing the nets one by one in order. The oracle (oracle/spec_oracle.py)
routes them one by one on the CPU; the device must give the same paths with the sequential, plain and any other
batch composition.
"""
import numpy as np
import pytest

from oracle import spec_oracle
from pcbroute_b200 import spec


def _small(seed):
    return spec.spec_board(seed, nx=96, ny=80, nl=3, nnets=28, margin=8, span=(10, 45))


@pytest.mark.parametrize("seed", [1, 2])
def test_oracle_paths_are_connected(seed):
    b = _small(seed)
    paths = spec_oracle.negotiate(b, 1, pres_of=spec.pres_of)
    nx, n = b["nx"], b["n"]
    for (x0, y0, x1, y1, s, t), p in zip(b["nets"], paths):
        assert len(p) >= 2 and p[0] == t and p[-1] == s
        for a, c in zip(p[:-1], p[1:]):
            la, ca = divmod(int(a), n)
            lc, cc = divmod(int(c), n)
            if la == lc:
                assert max(abs(ca % nx - cc % nx), abs(ca // nx - cc // nx)) == 1
            else:
                assert ca == cc
            assert x0 <= cc % nx < x1 and y0 <= cc // nx < y1


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [1, 2])
def test_device_rounds_match_the_sequential_oracle(gpu, seed):
    b = _small(seed)
    ref = spec_oracle.negotiate(b, 3, pres_of=spec.pres_of)
    got, stats = spec.negotiate(b, 3, spec.SEQUENTIAL, 1)
    assert all(s["wasted"] == 0 for s in stats)
    for k, (g, r) in enumerate(zip(got, ref)):
        assert np.array_equal(g, r), k


@pytest.mark.gpu
@pytest.mark.parametrize("width", [4, 16])
def test_speculation_never_changes_the_paths(gpu, width):
    """Plain speculation and a random batch composition commit the sequential paths, with searches wasted."""
    b = spec.spec_board(7, nx=128, ny=112, nl=4, nnets=48, margin=10, span=(12, 60))
    seq, s0 = spec.negotiate(b, 2, spec.SEQUENTIAL, 1)
    plain, s1 = spec.negotiate(b, 2, spec.PLAIN, width)
    rng = np.random.default_rng(width)

    def attach(r):
        r.set_scheduler(lambda cursor, cand: [c for c in cand if rng.random() < 0.5])

    rand, s2 = spec.negotiate(b, 2, spec.LEARNED, width, scheduler=attach)
    for k in range(len(seq)):
        assert np.array_equal(seq[k], plain[k]), k
        assert np.array_equal(seq[k], rand[k]), k
    assert sum(s["wasted"] for s in s1) > 0
    assert sum(s["batches"] for s in s1) < sum(s["batches"] for s in s0)
    assert all(s["commits"] == len(b["nets"]) for s in s0 + s1 + s2)
