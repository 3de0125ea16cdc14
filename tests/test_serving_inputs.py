"""The seeded serving workload (markovkit_b200.inputs.serving_requests) that bench.py replays:
deterministic, Poisson arrivals in order, models and sizes in the ranges the serving
configuration names, 1-D boxes whose grid halves down to at most 16 voxels."""

import math

import numpy as np

from markovkit_b200.inputs import SERVING_MODELS, serving_requests


def _states(r):
    if r["model"] == "cfg1":
        return (r["voxels"] + 1) ** 2  # box {1, 1}: (1 + V)^2 states
    return math.comb(r["voxels"] + r["cap"], r["cap"])


def test_deterministic_and_ordered():
    a, b = serving_requests(), serving_requests()
    assert a == b
    t = [r["arrival_s"] for r in a]
    assert all(x < y for x, y in zip(t, t[1:]))
    assert len({r["rhs_seed"] for r in a}) == len(a)


def test_ranges():
    reqs = serving_requests(count=400)
    assert {r["model"] for r in reqs} == set(SERVING_MODELS)
    for r in reqs:
        assert 0.1 <= r["shift"] <= 10.0
        if r["model"] == "bd1d":
            V = r["voxels"]
            assert 64 <= V <= 256 and V % 16 == 0
            assert 2 <= r["cap"] <= 4
            # the multigrid halves an even axis; it stops at an odd length of at most 16
            while V % 2 == 0 and V > 1:
                V //= 2
            assert V <= 16
    sizes = [_states(r) for r in reqs]
    assert min(sizes) == 969 and max(sizes) <= 186_043_585
    assert max(sizes) == 186_043_585  # V = 256, cap 4 is drawn at this count


def test_poisson_rate():
    reqs = serving_requests(count=4000, rate=20.0)
    gaps = np.diff([0.0] + [r["arrival_s"] for r in reqs])
    assert abs(gaps.mean() - 1 / 20.0) < 0.1 / 20.0
    # exponential: the standard deviation equals the mean
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.1
