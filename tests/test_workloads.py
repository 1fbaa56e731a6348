"""The seeded synthetic workloads the bench and the GPU tests build (host
side only): deterministic, and with the shapes and parameter ranges their
descriptions state."""
import math

import numpy as np

from omega_h_v1_b200 import workloads as W


def test_serving_stream_mix_and_ranges():
    jobs = W.serving_stream()
    assert len(jobs) == 200
    assert [j.index for j in jobs] == list(range(200))
    arrivals = [j.arrival for j in jobs]
    assert all(b > a for a, b in zip(arrivals, arrivals[1:]))
    # Poisson arrivals at 200/s: 200 jobs in about a second
    assert 0.5 < arrivals[-1] < 2.0
    front = [j for j in jobs if j.front is not None]
    uniform = [j for j in jobs if j.front is None]
    assert 60 < len(front) < 140 and len(front) + len(uniform) == 200
    for j in uniform:
        assert j.radial is None
        assert 1.0 / j.n <= j.size <= 1.6 / j.n
    for j in front:
        offset, weight, min_h, max_h = j.front
        assert j.size == 0.0 and j.radial is None
        assert 0.3 <= offset <= 0.7
        assert math.isclose(min_h, 0.5 / j.n) and math.isclose(max_h, 2.0 / j.n)
        assert math.isclose(weight, (max_h - min_h) / 2000.0)
        assert j.estimated_output_tets() > 0
    for j in jobs:
        assert j.n >= 2 and j.tets == 6 * j.n ** 3
        assert j.tets <= 2.2e6


def test_workloads_are_deterministic():
    a, b = W.serving_stream(), W.serving_stream()
    assert a == b
    assert W.batched_boxes() == W.batched_boxes()
    assert W.serving_stream(seed=3) != a


def test_batched_boxes_ranges():
    jobs = W.batched_boxes()
    assert len(jobs) == 512
    for j in jobs:
        assert 4 <= j.n <= 40
        assert 0.3 / j.n <= j.size <= 1.5 / j.n
        assert j.estimated_output_tets() >= 0.5 * j.tets


def test_front_field_zero_level():
    y = np.linspace(0.0, 1.0, 11)
    offset = 0.45
    x0 = offset + 0.1 * np.sin(2.0 * np.pi * y)
    on = np.stack([x0, y, np.zeros_like(y)], axis=1)
    u = W.front_field(on, offset)
    assert np.all(np.abs(u) < 1e-12)
    left = W.front_field(on - [0.05, 0.0, 0.0], offset)
    right = W.front_field(on + [0.05, 0.0, 0.0], offset)
    assert np.all(left < -0.9) and np.all(right > 0.9)


def test_serving_routing_assigns_every_job_once_in_arrival_order():
    from omega_h_v1_b200 import workloads as W
    jobs = W.serving_stream(200, seed=2, rate=200.0)
    for nb in (1, 2, 4, 8):
        bins = W.route_stream(jobs, nb)
        assert sorted(i for b in bins for i in b) == list(range(len(jobs)))
        for b in bins:
            assert [jobs[i].arrival for i in b] == sorted(jobs[i].arrival for i in b)
        loads = [sum(jobs[i].estimated_output_tets() for i in b) for b in bins]
        biggest = max(j.estimated_output_tets() for j in jobs)
        assert max(loads) - min(loads) <= biggest
