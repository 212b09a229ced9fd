"""Host logic of the job server (no GPU): the job mixes are seeded and follow the benchmark
distribution, terrains and vents are valid, arrival times are a Poisson trace."""
from __future__ import annotations

import numpy as np

from volcano_ca_mc_b200 import serve


def test_mix_is_seeded_and_in_range():
    a = serve.make_mix(96, 7)
    b = serve.make_mix(96, 7)
    assert [(j.nx, j.ny, j.nz, j.seed, j.neighborhood) for j in a] == [(j.nx, j.ny, j.nz, j.seed, j.neighborhood) for j in b]
    for j in a:
        if j.ny == 1:
            assert 128 <= j.nx <= 2048 and 128 <= j.nz <= 2048
        else:
            assert 64 <= j.nx <= 256 and j.ny == j.nx and j.nz == max(8, j.nx // 2)
            assert j.neighborhood != "hexagonal"
        assert 200 <= j.max_steps <= 600 and 20 <= j.mcs <= 100 and 1 <= j.n_vents <= 8 and j.Q in (32, 64, 128)
    share3 = np.mean([j.ny > 1 for j in serve.make_mix(2000, 3)])
    assert 0.25 < share3 < 0.35


def test_terrain_and_vents_valid():
    for j in serve.make_mix(20, 11, side_2d=(64, 256), side_3d=(32, 64)):
        h, vents = j.terrain()
        assert h.shape == (j.nx * j.ny,) and h.min() >= 0 and h.max() <= j.nz
        hm = h.reshape(j.ny, j.nx)
        for (x, y, z, f) in vents:
            assert 0 <= x < j.nx and 0 <= y < j.ny and z == hm[y, x] and z < j.nz


def test_poisson_arrivals():
    jobs = serve.make_mix(4000, 5, rate_hz=20.0)
    t = np.array([j.arrival_s for j in jobs])
    assert np.all(np.diff(t) >= 0)
    rate = len(t) / t[-1]
    assert 18.0 < rate < 22.0


def test_capacity_covers_every_job():
    jobs = serve.make_mix(50, 2, share_3d=0.0, side_2d=(64, 512))
    cap = serve.capacity(jobs)
    for j in jobs:
        assert j.nx <= cap.nx and j.ny <= cap.ny and j.nz <= cap.nz and j.max_steps <= cap.max_steps
