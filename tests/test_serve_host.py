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


def test_job_configs_pass_the_engine_validation(tmp_path):
    """Every job of a mix is an engine config in the reference's schema that the engine's own
    validation accepts (engine --validate: the same parser as a run)."""
    import json
    import os
    import subprocess

    from volcano_ca_mc_b200 import capi
    if not os.path.exists(capi.ENGINE_PATH):
        import pytest
        pytest.skip("engine not built")
    for j in serve.make_mix(12, 13, side_2d=(64, 256), side_3d=(32, 64)):
        path = tmp_path / f"job{j.job_id}.json"
        path.write_text(json.dumps(j.config(str(tmp_path))))
        r = subprocess.run([capi.ENGINE_PATH, "--validate", "--config", str(path)], capture_output=True, text=True)
        out = json.loads(r.stdout)
        assert r.returncode == 0 and out["ok"], out


def test_server_answers_refused_requests_without_a_gpu():
    """engine --serve answers each request line; refused configs come back as errors with the
    reference's message texts, the rest of the stream goes on, the summary counts them (exit code 5)."""
    import os

    import pytest

    from volcano_ca_mc_b200 import capi
    if not os.path.exists(capi.ENGINE_PATH):
        pytest.skip("engine not built")
    srv = serve.EngineServer(slots=2, batched=False)
    srv.submit({"id": "a", "json": {"space": {"nx": 0}}})
    srv.submit({"id": "b", "json": {"neighborhood": "hexagonal", "space": {"nx": 40, "ny": 30, "nz": 20}}})
    srv.submit({"id": "c", "config": "does/not/exist.json"})
    assert srv.close() == 5
    assert srv.answers["a"]["error"].startswith("Błąd konfiguracji: Parametr „space.nx” musi być z zakresu")
    assert "hexagonal" in srv.answers["b"]["error"]
    assert "Nie można otworzyć pliku konfiguracyjnego" in srv.answers["c"]["error"]
    assert srv.summary["failed"] == 3 and srv.summary["jobs"] == 0


def test_phase_sums_add_the_answers_sections():
    """The per-mode phase sums of the bench: every answer's times_ms sections added up; answers
    without times (refused requests) add nothing."""
    recs = [{"times_ms": {"caSim": 2.5, "save": 1.0, "digest": 0.25}},
            {"times_ms": {"caSim": 1.5, "mcSim": 3.0, "digest": 0.75}},
            {"status": "error"}]
    assert serve.phase_sums(recs) == {"caSim": 4.0, "save": 1.0, "digest": 1.0, "mcSim": 3.0}
    assert serve.phase_sums([]) == {}
