"""The host logic of bench.py's end-to-end measurement on CPU, with stand-in handles: jobs go through
the resident handles, one vca_ca_run at a time (each job computes alone), while another handle's
upload and download overlap it; every job runs once, and the phase medians and step sums add up."""
from __future__ import annotations

import os
import sys
import time

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


class FakeHandle:
    """Records the time intervals of its runs and downloads; run() and download() take set times."""

    def __init__(self, spans, run_s=0.03, copy_s=0.02, steps=7, fail_at=None):
        self.spans = spans
        self.run_s, self.copy_s, self.steps, self.fail_at = run_s, copy_s, steps, fail_at
        self.runs = 0

    def reset(self):
        pass

    def apply_terrain(self, heights):
        pass

    def place_seeds(self, vents):
        pass

    def run(self):
        self.runs += 1
        if self.fail_at == self.runs:
            raise RuntimeError("run failed")
        t0 = time.perf_counter()
        time.sleep(self.run_s)
        self.spans.append(("run", id(self), t0, time.perf_counter()))

    def download(self, out):
        t0 = time.perf_counter()
        time.sleep(self.copy_s)
        self.spans.append(("copy", id(self), t0, time.perf_counter()))

    def info(self):
        class I:  # noqa: E742
            steps = self.steps
        return I()


def fake_e2e(n_handles, **kw):
    e = object.__new__(bench.E2E)
    spans = []
    e.slots = [(FakeHandle(spans, **kw), None) for _ in range(n_handles)]
    e.heights, e.vents = None, []
    return e, spans


def overlaps(a, b):
    return a[2] < b[3] and b[2] < a[3]


def test_two_in_flight_run_one_at_a_time_and_overlap_copies():
    e, spans = fake_e2e(2)
    wall, steps, med = e.jobs(6)
    assert steps == 6 * 7
    assert sum(h.runs for h, _ in e.slots) == 6
    runs = [s for s in spans if s[0] == "run"]
    copies = [s for s in spans if s[0] == "copy"]
    assert not any(overlaps(a, b) for i, a in enumerate(runs) for b in runs[i + 1:]), "two runs at once"
    assert any(overlaps(c, r) for c in copies for r in runs if r[1] != c[1]), "no download overlapped a run"
    assert wall >= 6 * 30  # the runs are serialised
    assert set(med) == {"prep_ms", "run_ms", "download_ms"} and med["run_ms"] >= 25


def test_one_handle_is_the_plain_sequence():
    e, spans = fake_e2e(1)
    wall, steps, _ = e.jobs(3)
    assert steps == 21 and len(spans) == 6
    assert not any(overlaps(a, b) for i, a in enumerate(spans) for b in spans[i + 1:])
    assert wall >= 3 * (30 + 20)


def test_a_failing_job_is_raised():
    e, _ = fake_e2e(2, fail_at=2)
    with pytest.raises(RuntimeError, match="run failed"):
        e.jobs(6)
