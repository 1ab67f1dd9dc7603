"""The seeded workload generators reproduce their committed replay fixtures
(tests/golden/workload_traces.json, written by tests/golden/make_traces.py)."""
import dataclasses
import json
import os

from frforge_b200.workloads import c4_instances, served_trace

HERE = os.path.dirname(os.path.abspath(__file__))


def _fixture():
    with open(os.path.join(HERE, "golden", "workload_traces.json")) as f:
        return json.load(f)


def test_served_trace_replays():
    ref = _fixture()["served_trace"]
    got = [dataclasses.asdict(r) for r in served_trace()]
    assert got == ref
    assert len(got) == 32 and all(0 < a["arrival"] < b["arrival"] for a, b in zip(got, got[1:]))


def test_batched_instances_replay():
    ref = _fixture()["batched_instances"]
    got = [dataclasses.asdict(w) for w in c4_instances()]
    assert got == ref
    assert len(got) == 64
    assert 600_000 < sum(w["n"] ** 2 for w in got) < 900_000
