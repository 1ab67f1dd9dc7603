"""Write the replay fixtures of the seeded workloads: the served request
trace and the batched instance list, as JSON.

The generators (frforge_b200.workloads.served_trace / c4_instances) are
seeded SplitMix64 streams; the fixtures pin them, so a change to a generator
shows up as a failing regression test rather than as a silently different
benchmark.

Usage: python tests/golden/make_traces.py
"""
import dataclasses
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from frforge_b200.workloads import c4_instances, served_trace  # noqa: E402


def main():
    out = {
        "served_trace": [dataclasses.asdict(r) for r in served_trace()],
        "batched_instances": [dataclasses.asdict(w) for w in c4_instances()],
    }
    with open(os.path.join(HERE, "workload_traces.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
