"""The algorithmic operation counts behind bench.py's rooflines
(tests/golden/flop_counts.json) are reproducible: the oracle, instantiated
with a counting scalar type, gives the committed per-event figures again for
the headline map and the small map."""
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_flop_counts  # noqa: E402


@pytest.mark.parametrize("name", ["fe15648_1024x1024", "fe15648_64x64"])
def test_flop_counts_reproduce(name):
    want = json.load(open(os.path.join(HERE, "golden", "flop_counts.json")))[name]
    got = make_flop_counts.workload_counts(name)
    assert got["nl"] == want["nl"] and got["samples"] == want["samples"]
    for event, c in want.items():
        if not isinstance(c, dict):
            continue
        for op, v in c.items():
            assert got[event][op] == pytest.approx(v, rel=1e-12, abs=1e-9), (event, op)
