"""bench.py's reference arm runs the reference's own C core and nothing of
this library: neither the bench process nor its spawned worker processes map
libme_b200.so, and the line it prints is the reference arm's."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libmeref.so")

pytestmark = pytest.mark.skipif(not os.path.exists(REF),
                                reason="the reference's core is not built here")

PROBE = r"""
import json, pathlib, sys
sys.path.insert(0, {root!r})
import bench
pool = bench.CpuPool("fe15648_1024x1024", 2, 8, True)
_, prof = bench.sample_profiles(pool, "fe15648_1024x1024", 1048576, 8, 0)
res, _ = pool.invert(prof)
worker_maps = pool.pool.map(pathlib.Path.read_text, [pathlib.Path("/proc/self/maps")] * 4)
pool.close()
own = pathlib.Path("/proc/self/maps").read_text()
print(json.dumps({{"kind": pool.kind, "inverted": int((res[:, 9] > 0).sum()),
                  "workers_ref": all("libmeref.so" in m for m in worker_maps),
                  "workers_lib": any("libme_b200.so" in m for m in worker_maps),
                  "main_lib": "libme_b200.so" in own}}))
"""


def test_reference_arm_loads_nothing_of_the_library():
    out = subprocess.run([sys.executable, "-c", PROBE.format(root=ROOT)], capture_output=True,
                         text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    got = json.loads(out.stdout.strip().splitlines()[-1])
    assert got["kind"] == "reference" and got["inverted"] > 0
    assert got["workers_ref"], "the workers run the reference's core"
    assert not got["workers_lib"] and not got["main_lib"], got


def test_reference_arm_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                          "--warmup", "1", "--sample", "16"], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    assert line["config"]["workload"] == "fe15648_1024x1024"
