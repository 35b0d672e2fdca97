"""Each precision variant inverting first in a fresh process.

The round kernels exist once per synthesis precision and filter variant, each
with its own launch settings (the SVD kernel's shared-memory limit among
them).  A process that uses one variant only must find that variant's
settings made: inside one pytest process an earlier test has usually set up
another variant, which can hide a launch that picks the wrong one.  So each
case runs in a subprocess of its own.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = """
import sys
sys.path[:0] = [{pkg!r}, {root!r}]
import numpy as np
import me_b200, me_maps
name = {name!r}
lam = me_maps.wavelengths(name)
cfg = me_b200.parse_config_text(me_maps.control_text(name, precision={prec!r}))
with me_b200.Plan(cfg, lam, device=0) as plan:
    par = me_maps.draw_parameters(name, 64, 3)
    prof = me_maps.add_noise(plan.synthesize(par), {noise!r}, 3)
    res, st = plan.invert(prof)
assert st["valid"] == 64 and (res[:, 9] > 0).all(), st
print("ok", st["launches"])
"""


@pytest.mark.gpu
@pytest.mark.parametrize("name,prec,noise", [("fe15648_64x64", "FP64", 1e-3),
                                             ("fe15648_64x64", "FP32", 1e-3),
                                             ("fe6173_4096x4096", "FP64", 2e-3),
                                             ("fe6173_4096x4096", "FP32", 2e-3)])
def test_inversion_in_a_fresh_process(name, prec, noise):
    code = SCRIPT.format(pkg=os.path.join(ROOT, "milne-eddington_b200"), root=ROOT, name=name,
                         prec=prec, noise=noise)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok")
