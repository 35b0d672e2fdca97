"""The C ABI library: it loads without a GPU, exports every entry point that
include/me_b200.h declares, and has no CPU path (compute entry points fail with
ME_ERR_NODEVICE when no device is visible)."""
import os
import re
import subprocess

import numpy as np
import pytest

import me_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "me_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(me_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_expected_entry_points():
    assert set(header_symbols()) == set(me_b200.EXPORTED)


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", me_b200.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (me_[a-z0-9_]+)", out))
    missing = set(header_symbols()) - exported
    assert not missing, missing


def test_version_and_strerror():
    L = me_b200.lib()
    assert b"sm_100a" in L.me_version()
    assert L.me_strerror(-5) == b"no CUDA device (no CPU fallback)"


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback_without_gpu():
    import me_maps
    cfg = me_b200.parse_config_text(me_maps.control_text("fe15648_64x64"))
    with pytest.raises(me_b200.MeError) as e:
        me_b200.Plan(cfg, me_maps.wavelengths("fe15648_64x64"))
    assert e.value.status == -5
    with pytest.raises(me_b200.MeError) as e:
        me_b200.faddeeva(6, np.zeros(3), np.ones(3))
    assert e.value.status == -5


def test_svd_u_rejects_bad_arguments_before_the_device():
    """The U-only decomposition's unit entry point checks its order and lane
    count before it looks for a device (ME_ERR_ARG), and without a GPU has no
    CPU path (ME_ERR_NODEVICE)."""
    a = np.eye(9)[None].copy()
    for kw in ({"lanes": 3}, {"lanes": 64}):
        with pytest.raises(me_b200.MeError) as e:
            me_b200.svd_u(a, **kw)
        assert e.value.status == -1 and "lanes" in str(e.value)
    with pytest.raises(me_b200.MeError) as e:
        me_b200.svd_u(np.eye(10)[None].copy())
    assert e.value.status == -1
    if not _has_gpu():
        with pytest.raises(me_b200.MeError) as e:
            me_b200.svd_u(a, lanes=4)
        assert e.value.status == -5
