"""The entry point that allocates nothing (me_invert_batch_device_noalloc).

It is for callers that cannot allocate device memory while they invert:
pipelines and frameworks that reserve the GPU's memory for their own pool when
they start, and real-time loops at the instrument that cannot afford the device
synchronisation cudaMalloc / cudaFree may bring.  All of its scratch sits in a
fixed static device array, so it takes at most 65536 pixels per call, 8192 of
them in flight.

These tests call it through the C ABI and compare it with the allocating entry
point me_invert_batch_device on the same profiles, for two calls in a row that
continue one map (the second call starts from the LM chi^2 the first one
carried out), in both synthesis precisions; with a strong theta regularisation
that makes the carried chi^2 flip pixels' first ratio test, so that both entry
points re-run pixels; and for the largest batch, where every one of the 8192
slots serves eight pixels.  Both run the same one-thread-per-pixel round
kernels, so the results must agree to 1e-12 (in practice bit for bit).

The file name sorts it after every other test, so a run that stops at the
first failure has run the rest first.
"""
import numpy as np
import pytest

import me_b200
import me_maps

pytestmark = pytest.mark.gpu

NAME = "fe15648_64x64"
REGUL = {"Btheta_Regularization": "YES, 0.5, 1"}


def _map(npix, seed):
    """Seeded noisy profiles on the device, one pixel under Icriteria."""
    import torch
    lam = me_maps.wavelengths(NAME)
    gen = me_b200.Plan(me_b200.parse_config_text(me_maps.control_text(NAME, precision="FP64")),
                       lam)
    par = torch.from_numpy(me_maps.draw_parameters(NAME, npix, seed)).cuda()
    prof = torch.empty((npix, 4, lam.size), dtype=torch.float64, device="cuda")
    gen.synthesize_device(par.data_ptr(), npix, prof.data_ptr())
    gen.close()
    g = torch.Generator(device="cuda").manual_seed(seed)
    prof += 1e-3 * torch.randn(prof.shape, dtype=torch.float64, device="cuda", generator=g)
    prof[17] *= 1e-5  # a pixel under Icriteria: zeros from both entry points
    torch.cuda.synchronize()
    return lam, prof


def _compare(cfg, lam, prof, calls, per_call):
    """The map in `calls` consecutive calls of `per_call` pixels through both
    entry points; returns (no-alloc results, allocating results, carried chi^2
    of each, pixels the allocating path re-ran for the carried chi^2)."""
    import torch
    n = calls * per_call
    res_ref = torch.zeros((n, 10), dtype=torch.float64, device="cuda")
    redo = 0
    with me_b200.Plan(cfg, lam) as plan:
        # the no-alloc entry point runs one-thread-per-pixel LM rounds to the
        # end; the plan's lane-split rounds and tail kernel (the same
        # arithmetic up to summation order and multiply-add contraction) are
        # switched off so that the two can be compared bit for bit
        plan.tail_slots = 0
        plan.max_group = 1
        plan.carry_chisq = 0.0
        for c in range(calls):
            sl = slice(c * per_call, (c + 1) * per_call)
            st = plan.invert_device(prof[sl].data_ptr(), per_call, res_ref[sl].data_ptr())
            redo += st["redo_pixels"]
        carry_ref = plan.carry_chisq
    res = torch.full((n, 10), -1.0, dtype=torch.float64, device="cuda")
    carry = 0.0
    for c in range(calls):
        sl = slice(c * per_call, (c + 1) * per_call)
        carry = me_b200.invert_device_noalloc(cfg, lam, prof[sl].data_ptr(), per_call,
                                              res[sl].data_ptr(), carry)
    torch.cuda.synchronize()
    return res.cpu().numpy(), res_ref.cpu().numpy(), carry, carry_ref, redo


@pytest.mark.parametrize("regul", [False, True], ids=["default", "strong_theta_regul"])
@pytest.mark.parametrize("prec", ["FP32", "FP64"])
def test_noalloc_matches_allocating_entry_point_two_calls(prec, regul):
    lam, prof = _map(6000, 31)
    cfg = me_b200.parse_config_text(me_maps.control_text(NAME, precision=prec, seed=11,
                                                         extra=REGUL if regul else None))
    a, b, carry, carry_ref, redo = _compare(cfg, lam, prof, 2, 3000)
    assert np.all(a[17] == 0) and np.all(b[17] == 0)
    assert np.all(a[:, 9] >= 0)  # every pixel written (the buffer started at -1)
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)
    assert carry == pytest.approx(carry_ref, rel=1e-12, abs=1e-300)
    if regul:
        # the carried chi^2 flipped first ratio tests: pixels were re-run
        assert redo > 0
    print(f"{prec} regul={regul}: {a.shape[0]} pixels agree, re-run {redo}")


def test_noalloc_largest_batch_reuses_every_slot():
    """65536 pixels per call (the limit), twice: each of the 8192 slots takes
    eight pixels in turn, and the second call starts from the first call's
    state left in the shared array."""
    lam, prof = _map(2 * 65536, 47)
    cfg = me_b200.parse_config_text(me_maps.control_text(NAME, precision="FP32", seed=3))
    a, b, carry, carry_ref, _ = _compare(cfg, lam, prof, 2, 65536)
    assert np.all(a[:, 9] >= 0)
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)
    assert carry == pytest.approx(carry_ref, rel=1e-12, abs=1e-300)


def test_noalloc_rejects_oversized_batch():
    lam = me_maps.wavelengths(NAME)
    cfg = me_b200.parse_config_text(me_maps.control_text(NAME))
    with pytest.raises(me_b200.MeError) as e:
        me_b200.invert_device_noalloc(cfg, lam, 1, 65537, 1)
    assert e.value.status == -1 and "65536" in str(e.value)


def test_noalloc_keeps_the_cause_of_a_bad_grid():
    """A grid the plan set-up rejects keeps its own message in me_last_error."""
    lam = me_maps.wavelengths(NAME)
    cfg = me_b200.parse_config_text(me_maps.control_text(NAME))
    with pytest.raises(me_b200.MeError) as e:
        me_b200.invert_device_noalloc(cfg, lam[:3], 1, 16, 1)
    assert e.value.status == -1 and "nl must be in" in str(e.value)
