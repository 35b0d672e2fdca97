"""The entry point that allocates nothing (me_invert_batch_device_noalloc).

It serves callers that cannot allocate device memory while they invert --
code running during another stream's graph capture, pipelines that have handed
their GPU memory to their own pool, real-time loops that must not block in the
allocator -- by keeping all of its scratch in a fixed static device array (at
most 65536 pixels per call).  This checks it through the C ABI against the
allocating entry point me_invert_batch_device on the same profiles, for two
calls in a row that continue one map (the second call starts from the LM chi^2
the first one carried out), with the tolerance of the other inversion tests
(the same kernels run in both, so the results should agree exactly).

The file name sorts it after every other test, so a run that stops at the
first failure has run the rest first.
"""
import numpy as np
import pytest

import me_b200
import me_maps

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_entry_point_two_calls():
    import torch
    name = "fe15648_64x64"
    lam = me_maps.wavelengths(name)
    cfg = me_b200.parse_config_text(me_maps.control_text(name, precision="FP32", seed=11))
    npix = 3000
    gen = me_b200.Plan(me_b200.parse_config_text(me_maps.control_text(name, precision="FP64")),
                       lam)
    par = torch.from_numpy(me_maps.draw_parameters(name, 2 * npix, 31)).cuda()
    prof = torch.empty((2 * npix, 4, lam.size), dtype=torch.float64, device="cuda")
    gen.synthesize_device(par.data_ptr(), 2 * npix, prof.data_ptr())
    gen.close()
    g = torch.Generator(device="cuda").manual_seed(5)
    prof += 1e-3 * torch.randn(prof.shape, dtype=torch.float64, device="cuda", generator=g)
    prof[17] *= 1e-5  # a pixel under Icriteria: zeros in both
    torch.cuda.synchronize()

    res_ref = torch.zeros((2 * npix, 10), dtype=torch.float64, device="cuda")
    with me_b200.Plan(cfg, lam) as plan:
        # the no-alloc entry point runs one-thread-per-pixel LM rounds to the
        # end; the plan's lane-split rounds and tail kernel (the same
        # arithmetic up to summation order and multiply-add contraction) are
        # switched off so that the two can be compared bit for bit
        plan.tail_slots = 0
        plan.max_group = 1
        plan.carry_chisq = 0.0
        for c in range(2):
            sl = slice(c * npix, (c + 1) * npix)
            plan.invert_device(prof[sl].data_ptr(), npix, res_ref[sl].data_ptr())
        carry_ref = plan.carry_chisq

    res = torch.full((2 * npix, 10), -1.0, dtype=torch.float64, device="cuda")
    carry = 0.0
    for c in range(2):
        sl = slice(c * npix, (c + 1) * npix)
        carry = me_b200.invert_device_noalloc(cfg, lam, prof[sl].data_ptr(), npix,
                                              res[sl].data_ptr(), carry)
    torch.cuda.synchronize()
    a = res.cpu().numpy()
    b = res_ref.cpu().numpy()
    assert np.all(a[17] == 0) and np.all(b[17] == 0)
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)
    assert carry == pytest.approx(carry_ref, rel=1e-12, abs=1e-300)


def test_noalloc_rejects_oversized_batch():
    name = "fe15648_64x64"
    lam = me_maps.wavelengths(name)
    cfg = me_b200.parse_config_text(me_maps.control_text(name))
    with pytest.raises(me_b200.MeError) as e:
        me_b200.invert_device_noalloc(cfg, lam, 1, 65537, 1)
    assert e.value.status == -1 and "65536" in str(e.value)
