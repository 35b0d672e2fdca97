"""me_invert_batch from page-locked host memory: the map goes to the device in
chunks and the inversion starts on the first chunk while the rest is on its
way (queue positions are taken only once their chunk has landed).

* One thread per pixel throughout (no lane-split rounds, no tail kernel), the
  plain LM: each pixel's steps do not depend on when it is taken, so the
  chunked copy gives the whole-copy results bit for bit.
* A learned start with the queue order: each chunk's guesses and order
  (sorted within the chunk) are made as it lands; the order in which pixels
  meet the kernels changes, so results agree with the whole copy to rounding.
* From pageable memory the map is copied whole (same results).
"""
import numpy as np
import pytest

import me_b200
import me_maps

pytestmark = pytest.mark.gpu

NAME = "fe15648_64x64"
NPIX = 3 * 65536 + 1000  # four chunks, the last one short


def _map(prec, seed=77):
    import torch
    lam = me_maps.wavelengths(NAME)
    gen = me_b200.Plan(me_b200.parse_config_text(me_maps.control_text(NAME, precision="FP64")),
                       lam)
    par = torch.from_numpy(me_maps.draw_parameters(NAME, NPIX, seed)).cuda()
    prof = torch.empty((NPIX, 4, lam.size), dtype=torch.float64, device="cuda")
    gen.synthesize_device(par.data_ptr(), NPIX, prof.data_ptr())
    gen.close()
    g = torch.Generator(device="cuda").manual_seed(seed)
    prof += 1e-3 * torch.randn(prof.shape, dtype=torch.float64, device="cuda", generator=g)
    prof[12345] *= 1e-5  # under Icriteria
    h = torch.empty(prof.shape, dtype=torch.float64, pin_memory=True)
    h.copy_(prof)
    cfg = me_b200.parse_config_text(me_maps.control_text(NAME, precision=prec, seed=5))
    return lam, cfg, h


@pytest.mark.parametrize("prec", ["FP32", "FP64"])
def test_chunked_copy_matches_whole_copy(prec):
    lam, cfg, h = _map(prec)
    hp = h.numpy()
    out = {}
    with me_b200.Plan(cfg, lam) as plan:
        plan.max_group, plan.tail_slots = 1, 0
        for feed in (False, True):
            plan.set_feed(feed)
            plan.carry_chisq = 0.0
            out[feed] = plan.invert(hp)
        # pageable input: copied whole, the same results again
        plan.carry_chisq = 0.0
        res_pageable, _ = plan.invert(np.array(hp))
    (a, st_a), (b, st_b) = out[False], out[True]
    assert st_a["valid"] == st_b["valid"] == NPIX - 1
    assert np.all(b[12345] == 0)
    assert np.array_equal(a, b)
    assert np.array_equal(a, res_pageable)


def test_chunked_copy_learned_start():
    lam, cfg, h = _map("FP32", seed=78)
    hp = h.numpy()
    with me_b200.Plan(cfg, lam) as plan:
        init = me_b200.Initializer.train(plan, samples=1 << 16, batch=4096, epochs=2,
                                         **me_maps.train_prior(NAME))
        plan.set_initializer(init)
        res = {}
        for feed in (False, True):
            plan.set_feed(feed)
            plan.carry_chisq = 0.0
            res[feed] = plan.invert(hp)
        init.close()
    (a, st_a), (b, st_b) = res[False], res[True]
    assert st_a["valid"] == st_b["valid"] == NPIX - 1
    assert st_b["init_ms"] > 0
    v = a[:, 9] > 0
    ratio = b[v, 9] / a[v, 9]
    same = np.mean(np.all(a == b, axis=1))
    print(f"learned start: identical {same:.4f}, chi2 within 1.05 {np.mean(ratio <= 1.05):.4f}, "
          f"median ratio {np.median(ratio):.6f}, ended after the learned run "
          f"{st_a['learned_done']} / {st_b['learned_done']}")
    assert np.array_equal(a[:, 9] == 0, b[:, 9] == 0)
    # the pixels still in flight when the queue drains, and so the steps that
    # the lane-split rounds take (results agree to rounding), differ between
    # the two copies; with two waves of lanes after the drain 0.79 of the
    # pixels stayed identical on this map
    assert same > 0.7
    assert abs(np.median(ratio) - 1) < 1e-6
    assert np.mean(ratio <= 1.05) > 0.97
