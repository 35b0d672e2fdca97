"""The instrument filter (an extension of the synthesis; the reference has
none), on the configs' filtergram workload: Fe I 6173.3 A, 6 wavelengths at
+-34, +-103, +-172 mA, each seen through a Gaussian filter of 76 mA FWHM.

The oracle's filter is a weighted sum of its Milne-Eddington synthesis (the
restatement pinned to the reference) over the filter's sub-wavelengths; the
CPU tests pin that sum and the `filter` keyword's Gaussian table.  The GPU
tests compare the CUDA synthesis and Jacobian with the oracle, and the
inversion with the oracle under the same ulp-chaos bar as the unfiltered
path.
"""
import numpy as np
import pytest

import me_b200
import me_maps
import oracle_bind as ob

NAME = "fe6173_4096x4096"


def gaussian_table(fwhm, points):
    """The `filter = FWHM, points` table as documented: offsets uniform over
    +-1.5 FWHM, weights exp(-d^2 / 2 sigma^2) normalised to sum 1."""
    off = np.linspace(-1.5 * fwhm, 1.5 * fwhm, points)
    sigma = fwhm / (2 * np.sqrt(2 * np.log(2)))
    w = np.exp(-off ** 2 / (2 * sigma ** 2))
    return off, w / w.sum()


def cfg_of(precision="FP64", extra=None):
    return me_b200.parse_config_text(me_maps.control_text(NAME, precision=precision, extra=extra))


# ---------------------------------------------------------------- CPU ------

def test_oracle_filter_is_weighted_sum_of_subgrid_synthesis():
    lam = me_maps.wavelengths(NAME)
    off, w = gaussian_table(76.0, 21)
    filt = ob.Oracle(cfg_of(), lam)
    fine_lam = (lam[:, None] + off[None, :] * 1e-3).ravel()
    plain = ob.Oracle(cfg_of(extra={"filter": "0"}), fine_lam)
    par = me_maps.draw_parameters(NAME, 6, 3)
    for p in par:
        syn, jac = filt.synth(p, deriv=True, step7=0.1)
        fs, fj = plain.synth(p, deriv=True, step7=0.1)
        want = (fs.reshape(4, lam.size, 21) * w).sum(-1)
        wantj = (fj.reshape(4, 9, lam.size, 21) * w).sum(-1)
        np.testing.assert_allclose(syn, want, rtol=1e-13, atol=1e-15)
        np.testing.assert_allclose(jac, wantj, rtol=1e-12, atol=1e-13 * np.abs(wantj).max())


def test_filter_keyword_is_the_documented_gaussian():
    lam = me_maps.wavelengths(NAME)
    a = ob.Oracle(cfg_of(), lam)
    b = ob.Oracle(cfg_of(extra={"filter": "0"}), lam)
    b.set_filter(*gaussian_table(76.0, 21))
    par = me_maps.draw_parameters(NAME, 4, 8)
    for p in par:  # numpy's linspace rounds the offsets differently from the C formula
        np.testing.assert_allclose(a.synth(p), b.synth(p), rtol=1e-13, atol=1e-15)
    off, w = gaussian_table(76.0, 21)
    assert abs(w.sum() - 1) < 1e-15 and np.allclose(w, w[::-1])


def test_filter_keyword_errors():
    for bad in ("76", "76, 20", "76, 65", "-3, 21", "x"):
        with pytest.raises(me_b200.MeError):
            cfg_of(extra={"filter": bad})


# ---------------------------------------------------------------- GPU ------

@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol_syn,tol_jac", [("FP64", 1e-12, 1e-9), ("FP32", 2e-6, 2e-3)])
def test_filtered_synthesis_vs_oracle(prec, tol_syn, tol_jac):
    lam = me_maps.wavelengths(NAME)
    orc = ob.Oracle(cfg_of(), lam)
    par = me_maps.draw_parameters(NAME, 16, 5)
    with me_b200.Plan(cfg_of(prec), lam) as plan:
        syn, jac = plan.synthesize_jacobian(par, 0.1)
        fwd = plan.synthesize(par)
    for i, p in enumerate(par):
        s0, j0 = orc.synth(p, deriv=True, step7=0.1)
        assert np.max(np.abs(syn[i] - s0)) < tol_syn
        assert np.max(np.abs(fwd[i] - s0)) < tol_syn
        scale = np.abs(j0).max(axis=(1, 2), keepdims=True)
        assert np.max(np.abs(jac[i] - j0) / scale) < tol_jac


@pytest.mark.gpu
def test_removing_the_filter_restores_the_plain_path():
    lam = me_maps.wavelengths(NAME)
    par = me_maps.draw_parameters(NAME, 64, 6)
    with me_b200.Plan(cfg_of("FP32"), lam) as a, \
            me_b200.Plan(cfg_of("FP32", extra={"filter": "0"}), lam) as b:
        a.set_filter([0.0], [1.0])
        np.testing.assert_array_equal(a.synthesize(par), b.synthesize(par))
        prof = me_maps.add_noise(b.synthesize(par), 2e-3, 6)
        ra, _ = a.invert(prof)
        rb, _ = b.invert(prof)
        np.testing.assert_array_equal(ra, rb)


def ulp_perturb(prof, seed=5):
    rng = np.random.default_rng(seed)
    return prof * (1 + 2.3e-16 * rng.choice([-1, 1], prof.shape))


def agreement(res, base):
    same = (np.abs(res - base) <= 1e-6 * np.abs(base) + 1e-12).all(1)
    valid = base[:, 9] > 0
    ratio = np.ones(len(base))
    ratio[valid] = res[valid, 9] / base[valid, 9]
    return same.mean(), np.mean(ratio[valid] <= 1.05), np.median(ratio[valid])


@pytest.fixture(scope="module")
def filt_map():
    lam = me_maps.wavelengths(NAME)
    extra = {"num_run": "1"}
    orc = ob.Oracle(cfg_of(extra=extra), lam)
    par = me_maps.draw_parameters(NAME, 1024, 17)
    prof = me_maps.add_noise(orc.synth_many(par), 2e-3, 17)
    base = orc.invert(prof)
    pert = ob.Oracle(cfg_of(extra=extra), lam).invert(ulp_perturb(prof))
    return dict(lam=lam, prof=prof, base=base, extra=extra, self=agreement(pert, base))


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["FP64", "FP32"])
def test_filtered_inversion_parity_vs_oracle(filt_map, prec):
    m = filt_map
    with me_b200.Plan(cfg_of(prec, m["extra"]), m["lam"]) as plan:
        res, st = plan.invert(m["prof"])
    same, within, med = agreement(res, m["base"])
    s_same, s_within, _ = m["self"]
    print(f"filter {prec}: identical {same:.3f} (self {s_same:.3f}), chi2<=1.05x {within:.3f} "
          f"(self {s_within:.3f}), median ratio {med:.6f}")
    assert st["valid"] == np.sum(m["base"][:, 9] > 0)
    assert abs(med - 1) < 1e-3
    assert within >= s_within - 0.05
    if prec == "FP64":
        assert same >= s_same - 0.10


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["FP64", "FP32"])
def test_filtered_kernel_variants_agree(filt_map, prec):
    """The sub-wavelength grid (6 x 21 points) staged in shared memory, and
    the other kernel variants: each meets the oracle bar on the filtergram
    (they agree with the default variant to rounding)."""
    m = filt_map
    s_same, s_within, _ = m["self"]
    with me_b200.Plan(cfg_of(prec, m["extra"]), m["lam"]) as plan:
        plan.max_group, plan.tail_slots = 1, 0
        for v in (3, 4, 1, 5):
            plan.kernel_variant = v
            plan.carry_chisq = 0.0
            res, _ = plan.invert(m["prof"])
            same, within, med = agreement(res, m["base"])
            print(f"filter {prec} variant {v}: identical {same:.3f} (self {s_same:.3f}), "
                  f"chi2<=1.05x {within:.3f} (self {s_within:.3f})")
            assert abs(med - 1) < 1e-3 and within >= s_within - 0.05, v
            if prec == "FP64":
                assert same >= s_same - 0.10, v


@pytest.mark.gpu
def test_learned_start_with_queue_order_on_the_filtered_grid():
    """The learned start on the filtered grid, queue order on and off (the
    start-misfit kernel's filtered variant): the same pixels inverted, chi^2
    that agree under the ulp-chaos bar, and a reproducible order."""
    lam = me_maps.wavelengths(NAME)
    par = me_maps.draw_parameters(NAME, 8192, 29)
    with me_b200.Plan(cfg_of("FP32"), lam) as plan:
        prof = me_maps.add_noise(plan.synthesize(par), 2e-3, 29)
        init = me_b200.Initializer.train(plan, samples=1 << 18, epochs=4,
                                         doppler_range=(20.0, 50.0), noise=2e-3)
        plan.set_initializer(init)
        plan.window = 2048
        plan.set_queue_order(False)
        plan.carry_chisq = 0.0
        r0, s0 = plan.invert(prof)
        plan.set_queue_order(True)
        plan.carry_chisq = 0.0
        r1, s1 = plan.invert(prof)
        plan.carry_chisq = 0.0
        r2, _ = plan.invert(prof)
        plan.set_initializer(None)
        init.close()
    np.testing.assert_array_equal(r1, r2)
    assert s1["valid"] == s0["valid"] and s1["init_ms"] > 0
    valid = r0[:, 9] > 0
    ratio = r1[valid, 9] / r0[valid, 9]
    print(f"filtered learned start, queue order: chi2 within 1.05x {np.mean(ratio <= 1.05):.4f}")
    assert np.mean(ratio <= 1.05) > 0.97 and abs(np.median(ratio) - 1) < 1e-6


@pytest.mark.gpu
def test_initialiser_trained_on_the_filtered_grid():
    """The configs' filtergram run retrains the learned initialiser for its
    grid: training profiles go through the same filter."""
    lam = me_maps.wavelengths(NAME)
    with me_b200.Plan(cfg_of("FP32"), lam) as plan:
        init = me_b200.Initializer.train(plan, samples=1 << 20, epochs=8,
                                         doppler_range=(20.0, 50.0), noise=2e-3)
        assert init.shape()[:2] == (6, 32)
        par = me_maps.draw_parameters(NAME, 4096, 23)
        prof = me_maps.add_noise(plan.synthesize(par), 2e-3, 23)
        pred = init.predict(prof)
        guess, _, status = plan.init_guess(prof)
        ok = status == 0
        for k in (0, 3):  # field strength and velocity
            assert np.median(np.abs(pred[ok, k] - par[ok, k])) < \
                np.median(np.abs(guess[ok, k] - par[ok, k])), k
        init.close()
