"""CUDA building blocks against the reference's golden vectors and the oracle:
Voigt/Faraday (Faddeeva), Milne-Eddington synthesis + analytic Jacobian,
Golub-Reinsch SVD, initial guess.  Tolerances: FP64 paths agree to rounding
(libm and fused multiply-add differ from the reference's x86 build); FP32
paths within the FP32 error of the same formulas."""
import json
import os

import numpy as np
import pytest

import me_b200
import oracle_bind as ob

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["fe15648_run1", "fe6302_run1", "fe15648_fixed_hmi", "fe15648_regul_eta"]


def load(name):
    return np.load(os.path.join(GOLD, name + ".npz"))


@pytest.mark.parametrize("nf", [4, 5, 6, 7, 8])
@pytest.mark.parametrize("prec,tol", [(me_b200.ME_PREC_FP64, 1e-13), (me_b200.ME_PREC_FP32, 2e-6)])
def test_voigt_vs_reference(nf, prec, tol):
    f = load("faddeeva")
    H, L = me_b200.faddeeva(nf, f["nu"], f["a"], precision=prec)
    Hr, Lr = f[f"H{nf}"], f[f"L{nf}"]
    scale = np.abs(Hr) + np.abs(Lr)
    assert np.max(np.abs(H - Hr) / scale) < tol
    assert np.max(np.abs(L - Lr) / scale) < tol


def test_weideman_on_device_vs_scipy():
    """The FP32 Weideman series on the device (me_faddeeva_weideman) on the
    reference's golden (nu, a) points and a dense grid, against scipy's
    Faddeeva function: within 1.5e-6 of |H| + |L|."""
    from scipy.special import wofz
    f = load("faddeeva")
    rng = np.random.default_rng(5)
    nu = np.concatenate([f["nu"], rng.uniform(-40, 40, 100000)])
    a = np.concatenate([f["a"], rng.uniform(0, 1.6, 100000)])
    H, L = me_b200.faddeeva_weideman(nu, a)
    w = wofz(nu + 1j * a)
    scale = np.abs(w.real) + np.abs(w.imag)
    eh, el = np.max(np.abs(H - w.real) / scale), np.max(np.abs(L - w.imag) / scale)
    print(f"Weideman FP32 on the device: H {eh:.2e} L {el:.2e}")
    assert eh < 1.5e-6 and el < 1.5e-6


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("prec,tol_syn,tol_jac,fad", [("FP64", 1e-12, 1e-9, 0), ("FP32", 2e-6, 2e-3, 0),
                                                      ("FP32", 5e-6, 2e-3, 1)])
def test_synthesis_jacobian_vs_reference(case, prec, tol_syn, tol_jac, fad):
    """fad 1: Weideman's series in place of the reference's Faddeeva regions;
    the reference's own FP64 values carry up to 2.4e-6 (of |H| + |L|) of
    Faddeeva error at Nfigures = 6, hence the wider synthesis bound."""
    f = load(case)
    cfg = me_b200.parse_config_text(str(f["ctl"]) + f"precision = {prec}\n")
    with me_b200.Plan(cfg, f["lam"]) as plan:
        plan.faddeeva = fad
        assert plan.faddeeva == fad
        syn, jac = plan.synthesize_jacobian(f["par_true"][:1], 0.1)
        e_syn = np.max(np.abs(syn[0] - f["syn0"]))
        # derivatives normalised by the largest entry of their Stokes parameter
        # (some rows are analytically zero and only carry rounding)
        scale = np.abs(f["jac0"]).max(axis=(1, 2), keepdims=True)
        e_jac = np.max(np.abs(jac[0] - f["jac0"]) / scale)
        # forward-only entry point agrees with the Jacobian one
        e_fwd = np.max(np.abs(plan.synthesize(f["par_true"][:4])[0] - syn[0]))
        print(f"{case} {prec} faddeeva {fad}: syn {e_syn:.3e} jac {e_jac:.3e} fwd-vs-jac {e_fwd:.3e}")
        assert e_syn < tol_syn and e_jac < tol_jac and e_fwd < tol_syn


@pytest.mark.parametrize("case", CASES)
def test_plan_facts_vs_reference(case):
    f = load(case)
    cfg = me_b200.parse_config_text(str(f["ctl"]))
    facts = json.loads(str(f["facts"]))
    with me_b200.Plan(cfg, f["lam"]) as plan:
        got = plan.facts()
    for k in ("ncut", "ic", "i0", "i1", "npar"):
        assert got[k] == facts[k]
    keep = [i for i in range(9) if i != 7]
    np.testing.assert_array_equal(got["limits"][keep], np.array(facts["limits"])[keep])


def test_svd_vs_reference():
    """Golub-Reinsch output equals the reference's up to a common sign flip of
    a (u_j, v_j) column pair, the freedom rounding decides between."""
    f = load("svd")
    u, w, v = me_b200.svd(f["a"])
    for i in range(len(f["a"])):
        np.testing.assert_allclose(w[i], f["w"][i], rtol=1e-12, atol=1e-13 * f["w"][i].max())
        if np.ptp(f["w"][i]) < 1e-8:
            # an orthogonal input (the LM's later trials): all singular values
            # are 1 and the factors are not unique -- only the product is
            np.testing.assert_allclose((u[i] * w[i]) @ v[i].T, f["a"][i], atol=1e-13)
            continue
        s = np.sign(np.sum(u[i] * f["u"][i], axis=0))
        sv = np.sign(np.sum(v[i] * f["v"][i], axis=0))
        assert np.array_equal(s, sv), "unpaired column sign flip"
        assert np.max(np.abs(u[i] * s - f["u"][i])) < 1e-10
        assert np.max(np.abs(v[i] * s - f["v"][i])) < 1e-10
        rec = (u[i] * w[i]) @ v[i].T
        assert np.max(np.abs(rec - f["a"][i])) < 1e-12 * np.abs(f["a"][i]).max()


def test_svd_smaller_orders():
    rng = np.random.default_rng(1)
    for n in (1, 2, 5, 8):
        a = rng.normal(size=(6, n, n))
        u, w, v = me_b200.svd(a)
        for i in range(6):
            uo, wo, vo, _ = ob.oracle_svd(a[i])
            np.testing.assert_allclose(np.sort(w[i]), np.sort(wo), rtol=1e-12, atol=1e-14)
            np.testing.assert_allclose((u[i] * w[i]) @ v[i].T, a[i], atol=1e-12)


def _svd_u_inputs():
    """The reference's golden SVD inputs, plus the matrices the trial steps
    decompose: normal matrices J^T J of random Jacobians (first trials) and
    the orthogonal U factors of earlier decompositions (later trials), at the
    full order 9 and at 5 (four parameters fixed)."""
    rng = np.random.default_rng(11)
    out = [np.asarray(load("svd")["a"], dtype=np.float64)]
    for n in (9, 5):
        j = rng.normal(size=(64, 240, n)) * np.logspace(0, 2, n)
        h = np.einsum("mki,mkj->mij", j, j)
        q, _ = np.linalg.qr(rng.normal(size=(64, n, n)))
        out += [h, q]
    return out


@pytest.mark.parametrize("fast", [False, True])
def test_svd_u_lanes_and_forms(fast):
    """The U-only decomposition of the trial-step solve (one thread, the
    lane-split groups, the tail kernel's warp) against the full decomposition
    me_svd runs.  An orthogonal input (the later trials' U factors) has all
    singular values 1 and no unique U: the last bit of any operation picks
    another one, so there U is checked for orthogonality only.  Elsewhere U
    and w agree with me_svd's to rounding, whatever the lanes, up to the sign
    of a column (a QR sweep more or less, which rounding decides, can turn a
    rotation by pi); fast: the FP32 plans' Givens radius from one reciprocal
    square root (two ulps per rotation)."""
    for a in _svd_u_inputs():
        n = a.shape[1]
        u_ref, w_ref, _ = me_b200.svd(a)
        scale = np.abs(a).max(axis=(1, 2))
        ortho = np.ptp(w_ref, axis=1) < 1e-8
        # rounding moves a column by about eps * |a| / (gap to its neighbours)
        tol_u = 1e-9 if fast else 1e-10
        for lanes in (1, 2, 4, 8, 16, 32):
            u, w, hits = me_b200.svd_u(a, lanes=lanes, fast=fast)
            assert hits == 0
            assert np.max(np.abs(w - w_ref) / scale[:, None]) < 1e-13, lanes
            eye = np.einsum("mki,mkj->mij", u, u)
            assert np.max(np.abs(eye - np.eye(n))) < 1e-13, lanes
            if np.any(~ortho):
                ug, ur = u[~ortho], u_ref[~ortho]
                sign = np.sign(np.sum(ug * ur, axis=1))[:, None, :]
                assert np.max(np.abs(ug * sign - ur)) < tol_u, lanes


@pytest.mark.parametrize("case", CASES + ["fe15648_widened", "fe15648_run2_nr"])
def test_init_guess_vs_reference(case):
    f = load(case)
    cfg = me_b200.parse_config_text(str(f["ctl"]))
    with me_b200.Plan(cfg, f["lam"]) as plan:
        g, e, st = plan.init_guess(f["prof"])
    np.testing.assert_array_equal(st, f["guess_status"])
    ok = st == 0
    # v_los comes from a centroid minus lambda0 (a cancellation that turns
    # ulp-level libm differences into ~1e-10 relative)
    np.testing.assert_allclose(g[ok], f["guess"][ok], rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(e[ok], f["guess_extra"][ok], rtol=1e-12, atol=1e-15)
