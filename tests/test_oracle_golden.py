"""The CPU oracle against the golden fixtures made by the reference itself.

The fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py) are the
outputs of the reference's own C core on seeded synthetic profiles.  The oracle
keeps the reference's floating-point evaluation order, so on an x86-64 CPU with
glibc it reproduces them bit for bit; the comparisons here are exact.
"""
import glob
import json
import os

import numpy as np
import pytest

import me_b200
import oracle_bind as ob

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLD, "fe*.npz")))


def load(name):
    return np.load(os.path.join(GOLD, name + ".npz"))


def test_fixture_set_present():
    assert len(CASES) >= 6


def test_faddeeva_bit_exact():
    f = load("faddeeva")
    for nf in (4, 5, 6, 7, 8):
        H, L = ob.oracle_faddeeva(nf, f["nu"], f["a"])
        np.testing.assert_array_equal(H, f[f"H{nf}"])
        np.testing.assert_array_equal(L, f[f"L{nf}"])


def test_svd_bit_exact():
    f = load("svd")
    for a, u, w, v in zip(f["a"], f["u"], f["w"], f["v"]):
        uo, wo, vo, hit = ob.oracle_svd(a)
        assert hit == 0
        np.testing.assert_array_equal(uo, u)
        np.testing.assert_array_equal(wo, w)
        np.testing.assert_array_equal(vo, v)


@pytest.mark.parametrize("case", CASES)
def test_plan_facts(case):
    f = load(case)
    cfg = me_b200.parse_config_text(str(f["ctl"]))
    o = ob.Oracle(cfg, f["lam"])
    facts = json.loads(str(f["facts"]))
    got = o.facts()
    for k in ("ncut", "ic", "i0", "i1", "npar"):
        assert got[k] == facts[k], k
    # row 7 (S) is per-pixel state in the reference: Init_Guess rewrites
    # Para->Limits[7] for every pixel (Src/ME_SOLVER.c:664-665)
    keep = [i for i in range(9) if i != 7]
    np.testing.assert_array_equal(got["limits"][keep], np.array(facts["limits"])[keep])


@pytest.mark.parametrize("case", CASES)
def test_synthesis_and_jacobian_bit_exact(case):
    f = load(case)
    cfg = me_b200.parse_config_text(str(f["ctl"]))
    o = ob.Oracle(cfg, f["lam"])
    syn, jac = o.synth(f["par_true"][0], deriv=True, step7=0.1)
    np.testing.assert_array_equal(syn, f["syn0"])
    np.testing.assert_array_equal(jac, f["jac0"])


@pytest.mark.parametrize("case", CASES)
def test_init_guess_bit_exact(case):
    f = load(case)
    cfg = me_b200.parse_config_text(str(f["ctl"]))
    o = ob.Oracle(cfg, f["lam"])
    for i, p in enumerate(f["prof"]):
        st, g, e = o.init_guess(p)
        assert st == f["guess_status"][i]
        if st == 0:
            np.testing.assert_array_equal(g, f["guess"][i])
            np.testing.assert_array_equal(e, f["guess_extra"][i])


@pytest.mark.parametrize("case", CASES)
def test_inversion_bit_exact(case):
    """INVERSION_MULTI over the fixture pixels, including the pixel under
    Icriteria and the NaN pixel (zeros), and the LM chi^2 carried between
    pixels."""
    f = load(case)
    cfg = me_b200.parse_config_text(str(f["ctl"]))
    o = ob.Oracle(cfg, f["lam"])
    res = o.invert(f["prof"], rng_mode=ob.MEO_RNG_NR, nr_seed=int(f["nr_seed"]))
    np.testing.assert_array_equal(res, f["res"])
    assert o.carry[0] == float(f["carry_out"])
    assert np.all(res[5] == 0) and np.all(res[9] == 0)


def test_restart_draws_are_standard_normal():
    z = np.concatenate([ob.restart_draws(7, p, r) for p in range(300) for r in range(4, 12)])
    assert abs(z.mean()) < 0.05 and abs(z.std() - 1) < 0.05
    np.testing.assert_array_equal(ob.restart_draws(7, 12, 5), ob.restart_draws(7, 12, 5))
    assert not np.array_equal(ob.restart_draws(7, 12, 5), ob.restart_draws(7, 12, 6))
