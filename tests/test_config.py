"""Control-file reader: the reference's keyword table and parsing rules
(Src/RINPUT.c:361-563, Get_Keys Src/RINPUT.c:48-357, STR_READ_LINE
Src/STR.c:387-460)."""
import math

import pytest

import me_b200

BASE = "lines = 15648.5, 3.0\ndata_path = ./d.fits\nwavelength_path = ./w.fits\n"


def parse(extra=""):
    return me_b200.parse_config_text(BASE + extra)


def test_defaults_table():
    c = parse()
    assert c.nline == 1 and c.line_lambda0[0] == 15648.5 and c.line_geff[0] == 3.0
    assert (c.verbose, c.num_iter, c.num_run) == (1, 60, 4)
    assert c.convg_criteria == 1e-3 and c.chisq_criteria == 1.0
    assert list(c.weights) == [1.0] * 4
    assert list(c.sol_box) == [-1, -1, -1, -1]
    assert c.output_fit == 0 and c.damp == 1e-3
    assert (c.lambda_accept, c.lambda_reject) == (5.0, 5.0)
    assert list(c.lambda_limits) == [1e-5, 1e3]
    bounds = [[5, 6000], [0, math.pi], [0, math.pi], [-20, 20], [10, 80], [0.4, 0.8],
              [2, 90], [0, 1e6], [0.1, 0.85]]
    for i, (lo, hi) in enumerate(bounds):
        assert c.bounds[i][0] == pytest.approx(lo) and c.bounds[i][1] == pytest.approx(hi)
    assert list(c.fixed) == [0] * 9
    # theta regularisation is on by default, target 0.5 pi, weight 1e-4
    assert list(c.regul) == [0, 1, 0, 0, 0, 0, 0, 0, 0] and c.regul_any == 1
    assert c.regul_value[1] == pytest.approx(0.5 * math.pi) and c.regul_weight[1] == 1e-4
    assert (c.vcoeffi, c.lcoeffi, c.icriteria, c.svd_threshold) == (100.0, 250.0, 100.0, 1e-6)
    assert c.hmi_ref == 0 and c.nfigures == 6 and c.nprofiles == 20
    assert list(c.step) == [1000., 2., 2., 2., 20., 0.3, 30., 1e5, 0.3]
    assert c.precision == me_b200.ME_PREC_FP32 and c.rng_seed == 0


def test_comments_and_inline_bang():
    c = parse("# num_run = 9\n! num_iter = 3\n* damp = 5\n  num_run = 7 ! seven\n"
              "num_iter = 11 # not a comment for atoi\n")
    assert c.num_run == 7 and c.num_iter == 11 and c.damp == 1e-3


def test_case_sensitive_keys_and_unknown_ignored():
    c = parse("NUM_RUN = 9\nfoo = 1\nx= 3\n")
    assert c.num_run == 4


def test_redefinition_overwrites():
    assert parse("num_run = 2\nnum_run = 3\n").num_run == 3


def test_flags_yes_only():
    c = parse("HMI_REF = yes\noutput_fit = Y\nBmod_fixed = YES\n")
    assert c.hmi_ref == 1 and c.output_fit == 0 and c.fixed[0] == 1


def test_cache_prof_disables_fit_output():
    assert parse("output_fit = YES\nCache_prof = YES\n").output_fit == 0


def test_regularisation_triples():
    c = parse("Bphi_Regularization = Yes, 0.25, 2\nEta_Regularization = YES, 10.0, 2e-3\n"
              "Btheta_Regularization = NO\n")
    assert c.regul[2] == 1 and c.regul_value[2] == pytest.approx(0.25 * math.pi)
    assert c.regul[6] == 1 and c.regul_value[6] == 10.0 and c.regul_weight[6] == 2e-3
    assert c.regul[1] == 0


def test_multiple_lines_first_used():
    c = parse("lines = 6302.5, 2.5\n")
    assert c.nline == 2 and c.line_lambda0[1] == 6302.5


@pytest.mark.parametrize("bad", [
    "weights = 1, 2, 3\n", "Bounds_Dopp = 5 6\n", "sol_box = 1, 2\n", "Step = 1, 2\n",
    "lambda_accept = 1.2\n", "lambda_limits = 3\n", "Nfigures = 9\n", "precision = FP16\n",
    "lines = 15648.5\n"])
def test_malformed_values_are_errors(bad):
    with pytest.raises(me_b200.MeError) as e:
        parse(bad)
    assert e.value.status == -2


def test_required_keywords():
    with pytest.raises(me_b200.MeError):
        me_b200.parse_config_text("lines = 15648.5, 3\n")
    with pytest.raises(me_b200.MeError):
        me_b200.parse_config_text("data_path = a\nwavelength_path = b\n")


def test_too_many_lines():
    with pytest.raises(me_b200.MeError):
        parse("lines = 6302.5, 2.5\n" * 20)


def test_parse_file(tmp_path):
    p = tmp_path / "input"
    p.write_text(BASE + "num_run = 6\n")
    assert me_b200.parse_config(str(p)).num_run == 6
    with pytest.raises(me_b200.MeError) as e:
        me_b200.parse_config(str(tmp_path / "missing"))
    assert e.value.status == -3


def test_config_init_defaults():
    c = me_b200.default_config()
    assert c.num_iter == 60 and c.nfigures == 6 and c.lines_seen == 0


def test_reference_examples_parse():
    """The reference's example control files (keyword syntax only)."""
    text = ("verbose = 0\nnum_run = 6\nlines =  15648.5,  3.0\n"
            "data_path = ./data/niris_example.fits\nwavelength_path = ./niriswavelength.fits\n"
            "weights = 1, 8, 8, 12\n#weights = 1, 1.5, 1.5, 2\nBounds_Bmod = 5, 5000\n"
            "Bounds_Dopp = 50, 140\n#Btheta_Regularization = Yes, 0.5, 1\n"
            "sol_box = -1, -1, -1, -1\n!sol_box = 0, 100, 0, 5\nLCoeffi = 300\n")
    c = me_b200.parse_config_text(text)
    assert c.num_run == 6 and list(c.weights) == [1, 8, 8, 12] and c.bounds[4][1] == 140
    assert c.lcoeffi == 300 and list(c.sol_box) == [-1] * 4
