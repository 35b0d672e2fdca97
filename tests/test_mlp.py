"""The learned initialiser: its arithmetic against the numpy oracle
(oracle/mlp_oracle.py), its training, and its gain on the inversion.

CPU tests pin the oracle (finite differences, torch's bfloat16 rounding and
Adam) and the C ABI's argument checks; GPU tests compare the CUDA loss and
gradients with the oracle, check that training learns, and measure what the
learned start buys the inversion against the plain LM with restarts.
"""
import ctypes
import os

import numpy as np
import pytest

import me_b200
import me_maps
from oracle import mlp_oracle as mo

NIN_PAD = 256  # the Fe I 15648.5 A grid: 4 x 60 = 240 features, padded to 256


def random_params(nin_pad, nin_used, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    layers = []
    for l, (dout, din) in enumerate(mo.shapes(nin_pad)):
        W = rng.normal(0, scale * np.sqrt(2.0 / din), (dout, din))
        if l == 0:
            W[:, nin_used:] = 0
        if l == 3:
            W[mo.NOUT:, :] = 0
        b = rng.normal(0, 0.1, dout)
        if l == 3:
            b[mo.NOUT:] = 0
        layers.append((W, b))
    return mo.flatten(layers).astype(np.float32)


def random_batch(rows, nin_pad, nin_used, seed):
    rng = np.random.default_rng(seed + 1)
    x = rng.normal(0, 1, (rows, nin_pad)).astype(np.float32)
    x[:, nin_used:] = 0
    t = rng.normal(0, 1, (rows, mo.NOUT)).astype(np.float32)
    return x, t


# ---------------------------------------------------------------- CPU ------

def test_oracle_gradient_matches_finite_differences():
    nin_pad, nin = 64, 60
    p = random_params(nin_pad, nin, 1).astype(np.float64)
    x, t = random_batch(8, nin_pad, nin, 1)
    _, g = mo.loss_grad(p, x, t, nin_pad)
    rng = np.random.default_rng(3)
    sizes = [dout * din + dout for dout, din in mo.shapes(nin_pad)]
    starts = np.cumsum([0] + sizes[:-1])
    idx = []
    for l, (dout, din) in enumerate(mo.shapes(nin_pad)):
        used_rows = mo.NOUT if l == 3 else dout
        used_cols = nin if l == 0 else din
        for _ in range(6):
            r, c = rng.integers(used_rows), rng.integers(used_cols)
            idx.append(starts[l] + r * din + c)
        idx.append(starts[l] + dout * din + rng.integers(used_rows))
    for i in idx:
        h = 1e-6 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mo.loss_grad(pp, x, t, nin_pad)[0] - mo.loss_grad(pm, x, t, nin_pad)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1e-3, abs(g[i])) + 1e-9, (i, fd, g[i])


def test_oracle_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(7)
    v = np.concatenate([rng.normal(0, 1, 10000), rng.normal(0, 1e-30, 100),
                        [0.0, -0.0, 1.0, 65504.0, 1 + 2 ** -8, 1 + 3 * 2 ** -9]]).astype(np.float32)
    want = torch.from_numpy(v).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(mo.bf16_round(v), want)


def test_oracle_adam_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(9)
    p0 = rng.normal(0, 1, 50)
    w = torch.tensor(p0.copy(), requires_grad=True)
    opt = torch.optim.Adam([w], lr=1e-3, betas=(0.9, 0.999), eps=1e-8)
    p, m, v = p0.copy(), np.zeros(50), np.zeros(50)
    for step in range(1, 4):
        g = rng.normal(0, 1, 50)
        w.grad = torch.tensor(g)
        opt.step()
        p, m, v = mo.adam(p, m, v, g, step)
    np.testing.assert_allclose(p, w.detach().numpy(), rtol=1e-12, atol=1e-14)


def test_abi_argument_checks(tmp_path):
    L = me_b200.lib()
    tp = me_b200.mlp_train_params()
    assert tp.samples == 1 << 22 and tp.batch == 4096 and tp.epochs == 16
    assert tuple(tp.doppler_range) == (150.0, 350.0)
    h = ctypes.c_void_p()
    assert L.me_mlp_train(None, ctypes.byref(tp), ctypes.byref(h), None) == me_b200.ME_ERR_ARG
    assert L.me_mlp_load(str(tmp_path / "missing.bin").encode(), 0,
                         ctypes.byref(h)) == me_b200.ME_ERR_IO
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"NOTANMLP" + bytes(64))
    assert L.me_mlp_load(str(bad).encode(), 0, ctypes.byref(h)) == me_b200.ME_ERR_FORMAT
    assert L.me_plan_set_initializer(None, None) == me_b200.ME_ERR_ARG
    with pytest.raises(KeyError):
        me_b200.mlp_train_params(no_such_field=1)


# ---------------------------------------------------------------- GPU ------

def fe15648_plan(precision="FP32", widen=False, seed=0):
    name = "fe15648_1024x1024"
    cfg = me_b200.parse_config_text(me_maps.control_text(name, precision=precision, seed=seed,
                                                         widen_bounds=widen))
    return me_b200.Plan(cfg, me_maps.wavelengths(name))


@pytest.fixture(scope="module")
def trained():
    plan = fe15648_plan()
    init = me_b200.Initializer.train(plan, samples=1 << 20, epochs=8)
    yield plan, init
    init.close()
    plan.close()


@pytest.mark.gpu
@pytest.mark.parametrize("gemm", ["tcgen05", "mma_sync"])
def test_loss_and_gradient_match_oracle(gemm):
    plan = fe15648_plan()
    init = me_b200.Initializer.train(plan, samples=256, batch=256, epochs=0)
    init.set_gemm(gemm)
    before = init.gemm_launches()
    nl, nip, npar = init.shape()
    assert (nl, nip) == (60, NIN_PAD)
    assert npar == sum(o * i + o for o, i in mo.shapes(nip))
    p = random_params(nip, 4 * nl, 11)
    init.set_params(p)
    np.testing.assert_array_equal(init.get_params(), p)
    x, t = random_batch(512, nip, 4 * nl, 11)
    loss, g = init.loss_grad(x, t)
    # same bfloat16 roundings as the device: FP32 versus FP64 summation only
    l_b, g_b = mo.loss_grad(p.astype(np.float64), x, t, nip, bf16=True)
    assert abs(loss - l_b) <= 1e-5 * l_b
    rel = np.linalg.norm(g - g_b) / np.linalg.norm(g_b)
    assert rel < 2e-3, rel
    for l0, l1 in zip(np.cumsum([0] + [o * i + o for o, i in mo.shapes(nip)])[:-1],
                      np.cumsum([o * i + o for o, i in mo.shapes(nip)])):
        gl, bl = g[l0:l1], g_b[l0:l1]
        assert np.linalg.norm(gl - bl) <= 5e-3 * np.linalg.norm(bl) + 1e-12
    # against exact FP64 arithmetic: the bfloat16 operands cost ~1 % at most
    l_x, g_x = mo.loss_grad(p.astype(np.float64), x, t, nip)
    assert abs(loss - l_x) <= 2e-2 * l_x
    assert np.linalg.norm(g - g_x) / np.linalg.norm(g_x) < 5e-2
    # every GEMM of the forward and backward pass ran on the chosen kernel
    after = init.gemm_launches()
    other = "mma_sync" if gemm == "tcgen05" else "tcgen05"
    assert after[gemm] - before[gemm] == 4 + 4 + 3 and after[other] == before[other]
    init.close()
    plan.close()


@pytest.mark.gpu
def test_training_learns_and_beats_init_guess(trained):
    plan, init = trained
    assert init.final_loss < 0.25, init.final_loss  # standardised MSE (1.0 = predicting the mean)
    name = "fe15648_1024x1024"
    par = me_maps.draw_parameters(name, 4096, 123)
    prof = me_maps.add_noise(plan.synthesize(par), 1e-3, 123)
    pred = init.predict(prof)
    guess, _, status = plan.init_guess(prof)
    ok = status == 0
    err_mlp = np.abs(pred[ok] - par[ok])
    err_ig = np.abs(guess[ok] - par[ok])
    # field strength, inclination, velocity, eta0: the network is closer to the truth
    for k in (0, 1, 3, 6):
        assert np.median(err_mlp[:, k]) < np.median(err_ig[:, k]), k
    assert np.median(err_mlp[:, 0]) < 150.0
    assert np.median(err_mlp[:, 3]) < 0.2


@pytest.mark.gpu
def test_save_load_roundtrip(trained, tmp_path):
    plan, init = trained
    path = tmp_path / "init.bin"
    init.save(path)
    again = me_b200.Initializer.load(path)
    np.testing.assert_array_equal(again.get_params(), init.get_params())
    par = me_maps.draw_parameters("fe15648_1024x1024", 300, 5)
    prof = plan.synthesize(par)
    np.testing.assert_array_equal(again.predict(prof), init.predict(prof))
    again.close()


def read_initializer(path):
    """The initialiser file as numpy arrays: nl, nin_pad, feature and target
    standardisation, flat parameters (the documented layout)."""
    raw = open(path, "rb").read()
    assert raw[:8] == b"MEMLP001"
    nl, nip = np.frombuffer(raw, np.int32, 2, 8)
    f = np.frombuffer(raw, np.float32, offset=16)
    fmean, fistd = f[:nip], f[nip:2 * nip]
    tmean, tstd = f[2 * nip:2 * nip + 10], f[2 * nip + 10:2 * nip + 20]
    return int(nl), int(nip), fmean, fistd, tmean, tstd, f[2 * nip + 20:]


def oracle_predict(path, prof):
    """The inference restated in numpy: features (I / I_max - 1, 10 Q / I_max,
    10 U / I_max, 10 V / I_max), standardisation, the network with BF16
    operands (FP64 sums), de-standardisation and the parameter decode."""
    nl, nip, fmean, fistd, tmean, tstd, params = read_initializer(path)
    imax = np.maximum(prof[:, 0, :].max(1), 0.0)
    inv = np.where(imax > 0, 1.0 / np.where(imax > 0, imax, 1), 0.0)
    x = np.zeros((prof.shape[0], nip))
    feat = prof.reshape(prof.shape[0], 4 * nl) * inv[:, None]
    feat[:, :nl] -= 1.0
    feat[:, nl:] *= 10.0
    x[:, :4 * nl] = (feat - fmean[:4 * nl]) * fistd[:4 * nl]
    y, _ = mo.forward(params.astype(np.float64), x, nip, bf16=True)
    t = y[:, :10] * tstd + tmean
    par = np.zeros((prof.shape[0], 9))
    par[:, 0] = np.maximum(t[:, 0], 0)
    par[:, 1] = np.arccos(np.clip(t[:, 1], -1, 1))
    phi = 0.5 * np.arctan2(t[:, 2], t[:, 3])
    par[:, 2] = np.where(phi < 0, phi + np.pi, phi)
    par[:, 3:7] = t[:, 4:8]
    par[:, 7] = t[:, 9] * imax
    par[:, 8] = t[:, 8]
    return par


@pytest.mark.gpu
@pytest.mark.parametrize("aligned", [True, False])
def test_predict_matches_oracle_inference(trained, tmp_path, aligned):
    """Map inference (the warp-per-profile feature kernel, the four GEMMs and
    the decode) against the numpy restatement.  BF16 rounding of activations
    computed in FP32 on the device and FP64 in the oracle can fall on
    opposite sides of a rounding boundary, so the bound is statistical."""
    torch = pytest.importorskip("torch")
    plan, init = trained
    path = tmp_path / "init.bin"
    init.save(path)
    par = me_maps.draw_parameters("fe15648_1024x1024", 3000, 31)
    prof = me_maps.add_noise(plan.synthesize(par), 1e-3, 31)
    want = oracle_predict(path, prof)
    flat = torch.from_numpy(np.ascontiguousarray(prof).ravel()).cuda()
    if not aligned:  # profiles starting 8 bytes past a 16-byte boundary
        buf = torch.zeros(flat.numel() + 1, dtype=torch.float64, device="cuda")
        buf[1:] = flat
        flat = buf[1:]
    assert (flat.data_ptr() % 16 == 0) == aligned
    out = torch.zeros((prof.shape[0], 9), dtype=torch.float64, device="cuda")
    init.predict_device(flat.data_ptr(), prof.shape[0], out.data_ptr(), 0)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    np.testing.assert_array_equal(got, init.predict(prof))
    err = np.abs(got - want)
    err[:, 2] = np.minimum(err[:, 2], np.pi - err[:, 2])  # azimuth modulo pi
    spread = np.quantile(want, 0.95, axis=0) - np.quantile(want, 0.05, axis=0)
    assert np.all(np.median(err, 0) <= 2e-3 * spread), np.median(err, 0) / spread
    assert np.all(np.quantile(err, 0.99, axis=0) <= 2e-2 * spread)


@pytest.mark.gpu
def test_attach_detach_leaves_plain_path_unchanged(trained):
    _, init = trained
    name = "fe15648_1024x1024"
    par = me_maps.draw_parameters(name, 1024, 77)
    with fe15648_plan() as p1, fe15648_plan() as p2:
        prof = me_maps.add_noise(p1.synthesize(par), 1e-3, 77)
        r1, _ = p1.invert(prof)
        p2.set_initializer(init)
        r_learned, st = p2.invert(prof)
        assert st["learned_done"] > 0 and st["init_ms"] > 0
        p2.set_initializer(None)
        p2.carry_chisq = 0.0
        r2, _ = p2.invert(prof)
        np.testing.assert_array_equal(r1, r2)
        assert not np.array_equal(r1, r_learned)


@pytest.mark.gpu
def test_learned_start_gain(trained):
    """Learned start versus the plain LM with restarts on the benchmark's
    workload (num_run = 5, chisq_criteria = 1.5, Doppler and damping bounds
    widened to cover the drawn values): at least as good a fit for nearly every
    pixel, in far fewer LM runs and less device time.  (With the default
    Bounds_Dopp of 10-80 mA no start can fit the drawn 150-350 mA widths, the
    criterion is rarely met and every pixel falls back to the full schedule.)"""
    _, init = trained
    name = "fe15648_1024x1024"
    npix = 16384
    par = me_maps.draw_parameters(name, npix, 99)
    with fe15648_plan("FP64", True) as ref, fe15648_plan("FP32", True) as plain, \
            fe15648_plan("FP32", True) as learned:
        prof = me_maps.add_noise(ref.synthesize(par), 1e-3, 99)
        r_ref, _ = ref.invert(prof)
        plain.invert(prof[:2048])  # warm-up
        plain.carry_chisq = 0.0
        r_plain, s_plain = plain.invert(prof)
        learned.set_initializer(init)
        learned.invert(prof[:2048])
        learned.carry_chisq = 0.0
        r_learn, s_learn = learned.invert(prof)
    valid = r_ref[:, 9] > 0
    conv_plain = np.mean(r_plain[valid, 9] <= 1.05 * r_ref[valid, 9])
    conv_learn = np.mean(r_learn[valid, 9] <= 1.05 * r_ref[valid, 9])
    assert conv_learn >= max(conv_plain, 0.98), (conv_learn, conv_plain)
    assert s_learn["runs"] * 4 < s_plain["runs"], (s_learn["runs"], s_plain["runs"])
    # LM work (trial syntheses + syntheses with Jacobian) at least 4x smaller;
    # device time is reported (at this size it is bound by the latency of the
    # slowest pixels' run chains, not by throughput)
    work_plain = s_plain["trials"] + s_plain["jacobians"]
    work_learn = s_learn["trials"] + s_learn["jacobians"]
    print("plain", s_plain, "learned", s_learn)
    assert work_learn * 4 < work_plain, (work_learn, work_plain)
    assert s_learn["learned_done"] > 0.5 * valid.sum()
