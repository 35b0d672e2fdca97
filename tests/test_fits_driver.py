"""FITS I/O and the driver (me_run): the reference's MEINV around
INVERSION_MULTI (Src/ME_INV.c, Src/IO.c).

CPU tests check the FITS reader against files built here independently
(header cards and big-endian data from numpy), the writer's bytes, the
checkpoint file's format and the driver's input checks.  GPU tests run the
driver on small synthetic cubes and compare its result and fit files with
me_invert_batch on the same pixels, bit for bit: plain, chunked and batched
runs, a run interrupted and resumed from its checkpoint, Cache_prof, and two
plans taking batches in turn.
"""
import ctypes
import os

import numpy as np
import pytest

import me_b200
import me_maps


# ------------------------------------------------------------------ helpers --

def card(key, value=None, comment=None):
    if value is None:
        s = f"{key:<8}" + (comment or "")
    else:
        s = f"{key:<8}= {value:>20}" + (f" / {comment}" if comment else "")
    return s[:80].ljust(80)


def write_fits(path, data, bitpix, bscale=None, bzero=None, comments=0):
    """A primary-HDU FITS file built without the library: numpy shape
    (..., NAXIS2, NAXIS1) in C order is the FITS order."""
    data = np.asarray(data, dtype=np.float64)
    cards = [card("SIMPLE", "T"), card("BITPIX", str(bitpix)), card("NAXIS", str(data.ndim))]
    for i, n in enumerate(reversed(data.shape)):
        cards.append(card(f"NAXIS{i + 1}", str(n)))
    if bscale is not None:
        cards.append(card("BSCALE", repr(float(bscale)), "scale"))
    if bzero is not None:
        cards.append(card("BZERO", repr(float(bzero))))
    cards += [card("COMMENT", comment=f" filler card {i}") for i in range(comments)]
    cards.append(card("END"))
    hdr = "".join(cards).encode()
    hdr += b" " * (-len(hdr) % 2880)
    stored = data
    if bitpix > 0:
        stored = np.round((data - (bzero or 0.0)) / (bscale or 1.0))
    dt = {-64: ">f8", -32: ">f4", 16: ">i2", 32: ">i4", 8: "u1"}[bitpix]
    raw = stored.astype(dt).tobytes()
    raw += b"\0" * (-len(raw) % 2880)
    with open(path, "wb") as f:
        f.write(hdr + raw)


def parse_fits(path):
    """(header dict, data in C order) of a BITPIX -64 primary HDU."""
    blob = open(path, "rb").read()
    hdr, pos = {}, 0
    while True:
        c = blob[pos:pos + 80].decode()
        pos += 80
        key = c[:8].strip()
        if key == "END":
            break
        if c[8:10] == "= ":
            hdr[key] = c[10:].split("/")[0].strip()
    start = (pos + 2879) // 2880 * 2880
    n = int(hdr["NAXIS"])
    shape = [int(hdr[f"NAXIS{i}"]) for i in range(n, 0, -1)]
    count = int(np.prod(shape))
    assert hdr["BITPIX"] == "-64"
    data = np.frombuffer(blob, dtype=">f8", count=count, offset=start).reshape(shape)
    assert len(blob) % 2880 == 0
    return hdr, data


# ---------------------------------------------------------------- CPU ------

@pytest.mark.parametrize("bitpix", [-64, -32, 16])
def test_fits_read_matches_independent_file(tmp_path, bitpix):
    rng = np.random.default_rng(bitpix + 100)
    cube = rng.normal(1.0, 0.3, (3, 5, 4, 7))  # [ny][nx][4][nw]
    path = tmp_path / "cube.fits"
    kw = {}
    if bitpix == 16:
        kw = dict(bscale=1e-4, bzero=1.0)
    write_fits(path, cube, bitpix, comments=40, **kw)  # a header of two blocks
    b, shape = me_b200.fits_info(path)
    assert b == bitpix and shape == (7, 4, 5, 3)
    got = me_b200.fits_read(path)
    if bitpix == -64:
        want = cube.ravel()
    elif bitpix == -32:
        want = cube.astype(np.float32).astype(np.float64).ravel()
    else:
        want = 1.0 + 1e-4 * np.round((cube.ravel() - 1.0) / 1e-4)
    np.testing.assert_array_equal(got, want)
    # an element range from the middle
    np.testing.assert_array_equal(me_b200.fits_read(path, 29, 40), want[29:69])


def test_fits_create_and_write_bytes(tmp_path):
    path = tmp_path / "res.fits"
    me_b200.fits_create(path, (10, 6, 4))
    hdr, data = parse_fits(path)
    assert hdr["SIMPLE"] == "T" and hdr["NAXIS1"] == "10" and hdr["NAXIS3"] == "4"
    assert data.shape == (4, 6, 10) and not data.any()
    v = np.arange(35, dtype=np.float64) * 0.5 - 3
    me_b200.fits_write(path, 17, v)
    _, data = parse_fits(path)
    flat = data.ravel()
    np.testing.assert_array_equal(flat[17:52], v)
    assert not flat[:17].any() and not flat[52:].any()
    np.testing.assert_array_equal(me_b200.fits_read(path, 17, 35), v)


def test_fits_errors(tmp_path):
    L = me_b200.lib()
    bad = tmp_path / "bad.fits"
    bad.write_bytes(b"NOT FITS" + b" " * 3000)
    b, n = ctypes.c_int(), ctypes.c_int()
    ax = (ctypes.c_long * 8)()
    assert L.me_fits_image_info(str(bad).encode(), ctypes.byref(b), ctypes.byref(n),
                                ax) == me_b200.ME_ERR_FORMAT
    assert L.me_fits_image_info(str(tmp_path / "none.fits").encode(), ctypes.byref(b),
                                ctypes.byref(n), ax) == me_b200.ME_ERR_IO
    path = tmp_path / "small.fits"
    me_b200.fits_create(path, (4, 4))
    out = np.zeros(20)
    assert L.me_fits_read(str(path).encode(), 0, 20, out.ctypes.data_as(
        ctypes.POINTER(ctypes.c_double))) == me_b200.ME_ERR_ARG
    write_fits(tmp_path / "f32.fits", np.zeros((2, 2)), -32)
    v = np.zeros(2)
    assert L.me_fits_write(str(tmp_path / "f32.fits").encode(), 0, 2, v.ctypes.data_as(
        ctypes.POINTER(ctypes.c_double))) == me_b200.ME_ERR_FORMAT


def control_file(tmp_path, name="fe15648_64x64", extra=None, precision="FP32"):
    keys = {"data_path": str(tmp_path / "data.fits"),
            "wavelength_path": str(tmp_path / "wave.fits"),
            "result_path": str(tmp_path / "res.fits"), "fit_path": str(tmp_path / "fit.fits"),
            "cache_path": str(tmp_path / "cache")}
    keys.update(extra or {})
    text = me_maps.control_text(name, precision=precision, extra=keys)
    path = tmp_path / "input"
    path.write_text(text)
    return path


def test_driver_checks_and_checkpoint_format(tmp_path):
    """Without a GPU the driver still validates its inputs and lays down the
    checkpoint and result files (CACHE_INIT) before it needs the device."""
    lam = me_maps.wavelengths("fe15648_64x64")
    write_fits(tmp_path / "wave.fits", lam, -64)
    write_fits(tmp_path / "data.fits", np.ones((6, 9, 4, lam.size)), -32)
    ctl = control_file(tmp_path, extra={"sol_box": "2, 7, 1, 4", "nprofiles": "7",
                                        "Cache_inv": "YES", "output_fit": "YES"})
    L = me_b200.lib()
    st = L.me_run(str(ctl).encode(), None, None)
    assert st in (me_b200.ME_OK, me_b200.ME_ERR_NODEVICE, me_b200.ME_ERR_CUDA)
    blob = (tmp_path / "cache").read_bytes()
    nxc, nyc, nprof = 6, 4, 7
    ncache = nxc * nyc // nprof + 1
    assert blob[:4] == b"cach"
    assert np.frombuffer(blob[4:16], dtype="<i4").tolist() == [nxc, nyc, ncache]
    assert len(blob) == 16 + 4 * ncache
    hdr, res = parse_fits(tmp_path / "res.fits")
    assert res.shape == (nyc, nxc, 10)
    _, fit = parse_fits(tmp_path / "fit.fits")
    assert fit.shape == (nyc, nxc, 4, lam.size)
    # input checks
    write_fits(tmp_path / "wave.fits", lam[:-1], -64)
    assert L.me_run(str(ctl).encode(), None, None) == me_b200.ME_ERR_FORMAT
    write_fits(tmp_path / "wave.fits", lam, -64)
    write_fits(tmp_path / "data.fits", np.ones((6, 9, 3, lam.size)), -32)
    assert L.me_run(str(ctl).encode(), None, None) == me_b200.ME_ERR_FORMAT
    write_fits(tmp_path / "data.fits", np.ones((6, 9, 4, lam.size)), 32)
    assert L.me_run(str(ctl).encode(), None, None) == me_b200.ME_ERR_FORMAT


# ---------------------------------------------------------------- GPU ------

NX, NY = 24, 20
SOL = (3, 20, 2, 17)  # x0, x1, y0, y1


@pytest.fixture(scope="module")
def cube(tmp_path_factory):
    d = tmp_path_factory.mktemp("cube")
    name = "fe15648_64x64"
    lam = me_maps.wavelengths(name)
    cfg = me_b200.parse_config_text(me_maps.control_text(name, precision="FP64"))
    with me_b200.Plan(cfg, lam) as gen:
        par = me_maps.draw_parameters(name, NX * NY, 41)
        prof = me_maps.add_noise(gen.synthesize(par), 1e-3, 41)
    data = prof.reshape(NY, NX, 4, lam.size)
    return dict(dir=d, lam=lam, data=data)


def sol_pixels(data):
    x0, x1, y0, y1 = SOL
    return np.ascontiguousarray(data[y0:y1 + 1, x0:x1 + 1].reshape(-1, 4, data.shape[-1]))


def reference_run(ctl_text_path, prof, pieces, want_fit=True):
    """me_invert_batch over the pixel ranges `pieces`, one fresh plan per
    list (each carries its own LM chi^2 through its pieces in order), one
    thread per pixel throughout."""
    cfg = me_b200.parse_config(str(ctl_text_path))
    res = np.zeros((prof.shape[0], 10))
    fit = np.zeros_like(prof)
    for plan_pieces in pieces:
        with me_b200.Plan(cfg, me_maps.wavelengths("fe15648_64x64")) as plan:
            plan.max_group, plan.tail_slots = 1, 0
            for a, b in plan_pieces:
                r, f, _ = plan.invert(prof[a:b], want_fit=True)
                res[a:b] = r
                fit[a:b] = f
    return res, fit


def setup_run(tmp, cube, extra):
    write_fits(tmp / "wave.fits", cube["lam"], -64)
    write_fits(tmp / "data.fits", cube["data"], -64)
    return control_file(tmp, extra=dict({"sol_box": ", ".join(map(str, SOL))}, **extra))


@pytest.mark.gpu
def test_driver_matches_invert_batch(tmp_path, cube):
    ctl = setup_run(tmp_path, cube, {"nprofiles": "37", "output_fit": "YES"})
    rep = me_b200.run(ctl, batch_pixels=100, max_group=1, tail_slots=0)
    prof = sol_pixels(cube["data"])
    n = prof.shape[0]
    assert rep["counts"] == n and rep["chunk_pixels"] == 37
    assert rep["nchunks"] == (n + 36) // 37 and rep["pixels_inverted"] == n
    # batches of two chunks (74 pixels) on one plan: one carry chain over all
    res_ref, fit_ref = reference_run(ctl, prof, [[(0, n)]])
    _, res = parse_fits(tmp_path / "res.fits")
    _, fit = parse_fits(tmp_path / "fit.fits")
    np.testing.assert_array_equal(res.reshape(n, 10), res_ref)
    np.testing.assert_array_equal(fit.reshape(n, 4, -1), fit_ref)


@pytest.mark.gpu
def test_driver_checkpoint_resume(tmp_path, cube):
    ctl = setup_run(tmp_path, cube, {"nprofiles": "23", "Cache_inv": "YES"})
    prof = sol_pixels(cube["data"])
    n = prof.shape[0]
    nch = (n + 22) // 23
    r1 = me_b200.run(ctl, batch_pixels=46, max_group=1, tail_slots=0, stop_after_chunks=5)
    assert r1["chunks_done"] == 5 and r1["pixels_inverted"] == 5 * 23
    flags = np.frombuffer((tmp_path / "cache").read_bytes()[16:], dtype="<i4")
    assert flags[:5].tolist() == [1] * 5 and not flags[5:].any()
    r2 = me_b200.run(ctl, batch_pixels=46, max_group=1, tail_slots=0)
    assert r2["chunks_skipped"] == 5 and r2["chunks_done"] == nch - 5
    flags = np.frombuffer((tmp_path / "cache").read_bytes()[16:], dtype="<i4")
    assert flags[:nch].all()
    # the resumed run starts a new carry chain at chunk 5, as a new process does
    res_ref, _ = reference_run(ctl, prof, [[(0, 115)], [(115, n)]])
    _, res = parse_fits(tmp_path / "res.fits")
    np.testing.assert_array_equal(res.reshape(n, 10), res_ref)
    # a third run finds everything done
    r3 = me_b200.run(ctl, max_group=1, tail_slots=0)
    assert r3["chunks_done"] == 0 and r3["chunks_skipped"] == nch


@pytest.mark.gpu
def test_driver_cache_prof_and_two_plans(tmp_path, cube):
    prof = sol_pixels(cube["data"])
    n = prof.shape[0]
    ctl = setup_run(tmp_path, cube, {"Cache_prof": "YES", "output_fit": "YES"})
    rep = me_b200.run(ctl, max_group=1, tail_slots=0)
    assert rep["nchunks"] == 1 and rep["chunk_pixels"] == n
    assert not (tmp_path / "fit.fits").exists()  # Cache_prof turns output_fit off
    res_ref, _ = reference_run(ctl, prof, [[(0, n)]])
    _, res = parse_fits(tmp_path / "res.fits")
    np.testing.assert_array_equal(res.reshape(n, 10), res_ref)
    # two plans on this GPU take batches of 3 chunks in turn: plan 0 gets
    # batches 0, 2, 4, ...; plan 1 gets 1, 3, 5, ... (each its own carry chain)
    sub = tmp_path / "two"
    sub.mkdir()
    ctl2 = setup_run(sub, cube, {"nprofiles": "20"})
    rep = me_b200.run(ctl2, devices=[0, 0], batch_pixels=60, max_group=1, tail_slots=0)
    assert rep["pixels_inverted"] == n
    batches = [(a, min(a + 60, n)) for a in range(0, n, 60)]
    res_ref, _ = reference_run(ctl2, prof, [batches[0::2], batches[1::2]])
    _, res = parse_fits(sub / "res.fits")
    np.testing.assert_array_equal(res.reshape(n, 10), res_ref)


@pytest.mark.gpu
def test_me_inv_command(tmp_path, cube):
    """The command-line driver writes the same result file."""
    import subprocess
    ctl = setup_run(tmp_path, cube, {"nprofiles": "50"})
    exe = os.path.join(os.path.dirname(me_b200.LIB_PATH), "me_inv")
    out = subprocess.run([exe, str(ctl)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    _, res = parse_fits(tmp_path / "res.fits")
    prof = sol_pixels(cube["data"])
    assert (res.reshape(-1, 10)[:, 9] > 0).all()
    # same inputs through the library
    sub = tmp_path / "lib"
    sub.mkdir()
    ctl2 = setup_run(sub, cube, {"nprofiles": "50"})
    me_b200.run(ctl2)
    _, res2 = parse_fits(sub / "res.fits")
    np.testing.assert_array_equal(res, res2)
    assert res.reshape(-1, 10).shape[0] == prof.shape[0]
