"""Seeded synthetic Stokes maps for the benchmark workloads.

No public dataset is named for this path, so every map is synthesised from
seeded parameter draws with the project's own forward model (the GPU
synthesis on a GPU, the CPU oracle in the CPU tests) plus Gaussian noise.

Workloads (sizes and distributions of the reference-facing benchmark configs):

* ``fe15648_64x64``      64x64 px, Fe I 15648.5 A (g_eff = 3), nl = 60,
                          lambda_i = lambda0 - 1.2 + 0.04 i; B ~ U(0,3000) G,
                          cos(theta) ~ U(-1,1), phi ~ U(0,180) deg,
                          v ~ N(0,1.5) km/s, Doppler width ~ U(150,350) mA,
                          a ~ U(0.1,0.8), eta0 ~ U(2,30), S = 1, beta ~ U(0.1,0.6);
                          noise sigma = 1e-3; num_run = 1, 100 iterations,
                          default bounds, Icriteria lowered to 0.01 (S = 1 data).
* ``fe15648_1024x1024``  the same draws on 1024x1024 px, num_run = 5,
                          chisq_criteria = 1.5.
* ``fe6173_4096x4096``   4096x4096 px, Fe I 6173.3 A (g_eff = 2.5), a filtergram:
                          nl = 6 at lambda0 +-34, +-103, +-172 mA, each the mean
                          through a Gaussian instrument filter of 76 mA FWHM
                          (keyword ``filter = 76, 21``: 21 sub-wavelengths over
                          +-1.5 FWHM); draws as fe15648 but Doppler width
                          ~ U(20, 50) mA; noise sigma = 2e-3; num_run = 5,
                          chisq_criteria = 1.5, Bounds_Damp 0.05-1.0 (the
                          drawn damping reaches 0.1).
* ``fe6302_2048x1024``   2048x1024 px, Fe I 6302.5 A (g_eff = 2.5), nl = 112 at
                          21.5 mA centred on lambda0; 60 % weak-field pixels
                          (B ~ U(0,200) G, eta0 ~ U(1,10)), 40 % strong-field
                          (B ~ U(500,3500) G, eta0 ~ U(2,30)); the Doppler width
                          is not stated for this line, so it is drawn from the
                          15648 A range scaled by the wavelength ratio,
                          U(60,140) mA; weights 1,4,4,2; num_run = 10.

The literal default Bounds_Dopp (10-80 mA) cannot reach the drawn Doppler
widths of the 15648 A maps; the parity runs keep the literal defaults (what
the reference does with the same control file) and ``widen_bounds`` gives the
truth-recovery variant (Bounds_Dopp = 100, 400; Bounds_Damp = 0.05, 1.0).
"""
from __future__ import annotations

import numpy as np

C_LIGHT = 299792458.0

WORKLOADS = {
    "fe15648_64x64": dict(lam0=15648.5, geff=3.0, nl=60, npix=64 * 64, kind="fe15648",
                          ctl={"num_run": "1", "num_iter": "100", "Icriteria": "0.01"},
                          noise=1e-3),
    "fe15648_1024x1024": dict(lam0=15648.5, geff=3.0, nl=60, npix=1024 * 1024, kind="fe15648",
                              ctl={"num_run": "5", "num_iter": "100", "chisq_criteria": "1.5",
                                   "Icriteria": "0.01"},
                              noise=1e-3),
    "fe6173_4096x4096": dict(lam0=6173.3, geff=2.5, nl=6, npix=4096 * 4096, kind="fe6173",
                             ctl={"num_run": "5", "num_iter": "100", "chisq_criteria": "1.5",
                                  "Icriteria": "0.01", "filter": "76, 21",
                                  "Bounds_Damp": "0.05, 1.0"},
                             noise=2e-3),
    "fe6302_2048x1024": dict(lam0=6302.5, geff=2.5, nl=112, npix=2048 * 1024, kind="fe6302",
                             ctl={"num_run": "10", "num_iter": "100", "weights": "1, 4, 4, 2",
                                  "Icriteria": "0.01"},
                             noise=1e-3),
}


def wavelengths(name: str) -> np.ndarray:
    w = WORKLOADS[name]
    if w["kind"] == "fe15648":
        return w["lam0"] - 1.2 + 0.04 * np.arange(w["nl"])
    if w["kind"] == "fe6302":
        return w["lam0"] + 0.0215 * (np.arange(w["nl"]) - (w["nl"] - 1) / 2.0)
    if w["kind"] == "fe6173":
        return w["lam0"] + 1e-3 * np.array([-172.0, -103.0, -34.0, 34.0, 103.0, 172.0])
    raise KeyError(name)


def control_text(name: str, precision: str = "FP32", seed: int = 0, widen_bounds: bool = False,
                 extra: dict | None = None) -> str:
    """Control file in the reference's keyword syntax for one workload."""
    w = WORKLOADS[name]
    keys = {"verbose": "0", "lines": f"{w['lam0']}, {w['geff']}",
            "data_path": "./synthetic.fits", "wavelength_path": "./synthetic_wave.fits"}
    keys.update(w["ctl"])
    if widen_bounds:
        keys["Bounds_Dopp"] = "100, 400"
        keys["Bounds_Damp"] = "0.05, 1.0"
    keys["precision"] = precision
    keys["rng_seed"] = str(int(seed))
    if extra:
        keys.update(extra)
    return "".join(f"{k} = {v}\n" for k, v in keys.items())


def reference_control_text(name: str, widen_bounds: bool = False, extra: dict | None = None,
                           path: str = "./input") -> str:
    """Same control file without this library's own keywords (for the reference)."""
    w = WORKLOADS[name]
    keys = {"verbose": "0", "lines": f"{w['lam0']}, {w['geff']}",
            "data_path": path, "wavelength_path": path}
    keys.update(w["ctl"])
    if widen_bounds:
        keys["Bounds_Dopp"] = "100, 400"
        keys["Bounds_Damp"] = "0.05, 1.0"
    if extra:
        keys.update(extra)
    return "".join(f"{k} = {v}\n" for k, v in keys.items())


def draw_parameters(name: str, npix: int, seed: int) -> np.ndarray:
    """True parameters [npix][9] in the reference's units (rad, km/s, mA)."""
    w = WORKLOADS[name]
    rng = np.random.default_rng(seed)
    p = np.zeros((npix, 9))
    p[:, 1] = np.arccos(rng.uniform(-1.0, 1.0, npix))
    p[:, 2] = np.deg2rad(rng.uniform(0.0, 180.0, npix))
    p[:, 3] = rng.normal(0.0, 1.5, npix)
    p[:, 5] = rng.uniform(0.1, 0.8, npix)
    p[:, 7] = 1.0
    p[:, 8] = rng.uniform(0.1, 0.6, npix)
    if w["kind"] in ("fe15648", "fe6173"):
        p[:, 0] = rng.uniform(0.0, 3000.0, npix)
        p[:, 4] = rng.uniform(150.0, 350.0, npix) if w["kind"] == "fe15648" else \
            rng.uniform(20.0, 50.0, npix)
        p[:, 6] = rng.uniform(2.0, 30.0, npix)
    else:
        weak = rng.uniform(0.0, 1.0, npix) < 0.6
        p[:, 0] = np.where(weak, rng.uniform(0.0, 200.0, npix), rng.uniform(500.0, 3500.0, npix))
        p[:, 6] = np.where(weak, rng.uniform(1.0, 10.0, npix), rng.uniform(2.0, 30.0, npix))
        p[:, 4] = rng.uniform(60.0, 140.0, npix)
    return p


def train_prior(name: str) -> dict:
    """Training-set overrides of me_mlp_train_params for a workload's learned
    initialiser (its parameter distributions and noise; the defaults are the
    Fe I 15648.5 A maps')."""
    w = WORKLOADS[name]
    if w["kind"] == "fe6173":
        return {"doppler_range": (20.0, 50.0), "noise": w["noise"]}
    if w["kind"] == "fe6302":
        # the map's two populations: 40 % strong-field, 60 % weak-field
        return {"b_range": (500.0, 3500.0), "eta_range": (2.0, 30.0),
                "mix_weight": 0.6, "mix_b_range": (0.0, 200.0), "mix_eta_range": (1.0, 10.0),
                "doppler_range": (60.0, 140.0), "noise": w["noise"]}
    return {}


def add_noise(prof: np.ndarray, sigma: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed + 7919)
    return prof + rng.normal(0.0, sigma, prof.shape)


def sample_indices(npix: int, nsample: int, seed: int = 7) -> np.ndarray:
    """Sorted indices of a seeded sample of a map's pixels (the pixels whose
    chi^2 is compared with the reference's, and the reference arm's input)."""
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(npix, size=min(nsample, npix), replace=False))


def sample_noise(name: str, nsample: int, map_seed: int) -> np.ndarray:
    """Gaussian noise [nsample][4][nl] of a map's sample pixels, drawn on the
    host so that every process that builds the sample gets the same values."""
    w = WORKLOADS[name]
    rng = np.random.default_rng(map_seed + 104729)
    return rng.normal(0.0, w["noise"], (nsample, 4, w["nl"]))
