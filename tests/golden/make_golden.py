"""Generates the golden fixtures in tests/golden/ from the reference's own C core.

The reference (HaoLi-70/Milne-Eddington) ships no tests, data cube or golden
vectors, so the fixtures are outputs of the reference itself: its unmodified
Src/ core compiled by oracle/Makefile into oracle/_ref/libmeref.so and driven
through oracle/ref_harness.c.  Every input is a seeded synthetic profile.

    make -C oracle ref && python tests/golden/make_golden.py

The reference core keeps per-process state that INIT_INV sets once, so each
fixture family is produced in its own child process.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "milne-eddington_b200"))

# (fixture name, workload, number of pixels, extra control keys, NR seed)
CASES = [
    ("fe15648_run1", "fe15648_64x64", 48, {}, 0),
    ("fe15648_run2_nr", "fe15648_64x64", 32, {"num_run": "2"}, 4242),
    ("fe15648_widened", "fe15648_64x64", 32, {"Bounds_Dopp": "100, 400",
                                              "Bounds_Damp": "0.05, 1.0"}, 0),
    ("fe6302_run1", "fe6302_2048x1024", 32, {"num_run": "1"}, 0),
    ("fe15648_fixed_hmi", "fe15648_64x64", 24, {"Bmod_fixed": "YES", "HMI_REF": "YES",
                                                "Btheta_Regularization": "NO",
                                                "Nfigures": "4"}, 0),
    ("fe15648_regul_eta", "fe15648_64x64", 24, {"Eta_Regularization": "YES, 10.0, 2e-3",
                                                "Dopp_Regularization": "YES, 60, 1e-3",
                                                "Nfigures": "5"}, 0),
]


def one_case(name, workload, npix, extra, seed):
    import me_maps
    import oracle_bind as ob

    lam = me_maps.wavelengths(workload)
    ctl = me_maps.reference_control_text(workload, extra=extra)
    ref = ob.Reference(ctl, lam, npix, seed=seed)
    par = me_maps.draw_parameters(workload, npix, seed=1000 + len(name))
    prof = np.stack([ref.synth(p) for p in par])
    prof = me_maps.add_noise(prof, me_maps.WORKLOADS[workload]["noise"], seed=17)
    # edge cases: a pixel under Icriteria and a NaN pixel (both written as zeros)
    prof[5] *= 1e-4
    prof[9, 0, 3] = np.nan
    guess = np.zeros((npix, 9))
    gextra = np.zeros((npix, 5))
    gstat = np.zeros(npix, dtype=np.int32)
    for i in range(npix):
        st, g, e = ref.init_guess(prof[i])
        gstat[i] = st
        guess[i] = g
        gextra[i] = e
    syn, jac = ref.synth(par[0], True, 0.1)
    ref.lm_chisq = 0.0
    res = ref.invert(prof)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), ctl=np.array(ctl), lam=lam,
                        par_true=par, prof=prof, res=res, guess=guess, guess_extra=gextra,
                        guess_status=gstat, syn0=syn, jac0=jac, nr_seed=np.array(seed),
                        carry_out=np.array(ref.lm_chisq), facts=np.array(json.dumps(
                            {k: (v.tolist() if hasattr(v, "tolist") else v)
                             for k, v in ref.facts().items()})))


def units():
    import oracle_bind as ob

    rng = np.random.default_rng(2024)
    nu = np.concatenate([rng.uniform(-12, 12, 1500), rng.uniform(-400, 400, 300),
                         np.sign(rng.uniform(-1, 1, 200)) * 10 ** rng.uniform(-4, 5, 200),
                         np.zeros(10), rng.uniform(-5, 5, 40)])
    a = np.concatenate([rng.uniform(0.005, 1.6, nu.size - 50), np.zeros(40), rng.uniform(0.1, 1, 10)])
    out = {"nu": nu, "a": a}
    for nf in (4, 5, 6, 7, 8):
        H, L = ob.ref_faddeeva(nf, nu, a)
        out[f"H{nf}"] = H
        out[f"L{nf}"] = L
    np.savez_compressed(os.path.join(HERE, "faddeeva.npz"), **out)
    mats = []
    A = rng.normal(size=(16, 9, 9))
    mats.extend(A @ A.transpose(0, 2, 1))
    mats.extend(rng.normal(size=(8, 9, 9)))
    Q, _ = np.linalg.qr(rng.normal(size=(9, 9)))
    mats.append(Q)  # orthogonal input: the trial-2+ case of the LM (SVD of U)
    U = []
    W = []
    V = []
    for m in mats:
        u, w, v = ob.ref_svd(m)
        U.append(u)
        W.append(w)
        V.append(v)
    np.savez_compressed(os.path.join(HERE, "svd.npz"), a=np.array(mats), u=np.array(U),
                        w=np.array(W), v=np.array(V))
    np.savez_compressed(os.path.join(HERE, "rng.npz"), seed=np.array(4242),
                        gauss=ob.ref_rng_gauss(4242, 64))


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--case":
        i = int(sys.argv[2])
        one_case(*CASES[i])
        sys.exit(0)
    if len(sys.argv) > 1 and sys.argv[1] == "--units":
        units()
        sys.exit(0)
    subprocess.check_call([sys.executable, __file__, "--units"])
    for i in range(len(CASES)):
        subprocess.check_call([sys.executable, __file__, "--case", str(i)])
    print("fixtures written to", HERE)
