"""Algorithmic operation counts of the reference's per-pixel algorithm.

Runs the oracle's numeric kernels instantiated with a counting scalar type
(oracle/flop_count.h) and writes tests/golden/flop_counts.json, the per-event
figures bench.py multiplies by the event counts the CUDA kernel reports:

* forward synthesis, per wavelength   (Milne_Eddington_Single, Deriv=0,
                                       Src/ME_SOLVER.c:101-366, + Loss_Function)
* synthesis with Jacobian, per wavelength (Deriv=1) + Hessian_Compute's
                                       normal equations (Src/LM_FIT.c:240-350)
* SVD solve (svdcmp + truncation ladder + svbksb, Src/LM_FIT.c:400-469) of the
  normal matrix (the first trial of an iteration) and of an orthogonal U
  factor (every later trial: the reference re-decomposes the previous U).

Synthesis counts depend on the Voigt region mix, so they are averaged over the
parameters the LM actually visits: the initial guesses and the oracle's final
fits of a seeded sample of each workload.  Counts: add/sub, mul, div, sqrt,
exp/log, sin/cos, erfc, compares.  FLOPs = add + mul + div + sqrt; the
transcendental calls are reported separately.

    python tests/golden/make_flop_counts.py
"""
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "tests"), os.path.join(ROOT, "milne-eddington_b200")]

import me_b200  # noqa: E402
import me_maps  # noqa: E402
import oracle_bind as ob  # noqa: E402

KEYS = ["add", "mul", "div", "sqrt", "exp_log", "sin_cos", "erfc", "cmp"]
D = ctypes.POINTER(ctypes.c_double)


def counts(vec):
    return {k: float(v) for k, v in zip(KEYS, vec)}


def main(npix=96):
    out = {name: workload_counts(name, npix) for name in me_maps.WORKLOADS}
    path = os.path.join(HERE, "flop_counts.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


def workload_counts(name, npix=96):
    """The per-event counts of one workload (the entry flop_counts.json holds)."""
    L = ob.oracle_lib()
    L.meo_count_synth.argtypes = [ctypes.c_void_p, D, ctypes.c_int, D]
    L.meo_count_svd_solve.argtypes = [D, D, ctypes.c_int, ctypes.c_double, D]
    lam = me_maps.wavelengths(name)
    nl = lam.size
    cfg = me_b200.parse_config_text(me_maps.control_text(name, precision="FP64"))
    o = ob.Oracle(cfg, lam)
    par = me_maps.draw_parameters(name, npix, 77)
    prof = me_maps.add_noise(o.synth_many(par), 1e-3, 77)
    res = o.invert(prof)
    visited = []
    for i in range(npix):
        st, g, e = o.init_guess(prof[i])
        if st == 0:
            visited.append((g, e))
        if res[i, 9] > 0:
            visited.append((res[i, :9], e))
    fwd = np.zeros(8)
    der = np.zeros(8)
    svd1 = np.zeros(8)
    svd2 = np.zeros(8)
    for p, e in visited:
        c = np.zeros(8)
        L.meo_count_synth(o.h, np.ascontiguousarray(p).ctypes.data_as(D), 0, c.ctypes.data_as(D))
        fwd += c
        L.meo_count_synth(o.h, np.ascontiguousarray(p).ctypes.data_as(D), 1, c.ctypes.data_as(D))
        der += c
        H, g, _ = o.normal_equations(prof[0], p, e[4], e[0])
        H = np.ascontiguousarray(H)
        g = np.ascontiguousarray(g)
        L.meo_count_svd_solve(H.ctypes.data_as(D), g.ctypes.data_as(D), 9, 1e-6,
                              c.ctypes.data_as(D))
        svd1 += c
        u, w, v, _ = ob.oracle_svd(H)
        u = np.ascontiguousarray(u)
        L.meo_count_svd_solve(u.ctypes.data_as(D), g.ctypes.data_as(D), 9, 1e-6,
                              c.ctypes.data_as(D))
        svd2 += c
    n = len(visited)
    fwd /= n * nl
    der /= n * nl
    svd1 /= n
    svd2 /= n
    npar = 9
    normal = {"add": 4 * (npar * (npar + 1) // 2) + 8 * npar, "mul": 8 * (npar * (npar + 1) // 2)
              + 8 * npar}  # s += iv*Ji*Jj per Stokes; s -= iv*Ji*(syn-obs)
    loss = {"add": 8.0, "mul": 8.0}  # diff, diff*diff*iv, += per Stokes
    return {"nl": nl, "samples": n,
            "forward_per_lambda": counts(fwd),
            "jacobian_per_lambda": counts(der),
            "normal_equations_per_lambda": normal,
            "loss_per_lambda": loss,
            "svd_solve_normal_matrix": counts(svd1),
            "svd_solve_orthogonal": counts(svd2)}


if __name__ == "__main__":
    main()
