"""ctypes bindings of the CPU checkers (test infrastructure only).

* ``Oracle``     oracle/libme_oracle.so, this project's C++ restatement of the
                 reference's per-pixel inversion.
* ``Reference``  oracle/_ref/libmeref.so, the reference's own C core compiled
                 unmodified with ref_harness.c; present only where it was built
                 (it travels with the repository snapshot).
"""
from __future__ import annotations

import ctypes
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "milne-eddington_b200")
if PKG not in sys.path:
    sys.path.insert(0, PKG)


ORACLE_SO = os.path.join(ROOT, "oracle", "libme_oracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libmeref.so")
MEO_RNG_COUNTER = 0
MEO_RNG_NR = 1

_D = ctypes.POINTER(ctypes.c_double)
_LL = ctypes.POINTER(ctypes.c_longlong)


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_D)


_olib = None


def oracle_lib():
    global _olib
    if _olib is None:
        # the oracle shares the product's control-file structure (me_config);
        # only the Oracle class needs it, so the Reference class below loads
        # nothing of the product
        import me_b200
        L = ctypes.CDLL(ORACLE_SO)
        L.meo_plan_create.argtypes = [ctypes.POINTER(me_b200.MeConfig), _D, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_void_p)]
        L.meo_plan_set_filter.argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_int]
        L.meo_plan_destroy.argtypes = [ctypes.c_void_p]
        L.meo_plan_destroy.restype = None
        L.meo_plan_facts.argtypes = [ctypes.c_void_p, ctypes.POINTER(me_b200.MePlanFacts)]
        L.meo_invert.argtypes = [ctypes.c_void_p, _D, ctypes.c_long, ctypes.c_long, _D, _D,
                                 ctypes.c_int, ctypes.c_int, _D, _LL]
        L.meo_synth.argtypes = [ctypes.c_void_p, _D, ctypes.c_int, ctypes.c_double, _D, _D]
        L.meo_faddeeva.argtypes = [ctypes.c_int, _D, _D, ctypes.c_long, _D, _D]
        L.meo_svd.argtypes = [_D, ctypes.c_int, _D, _D]
        L.meo_svbksb.argtypes = [_D, _D, _D, _D, ctypes.c_int, _D]
        L.meo_init_guess.argtypes = [ctypes.c_void_p, _D, _D, _D]
        L.meo_normal_equations.argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_double,
                                           ctypes.c_double, _D, _D, _D]
        L.meo_restart_draws.argtypes = [ctypes.c_ulonglong, ctypes.c_longlong, ctypes.c_int, _D]
        L.meo_restart_draws.restype = None
        _olib = L
    return _olib


class Oracle:
    def __init__(self, cfg: "me_b200.MeConfig", wavelengths):
        self.cfg = cfg
        self.lam = np.ascontiguousarray(wavelengths, dtype=np.float64)
        self.nl = self.lam.size
        h = ctypes.c_void_p()
        st = oracle_lib().meo_plan_create(ctypes.byref(cfg), _p(self.lam), self.nl,
                                          ctypes.byref(h))
        assert st == 0, st
        self.h = h
        self.carry = np.zeros(1)

    def set_filter(self, offsets_mA, weights):
        off = np.ascontiguousarray(offsets_mA, dtype=np.float64)
        w = np.ascontiguousarray(weights, dtype=np.float64)
        st = oracle_lib().meo_plan_set_filter(self.h, _p(off), _p(w), off.size)
        assert st == 0, st

    def close(self):
        if self.h:
            oracle_lib().meo_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def facts(self):
        import me_b200
        f = me_b200.MePlanFacts()
        oracle_lib().meo_plan_facts(self.h, ctypes.byref(f))
        return {"nl": f.nl, "ncut": f.ncut, "ic": f.ic, "i0": f.i0, "i1": f.i1, "npar": f.npar,
                "bshift": f.bshift,
                "limits": np.array([[f.limits[i][0], f.limits[i][1]] for i in range(9)]),
                "fadd_a": f.fadd_a}

    def invert(self, prof, pixel_offset=0, rng_mode=MEO_RNG_COUNTER, nr_seed=0,
               want_fit=False, counters=False):
        prof = np.ascontiguousarray(prof, dtype=np.float64)
        n = prof.shape[0]
        res = np.zeros((n, 10))
        fit = np.zeros((n, 4, self.nl)) if want_fit else None
        cnt = np.zeros((n, 8), dtype=np.int64) if counters else None
        st = oracle_lib().meo_invert(self.h, _p(prof), n, pixel_offset, _p(res), _p(fit),
                                     rng_mode, nr_seed, _p(self.carry),
                                     cnt.ctypes.data_as(_LL) if counters else None)
        assert st == 0
        out = [res]
        if want_fit:
            out.append(fit)
        if counters:
            out.append(cnt)
        return out[0] if len(out) == 1 else tuple(out)

    def synth(self, par, deriv=False, step7=1e5):
        par = np.ascontiguousarray(par, dtype=np.float64)
        syn = np.zeros(4 * self.nl)
        jac = np.zeros(36 * self.nl) if deriv else None
        oracle_lib().meo_synth(self.h, _p(par), int(deriv), step7, _p(syn), _p(jac))
        return (syn.reshape(4, self.nl), jac.reshape(4, 9, self.nl)) if deriv \
            else syn.reshape(4, self.nl)

    def synth_many(self, pars):
        return np.stack([self.synth(p) for p in np.atleast_2d(pars)])

    def init_guess(self, prof):
        g = np.zeros(9)
        e = np.zeros(5)
        st = oracle_lib().meo_init_guess(self.h, _p(np.ascontiguousarray(prof, dtype=np.float64)),
                                         _p(g), _p(e))
        return st, g, e

    def normal_equations(self, prof, par, step7, norm0):
        n = 9 - sum(self.cfg.fixed)
        H = np.zeros(n * n)
        g = np.zeros(n)
        chi = np.zeros(1)
        oracle_lib().meo_normal_equations(self.h, _p(np.ascontiguousarray(prof, dtype=np.float64)),
                                          _p(np.ascontiguousarray(par, dtype=np.float64)), step7,
                                          norm0, _p(H), _p(g), _p(chi))
        return H.reshape(n, n), g, chi[0]


def oracle_faddeeva(nfigures, nu, a):
    nu = np.ascontiguousarray(nu, dtype=np.float64).ravel()
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    H = np.zeros_like(nu)
    L = np.zeros_like(nu)
    oracle_lib().meo_faddeeva(nfigures, _p(nu), _p(a), nu.size, _p(H), _p(L))
    return H, L


def oracle_svd(a):
    a = np.array(a, dtype=np.float64, copy=True, order="C")
    n = a.shape[0]
    w = np.zeros(n)
    v = np.zeros((n, n))
    hit = oracle_lib().meo_svd(_p(a), n, _p(w), _p(v))
    return a, w, v, hit


def restart_draws(seed, pixel, run):
    out = np.zeros(8)
    oracle_lib().meo_restart_draws(seed, pixel, run, _p(out))
    return out


# ---------------------------------------------------------------------------
# the reference's own C core
# ---------------------------------------------------------------------------
_rlib = None


def reference_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _rlib
    if _rlib is None:
        L = ctypes.CDLL(REF_SO)
        L.meref_setup.argtypes = [ctypes.c_char_p, _D, ctypes.c_int, ctypes.c_long, ctypes.c_int,
                                  ctypes.c_char_p]
        L.meref_invert.argtypes = [_D, ctypes.c_long, _D, _D]
        L.meref_plan_facts.argtypes = [ctypes.POINTER(ctypes.c_int), _D]
        L.meref_get_lm_chisq.restype = ctypes.c_double
        L.meref_set_lm_chisq.argtypes = [ctypes.c_double]
        L.meref_set_lm_chisq.restype = None
        L.meref_synth.argtypes = [_D, ctypes.c_int, ctypes.c_double, _D, _D]
        L.meref_faddeeva.argtypes = [ctypes.c_int, _D, _D, ctypes.c_long, _D, _D]
        L.meref_svd.argtypes = [_D, ctypes.c_int, _D, _D]
        L.meref_svbksb.argtypes = [_D, _D, _D, _D, ctypes.c_int, _D]
        L.meref_init_guess.argtypes = [_D, _D, _D]
        L.meref_bounds.argtypes = [_D, _D]
        L.meref_rng_gauss.argtypes = [ctypes.c_int, ctypes.c_long, _D]
        L.meref_reseed.argtypes = [ctypes.c_int]
        _rlib = L
    return _rlib


class Reference:
    """The reference core, set up once per process (INIT_INV has no teardown)."""

    def __init__(self, ctl_text: str, wavelengths, npix_max: int, seed: int = 12345):
        self.dir = tempfile.mkdtemp(prefix="meref_")
        self.ctl = os.path.join(self.dir, "input")
        with open(self.ctl, "w") as f:
            f.write(ctl_text.replace("./input", self.ctl))
        self.lam = np.ascontiguousarray(wavelengths, dtype=np.float64)
        self.nl = self.lam.size
        self.npix_max = npix_max
        st = ref_lib().meref_setup(self.ctl.encode(), _p(self.lam), self.nl, npix_max, seed,
                                   self.dir.encode())
        assert st == 0, f"meref_setup: {st}"

    def invert(self, prof, want_fit=False):
        prof = np.ascontiguousarray(prof, dtype=np.float64)
        n = prof.shape[0]
        res = np.zeros((n, 10))
        fit = np.zeros((n, 4, self.nl)) if want_fit else None
        for s in range(0, n, self.npix_max):
            e = min(n, s + self.npix_max)
            st = ref_lib().meref_invert(_p(prof[s:e]), e - s, _p(res[s:e]),
                                        _p(fit[s:e]) if want_fit else None)
            assert st == 0, st
        return (res, fit) if want_fit else res

    def reseed(self, seed: int):
        """The RNG state of a fresh set-up with `seed`, carried LM chi^2 zeroed."""
        st = ref_lib().meref_reseed(int(seed))
        assert st == 0, st

    @property
    def lm_chisq(self):
        return ref_lib().meref_get_lm_chisq()

    @lm_chisq.setter
    def lm_chisq(self, v):
        ref_lib().meref_set_lm_chisq(float(v))

    def facts(self):
        ints = (ctypes.c_int * 5)()
        lim = np.zeros(18)
        ref_lib().meref_plan_facts(ints, _p(lim))
        return {"ncut": ints[0], "ic": ints[1], "i0": ints[2], "i1": ints[3], "npar": ints[4],
                "limits": lim.reshape(9, 2)}

    def synth(self, par, deriv=False, step7=1e5):
        par = np.ascontiguousarray(par, dtype=np.float64)
        syn = np.zeros(4 * self.nl)
        jac = np.zeros(36 * self.nl)
        ref_lib().meref_synth(_p(par), int(deriv), step7, _p(syn), _p(jac))
        return (syn.reshape(4, self.nl), jac.reshape(4, 9, self.nl)) if deriv \
            else syn.reshape(4, self.nl)

    def init_guess(self, prof):
        g = np.zeros(9)
        e = np.zeros(5)
        st = ref_lib().meref_init_guess(_p(np.ascontiguousarray(prof, dtype=np.float64)), _p(g),
                                        _p(e))
        return st, g, e


def ref_faddeeva(nfigures, nu, a):
    nu = np.ascontiguousarray(nu, dtype=np.float64).ravel()
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    H = np.zeros_like(nu)
    L = np.zeros_like(nu)
    ref_lib().meref_faddeeva(nfigures, _p(nu), _p(a), nu.size, _p(H), _p(L))
    return H, L


def ref_svd(a):
    a = np.array(a, dtype=np.float64, copy=True, order="C")
    n = a.shape[0]
    w = np.zeros(n)
    v = np.zeros((n, n))
    ref_lib().meref_svd(_p(a), n, _p(w), _p(v))
    return a, w, v


def ref_rng_gauss(seed, n):
    out = np.zeros(n)
    ref_lib().meref_rng_gauss(seed, n, _p(out))
    return out


# ---------------------------------------------------------------------------
# the oracle over host cores: contiguous chunks of a map in spawned processes
# ---------------------------------------------------------------------------
_PW = {}


def _pool_init(ctl_text, lam):
    for p in (PKG, os.path.dirname(os.path.abspath(__file__))):
        if p not in sys.path:
            sys.path.insert(0, p)
    import me_b200
    _PW["orc"] = Oracle(me_b200.parse_config_text(ctl_text), lam)


def _pool_invert(job):
    prof, offset, rng_mode, nr_seed = job
    orc = _PW["orc"]
    orc.carry[0] = 0.0
    return orc.invert(prof, pixel_offset=offset, rng_mode=rng_mode, nr_seed=nr_seed)


def oracle_invert_chunks(ctl_text, lam, prof, chunk, procs=None, rng_mode=MEO_RNG_COUNTER,
                         nr_seed=0):
    """The oracle on prof [n][4][nl] in contiguous chunks of `chunk` pixels,
    each chunk a fresh run (carried LM chi^2 0 at its first pixel, as a new
    reference process starts; per-pixel restart draws keyed by the pixel's
    index in the whole map), the chunks spread over `procs` spawned
    processes.  Compare with a GPU plan inverting the same chunks with its
    carried chi^2 reset to 0 before each."""
    import multiprocessing as mp
    n = prof.shape[0]
    jobs = [(np.ascontiguousarray(prof[s:s + chunk]), s, rng_mode, nr_seed)
            for s in range(0, n, chunk)]
    procs = procs or min(len(jobs), os.cpu_count() or 1)
    with mp.get_context("spawn").Pool(procs, initializer=_pool_init,
                                      initargs=(ctl_text, np.asarray(lam))) as pool:
        return np.concatenate(pool.map(_pool_invert, jobs))


# ---------------------------------------------------------------------------
# the reference's core and the GPU adapter that replaces its INVERSION_MULTI
# (milne-eddington_b200/shim/me_inversion_multi.c) on one set-up
# ---------------------------------------------------------------------------
SHIM_SO = os.path.join(ROOT, "oracle", "_ref", "libmeshim.so")
_slib = None


def shim_available() -> bool:
    return os.path.exists(SHIM_SO)


def shim_lib():
    global _slib
    if _slib is None:
        import me_b200  # the adapter links the product library
        L = ctypes.CDLL(SHIM_SO)
        L.meref_setup.argtypes = [ctypes.c_char_p, _D, ctypes.c_int, ctypes.c_long, ctypes.c_int,
                                  ctypes.c_char_p]
        L.meref_invert.argtypes = [_D, ctypes.c_long, _D, _D]
        L.meref_invert_shim.argtypes = [_D, ctypes.c_long, _D, _D, ctypes.c_int]
        L.meref_shim_config.argtypes = [ctypes.POINTER(me_b200.MeConfig)]
        L.meref_get_lm_chisq.restype = ctypes.c_double
        L.meref_set_lm_chisq.argtypes = [ctypes.c_double]
        L.meref_set_lm_chisq.restype = None
        _slib = L
    return _slib


class ShimHarness:
    """RDINPUT + INIT_INV of the reference once per process (in libmeshim.so),
    then the same structures through the reference's INVERSION_MULTI or
    through me_inversion_multi (the GPU)."""

    def __init__(self, ctl_text: str, wavelengths, npix_max: int, seed: int = 12345):
        self.dir = tempfile.mkdtemp(prefix="meshim_")
        self.ctl = os.path.join(self.dir, "input")
        with open(self.ctl, "w") as f:
            f.write(ctl_text.replace("./input", self.ctl))
        self.lam = np.ascontiguousarray(wavelengths, dtype=np.float64)
        self.nl = self.lam.size
        self.npix_max = npix_max
        st = shim_lib().meref_setup(self.ctl.encode(), _p(self.lam), self.nl, npix_max, seed,
                                    self.dir.encode())
        assert st == 0, f"meref_setup: {st}"

    def _run(self, prof, shim, precision):
        prof = np.ascontiguousarray(prof, dtype=np.float64)
        n = prof.shape[0]
        assert n <= self.npix_max
        res = np.zeros((n, 10))
        if shim:
            st = shim_lib().meref_invert_shim(_p(prof), n, _p(res), None, precision)
        else:
            st = shim_lib().meref_invert(_p(prof), n, _p(res), None)
        assert st == 0, st
        return res

    def invert_reference(self, prof):
        return self._run(prof, False, 0)

    def invert_shim(self, prof, precision):
        return self._run(prof, True, precision)

    def config(self):
        import me_b200
        cfg = me_b200.MeConfig()
        assert shim_lib().meref_shim_config(ctypes.byref(cfg)) == 0
        return cfg

    @property
    def lm_chisq(self):
        return shim_lib().meref_get_lm_chisq()

    @lm_chisq.setter
    def lm_chisq(self, v):
        shim_lib().meref_set_lm_chisq(float(v))
