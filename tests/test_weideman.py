"""Weideman's 16-term series for the Faddeeva function (the FP32 syntheses'
alternative to the reference's region table, me_plan_set_faddeeva): the
library's coefficients against the paper's construction, recomputed here
(J. A. C. Weideman, SIAM J. Numer. Anal. 31 (1994) 1497-1518), and the FP32
series, evaluated in numpy, against scipy's Faddeeva function."""
import numpy as np
import pytest
from scipy.special import wofz

import me_b200

N = 16


def paper_coefficients(n):
    """c_0..c_{n-1} and L of the n-term series: the real parts of the
    length-4n DFT of f(t) = exp(-t^2) (L^2 + t^2) at t = L tan(theta / 2),
    theta = k pi / (2n), k = -2n+1 .. 2n-1 (a zero prepended), over 4n."""
    m = 2 * n
    L = np.sqrt(n / np.sqrt(2.0))
    theta = np.arange(-m + 1, m) * np.pi / m
    t = L * np.tan(theta / 2)
    f = np.concatenate([[0.0], np.exp(-t * t) * (L * L + t * t)])
    a = np.real(np.fft.fft(np.fft.fftshift(f))) / (2 * m)
    return a[1:n + 1], L


def series_f32(nu, y, c, L):
    """The device formula, step for step, in FP32."""
    f = np.float32
    nu, y, c, L = nu.astype(f), y.astype(f), c.astype(f), f(L)
    dre = L + y
    r = f(1) / (dre * dre + nu * nu)
    ire, iim = dre * r, nu * r
    nre = L - y
    zre, zim = nre * ire - nu * iim, nre * iim + nu * ire
    pre, pim = np.zeros_like(nu), np.zeros_like(nu)
    for n in range(len(c) - 1, -1, -1):
        pre, pim = pre * zre - pim * zim + c[n], pre * zim + pim * zre
    i2re, i2im = ire * ire - iim * iim, f(2) * ire * iim
    rsp = f(1 / np.sqrt(np.pi))
    return (f(2) * (pre * i2re - pim * i2im) + ire * rsp).astype(np.float64), \
           (f(2) * (pre * i2im + pim * i2re) + iim * rsp).astype(np.float64)


def test_coefficients_are_the_papers():
    c, L = me_b200.weideman16()
    ref, Lref = paper_coefficients(N)
    assert abs(L - Lref) < 1e-6
    np.testing.assert_allclose(c, ref.astype(np.float32), rtol=1e-6, atol=1e-12)


@pytest.mark.parametrize("lo,hi", [(-4, 4), (-40, 40), (-1e5, 1e5)])
def test_series_accuracy_fp32(lo, hi):
    rng = np.random.default_rng(11)
    nu = rng.uniform(lo, hi, 200000)
    y = np.concatenate([np.zeros(1000), rng.uniform(0, 1.6, 199000)])
    c, L = me_b200.weideman16()
    H, Lf = series_f32(nu, y, c, L)
    w = wofz(nu + 1j * y)
    scale = np.abs(w.real) + np.abs(w.imag)
    assert np.max(np.abs(H - w.real) / scale) < 1.5e-6
    assert np.max(np.abs(Lf - w.imag) / scale) < 1.5e-6
