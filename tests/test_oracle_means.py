"""CPU: the oracle's Planck / Rosseland mean sums and transmission function
(resample.h:541-773) against closed forms.

Known answers: for a constant opacity both means equal it; the end-weighted
sums of B and dB/dT times dnu approach sigma T^4 / pi and 4 sigma T^3 / pi
(the reference's own analytic check, heliosk.cu:1991-1993); the end weights
sum to -1, so a constant K gives Tr(m) = exp(-K m) exactly up to rounding,
and the Nxmin part mixes in exp(-kmin m) by the fraction Nxmin / Nxb.
"""
import math

import numpy as np
import pytest

import oracle

KB, H, C = 1.3806489e-16, 6.62606957e-27, 2.99792458e10
SIGMA = 2.0 * KB**4 / (H**3 * C**2 * 15.0) * math.pi**5


def test_planck_closed_form():
    for nu, T in ((1000.0, 300.0), (5000.0, 1500.0), (20000.0, 3000.0)):
        B, R = oracle.planck(nu, T)
        x = H * C * nu / (KB * T)
        assert B == pytest.approx(2.0 * H * C * C * nu**3 / math.expm1(x), rel=1e-13)
        assert R == pytest.approx(B * x * math.exp(x) / (T * math.expm1(x)), rel=1e-12)
    assert oracle.planck(0.0, 1000.0) == (0.0, 0.0)
    # cold: exp overflows to inf, both vanish (Mean_kernel's rewritten dB/dT)
    assert oracle.planck(30000.0, 10.0) == (0.0, 0.0)


@pytest.mark.parametrize("T", [500.0, 1500.0, 3000.0])
def test_means_known_answers(T):
    dnu = 0.2  # 0-60000 cm^-1: the Planck tail beyond is < 1e-9 of the integral at 3000 K
    x = np.arange(0, 300000) * dnu
    K = np.full(len(x), 3.25)
    m = oracle.means(x, K, T)
    assert m[0] / m[2] == pytest.approx(3.25, rel=1e-12)   # Planck mean
    assert m[3] / m[1] == pytest.approx(3.25, rel=1e-12)   # Rosseland mean
    assert m[2] * dnu == pytest.approx(SIGMA * T**4 / math.pi, rel=1e-7)
    assert m[3] * dnu == pytest.approx(4.0 * SIGMA * T**3 / math.pi, rel=1e-7)
    # zero opacity points are skipped in the Rosseland sum, not divided by
    K[1000:2000] = 0.0
    m2 = oracle.means(x, K, T)
    assert np.isfinite(m2).all() and m2[1] < m[1]


def test_transmission_known_answers():
    nxb, nbins, nTr, dTr = 1000, 3, 40, 0.25
    K = np.repeat([0.2, 1.5, 0.0], nxb)
    nxmin = np.array([0, 250, 999], np.int32)
    kmin = 0.01
    Tr = oracle.transmission(K, nxb, nbins, nxmin, kmin, nTr, dTr)
    m = np.exp((np.arange(nTr) - nTr // 2) * dTr)
    for b, k in enumerate((0.2, 1.5, 0.0)):
        f = nxmin[b] / nxb
        want = np.exp(-k * m) * (1.0 - f) + np.exp(-kmin * m) * f
        np.testing.assert_allclose(Tr[b], want, rtol=1e-13, atol=0)
    # without Nxmin (no resampling) and sorted K: decreasing in m, Tr(m -> 0) -> 1
    Ks = np.sort(np.random.default_rng(1).lognormal(0.0, 2.0, nxb))
    T1 = oracle.transmission(Ks, nxb, 1, None, 0.0, nTr, dTr)[0]
    assert np.all(np.diff(T1) < 0) and 0.9 < T1[0] <= 1.0
