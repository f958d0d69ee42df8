"""CPU: the oracle's gradient (vjp_hitran: hko_vjp_sums + the chain rule of
the line scaling) against central differences of the oracle's own forward,
for the four profiles (Voigt, Lorentz, Doppler, binned Gaussian).  This
pins the reference gradient the GPU adjoint is tested against.

Loss = sum_i w_i log K_i.  Steps: T0 +- 0.2 K and +- 0.1 K stay inside one
1 K segment of the partition table (Q(T) is piecewise linear), P and the
per-line multipliers by 2.5e-4 and 1.25e-4 relative; the two steps are
Richardson-extrapolated.  Tolerance 1e-6 relative.
"""
import numpy as np
import pytest

import oracle
from hkb import synth

NUMIN, NUMAX, DNU, CUT = 1000.0, 1100.0, 0.01, 25.0
T0, P0 = 800.5, 0.7


@pytest.fixture(scope="module")
def case():
    L = synth.hitran_lines(300, seed=17, nu_min=NUMIN - 20.0, nu_max=NUMAX + 20.0)
    L["delta"] = np.random.default_rng(2).uniform(-0.01, 0.01, 300)
    Tq, Qq = synth.q_table()
    nx = oracle.grid_nx(NUMIN, NUMAX, DNU)
    w = np.random.default_rng(6).standard_normal(nx)
    return dict(L=L, Tq=Tq, Qq=Qq, nx=nx, w=w)


def _loss(d, T, P, profile, s_scale=None, g_scale=None, kmin=0.0):
    Q = oracle.partition(d["Tq"], d["Qq"], T)
    nu, S, iad, vy = oracle.prep_hitran(d["L"], [synth.MASS], [1.0], [Q], T, P, qalphaL=1.0)
    if s_scale is not None:
        S = S * s_scale
    if g_scale is not None:
        vy = vy * g_scale
    win = oracle.windows(nu, S, iad, vy, NUMIN, DNU, d["nx"], 0, CUT, profile=profile)
    K, _ = oracle.opacity(nu, S, iad, vy, win, NUMIN, DNU, d["nx"], kmin=kmin, profile=profile)
    assert np.all(K > 0.0)
    return float(np.sum(d["w"] * np.log(K)))


def _richardson(f, h):
    c1 = (f(h) - f(-h)) / (2 * h)
    c2 = (f(h / 2) - f(-h / 2)) / h
    return (4.0 * c2 - c1) / 3.0


@pytest.mark.parametrize("profile", [1, 2, 3, 4])
def test_oracle_gradient_vs_central_differences(case, profile):
    d = case
    Q = oracle.partition(d["Tq"], d["Qq"], T0)
    nu, S, iad, vy = oracle.prep_hitran(d["L"], [synth.MASS], [1.0], [Q], T0, P0, qalphaL=1.0)
    win = oracle.windows(nu, S, iad, vy, NUMIN, DNU, d["nx"], 0, CUT, profile=profile)
    K, _ = oracle.opacity(nu, S, iad, vy, win, NUMIN, DNU, d["nx"], profile=profile)
    # the Doppler and binned-Gaussian cores leave most points empty: a floor
    # kmin (constant in T, P and the line parameters) keeps log K finite
    kmin = 1e-12 * K.max()
    K = K + kmin
    u = d["w"] / K
    rT, rP, rS, rG = oracle.vjp_hitran(d["L"], synth.MASS, d["Tq"], d["Qq"], T0, P0, u, NUMIN,
                                       DNU, d["nx"], profile=profile)
    fT = _richardson(lambda h: _loss(d, T0 + h, P0, profile, kmin=kmin), 0.2)
    fP = _richardson(lambda h: _loss(d, T0, P0 + h, profile, kmin=kmin), 2.5e-4 * P0)
    print(f"profile {profile}: dT {rT:.8g} fd {fT:.8g}; dP {rP:.8g} fd {fP:.8g}")
    assert abs(fT - rT) < 1e-6 * abs(rT)
    assert abs(fP - rP) < 1e-6 * abs(rP)
    n = len(nu)
    aL = vy / iad  # gammaL of each line at (T0, P0)
    for l in np.argsort(-np.abs(rS))[:2]:
        def fs(h, l=l):
            s = np.ones(n)
            s[l] = np.exp(h)
            return _loss(d, T0, P0, profile, s_scale=s, kmin=kmin)
        fS = _richardson(fs, 2.5e-4)
        assert abs(fS - rS[l]) < 1e-6 * abs(rS[l])
    if profile >= 3:  # no Lorentz width in the Doppler and binned Gaussian shapes
        assert np.all(rG == 0.0)
        return
    for l in np.argsort(-np.abs(rG * aL))[:2]:
        def fg(h, l=l):
            g = np.ones(n)
            g[l] = np.exp(h)
            return _loss(d, T0, P0, profile, g_scale=g, kmin=kmin)
        fG = _richardson(fg, 2.5e-4)
        # d/dlog gammaL = gammaL * dLoss/dgammaL
        assert abs(fG - rG[l] * aL[l]) < 1e-6 * abs(rG[l] * aL[l])
