"""CPU: the oracle's profiles 2-4 and plinth removal (voigt.h:1091-1262)
against closed forms, for one line on a uniform grid.

Line strength S here is the reference's scaled strength, which carries the
1/alphaD factor (voigt.h:349-363): S = S_true / alphaD.  Then
  Lorentz    K = S_true gamma / (pi (dnu^2 + gamma^2)),
  Doppler    K = S_true / (alphaD sqrt(pi)) exp(-(dnu / alphaD)^2),
  binned     sum_i K_i dnu = S_true (erf(x + vb/2) - erf(x - vb/2) telescopes
  Gaussian   over the window to ~2),
and with plinth removal K drops by the profile's value at the cut edge.
"""
import math

import numpy as np
import pytest

import oracle

NUMIN, DNU, NX = 0.0, 0.01, 20000
NU0, STRUE, ALPHA, GAMMA, CUT = 100.0037, 2.5e-20, 0.03, 0.2, 25.0


def one_line(profile, cutMode=0, cut=CUT, plinth=False):
    nu = np.array([NU0])
    iad = np.array([1.0 / ALPHA])
    vy = np.array([GAMMA / ALPHA])
    S = np.array([STRUE / ALPHA])
    win = oracle.windows(nu, S, iad, vy, NUMIN, DNU, NX, cutMode, cut, profile=profile)
    pl = oracle.plinth(S, iad, vy, win, cutMode, cut, profile) if plinth else None
    K, pairs = oracle.opacity(nu, S, iad, vy, win, NUMIN, DNU, NX, profile=profile, plinth=pl)
    return K, win[0], pairs, pl


def test_profiles_have_no_b_c_regions():
    for p in (2, 3, 4):
        _, w, pairs, _ = one_line(p)
        assert w[1] == w[2] == w[3] == w[4] and pairs[1] == pairs[2] == 0
        assert pairs[0] == w[5] - w[0] > 0
    _, w, pairs, _ = one_line(1)
    assert pairs[1] > 0 and pairs[2] > 0


def test_lorentz_and_doppler_closed_forms():
    x = NUMIN + DNU * np.arange(NX)
    d = x - NU0
    inside = np.abs(d) < CUT
    K2, _, _, _ = one_line(2)
    want2 = np.where(inside, STRUE * GAMMA / (math.pi * (d * d + GAMMA * GAMMA)), 0.0)
    np.testing.assert_allclose(K2, want2, rtol=1e-13, atol=0)
    K3, _, _, _ = one_line(3)
    want3 = np.where(inside, STRUE / (ALPHA * math.sqrt(math.pi)) * np.exp(-(d / ALPHA) ** 2), 0.0)
    np.testing.assert_allclose(K3, want3, rtol=1e-12, atol=1e-300)


def test_binned_gaussian_integrates_to_strength():
    K4, w, _, _ = one_line(4)
    assert K4.sum() * DNU == pytest.approx(STRUE, rel=1e-12)
    # and it is the bin average of the Doppler profile
    K3, _, _, _ = one_line(3)
    c = int(np.argmax(K3))
    assert K4[c] == pytest.approx(K3[c], rel=2e-2) and K4[c] < K3[c]


# the Doppler profile's edge value underflows unless the cut is a few
# Doppler widths (x_c = 1.7, 2, 2.5 here)
PLINTH_CASES = [(p, m, c) for p in (1, 2) for m, c in ((0, 1.0), (1, 40.0), (2, 60.0))] + [
    (3, 0, 0.05), (3, 1, 0.3), (3, 2, 2.5)]


@pytest.mark.parametrize("profile,cutMode,cut", PLINTH_CASES)
def test_plinth_is_the_cut_edge_value(profile, cutMode, cut):
    K, w, _, _ = one_line(profile, cutMode, cut)
    Kp, _, _, pl = one_line(profile, cutMode, cut, plinth=True)
    assert pl[0] > 0.0
    inside = np.zeros(NX, bool)
    inside[w[0]:w[5]] = True
    np.testing.assert_allclose(Kp[inside], K[inside] - pl[0], rtol=1e-12, atol=1e-12 * K.max())
    assert np.array_equal(Kp[~inside], K[~inside])
    # the plinth is the profile at exactly the cut edge x_c (Doppler units)
    y = GAMMA / ALPHA
    xc = {0: cut / ALPHA, 1: cut * y, 2: cut}[cutMode]
    if profile == 2:
        dc = xc * ALPHA
        assert pl[0] == pytest.approx(STRUE * GAMMA / (math.pi * (dc * dc + GAMMA * GAMMA)), rel=1e-13)
    elif profile == 3:
        assert pl[0] == pytest.approx(STRUE / (ALPHA * math.sqrt(math.pi)) * math.exp(-xc * xc), rel=1e-13)
    else:
        # Voigt far from the core: within 1 % of the Lorentz value there
        dc = xc * ALPHA
        assert pl[0] == pytest.approx(STRUE * GAMMA / (math.pi * (dc * dc + GAMMA * GAMMA)), rel=1e-2)
    assert oracle.plinth(np.array([1.0]), np.array([1.0]), np.array([1.0]), w[None, :], 0, 5.0, 4)[0] == 0.0


SL14 = [3.0, 10.0, 20.0, 0.09, -0.05, 0.004, 0.05, 0.02, 0.003, 0.02, 0.0, 0.0, 95.0, 130.0]


@pytest.mark.parametrize("profile", [1, 2])
def test_sublorentz_factor(profile):
    """chi(|x - nu|) x / nu inside (x_lo, x_hi), 1 outside; chi = 1 within
    sigma1 of the centre, continuous at the breakpoints (voigt.h:47-72)."""
    T = 700.0
    nu = np.array([NU0])
    iad = np.array([1.0 / ALPHA])
    vy = np.array([GAMMA / ALPHA])
    S = np.array([STRUE / ALPHA])
    win = oracle.windows(nu, S, iad, vy, NUMIN, DNU, NX, 0, CUT, profile=profile)
    K, _ = oracle.opacity(nu, S, iad, vy, win, NUMIN, DNU, NX, profile=profile)
    sl = oracle.sublorentz_params(SL14, T)
    Ks, _ = oracle.opacity(nu, S, iad, vy, win, NUMIN, DNU, NX, profile=profile, sublorentz=sl)
    x = NUMIN + DNU * np.arange(NX)
    d = np.abs(x - NU0)
    B = sl[3:6]
    chi = np.where(d < 3.0, 1.0, np.where(d < 10.0, np.exp(-B[0] * (d - 3.0)), np.where(
        d < 20.0, np.exp(-B[0] * 7.0 - B[1] * (d - 10.0)),
        np.exp(-B[0] * 7.0 - B[1] * 10.0 - B[2] * (d - 20.0)))))
    f = np.where((x > 95.0) & (x < 130.0), chi * x / NU0, 1.0)
    m = K > 0
    np.testing.assert_allclose(Ks[m], K[m] * f[m], rtol=1e-13)
    assert np.array_equal(Ks[~m], K[~m])
    assert sl[3] == pytest.approx(0.09 - 0.05 * math.exp(-0.004 * T), rel=1e-15)
