"""CPU: the oracle's ExoMol line scaling (oracle.prep_exomol) against the
reference's formulas evaluated by hand, record by record, in plain Python:
L_kernelExomol (voigt.h:484-504) forms 1/alphaD at the line, A / (4 pi c),
the default width and S_file Ab Sscale / Q; Sf_kernel (voigt.h:365-397)
applies exp(-c1 E'') (1 - exp(-c1 nu)) / alphaD, the width at P / 1 bar and
(T0 / T)^n plus the natural width, and zeroes lines at nu = 0.  The caller's
constants are heliosk.cu:985-986 (c1 = h c / (kB T), T1 = T0 / T) and the
units = 0 mass scaling of heliosk.cu:1064-1070.  Constants: define.h:36-45.

Tolerance: 1e-15 relative (the same IEEE operations in the same order; only
libm's exp and pow could differ in the last bit).
"""
import math

import numpy as np

import oracle

KB, H, C, NA = 1.3806489e-16, 6.62606957e-27, 2.99792458e10, 6.0221412927e23
T0, PO_BAR = 296.0, 0.986923


def hand(nu, S_file, EL, A, mass_g, ab, Q, defaultL, defaultn, T, P, gammaF=1.0,
         meanMass=None, Sscale=1.0):
    if meanMass is None:
        meanMass = ab * mass_g * Sscale
    m = mass_g / NA
    Ab = ab * (mass_g / meanMass)          # units = 0
    Ss = Sscale * (mass_g / meanMass)
    c1 = H * C / (KB * T)
    T1 = T0 / T
    # L_kernelExomol
    iad0 = C * math.sqrt(m / (2.0 * KB * T))
    Ad = A / (4.0 * math.pi * C)
    vy = defaultL * gammaF
    S = S_file * Ab * Ss / Q
    # Sf_kernel
    iad = iad0 / nu if nu != 0.0 else math.inf
    if nu != 0.0:
        S *= math.exp(-c1 * EL) * (1.0 - math.exp(-c1 * nu)) * iad
    aL = vy * ((P / PO_BAR) * math.pow(T1, defaultn))
    aL = aL + Ad
    y = aL * iad
    if nu == 0.0:
        return 0.0, 0.0, 0.0, 0.0
    return nu, S, iad, y


def test_prep_exomol_against_hand_evaluation():
    rng = np.random.default_rng(21)
    n = 64
    L = {"nu": rng.uniform(0.5, 40000.0, n), "S": 10.0 ** rng.uniform(-40, -18, n) * 1e25,
         "EL": rng.exponential(8000.0, n), "A": rng.uniform(0.0, 50.0, n)}
    L["nu"][3] = 0.0          # zeroed by Sf_kernel
    L["A"][5] = 0.0
    mass, ab, defaultL, defaultn = 18.0, 0.997, 0.07, 0.5
    for T, P, Q in ((500.0, 1e-4, 123.4), (2500.0, 10.0, 9876.5), (1200.0, 0.3, 1.0)):
        got = oracle.prep_exomol(L, mass, ab, Q, defaultL, defaultn, T, P)
        for i in range(n):
            want = hand(L["nu"][i], L["S"][i], L["EL"][i], L["A"][i], mass, ab, Q, defaultL,
                        defaultn, T, P)
            for k in range(4):
                g, w = float(got[k][i]), want[k]
                if w == 0.0:
                    assert g == 0.0, (T, i, k)
                else:
                    assert abs(g - w) <= 1e-15 * abs(w), (T, i, k, g, w)


def test_prep_exomol_units_and_scales():
    """gammaF scales the default width; Sscale and the mean molar mass enter
    the strength as Ab (m / meanMass) Sscale (m / meanMass) (units = 0)."""
    L = {"nu": np.array([1234.5]), "S": np.array([3e-21]), "EL": np.array([700.0]),
         "A": np.array([2.5])}
    got = oracle.prep_exomol(L, 18.0, 0.9, 50.0, 0.07, 0.5, 800.0, 2.0, gammaF=1.3,
                             meanMass=25.0, Sscale=0.01)
    want = hand(1234.5, 3e-21, 700.0, 2.5, 18.0, 0.9, 50.0, 0.07, 0.5, 800.0, 2.0, gammaF=1.3,
                meanMass=25.0, Sscale=0.01)
    for k in range(4):
        assert abs(float(got[k][0]) - want[k]) <= 1e-15 * abs(want[k])
